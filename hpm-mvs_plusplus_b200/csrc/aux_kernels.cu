// Joint bilateral upsampling between pyramid levels (sm_100a).
//
// JBU_cu / RunJBU (HPM.cu:3037-3095, HPM.cpp:1266-1319) and JBU_cu_prior /
// JointBilateralUpsampling_prior (HPM.cu:3130-3197, HPM.cpp:1323-1392).  One
// thread per fine pixel gathers a (s^2+1) x (s^2+1) window of the coarse map;
// the Gaussian weights are evaluated in double as in the reference (its
// arguments are double expressions), the reductions in float.  The NaN
// fallback of RunJBU is folded into the kernel.  IEEE arithmetic, no implicit
// contraction (include/hpm_fp.h).
#include <cuda_runtime.h>
#include <stdint.h>

#include "aux_kernels.cuh"

namespace hpm {

__device__ __forceinline__ int clampi_(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ float jbu_spatial(float x1, float y1, float x2, float y2) {
    const float dx = x1 - x2, dy = y1 - y2;
    const float dis = dx * dx + dy * dy - 0.0f;  // pow(., 2) of floats (HPM.cu:144)
    const float sigma = 0.50f;
    return (float)exp(-1.0 * dis / (2 * sigma * sigma));
}

__device__ __forceinline__ float jbu_range(float x) {
    const float sigma = 25.5f;
    return (float)exp(-1.0 * (x * x) / (2 * sigma * sigma));
}

template <bool PRIOR>
__global__ void k_jbu(const float* __restrict__ image, int W, int H, const float* __restrict__ sdepth,
                      const float* __restrict__ snormal, int sw, int sh, float* __restrict__ out_depth,
                      float* __restrict__ out_normal) {
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    const int py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= W || py >= H) return;
    const float scale = (float)(1.0 * sw / W);
    const int a = H / sh, b = W / sw;
    const int image_scale = a > b ? a : b;
    const int nn = (image_scale * image_scale + 1) / 2;
    const float o_y = py * scale, o_x = px * scale;
    const float ref_pix = image[(size_t)py * W + px];
    float nf = 0.0f, val = 0.0f, n0 = 0.0f, n1 = 0.0f, n2 = 0.0f;
    for (int j = -nn; j <= nn; ++j) {
        int r_y = __float2int_rz(o_y + j);
        r_y = (r_y > 0 ? (r_y < sh ? r_y : sh - 1) : 0);
        const int r_ys = clampi_(py + j, 0, H - 1);
        for (int i = -nn; i <= nn; ++i) {
            int r_x = __float2int_rz(o_x + i);
            r_x = (r_x > 0 ? (r_x < sw ? r_x : sw - 1) : 0);
            const size_t s = (size_t)r_y * sw + r_x;
            const float sp = sdepth[s];
            const float nb = image[(size_t)r_ys * W + clampi_(px + i, 0, W - 1)];
            const float tg = jbu_spatial(o_x, o_y, (float)r_x, (float)r_y) * jbu_range(fabsf(ref_pix - nb));
            nf += tg;
            val += sp * tg;
            if (PRIOR) {
                n0 = n0 + snormal[3 * s] * tg;
                n1 = n1 + snormal[3 * s + 1] * tg;
                n2 = n2 + snormal[3 * s + 2] * tg;
            }
        }
    }
    float d = val / nf;
    const size_t c = (size_t)py * W + px;
    if (PRIOR) {
        const float x = n0 / nf, y = n1 / nf, z = n2 / nf;
        const float inv = 1.0f / sqrtf(x * x + y * y + z * z);
        out_normal[3 * c] = x * inv;
        out_normal[3 * c + 1] = y * inv;
        out_normal[3 * c + 2] = z * inv;
    } else if (d != d) {
        // RunJBU replaces NaN by src_depthmap(j/2, i/2) (HPM.cpp:1297-1300); the clamp keeps
        // the read inside the coarse map when the scale exceeds 2
        d = sdepth[(size_t)clampi_(py / 2, 0, sh - 1) * sw + clampi_(px / 2, 0, sw - 1)];
    }
    out_depth[c] = d;
}

cudaError_t launch_jbu(const float* image, int W, int H, const float* sdepth, int sw, int sh, float* out,
                       cudaStream_t st) {
    dim3 block(32, 8), grid((W + 31) / 32, (H + 7) / 8);
    k_jbu<false><<<grid, block, 0, st>>>(image, W, H, sdepth, nullptr, sw, sh, out, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_jbu_prior(const float* image, int W, int H, const float* sdepth, const float* snormal, int sw,
                             int sh, float* out_depth, float* out_normal, cudaStream_t st) {
    dim3 block(32, 8), grid((W + 31) / 32, (H + 7) / 8);
    k_jbu<true><<<grid, block, 0, st>>>(image, W, H, sdepth, snormal, sw, sh, out_depth, out_normal);
    return cudaGetLastError();
}

}  // namespace hpm
