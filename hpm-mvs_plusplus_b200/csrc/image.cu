// Image preparation of a pyramid level on the GPU (PrepareScaleImages,
// main.cpp:107-161; InuputInitialization's grey conversion, HPM.cpp:658-662;
// cv::Canny(image, 50, 150) of ProcessProblem, main.cpp:287):
//   k_resize_u8c3  cv::resize INTER_LINEAR of 8-bit BGR: float source
//                  coordinate, 11-bit fixed-point weights, exact 22-bit
//                  rounding (bit-exact with OpenCV for the integer factors of
//                  the pyramid; within one level otherwise)
//   k_gray         BGR -> grey with 16-bit fixed-point weights (7470, 38470,
//                  19596; round half up), equal to cv2.cvtColor BGR2GRAY on
//                  all 2^24 colours, as float
//   k_canny_*      3x3 Sobel per channel (replicated border), L1 magnitude of
//                  the strongest channel, tangent-sector non-maximum
//                  suppression, hysteresis over 8-connected weak pixels
//                  (tile-local propagation to a fixed point, repeated until
//                  no tile changes).
#include "aux_kernels.cuh"
#include "ctx.hpp"

#include <algorithm>

namespace hpm {

__global__ void k_resize_u8c3(const uint8_t* __restrict__ src, int sw, int sh, uint8_t* __restrict__ dst, int dw,
                              int dh) {
    const int dx = blockIdx.x * blockDim.x + threadIdx.x;
    const int dy = blockIdx.y * blockDim.y + threadIdx.y;
    if (dx >= dw || dy >= dh) return;
    const double sxs = 1.0 / ((double)dw / sw), sys = 1.0 / ((double)dh / sh);
    float fx = (float)((dx + 0.5) * sxs - 0.5);
    int sx = (int)floorf(fx);
    fx -= sx;
    if (sx < 0) { fx = 0.f; sx = 0; }
    if (sx >= sw - 1) { fx = 0.f; sx = sw - 1; }
    const int sx1 = min(sx + 1, sw - 1);
    float fy = (float)((dy + 0.5) * sys - 0.5);
    int sy = (int)floorf(fy);
    fy -= sy;
    if (sy < 0) { fy = 0.f; sy = 0; }
    if (sy >= sh - 1) { fy = 0.f; sy = sh - 1; }
    const int sy1 = min(sy + 1, sh - 1);
    const int a0 = __float2int_rn((1.0f - fx) * 2048.0f), a1 = __float2int_rn(fx * 2048.0f);
    const long long b0 = __float2int_rn((1.0f - fy) * 2048.0f), b1 = __float2int_rn(fy * 2048.0f);
    const uint8_t* r0 = src + (size_t)sy * sw * 3;
    const uint8_t* r1 = src + (size_t)sy1 * sw * 3;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const long long h0 = (long long)r0[3 * sx + c] * a0 + (long long)r0[3 * sx1 + c] * a1;
        const long long h1 = (long long)r1[3 * sx + c] * a0 + (long long)r1[3 * sx1 + c] * a1;
        long long v = (h0 * b0 + h1 * b1 + (1LL << 21)) >> 22;
        v = v < 0 ? 0 : (v > 255 ? 255 : v);
        dst[((size_t)dy * dw + dx) * 3 + c] = (uint8_t)v;
    }
}

__global__ void k_gray(const uint8_t* __restrict__ bgr, int n, float* __restrict__ gray) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b = bgr[3 * (size_t)i], g = bgr[3 * (size_t)i + 1], r = bgr[3 * (size_t)i + 2];
    gray[i] = (float)((b * 7470 + g * 38470 + r * 19596 + (1 << 15)) >> 16);
}

// Sobel 3x3 (replicated border), strongest channel by |dx|+|dy| (first on ties),
// and the non-maximum suppression class: 0 none, 1 weak, 2 strong.
__global__ void k_canny_grad(const uint8_t* __restrict__ bgr, int W, int H, int* __restrict__ mag,
                             short2* __restrict__ grad) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const int xm = max(x - 1, 0), xp = min(x + 1, W - 1), ym = max(y - 1, 0), yp = min(y + 1, H - 1);
    int best = -1, bdx = 0, bdy = 0;
    for (int c = 0; c < 3; ++c) {
        auto P = [&](int xx, int yy) { return (int)bgr[((size_t)yy * W + xx) * 3 + c]; };
        const int dx = (P(xp, ym) + 2 * P(xp, y) + P(xp, yp)) - (P(xm, ym) + 2 * P(xm, y) + P(xm, yp));
        const int dy = (P(xm, yp) + 2 * P(x, yp) + P(xp, yp)) - (P(xm, ym) + 2 * P(x, ym) + P(xp, ym));
        const int m = abs(dx) + abs(dy);
        if (m > best) { best = m; bdx = dx; bdy = dy; }
    }
    mag[(size_t)y * W + x] = best;
    grad[(size_t)y * W + x] = make_short2((short)bdx, (short)bdy);
}

__global__ void k_canny_nms(const int* __restrict__ mag, const short2* __restrict__ grad, int W, int H, int low,
                            int high, uint8_t* __restrict__ state) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    auto M = [&](int xx, int yy) { return (xx < 0 || xx >= W || yy < 0 || yy >= H) ? 0 : mag[(size_t)yy * W + xx]; };
    const int m = mag[(size_t)y * W + x];
    uint8_t s = 0;
    if (m > low) {
        const short2 g = grad[(size_t)y * W + x];
        const long long xs = abs((int)g.x);
        const long long ys = (long long)abs((int)g.y) << 15;
        const long long tg22x = xs * 13573;  // round(tan(22.5 deg) * 2^15)
        bool ok;
        if (ys < tg22x) {
            ok = m > M(x - 1, y) && m >= M(x + 1, y);
        } else {
            const long long tg67x = tg22x + (xs << 16);
            if (ys > tg67x) {
                ok = m > M(x, y - 1) && m >= M(x, y + 1);
            } else {
                const int sgn = (((int)g.x ^ (int)g.y) < 0) ? -1 : 1;
                ok = m > M(x - sgn, y - 1) && m > M(x + sgn, y + 1);
            }
        }
        if (ok) s = m > high ? 2 : 1;
    }
    state[(size_t)y * W + x] = s;
}

// Hysteresis: weak pixels 8-connected to a strong pixel become strong.  Each
// block propagates inside its 32x8 tile (plus a one-pixel halo it reads) to a
// fixed point; the host repeats the launch until no block changed anything.
constexpr int kHystTile = 32;  // hysteresis tiles are 32 x 32 pixels, one thread each

__global__ void k_canny_hyst(uint8_t* __restrict__ state, int W, int H, int* __restrict__ changed) {
    __shared__ uint8_t t[kHystTile + 2][kHystTile + 2];
    __shared__ int any;
    const int x0 = blockIdx.x * kHystTile, y0 = blockIdx.y * kHystTile;
    for (int k = threadIdx.y * kHystTile + threadIdx.x; k < (kHystTile + 2) * (kHystTile + 2);
         k += kHystTile * kHystTile) {
        const int ty = k / (kHystTile + 2), tx = k % (kHystTile + 2);
        const int gx = x0 + tx - 1, gy = y0 + ty - 1;
        t[ty][tx] = (gx >= 0 && gx < W && gy >= 0 && gy < H) ? state[(size_t)gy * W + gx] : 0;
    }
    __syncthreads();
    const int lx = threadIdx.x + 1, ly = threadIdx.y + 1;
    const int gx = x0 + threadIdx.x, gy = y0 + threadIdx.y;
    bool mine = false;
    for (int iter = 0; iter < kHystTile * kHystTile; ++iter) {  // a path inside a tile has at most 1024 pixels
        if (threadIdx.x == 0 && threadIdx.y == 0) any = 0;
        __syncthreads();
        if (gx < W && gy < H && t[ly][lx] == 1) {
            bool strong = false;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) strong = strong || t[ly + dy][lx + dx] == 2;
            if (strong) { t[ly][lx] = 2; mine = true; any = 1; }
        }
        __syncthreads();
        if (!any) break;
        __syncthreads();
    }
    if (mine) {
        state[(size_t)gy * W + gx] = 2;
        *changed = 1;
    }
}

__global__ void k_canny_out(const uint8_t* __restrict__ state, int n, uint8_t* __restrict__ edges) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) edges[i] = state[i] == 2 ? 255 : 0;
}

template <class T>
static cudaError_t ensure_i(T*& p, size_t& cap, size_t n) {
    if (n <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) cap = n;
    return e;
}

// Builds the level image of a view from its original BGR image: resize (when
// the target differs), colour for fusion, grey + texture, Canny edges.
int Ctx::prepare_level_image(int view, int w, int h, const hpm_camera& cam) {
    cudaSetDevice(device);
    ViewState& v = views[view];
    if (!v.orig || v.orig_w <= 0) return fail(HPM_E_STATE, "view %d has no original image", view);
    const size_t n = (size_t)w * h;
    cudaError_t e = ensure_i(v.color, v.color_cap, n * 3);
    if (e != cudaSuccess) return cuda_fail(e, "alloc level colour");
    if (w == v.orig_w && h == v.orig_h) {
        e = cudaMemcpyAsync(v.color, v.orig, n * 3, cudaMemcpyDeviceToDevice, stream);
    } else {
        dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
        k_resize_u8c3<<<g, b, 0, stream>>>(v.orig, v.orig_w, v.orig_h, v.color, w, h);
        ++launches;
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return cuda_fail(e, "level resize");
    v.color_w = w;
    v.color_h = h;
    e = ensure_i(v.gray, v.gray_cap, n);
    if (e != cudaSuccess) return cuda_fail(e, "alloc grey");
    k_gray<<<(int)((n + 255) / 256), 256, 0, stream>>>(v.color, (int)n, v.gray);
    ++launches;
    v.w = w;
    v.h = h;
    v.cam = cam;
    v.cam.width = w;
    v.cam.height = h;
    int rc = bind_texture(view);
    if (rc) return rc;
    return canny_view(view);
}

int Ctx::canny_view(int view) {
    ViewState& v = views[view];
    const int W = v.color_w, H = v.color_h;
    const size_t n = (size_t)W * H;
    cudaError_t e = ensure_i(canny_mag, canny_mag_cap, n);
    if (e == cudaSuccess) e = ensure_i(canny_grad, canny_grad_cap, n);
    if (e == cudaSuccess) e = ensure_i(canny_state, canny_state_cap, n + 64);
    if (e == cudaSuccess) e = ensure_i(v.canny, v.canny_cap, n);
    if (e != cudaSuccess) return cuda_fail(e, "alloc canny");
    dim3 b(32, 8), g((W + 31) / 32, (H + 7) / 8);
    k_canny_grad<<<g, b, 0, stream>>>(v.color, W, H, canny_mag, canny_grad);
    k_canny_nms<<<g, b, 0, stream>>>(canny_mag, canny_grad, W, H, 50, 150, canny_state);
    launches += 2;
    int* d_changed = reinterpret_cast<int*>(canny_state + ((n + 3) & ~size_t(3)));  // one flag per round
    // A round grows every weak path to the end of its tile and one pixel into the next, so a path
    // crossing k tiles takes k rounds; long weak chains (flat, noisy regions) take hundreds.  Rounds
    // run kHystRounds at a time between host reads of their change flags: a round after one that
    // changed nothing finds the same state and changes nothing, so the extra rounds leave the edge
    // map as it was when the first of them had converged.
    constexpr int kHystRounds = 8;
    const dim3 hg((W + kHystTile - 1) / kHystTile, (H + kHystTile - 1) / kHystTile);
    // every round before the last marks at least one weak pixel strong, so the loop ends by itself
    // within (weak pixels + 1) rounds; n + 2 only bounds it
    const int max_rounds = (int)std::min<size_t>(n + 2, 0x7fffffff);
    for (int r0 = 0; r0 < max_rounds; r0 += kHystRounds) {
        const int batch = std::min(kHystRounds, max_rounds - r0);
        cudaMemsetAsync(d_changed, 0, 4 * (size_t)batch, stream);
        for (int r = 0; r < batch; ++r)
            k_canny_hyst<<<hg, dim3(kHystTile, kHystTile), 0, stream>>>(canny_state, W, H, d_changed + r);
        launches += batch;
        int changed[kHystRounds];
        e = cudaMemcpyAsync(changed, d_changed, 4 * (size_t)batch, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "canny hysteresis");
        bool done = false;
        for (int r = 0; r < batch; ++r) done = done || !changed[r];
        if (done) break;
    }
    k_canny_out<<<(int)((n + 255) / 256), 256, 0, stream>>>(canny_state, (int)n, v.canny);
    ++launches;
    v.canny_w = W;
    v.canny_h = H;
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "canny");
    return HPM_OK;
}

}  // namespace hpm
