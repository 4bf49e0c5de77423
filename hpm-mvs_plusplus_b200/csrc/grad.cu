// Differentiable form of the bilateral NCC and its adjoint (no counterpart in
// the reference, which only evaluates the cost: ComputeBilateralNCC,
// HPM.cu:375-448).
//
// Cost of pixel p under the camera-frame plane theta = (depth, nx, ny),
// nz = -sqrt(1 - nx^2 - ny^2), against source view j: the reference's
// bilateral NCC with the source sampled by exact bilinear interpolation (the
// texture unit's 8-bit weights are not differentiable).  The gradient is
// formed in three passes over the 36 warped samples, recomputing them rather
// than storing them: the weighted source mean, the centred second moments
// (compensated: no E[v^2] - E[v]^2 cancellation), then
//   dc/dv_k = (w_k / W) (-(r_k - mean_r) / sigma + cov (v_k - mean_s) / (sigma var_s))
//   dv_k/dm = -(g_k . b) u_k,   g_k = (Ix, Iy, -(Ix X + Iy Y)) / q_z
// through the homography H = A - b m^T, m = Kr^-T n / w, w = -depth (n . ray).
//
// k_cost_grad  costs and d cost / d theta for (pixel, hypothesis) pairs x S views;
// k_gn_refine  Gauss-Newton steps on the views' costs, per pixel of a view's maps.
#include "ctx.hpp"
#include "hpm_device.cuh"
#include "hpm_geometry.h"

namespace hpm {

struct SrcImages {
    const float* img[32];  // index j + 1: grey image of source j (row-major)
    int w[32], h[32];
};

namespace {

// Self-check of the gradient kernels: an index outside its buffer (which the
// clamping below rules out) is counted here and the access skipped, so a
// wrong index surfaces as an error status instead of a memory fault.
__device__ unsigned int g_grad_oob;

__device__ __forceinline__ float texel_c(const float* img, int w, int h, int x, int y) {
    x = min(max(x, 0), w - 1);
    y = min(max(y, 0), h - 1);
    if (!img || x < 0 || y < 0 || w <= 0 || h <= 0) {
        atomicAdd(&g_grad_oob, 1u);
        return 0.0f;
    }
    return __ldg(img + (size_t)y * w + x);
}

// Exact bilinear sample with clamp-to-edge addressing.  The position is first
// clamped to [-2, size + 1] (a NaN to -2): outside that range every tap reads
// the edge texel, so the value and the (zero) gradient are unchanged, and the
// integer tap index x0 + 1 cannot overflow for a sample position near a
// plane's horizon, where X grows without bound.
__device__ __forceinline__ float bilinear(const float* img, int w, int h, float X, float Y, float& gx, float& gy) {
    X = fminf(fmaxf(X, -2.0f), (float)w + 1.0f);
    Y = fminf(fmaxf(Y, -2.0f), (float)h + 1.0f);
    const float fx = floorf(X), fy = floorf(Y);
    const int x0 = __float2int_rz(fx), y0 = __float2int_rz(fy);
    const float ax = X - fx, ay = Y - fy;
    const float i00 = texel_c(img, w, h, x0, y0), i10 = texel_c(img, w, h, x0 + 1, y0);
    const float i01 = texel_c(img, w, h, x0, y0 + 1), i11 = texel_c(img, w, h, x0 + 1, y0 + 1);
    gx = (1 - ay) * (i10 - i00) + ay * (i11 - i01);
    gy = (1 - ax) * (i01 - i00) + ax * (i11 - i10);
    return (1 - ay) * ((1 - ax) * i00 + ax * i10) + ay * ((1 - ax) * i01 + ax * i11);
}

struct RefPatch {
    float w[36], r[36];
    float W, mean, var;
};

__device__ void ref_patch(const RunArgs& a, int px, int py, RefPatch& P) {
    const float center = texel_c(a.ref_img, a.W, a.H, px, py);
    const float two_ss = 2.0f * a.prm.sigma_spatial * a.prm.sigma_spatial;
    const float two_sc = 2.0f * a.prm.sigma_color * a.prm.sigma_color;
    float W = 0.f, Sr = 0.f;
#pragma unroll
    for (int k = 0; k < 36; ++k) {
        const int dx = -5 + 2 * (k / 6), dy = -5 + 2 * (k % 6);
        const float r = texel_c(a.ref_img, a.W, a.H, px + dx, py + dy);
        const float w = expf(-sqrtf((float)(dx * dx + dy * dy)) / two_ss - fabsf(r - center) / two_sc);
        P.w[k] = w;
        P.r[k] = r;
        W += w;
        Sr += w * r;
    }
    P.W = W;
    P.mean = Sr / W;
    float v = 0.f;
#pragma unroll
    for (int k = 0; k < 36; ++k) v += P.w[k] * (P.r[k] - P.mean) * (P.r[k] - P.mean);
    P.var = v / W;
}

// Cost of one view and, when grad is not null, d cost / d theta.
__device__ float cost_grad_view(const RunArgs& a, const SrcImages& si, const RefPatch& P, int px, int py,
                                const float theta[3], int j, float* grad) {
    if (grad) grad[0] = grad[1] = grad[2] = 0.f;
    if (P.var < 1e-5f) return 2.0f;
    const float nx = theta[1], ny = theta[2];
    const float nn = 1.0f - nx * nx - ny * ny;
    if (!(nn > 0.0f)) return 2.0f;
    const float nz = -sqrtf(nn);
    const hpm_camera& rc = a.cams[0];
    const float fx = rc.K[0], fy = rc.K[4], cx = rc.K[2], cy = rc.K[5];
    const float ray[3] = { (px - cx) / fx, (py - cy) / fy, 1.0f };
    const float nr = nx * ray[0] + ny * ray[1] + nz * ray[2];
    const float w = -theta[0] * nr;
    const float t[3] = { nx / fx, ny / fy, nz - nx * cx / fx - ny * cy / fy };
    const float m[3] = { t[0] / w, t[1] / w, t[2] / w };
    const float* A = a.basis[j + 1].A;
    const float* b = a.basis[j + 1].b;
    float H[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) H[3 * r + k] = A[3 * r + k] - b[r] * m[k];
    if (j < 0 || j > 30) {
        atomicAdd(&g_grad_oob, 1u);
        return 2.0f;
    }
    const float* img = si.img[j + 1];
    const int sw = si.w[j + 1], sh = si.h[j + 1];
    {
        const float qz = H[6] * px + H[7] * py + H[8];
        const float X = (H[0] * px + H[1] * py + H[2]) / qz, Y = (H[3] * px + H[4] * py + H[5]) / qz;
        if (!(X < sw && X >= 0.0f && Y < sh && Y >= 0.0f)) return 2.0f;
    }
    auto sample = [&](int k, float& X, float& Y, float& qz, float& gx, float& gy) -> float {
        const float ux = (float)(px - 5 + 2 * (k / 6)), uy = (float)(py - 5 + 2 * (k % 6));
        qz = H[6] * ux + H[7] * uy + H[8];
        X = (H[0] * ux + H[1] * uy + H[2]) / qz;
        Y = (H[3] * ux + H[4] * uy + H[5]) / qz;
        return bilinear(img, sw, sh, X, Y, gx, gy);
    };
    float X, Y, qz, gx, gy;
    float Ss = 0.f;
    for (int k = 0; k < 36; ++k) Ss += P.w[k] * sample(k, X, Y, qz, gx, gy);
    Ss /= P.W;
    float vs = 0.f, cv = 0.f;
    for (int k = 0; k < 36; ++k) {
        const float d = sample(k, X, Y, qz, gx, gy) - Ss;
        vs += P.w[k] * d * d;
        cv += P.w[k] * (P.r[k] - P.mean) * d;
    }
    const float var_s = vs / P.W, cov = cv / P.W;
    if (var_s < 1e-5f) return 2.0f;
    const float sig = sqrtf(P.var * var_s);
    const float c = 1.0f - cov / sig;
    if (c < 0.0f) return 0.0f;
    if (c > 2.0f) return 2.0f;
    if (!grad) return c;
    float dm0 = 0.f, dm1 = 0.f, dm2 = 0.f;
    for (int k = 0; k < 36; ++k) {
        const float v = sample(k, X, Y, qz, gx, gy);
        const float dcdv = P.w[k] / P.W * (-(P.r[k] - P.mean) / sig + cov * (v - Ss) / (sig * var_s));
        const float gb = (gx * b[0] + gy * b[1] - (gx * X + gy * Y) * b[2]) / qz;
        const float f = -dcdv * gb;
        dm0 += f * (float)(px - 5 + 2 * (k / 6));
        dm1 += f * (float)(py - 5 + 2 * (k % 6));
        dm2 += f;
    }
    const float dw = -(dm0 * m[0] + dm1 * m[1] + dm2 * m[2]) / w;
    float dn0 = (dm0 / fx - dm2 * cx / fx) / w, dn1 = (dm1 / fy - dm2 * cy / fy) / w, dn2 = dm2 / w;
    dn0 += dw * (-theta[0] * ray[0]);
    dn1 += dw * (-theta[0] * ray[1]);
    dn2 += dw * (-theta[0] * ray[2]);
    grad[0] = dw * (-nr);
    grad[1] = dn0 + dn2 * (-nx / nz);
    grad[2] = dn1 + dn2 * (-ny / nz);
    return c;
}

__global__ void k_cost_grad(const __grid_constant__ RunArgs a, const __grid_constant__ SrcImages si, int n,
                            const int32_t* __restrict__ px, const float* __restrict__ theta,
                            float* __restrict__ cost, float* __restrict__ grad) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int x = px[2 * k], y = px[2 * k + 1];
    if (x < 0 || x >= a.W || y < 0 || y >= a.H) {
        atomicAdd(&g_grad_oob, 1u);
        return;
    }
    RefPatch P;
    ref_patch(a, x, y, P);
    const float th[3] = { theta[3 * k], theta[3 * k + 1], theta[3 * k + 2] };
    for (int j = 0; j < a.S; ++j) {
        float g[3];
        const float c = cost_grad_view(a, si, P, x, y, th, j, grad ? g : nullptr);
        cost[(size_t)k * a.S + j] = c;
        if (grad)
            for (int q = 0; q < 3; ++q) grad[((size_t)k * a.S + j) * 3 + q] = g[q];
    }
}

// d = M^-1 rhs for a 3x3 M through its adjugate; false when M is singular.
__device__ bool solve3(const float M[9], const float rhs[3], float d[3]) {
    const float a00 = M[4] * M[8] - M[5] * M[7], a01 = M[2] * M[7] - M[1] * M[8], a02 = M[1] * M[5] - M[2] * M[4];
    const float a10 = M[5] * M[6] - M[3] * M[8], a11 = M[0] * M[8] - M[2] * M[6], a12 = M[2] * M[3] - M[0] * M[5];
    const float a20 = M[3] * M[7] - M[4] * M[6], a21 = M[1] * M[6] - M[0] * M[7], a22 = M[0] * M[4] - M[1] * M[3];
    const float det = M[0] * a00 + M[1] * a10 + M[2] * a20;
    if (!(fabsf(det) > 1e-30f)) return false;
    const float inv = 1.0f / det;
    d[0] = (a00 * rhs[0] + a01 * rhs[1] + a02 * rhs[2]) * inv;
    d[1] = (a10 * rhs[0] + a11 * rhs[1] + a12 * rhs[2]) * inv;
    d[2] = (a20 * rhs[0] + a21 * rhs[1] + a22 * rhs[2]) * inv;
    return true;
}

// Gauss-Newton on the sum of squared per-view costs, a Levenberg damping that
// grows tenfold on every rejected step; the valid views are those with a cost
// in (0, 2) at the start.  Depth stays in [dmin, dmax].
__global__ void k_gn_refine(const __grid_constant__ RunArgs a, const __grid_constant__ SrcImages si, int steps,
                            float* __restrict__ depth, float* __restrict__ normal, float* __restrict__ cost_out,
                            size_t n_px) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.W || y >= a.H) return;
    const size_t i = (size_t)y * a.W + x;
    if (i >= n_px) {
        atomicAdd(&g_grad_oob, 1u);
        return;
    }
    const hpm_camera& c0 = a.cams[0];
    float d0 = depth[i];
    if (!(d0 > 0.0f)) return;
    // world normal -> camera frame (R n)
    const float nwx = normal[3 * i], nwy = normal[3 * i + 1], nwz = normal[3 * i + 2];
    float n[3] = { c0.R[0] * nwx + c0.R[1] * nwy + c0.R[2] * nwz, c0.R[3] * nwx + c0.R[4] * nwy + c0.R[5] * nwz,
                   c0.R[6] * nwx + c0.R[7] * nwy + c0.R[8] * nwz };
    const float len = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    if (!(len > 0.0f)) return;
    if (n[2] > 0.0f) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
    float th[3] = { d0, n[0] / len, n[1] / len };
    RefPatch P;
    ref_patch(a, x, y, P);
    uint32_t valid = 0;
    float e0 = 0.f;
    for (int j = 0; j < a.S; ++j) {
        const float c = cost_grad_view(a, si, P, x, y, th, j, nullptr);
        if (c > 0.0f && c < 2.0f) { valid |= 1u << j; e0 += c * c; }
    }
    if (__popc(valid) < 2) return;
    float lambda = 1e-3f;
    for (int it = 0; it < steps; ++it) {
        float JtJ[9] = { 0.f }, Jtr[3] = { 0.f, 0.f, 0.f };
        for (int j = 0; j < a.S; ++j) {
            if (!((valid >> j) & 1u)) continue;
            float g[3];
            const float c = cost_grad_view(a, si, P, x, y, th, j, g);
            for (int r = 0; r < 3; ++r) {
                Jtr[r] += g[r] * c;
                for (int q = 0; q < 3; ++q) JtJ[3 * r + q] += g[r] * g[q];
            }
        }
        bool accepted = false;
        for (int attempt = 0; attempt < 4 && !accepted; ++attempt) {
            float M[9], rhs[3] = { -Jtr[0], -Jtr[1], -Jtr[2] }, dlt[3];
            for (int q = 0; q < 9; ++q) M[q] = JtJ[q];
            for (int q = 0; q < 3; ++q) M[4 * q] += lambda * (JtJ[4 * q] + 1e-12f);
            if (!solve3(M, rhs, dlt)) { lambda *= 10.f; continue; }
            float tn[3] = { th[0] + dlt[0], th[1] + dlt[1], th[2] + dlt[2] };
            if (!(tn[0] >= a.prm.depth_min && tn[0] <= a.prm.depth_max) ||
                !(tn[1] * tn[1] + tn[2] * tn[2] < 0.999f)) { lambda *= 10.f; continue; }
            float e1 = 0.f;
            for (int j = 0; j < a.S; ++j)
                if ((valid >> j) & 1u) { const float c = cost_grad_view(a, si, P, x, y, tn, j, nullptr); e1 += c * c; }
            if (e1 < e0) {
                th[0] = tn[0]; th[1] = tn[1]; th[2] = tn[2];
                e0 = e1;
                lambda = fmaxf(lambda * 0.1f, 1e-6f);
                accepted = true;
            } else {
                lambda *= 10.f;
            }
        }
        if (!accepted) break;
    }
    // camera-frame normal -> world frame (R^T n)
    const float nz = -sqrtf(fmaxf(0.f, 1.f - th[1] * th[1] - th[2] * th[2]));
    depth[i] = th[0];
    normal[3 * i] = c0.R[0] * th[1] + c0.R[3] * th[2] + c0.R[6] * nz;
    normal[3 * i + 1] = c0.R[1] * th[1] + c0.R[4] * th[2] + c0.R[7] * nz;
    normal[3 * i + 2] = c0.R[2] * th[1] + c0.R[5] * th[2] + c0.R[8] * nz;
    if (cost_out) cost_out[i] = sqrtf(e0 / __popc(valid));
}

// Resets the self-check counter before a launch and reads it after one.
static cudaError_t grad_oob_reset(cudaStream_t st) {
    const unsigned int zero = 0;
    return cudaMemcpyToSymbolAsync(g_grad_oob, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, st);
}

static cudaError_t grad_oob_read(cudaStream_t st, unsigned int* n) {
    cudaError_t e = cudaMemcpyFromSymbolAsync(n, g_grad_oob, sizeof(*n), 0, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
}

}  // namespace

int Ctx::fill_src_images(const int32_t* srcs, int n_src, SrcImages& si) {
    for (int j = 0; j < n_src; ++j) {
        const ViewState& v = views[srcs[j]];
        if (!v.gray) return fail(HPM_E_STATE, "source view %d has no grey image", srcs[j]);
        si.img[j + 1] = v.gray;
        si.w[j + 1] = v.w;
        si.h[j + 1] = v.h;
    }
    return HPM_OK;
}

int Ctx::eval_cost_grad(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int n, const int32_t* px,
                        const float* theta, float* cost, float* grad) {
    cudaSetDevice(device);
    if (n < 0 || (n > 0 && (!px || !theta || !cost))) return fail(HPM_E_INVALID, "hpm_eval_cost_grad: bad arguments");
    RunArgs a;
    int rc = fill_run_args(ref, srcs, n_src, params, a);
    if (rc) return rc;
    SrcImages si{};
    if ((rc = fill_src_images(srcs, n_src, si))) return rc;
    if (n == 0) return HPM_OK;
    for (int k = 0; k < n; ++k)
        if (px[2 * k] < 0 || px[2 * k] >= a.W || px[2 * k + 1] < 0 || px[2 * k + 1] >= a.H)
            return fail(HPM_E_INVALID, "pixel %d outside the reference image", k);
    const size_t bytes = (size_t)n * (8 + 12) + (size_t)n * n_src * 16 + 256;
    cudaError_t e = ensure_scratch(bytes);
    if (e != cudaSuccess) return cuda_fail(e, "alloc scratch");
    int32_t* d_px = reinterpret_cast<int32_t*>(scratch);
    float* d_th = reinterpret_cast<float*>(scratch + (size_t)n * 8);
    float* d_c = reinterpret_cast<float*>(scratch + (size_t)n * 20);
    float* d_g = d_c + (size_t)n * n_src;
    e = cudaMemcpyAsync(d_px, px, (size_t)n * 8, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_th, theta, (size_t)n * 12, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return cuda_fail(e, "upload hypotheses");
    if ((e = grad_oob_reset(stream)) != cudaSuccess) return cuda_fail(e, "self-check reset");
    k_cost_grad<<<(n + 127) / 128, 128, 0, stream>>>(a, si, n, d_px, d_th, d_c, grad ? d_g : nullptr);
    ++launches;
    unsigned int oob = 0;
    if ((e = grad_oob_read(stream, &oob)) != cudaSuccess) return cuda_fail(e, "cost gradient");
    if (oob) return fail(HPM_E_CUDA, "cost gradient: %u out-of-range accesses skipped", oob);
    e = cudaMemcpyAsync(cost, d_c, (size_t)n * n_src * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && grad) e = cudaMemcpyAsync(grad, d_g, (size_t)n * n_src * 12, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "download costs");
    return HPM_OK;
}

int Ctx::eval_cost_grad_device(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int n,
                               const int32_t* d_px, const float* d_theta, float* d_cost, float* d_grad) {
    cudaSetDevice(device);
    if (n < 0 || (n > 0 && (!d_px || !d_theta || !d_cost)))
        return fail(HPM_E_INVALID, "hpm_eval_cost_grad_device: bad arguments");
    RunArgs a;
    int rc = fill_run_args(ref, srcs, n_src, params, a);
    if (rc) return rc;
    SrcImages si{};
    if ((rc = fill_src_images(srcs, n_src, si))) return rc;
    if (n == 0) return HPM_OK;
    cudaError_t e;
    if ((e = grad_oob_reset(stream)) != cudaSuccess) return cuda_fail(e, "self-check reset");
    // pixels outside the reference image are skipped and counted by the kernel (no host copy to check them)
    k_cost_grad<<<(n + 127) / 128, 128, 0, stream>>>(a, si, n, d_px, d_theta, d_cost, d_grad);
    ++launches;
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "cost gradient launch");
    unsigned int oob = 0;
    if ((e = grad_oob_read(stream, &oob)) != cudaSuccess) return cuda_fail(e, "cost gradient");
    if (oob) return fail(HPM_E_INVALID, "cost gradient: %u pixels or samples outside their images skipped", oob);
    return HPM_OK;
}

int Ctx::gn_refine(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int depth_kind, int steps) {
    cudaSetDevice(device);
    if (steps < 0 || steps > 100) return fail(HPM_E_INVALID, "steps must be 0..100");
    if (depth_kind != HPM_MAP_DEPTH && depth_kind != HPM_MAP_DEPTH_GEOM)
        return fail(HPM_E_INVALID, "depth_kind must be HPM_MAP_DEPTH or HPM_MAP_DEPTH_GEOM");
    RunArgs a;
    int rc = fill_run_args(ref, srcs, n_src, params, a);
    if (rc) return rc;
    SrcImages si{};
    if ((rc = fill_src_images(srcs, n_src, si))) return rc;
    ViewState& v = views[ref];
    DevMap& dm = v.maps[depth_kind];
    DevMap& nm = v.maps[HPM_MAP_NORMAL];
    if (!dm.ptr || dm.w != v.w || dm.h != v.h || !nm.ptr || nm.w != v.w || nm.h != v.h)
        return fail(HPM_E_STATE, "view %d needs depth and normal maps of its size", ref);
    cudaError_t e = ensure_map(ref, HPM_MAP_COST, v.w, v.h);
    if (e != cudaSuccess) return cuda_fail(e, "alloc cost map");
    dim3 block(16, 8), grid((v.w + 15) / 16, (v.h + 7) / 8);
    if ((e = grad_oob_reset(stream)) != cudaSuccess) return cuda_fail(e, "self-check reset");
    k_gn_refine<<<grid, block, 0, stream>>>(a, si, steps, dm.ptr, nm.ptr, v.maps[HPM_MAP_COST].ptr,
                                            (size_t)v.w * v.h);
    ++launches;
    e = cudaGetLastError();
    unsigned int oob = 0;
    if (e == cudaSuccess) e = grad_oob_read(stream, &oob);
    if (e != cudaSuccess) return cuda_fail(e, "gauss-newton refinement");
    if (oob) return fail(HPM_E_CUDA, "gauss-newton refinement: %u out-of-range accesses skipped", oob);
    return HPM_OK;
}

}  // namespace hpm

extern "C" {

int hpm_eval_cost_grad(hpm_ctx* ctx, int ref, const int32_t* srcs, int n_src, const hpm_params* params, int n,
                       const int32_t* px, const float* theta, float* cost, float* grad) {
    if (!ctx) return HPM_E_INVALID;
    return reinterpret_cast<hpm::Ctx*>(ctx)->eval_cost_grad(ref, srcs, n_src, params, n, px, theta, cost, grad);
}

int hpm_eval_cost_grad_device(hpm_ctx* ctx, int ref, const int32_t* srcs, int n_src, const hpm_params* params,
                              int n, const int32_t* d_px, const float* d_theta, float* d_cost, float* d_grad) {
    if (!ctx) return HPM_E_INVALID;
    return reinterpret_cast<hpm::Ctx*>(ctx)->eval_cost_grad_device(ref, srcs, n_src, params, n, d_px, d_theta, d_cost,
                                                                   d_grad);
}

int hpm_gn_refine(hpm_ctx* ctx, int ref, const int32_t* srcs, int n_src, const hpm_params* params, int depth_kind,
                  int steps) {
    if (!ctx) return HPM_E_INVALID;
    return reinterpret_cast<hpm::Ctx*>(ctx)->gn_refine(ref, srcs, n_src, params, depth_kind, steps);
}

}  // extern "C"
