// PatchMatch kernels of the plain FP32 path (sm_100a): random initialisation,
// red/black checkerboard propagation with the non-local sampling pattern, joint
// view selection and refinement, and the depth/normal export.
//
// Algorithm: HPM-MVS++ HPM.cu:567-842 (init, refinement), 843-1873 (standard
// propagation), 1875-2791 (mandatory consistency), 2793-2842 (schedule,
// export).  The kernels are laid out differently:
//   * one thread per pixel of the active colour, block 32 x (BLK/32) over
//     (x, row pair) so a warp covers a 32 x 2 strip (coherent texture reads);
//   * the pixel's reference patch (weights and weighted texels) lives in
//     registers and is built once per launch instead of once per NCC;
//   * per-pixel cost rows, view weights, final costs and positions live in a
//     per-thread column of shared memory (stride BLK, conflict-free);
//   * NCCs whose view weight is zero are not evaluated (their product with the
//     zero weight is exactly 0 because the NCC is never NaN), and a reference
//     patch with variance < 1e-5 yields cost 2 for every hypothesis without
//     sampling (exactly the reference's result).
// Arithmetic follows include/hpm_fp.h (IEEE fp32, explicit fused multiply-adds),
// which the CPU oracle shares, so the two differ only where the texture unit's
// filtered sample does (about 0.6 % of samples, by one ulp).
#include "hpm_device.cuh"
#include "pm_kernels.cuh"

#include <float.h>

namespace hpm {


// CNT: the counting build of a kernel (profiling); the timed build has it off
// so the counters do not change its code.
template <int NS, int BLK, bool CNT = false>
struct Scratch {
    float* base;  // smem + threadIdx linear
    static constexpr bool kCount = CNT;
    // cost rows 0-7 (directions), row 8 (the hypothesis costed against the
    // selected views), view weights, final costs, candidate positions
    static constexpr int kWords = 10 * NS + 16;
    __device__ __forceinline__ float& ca(int d, int j) const { return base[(d * NS + j) * BLK]; }
    __device__ __forceinline__ float& vw(int j) const { return base[(9 * NS + j) * BLK]; }
    __device__ __forceinline__ float& fc(int d) const { return base[(10 * NS + d) * BLK]; }
    __device__ __forceinline__ int& pos(int d) const { return reinterpret_cast<int*>(base)[(10 * NS + 8 + d) * BLK]; }
};

// Statistics of a pixel's reference patch (the view-independent part of the NCC).
struct RefStats {
    float mean;   // sum_ref / weight_sum
    float var;    // reference variance
    float inv_w;  // 1 / weight_sum
};

struct Patch {
    float2 p[kPatchSamples];  // (w_k, w_k * r_k)
    RefStats rs;
};

__device__ __forceinline__ void build_patch(const RunArgs& a, int px, int py, Patch& P) {
    const float* __restrict__ ref = a.ref_img;
    const int W = a.W, H = a.H;
    const float center = __ldg(ref + (size_t)clampi(py, 0, H - 1) * W + clampi(px, 0, W - 1));
    const float two_ss = 2.0f * a.prm.sigma_spatial * a.prm.sigma_spatial;
    const float two_sc = 2.0f * a.prm.sigma_color * a.prm.sigma_color;
    // shifted moments (precision form): the patch relative to its centre texel; shift 0 is the plain arithmetic
    const float cs = a.ncc_shift ? center : 0.0f;
    float s_r = 0.f, s_rr = 0.f, s_w = 0.f;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        float r_r = 0.f, r_rr = 0.f, r_w = 0.f;
        const int dx = -kPatchRadius + kPatchStep * i;
        const int x = clampi(px + dx, 0, W - 1);
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            const int dy = -kPatchRadius + kPatchStep * j;
            const float r = __ldg(ref + (size_t)clampi(py + dy, 0, H - 1) * W + x);
            const float sd = sqrtf((float)(dx * dx + dy * dy));
            const float w = hpm_expf(-sd / two_ss - fabsf(r - center) / two_sc);
            const float rs = r - cs;
            const float wr = w * rs;
            P.p[i * 6 + j] = make_float2(w, wr);
            r_r += wr;
            r_rr = hpm_fma(wr, rs, r_rr);
            r_w += w;
        }
        s_r += r_r; s_rr += r_rr; s_w += r_w;
    }
    P.rs.inv_w = 1.0f / s_w;
    P.rs.mean = s_r * P.rs.inv_w;
    P.rs.var = s_rr * P.rs.inv_w - P.rs.mean * P.rs.mean;
}

// m = Kr^-T n / d of a camera-frame hypothesis: the view-independent part of
// its homographies (include/hpm_geometry.h).
struct PlaneM {
    float m[3];
};

__device__ __forceinline__ PlaneM plane_m(const RunArgs& a, float4 pl) {
    PlaneM r;
    hpm_plane_m(a.kinv, pl.x, pl.y, pl.z, pl.w, r.m);
    return r;
}

// One bilateral NCC (HPM.cu:375-448) with the patch in registers.  CNT: the
// counting build also counts the NCCs that sample the source (hyp_count[2]).
template <bool CNT = false>
__device__ __forceinline__ float ncc_view(const RunArgs& a, const Patch& P, int px, int py, const PlaneM& pm, int j) {
    const float cost_max = 2.0f;
    if (P.rs.var < 1e-5f) return cost_max;
    const hpm_camera& sc = a.cams[j + 1];
    float H[9];
    hpm_homography(a.basis[j + 1].A, a.basis[j + 1].b, pm.m, H);
    const int sw = sc.width, sh = sc.height;
    float iz_c;
    {
        const float fx = (float)px, fy = (float)py;
        const float cx = hpm_fma(H[0], fx, hpm_fma(H[1], fy, H[2]));
        const float cy = hpm_fma(H[3], fx, hpm_fma(H[4], fy, H[5]));
        const float cz = hpm_fma(H[6], fx, hpm_fma(H[7], fy, H[8]));
        iz_c = 1.0f / cz;
        const float ux = cx * iz_c, uy = cy * iz_c;
        if (ux >= sw || ux < 0.0f || uy >= sh || uy < 0.0f) return cost_max;
    }
    if (CNT) {  // one atomic per group of converged lanes
        unsigned lane;
        asm("mov.u32 %0, %%laneid;" : "=r"(lane));
        const unsigned m = __activemask();
        if (lane == (unsigned)(__ffs(m) - 1)) atomicAdd(a.hyp_count + 2, (unsigned long long)__popc(m));
    }
    const cudaTextureObject_t tex = a.tex[j + 1];
    float s_s = 0.f, s_ss = 0.f, s_rs = 0.f;
    float vshift = 0.0f;  // shifted moments: the source patch relative to its first sample
    // two patch columns (12 fetches) are issued before their moments are summed: more fetches in
    // flight per warp at the same register budget; the summation order is the oracle's
#pragma unroll
    for (int i0 = 0; i0 < 6; i0 += 2) {
        float v[2][6];
#pragma unroll
        for (int g = 0; g < 2; ++g) {
            const float x = (float)(px - kPatchRadius + kPatchStep * (i0 + g));
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                const float y = (float)(py - kPatchRadius + kPatchStep * k);
                const float qx = hpm_fma(H[0], x, hpm_fma(H[1], y, H[2]));
                const float qy = hpm_fma(H[3], x, hpm_fma(H[4], y, H[5]));
                const float qz = hpm_fma(H[6], x, hpm_fma(H[7], y, H[8]));
                const float iz = hpm_recip_near(qz, iz_c);
                v[g][k] = tex2D<float>(tex, hpm_fma(qx, iz, 0.5f), hpm_fma(qy, iz, 0.5f));
            }
        }
#pragma unroll
        for (int g = 0; g < 2; ++g) {
            const int i = i0 + g;
            if (i == 0 && a.ncc_shift) vshift = v[0][0];
            float r_s = 0.f, r_ss = 0.f, r_rs = 0.f;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                const float2 w = P.p[i * 6 + k];
                const float vk = v[g][k] - vshift;
                const float ws = w.x * vk;
                r_s += ws;
                r_ss = hpm_fma(ws, vk, r_ss);
                r_rs = hpm_fma(w.y, vk, r_rs);
            }
            s_s += r_s; s_ss += r_ss; s_rs += r_rs;
        }
    }
    s_s *= P.rs.inv_w; s_ss *= P.rs.inv_w; s_rs *= P.rs.inv_w;
    const float var_s = s_ss - s_s * s_s;
    if (var_s < a.var_s_min) return cost_max;
    const float cov = s_rs - P.rs.mean * s_s;
    const float vrs = sqrtf(P.rs.var * var_s);
    return fmaxf(0.0f, fminf(cost_max, 1.0f - cov / vrs));
}

// ---------------------------------------------------------------- init

template <int NS, int BLK, bool CNT>
__device__ float initial_cost(const RunArgs& a, const Patch& P, int px, int py, float4 pl, uint32_t* sel_out,
                              const Scratch<NS, BLK, CNT>& s) {
    const float cost_max = 2.0f;
    const int S = a.S;
    int valid = 0;
    if (CNT) atomicAdd(a.hyp_count, (unsigned long long)a.S);
    const PlaneM pm = plane_m(a, pl);
#pragma unroll 1
    for (int j = 0; j < S; ++j) {
        const float c = ncc_view(a, P, px, py, pm, j);
        s.ca(0, j) = c;
        s.ca(1, j) = c;
        if (c < cost_max) ++valid;
    }
    // insertion sort of row 1 (HPM.cu:15-24)
    for (int i = 1; i < S; ++i) {
        const float t = s.ca(1, i);
        int k = i;
        for (; k >= 1 && t < s.ca(1, k - 1); --k) s.ca(1, k) = s.ca(1, k - 1);
        s.ca(1, k) = t;
    }
    uint32_t sel = 0;
    const int top_k = min(valid, a.prm.top_k);
    float result = cost_max;
    if (top_k > 0) {
        float cost = 0.0f;
        for (int i = 0; i < top_k; ++i) cost += s.ca(1, i);
        const float thr = s.ca(1, top_k - 1);
        for (int i = 0; i < S; ++i)
            if (s.ca(0, i) <= thr) sel |= (1u << i);
        result = cost / top_k;
    }
    *sel_out = sel;
    return result;
}

__device__ __forceinline__ float spatial_gauss(float x1, float y1, float x2, float y2, float sigma) {
    const float dx = x1 - x2, dy = y1 - y2;
    const float dis = dx * dx + dy * dy - 0.0f;
    return (float)exp(-1.0 * dis / (2 * sigma * sigma));
}

__device__ __forceinline__ float range_gauss(float x, float sigma) {
    return (float)exp(-1.0 * (x * x) / (2 * sigma * sigma));
}

template <int NS, int BLK, bool CNT>
__device__ __forceinline__ void init_pixel(const RunArgs& a, const Scratch<NS, BLK, CNT>& s, int px, int py) {
    const int W = a.W, H = a.H;
    if (px >= W || py >= H) return;
    const int center = py * W + px;
    const hpm_camera& c0 = a.cams[0];
    const uint32_t mode = a.prm.mode;
    const bool geom = mode & HPM_MODE_GEOM, prior = mode & HPM_MODE_PRIOR, hier = mode & HPM_MODE_HIERARCHY;
    const bool ups = mode & HPM_MODE_UPSAMPLE, mand = mode & HPM_MODE_MAND;
    PixelRng rng;
    rng.init(a.seed, a.view_id, px, py, 0);

    if (!prior && !mand) a.texture[center] = texture_term(a.canny, W, H, px, py);

    Patch P;
    build_patch(a, px, py, P);
    uint32_t sel = 0;
    if (!geom && !hier && !prior) {
        const float depth = rng.uniform() * (a.prm.depth_max - a.prm.depth_min) + a.prm.depth_min;
        float4 pl = random_normal(c0, px, py, rng, depth);
        pl.w = distance_to_origin(c0, px, py, depth, pl);
        a.planes[center] = pl;
        a.costs[center] = initial_cost(a, P, px, py, pl, &sel, s);
        a.sel[center] = sel;
    } else if (prior) {
        if (a.pmask[center] > 0) {
            if (a.conf[center] > 0.3) {
                float4 pl = a.planes[center];
                pl.w = distance_to_origin(c0, px, py, pl.w, pl);
                a.planes[center] = pl;
                a.costs[center] = 0.1f;
            } else if (a.costs[center] > 0.1f) {
                const float perturbation = 0.02f;
                const float4 pp = a.prior[center];
                float dp = pp.w;  // the prior's offset is used as a depth (HPM.cu:603-604)
                const float dmin_p = (1 - 3 * perturbation) * dp;
                const float dmax_p = (1 + 3 * perturbation) * dp;
                dp = rng.uniform() * (dmax_p - dmin_p) + dmin_p;
                float4 pl = perturbed_normal(c0, px, py, pp, rng, (float)(3 * perturbation * 3.14159265358979323846));
                pl.w = dp;
                a.planes[center] = pl;
                a.costs[center] = initial_cost(a, P, px, py, pl, &sel, s);
                a.sel[center] = sel;
            } else {
                float4 pl = a.planes[center];
                pl.w = distance_to_origin(c0, px, py, pl.w, pl);
                a.planes[center] = pl;
                a.costs[center] = initial_cost(a, P, px, py, pl, &sel, s);
                a.sel[center] = sel;
            }
        } else {
            float4 pl = a.planes[center];
            pl.w = distance_to_origin(c0, px, py, pl.w, pl);
            a.planes[center] = pl;
            if (a.conf[center] > 0.3) a.costs[center] = 0.1f;
        }
    } else if (ups) {
        const int scols = a.prm.scaled_cols, srows = a.prm.scaled_rows;
        const float sc_f = (float)scols, sr_f = (float)srows;
        const float scale = (float)(1.0 * sc_f / W);
        const float sigmad = 0.50f, sigmar = 25.5f;
        const int image_scale = (int)fmaxf(W / sc_f, H / sr_f);
        const int nn = (image_scale * image_scale + 1) / 2;
        const float o_y = py * scale, o_x = px * scale;
        const float ref_pix = __ldg(a.ref_img + center);
        float nf = 0.0f;
        float n0 = 0.0f, n1 = 0.0f, n2 = 0.0f;
        for (int j = -nn; j <= nn; ++j) {
            int r_y = __float2int_rz(o_y + j);
            r_y = (r_y > 0 ? (r_y < sr_f ? r_y : srows - 1) : 0);
            const int r_ys = clampi(py + j, 0, H - 1);
            for (int i = -nn; i <= nn; ++i) {
                int r_x = __float2int_rz(o_x + i);
                r_x = (r_x > 0 ? (r_x < sc_f ? r_x : scols - 1) : 0);
                const int s_center = (int)(r_y * sc_f + r_x);
                const float4 sn = a.scaled[s_center];
                const float nb = __ldg(a.ref_img + (size_t)r_ys * W + clampi(px + i, 0, W - 1));
                const float tg = spatial_gauss(o_x, o_y, (float)r_x, (float)r_y, sigmad) *
                                 range_gauss(fabsf(ref_pix - nb), sigmar);
                nf += tg;
                n0 = n0 + sn.x * tg; n1 = n1 + sn.y * tg; n2 = n2 + sn.z * tg;
            }
        }
        float4 nt = make_float4(n0 / nf, n1 / nf, n2 / nf, 0.0f);
        normalize3(nt);
        const float4 cur = a.planes[center];
        // pre-cost plane: zero normal, upsampled depth as offset (HPM.cu:689, HPM.cpp:894-901)
        const float pre = initial_cost(a, P, px, py, make_float4(0.f, 0.f, 0.f, cur.w), &sel, s);
        a.pre_costs[center] = pre;
        float4 pl = rotate_to_cam(c0, nt);
        pl.w = distance_to_origin(c0, px, py, cur.w, pl);
        a.planes[center] = pl;
        a.costs[center] = initial_cost(a, P, px, py, pl, &sel, s);
        a.sel[center] = sel;
    } else {
        if (mand && !(a.conf[center] >= 0.3)) {
            if (texture_term(a.canny, W, H, px, py) > 0.5) a.conf[center] = 0.1f;
        }
        float4 pl = hier ? a.scaled[center] : a.planes[center];
        pl = rotate_to_cam(c0, pl);
        pl.w = distance_to_origin(c0, px, py, pl.w, pl);
        a.planes[center] = pl;
        a.costs[center] = initial_cost(a, P, px, py, pl, &sel, s);
        a.sel[center] = sel;
    }
    a.rng[center] = rng.draw;
}

template <int NS, int BLK, bool CNT>
// 3 blocks per SM (at most 168 registers): 12 warps, against 8 at the unbounded 174 registers; 1.5 ms
// instead of 1.8 ms per 1600x1200 initialisation with 32 x 4 blocks
__global__ void __launch_bounds__(BLK, 3) k_random_init(const __grid_constant__ RunArgs a) {
    extern __shared__ float smem[];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const Scratch<NS, BLK, CNT> s{ smem + tid };
    init_pixel<NS, BLK, CNT>(a, s, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y);
}

// ---------------------------------------------------------------- batched launches
//
// The batching form: the runs of several reference views (one pass of the
// schedule over the views of a pyramid level, main.cpp:1253-1255) share one
// launch per stage.  Their RunArgs sit in device memory; block b of the launch
// is tile b - tile_start[k] of run k, the last run with tile_start[k] <= b.
// A tile is the block footprint of the single-view launch, so every pixel sees
// exactly the arithmetic of the per-view kernels.  With gridDim.x smaller than
// the tile count the launch is persistent: each block walks the tiles b,
// b + gridDim.x, ...  The per-view kernels launch one view at a time and wait
// for each launch (HPM.cu:2987-3035); here the tail of one view's grid overlaps
// the next view's tiles.

__device__ __forceinline__ int batch_run_of(const int* __restrict__ tile_start, int n, int b) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(tile_start + mid) <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int NS, int BLK, bool CNT>
__global__ void __launch_bounds__(BLK) k_random_init_batch(const RunArgs* __restrict__ args,
                                                           const int* __restrict__ tile_start, int n) {
    extern __shared__ float smem[];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const Scratch<NS, BLK, CNT> s{ smem + tid };
    const int total = __ldg(tile_start + n);
    for (int b = blockIdx.x; b < total; b += gridDim.x) {
        const int k = batch_run_of(tile_start, n, b);
        const RunArgs& a = args[k];
        const int t = b - __ldg(tile_start + k);
        const int tx = (a.W + blockDim.x - 1) / blockDim.x;
        init_pixel<NS, BLK, CNT>(a, s, (t % tx) * blockDim.x + threadIdx.x, (t / tx) * blockDim.y + threadIdx.y);
    }
}

// ---------------------------------------------------------------- propagation

// Costs of one hypothesis (its PlaneM) against the source views in `mask`,
// into scratch row `row` (ComputeMultiViewCostVector, HPM.cu:490-495).  The
// only place a half-sweep evaluates the NCC, so the kernel carries one copy.
// The loop runs over view indices, the same for every lane: a variant in which
// each lane took its own k-th selected view ran three times slower on B200,
// because texture fetches with different texture objects across a warp
// serialise.
template <int NS, int BLK, bool CNT>
__device__ __forceinline__ void eval_row(const RunArgs& a, const Patch& P, int px, int py, const PlaneM& pm,
                                         uint32_t mask, int row, const Scratch<NS, BLK, CNT>& s) {
#pragma unroll 1
    for (int j = 0; j < a.S; ++j)
        if ((mask >> j) & 1u) s.ca(row, j) = ncc_view<CNT>(a, P, px, py, pm, j);
}

__device__ __forceinline__ void v_path_scan(const float* __restrict__ costs, int W, int H, int x, int y, int ax,
                                            int ay, int bx, int by, float& bc, int& best) {
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        if (i % 2 == 0) { x += ax; y += ay; } else { x += bx; y += by; }
        if (x >= 0 && x < W && y < H && y >= 0) {
            const int q = y * W + x;
            const float c = costs[q];
            if (c < bc) { bc = c; best = q; }
        } else break;
    }
}

// First candidate 5 px away along (dx, dy), then up to 4 more every 2 px while
// inside the image (HPM.cu:1385-1475).  right_far keeps the maximum (HPM.cu:1464).
__device__ __forceinline__ bool far_search(const float* __restrict__ costs, int W, int H, int px, int py, int dx,
                                           int dy, bool keep_max, int& pos) {
    const int x = px + 5 * dx, y = py + 5 * dy;
    if (x < 0 || x >= W || y < 0 || y >= H) return false;
    int best = y * W + x;
    float bc = costs[best];
#pragma unroll
    for (int i = 1; i < 5; ++i) {
        const int xi = px + (5 + 2 * i) * dx, yi = py + (5 + 2 * i) * dy;
        if (xi < 0 || xi >= W || yi < 0 || yi >= H) break;
        const int q = yi * W + xi;
        const float c = costs[q];
        if (keep_max ? (bc < c) : (c < bc)) { bc = c; best = q; }
    }
    pos = best;
    return true;
}

// Non-local candidate positions of the eight directions (HPM.cu:1367-1608);
// returns the bitmask of valid directions and leaves the positions in scratch.
template <int NS, int BLK, bool CNT>
__device__ __forceinline__ uint32_t direction_search(const RunArgs& a, int px, int py,
                                                     const Scratch<NS, BLK, CNT>& s) {
    const int W = a.W, H = a.H;
    const int center = py * W + px;
    const float* __restrict__ costs = a.costs;
    uint32_t flags = 0;
    int pos[8];
    pos[0] = center - 5 - 6 * W; pos[1] = center - 5 * W; pos[2] = center + 6 - 5 * W; pos[3] = center + 5 * W;
    pos[4] = center + 5 + 6 * W; pos[5] = center - 5; pos[6] = center - 6 + 5 * W; pos[7] = center + 5;
    if (far_search(costs, W, H, px, py, 0, -1, false, pos[1])) flags |= 1u << 1;
    if (far_search(costs, W, H, px, py, 0, 1, false, pos[3])) flags |= 1u << 3;
    if (far_search(costs, W, H, px, py, -1, 0, false, pos[5])) flags |= 1u << 5;
    if (far_search(costs, W, H, px, py, 1, 0, true, pos[7])) flags |= 1u << 7;
    if (px > 4 && py > 5) {
        flags |= 1u << 0;
        float bc = costs[pos[0]]; int best = pos[0];
        v_path_scan(costs, W, H, px - 5, py - 6, -2, 0, 0, -2, bc, best);
        pos[0] = best;
    }
    if (px < W - 6 && py > 4) {
        flags |= 1u << 2;
        float bc = costs[pos[2]]; int best = pos[2];
        v_path_scan(costs, W, H, px + 6, py - 5, 0, -2, 2, 0, bc, best);
        pos[2] = best;
    }
    if (px < W - 5 && py < H - 6) {
        flags |= 1u << 4;
        float bc = costs[pos[4]]; int best = pos[4];
        v_path_scan(costs, W, H, px + 5, py + 6, 2, 0, 0, 2, bc, best);
        pos[4] = best;
    }
    if (px > 5 && py < H - 5) {
        flags |= 1u << 6;
        float bc = costs[pos[6]]; int best = pos[6];
        v_path_scan(costs, W, H, px - 6, py + 5, 0, 2, -2, 0, bc, best);
        pos[6] = best;
    }
#pragma unroll
    for (int d = 0; d < 8; ++d) s.pos(d) = pos[d];
    return flags;
}

struct Selection {
    uint32_t temp_selected;
    int num_selected;
    float weight_norm;
};

// Joint view selection and the eight final costs (HPM.cu:1686-1771), from the
// cost rows of the directions; weights to scratch vw, final costs to fc.
template <int NS, int BLK, bool CNT>
__device__ __forceinline__ Selection view_selection(const RunArgs& a, int px, int py, int iter, uint32_t flags,
                                                    PixelRng& rng, const Scratch<NS, BLK, CNT>& s) {
    const int W = a.W, S = a.S;
    const int center = py * W + px;
    const bool geom = a.prm.mode & HPM_MODE_GEOM;
    float priors[NS];
#pragma unroll
    for (int j = 0; j < NS; ++j) priors[j] = 0.0f;
    const int nbr[4] = { center - W * 5, center + W * 5, center - 5, center + 5 };
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (flags & (1u << (2 * i + 1))) {
            const uint32_t m = a.sel[nbr[i]];
#pragma unroll
            for (int j = 0; j < NS; ++j)
                if (j < S) priors[j] += ((m >> j) & 1u) ? 0.9f : 0.1f;
        }
    }
    const float cost_thr = (float)(0.8 * hpm_expf((float)(iter * iter) / (-90.0f)));
    float probs[NS];
#pragma unroll
    for (int j = 0; j < NS; ++j) {
        probs[j] = 0.0f;
        if (j < S) {
            float count = 0.0f, tmpw = 0.0f;
            int count_false = 0;
#pragma unroll
            for (int d = 0; d < 8; ++d) {
                const float c = s.ca(d, j);
                if (c < cost_thr) { tmpw += hpm_expf(c * c / (-0.18f)); count += 1.0f; }
                if (c > 1.2f) ++count_false;
            }
            if (count > 2 && count_false < 3) probs[j] = tmpw / count;
            else if (count_false < 3) probs[j] = hpm_expf(cost_thr * cost_thr / (-0.32f));
            probs[j] = probs[j] * priors[j];
        }
    }
    {
        float sum = 0.0f;
#pragma unroll
        for (int j = 0; j < NS; ++j) if (j < S) sum += probs[j];
        const float inv = 1.0f / sum;
        float cum = 0.0f;
#pragma unroll
        for (int j = 0; j < NS; ++j) if (j < S) { cum += probs[j] * inv; probs[j] = cum; }
    }
    float vw[NS];
#pragma unroll
    for (int j = 0; j < NS; ++j) vw[j] = 0.0f;
    for (int smp = 0; smp < 15; ++smp) {
        const float rp = rng.uniform() - FLT_EPSILON;
        bool done = false;
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            if (!done && j < S && probs[j] > rp) { vw[j] += 1.0f; done = true; }
        }
    }
    Selection o;
    o.temp_selected = 0; o.num_selected = 0; o.weight_norm = 0.0f;
#pragma unroll
    for (int j = 0; j < NS; ++j) {
        s.vw(j) = vw[j];
        if (j < S && vw[j] > 0) {
            o.temp_selected |= 1u << j;
            o.weight_norm += vw[j];
            o.num_selected++;
        }
    }
#pragma unroll 1
    for (int d = 0; d < 8; ++d) {
        float fc = 0.0f;
        const bool valid = flags & (1u << d);
        float depth = 0.0f;
        if (geom && valid) depth = depth_from_plane(a.cams[0], a.planes[s.pos(d)], px, py);
        for (int j = 0; j < S; ++j) {
            const float w = s.vw(j);
            if (w > 0) {
                if (geom) {
                    if (valid)
                        fc += w * (s.ca(d, j) + 0.2f * geom_cost(a.depth_src[j + 1], a.dsw[j + 1], a.dsh[j + 1],
                                                                   a.fwd[j + 1].A, a.fwd[j + 1].b, a.bwd[j + 1].A,
                                                                   a.bwd[j + 1].b, depth, px, py));
                    else
                        fc += w * (s.ca(d, j) + 0.1f * 3.0f);
                } else {
                    fc += w * s.ca(d, j);
                }
            }
        }
        s.fc(d) = fc / o.weight_norm;
    }
    return o;
}

// Weighted cost over the selected views of the hypothesis whose NCCs are in
// scratch row 8 (HPM.cu:1775-1786, 805-817).
template <int NS, int BLK, bool CNT>
__device__ __forceinline__ float selected_cost(const RunArgs& a, int px, int py, float4 pl, uint32_t selmask,
                                               float weight_norm, const Scratch<NS, BLK, CNT>& s) {
    const bool geom = a.prm.mode & HPM_MODE_GEOM;
    const float depth = geom ? depth_from_plane(a.cams[0], pl, px, py) : 0.0f;
    float c = 0.0f;
#pragma unroll 1
    for (int j = 0; j < a.S; ++j) {
        if (!((selmask >> j) & 1u)) continue;
        const float w = s.vw(j);
        const float n = s.ca(8, j);
        if (geom) c += w * (n + 0.2f * geom_cost(a.depth_src[j + 1], a.dsw[j + 1], a.dsh[j + 1], a.fwd[j + 1].A,
                                                  a.fwd[j + 1].b, a.bwd[j + 1].A, a.bwd[j + 1].b, depth, px,
                                                  py));
        else c += w * n;
    }
    return c / weight_norm;
}

__device__ __forceinline__ int find_min_index8(const float* v) {  // ties -> last (HPM.cu:41-52)
    float m = v[0]; int idx = 0;
#pragma unroll
    for (int i = 1; i < 8; ++i) if (v[i] <= m) { m = v[i]; idx = i; }
    return idx;
}

__device__ __forceinline__ int find_max_index8(const float* v) {  // ties -> last (HPM.cu:54-65)
    float m = v[0]; int idx = 0;
#pragma unroll
    for (int i = 1; i < 8; ++i) if (v[i] >= m) { m = v[i]; idx = i; }
    return idx;
}

__device__ __forceinline__ float prior_score(float final_cost, float depth_now, float depth_prior, float4 pp,
                                             float4 pl, float texture, float two_dss, float two_ass) {
    const float gamma = 0.5f, beta = 0.18f;
    const float dd = depth_now - depth_prior;
    const float nd = fabsf(pp.x - pl.x) + fabsf(pp.y - pl.y) + fabsf(pp.z - pl.z);
    const float prior = (float)(gamma * (1.2 - 0.2 * texture) + (double)(hpm_expf(-dd * dd / two_dss) * hpm_expf(-nd * nd / two_ass)));
    return (float)(exp(-final_cost * final_cost / beta * (1 + 0.2 * texture)) * (double)prior);
}

// One pixel of a black or red half-sweep: CheckerboardPropagation (HPM.cu:1347-1873)
// or, with MAND, CheckerboardPropagation_MandatoryConsistency (HPM.cu:1875-2791).
//
// The NCC work runs in one loop of 17 slots, each costing at most one
// hypothesis through eval_row:
//   slots 0-7    the eight direction candidates, against all sources;
//   slots 8-10   the three rounds of the left-up extension (HPM.cu:1063-1126);
//   slot  11     view selection, then the current plane against the selected views;
//   slots 12-16  the five PlaneHypothesisRefinement candidates (HPM.cu:765-841),
//                built from the state at entry and accepted greedily in order.
// The decisions between slots are the reference's, in its order, and the
// random draws happen in the same sequence.
#ifndef HPM_SWEEP_MIN_BLOCKS
#define HPM_SWEEP_MIN_BLOCKS 3  // 3 blocks of 128 threads per SM: at most 170 registers
#endif

template <int NS, int BLK, bool MAND, bool CNT>
__device__ __forceinline__ void sweep_pixel(const RunArgs& a, const Scratch<NS, BLK, CNT>& s, int px, int pair,
                                            int color, int iter) {
    const int py = 2 * pair + ((px & 1) ^ color);
    const int W = a.W, H = a.H, S = a.S;
    if (px >= W || py >= H || pair >= a.cover_pairs) return;
    const int center = py * W + px;
    const hpm_camera& c0 = a.cams[0];
    const uint32_t mode = a.prm.mode;
    const bool prior = mode & HPM_MODE_PRIOR, hier = mode & HPM_MODE_HIERARCHY;
    const float dmin = a.prm.depth_min, dmax = a.prm.depth_max;

    if (!MAND && prior) {
        if (a.conf[center] > 0.3) return;
        if (a.pmask[center] == 0) return;
    }
    PixelRng rng;
    rng.init(a.seed, a.view_id, px, py, a.rng[center]);
    Patch P;
    build_patch(a, px, py, P);
    const bool reliable = MAND ? (a.conf[center] >= 0.3) : true;
    const uint32_t all_views = (S >= 32) ? 0xffffffffu : ((1u << S) - 1u);

    // `float cost_array[8][32] = { 2.0f }` (HPM.cu:1378): only [0][0] is 2, the rest 0.
    for (int d = 0; d < 8; ++d)
        for (int j = 0; j < S; ++j) s.ca(d, j) = 0.0f;
    s.ca(0, 0) = 2.0f;
    const uint32_t flags = direction_search(a, px, py, s);

    // state carried across slots
    bool extending = flags & 1u;  // left-up extension still active
    Selection sel{ 0u, 0, 0.0f };
    bool refine = false;          // slots 12-16 run
    bool use_prior = false;
    float4 cur = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 plane_now = cur;
    float depth_now = 0.0f, cost_now = 0.0f, restricted_cost = 0.0f, texture = 0.0f, depth_prior = 0.0f;
    float4 pp = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 plane0 = cur, plane_rand = cur, plane_pert = cur;
    float depth0 = 0.0f, depth_rand = 0.0f, depth_pert = 0.0f;
    const float depth_sigma = (dmax - dmin) / 64.0f;
    const float two_dss = 2 * depth_sigma * depth_sigma;
    const float angle_sigma = (float)(3.14159265358979323846 * (5.0f / 180.0f));
    const float two_ass = 2 * angle_sigma * angle_sigma;

#pragma unroll 1
    for (int t = 0; t < 17; ++t) {
        bool run = false;
        float4 pl = make_float4(0.f, 0.f, 0.f, 0.f);
        uint32_t mask = all_views;
        int row = 8;
        if (t < 8) {
            run = (flags >> t) & 1u;
            if (run) pl = a.planes[s.pos(t)];
            row = t;
        } else if (t < 11) {
            // Extended propagation: only orientation 0 (left_up) is active because
            // `bool symbol_eight_orientations[10] = { true }` (HPM.cu:1612, 1063-1126).
            const int it = t - 8;
            if (extending) {
                const float good_thr = (float)(0.8 * exp(-iter * iter * (3 - it) / 90.0));
                int good = 0, bad = 0;
                for (int j = 0; j < S; ++j) {
                    const float c = s.ca(0, j);
                    if (c < good_thr) ++good;
                    if (c > 1.2f) ++bad;
                }
                if (good >= 1 && bad <= 2) {
                    extending = false;
                } else if (px > 4 + 8 * it && py > 5 + 8 * it) {
                    const int sx = px - 5 - 8 * it, sy = py - 6 - 8 * it;
                    int best = sy * W + sx;
                    float bc = a.costs[best];
                    v_path_scan(a.costs, W, H, sx, sy, -2, 0, 0, -2, bc, best);
                    const int prev = s.pos(0);
                    if (bc > a.costs[prev]) {
                        best = prev;
                    } else if (best != prev) {
                        run = true;
                        pl = a.planes[best];
                        row = 0;
                    }
                    // best == prev recomputes the same row in the reference: identical values
                    s.pos(0) = best;
                }
            }
        } else if (t == 11) {
            sel = view_selection(a, px, py, iter, flags, rng, s);
            cur = a.planes[center];
            run = true;
            pl = cur;
            mask = sel.temp_selected;
        } else if (refine) {
            const int i = t - 12;
            // candidates (depth, normal): (rand, entry) (entry, rand) (rand, rand) (entry, perturbed) (perturbed, entry)
            pl = (i == 1 || i == 2) ? plane_rand : (i == 3 ? plane_pert : plane0);
            const float dc = (i == 0 || i == 2) ? depth_rand : (i == 4 ? depth_pert : depth0);
            pl.w = distance_to_origin(c0, px, py, dc, pl);
            run = true;
            mask = sel.temp_selected;
        }

        if (run) {
            if (CNT) atomicAdd(a.hyp_count + 1, (unsigned long long)S);
            const PlaneM pm = plane_m(a, pl);
            eval_row(a, P, px, py, pm, mask, row, s);
        }

        if (t == 11) {
            float fcl[8];
#pragma unroll
            for (int d = 0; d < 8; ++d) fcl[d] = s.fc(d);
            if (!MAND || reliable) {
                const int min_idx = find_min_index8(fcl);
                const bool min_valid = flags & (1u << min_idx);
                cost_now = selected_cost(a, px, py, cur, sel.temp_selected, sel.weight_norm, s);
                a.costs[center] = cost_now;
                const float cost_chk = cost_now;  // costs[center] as read by the NaN test
                depth_now = depth_from_plane(c0, cur, px, py);
                restricted_cost = 0.0f;
                texture = 0.0f;
                float4 prior_pick = cur;  // prior mode: the maximum-score neighbour's plane, when valid
                bool has_pick = false;
                if (!MAND && prior) {
                    pp = a.prior[center];
                    depth_prior = depth_from_plane(c0, pp, px, py);
                    texture = texture_term(a.canny, W, H, px, py);
                    if (a.pmask[center] > 0) {
                        float rfc[8];
#pragma unroll
                        for (int d = 0; d < 8; ++d) {
                            rfc[d] = 0.0f;
                            if (flags & (1u << d)) {
                                const float4 pd = a.planes[s.pos(d)];
                                const float dn = depth_from_plane(c0, pd, px, py);
                                rfc[d] = prior_score(fcl[d], dn, depth_prior, pp, pd, texture, two_dss, two_ass);
                            }
                        }
                        const int max_idx = find_max_index8(rfc);
                        const float rnow = prior_score(cost_now, depth_now, depth_prior, pp, cur, texture, two_dss,
                                                       two_ass);
                        if (flags & (1u << max_idx)) {
                            const float4 pd = a.planes[s.pos(max_idx)];
                            const float db = depth_from_plane(c0, pd, px, py);
                            prior_pick = pd;
                            has_pick = true;
                            if (db >= dmin && db <= dmax && rfc[max_idx] > rnow) {
                                // depth_now is left alone: HPM.cu:1815 shadows it in this block, so
                                // the refinement receives the pre-acceptance depth
                                cur = pd;
                                a.planes[center] = pd;
                                a.costs[center] = fcl[max_idx];
                                restricted_cost = rfc[max_idx];
                                a.sel[center] = sel.temp_selected;
                            }
                        }
                    } else if (min_valid) {
                        const float4 pd = a.planes[s.pos(min_idx)];
                        const float db = depth_from_plane(c0, pd, px, py);
                        if (db >= dmin && db <= dmax && fcl[min_idx] < cost_now) {
                            depth_now = db;
                            cur = pd;
                            a.planes[center] = pd;
                            a.costs[center] = fcl[min_idx];
                        }
                    }
                }
                // plane_hypotheses_now (HPM.cu:1844, 2299) is assigned only when the neighbour
                // is accepted; the reference as compiled holds the minimum-cost neighbour's plane
                // whenever that direction is valid; prior mode never assigns it and holds the
                // maximum-score neighbour's plane when valid.  Otherwise it starts as the
                // pixel's current plane.
                plane_now = (!MAND && prior && has_pick) ? prior_pick : cur;
                if ((MAND || !prior) && min_valid) {
                    const float4 pd = a.planes[s.pos(min_idx)];
                    const float db = depth_from_plane(c0, pd, px, py);
                    plane_now = pd;
                    if (db >= dmin && db <= dmax && fcl[min_idx] < cost_now) {
                        depth_now = db; plane_now = pd; cost_now = fcl[min_idx];
                        a.sel[center] = sel.temp_selected;
                    }
                    if (cost_chk != cost_chk) {
                        if (!MAND) depth_now = db;
                        plane_now = pd; cost_now = fcl[min_idx];
                        a.sel[center] = sel.temp_selected;
                    }
                }
                // PlaneHypothesisRefinement's random draws (HPM.cu:765-799), before any candidate is costed
                refine = true;
                use_prior = prior && a.pmask[center] > 0;
                const float perturbation = 0.02f;
                if (use_prior) {
                    depth_rand = rng.uniform() * 6 * depth_sigma + (depth_prior - 3 * depth_sigma);
                    plane_rand = perturbed_normal(c0, px, py, pp, rng, angle_sigma);
                } else {
                    depth_rand = rng.uniform() * (dmax - dmin) + dmin;
                    plane_rand = random_normal(c0, px, py, rng, depth_now);
                }
                const float dmin_p = (1 - perturbation) * depth_now;
                const float dmax_p = (1 + perturbation) * depth_now;
                depth_pert = rng.uniform() * (dmax_p - dmin_p) + dmin_p;
                plane_pert = perturbed_normal(c0, px, py, plane_now, rng,
                                              (float)(perturbation * 3.14159265358979323846));
                plane0 = plane_now;
                depth0 = depth_now;
            } else {
                // mandatory consistency, unreliable pixel (HPM.cu:2684-2789)
                const float beta = 0.18f;
                float rfc[8];
                const float mmc = sel.num_selected * 0.5f;
#pragma unroll
                for (int d = 0; d < 8; ++d) {
                    rfc[d] = 0.0f;
                    if (flags & (1u << d)) {
                        const float cp = a.conf[s.pos(d)];
                        const float gce = hpm_expf(-fcl[d] * fcl[d] / beta);
                        const float dm = fmaxf(0.0f, mmc - cp);
                        const float mce = (float)(0.5f + exp(-dm * dm / (mmc * mmc * 1.0)));
                        rfc[d] = (cp > 0) ? fmaxf(3.0f, mce) * gce : mce * gce;
                        if (cp > 0) fcl[d] = (float)(fcl[d] * fmin((double)hpm_expf(-cp * 2), 0.35));
                    }
                }
                const int max_idx = find_max_index8(rfc);
                float cost_u = selected_cost(a, px, py, cur, sel.temp_selected, sel.weight_norm, s);
                const float cost_chk = cost_u;
                const float cc = a.conf[center];
                const float gce = hpm_expf(-cost_u * cost_u / beta);
                const float dm = fmaxf(0.0f, mmc - cc);
                const float mce = (float)(0.5f + exp(-dm * dm / (mmc * mmc * 1.0)));
                const float rnow = (cc > 0) ? fmaxf(3.0f, mce) * gce : mce * gce;
                if (cc < 0.3) cost_u = (float)(cost_u * exp(0.2 + cc * 2));
                else cost_u = cost_u * hpm_expf(-cc * 2);
                float4 pu = cur;  // HPM.cu:2761: the neighbour's plane whenever that direction is valid
                if (flags & (1u << max_idx)) {
                    const int pm = s.pos(max_idx);
                    const float4 pd = a.planes[pm];
                    pu = pd;
                    const float db = depth_from_plane(c0, pd, px, py);
                    if (db >= dmin && db <= dmax && rfc[max_idx] > rnow) {
                        pu = pd; cost_u = fcl[max_idx];
                        a.sel[center] = sel.temp_selected;
                        a.conf[center] = (float)(0.5 * a.conf[pm]);
                    }
                    if (cost_chk != cost_chk) {
                        pu = pd; cost_u = fcl[max_idx];
                        a.sel[center] = sel.temp_selected;
                        a.conf[center] = (float)(0.5 * a.conf[pm]);
                    }
                }
                a.costs[center] = cost_u;
                a.planes[center] = pu;
            }
        } else if (t >= 12 && refine) {
            const int i = t - 12;
            const float dc = (i == 0 || i == 2) ? depth_rand : (i == 4 ? depth_pert : depth0);
            const float tc = selected_cost(a, px, py, pl, sel.temp_selected, sel.weight_norm, s);
            const float db = depth_from_plane(c0, pl, px, py);
            if (use_prior) {
                const float rt = prior_score(tc, dc, depth_prior, pp, pl, texture, two_dss, two_ass);
                if (db >= dmin && db <= dmax && rt > restricted_cost) {
                    depth_now = db; plane_now = pl; cost_now = tc; restricted_cost = rt;
                }
            } else if (db >= dmin && db <= dmax && tc < cost_now) {
                depth_now = db; plane_now = pl; cost_now = tc;
            }
        }
    }

    if (refine) {
        if (!MAND && hier) {
            if (cost_now < a.pre_costs[center] - 0.1f) {
                a.costs[center] = cost_now;
                a.planes[center] = plane_now;
            }
        } else {
            a.costs[center] = cost_now;
            a.planes[center] = plane_now;
        }
    }
    a.rng[center] = rng.draw;
}

template <int NS, int BLK, bool MAND, bool CNT>
__global__ void __launch_bounds__(BLK, HPM_SWEEP_MIN_BLOCKS) k_half_sweep(const __grid_constant__ RunArgs a, int color, int iter) {
    extern __shared__ float smem[];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const Scratch<NS, BLK, CNT> s{ smem + tid };
    sweep_pixel<NS, BLK, MAND, CNT>(a, s, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y,
                                    color, iter);
}

// Prior mode with work lists (RunArgs::active_px): thread x of a row pair takes the x-th pixel the
// sweep updates, so the pixels that return at once (confident, or outside the prior mask) leave
// whole warps idle instead of holding lanes of working ones.  Pixels of one colour read only the
// other colour's state, so the mapping does not change any result.
template <int NS, int BLK, bool CNT>
__global__ void __launch_bounds__(BLK, HPM_SWEEP_MIN_BLOCKS) k_half_sweep_listed(const __grid_constant__ RunArgs a,
                                                                                 int color, int iter) {
    extern __shared__ float smem[];
    const int pair = blockIdx.y * blockDim.y + threadIdx.y;
    if (pair >= a.cover_pairs) return;
    const int k = color * a.cover_pairs + pair;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= a.active_n[k]) return;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const Scratch<NS, BLK, CNT> s{ smem + tid };
    sweep_pixel<NS, BLK, false, CNT>(a, s, a.active_px[(size_t)k * a.W + x], pair, color, iter);
}

// The pixels a prior-mode half-sweep updates (CheckerboardPropagation returns at once where
// confidence > 0.3 or the prior mask is clear, HPM.cu:1352-1365): one warp per (row pair, colour)
// writes their columns in increasing order and their count.
__global__ void k_prior_active(const __grid_constant__ RunArgs a, int* __restrict__ out_px, int* __restrict__ out_n) {
    const int pair = blockIdx.x, color = blockIdx.y, lane = threadIdx.x;
    const int W = a.W, H = a.H;
    int* row = out_px + ((size_t)color * a.cover_pairs + pair) * W;
    int n = 0;
    for (int x0 = 0; x0 < W; x0 += 32) {
        const int px = x0 + lane;
        const int py = 2 * pair + ((px & 1) ^ color);
        bool act = false;
        if (px < W && py < H) {
            const int c = py * W + px;
            act = !(a.conf[c] > 0.3) && a.pmask[c] != 0;
        }
        const unsigned m = __ballot_sync(0xffffffffu, act);
        if (act) row[n + __popc(m & ((1u << lane) - 1u))] = px;
        n += __popc(m);
    }
    if (lane == 0) out_n[color * a.cover_pairs + pair] = n;
}

cudaError_t launch_prior_active(const RunArgs& a, int* px, int* n, cudaStream_t st) {
    if (a.cover_pairs <= 0) return cudaSuccess;
    k_prior_active<<<dim3(a.cover_pairs, 2), 32, 0, st>>>(a, px, n);
    return cudaGetLastError();
}

// The batched form of k_half_sweep_listed: tile t of run k maps to columns of that run's work lists.
template <int NS, int BLK, bool CNT>
__global__ void __launch_bounds__(BLK, HPM_SWEEP_MIN_BLOCKS)
    k_half_sweep_batch_listed(const RunArgs* __restrict__ args, const int* __restrict__ tile_start, int n,
                              int color, int iter) {
    extern __shared__ float smem[];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const Scratch<NS, BLK, CNT> s{ smem + tid };
    const int total = __ldg(tile_start + n);
    for (int b = blockIdx.x; b < total; b += gridDim.x) {
        const int k = batch_run_of(tile_start, n, b);
        const RunArgs& a = args[k];
        const int t = b - __ldg(tile_start + k);
        const int tx = (a.W + blockDim.x - 1) / blockDim.x;
        const int x = (t % tx) * blockDim.x + threadIdx.x;
        const int pair = (t / tx) * blockDim.y + threadIdx.y;
        if (pair >= a.cover_pairs) continue;
        const int r = color * a.cover_pairs + pair;
        if (x >= a.active_n[r]) continue;
        sweep_pixel<NS, BLK, false, CNT>(a, s, a.active_px[(size_t)r * a.W + x], pair, color, iter);
    }
}

template <int NS, int BLK, bool MAND, bool CNT>
__global__ void __launch_bounds__(BLK, HPM_SWEEP_MIN_BLOCKS)
    k_half_sweep_batch(const RunArgs* __restrict__ args, const int* __restrict__ tile_start, int n, int color,
                       int iter) {
    extern __shared__ float smem[];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const Scratch<NS, BLK, CNT> s{ smem + tid };
    const int total = __ldg(tile_start + n);
    for (int b = blockIdx.x; b < total; b += gridDim.x) {
        const int k = batch_run_of(tile_start, n, b);
        const RunArgs& a = args[k];
        const int t = b - __ldg(tile_start + k);
        const int tx = (a.W + blockDim.x - 1) / blockDim.x;
        sweep_pixel<NS, BLK, MAND, CNT>(a, s, (t % tx) * blockDim.x + threadIdx.x,
                                        (t / tx) * blockDim.y + threadIdx.y, color, iter);
    }
}

__global__ void k_export(const __grid_constant__ RunArgs a) {
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    const int py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= a.W || py >= a.H) return;
    const int center = py * a.W + px;
    float4 pl = a.planes[center];
    pl.w = depth_from_plane(a.cams[0], pl, px, py);
    a.planes[center] = rotate_to_world(a.cams[0], pl);
}

__global__ void k_eval_costs(const __grid_constant__ RunArgs a, int n, const int32_t* __restrict__ px,
                             const float4* __restrict__ planes, float* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int x = px[2 * k], y = px[2 * k + 1];
    Patch P;
    build_patch(a, x, y, P);
    const float4 pl = planes[k];
    const PlaneM pm = plane_m(a, pl);
    for (int j = 0; j < a.S; ++j) out[(size_t)k * a.S + j] = ncc_view(a, P, x, y, pm, j);
}

// ---------------------------------------------------------------- launchers

template <int NS>
static constexpr int block_threads() { return NS <= 10 ? 128 : (NS <= 16 ? 64 : 32); }

template <int NS, bool CNT>
static cudaError_t init_impl(const RunArgs& a, cudaStream_t st) {
    constexpr int BLK = 128;
    const size_t shm = sizeof(float) * Scratch<NS, BLK>::kWords * BLK;
    auto k = k_random_init<NS, BLK, CNT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    if (e != cudaSuccess) return e;
    dim3 block(32, 4), grid((a.W + 31) / 32, (a.H + 3) / 4);
    k<<<grid, block, shm, st>>>(a);
    return cudaGetLastError();
}

template <int NS, bool MAND, bool CNT>
static cudaError_t sweep_impl(const RunArgs& a, int color, int iter, cudaStream_t st) {
    constexpr int BLK = block_threads<NS>();
    const size_t shm = sizeof(float) * Scratch<NS, BLK>::kWords * BLK;
    auto k = k_half_sweep<NS, BLK, MAND, CNT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    if (e != cudaSuccess) return e;
#ifndef HPM_SWEEP_BX
#define HPM_SWEEP_BX 32
#endif
    constexpr int BX = HPM_SWEEP_BX < BLK ? HPM_SWEEP_BX : BLK;
    dim3 block(BX, BLK / BX), grid((a.W + BX - 1) / BX, (a.cover_pairs + BLK / BX - 1) / (BLK / BX));
    if (!MAND && a.active_px) {
        auto kl = k_half_sweep_listed<NS, BLK, CNT>;
        if ((e = cudaFuncSetAttribute(kl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm)) != cudaSuccess)
            return e;
        kl<<<grid, block, shm, st>>>(a, color, iter);
        return cudaGetLastError();
    }
    k<<<grid, block, shm, st>>>(a, color, iter);
    return cudaGetLastError();
}

template <int NS, bool CNT>
static cudaError_t init_batch_impl(const BatchLaunch& bl, cudaStream_t st) {
    constexpr int BLK = 128;
    const size_t shm = sizeof(float) * Scratch<NS, BLK>::kWords * BLK;
    auto k = k_random_init_batch<NS, BLK, CNT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    if (e != cudaSuccess) return e;
    const int grid = bl.grid_blocks > 0 && bl.grid_blocks < bl.tiles ? bl.grid_blocks : bl.tiles;
    k<<<grid, dim3(16, 8), shm, st>>>(bl.args, bl.tile_start, bl.n);
    return cudaGetLastError();
}

template <int NS, bool MAND, bool CNT>
static cudaError_t sweep_batch_impl(const BatchLaunch& bl, int color, int iter, cudaStream_t st) {
    constexpr int BLK = block_threads<NS>();
    const size_t shm = sizeof(float) * Scratch<NS, BLK>::kWords * BLK;
    auto k = (!MAND && bl.listed) ? k_half_sweep_batch_listed<NS, BLK, CNT> : k_half_sweep_batch<NS, BLK, MAND, CNT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    if (e != cudaSuccess) return e;
    const int grid = bl.grid_blocks > 0 && bl.grid_blocks < bl.tiles ? bl.grid_blocks : bl.tiles;
    const int bx = (bl.bx > 0 && bl.bx <= BLK) ? bl.bx : 32;
    k<<<grid, dim3(bx, BLK / bx), shm, st>>>(bl.args, bl.tile_start, bl.n, color, iter);
    return cudaGetLastError();
}

template <int NS, bool MAND, bool CNT>
static int sweep_batch_occupancy() {
    constexpr int BLK = block_threads<NS>();
    const size_t shm = sizeof(float) * Scratch<NS, BLK>::kWords * BLK;
    auto k = k_half_sweep_batch<NS, BLK, MAND, CNT>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm) != cudaSuccess) return 0;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, BLK, shm) != cudaSuccess) return 0;
    return blocks;
}

template <bool CNT>
static cudaError_t init_dispatch(const RunArgs& a, cudaStream_t st) {
    if (a.S <= 4) return init_impl<4, CNT>(a, st);
    if (a.S <= 10) return init_impl<10, CNT>(a, st);
    if (a.S <= 16) return init_impl<16, CNT>(a, st);
    return init_impl<31, CNT>(a, st);
}

cudaError_t launch_random_init(const RunArgs& a, cudaStream_t st) {
    return a.hyp_count ? init_dispatch<true>(a, st) : init_dispatch<false>(a, st);
}

template <bool MAND, bool CNT>
static cudaError_t sweep_dispatch(const RunArgs& a, int color, int iter, cudaStream_t st) {
    if (a.S <= 4) return sweep_impl<4, MAND, CNT>(a, color, iter, st);
    if (a.S <= 10) return sweep_impl<10, MAND, CNT>(a, color, iter, st);
    if (a.S <= 16) return sweep_impl<16, MAND, CNT>(a, color, iter, st);
    return sweep_impl<31, MAND, CNT>(a, color, iter, st);
}

cudaError_t launch_half_sweep(const RunArgs& a, int color, int iter, cudaStream_t st) {
    const bool mand = a.prm.mode & HPM_MODE_MAND;
    if (a.hyp_count)
        return mand ? sweep_dispatch<true, true>(a, color, iter, st) : sweep_dispatch<false, true>(a, color, iter, st);
    return mand ? sweep_dispatch<true, false>(a, color, iter, st) : sweep_dispatch<false, false>(a, color, iter, st);
}

template <bool CNT>
static cudaError_t init_batch_dispatch(const BatchLaunch& bl, cudaStream_t st) {
    if (bl.max_s <= 4) return init_batch_impl<4, CNT>(bl, st);
    if (bl.max_s <= 10) return init_batch_impl<10, CNT>(bl, st);
    if (bl.max_s <= 16) return init_batch_impl<16, CNT>(bl, st);
    return init_batch_impl<31, CNT>(bl, st);
}

cudaError_t launch_random_init_batch(const BatchLaunch& bl, cudaStream_t st) {
    return bl.count ? init_batch_dispatch<true>(bl, st) : init_batch_dispatch<false>(bl, st);
}

template <bool MAND, bool CNT>
static cudaError_t sweep_batch_dispatch(const BatchLaunch& bl, int color, int iter, cudaStream_t st) {
    if (bl.max_s <= 4) return sweep_batch_impl<4, MAND, CNT>(bl, color, iter, st);
    if (bl.max_s <= 10) return sweep_batch_impl<10, MAND, CNT>(bl, color, iter, st);
    if (bl.max_s <= 16) return sweep_batch_impl<16, MAND, CNT>(bl, color, iter, st);
    return sweep_batch_impl<31, MAND, CNT>(bl, color, iter, st);
}

cudaError_t launch_half_sweep_batch(const BatchLaunch& bl, int color, int iter, cudaStream_t st) {
    if (bl.count)
        return bl.mand ? sweep_batch_dispatch<true, true>(bl, color, iter, st)
                       : sweep_batch_dispatch<false, true>(bl, color, iter, st);
    return bl.mand ? sweep_batch_dispatch<true, false>(bl, color, iter, st)
                   : sweep_batch_dispatch<false, false>(bl, color, iter, st);
}

int half_sweep_batch_occupancy(int max_s, bool mand) {
    if (max_s <= 4) return mand ? sweep_batch_occupancy<4, true, false>() : sweep_batch_occupancy<4, false, false>();
    if (max_s <= 10) return mand ? sweep_batch_occupancy<10, true, false>() : sweep_batch_occupancy<10, false, false>();
    if (max_s <= 16) return mand ? sweep_batch_occupancy<16, true, false>() : sweep_batch_occupancy<16, false, false>();
    return mand ? sweep_batch_occupancy<31, true, false>() : sweep_batch_occupancy<31, false, false>();
}

int half_sweep_block_threads(int max_s) { return max_s <= 10 ? 128 : (max_s <= 16 ? 64 : 32); }

cudaError_t launch_export(const RunArgs& a, cudaStream_t st) {
    dim3 block(32, 8), grid((a.W + 31) / 32, (a.H + 7) / 8);
    k_export<<<grid, block, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_eval_costs(const RunArgs& a, int n, const int32_t* px, const float4* planes, float* out,
                              cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_eval_costs<<<(n + 127) / 128, 128, 0, st>>>(a, n, px, planes, out);
    return cudaGetLastError();
}

}  // namespace hpm
