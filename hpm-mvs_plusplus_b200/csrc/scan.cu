// ConfidenceEvaluation (main.cpp:959-1109) and RunFusion / RunFusion_Sky_Strict
// (main.cpp:659-957) on the GPU with the reference's sequential semantics.
//
// The reference scans views in order and each view's pixels in raster order.
// A pixel is accepted when enough source views agree; accepting it marks the
// source pixels in `used_list` as used, and `used_list` keeps the last passing
// position of every source across pixels (it is declared per view, not per
// pixel), so stale positions are re-marked.  Later pixels skip marked source
// pixels.  The result depends on that order.
//
// Parallel form used here, per view i (views stay sequential):
//   1. candidates (parallel over pixels q and sources j): the source pixel
//      P[q][j] and whether the geometric test passes, T[q][j], ignoring masks;
//   2. a causal fixed point: eff[q][j] = T[q][j] and P[q][j] not marked before q.
//      Each Jacobi iteration computes acceptance from eff, the last counted
//      pixel of every source up to q (a max-scan over q), the first pixel that
//      marks each source pixel (atomicMin), and eff again.  eff[q] depends only
//      on pixels before q, so the system has one solution and an iteration that
//      changes nothing has reached it; iterations are capped and a sequential
//      pass takes over beyond the cap;
//   3. marks become permanent, confidences take the value of the last pixel
//      that marked them (atomicMax), points are compacted in raster order.
// Arithmetic mirrors the host code of the reference (g++ without -ffast-math):
// float geometry, double where pow(float, int) promotes; exp(float) is the
// float function there (the double exp rounded to float here).  No implicit
// contraction.
#include "aux_kernels.cuh"
#include "ctx.hpp"

#include <algorithm>
#include <climits>
#include <vector>

namespace hpm {

constexpr int kScanBlock = 1024;
constexpr int kMaxScanIterations = 256;
// fixed-point rounds launched between host reads of their change flags: at 4 the extra rounds after
// the fixed point cost more device time than the host round trips they save (confidence scans
// 19.9 -> 21.5 ms per view on the 49-view 1600x1200 workload), so one
constexpr int kRoundsPerCheck = 1;
// "not marked" value of marktime: the byte pattern 0x7f written by cudaMemset
constexpr int32_t kUnmarked = 0x7F7F7F7F;

__device__ __forceinline__ float3 sc_world_point(int x, int y, float depth, const hpm_camera& c) {
    const float X0 = depth * (x - c.K[2]) / c.K[0];
    const float X1 = depth * (y - c.K[5]) / c.K[4];
    const float X2 = depth;
    const float T0 = c.R[0] * X0 + c.R[3] * X1 + c.R[6] * X2;
    const float T1 = c.R[1] * X0 + c.R[4] * X1 + c.R[7] * X2;
    const float T2 = c.R[2] * X0 + c.R[5] * X1 + c.R[8] * X2;
    const float C0 = -(c.R[0] * c.t[0] + c.R[3] * c.t[1] + c.R[6] * c.t[2]);
    const float C1 = -(c.R[1] * c.t[0] + c.R[4] * c.t[1] + c.R[7] * c.t[2]);
    const float C2 = -(c.R[2] * c.t[0] + c.R[5] * c.t[1] + c.R[8] * c.t[2]);
    return make_float3(T0 + C0, T1 + C1, T2 + C2);
}

__device__ __forceinline__ float2 sc_project(float3 X, const hpm_camera& c, float& depth) {
    const float T0 = c.R[0] * X.x + c.R[1] * X.y + c.R[2] * X.z + c.t[0];
    const float T1 = c.R[3] * X.x + c.R[4] * X.y + c.R[5] * X.z + c.t[1];
    const float T2 = c.R[6] * X.x + c.R[7] * X.y + c.R[8] * X.z + c.t[2];
    depth = c.K[6] * T0 + c.K[7] * T1 + c.K[8] * T2;
    return make_float2((c.K[0] * T0 + c.K[1] * T1 + c.K[2] * T2) / depth,
                       (c.K[3] * T0 + c.K[4] * T1 + c.K[5] * T2) / depth);
}

// int(v) of the x86 host: truncation, NaN and out-of-range give INT_MIN.
__device__ __forceinline__ int host_trunc(float v) {
    if (!(v > -2147483648.0f && v < 2147483648.0f)) return INT_MIN;
    return __float2int_rz(v);
}

__device__ __forceinline__ float host_angle(const float* a, const float* b) {  // HPM.cpp:281-290
    const float dot = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    const float ang = (float)acos((double)dot);
    return ang != ang ? 0.0f : ang;
}

template <int MODE>
__global__ void k_candidates(const ScanView* __restrict__ views, int i, const int32_t* __restrict__ srcs, int n_ngb,
                             int32_t* __restrict__ pos, double* __restrict__ wexp, uint32_t* __restrict__ test,
                             int npix) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npix) return;
    const ScanView& vi = views[i];
    const int W = vi.W;
    const int r = q / W, c = q - r * W;
    uint32_t T = 0;
    const float ref_depth = vi.depth[q];
    bool valid = vi.mask[q] != 1 && ref_depth > 0.0f;
    if (MODE == 0 && valid && (ref_depth < vi.cam.depth_min || ref_depth > vi.cam.depth_max)) valid = false;
    float3 X = make_float3(0.f, 0.f, 0.f);
    if (valid) X = sc_world_point(c, r, ref_depth, vi.cam);
    const float* rn = vi.normal + 3 * (size_t)q;
    for (int j = 0; j < n_ngb; ++j) {
        int p = -1;
        if (valid) {
            const ScanView& vs = views[srcs[j]];
            float pd;
            const float2 pt = sc_project(X, vs.cam, pd);
            const int sr = host_trunc(pt.y + 0.5f);
            const int scc = host_trunc(pt.x + 0.5f);
            if (scc >= 0 && scc < vs.W && sr >= 0 && sr < vs.H) {
                p = sr * vs.W + scc;
                const float sd = vs.depth[p];
                bool ok = sd > 0.0f;
                if (MODE == 0 && ok && (sd < vi.cam.depth_min || sd > vi.cam.depth_max)) ok = false;
                if (ok) {
                    const float3 tX = sc_world_point(scc, sr, sd, vs.cam);
                    float proj;
                    const float2 tp = sc_project(tX, vi.cam, proj);
                    const double dx = (double)(c - tp.x), dy = (double)(r - tp.y);
                    const float reproj = (float)sqrt(dx * dx + dy * dy);
                    const float rel = (float)(fabs((double)(proj - ref_depth)) / (double)ref_depth);
                    const float ang = host_angle(rn, vs.normal + 3 * (size_t)p);
                    if (reproj < 2.0f && rel < 0.01f && ang < 0.174533f) {
                        const float idx = reproj + 200 * rel + ang * 10;
                        T |= 1u << j;
                        // exp(float) of the reference's host code: the float function
                        wexp[(size_t)q * n_ngb + j] = (double)(float)exp((double)(-idx));
                    }
                }
            }
        }
        pos[(size_t)q * n_ngb + j] = p;
    }
    test[q] = T;
}

// eff = T minus pairs whose source pixel is masked or marked before q.
__global__ void k_update_eff(const ScanView* __restrict__ views, const int32_t* __restrict__ srcs, int n_ngb,
                             const int32_t* __restrict__ pos, const uint32_t* __restrict__ test,
                             uint32_t* __restrict__ eff, int* __restrict__ changed, int npix, int use_marks) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npix) return;
    const uint32_t T = test[q];
    uint32_t e = T;
    for (int j = 0; j < n_ngb; ++j) {
        if (!((T >> j) & 1u)) continue;
        const ScanView& vs = views[srcs[j]];
        const int p = pos[(size_t)q * n_ngb + j];
        bool blocked = vs.mask[p] == 1;
        if (use_marks && vs.marktime[p] < q) blocked = true;
        if (blocked) e &= ~(1u << j);
    }
    if (e != eff[q]) {
        eff[q] = e;
        if (changed) *changed = 1;
    }
}

__global__ void k_accept(const uint32_t* __restrict__ eff, const double* __restrict__ wexp, int n_ngb,
                         float* __restrict__ dyn, uint8_t* __restrict__ acc, int npix) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npix) return;
    const uint32_t e = eff[q];
    float d = 0.0f;
    int n = 0;
    for (int j = 0; j < n_ngb; ++j)
        if ((e >> j) & 1u) {
            d = (float)((double)d + wexp[(size_t)q * n_ngb + j]);
            ++n;
        }
    dyn[q] = d;
    acc[q] = (n >= 1 && (double)d > 0.3 * n) ? 1 : 0;
}

// last[q][j] = max{q' <= q : eff[q'] has bit j}, per block of kScanBlock pixels.
__global__ void k_last_local(const uint32_t* __restrict__ eff, int n_ngb, int32_t* __restrict__ last,
                             int32_t* __restrict__ block_max, int npix) {
    __shared__ int32_t s[kScanBlock];
    const int j = blockIdx.y;
    const int q = blockIdx.x * kScanBlock + threadIdx.x;
    int v = -1;
    if (q < npix && ((eff[q] >> j) & 1u)) v = q;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < kScanBlock; off <<= 1) {
        const int t = (int)threadIdx.x >= off ? s[threadIdx.x - off] : -1;
        __syncthreads();
        s[threadIdx.x] = max(s[threadIdx.x], t);
        __syncthreads();
    }
    if (q < npix) last[(size_t)q * n_ngb + j] = s[threadIdx.x];
    if (threadIdx.x == kScanBlock - 1) block_max[(size_t)j * gridDim.x + blockIdx.x] = s[threadIdx.x];
}

__global__ void k_last_blocks(int32_t* __restrict__ block_max, int nblocks, int n_ngb) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_ngb) return;
    int run = -1;
    for (int b = 0; b < nblocks; ++b) {  // exclusive prefix max over blocks
        const int v = block_max[(size_t)j * nblocks + b];
        block_max[(size_t)j * nblocks + b] = run;
        run = max(run, v);
    }
}

__global__ void k_last_combine(int32_t* __restrict__ last, const int32_t* __restrict__ block_max, int n_ngb,
                               int npix, int nblocks) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npix) return;
    const int b = q / kScanBlock;
    for (int j = 0; j < n_ngb; ++j) {
        const int pre = block_max[(size_t)j * nblocks + b];
        int32_t& v = last[(size_t)q * n_ngb + j];
        v = max(v, pre);
    }
}

// The marks of every source of the current view back to "not marked" (marktime) and -1
// (marklast, confidence mode): one launch for all sources of a round, row j of the grid for
// source j.
__global__ void k_reset_marks(const ScanView* __restrict__ views, const int32_t* __restrict__ srcs, int with_last) {
    const ScanView& vs = views[srcs[blockIdx.y]];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= vs.W * vs.H) return;
    vs.marktime[p] = kUnmarked;
    if (with_last) vs.marklast[p] = -1;
}

template <int MODE>
__global__ void k_marks(const ScanView* __restrict__ views, const int32_t* __restrict__ srcs, int n_ngb,
                        const int32_t* __restrict__ pos, const int32_t* __restrict__ last,
                        const uint8_t* __restrict__ acc, int npix) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npix || !acc[q]) return;
    for (int j = 0; j < n_ngb; ++j) {
        const int L = last[(size_t)q * n_ngb + j];
        if (L < 0) continue;
        const ScanView& vs = views[srcs[j]];
        const int p = pos[(size_t)L * n_ngb + j];
        atomicMin(&vs.marktime[p], q);
        if (MODE == 0) atomicMax(&vs.marklast[p], q);
    }
}

// Exact sequential pass (the reference loop) over the precomputed candidates;
// used when the fixed point has not settled within kMaxScanIterations.
template <int MODE>
__global__ void k_sequential(const ScanView* __restrict__ views, const int32_t* __restrict__ srcs, int n_ngb,
                             const int32_t* __restrict__ pos, const double* __restrict__ wexp,
                             const uint32_t* __restrict__ test, float* __restrict__ dyn, uint8_t* __restrict__ acc,
                             int npix) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int used[32];
    for (int j = 0; j < n_ngb; ++j) used[j] = -1;
    for (int q = 0; q < npix; ++q) {
        const uint32_t T = test[q];
        float d = 0.0f;
        int n = 0;
        for (int j = 0; j < n_ngb; ++j) {
            if (!((T >> j) & 1u)) continue;
            const ScanView& vs = views[srcs[j]];
            const int p = pos[(size_t)q * n_ngb + j];
            if (vs.mask[p] == 1 || vs.marktime[p] != kUnmarked) continue;
            used[j] = p;
            d = (float)((double)d + wexp[(size_t)q * n_ngb + j]);
            ++n;
        }
        const bool a = n >= 1 && (double)d > 0.3 * n;
        dyn[q] = d;
        acc[q] = a ? 1 : 0;
        if (a)
            for (int j = 0; j < n_ngb; ++j)
                if (used[j] >= 0) {
                    const ScanView& vs = views[srcs[j]];
                    if (vs.marktime[used[j]] == kUnmarked) vs.marktime[used[j]] = q;
                    if (MODE == 0) vs.marklast[used[j]] = q;
                }
    }
}

template <int MODE>
__global__ void k_apply_marks(ScanView* __restrict__ views, int sid, const float* __restrict__ dyn) {
    ScanView& vs = views[sid];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= vs.W * vs.H) return;
    if (vs.marktime[p] != kUnmarked) {
        vs.mask[p] = 1;
        if (MODE == 0) vs.cons[p] = dyn[vs.marklast[p]];
    }
}

__global__ void k_conf_own(ScanView* __restrict__ views, int i, const float* __restrict__ dyn,
                           const uint8_t* __restrict__ acc, float* __restrict__ out, int npix) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npix) return;
    float* cons = views[i].cons;
    if (acc[q]) cons[q] = dyn[q];
    out[q] = cons[q];  // confidence.dmb of view i is written after its own scan (main.cpp:1091-1095)
}

// Fusion output: keep flag (sky test of RunFusion_Sky_Strict, main.cpp:805) and points.
__global__ void k_fuse_flags(const ScanView* __restrict__ views, int i, const uint8_t* __restrict__ acc,
                             int32_t* __restrict__ keep, int npix) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npix) return;
    const ScanView& v = views[i];
    int k = acc[q];
    if (k && v.sky) {
        const uint8_t* s = v.sky + 3 * (size_t)q;
        k = ((int)s[0] != 234 && (int)s[1] != 235 && (int)s[2] != 55) ? 1 : 0;
    }
    keep[q] = k;
}

__global__ void k_fuse_emit(const ScanView* __restrict__ views, int i, const int32_t* __restrict__ keep,
                            const int32_t* __restrict__ offset, hpm_point* __restrict__ out, int64_t base,
                            int64_t capacity, int npix) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npix || !keep[q]) return;
    const int64_t k = base + offset[q];
    if (k >= capacity) return;
    const ScanView& v = views[i];
    const int r = q / v.W, c = q - r * v.W;
    const float3 X = sc_world_point(c, r, v.depth[q], v.cam);
    hpm_point p;
    p.coord[0] = X.x; p.coord[1] = X.y; p.coord[2] = X.z;
    p.normal[0] = v.normal[3 * (size_t)q]; p.normal[1] = v.normal[3 * (size_t)q + 1];
    p.normal[2] = v.normal[3 * (size_t)q + 2];
    p.color[0] = (float)v.color[3 * (size_t)q]; p.color[1] = (float)v.color[3 * (size_t)q + 1];
    p.color[2] = (float)v.color[3 * (size_t)q + 2];
    out[k] = p;
}

// Compaction offsets of the fused points: an exclusive prefix sum of the keep
// flags in three launches over tiles of kScanBlock pixels -- tile totals, an
// exclusive scan of the totals (one block), and each tile's scan plus its
// offset.  Warp scans by shuffle, then a scan of the 32 warp totals.
__device__ __forceinline__ int32_t warp_inclusive_sum(int32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Inclusive sum over a block of kScanBlock threads; ws[31] holds the block
// total when it returns.  The caller syncs before ws is written again.
__device__ __forceinline__ int32_t block_inclusive_sum(int32_t v, int32_t* ws) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warp_inclusive_sum(v);
    if (lane == 31) ws[w] = v;
    __syncthreads();
    if (w == 0) ws[lane] = warp_inclusive_sum(ws[lane]);
    __syncthreads();
    return v + (w > 0 ? ws[w - 1] : 0);
}

__global__ void __launch_bounds__(kScanBlock) k_tile_sums(const int32_t* __restrict__ in, int n,
                                                          int32_t* __restrict__ tile_sum) {
    __shared__ int32_t ws[32];
    const int q = blockIdx.x * kScanBlock + threadIdx.x;
    block_inclusive_sum(q < n ? in[q] : 0, ws);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = ws[31];
}

// exclusive scan of the tile totals in place (one block, chunks with a carry); total = sum of all
__global__ void __launch_bounds__(kScanBlock) k_scan_tile_sums(int32_t* __restrict__ tile_sum, int ntiles,
                                                               int32_t* __restrict__ total) {
    __shared__ int32_t ws[32];
    int32_t carry = 0;
    for (int base = 0; base < ntiles; base += kScanBlock) {
        const int q = base + threadIdx.x;
        const int32_t v = q < ntiles ? tile_sum[q] : 0;
        const int32_t inc = block_inclusive_sum(v, ws);
        if (q < ntiles) tile_sum[q] = carry + inc - v;
        carry += ws[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_tiles(const int32_t* __restrict__ in, int n,
                                                           const int32_t* __restrict__ tile_off,
                                                           int32_t* __restrict__ out) {
    __shared__ int32_t ws[32];
    const int q = blockIdx.x * kScanBlock + threadIdx.x;
    const int32_t v = q < n ? in[q] : 0;
    const int32_t inc = block_inclusive_sum(v, ws);
    if (q < n) out[q] = tile_off[blockIdx.x] + inc - v;
}

// ---------------------------------------------------------------- host driver

template <class T>
static cudaError_t ensure_dev(T*& p, size_t& cap, size_t n) {
    if (n <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) cap = n;
    return e;
}

int Ctx::consistency_scan(int mode, int n_views, const int32_t* src_off, const int32_t* src_ids, int depth_kind,
                          const uint8_t* const* sky_host, hpm_point* out, int64_t capacity, int64_t* n_points,
                          int* max_iterations_used) {
    cudaSetDevice(device);
    if (n_views < 1 || n_views > HPM_MAX_VIEWS || !src_off || !src_ids)
        return fail(HPM_E_INVALID, "consistency scan: bad arguments");
    if (depth_kind != HPM_MAP_DEPTH && depth_kind != HPM_MAP_DEPTH_GEOM)
        return fail(HPM_E_INVALID, "consistency scan: depth kind must be DEPTH or DEPTH_GEOM");
    std::vector<ScanView> hv(n_views);
    size_t max_pix = 0, total_pix = 0;
    int max_ngb = 0;
    for (int v = 0; v < n_views; ++v) {
        ViewState& vs = views[v];
        const DevMap& dm = vs.maps[depth_kind];
        const DevMap& nm = vs.maps[HPM_MAP_NORMAL];
        if (!dm.ptr || !nm.ptr || dm.w != nm.w || dm.h != nm.h)
            return fail(HPM_E_STATE, "view %d lacks depth/normal maps of one size", v);
        if (vs.w != dm.w || vs.h != dm.h)
            return fail(HPM_E_STATE, "view %d: camera size %dx%d differs from its maps %dx%d", v, vs.w, vs.h, dm.w, dm.h);
        const int ng = src_off[v + 1] - src_off[v];
        if (ng < 0 || ng > 31) return fail(HPM_E_INVALID, "view %d has %d sources (max 31)", v, ng);
        for (int k = src_off[v]; k < src_off[v + 1]; ++k)
            if (src_ids[k] < 0 || src_ids[k] >= n_views || src_ids[k] == v)
                return fail(HPM_E_INVALID, "view %d: invalid source id %d", v, src_ids[k]);
        max_ngb = std::max(max_ngb, ng);
        if (mode == 1 && (!vs.color || vs.color_w != dm.w || vs.color_h != dm.h))
            return fail(HPM_E_STATE, "view %d lacks a colour image of its map size", v);
        ScanView s{};
        s.depth = dm.ptr;
        s.normal = nm.ptr;
        s.color = vs.color;
        s.W = dm.w;
        s.H = dm.h;
        s.cam = vs.cam;
        hv[v] = s;
        max_pix = std::max(max_pix, (size_t)dm.w * dm.h);
        total_pix += (size_t)dm.w * dm.h;
    }
    // per-view scan state, carved out of one allocation in 256-byte aligned pieces
    auto al = [](size_t bytes) { return (bytes + 255) & ~size_t(255); };
    size_t state_bytes = al(sizeof(ScanView) * n_views) + al(4 * (size_t)src_off[n_views] + 4);
    for (int v = 0; v < n_views; ++v) {
        const size_t n = (size_t)hv[v].W * hv[v].H;
        state_bytes += al(n) + 3 * al(4 * n) + (mode == 1 ? al(3 * n) : 0);
    }
    cudaError_t e = ensure_dev(scan_state, scan_state_cap, state_bytes);
    if (e != cudaSuccess) return cuda_fail(e, "alloc scan state");
    uint8_t* cur = scan_state;
    auto carve = [&](size_t bytes) { uint8_t* p = cur; cur += al(bytes); return p; };
    for (int v = 0; v < n_views; ++v) {
        const size_t n = (size_t)hv[v].W * hv[v].H;
        hv[v].mask = carve(n);
        hv[v].cons = reinterpret_cast<float*>(carve(4 * n));
        hv[v].marktime = reinterpret_cast<int32_t*>(carve(4 * n));
        hv[v].marklast = reinterpret_cast<int32_t*>(carve(4 * n));
        if (mode == 1 && sky_host && sky_host[v]) {
            uint8_t* sky = carve(3 * n);
            e = cudaMemcpyAsync(sky, sky_host[v], 3 * n, cudaMemcpyHostToDevice, stream);
            if (e != cudaSuccess) return cuda_fail(e, "upload sky mask");
            hv[v].sky = sky;
        }
        cudaMemsetAsync(hv[v].mask, 0, n, stream);
        cudaMemsetAsync(hv[v].cons, 0, 4 * n, stream);
        cudaMemsetAsync(hv[v].marktime, 0x7f, 4 * n, stream);
    }
    ScanView* d_views = reinterpret_cast<ScanView*>(carve(sizeof(ScanView) * n_views));
    int32_t* d_srcs = reinterpret_cast<int32_t*>(carve(4 * (size_t)src_off[n_views] + 4));
    e = cudaMemcpyAsync(d_views, hv.data(), sizeof(ScanView) * n_views, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_srcs, src_ids, 4 * (size_t)src_off[n_views], cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return cuda_fail(e, "upload scan views");

    // per-pixel work buffers (sized for the largest view)
    const size_t nblocks_max = (max_pix + kScanBlock - 1) / kScanBlock;
    const size_t ng = std::max(1, max_ngb);
    const size_t wbytes = al(4 * max_pix * ng) + al(8 * max_pix * ng) + al(4 * max_pix * ng) + 5 * al(4 * max_pix) +
                          al(max_pix) + al(4 * nblocks_max * ng) + al(64) + al(4 * kMaxScanIterations);
    e = ensure_dev(scan_work, scan_work_cap, wbytes);
    if (e != cudaSuccess) return cuda_fail(e, "alloc scan work");
    cur = scan_work;
    int32_t* pos = reinterpret_cast<int32_t*>(carve(4 * max_pix * ng));
    double* wexp = reinterpret_cast<double*>(carve(8 * max_pix * ng));
    int32_t* last = reinterpret_cast<int32_t*>(carve(4 * max_pix * ng));
    uint32_t* test = reinterpret_cast<uint32_t*>(carve(4 * max_pix));
    uint32_t* eff = reinterpret_cast<uint32_t*>(carve(4 * max_pix));
    float* dyn = reinterpret_cast<float*>(carve(4 * max_pix));
    uint8_t* acc = carve(max_pix);
    int32_t* keep = reinterpret_cast<int32_t*>(carve(4 * max_pix));
    int32_t* offs = reinterpret_cast<int32_t*>(carve(4 * max_pix));
    int32_t* block_max = reinterpret_cast<int32_t*>(carve(4 * nblocks_max * ng));
    int32_t* d_total = reinterpret_cast<int32_t*>(carve(64));
    int* d_changed = reinterpret_cast<int*>(carve(4 * kMaxScanIterations));  // one flag per round

    int64_t emitted = 0;
    int max_iter = 0;
    for (int i = 0; i < n_views; ++i) {
        const int npix = hv[i].W * hv[i].H;
        const int n_ngb = src_off[i + 1] - src_off[i];
        const int32_t* srcs = d_srcs + src_off[i];
        const int blocks = (npix + 255) / 256;
        const int nblocks = (npix + kScanBlock - 1) / kScanBlock;
        if (mode == 0) k_candidates<0><<<blocks, 256, 0, stream>>>(d_views, i, srcs, n_ngb, pos, wexp, test, npix);
        else k_candidates<1><<<blocks, 256, 0, stream>>>(d_views, i, srcs, n_ngb, pos, wexp, test, npix);
        cudaMemsetAsync(eff, 0xff, 4 * (size_t)npix, stream);
        k_update_eff<<<blocks, 256, 0, stream>>>(d_views, srcs, n_ngb, pos, test, eff, nullptr, npix, 0);
        launches += 2;
        bool converged = n_ngb == 0;
        int it = 0;
        int max_sp = 0;
        for (int j = 0; j < n_ngb; ++j) {
            const ScanView& vs = hv[src_ids[src_off[i] + j]];
            max_sp = std::max(max_sp, vs.W * vs.H);
        }
        const dim3 reset_grid((max_sp + 255) / 256, std::max(1, n_ngb));
        // rounds of the fixed point run kRoundsPerCheck at a time between reads of their change
        // flags; a round after the one that changed nothing recomputes the same state from the same
        // eff, so extra rounds would leave every result as it was at the fixed point
        while (!converged && it < kMaxScanIterations) {
            const int batch = std::min(kRoundsPerCheck, kMaxScanIterations - it);
            cudaMemsetAsync(d_changed + it, 0, 4 * (size_t)batch, stream);
            for (int r = 0; r < batch; ++r) {
                k_accept<<<blocks, 256, 0, stream>>>(eff, wexp, n_ngb, dyn, acc, npix);
                k_last_local<<<dim3(nblocks, n_ngb), kScanBlock, 0, stream>>>(eff, n_ngb, last, block_max, npix);
                k_last_blocks<<<1, 32, 0, stream>>>(block_max, nblocks, n_ngb);
                k_last_combine<<<blocks, 256, 0, stream>>>(last, block_max, n_ngb, npix, nblocks);
                k_reset_marks<<<reset_grid, 256, 0, stream>>>(d_views, srcs, mode == 0 ? 1 : 0);
                if (mode == 0) k_marks<0><<<blocks, 256, 0, stream>>>(d_views, srcs, n_ngb, pos, last, acc, npix);
                else k_marks<1><<<blocks, 256, 0, stream>>>(d_views, srcs, n_ngb, pos, last, acc, npix);
                k_update_eff<<<blocks, 256, 0, stream>>>(d_views, srcs, n_ngb, pos, test, eff, d_changed + it + r,
                                                         npix, 1);
                launches += 7;
            }
            int changed[kRoundsPerCheck];
            e = cudaMemcpyAsync(changed, d_changed + it, 4 * (size_t)batch, cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) return cuda_fail(e, "consistency iteration");
            int r = 0;
            while (r < batch && changed[r] != 0) ++r;
            if (r < batch) {
                converged = true;
                it += r + 1;
            } else {
                it += batch;
            }
        }
        if (!converged) {
            for (int j = 0; j < n_ngb; ++j) {
                const ScanView& vs = hv[src_ids[src_off[i] + j]];
                cudaMemsetAsync(vs.marktime, 0x7f, 4 * (size_t)vs.W * vs.H, stream);
                if (mode == 0) cudaMemsetAsync(vs.marklast, 0xff, 4 * (size_t)vs.W * vs.H, stream);
            }
            if (mode == 0) k_sequential<0><<<1, 32, 0, stream>>>(d_views, srcs, n_ngb, pos, wexp, test, dyn, acc, npix);
            else k_sequential<1><<<1, 32, 0, stream>>>(d_views, srcs, n_ngb, pos, wexp, test, dyn, acc, npix);
            ++launches;
        } else if (n_ngb == 0) {
            cudaMemsetAsync(acc, 0, npix, stream);
        }
        max_iter = std::max(max_iter, converged ? it : kMaxScanIterations + 1);
        for (int j = 0; j < n_ngb; ++j) {
            const int sid = src_ids[src_off[i] + j];
            const int sp = hv[sid].W * hv[sid].H;
            if (mode == 0) k_apply_marks<0><<<(sp + 255) / 256, 256, 0, stream>>>(d_views, sid, dyn);
            else k_apply_marks<1><<<(sp + 255) / 256, 256, 0, stream>>>(d_views, sid, dyn);
            ++launches;
        }
        if (mode == 0) {
            e = ensure_map(i, HPM_MAP_CONF, hv[i].W, hv[i].H);
            if (e != cudaSuccess) return cuda_fail(e, "alloc confidence map");
            k_conf_own<<<blocks, 256, 0, stream>>>(d_views, i, dyn, acc, views[i].maps[HPM_MAP_CONF].ptr, npix);
            ++launches;
        } else {
            k_fuse_flags<<<blocks, 256, 0, stream>>>(d_views, i, acc, keep, npix);
            // block_max is free here (the mark iterations of view i are done): tile totals
            k_tile_sums<<<nblocks, kScanBlock, 0, stream>>>(keep, npix, block_max);
            k_scan_tile_sums<<<1, kScanBlock, 0, stream>>>(block_max, nblocks, d_total);
            if (out) {
                k_scan_tiles<<<nblocks, kScanBlock, 0, stream>>>(keep, npix, block_max, offs);
                k_fuse_emit<<<blocks, 256, 0, stream>>>(d_views, i, keep, offs, out, emitted, capacity, npix);
            }
            launches += out ? 5 : 3;
            int32_t total = 0;
            e = cudaMemcpyAsync(&total, d_total, 4, cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) return cuda_fail(e, "fusion count");
            emitted += total;
        }
    }
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "consistency scan");
    if (n_points) *n_points = emitted;
    if (max_iterations_used) *max_iterations_used = max_iter;
    return HPM_OK;
}

}  // namespace hpm
