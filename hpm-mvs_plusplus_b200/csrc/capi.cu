// C ABI implementation: a context owns every view's grey image (as a
// linear-filtered texture), its resident "dmb" maps and the work buffers of a
// PatchMatch run.  See include/hpm_capi.h for the contract.
#include "hpm_capi.h"
#include "ctx.hpp"
#include "pm_kernels.cuh"
#include "aux_kernels.cuh"
#include <cmath>
#include <vector>

namespace hpm {
int delaunay_triangulate(const int32_t* xy, int n, int width, int height, std::vector<hpm_triangle>& out);
}

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

using namespace hpm;

namespace hpm {

int Ctx::fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    err = buf;
    return code;
}

int Ctx::cuda_fail(cudaError_t e, const char* what) {
    cudaGetLastError();  // clear the runtime's last-error state so the next launch check is not stale
    return fail(HPM_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

template <class T>
static cudaError_t ensure(T*& p, size_t& cap, size_t n) {
    if (n <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) cap = n;
    return e;
}

cudaError_t Ctx::ensure_map(int view, int kind, int w, int h) {
    DevMap& m = views[view].maps[kind];
    const int ch = (kind == HPM_MAP_NORMAL) ? 3 : 1;
    cudaError_t e = ensure(m.ptr, m.cap, (size_t)w * h * ch);
    if (e == cudaSuccess) { m.w = w; m.h = h; m.ch = ch; }
    return e;
}

cudaError_t Ctx::ensure_run(size_t n) {
    cudaError_t e;
    if ((e = ensure(planes, run_cap_planes, n)) != cudaSuccess) return e;
    if ((e = ensure(costs, run_cap_costs, n)) != cudaSuccess) return e;
    if ((e = ensure(pre_costs, run_cap_pre, n)) != cudaSuccess) return e;
    if ((e = ensure(sel, run_cap_sel, n)) != cudaSuccess) return e;
    if ((e = ensure(rng, run_cap_rng, n)) != cudaSuccess) return e;
    if ((e = ensure(conf, run_cap_conf, n)) != cudaSuccess) return e;
    return cudaSuccess;
}

Ctx::~Ctx() {
    for (auto& v : views) {
        if (v.tex) cudaDestroyTextureObject(v.tex);
        if (v.arr) cudaFreeArray(v.arr);
        if (v.gray) cudaFree(v.gray);
        for (auto& m : v.maps) if (m.ptr) cudaFree(m.ptr);
        if (v.canny) cudaFree(v.canny);
        if (v.prior) cudaFree(v.prior);
        if (v.pmask) cudaFree(v.pmask);
        if (v.color) cudaFree(v.color);
        if (v.orig) cudaFree(v.orig);
    }
    for (auto& g : batch_graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    for (void* p : { (void*)b_planes, (void*)b_costs, (void*)b_pre, (void*)b_sel, (void*)b_rng, (void*)b_conf,
                     (void*)b_scaled, (void*)d_bargs, (void*)d_btiles })
        if (p) cudaFree(p);
    if (h_bargs) cudaFreeHost(h_bargs);
    if (h_btiles) cudaFreeHost(h_btiles);
    for (void* p : { (void*)planes, (void*)costs, (void*)pre_costs, (void*)sel, (void*)rng, (void*)conf,
                     (void*)active_px, (void*)active_n, (void*)b_active,
                     (void*)scaled, (void*)scratch, (void*)scan_state, (void*)scan_work, (void*)points,
                     (void*)prior_small, (void*)prior_tris, (void*)prior_label, (void*)prior_work,
                     (void*)prior_unormal, (void*)canny_mag, (void*)canny_grad, (void*)canny_state })
        if (p) cudaFree(p);
    for (auto& t : prof_events) {
        cudaEventDestroy(t.start);
        cudaEventDestroy(t.stop);
    }
    if (prof_hyp) cudaFree(prof_hyp);
    if (half_stage) cudaFree(half_stage);
    if (stream) cudaStreamDestroy(stream);
}

// ---------------------------------------------------------------- small kernels

__global__ void k_pack_planes(const float* __restrict__ normal, const float* __restrict__ depth,
                              float4* __restrict__ planes, const float* __restrict__ cost_in,
                              float* __restrict__ cost_out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p;
    p.x = normal ? normal[3 * (size_t)i] : 0.0f;
    p.y = normal ? normal[3 * (size_t)i + 1] : 0.0f;
    p.z = normal ? normal[3 * (size_t)i + 2] : 0.0f;
    p.w = depth[i];
    planes[i] = p;
    if (cost_out) cost_out[i] = cost_in[i];
}

// Hierarchy input map (HPM.cpp:877-892): coarse normals with the coarse cost
// (upsample) or the depth as w.
__global__ void k_pack_scaled(const float* __restrict__ normal, const float* __restrict__ w_src,
                              float4* __restrict__ out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = make_float4(normal[3 * (size_t)i], normal[3 * (size_t)i + 1], normal[3 * (size_t)i + 2], w_src[i]);
}

__global__ void k_unpack_planes(const float4* __restrict__ planes, float* __restrict__ depth,
                                float* __restrict__ normal, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = planes[i];
    depth[i] = p.w;
    normal[3 * (size_t)i] = p.x;
    normal[3 * (size_t)i + 1] = p.y;
    normal[3 * (size_t)i + 2] = p.z;
}

}  // namespace hpm

// ---------------------------------------------------------------- C ABI

extern "C" {

int hpm_create(int device, hpm_ctx** out) {
    if (!out) return HPM_E_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return HPM_E_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return HPM_E_CUDA;
    Ctx* c = new (std::nothrow) Ctx();
    if (!c) return HPM_E_NOMEM;
    c->device = device;
    c->views.resize(HPM_MAX_VIEWS);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return HPM_E_CUDA;
    }
    *out = reinterpret_cast<hpm_ctx*>(c);
    return HPM_OK;
}

void hpm_destroy(hpm_ctx* ctx) {
    if (!ctx) return;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    delete c;
}

const char* hpm_last_error(const hpm_ctx* ctx) {
    if (!ctx) return "null context";
    return reinterpret_cast<const Ctx*>(ctx)->err.c_str();
}

int hpm_set_address_mode(hpm_ctx* ctx, int mode) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (mode != 0 && mode != 1) return c->fail(HPM_E_INVALID, "address mode must be 0 (clamp) or 1 (wrap)");
    c->addr_mode = mode;
    return HPM_OK;
}

int hpm_set_texture_format(hpm_ctx* ctx, int format) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (format != HPM_TEX_F32 && format != HPM_TEX_F16 && format != HPM_TEX_U8)
        return c->fail(HPM_E_INVALID, "texture format must be HPM_TEX_F32, HPM_TEX_F16 or HPM_TEX_U8");
    c->tex_format = format;
    return HPM_OK;
}

int hpm_set_ncc_mode(hpm_ctx* ctx, int mode) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (mode != HPM_NCC_PLAIN && mode != HPM_NCC_SHIFTED)
        return c->fail(HPM_E_INVALID, "NCC mode must be HPM_NCC_PLAIN or HPM_NCC_SHIFTED");
    c->ncc_mode = mode;
    return HPM_OK;
}

int64_t hpm_launch_count(const hpm_ctx* ctx) { return ctx ? reinterpret_cast<const Ctx*>(ctx)->launches : 0; }

int hpm_synchronize(hpm_ctx* ctx) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "synchronize");
    return HPM_OK;
}

int hpm_set_view(hpm_ctx* ctx, int view, const float* gray, int w, int h, const hpm_camera* cam) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (view < 0 || view >= HPM_MAX_VIEWS || !gray || !cam || w <= 0 || h <= 0)
        return c->fail(HPM_E_INVALID, "hpm_set_view: bad arguments");
    cudaSetDevice(c->device);
    ViewState& v = c->views[view];
    cudaError_t e = ensure(v.gray, v.gray_cap, (size_t)w * h);
    if (e != cudaSuccess) return c->cuda_fail(e, "alloc grey image");
    e = cudaMemcpyAsync(v.gray, gray, sizeof(float) * w * h, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "upload grey image");
    v.w = w; v.h = h; v.cam = *cam;
    v.cam.width = w; v.cam.height = h;
    return c->bind_texture(view);
}

int hpm_set_map(hpm_ctx* ctx, int view, int kind, const float* data, int w, int h) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (view < 0 || view >= HPM_MAX_VIEWS || kind < 0 || kind >= kNumMaps || !data || w <= 0 || h <= 0)
        return c->fail(HPM_E_INVALID, "hpm_set_map: bad arguments");
    cudaSetDevice(c->device);
    cudaError_t e = c->ensure_map(view, kind, w, h);
    if (e != cudaSuccess) return c->cuda_fail(e, "alloc map");
    const DevMap& m = c->views[view].maps[kind];
    e = cudaMemcpyAsync(m.ptr, data, sizeof(float) * (size_t)w * h * m.ch, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "upload map");
    return HPM_OK;
}

int hpm_get_map(hpm_ctx* ctx, int view, int kind, float* data, size_t capacity, int* w, int* h) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (view < 0 || view >= HPM_MAX_VIEWS || kind < 0 || kind >= kNumMaps)
        return c->fail(HPM_E_INVALID, "hpm_get_map: bad arguments");
    const DevMap& m = c->views[view].maps[kind];
    if (!m.ptr || m.w == 0) return c->fail(HPM_E_STATE, "view %d has no map %d", view, kind);
    if (w) *w = m.w;
    if (h) *h = m.h;
    const size_t n = (size_t)m.w * m.h * m.ch;
    if (!data) return HPM_OK;
    if (capacity < n) return c->fail(HPM_E_INVALID, "hpm_get_map: capacity %zu < %zu", capacity, n);
    cudaSetDevice(c->device);
    cudaError_t e = cudaMemcpyAsync(data, m.ptr, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "download map");
    return HPM_OK;
}

int hpm_set_canny(hpm_ctx* ctx, int view, const uint8_t* edges, int w, int h) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (view < 0 || view >= HPM_MAX_VIEWS || !edges || w <= 0 || h <= 0)
        return c->fail(HPM_E_INVALID, "hpm_set_canny: bad arguments");
    cudaSetDevice(c->device);
    ViewState& v = c->views[view];
    cudaError_t e = ensure(v.canny, v.canny_cap, (size_t)w * h);
    if (e != cudaSuccess) return c->cuda_fail(e, "alloc canny");
    e = cudaMemcpyAsync(v.canny, edges, (size_t)w * h, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "upload canny");
    v.canny_w = w; v.canny_h = h;
    return HPM_OK;
}

int hpm_set_prior(hpm_ctx* ctx, int view, const float* planes, const uint8_t* mask, int w, int h) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (view < 0 || view >= HPM_MAX_VIEWS || !planes || !mask || w <= 0 || h <= 0)
        return c->fail(HPM_E_INVALID, "hpm_set_prior: bad arguments");
    cudaSetDevice(c->device);
    ViewState& v = c->views[view];
    cudaError_t e = ensure(v.prior, v.prior_cap, (size_t)w * h);
    if (e == cudaSuccess) e = ensure(v.pmask, v.pmask_cap, (size_t)w * h);
    if (e != cudaSuccess) return c->cuda_fail(e, "alloc prior");
    e = cudaMemcpyAsync(v.prior, planes, sizeof(float4) * w * h, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(v.pmask, mask, (size_t)w * h, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "upload prior");
    v.prior_w = w; v.prior_h = h;
    return HPM_OK;
}

int hpm_run_patchmatch(hpm_ctx* ctx, int ref, const int32_t* srcs, int n_src, const hpm_params* params,
                       int texture_level, uint64_t seed) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    return c->run_patchmatch(ref, srcs, n_src, params, texture_level, seed);
}

int hpm_run_batch(hpm_ctx* ctx, int n, const int32_t* refs, const int32_t* src_off, const int32_t* src_ids,
                  const hpm_params* params, int texture_level, const uint64_t* seeds) {
    if (!ctx) return HPM_E_INVALID;
    return reinterpret_cast<Ctx*>(ctx)->run_batch(n, refs, src_off, src_ids, params, texture_level, seeds);
}

int hpm_set_batch_options(hpm_ctx* ctx, int flags) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (flags & ~(HPM_BATCH_AUTOTUNE | HPM_BATCH_GRAPH | HPM_BATCH_PER_VIEW))
        return c->fail(HPM_E_INVALID, "hpm_set_batch_options: unknown flags 0x%x", flags);
    c->batch_flags = flags;
    return HPM_OK;
}

int hpm_eval_costs(hpm_ctx* ctx, int ref, const int32_t* srcs, int n_src, const hpm_params* params, int n,
                   const int32_t* px, const float* planes, float* out) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    return c->eval_costs(ref, srcs, n_src, params, n, px, planes, out);
}

int hpm_set_color(hpm_ctx* ctx, int view, const uint8_t* bgr, int w, int h) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (view < 0 || view >= HPM_MAX_VIEWS || !bgr || w <= 0 || h <= 0)
        return c->fail(HPM_E_INVALID, "hpm_set_color: bad arguments");
    cudaSetDevice(c->device);
    ViewState& v = c->views[view];
    cudaError_t e = ensure(v.color, v.color_cap, (size_t)w * h * 3);
    if (e != cudaSuccess) return c->cuda_fail(e, "alloc colour");
    e = cudaMemcpyAsync(v.color, bgr, (size_t)w * h * 3, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "upload colour");
    v.color_w = w; v.color_h = h;
    return HPM_OK;
}

int hpm_jbu(hpm_ctx* ctx, int view, int* applied) {
    if (!ctx) return HPM_E_INVALID;
    return reinterpret_cast<Ctx*>(ctx)->jbu_view(view, applied);
}

int hpm_jbu_maps(hpm_ctx* ctx, int view, const float* src_depth, const float* src_normal, int sw, int sh,
                 float* out_depth, float* out_normal) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (view < 0 || view >= HPM_MAX_VIEWS || c->views[view].w == 0) return c->fail(HPM_E_STATE, "view %d not set", view);
    if (!src_depth || !out_depth || sw <= 0 || sh <= 0 || (src_normal && !out_normal))
        return c->fail(HPM_E_INVALID, "hpm_jbu_maps: bad arguments");
    cudaSetDevice(c->device);
    const ViewState& v = c->views[view];
    const size_t ns = (size_t)sw * sh, nf = (size_t)v.w * v.h;
    cudaError_t e = ensure(c->scratch, c->scratch_cap, ns * 16 + nf * 16 + 256);
    if (e != cudaSuccess) return c->cuda_fail(e, "alloc scratch");
    float* d_sd = reinterpret_cast<float*>(c->scratch);
    float* d_sn = d_sd + ns;
    float* d_od = d_sn + 3 * ns;
    float* d_on = d_od + nf;
    e = cudaMemcpyAsync(d_sd, src_depth, 4 * ns, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && src_normal) e = cudaMemcpyAsync(d_sn, src_normal, 12 * ns, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "upload JBU input");
    e = src_normal ? launch_jbu_prior(v.gray, v.w, v.h, d_sd, d_sn, sw, sh, d_od, d_on, c->stream)
                   : launch_jbu(v.gray, v.w, v.h, d_sd, sw, sh, d_od, c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "JBU launch");
    ++c->launches;
    e = cudaMemcpyAsync(out_depth, d_od, 4 * nf, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && src_normal) e = cudaMemcpyAsync(out_normal, d_on, 12 * nf, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "download JBU output");
    return HPM_OK;
}

int hpm_confidence_eval(hpm_ctx* ctx, int n_views, const int32_t* src_off, const int32_t* src_ids, int depth_kind,
                        int* iterations) {
    if (!ctx) return HPM_E_INVALID;
    return reinterpret_cast<Ctx*>(ctx)->consistency_scan(0, n_views, src_off, src_ids, depth_kind, nullptr, nullptr,
                                                         0, nullptr, iterations);
}

int hpm_fuse(hpm_ctx* ctx, int n_views, const int32_t* src_off, const int32_t* src_ids, int depth_kind,
             const uint8_t* const* sky_masks, hpm_point* out, int64_t capacity, int64_t* n_points) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (n_views < 1 || n_views > HPM_MAX_VIEWS) return c->fail(HPM_E_INVALID, "hpm_fuse: bad view count");
    // checked before the maps are read to size the point buffer
    if (depth_kind != HPM_MAP_DEPTH && depth_kind != HPM_MAP_DEPTH_GEOM)
        return c->fail(HPM_E_INVALID, "hpm_fuse: depth_kind must be HPM_MAP_DEPTH or HPM_MAP_DEPTH_GEOM");
    if (!src_off || !src_ids) return c->fail(HPM_E_INVALID, "hpm_fuse: null source lists");
    cudaSetDevice(c->device);
    size_t total = 0;
    for (int v = 0; v < n_views; ++v) total += (size_t)c->views[v].maps[depth_kind].w * c->views[v].maps[depth_kind].h;
    cudaError_t e = ensure(c->points, c->points_cap, total + 1);
    if (e != cudaSuccess) return c->cuda_fail(e, "alloc points");
    int64_t n = 0;
    int rc = c->consistency_scan(1, n_views, src_off, src_ids, depth_kind, sky_masks, c->points, (int64_t)total, &n,
                                 nullptr);
    if (rc) return rc;
    c->n_points = n;
    if (n_points) *n_points = n;
    if (out && capacity > 0) {
        const int64_t m = n < capacity ? n : capacity;
        e = cudaMemcpyAsync(out, c->points, sizeof(hpm_point) * (size_t)m, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return c->cuda_fail(e, "download points");
    }
    return HPM_OK;
}

int hpm_support_points(hpm_ctx* ctx, int view, int distance, int32_t* xy, int capacity, int* n, int* w, int* h) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (view < 0 || view >= HPM_MAX_VIEWS || c->views[view].w == 0) return c->fail(HPM_E_STATE, "view %d not set", view);
    if (distance < 0 || distance > 2) return c->fail(HPM_E_INVALID, "prior scale distance must be 0, 1 or 2");
    std::vector<int32_t> pts;
    int sw = 0, sh = 0;
    int rc = c->support_points(view, distance, pts, sw, sh);
    if (rc) return rc;
    const int np = (int)pts.size() / 2;
    if (n) *n = np;
    if (w) *w = sw;
    if (h) *h = sh;
    if (xy) std::copy(pts.begin(), pts.begin() + 2 * std::min(np, std::max(capacity, 0)), xy);
    return HPM_OK;
}

int hpm_delaunay(const int32_t* xy, int n, int w, int h, hpm_triangle* out, int capacity, int* n_out) {
    if (n < 0 || (n > 0 && !xy) || w <= 0 || h <= 0) return HPM_E_INVALID;
    std::vector<hpm_triangle> tris;
    delaunay_triangulate(xy, n, w, h, tris);
    if (n_out) *n_out = (int)tris.size();
    if (out) std::copy(tris.begin(), tris.begin() + std::min((int)tris.size(), std::max(capacity, 0)), out);
    return HPM_OK;
}

int hpm_prior_from_triangles(hpm_ctx* ctx, int view, int distance, const hpm_triangle* tris, int n_tris) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (view < 0 || view >= HPM_MAX_VIEWS || c->views[view].w == 0) return c->fail(HPM_E_STATE, "view %d not set", view);
    if (distance < 0 || distance > 2 || n_tris < 0 || (n_tris > 0 && !tris))
        return c->fail(HPM_E_INVALID, "hpm_prior_from_triangles: bad arguments");
    int sw = c->views[view].w, sh = c->views[view].h;
    if (distance > 0) {
        const float f = 1.0f / (distance * 2);
        sw = (int)std::round(sw * f);
        sh = (int)std::round(sh * f);
    }
    return c->prior_from_triangles(view, distance, tris, n_tris, sw, sh);
}

int hpm_build_prior(hpm_ctx* ctx, int view, int distance, int* n_points, int* n_triangles) {
    if (!ctx) return HPM_E_INVALID;
    return reinterpret_cast<Ctx*>(ctx)->build_prior(view, distance, n_points, n_triangles);
}

int hpm_get_prior(hpm_ctx* ctx, int view, float* planes, uint8_t* mask) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (view < 0 || view >= HPM_MAX_VIEWS || !c->views[view].prior) return c->fail(HPM_E_STATE, "view %d has no prior", view);
    const ViewState& v = c->views[view];
    const size_t n = (size_t)v.prior_w * v.prior_h;
    cudaError_t e = cudaSuccess;
    if (planes) e = cudaMemcpyAsync(planes, v.prior, 16 * n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && mask) e = cudaMemcpyAsync(mask, v.pmask, n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "download prior");
    return HPM_OK;
}

int hpm_set_image(hpm_ctx* ctx, int view, const uint8_t* bgr, int w, int h) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (view < 0 || view >= HPM_MAX_VIEWS || !bgr || w <= 0 || h <= 0)
        return c->fail(HPM_E_INVALID, "hpm_set_image: bad arguments");
    cudaSetDevice(c->device);
    ViewState& v = c->views[view];
    cudaError_t e = ensure(v.orig, v.orig_cap, (size_t)w * h * 3);
    if (e != cudaSuccess) return c->cuda_fail(e, "alloc image");
    e = cudaMemcpyAsync(v.orig, bgr, (size_t)w * h * 3, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "upload image");
    v.orig_w = w; v.orig_h = h;
    return HPM_OK;
}

int hpm_prepare_level(hpm_ctx* ctx, int view, int w, int h, const hpm_camera* cam) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (view < 0 || view >= HPM_MAX_VIEWS || !cam || w <= 0 || h <= 0)
        return c->fail(HPM_E_INVALID, "hpm_prepare_level: bad arguments");
    return c->prepare_level_image(view, w, h, *cam);
}

int hpm_get_level(hpm_ctx* ctx, int view, uint8_t* bgr, float* gray, uint8_t* edges) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (view < 0 || view >= HPM_MAX_VIEWS || c->views[view].w == 0) return c->fail(HPM_E_STATE, "view %d not set", view);
    const ViewState& v = c->views[view];
    const size_t n = (size_t)v.w * v.h;
    cudaError_t e = cudaSuccess;
    if (bgr && v.color) e = cudaMemcpyAsync(bgr, v.color, n * 3, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && gray) e = cudaMemcpyAsync(gray, v.gray, n * 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && edges && v.canny) e = cudaMemcpyAsync(edges, v.canny, n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "download level image");
    return HPM_OK;
}

int hpm_reconstruct(hpm_ctx* ctx, int n_views, const hpm_camera* cams, const int32_t* src_off, const int32_t* src_ids,
                    const hpm_recon_options* opt, int64_t* n_points) {
    if (!ctx) return HPM_E_INVALID;
    return reinterpret_cast<Ctx*>(ctx)->reconstruct(n_views, cams, src_off, src_ids, opt, n_points);
}

int hpm_get_points(hpm_ctx* ctx, hpm_point* out, int64_t capacity, int64_t* n_points) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (n_points) *n_points = c->n_points;
    if (!out || capacity <= 0 || c->n_points == 0) return HPM_OK;
    const int64_t m = c->n_points < capacity ? c->n_points : capacity;
    cudaError_t e = cudaMemcpyAsync(out, c->points, sizeof(hpm_point) * (size_t)m, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "download points");
    return HPM_OK;
}

int hpm_sample_view(hpm_ctx* ctx, int view, int n, const float* xy, float* out) {
    if (!ctx) return HPM_E_INVALID;
    return reinterpret_cast<Ctx*>(ctx)->sample_view(view, n, xy, out);
}

int hpm_debug_run_partial(hpm_ctx* ctx, int ref, const int32_t* srcs, int n_src, const hpm_params* params,
                          int texture_level, uint64_t seed, int n_half_sweeps, float* planes, float* costs,
                          uint32_t* selected_views, uint32_t* draws) {
    if (!ctx) return HPM_E_INVALID;
    return reinterpret_cast<Ctx*>(ctx)->debug_run_partial(ref, srcs, n_src, params, texture_level, seed,
                                                          n_half_sweeps, planes, costs, selected_views, draws);
}

}  // extern "C"
