// PatchMatch run orchestration behind hpm_run_patchmatch / hpm_eval_costs:
// the device-resident replacement of HPM::CudaSpaceInitialization's reloads
// (HPM.cpp:741-906, 942-984), HPM::RunPatchMatch (HPM.cu:2987-3035) and the
// result hand-off of ProcessProblem (main.cpp:599-626).
#include "ctx.hpp"

#include <cuda_fp16.h>
#include "hpm_geometry.h"
#include "pm_kernels.cuh"
#include "aux_kernels.cuh"

#include <algorithm>
#include <cstring>

namespace hpm {

__global__ void k_pack_planes(const float* __restrict__ normal, const float* __restrict__ depth,
                              float4* __restrict__ planes, const float* __restrict__ cost_in,
                              float* __restrict__ cost_out, int n);
__global__ void k_pack_scaled(const float* __restrict__ normal, const float* __restrict__ w_src,
                              float4* __restrict__ out, int n);
__global__ void k_unpack_planes(const float4* __restrict__ planes, float* __restrict__ depth,
                                float* __restrict__ normal, int n);

template <class T>
static cudaError_t ensure_buf(T*& p, size_t& cap, size_t n) {
    if (n <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) cap = n;
    return e;
}

__global__ void k_to_half(const float* __restrict__ src, int n, uint16_t* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = __half_as_ushort(__float2half_rn(src[i]));
}

__global__ void k_to_u8(const float* __restrict__ src, int n, uint8_t* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = (uint8_t)fminf(255.0f, fmaxf(0.0f, rintf(src[i])));
}

int Ctx::bind_texture(int view) {
    ViewState& v = views[view];
    cudaError_t e;
    if (!v.arr || v.arr_w != v.w || v.arr_h != v.h || v.arr_mode != addr_mode || v.arr_fmt != tex_format) {
        if (v.tex) { cudaDestroyTextureObject(v.tex); v.tex = 0; }
        if (v.arr && (v.arr_w != v.w || v.arr_h != v.h || v.arr_fmt != tex_format)) {
            cudaFreeArray(v.arr);
            v.arr = nullptr;
        }
        if (!v.arr) {
            // float texels, or half texels: the 0..255 grey levels are exact, the filtered sample is
            // returned rounded to half precision
            cudaChannelFormatDesc fd = tex_format == HPM_TEX_F16
                                           ? cudaCreateChannelDesc(16, 0, 0, 0, cudaChannelFormatKindFloat)
                                           : (tex_format == HPM_TEX_U8
                                                  ? cudaCreateChannelDesc(8, 0, 0, 0, cudaChannelFormatKindUnsigned)
                                                  : cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat));
            e = cudaMallocArray(&v.arr, &fd, v.w, v.h);
            if (e != cudaSuccess) return cuda_fail(e, "alloc image array");
            v.arr_w = v.w; v.arr_h = v.h;
            v.arr_fmt = tex_format;
        }
        cudaResourceDesc rd;
        memset(&rd, 0, sizeof(rd));
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = v.arr;
        cudaTextureDesc td;
        memset(&td, 0, sizeof(td));
        const cudaTextureAddressMode am = addr_mode == 1 ? cudaAddressModeWrap : cudaAddressModeClamp;
        td.addressMode[0] = am;
        td.addressMode[1] = am;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = tex_format == HPM_TEX_U8 ? cudaReadModeNormalizedFloat : cudaReadModeElementType;
        td.normalizedCoords = 0;
        e = cudaCreateTextureObject(&v.tex, &rd, &td, nullptr);
        if (e != cudaSuccess) return cuda_fail(e, "create texture");
        v.arr_mode = addr_mode;
    }
    if (tex_format == HPM_TEX_F16) {
        const size_t n = (size_t)v.w * v.h;
        e = ensure_buf(half_stage, half_stage_cap, n);
        if (e != cudaSuccess) return cuda_fail(e, "alloc half staging");
        k_to_half<<<(int)((n + 255) / 256), 256, 0, stream>>>(v.gray, (int)n, half_stage);
        ++launches;
        e = cudaMemcpy2DToArrayAsync(v.arr, 0, 0, half_stage, 2 * (size_t)v.w, 2 * (size_t)v.w, v.h,
                                     cudaMemcpyDeviceToDevice, stream);
    } else if (tex_format == HPM_TEX_U8) {
        const size_t n = (size_t)v.w * v.h;
        e = ensure_buf(half_stage, half_stage_cap, n);  // n bytes fit in the n half words
        if (e != cudaSuccess) return cuda_fail(e, "alloc byte staging");
        uint8_t* bytes = reinterpret_cast<uint8_t*>(half_stage);
        k_to_u8<<<(int)((n + 255) / 256), 256, 0, stream>>>(v.gray, (int)n, bytes);
        ++launches;
        e = cudaMemcpy2DToArrayAsync(v.arr, 0, 0, bytes, (size_t)v.w, (size_t)v.w, v.h, cudaMemcpyDeviceToDevice,
                                     stream);
    } else {
        e = cudaMemcpy2DToArrayAsync(v.arr, 0, 0, v.gray, sizeof(float) * v.w, sizeof(float) * v.w, v.h,
                                     cudaMemcpyDeviceToDevice, stream);
    }
    if (e != cudaSuccess) return cuda_fail(e, "copy image to array");
    return HPM_OK;
}

int Ctx::fill_run_args(int ref, const int32_t* srcs, int n_src, const hpm_params* params, RunArgs& a) {
    if (!params) return fail(HPM_E_INVALID, "null params");
    if (ref < 0 || ref >= HPM_MAX_VIEWS || views[ref].w == 0) return fail(HPM_E_STATE, "reference view %d not set", ref);
    if (n_src < 1 || n_src > HPM_MAX_SRC || !srcs) return fail(HPM_E_INVALID, "need 1..31 source views, got %d", n_src);
    if (params->patch_size != 11 || params->radius_increment != 2)
        return fail(HPM_E_INVALID, "patch_size 11 / radius_increment 2 required (got %d / %d)", params->patch_size,
                    params->radius_increment);
    if (params->num_images != n_src + 1)
        return fail(HPM_E_INVALID, "params.num_images (%d) != n_src + 1 (%d)", params->num_images, n_src + 1);
    memset(&a, 0, sizeof(a));
    const ViewState& rv = views[ref];
    a.cams[0] = rv.cam;
    for (int j = 0; j < n_src; ++j) {
        const int s = srcs[j];
        if (s < 0 || s >= HPM_MAX_VIEWS || views[s].w == 0) return fail(HPM_E_STATE, "source view %d not set", s);
        a.cams[j + 1] = views[s].cam;
        a.tex[j + 1] = views[s].tex;
        hpm_view_basis(&rv.cam, &views[s].cam, a.basis[j + 1].A, a.basis[j + 1].b);
        hpm_view_transfer(&rv.cam, &views[s].cam, a.fwd[j + 1].A, a.fwd[j + 1].b);
        hpm_view_transfer(&views[s].cam, &rv.cam, a.bwd[j + 1].A, a.bwd[j + 1].b);
    }
    hpm_ref_kinv(&rv.cam, a.kinv);
    // 8-bit textures return grey / 255; the NCC is scale-free, only the flat-source test scales
    a.var_s_min = tex_format == HPM_TEX_U8 ? 1e-5f / (255.0f * 255.0f) : 1e-5f;
    a.ncc_shift = ncc_mode == HPM_NCC_SHIFTED ? 1 : 0;
    a.ref_img = rv.gray;
    a.prm = *params;
    a.S = n_src;
    a.W = rv.w;
    a.H = rv.h;
    a.cover_pairs = covered_row_pairs(rv.h);
    a.view_id = (uint32_t)ref;
    a.hyp_count = (prof_flags & HPM_PROFILE_COUNT) ? prof_hyp : nullptr;
    return HPM_OK;
}

int Ctx::prepare_run(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int texture_level,
                     uint64_t seed, RunArgs& a) {
    cudaSetDevice(device);
    if (ref < 0 || ref >= HPM_MAX_VIEWS || views[ref].w == 0) return fail(HPM_E_STATE, "reference view %d not set", ref);
    cudaError_t e = ensure_run((size_t)views[ref].w * views[ref].h);
    if (e != cudaSuccess) return cuda_fail(e, "alloc run buffers");
    RunBufs b;
    b.planes = planes; b.costs = costs; b.pre_costs = pre_costs; b.sel = sel; b.rng = rng; b.conf = conf;
    return prepare_run_into(ref, srcs, n_src, params, texture_level, seed, b, a);
}

// The hypothesis reload and run setup of one run (HPM.cpp:741-906, 942-984)
// into the run buffers `b`: fills `a` and issues the per-run copies and packing
// kernels on the context's stream.
int Ctx::prepare_run_into(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int texture_level,
                          uint64_t seed, const RunBufs& b, RunArgs& a) {
    int rc = fill_run_args(ref, srcs, n_src, params, a);
    if (rc) return rc;
    if (texture_level < 0 || texture_level >= 8) return fail(HPM_E_INVALID, "texture_level must be 0..7");
    ViewState& rv = views[ref];
    const int W = rv.w, H = rv.h;
    const int n = W * H;
    const uint32_t mode = params->mode;
    const bool geom = mode & HPM_MODE_GEOM, prior = mode & HPM_MODE_PRIOR, hier = mode & HPM_MODE_HIERARCHY;
    const bool mand = mode & HPM_MODE_MAND, multi = mode & HPM_MODE_MULTIGEOM;
    if (mand && !geom) return fail(HPM_E_INVALID, "mandatory consistency requires the geometric mode");
    if (!rv.canny || rv.canny_w != W || rv.canny_h != H) return fail(HPM_E_STATE, "view %d has no Canny map of its size", ref);
    cudaError_t e;
    float4* const planes = b.planes;
    float* const costs = b.costs;
    float* const conf = b.conf;
    a.seed = seed;
    a.planes = b.planes; a.costs = b.costs; a.pre_costs = b.pre_costs; a.sel = b.sel; a.rng = b.rng; a.conf = b.conf;
    a.canny = rv.canny;
    // selected_views starts at zero at every run (fresh allocation in the reference, HPM.cpp:782)
    e = cudaMemsetAsync(b.sel, 0, sizeof(uint32_t) * n, stream);
    if (e != cudaSuccess) return cuda_fail(e, "clear view masks");
    const int blocks = (n + 255) / 256;
    const int depth_kind = multi ? HPM_MAP_DEPTH_GEOM : HPM_MAP_DEPTH;
    auto map_ok = [&](int v, int kind, int w, int h) {
        const DevMap& m = views[v].maps[kind];
        return m.ptr && m.w == w && m.h == h;
    };

    if (geom || prior) {
        // hypotheses reload: normals.dmb + depths(_geom).dmb + costs.dmb (HPM.cpp:813-846, 942-962)
        if (!map_ok(ref, depth_kind, W, H) || !map_ok(ref, HPM_MAP_NORMAL, W, H) || !map_ok(ref, HPM_MAP_COST, W, H))
            return fail(HPM_E_STATE, "view %d lacks depth/normal/cost maps of size %dx%d", ref, W, H);
        k_pack_planes<<<blocks, 256, 0, stream>>>(rv.maps[HPM_MAP_NORMAL].ptr, rv.maps[depth_kind].ptr, planes,
                                                   rv.maps[HPM_MAP_COST].ptr, costs, n);
        ++launches;
    }
    if (geom) {
        for (int j = 0; j < n_src; ++j) {
            const ViewState& sv = views[srcs[j]];
            const DevMap& m = sv.maps[depth_kind];
            if (!m.ptr || m.w <= 0) return fail(HPM_E_STATE, "source view %d lacks its depth map", srcs[j]);
            a.depth_src[j + 1] = m.ptr;
            a.dsw[j + 1] = m.w;
            a.dsh[j + 1] = m.h;
        }
    }
    if (prior || mand) {
        if (!map_ok(ref, HPM_MAP_CONF, W, H)) return fail(HPM_E_STATE, "view %d lacks a confidence map", ref);
        e = cudaMemcpyAsync(conf, rv.maps[HPM_MAP_CONF].ptr, sizeof(float) * n, cudaMemcpyDeviceToDevice, stream);
        if (e != cudaSuccess) return cuda_fail(e, "copy confidences");
    }
    if (prior) {
        if (!rv.prior || rv.prior_w != W || rv.prior_h != H) return fail(HPM_E_STATE, "view %d has no prior", ref);
        a.prior = rv.prior;
        a.pmask = rv.pmask;
    }
    if (hier && !geom && !prior) {
        // HPM.cpp:849-905: fine depth from JBU, coarse normals and costs
        const DevMap& dm = rv.maps[HPM_MAP_DEPTH];
        const DevMap& nm = rv.maps[HPM_MAP_NORMAL];
        const DevMap& cm = rv.maps[HPM_MAP_COST];
        if (!dm.ptr || dm.w != W || dm.h != H) return fail(HPM_E_STATE, "hierarchy: view %d depth map is not %dx%d", ref, W, H);
        if (!nm.ptr || !cm.ptr || cm.w != nm.w || cm.h != nm.h)
            return fail(HPM_E_STATE, "hierarchy: view %d lacks coarse normal/cost maps", ref);
        // the reference compares the map width with the image rows (HPM.cpp:869)
        const bool upsample = (nm.w != H || nm.h != W);
        if (!upsample && (nm.w != W || nm.h != H))
            return fail(HPM_E_STATE, "hierarchy: non-upsampled maps must match the image size");
        const int ns = nm.w * nm.h;
        float4* sc = b.scaled;
        if (!sc) {
            e = ensure_buf(scaled, scaled_cap, (size_t)ns);
            if (e != cudaSuccess) return cuda_fail(e, "alloc scaled map");
            sc = scaled;
        }
        k_pack_scaled<<<(ns + 255) / 256, 256, 0, stream>>>(nm.ptr, upsample ? cm.ptr : dm.ptr, sc, ns);
        k_pack_planes<<<blocks, 256, 0, stream>>>(nullptr, dm.ptr, planes, nullptr, nullptr, n);
        launches += 2;
        a.scaled = sc;
        a.prm.scaled_cols = nm.w;
        a.prm.scaled_rows = nm.h;
        if (upsample) a.prm.mode |= HPM_MODE_UPSAMPLE;
        else a.prm.mode &= ~HPM_MODE_UPSAMPLE;
    } else {
        a.prm.mode &= ~HPM_MODE_UPSAMPLE;
    }
    const bool want_texture = !prior && !mand;
    if (want_texture) {
        e = ensure_map(ref, HPM_MAP_TEXTURE0 + texture_level, W, H);
        if (e != cudaSuccess) return cuda_fail(e, "alloc texture map");
        a.texture = rv.maps[HPM_MAP_TEXTURE0 + texture_level].ptr;
    }

    return HPM_OK;
}

int Ctx::record_start(int kind, TimedLaunch*& slot) {
    slot = nullptr;
    if (!(prof_flags & HPM_PROFILE_TIMING)) return HPM_OK;
    if (prof_used == prof_events.size()) {
        TimedLaunch t{};
        cudaError_t e = cudaEventCreate(&t.start);
        if (e == cudaSuccess) e = cudaEventCreate(&t.stop);
        if (e != cudaSuccess) return cuda_fail(e, "profiling event");
        prof_events.push_back(t);
    }
    slot = &prof_events[prof_used++];
    slot->kind = kind;
    cudaError_t e = cudaEventRecord(slot->start, stream);
    return e == cudaSuccess ? HPM_OK : cuda_fail(e, "profiling event record");
}

int Ctx::launch_schedule(const RunArgs& a0, int n_half_sweeps) {
    cudaError_t e;
    TimedLaunch* t = nullptr;
    int rc = record_start(0, t);
    if (rc) return rc;
    if ((e = launch_random_init(a0, stream)) != cudaSuccess) return cuda_fail(e, "init launch");
    if (t) cudaEventRecord(t->stop, stream);
    ++launches;
    RunArgs a = a0;
    const uint32_t mode = a0.prm.mode;
    if ((mode & HPM_MODE_PRIOR) && !(mode & HPM_MODE_MAND) && n_half_sweeps > 0) {
        // confidences and the prior mask do not change during a prior-mode run: the pixels its
        // half-sweeps update are listed once, after the initialisation
        const size_t rows = 2 * (size_t)a0.cover_pairs;
        if ((e = ensure_buf(active_px, active_px_cap, rows * a0.W)) != cudaSuccess ||
            (e = ensure_buf(active_n, active_n_cap, rows)) != cudaSuccess)
            return cuda_fail(e, "alloc prior work lists");
        if ((e = launch_prior_active(a0, active_px, active_n, stream)) != cudaSuccess)
            return cuda_fail(e, "prior work lists");
        ++launches;
        a.active_px = active_px;
        a.active_n = active_n;
    }
    for (int k = 0; k < n_half_sweeps; ++k) {
        if ((rc = record_start(1, t))) return rc;
        if ((e = launch_half_sweep(a, k & 1, k >> 1, stream)) != cudaSuccess) return cuda_fail(e, "half sweep");
        if (t) cudaEventRecord(t->stop, stream);
        ++launches;
    }
    return HPM_OK;
}

int Ctx::profile_read(hpm_profile* out) {
    cudaSetDevice(device);
    memset(out, 0, sizeof(*out));
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "profile read");
    for (size_t i = 0; i < prof_used; ++i) {
        float ms = 0.0f;
        e = cudaEventElapsedTime(&ms, prof_events[i].start, prof_events[i].stop);
        if (e != cudaSuccess) return cuda_fail(e, "profiling event time");
        switch (prof_events[i].kind) {
        case HPM_STAGE_INIT: out->init_launches++; out->init_ms += ms; break;
        case HPM_STAGE_SWEEP: out->sweep_launches++; out->sweep_ms += ms; break;
        case HPM_STAGE_CONFIDENCE: out->confidence_ms += ms; break;
        case HPM_STAGE_PRIOR: out->prior_ms += ms; break;
        case HPM_STAGE_JBU: out->jbu_ms += ms; break;
        case HPM_STAGE_LEVEL: out->level_ms += ms; break;
        default: out->fusion_ms += ms; break;
        }
    }
    prof_used = 0;
    if (prof_hyp) {
        unsigned long long h[3] = {0, 0, 0};
        e = cudaMemcpy(h, prof_hyp, sizeof(h), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemset(prof_hyp, 0, sizeof(h));
        if (e != cudaSuccess) return cuda_fail(e, "hypothesis counters");
        out->init_view_evals = h[0];
        out->sweep_view_evals = h[1];
        out->sweep_sampled = h[2];
    }
    return HPM_OK;
}

int Ctx::run_patchmatch(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int texture_level,
                        uint64_t seed) {
    RunArgs a;
    int rc = prepare_run(ref, srcs, n_src, params, texture_level, seed, a);
    if (rc) return rc;
    rc = launch_schedule(a, 2 * params->max_iterations);
    if (rc) return rc;
    return finish_run(ref, a, params->mode & HPM_MODE_GEOM);
}

// GetDepthandNormal (HPM.cu:2829-2842) and the hand-off of the run's results to
// the view's resident maps (ProcessProblem, main.cpp:599-626).
int Ctx::finish_run(int ref, const RunArgs& a, bool geom) {
    cudaError_t e;
    if ((e = launch_export(a, stream)) != cudaSuccess) return cuda_fail(e, "export launch");
    ++launches;
    ViewState& rv = views[ref];
    const int W = rv.w, H = rv.h;
    const int n = W * H;
    const int blocks = (n + 255) / 256;
    const int out_depth = geom ? HPM_MAP_DEPTH_GEOM : HPM_MAP_DEPTH;
    if ((e = ensure_map(ref, out_depth, W, H)) != cudaSuccess) return cuda_fail(e, "alloc depth map");
    if ((e = ensure_map(ref, HPM_MAP_NORMAL, W, H)) != cudaSuccess) return cuda_fail(e, "alloc normal map");
    if ((e = ensure_map(ref, HPM_MAP_COST, W, H)) != cudaSuccess) return cuda_fail(e, "alloc cost map");
    k_unpack_planes<<<blocks, 256, 0, stream>>>(a.planes, rv.maps[out_depth].ptr, rv.maps[HPM_MAP_NORMAL].ptr, n);
    ++launches;
    e = cudaMemcpyAsync(rv.maps[HPM_MAP_COST].ptr, a.costs, sizeof(float) * n, cudaMemcpyDeviceToDevice, stream);
    if (e != cudaSuccess) return cuda_fail(e, "store costs");
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "patchmatch run");
    return HPM_OK;
}

int Ctx::debug_run_partial(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int texture_level,
                           uint64_t seed, int n_half_sweeps, float* planes_out, float* costs_out, uint32_t* sel_out,
                           uint32_t* draws_out) {
    if (n_half_sweeps < 0 || n_half_sweeps > 64) return fail(HPM_E_INVALID, "n_half_sweeps must be 0..64");
    RunArgs a;
    int rc = prepare_run(ref, srcs, n_src, params, texture_level, seed, a);
    if (rc) return rc;
    rc = launch_schedule(a, n_half_sweeps);
    if (rc) return rc;
    const size_t n = (size_t)a.W * a.H;
    cudaError_t e = cudaSuccess;
    if (planes_out) e = cudaMemcpyAsync(planes_out, planes, n * sizeof(float4), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && costs_out) e = cudaMemcpyAsync(costs_out, costs, n * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && sel_out) e = cudaMemcpyAsync(sel_out, sel, n * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && draws_out) e = cudaMemcpyAsync(draws_out, rng, n * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "download run state");
    return HPM_OK;
}

__global__ void k_sample_view(cudaTextureObject_t tex, int n, const float2* __restrict__ xy, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = tex2D<float>(tex, xy[i].x, xy[i].y);
}

int Ctx::sample_view(int view, int n, const float* xy, float* out) {
    cudaSetDevice(device);
    if (view < 0 || view >= HPM_MAX_VIEWS || views[view].w == 0) return fail(HPM_E_STATE, "view %d not set", view);
    if (n < 0 || (n > 0 && (!xy || !out))) return fail(HPM_E_INVALID, "hpm_sample_view: bad arguments");
    if (n == 0) return HPM_OK;
    cudaError_t e = ensure_buf(scratch, scratch_cap, (size_t)n * 12 + 64);
    if (e != cudaSuccess) return cuda_fail(e, "alloc scratch");
    float2* d_xy = reinterpret_cast<float2*>(scratch);
    float* d_out = reinterpret_cast<float*>(scratch + (size_t)n * 8);
    e = cudaMemcpyAsync(d_xy, xy, (size_t)n * 8, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return cuda_fail(e, "upload coordinates");
    k_sample_view<<<(n + 255) / 256, 256, 0, stream>>>(views[view].tex, n, d_xy, d_out);
    ++launches;
    e = cudaMemcpyAsync(out, d_out, (size_t)n * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "download samples");
    return HPM_OK;
}

// RunJBU (HPM.cpp:1266-1319): the coarser depths_geom map of a view upsampled to
// the view's current image size into its depths map; nothing happens when the
// integer scale is 1 (HPM.cpp:1272-1275).
int Ctx::jbu_view(int view, int* applied) {
    cudaSetDevice(device);
    if (applied) *applied = 0;
    if (view < 0 || view >= HPM_MAX_VIEWS || views[view].w == 0) return fail(HPM_E_STATE, "view %d not set", view);
    ViewState& v = views[view];
    const DevMap& src = v.maps[HPM_MAP_DEPTH_GEOM];
    if (!src.ptr || src.w <= 0) return fail(HPM_E_STATE, "view %d has no depths_geom map", view);
    const int scale = std::max(v.h / src.h, v.w / src.w);
    if (scale == 1) return HPM_OK;
    if (src.w * 1LL * src.h > (long long)v.w * v.h) return fail(HPM_E_STATE, "JBU source larger than the image");
    // the source map must survive while the output is written: stage it in scratch
    const size_t ns = (size_t)src.w * src.h;
    cudaError_t e = ensure_buf(scratch, scratch_cap, ns * 4 + 256);
    if (e != cudaSuccess) return cuda_fail(e, "alloc scratch");
    float* d_src = reinterpret_cast<float*>(scratch);
    const int sw = src.w, sh = src.h;
    e = cudaMemcpyAsync(d_src, src.ptr, ns * 4, cudaMemcpyDeviceToDevice, stream);
    if (e != cudaSuccess) return cuda_fail(e, "stage JBU source");
    e = ensure_map(view, HPM_MAP_DEPTH, v.w, v.h);
    if (e != cudaSuccess) return cuda_fail(e, "alloc depth map");
    e = launch_jbu(v.gray, v.w, v.h, d_src, sw, sh, v.maps[HPM_MAP_DEPTH].ptr, stream);
    if (e != cudaSuccess) return cuda_fail(e, "JBU launch");
    ++launches;
    if (applied) *applied = 1;
    return HPM_OK;
}

cudaError_t Ctx::ensure_scratch(size_t bytes) { return ensure_buf(scratch, scratch_cap, bytes); }

int Ctx::eval_costs(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int n, const int32_t* px,
                    const float* planes_h, float* out) {
    cudaSetDevice(device);
    if (n < 0 || (n > 0 && (!px || !planes_h || !out))) return fail(HPM_E_INVALID, "hpm_eval_costs: bad arguments");
    RunArgs a;
    int rc = fill_run_args(ref, srcs, n_src, params, a);
    if (rc) return rc;
    if (n == 0) return HPM_OK;
    for (int k = 0; k < n; ++k)
        if (px[2 * k] < 0 || px[2 * k] >= a.W || px[2 * k + 1] < 0 || px[2 * k + 1] >= a.H)
            return fail(HPM_E_INVALID, "pixel %d outside the reference image", k);
    const size_t bytes = (size_t)n * (8 + 16) + (size_t)n * n_src * 4 + 64;
    cudaError_t e = ensure_buf(scratch, scratch_cap, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "alloc scratch");
    float4* d_planes = reinterpret_cast<float4*>(scratch);
    int32_t* d_px = reinterpret_cast<int32_t*>(scratch + (size_t)n * 16);
    float* d_out = reinterpret_cast<float*>(scratch + (size_t)n * 24);
    e = cudaMemcpyAsync(d_planes, planes_h, (size_t)n * 16, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_px, px, (size_t)n * 8, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return cuda_fail(e, "upload hypotheses");
    if ((e = launch_eval_costs(a, n, d_px, d_planes, d_out, stream)) != cudaSuccess) return cuda_fail(e, "eval launch");
    ++launches;
    e = cudaMemcpyAsync(out, d_out, (size_t)n * n_src * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "download costs");
    return HPM_OK;
}

}  // namespace hpm
