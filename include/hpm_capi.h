/*
 * C ABI of libhpm_cuda.so: the drop-in boundary of the HPM-MVS++ depth/normal
 * hot path.
 *
 * The reference exposes this path as the C++ class `HPM` (HPM.h:58-170) plus
 * `RunJBU` (HPM.h:20), `ConfidenceEvaluation` and `RunFusion` (main.cpp:823-1109).
 * Each of those uploads its inputs, runs, downloads and goes through .dmb files
 * on disk.  This ABI keeps every view's images and "dmb maps" resident on the
 * GPU inside one context, so a whole reconstruction schedule runs without
 * host round trips; the host C++ `HPM` class (host/hpm.hpp) is rebuilt on top.
 *
 * Conventions: plain pointers and sizes, host memory unless a name says
 * `_device`; every function returns 0 on success or a positive HPM_E* code and
 * never exits or throws (the reference calls exit(EXIT_FAILURE), HPM.cpp:68-76);
 * hpm_last_error() describes the last failure.  One CUDA stream per context;
 * calls on one context are not thread-safe.
 */
#ifndef HPM_CAPI_H
#define HPM_CAPI_H

#include <stddef.h>
#include <stdint.h>
#include "hpm_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hpm_ctx hpm_ctx;

enum {
    HPM_OK = 0,
    HPM_E_INVALID = 1,   /* bad argument */
    HPM_E_CUDA = 2,      /* CUDA runtime error */
    HPM_E_STATE = 3,     /* missing input (view, map, prior) for the requested mode */
    HPM_E_NOMEM = 4
};

/* Per-view resident maps: the reference's per-view .dmb files
 * (depths.dmb, depths_geom.dmb, normals.dmb, costs.dmb, confidence.dmb,
 * texture<k>.dmb; main.cpp:612-626, 1094). */
enum {
    HPM_MAP_DEPTH = 0,
    HPM_MAP_DEPTH_GEOM = 1,
    HPM_MAP_NORMAL = 2,      /* 3 floats per pixel, world frame */
    HPM_MAP_COST = 3,
    HPM_MAP_CONF = 4,
    HPM_MAP_TEXTURE0 = 8     /* HPM_MAP_TEXTURE0 + k holds texture<k>.dmb, k < 8 */
};

/* Create a context on CUDA device `device`.  Replaces the per-problem
 * allocation of HPM::CudaSpaceInitialization (HPM.cpp:741-906). */
int hpm_create(int device, hpm_ctx **out);
void hpm_destroy(hpm_ctx *ctx);
const char *hpm_last_error(const hpm_ctx *ctx);

/* Upload the grey image (float, 0..255, row-major) and camera of view `view`
 * at the current pyramid level.  Replaces the texture setup of
 * HPM::InuputInitialization / CudaSpaceInitialization (HPM.cpp:644-767).
 * `cam` must already be scaled to w x h. */
int hpm_set_view(hpm_ctx *ctx, int view, const float *gray, int w, int h, const hpm_camera *cam);

/* Upload / download one map of a view (see HPM_MAP_*).  Normal maps have 3
 * channels.  hpm_get_map writes w*h*channels floats and the size. */
int hpm_set_map(hpm_ctx *ctx, int view, int kind, const float *data, int w, int h);
int hpm_get_map(hpm_ctx *ctx, int view, int kind, float *data, size_t capacity, int *w, int *h);

/* Canny edge map (0 or 255) of the reference view at the current level
 * (HPM::CudaCannyInitialization, HPM.cpp:908-920). */
int hpm_set_canny(hpm_ctx *ctx, int view, const uint8_t *edges, int w, int h);

/* Planar prior of a view: per-pixel prior plane (4 floats, camera frame:
 * n, offset) and mask (HPM::CudaPlanarPriorInitialization HPM.cpp:964-984 /
 * ReloadPlanarPriorInitialization HPM.cpp:1433-1453). */
int hpm_set_prior(hpm_ctx *ctx, int view, const float *planes, const uint8_t *mask, int w, int h);

/* One PatchMatch run of reference view `ref` against `n_src` source views:
 * HPM::RunPatchMatch (HPM.cu:2987-3035) with the hypothesis reload and result
 * hand-off of ProcessProblem (main.cpp:237-634).  params->mode selects the
 * pass; inputs come from the resident maps:
 *   geom:      ref DEPTH (DEPTH_GEOM with MULTIGEOM), NORMAL, COST; sources' same depth kind
 *   hierarchy: ref DEPTH at this level, NORMAL and COST from the coarser level
 *   prior:     ref DEPTH, NORMAL, COST, CONF and the prior set by hpm_set_prior
 *   mandatory: geom inputs plus CONF
 * Outputs: DEPTH (DEPTH_GEOM in geom/mandatory passes), NORMAL, COST and, when
 * neither prior nor mandatory, TEXTURE0 + texture_level.
 * depth_min/max in params are the widened range of HPM.cpp:685-686.  `seed`
 * keys the counter-based random stream of this run. */
int hpm_run_patchmatch(hpm_ctx *ctx, int ref, const int32_t *srcs, int n_src, const hpm_params *params,
                       int texture_level, uint64_t seed);

/* Fixed-hypothesis costs (no reference counterpart: parity entry point).
 * out[k*n_src + j] = bilateral NCC (HPM.cu:375-448) of pixel (px[2k], px[2k+1])
 * under plane k (camera frame) against source j. */
int hpm_eval_costs(hpm_ctx *ctx, int ref, const int32_t *srcs, int n_src, const hpm_params *params, int n,
                   const int32_t *px, const float *planes, float *out);

/* Diagnostic: n linear-filtered fetches of view `view`'s image through the
 * texture unit at unnormalised coordinates xy[2k], xy[2k+1] (tex2D as used by
 * HPM.cu:409).  No reference counterpart: pins the filter model of the tests. */
int hpm_sample_view(hpm_ctx *ctx, int view, int n, const float *xy, float *out);

/* Diagnostic: the first part of a PatchMatch run -- initialisation followed by
 * `n_half_sweeps` black/red half-sweeps, no export -- returning the raw run
 * state (camera-frame planes, costs, view masks, per-pixel draw counters), each
 * w*h of the reference (planes 4 floats per pixel).  No reference counterpart:
 * used for step-by-step parity against the oracle. */
int hpm_debug_run_partial(hpm_ctx *ctx, int ref, const int32_t *srcs, int n_src, const hpm_params *params,
                          int texture_level, uint64_t seed, int n_half_sweeps, float *planes, float *costs,
                          uint32_t *selected_views, uint32_t *draws);

/* Texture address mode of the source images: 0 = clamp (default), 1 = wrap
 * (what HPM.cpp:760-761 requests with unnormalised coordinates). */
int hpm_set_address_mode(hpm_ctx *ctx, int mode);

/* Kernel launches issued by this context since creation (for accounting). */
int64_t hpm_launch_count(const hpm_ctx *ctx);

/* Wait for all work of the context. */
int hpm_synchronize(hpm_ctx *ctx);

#ifdef __cplusplus
}
#endif

#endif /* HPM_CAPI_H */
