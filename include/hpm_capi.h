/*
 * C ABI of libhpm_cuda.so: the drop-in boundary of the HPM-MVS++ depth/normal
 * hot path.
 *
 * The reference exposes this path as the C++ class `HPM` (HPM.h:57-140) plus
 * `RunJBU` (HPM.h:20), `ConfidenceEvaluation` and `RunFusion` (main.cpp:823-1109).
 * Each of those uploads its inputs, runs, downloads and goes through .dmb files
 * on disk.  This ABI keeps every view's images and "dmb maps" resident on the
 * GPU inside one context, so a whole reconstruction schedule runs without
 * host round trips; the host C++ `HPM` class (host/hpm_class.hpp) is rebuilt on top.
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

/* Options of a whole reconstruction (the command line of main.cpp:1143-1181). */
typedef struct hpm_recon_options {
    int32_t initial_image_scale; /* --initial-image-scale N (default 4) */
    int32_t geom_iterations;     /* geometric iterations per level (3, main.cpp:1236) */
    int32_t fuse;                /* run fusion after the last level */
    int32_t level_max_side;      /* 0: 1000, the pyramid bound of ComputeMultiScaleSettings (main.cpp:205);
                                    smaller values build more levels on small inputs */
    int32_t batch;               /* batching form (hpm_run_batch): HPM_RECON_SEQUENTIAL runs the views of a
                                    pass one after another as main.cpp:1253-1255 does; HPM_RECON_BATCH_EXACT
                                    batches every pass whose runs read no map of the same pass (same
                                    result); HPM_RECON_BATCH_ALL also batches the multi-geometry passes,
                                    which then read the previous pass's depth maps (Jacobi) */
    int32_t batch_views;         /* views per batch (0: all views of the pass) */
    uint64_t seed;               /* key of the random streams of all runs */
} hpm_recon_options;

enum { HPM_RECON_SEQUENTIAL = 0, HPM_RECON_BATCH_EXACT = 1, HPM_RECON_BATCH_ALL = 2 };

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

/* Batching form: n PatchMatch runs -- reference view refs[k] against sources
 * src_ids[src_off[k] .. src_off[k+1]) with params[k] and seeds[k] -- in one
 * launch per stage (initialisation, each half-sweep) over all n views.  It
 * replaces the per-view loop of main.cpp:1253-1255 around HPM::RunPatchMatch
 * (HPM.cu:2987-3035), which launches and synchronises one view at a time.
 * Inputs and outputs are those of hpm_run_patchmatch for each run.  Every run
 * reads the resident maps as they were before the call and writes its outputs
 * after all runs have finished, so the result equals n calls of
 * hpm_run_patchmatch in order whenever no run reads a map another run of the
 * batch writes (the photometric, prior, hierarchy and first geometric passes);
 * in multi-geometry passes it is the Jacobi form of the reference's
 * Gauss-Seidel view loop.  All runs share one mode and iteration count; a view
 * appears at most once.  Run buffers for all n views stay resident. */
int hpm_run_batch(hpm_ctx *ctx, int n, const int32_t *refs, const int32_t *src_off, const int32_t *src_ids,
                  const hpm_params *params, int texture_level, const uint64_t *seeds);

/* Options of hpm_run_batch (bit set; default HPM_BATCH_AUTOTUNE):
 *   HPM_BATCH_AUTOTUNE    the first batch of each (source count, mode, size class)
 *                         times the candidate launch shapes of the half-sweep (block
 *                         width 32, 16 or 8 pixels; one block per tile or a persistent
 *                         grid; or one single-view launch per run) on a copy of its
 *                         state and keeps the fastest; results do not depend on the shape
 *   HPM_BATCH_GRAPH       the initialisation and half-sweeps of a batch are captured once
 *                         per batch shape in a CUDA graph and replayed (not for the
 *                         single-view shape)
 *   HPM_BATCH_PER_VIEW    the half-sweeps use the single-view shape without tuning */
#define HPM_BATCH_AUTOTUNE 1
#define HPM_BATCH_GRAPH 2
#define HPM_BATCH_PER_VIEW 4
int hpm_set_batch_options(hpm_ctx *ctx, int flags);

/* Fixed-hypothesis costs (no reference counterpart: parity entry point).
 * out[k*n_src + j] = bilateral NCC (HPM.cu:375-448) of pixel (px[2k], px[2k+1])
 * under plane k (camera frame) against source j. */
int hpm_eval_costs(hpm_ctx *ctx, int ref, const int32_t *srcs, int n_src, const hpm_params *params, int n,
                   const int32_t *px, const float *planes, float *out);

/* hpm_eval_costs without any device allocation.  No counterpart in the
 * reference.  For callers that must not have cudaMalloc/cudaFree run under them
 * (those calls can synchronise the whole device and can fail when the process's
 * device memory is owned by another allocator with a fixed budget).  Same
 * arguments and results as hpm_eval_costs; the device staging lives in one
 * fixed 4 MiB array per GPU, so n * (24 + 4 * n_src) bytes (plus alignment)
 * must fit, else HPM_E_INVALID.  All calls on a device share that array: calls
 * that overlap on the GPU race.  The first call on a device looks up the
 * array's address; make it before any stream capture. */
int hpm_eval_costs_noalloc(hpm_ctx *ctx, int ref, const int32_t *srcs, int n_src, const hpm_params *params, int n,
                           const int32_t *px, const float *planes, float *out);

/* Differentiable form of the bilateral NCC (HPM.cu:375-448 with exact
 * bilinear sampling of the sources) and its adjoint; no counterpart in the
 * reference.  For n (pixel, hypothesis) pairs, theta[3k..3k+2] = (depth, nx,
 * ny) in the reference camera frame with nz = -sqrt(1 - nx^2 - ny^2):
 * cost[k*n_src + j] and, when grad is not null, grad[(k*n_src + j)*3 + a] =
 * d cost / d theta_a.  Costs of 2 (out-of-image centre, flat patch) and
 * clamped costs have zero gradient.  The warped samples are recomputed, not
 * stored. */
int hpm_eval_cost_grad(hpm_ctx *ctx, int ref, const int32_t *srcs, int n_src, const hpm_params *params, int n,
                       const int32_t *px, const float *theta, float *cost, float *grad);

/* hpm_eval_cost_grad on device buffers: px, theta, cost and grad are device
 * pointers of the context's GPU, read and written on the context's stream
 * (hpm_get_stream); the caller orders its own producers before the call.  The
 * call returns when the kernel has finished.  A pixel outside the reference
 * image is skipped and the call returns HPM_E_INVALID. */
int hpm_eval_cost_grad_device(hpm_ctx *ctx, int ref, const int32_t *srcs, int n_src, const hpm_params *params, int n,
                              const int32_t *d_px, const float *d_theta, float *d_cost, float *d_grad);

/* Gauss-Newton refinement of a view's resident planes (no counterpart in the
 * reference, where refinement is PlaneHypothesisRefinement's random
 * perturbations, HPM.cu:765-841): `steps` damped Gauss-Newton steps per pixel
 * on the sum of squared costs of hpm_eval_cost_grad over the sources whose
 * cost starts in (0, 2), updating the view's `depth_kind` (DEPTH or
 * DEPTH_GEOM) and NORMAL maps in place and writing the RMS cost to COST.
 * Depths stay in params' [depth_min, depth_max]. */
int hpm_gn_refine(hpm_ctx *ctx, int ref, const int32_t *srcs, int n_src, const hpm_params *params, int depth_kind,
                  int steps);

/* Colour image (BGR, 8 bits) of a view at the size of its maps, for the point
 * colours of fusion (the rescaled image of RunFusion, main.cpp:863-865). */
int hpm_set_color(hpm_ctx *ctx, int view, const uint8_t *bgr, int w, int h);

/* RunJBU (HPM.cpp:1266-1319) + JointBilateralUpsampling (main.cpp:636-657):
 * the view's coarser DEPTH_GEOM map upsampled, guided by the view's grey image,
 * into its DEPTH map at the image size.  *applied = 0 and nothing is written
 * when the integer scale is 1 (HPM.cpp:1272-1275). */
int hpm_jbu(hpm_ctx *ctx, int view, int *applied);

/* JBU_cu / JBU_cu_prior (HPM.cu:3037-3197) on host buffers: src_depth (sw x sh)
 * and, when src_normal (3 floats/px) is given, normals, upsampled to the view's
 * image size guided by its grey image.  Without normals the NaN fallback of
 * RunJBU (HPM.cpp:1297-1300) applies. */
int hpm_jbu_maps(hpm_ctx *ctx, int view, const float *src_depth, const float *src_normal, int sw, int sh,
                 float *out_depth, float *out_normal);

/* ConfidenceEvaluation (main.cpp:959-1109) over views 0..n_views-1 (view id ==
 * index, as the reference assumes): reads each view's depth map of
 * `depth_kind` (DEPTH or DEPTH_GEOM) and NORMAL, with the view's camera scaled
 * to the map size; writes each view's CONF map.  Source lists are
 * src_ids[src_off[i] .. src_off[i+1]).  *iterations receives the largest
 * number of fixed-point iterations a view needed. */
int hpm_confidence_eval(hpm_ctx *ctx, int n_views, const int32_t *src_off, const int32_t *src_ids, int depth_kind,
                        int *iterations);

/* RunFusion (main.cpp:823-957), or RunFusion_Sky_Strict (main.cpp:659-821) when
 * sky_masks (per view, BGR at the map size) is given.  Points in the
 * reference's order; up to `capacity` are copied to `out`, the total count goes
 * to *n_points.  Colours come from hpm_set_color. */
int hpm_fuse(hpm_ctx *ctx, int n_views, const int32_t *src_off, const int32_t *src_ids, int depth_kind,
             const uint8_t *const *sky_masks, hpm_point *out, int64_t capacity, int64_t *n_points);

/* Support points of the planar prior (GetSupportPoints_Classify_Check,
 * HPM.cpp:1026-1073) from the view's COST and CONF maps; with distance 1 or 2
 * the maps are first downsampled by 1/(2*distance) (main.cpp:444-454).  Up to
 * `capacity` (x, y) pairs are written, *n gets the count, *w x *h the size of
 * the rectangle they live in. */
int hpm_support_points(hpm_ctx *ctx, int view, int distance, int32_t *xy, int capacity, int *n, int *w, int *h);

/* Delaunay triangulation of integer points inside [0,w)x[0,h) (the role of
 * cv::Subdiv2D in HPM::DelaunayTriangulation, HPM.cpp:1075-1097).  Host only;
 * duplicate points are ignored. */
int hpm_delaunay(const int32_t *xy, int n, int w, int h, hpm_triangle *out, int capacity, int *n_out);

/* Planar prior of a view from a triangle list: raster (main.cpp:389-409),
 * 3-point plane fits in double (HPM.cpp:1099-1167), prior depth mask and, for
 * distance 1 or 2, prior JBU and reload (main.cpp:443-576).  The result is the
 * prior hpm_run_patchmatch uses in prior mode. */
int hpm_prior_from_triangles(hpm_ctx *ctx, int view, int distance, const hpm_triangle *tris, int n_tris);

/* Support points -> Delaunay -> hpm_prior_from_triangles in one call. */
int hpm_build_prior(hpm_ctx *ctx, int view, int distance, int *n_points, int *n_triangles);

/* Download a view's prior: planes (4 floats per pixel) and mask (0/1). */
int hpm_get_prior(hpm_ctx *ctx, int view, float *planes, uint8_t *mask);

/* Original BGR image of a view (what images/%08d.jpg decodes to). */
int hpm_set_image(hpm_ctx *ctx, int view, const uint8_t *bgr, int w, int h);

/* Builds a view's pyramid-level image from its original: cv::resize INTER_LINEAR
 * to w x h (PrepareScaleImages, main.cpp:107-161), BGR->grey as float
 * (HPM.cpp:658-662), the level colour for fusion, and the Canny(50, 150) edge
 * map (main.cpp:287).  `cam` is the camera scaled to w x h. */
int hpm_prepare_level(hpm_ctx *ctx, int view, int w, int h, const hpm_camera *cam);

/* Download a view's level image: BGR (w*h*3) and/or Canny edges (w*h). */
int hpm_get_level(hpm_ctx *ctx, int view, uint8_t *bgr, float *gray, uint8_t *edges);

/* The whole HPM-MVS++ schedule of main.cpp:1183-1359 on resident data: for
 * views 0..n_views-1 with original images set by hpm_set_image and original
 * cameras `cams` (as read from cams/%08d_cam.txt), source lists
 * src_ids[src_off[i]..src_off[i+1]): pyramid levels, photometric, prior,
 * hierarchy and geometric PatchMatch passes, JBU, confidence evaluations and
 * (opt->fuse) fusion.  Final maps stay resident (DEPTH_GEOM, NORMAL, ...);
 * points are read with hpm_get_points.  *n_points gets the fused count. */
int hpm_reconstruct(hpm_ctx *ctx, int n_views, const hpm_camera *cams, const int32_t *src_off,
                    const int32_t *src_ids, const hpm_recon_options *opt, int64_t *n_points);

/* Copy up to `capacity` fused points of the last hpm_reconstruct / hpm_fuse. */
int hpm_get_points(hpm_ctx *ctx, hpm_point *out, int64_t capacity, int64_t *n_points);

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

/* Texel type of the source-image textures bound from now on (hpm_set_view,
 * hpm_prepare_level): HPM_TEX_F32 (default, the reference's float textures,
 * HPM.cpp:750-768) or HPM_TEX_F16, the precision form: half the bytes through
 * the texture path.  The 8-bit grey levels are stored exactly, but the
 * filtered sample comes back rounded to half precision (within 1/16 of a grey
 * level), so F16 results are close to, not equal to, F32 results. */
#define HPM_TEX_F32 0
#define HPM_TEX_F16 1
#define HPM_TEX_U8 2  /* 8-bit texels read as grey/255; the NCC is scale-free, its flat-source test is rescaled */
int hpm_set_texture_format(hpm_ctx *ctx, int format);

/* Arithmetic of the bilateral NCC moments (HPM.cu:375-448) from now on:
 * HPM_NCC_PLAIN (default) forms the variances as E[x^2] - E[x]^2 as the
 * reference does; HPM_NCC_SHIFTED, the precision form, accumulates the
 * reference patch relative to its centre texel and each source patch relative
 * to its first sample, so that flat (textureless) patches keep their variance
 * instead of losing it to cancellation.  The NCC is shift-invariant: the two
 * differ only by rounding, which the shifted form makes smaller. */
#define HPM_NCC_PLAIN 0
#define HPM_NCC_SHIFTED 1
int hpm_set_ncc_mode(hpm_ctx *ctx, int mode);

/* Kernel launches issued by this context since creation (for accounting). */
int64_t hpm_launch_count(const hpm_ctx *ctx);

/* Wait for all work of the context. */
int hpm_synchronize(hpm_ctx *ctx);

/* ---- measurement (no reference counterpart; the reference has only its
 * wall-clock timer, main.cpp:10-23) ---- */

/* The CUDA stream all work of the context is issued on (a cudaStream_t), so a
 * caller can record its own events around calls. */
int hpm_get_stream(hpm_ctx *ctx, void **stream);

#define HPM_PROFILE_TIMING 1 /* CUDA events around every PatchMatch kernel launch */
#define HPM_PROFILE_COUNT 2  /* count (hypothesis, source view) cost evaluations */

typedef struct hpm_profile {
    int64_t init_launches;     /* random-initialisation launches timed */
    int64_t sweep_launches;    /* black/red half-sweep launches timed */
    double init_ms;            /* their summed device time */
    double sweep_ms;
    uint64_t init_view_evals;  /* (hypothesis, source view) pairs costed, each 36 patch samples, */
    uint64_t sweep_view_evals; /*   every hypothesis against all S sources as the reference does */
    uint64_t sweep_sampled;    /* (hypothesis, source view) NCCs of the half-sweeps that sampled the source
                                  (36 filtered fetches each): the credited ones minus those skipped for a
                                  zero view weight, an out-of-image centre or a flat reference patch */
    double confidence_ms;      /* device time of hpm_reconstruct's other stages: ConfidenceEvaluation, */
    double prior_ms;           /*   prior construction (support points, raster, fits, reload; the host */
    double jbu_ms;             /*   Delaunay triangulations overlap it and are not included), JBU and */
    double fusion_ms;          /*   fusion */
    double level_ms;           /* device time of the level images: resize, grey conversion, Canny */
} hpm_profile;

/* Turns profiling on (flags) or off (0).  Timing adds two event records per
 * launch; counting adds one atomic per costed hypothesis. */
int hpm_profile_enable(hpm_ctx *ctx, int flags);

/* Waits for the context's work, returns what was gathered since the last read
 * and resets it. */
int hpm_profile_read(hpm_ctx *ctx, hpm_profile *out);

/* FP32 FMA throughput of the device in TFLOP/s (2 flops per FMA), from a
 * dependent-chain kernel over all SMs timed with CUDA events. */
int hpm_measure_fp32_peak(int device, double *tflops);

/* Linear-filtered texture fetches per second (in units of 1e9) of the device
 * for source textures of `format` (HPM_TEX_F32, HPM_TEX_F16 or HPM_TEX_U8),
 * from fetches in the half-sweep's access pattern timed with CUDA events: the
 * roof of the NCC sampling, which issues one filtered fetch per patch sample. */
int hpm_measure_tex_peak(int device, int format, double *gsamples);

/* hpm_measure_tex_peak with the lanes of a warp apart: every lane's patch is
 * moved by its own offset, uniform in [-jitter, jitter] pixels per axis
 * (0 <= jitter <= 64) and redrawn for every six fetches, as when neighbouring
 * pixels sample under different planes.  jitter = 0 is hpm_measure_tex_peak. */
int hpm_measure_tex_rate(int device, int format, float jitter, double *gsamples);

#ifdef __cplusplus
}
#endif

#endif /* HPM_CAPI_H */
