/*
 * CPU ORACLE -- test infrastructure only.
 *
 * A plain-C restatement of the HPM-MVS++ depth/normal hot path, written from
 * the reference sources (HPM.cu, HPM.cpp, main.cpp; every function cites the
 * lines it restates).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline legs load it, and only as the checker: the product never calls it.
 *
 * Pinning: the reference ships no tests, golden vectors or fixtures for this
 * path.  The oracle is pinned against the reference's own CUDA code built from
 * source (oracle/ref_build.mk -> oracle/_ref/libhpmref.so): function by
 * function through golden vectors of its __device__ functions
 * (tests/golden/ref_probe.npz, checked on the CPU by tests/test_golden_ref.py),
 * whole runs statistically on a B200 (tests/test_ref_build.py), and against
 * the hand-derived known-answer cases in tests/test_oracle.py.
 *
 * Conventions shared with the CUDA path:
 *  - images are row-major float32 grey levels (0..255), index y*width + x;
 *  - planes are float4 (nx, ny, nz, w) in the reference camera frame during a
 *    run, (world normal, depth) after the export step (HPM.cu:2829-2842);
 *  - random draws come from include/hpm_philox.h with one 32-bit draw counter
 *    per pixel (reset to 0 by the init kernel, as curand_init is, HPM.cu:579);
 *  - texture fetches follow the linear filter of the B200 texture unit with
 *    clamp addressing (ora_tex2d; measured by tests/test_gpu_parity.py).
 *
 * Where the reference reads uninitialised memory this oracle and the CUDA path
 * use the same defined value:
 *  - plane_hypotheses_now (HPM.cu:1844, 2299, 2761) holds the best valid
 *    neighbour's plane (minimum cost; maximum score in prior mode and for
 *    unreliable mandatory pixels), as the compiled reference does, else the
 *    pixel's current plane;
 *  - the hierarchy pre-cost plane (HPM.cpp:894-901 leaves xyz unset) has a zero
 *    normal;
 *  - selected_views starts at zero at every run (fresh cudaMalloc, HPM.cpp:782).
 */
#ifndef HPM_ORACLE_H
#define HPM_ORACLE_H

#include <stdint.h>
#include "hpm_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Per-run state of one reference view (all arrays width*height of the reference). */
typedef struct ora_state {
    float *planes;           /* 4 floats per pixel */
    float *costs;
    float *pre_costs;        /* hierarchy only */
    uint32_t *selected_views;
    uint32_t *rng_draw;      /* per-pixel draw counter */
    const float *prior_planes; /* 4 floats per pixel, prior mode */
    const uint32_t *plane_masks; /* prior mode */
    float *confidences;      /* prior / mandatory modes */
    const uint8_t *canny;    /* 0 / 255 edge map */
    float *texture;          /* written when neither prior nor mandatory */
    const float *scaled_planes; /* hierarchy: scaled_rows*scaled_cols float4 */
} ora_state;

/* Texture filter model: 0 = as measured on B200 (8-bit weights and 8-bit cross
 * weight), 1 = separable 8-bit weights of the CUDA Programming Guide. */
void ora_set_texture_model(int model);
/* Shifted-moment NCC of the precision form (0: plain arithmetic). */
void ora_set_ncc_shift(int on);
/* The bilateral NCC of ora_bilateral_ncc's own samples with its moments in double. */
double ora_bilateral_ncc64(const float *ref, const hpm_camera *ref_cam, const float *src, const hpm_camera *src_cam,
                           int px, int py, const float plane[4], const hpm_params *prm);
int ora_get_texture_model(void);
float ora_tex2d(const float *img, int width, int height, float x, float y);

/* Bilateral NCC of one (pixel, plane, source view) (HPM.cu:375-448). */
float ora_bilateral_ncc(const float *ref, const hpm_camera *ref_cam,
                        const float *src, const hpm_camera *src_cam,
                        int px, int py, const float plane[4], const hpm_params *params);

/* Fixed-hypothesis mode: out[k*S + j] = NCC of (px[2k], px[2k+1]) under plane k
 * against source view j+1.  images[0] is the reference view. */
void ora_eval_costs(const float *const *images, const hpm_camera *cams, int num_images,
                    const hpm_params *params, int n, const int32_t *px, const float *planes,
                    float *out);

/* Geometric consistency cost (HPM.cu:539-564) of plane at (px,py) against the
 * source depth map `src_depth` (src_cam.height x src_cam.width). */
float ora_geom_cost(const float *src_depth, const hpm_camera *ref_cam, const hpm_camera *src_cam,
                    const float plane[4], int px, int py);

/* Depth of a camera-frame plane at pixel (px, py) (ComputeDepthfromPlaneHypothesis, HPM.cu:154-157). */
float ora_depth_from_plane(const hpm_camera *cam, const float plane[4], int px, int py);

/* Multi-view initial cost and view mask (HPM.cu:450-488). */
float ora_initial_cost(const float *const *images, const hpm_camera *cams, int num_images,
                       const hpm_params *params, int px, int py, const float plane[4],
                       uint32_t *selected);

/* Edge-density texture term (HPM.cu:349-373). */
float ora_texture(const uint8_t *canny, int width, int height, int px, int py);

/* RandomInitialization (HPM.cu:567-763). */
void ora_random_init(const float *const *images, const hpm_camera *cams, int num_images,
                     const hpm_params *params, ora_state *st, uint64_t seed, uint32_t view_id);

/* One Black (color 0) or Red (color 1) half-sweep (HPM.cu:2793-2827). */
void ora_half_sweep(const float *const *images, const float *const *depths,
                    const hpm_camera *cams, int num_images, const hpm_params *params,
                    ora_state *st, int color, int iter, uint64_t seed, uint32_t view_id);

/* GetDepthandNormal (HPM.cu:2829-2842). */
void ora_export(const hpm_camera *ref_cam, float *planes);

/* RunPatchMatch (HPM.cu:2987-3035): init, iterations x (black, red), export. */
void ora_run_patchmatch(const float *const *images, const float *const *depths,
                        const hpm_camera *cams, int num_images, const hpm_params *params,
                        ora_state *st, uint64_t seed, uint32_t view_id);

/* JBU_cu (HPM.cu:3037-3095) + the NaN fallback of RunJBU (HPM.cpp:1294-1303). */
void ora_jbu(const float *image, int width, int height, const float *src_depth,
             int s_width, int s_height, float *out_depth);

/* JBU_cu_prior (HPM.cu:3130-3197) + JointBilateralUpsampling_prior (HPM.cpp:1323-1392):
 * out_depth (w*h), out_normal (3 floats per pixel). src_normal has 3 floats/px. */
void ora_jbu_prior(const float *image, int width, int height, const float *src_depth,
                   const float *src_normal, int s_width, int s_height,
                   float *out_depth, float *out_normal);

/* ---- host stages (main.cpp / HPM.cpp) ---- */

/* ConfidenceEvaluation (main.cpp:959-1109) over all views at once.
 * depths[i], normals[i] (3 floats/px) have size cams[i].height x cams[i].width
 * (cams already rescaled to the depth-map size).  src lists are concatenated in
 * src_ids with offsets src_off[i]..src_off[i+1].  conf_out[i] receives view i's
 * confidence map as written to confidence.dmb. */
void ora_confidence_eval(int num_views, const hpm_camera *cams, const float *const *depths,
                         const float *const *normals, const int32_t *src_off,
                         const int32_t *src_ids, float *const *conf_out);

/* RunFusion (main.cpp:823-957); with sky_masks != NULL, RunFusion_Sky_Strict
 * (main.cpp:659-821).  colors[i] is BGR uint8 at the depth-map size.  Returns
 * the number of points written (at most max_points) and the total count in
 * *n_total. */
int64_t ora_fusion(int num_views, const hpm_camera *cams, const float *const *depths,
                   const float *const *normals, const uint8_t *const *colors,
                   const uint8_t *const *sky_masks, const int32_t *src_off,
                   const int32_t *src_ids, hpm_point *out, int64_t max_points,
                   int64_t *n_total);

/* GetSupportPoints_Classify_Check (HPM.cpp:1026-1073). Returns the number of
 * points (x, y pairs in out_xy, capacity max_points). costs/conf are w x h,
 * texture has tex_w columns. */
int32_t ora_support_points(const float *costs, const float *conf, const float *texture,
                           int tex_w, int width, int height, int32_t *out_xy, int32_t max_points);

/* Triangle raster of main.cpp:389-409 (labels idx+1 as float, later
 * triangles overwrite) + plane fits (HPM.cpp:1099-1167, `factor` = 1 gives the
 * unscaled variant) + prior depth mask (main.cpp:411-424 when mode 0;
 * main.cpp:516-535 when mode 1).  Only triangles with all vertices inside
 * [0,width)x[0,height) are labelled.  planes_out receives 4 floats per
 * accepted triangle; mask_out (width*height float labels); prior_depth_out and,
 * in mode 1, prior_normal_out (world frame, 3 floats/px).  Returns the number
 * of accepted triangles. */
int32_t ora_planar_prior(const hpm_triangle *tris, int32_t n_tris, const float *depths,
                         int width, int height, const hpm_camera *ref_cam, float factor,
                         float depth_min, float depth_max, int mode,
                         float *mask_out, float *planes_out, float *prior_depth_out,
                         float *prior_normal_out);

/* Reload of an upsampled prior (main.cpp:548-570): camera-frame planes and mask. */
void ora_prior_reload(const float *udepth, const float *unormal, int W, int H, const hpm_camera *c, float dmin,
                      float dmax, float *prior, uint8_t *mask);

/* Philox4x32-10 block and uniform draw of include/hpm_philox.h. */
void ora_philox(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]);
float ora_uniform(uint64_t seed, uint32_t view, uint32_t x, uint32_t y, uint32_t draw);

/* cv::resize INTER_LINEAR for a single-channel float image. */
void ora_resize_linear_f32(const float *src, int sw, int sh, float *dst, int dw, int dh);

/* FP64 differentiable bilateral NCC of pixel (px, py) under the camera-frame
 * plane theta = (depth, nx, ny), nz = -sqrt(1 - nx^2 - ny^2), against one
 * source view (exact bilinear sampling); returns the cost and, when grad is
 * not null, d cost / d theta (hpm_oracle_grad.c). */
double ora_cost_grad64(const float *ref, const hpm_camera *rc, const float *src, const hpm_camera *sc,
                       const hpm_params *prm, int px, int py, const double theta[3], double grad[3]);

#ifdef __cplusplus
}
#endif

#endif /* HPM_ORACLE_H */
