/*
 * Plain-old-data types shared by the C ABI (hpm_capi.h), the CUDA kernels and
 * the CPU oracle.  Layouts are fixed: every field is 4 bytes, no padding.
 *
 * hpm_camera  mirrors `struct Camera` of HPM-MVS++ (main.h:39-47) byte for byte:
 *             K[9], R[9], t[3] (world->camera: x_cam = R x_world + t),
 *             height, width, depth_min, depth_max  -> 100 bytes.
 * hpm_params  carries the fields of `PatchMatchParams` (HPM.h:32-55) that the
 *             hot path reads, as ints/floats so the struct is ABI stable.
 */
#ifndef HPM_TYPES_H
#define HPM_TYPES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hpm_camera {
    float K[9];
    float R[9];
    float t[3];
    int32_t height;
    int32_t width;
    float depth_min;
    float depth_max;
} hpm_camera;

/* Mode bits of one PatchMatch run (the bools of PatchMatchParams, HPM.h:49-54). */
enum {
    HPM_MODE_GEOM      = 1u << 0, /* geom_consistency  */
    HPM_MODE_PRIOR     = 1u << 1, /* prior_consistency */
    HPM_MODE_MULTIGEOM = 1u << 2, /* multi_geometry (which depth file a geom pass reads) */
    HPM_MODE_HIERARCHY = 1u << 3, /* hierarchy         */
    HPM_MODE_UPSAMPLE  = 1u << 4, /* upsample (hierarchy with a coarser hypothesis map) */
    HPM_MODE_MAND      = 1u << 5  /* mand_consistency  */
};

typedef struct hpm_params {
    int32_t max_iterations;   /* red/black iterations; RunPatchMatch hard-codes 3 (HPM.cu:3013) */
    int32_t patch_size;       /* 11 */
    int32_t num_images;       /* 1 + number of source views (<= 32) */
    int32_t radius_increment; /* 2  */
    float   sigma_spatial;    /* 5  */
    float   sigma_color;      /* 3  */
    int32_t top_k;            /* 4  */
    float   depth_min;        /* 0.6 * cam.depth_min (HPM.cpp:685) */
    float   depth_max;        /* 1.2 * cam.depth_max (HPM.cpp:686) */
    int32_t scaled_cols;      /* width of the coarser hypothesis map (upsample mode) */
    int32_t scaled_rows;      /* height of the coarser hypothesis map (upsample mode) */
    uint32_t mode;            /* HPM_MODE_* bits */
} hpm_params;

/* One fused point: PointList of main.h:92-96 (world xyz, world normal, BGR colour). */
typedef struct hpm_point {
    float coord[3];
    float normal[3];
    float color[3];
} hpm_point;

/* Triangle with integer vertices (struct Triangle, main.h:86-90). */
typedef struct hpm_triangle {
    int32_t x1, y1, x2, y2, x3, y3;
} hpm_triangle;

#define HPM_MAX_SRC 31      /* 32-bit view masks and cost_vector[32] (HPM.cu:453) cap S at 31 */
#define HPM_MAX_VIEWS 256   /* MAX_IMAGES (main.h:36) */

/* Seed of the PatchMatch run of `view` in pass `pass` of a reconstruction
 * keyed by `base` (a splitmix64-style mix): hpm_reconstruct uses it with
 * passes counted from 1 in schedule order, so a caller that drives the same
 * schedule run by run draws the same random streams. */
static inline uint64_t hpm_run_seed(uint64_t base, uint64_t pass, uint64_t view)
{
    uint64_t z = base ^ (pass * 0x9E3779B97F4A7C15ULL) ^ (view * 0xBF58476D1CE4E5B9ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

#ifdef __cplusplus
}
#endif

#endif /* HPM_TYPES_H */
