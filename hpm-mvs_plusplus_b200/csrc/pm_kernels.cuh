// PatchMatch run arguments and kernel declarations shared by pm_kernels.cu and
// the host-side launcher.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include "hpm_types.h"

namespace hpm {

// Per-view basis of the plane-induced homography H = A - b m^T
// (include/hpm_geometry.h, ComputeHomography HPM.cu:251-311).
struct ViewBasis {
    float A[9];
    float b[3];
};

// Everything one PatchMatch run of one reference view reads.  Passed by value
// as a __grid_constant__ kernel parameter (about 6 KB).
struct RunArgs {
    hpm_camera cams[32];            // 0 = reference
    ViewBasis basis[32];
    ViewBasis fwd[32], bwd[32];     // geometric cost: point transfer reference -> source j+1 and back            // homography basis of source j+1 w.r.t. the reference
    float kinv[4];                  // 1/fx, 1/fy, cx/fx, cy/fy of the reference camera
    float var_s_min;                // flat-source threshold: 1e-5 (HPM.cu:434) in the textures' grey units
    int ncc_shift;                  // 1: shifted NCC moments (precision form); 0: the plain arithmetic
    cudaTextureObject_t tex[32];    // linear-filtered source images (index j+1)
    const float* depth_src[32];     // geometric mode: source depth maps (index j+1)
    int dsw[32], dsh[32];           // their sizes
    const float* ref_img;           // reference grey image (row-major float)
    float4* planes;                 // per-pixel plane hypothesis (n, w)
    float* costs;
    float* pre_costs;
    uint32_t* sel;                  // selected-view bitmask
    uint32_t* rng;                  // per-pixel draw counter
    const float4* prior;            // prior planes (prior mode)
    const uint8_t* pmask;           // prior plane mask (prior mode)
    float* conf;                    // confidences (prior / mandatory)
    const uint8_t* canny;           // 0/255 edge map
    float* texture;                 // edge-density output
    const float4* scaled;           // hierarchy input map (scaled_cols x scaled_rows)
    // prior mode: per colour and row pair, the columns of the pixels a half-sweep updates, compacted
    // to the left (k_prior_active); null: every pixel of the colour is visited and skips itself
    const int* active_px;           // [(colour * cover_pairs + pair) * W + k]
    const int* active_n;            // [colour * cover_pairs + pair]
    hpm_params prm;
    int S, W, H, cover_pairs;
    uint64_t seed;
    uint32_t view_id;
    // profiling only (null otherwise): (hypothesis, source view) pairs costed
    // by [0] the initialisation and [1] the half-sweeps, counted as the
    // reference evaluates them: every hypothesis against all S sources
    // (ComputeMultiViewCostVector, HPM.cu:490-495); [2] the half-sweeps' NCCs
    // that sampled the source (36 filtered fetches each)
    unsigned long long* hyp_count;
};

// Passed by value as a kernel parameter: sm_70 and later accept up to 32764 bytes.
static_assert(sizeof(RunArgs) <= 32764, "RunArgs exceeds the kernel parameter limit");


// Host launchers (pm_kernels.cu).  Return cudaError_t of the launch.
cudaError_t launch_random_init(const RunArgs& a, cudaStream_t st);
cudaError_t launch_half_sweep(const RunArgs& a, int color, int iter, cudaStream_t st);
// Prior mode: the compacted columns of the pixels the half-sweeps update (W * cover_pairs ints and
// cover_pairs counts per colour in px / n), for RunArgs::active_px / active_n.
cudaError_t launch_prior_active(const RunArgs& a, int* px, int* n, cudaStream_t st);
cudaError_t launch_export(const RunArgs& a, cudaStream_t st);
// Fixed-hypothesis costs: out[k*S + j] for pixels px[2k], px[2k+1] and planes[k].
cudaError_t launch_eval_costs(const RunArgs& a, int n, const int32_t* px, const float4* planes, float* out,
                              cudaStream_t st);

// One launch of the batching form over several runs (pm_kernels.cu): the runs'
// RunArgs and the prefix sums of their tile counts (n + 1 entries) in device
// memory.  Tiles are the per-view launches' blocks: 16 x 8 pixels for the
// initialisation, 32 x (block_threads / 32) row pairs for a half-sweep.
struct BatchLaunch {
    const RunArgs* args;
    const int* tile_start;
    int n;            // runs
    int tiles;        // tile_start[n]
    int max_s;        // largest source count (kernel specialisation)
    int grid_blocks;  // 0 or >= tiles: one block per tile; else a persistent grid of this many blocks
    int bx;           // half-sweep block width in pixels (32, 16 or 8); the initialisation uses 16 x 8
    bool mand;        // mandatory-consistency kernel
    bool listed;      // prior mode with work lists (RunArgs::active_px of every run set)
    bool count;       // counting build (hyp_count of every run set)
};

cudaError_t launch_random_init_batch(const BatchLaunch& bl, cudaStream_t st);
cudaError_t launch_half_sweep_batch(const BatchLaunch& bl, int color, int iter, cudaStream_t st);
// Resident blocks per SM of the batched half-sweep kernel, and its block size.
int half_sweep_batch_occupancy(int max_s, bool mand);
int half_sweep_block_threads(int max_s);

// Rows covered by the checkerboard launch of RunPatchMatch (HPM.cu:3004-3011):
// the grid spans ceil(floor(H/2)/16)*16 row pairs.
inline int covered_row_pairs(int H) { return ((H / 2 + 15) / 16) * 16; }

}  // namespace hpm
