// Declarations of the auxiliary kernels (JBU, consistency scan, prior
// construction, image preparation).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include "hpm_types.h"

namespace hpm {

cudaError_t launch_jbu(const float* image, int W, int H, const float* sdepth, int sw, int sh, float* out,
                       cudaStream_t st);
cudaError_t launch_jbu_prior(const float* image, int W, int H, const float* sdepth, const float* snormal, int sw,
                             int sh, float* out_depth, float* out_normal, cudaStream_t st);

// ---- consistency scan (ConfidenceEvaluation / RunFusion) ----------------------------

// Per-view data of a scan (device pointers).
struct ScanView {
    const float* depth;     // H x W
    const float* normal;    // H x W x 3
    const uint8_t* color;   // H x W x 3 BGR (fusion only)
    const uint8_t* sky;     // H x W x 3 BGR sky mask or null
    uint8_t* mask;          // H x W, persistent across the views of one scan
    float* cons;            // H x W working confidence (confidence mode)
    int32_t* marktime;      // H x W first marking pixel of the current view scan
    int32_t* marklast;      // H x W last marking pixel (confidence mode)
    int W, H;
    hpm_camera cam;         // scaled to W x H
};

struct ScanBuffers {
    int32_t* pos;           // npix x n_ngb source pixel index (or -1)
    float* wexp;            // npix x n_ngb exp(-index) of passing pairs
    uint32_t* test;         // npix: bit j = geometric test passed (masks ignored)
    uint32_t* eff;          // npix: bit j = counted (masks applied)
    int32_t* last;          // npix x n_ngb: last pixel <= q whose bit j is counted, or -1
    float* dyn;             // npix
    uint8_t* acc;           // npix: accepted
    int32_t* block_max;     // scan partials
    int* changed;           // device flag
    size_t cap_pix = 0;
};

// mode 0: confidence, 1: fusion.  Scans view `i` against `srcs` (device array of
// ScanView indices).  `views` is a device array of all views.
cudaError_t scan_view_candidates(int mode, const ScanView* views, int i, const int32_t* srcs, int n_ngb,
                                 const ScanBuffers& b, int npix, int W, cudaStream_t st);

}  // namespace hpm
