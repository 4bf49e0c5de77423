// Context object behind the C ABI (hpm_capi.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <utility>
#include <vector>

#include "hpm_capi.h"
#include "pm_kernels.cuh"

namespace hpm {

constexpr int kNumMaps = 16;

// Kinds of the profiling events (hpm_profile): PatchMatch launches and the other stages of hpm_reconstruct.
enum { HPM_STAGE_INIT = 0, HPM_STAGE_SWEEP = 1, HPM_STAGE_CONFIDENCE = 2, HPM_STAGE_PRIOR = 3, HPM_STAGE_JBU = 4,
       HPM_STAGE_FUSION = 5, HPM_STAGE_LEVEL = 6 };

struct DevMap {
    float* ptr = nullptr;
    size_t cap = 0;
    int w = 0, h = 0, ch = 1;
};

struct ViewState {
    int w = 0, h = 0;
    hpm_camera cam{};
    float* gray = nullptr;
    size_t gray_cap = 0;
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
    int arr_w = 0, arr_h = 0, arr_mode = -1, arr_fmt = -1;
    DevMap maps[kNumMaps];
    uint8_t* canny = nullptr;
    size_t canny_cap = 0;
    int canny_w = 0, canny_h = 0;
    float4* prior = nullptr;
    size_t prior_cap = 0;
    uint8_t* pmask = nullptr;
    size_t pmask_cap = 0;
    int prior_w = 0, prior_h = 0;
    uint8_t* orig = nullptr;   // original BGR image (images/%08d.jpg)
    size_t orig_cap = 0;
    int orig_w = 0, orig_h = 0;
    uint8_t* color = nullptr;  // BGR at the map size (fusion colours)
    size_t color_cap = 0;
    int color_w = 0, color_h = 0;
};


struct SrcImages;

// Device buffers of one PatchMatch run: the context's own (single runs) or one
// run's slices of the batch buffers (hpm_run_batch).  scaled == nullptr: the
// hierarchy input goes to the context's own `scaled` buffer.
struct RunBufs {
    float4* planes = nullptr;
    float* costs = nullptr;
    float* pre_costs = nullptr;
    uint32_t* sel = nullptr;
    uint32_t* rng = nullptr;
    float* conf = nullptr;
    float4* scaled = nullptr;
};

// One tuned launch shape of the batched half-sweep (the autotuner's choice).
struct BatchShape {
    int bx = 32;       // block width in pixels (block height = block threads / bx row pairs)
    int persist = 0;   // 0: one block per tile; k > 0: a persistent grid of k x resident blocks
    bool perview = false;  // one launch of the single-view kernel per run and stage (large views)
    float ms = 0.0f;   // measured time of one half-sweep with this shape
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    std::vector<ViewState> views;
    int addr_mode = 0;
    int tex_format = 0;  // HPM_TEX_F32, HPM_TEX_F16 or HPM_TEX_U8: texel type of the source-image textures
    int ncc_mode = 0;    // HPM_NCC_PLAIN or HPM_NCC_SHIFTED
    uint16_t* half_stage = nullptr; size_t half_stage_cap = 0;
    int64_t launches = 0;

    // work buffers of one PatchMatch run (sized for the largest reference view)
    float4* planes = nullptr; size_t run_cap_planes = 0;
    float* costs = nullptr; size_t run_cap_costs = 0;
    float* pre_costs = nullptr; size_t run_cap_pre = 0;
    uint32_t* sel = nullptr; size_t run_cap_sel = 0;
    uint32_t* rng = nullptr; size_t run_cap_rng = 0;
    float* conf = nullptr; size_t run_cap_conf = 0;
    int* active_px = nullptr; size_t active_px_cap = 0;  // prior-mode compaction (k_prior_active)
    int* active_n = nullptr; size_t active_n_cap = 0;
    int* b_active = nullptr; size_t b_active_cap = 0;    // the same for every run of a prior-mode batch
    float4* scaled = nullptr; size_t scaled_cap = 0;
    uint8_t* scratch = nullptr; size_t scratch_cap = 0;
    uint8_t* scan_state = nullptr; size_t scan_state_cap = 0;
    uint8_t* scan_work = nullptr; size_t scan_work_cap = 0;
    hpm_point* points = nullptr; size_t points_cap = 0;
    float* prior_small = nullptr; size_t prior_small_cap = 0;
    uint8_t* prior_tris = nullptr; size_t prior_tris_cap = 0;
    int* prior_label = nullptr; size_t prior_label_cap = 0;
    float* prior_work = nullptr; size_t prior_work_cap = 0;
    float* prior_unormal = nullptr; size_t prior_unormal_cap = 0;
    int* canny_mag = nullptr; size_t canny_mag_cap = 0;
    short2* canny_grad = nullptr; size_t canny_grad_cap = 0;
    uint8_t* canny_state = nullptr; size_t canny_state_cap = 0;
    int64_t n_points = 0;

    // batching form (hpm_run_batch): per-run slices of these buffers, the runs'
    // RunArgs and tile prefix sums in device memory, and the tuned shapes
    float4* b_planes = nullptr; size_t b_cap_planes = 0;
    float* b_costs = nullptr; size_t b_cap_costs = 0;
    float* b_pre = nullptr; size_t b_cap_pre = 0;
    uint32_t* b_sel = nullptr; size_t b_cap_sel = 0;
    uint32_t* b_rng = nullptr; size_t b_cap_rng = 0;
    float* b_conf = nullptr; size_t b_cap_conf = 0;
    float4* b_scaled = nullptr; size_t b_cap_scaled = 0;
    RunArgs* d_bargs = nullptr; size_t d_bargs_cap = 0;
    int* d_btiles = nullptr; size_t d_btiles_cap = 0;    // init tiles (n+1), then sweep tiles (n+1)
    RunArgs* h_bargs = nullptr; size_t h_bargs_cap = 0;  // pinned staging of the RunArgs
    int* h_btiles = nullptr; size_t h_btiles_cap = 0;
    int batch_flags = HPM_BATCH_AUTOTUNE;
    std::vector<std::pair<uint64_t, BatchShape>> batch_shapes;  // autotuner cache: key -> shape
    struct BatchGraph {
        int n = 0, init_tiles = 0, sweep_tiles = 0, max_s = 0, iters = 0, bx = 0, grid = 0;
        bool mand = false, perview = false;
        cudaGraphExec_t exec = nullptr;
    };
    std::vector<BatchGraph> batch_graphs;

    // profiling (hpm_profile_enable): CUDA events around every PatchMatch
    // kernel launch, read back and summed by hpm_profile_read
    int prof_flags = 0;
    struct TimedLaunch { cudaEvent_t start, stop; int kind; };
    std::vector<TimedLaunch> prof_events;  // pool; the first prof_used are pending
    size_t prof_used = 0;
    unsigned long long* prof_hyp = nullptr;  // device counters [init, sweep credited, sweep sampled]
    int record_start(int kind, TimedLaunch*& slot);
    int profile_read(hpm_profile* out);

    ~Ctx();
    int fail(int code, const char* fmt, ...);
    int cuda_fail(cudaError_t e, const char* what);
    cudaError_t ensure_map(int view, int kind, int w, int h);
    cudaError_t ensure_run(size_t n);
    int bind_texture(int view);
    int fill_run_args(int ref, const int32_t* srcs, int n_src, const hpm_params* params, RunArgs& a);
    int prepare_run(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int texture_level,
                    uint64_t seed, RunArgs& a);
    int prepare_run_into(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int texture_level,
                         uint64_t seed, const RunBufs& b, RunArgs& a);
    int finish_run(int ref, const RunArgs& a, bool geom);
    int run_batch(int n, const int32_t* refs, const int32_t* src_off, const int32_t* src_ids,
                  const hpm_params* params, int texture_level, const uint64_t* seeds);
    int tune_batch(const BatchLaunch& bl, int n, size_t total_px, uint64_t key, BatchShape& out);
    int launch_schedule(const RunArgs& a, int n_half_sweeps);
    int debug_run_partial(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int texture_level,
                          uint64_t seed, int n_half_sweeps, float* planes_out, float* costs_out, uint32_t* sel_out,
                          uint32_t* draws_out);
    int sample_view(int view, int n, const float* xy, float* out);
    int run_patchmatch(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int texture_level,
                       uint64_t seed);
    int consistency_scan(int mode, int n_views, const int32_t* src_off, const int32_t* src_ids, int depth_kind,
                         const uint8_t* const* sky_host, hpm_point* out_device, int64_t capacity, int64_t* n_points,
                         int* max_iterations_used);
    int jbu_view(int view, int* applied);
    int prior_downsample(int view, int distance, int& hw, int& hh);
    int support_points(int view, int distance, std::vector<int32_t>& xy, int& sup_w, int& sup_h);
    int prior_from_triangles(int view, int distance, const hpm_triangle* tris, int n_tris, int sup_w, int sup_h);
    int build_prior(int view, int distance, int* n_points, int* n_triangles);
    int prepare_level_image(int view, int w, int h, const hpm_camera& cam);
    int canny_view(int view);
    int reconstruct(int n_views, const hpm_camera* cams, const int32_t* src_off, const int32_t* src_ids,
                    const hpm_recon_options* opt, int64_t* n_points_out);
    cudaError_t ensure_scratch(size_t bytes);
    int fill_src_images(const int32_t* srcs, int n_src, SrcImages& si);
    int eval_cost_grad(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int n, const int32_t* px,
                       const float* theta, float* cost, float* grad);
    int eval_cost_grad_device(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int n,
                              const int32_t* d_px, const float* d_theta, float* d_cost, float* d_grad);
    int gn_refine(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int depth_kind, int steps);
    int eval_costs(int ref, const int32_t* srcs, int n_src, const hpm_params* params, int n, const int32_t* px,
                   const float* planes, float* out);
};

}  // namespace hpm
