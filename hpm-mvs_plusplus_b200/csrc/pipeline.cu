// The reconstruction schedule of HPM-MVS++ main() (main.cpp:1183-1359) on
// resident GPU data.  Where the reference hands every stage's result to the
// next through .dmb files, the passes here read and write the per-view maps of
// the context; the order of passes and of views inside a pass is the
// reference's, so the geometric iterations that read neighbours' depths_geom
// maps rewritten earlier in the same pass see the same (Gauss-Seidel) state.
#include "ctx.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <future>
#include <thread>
#include <vector>

namespace hpm {

int delaunay_triangulate(const int32_t* xy, int n, int width, int height, std::vector<hpm_triangle>& out);

int Ctx::reconstruct(int n_views, const hpm_camera* cams, const int32_t* src_off, const int32_t* src_ids,
                     const hpm_recon_options* opt, int64_t* n_points_out) {
    cudaSetDevice(device);
    if (n_views < 1 || n_views > HPM_MAX_VIEWS || !cams || !src_off || !src_ids || !opt)
        return fail(HPM_E_INVALID, "hpm_reconstruct: bad arguments");
    if (opt->initial_image_scale < 1) return fail(HPM_E_INVALID, "--initial-image-scale must be at least 1");
    for (int i = 0; i < n_views; ++i) {
        if (!views[i].orig || views[i].orig_w <= 0) return fail(HPM_E_STATE, "view %d has no image", i);
        const int ns = src_off[i + 1] - src_off[i];
        if (ns < 1 || ns > HPM_MAX_SRC) return fail(HPM_E_INVALID, "view %d has %d sources (1..31)", i, ns);
    }
    const int scale = opt->initial_image_scale;
    const int geom_iterations = opt->geom_iterations > 0 ? opt->geom_iterations : 3;
    const int size_bound = opt->level_max_side > 0 ? opt->level_max_side : 1000;

    // ComputeMultiScaleSettings (main.cpp:202-235)
    std::vector<int> initial_max_side(n_views), num_downscale(n_views), cur_max_side(n_views, 0);
    int max_num_downscale = -1;
    for (int i = 0; i < n_views; ++i) {
        const int original = std::max(views[i].orig_w, views[i].orig_h);
        initial_max_side[i] = std::max(1, (original + scale / 2) / scale);
        int k = 0, side = initial_max_side[i];
        while (side > size_bound) { side /= 2; ++k; }
        num_downscale[i] = k;
        max_num_downscale = std::max(max_num_downscale, k);
    }
    const int max_hpm_scale = max_num_downscale;
    std::vector<int> ids(n_views);
    for (int i = 0; i < n_views; ++i) ids[i] = i;
    int pass = 0;
    int rc = HPM_OK;

    if (opt->batch < HPM_RECON_SEQUENTIAL || opt->batch > HPM_RECON_BATCH_ALL || opt->batch_views < 0)
        return fail(HPM_E_INVALID, "hpm_reconstruct: bad batch options");
    auto make_params = [&](int i, uint32_t mode) -> hpm_params {
        const hpm_camera& c = views[i].cam;
        hpm_params p;
        p.max_iterations = 3;  // RunPatchMatch hard-codes 3 (HPM.cu:3013)
        p.patch_size = 11;
        p.radius_increment = 2;
        p.sigma_spatial = 5.0f;
        p.sigma_color = 3.0f;
        p.top_k = 4;
        p.depth_min = c.depth_min * 0.6f;
        p.depth_max = c.depth_max * 1.2f;
        p.num_images = src_off[i + 1] - src_off[i] + 1;
        p.scaled_cols = 0;
        p.scaled_rows = 0;
        p.mode = mode;
        return p;
    };
    auto run = [&](int i, uint32_t mode, int texture_level) -> int {
        const hpm_params p = make_params(i, mode);
        return run_patchmatch(i, src_ids + src_off[i], p.num_images - 1, &p, texture_level,
                              hpm_run_seed(opt->seed, (uint64_t)pass, (uint64_t)i));
    };
    // views [first, last) of a pass in one hpm_run_batch: same seeds and inputs as their single runs
    auto run_group = [&](int first, int last, uint32_t mode, int texture_level) -> int {
        std::vector<int32_t> refs, off(1, 0), ids;
        std::vector<hpm_params> prm;
        std::vector<uint64_t> seeds;
        for (int i = first; i < last; ++i) {
            refs.push_back(i);
            ids.insert(ids.end(), src_ids + src_off[i], src_ids + src_off[i + 1]);
            off.push_back((int32_t)ids.size());
            prm.push_back(make_params(i, mode));
            seeds.push_back(hpm_run_seed(opt->seed, (uint64_t)pass, (uint64_t)i));
        }
        return run_batch((int)refs.size(), refs.data(), off.data(), ids.data(), prm.data(), texture_level,
                         seeds.data());
    };
    // a whole pass: batched when the options allow it for this mode, else view by view in order
    const int group = opt->batch_views > 0 ? opt->batch_views : n_views;
    auto run_pass = [&](uint32_t mode, int texture_level) -> int {
        const bool jacobi = mode & HPM_MODE_MULTIGEOM;  // reads depths_geom maps the same pass writes
        const bool batched = opt->batch == HPM_RECON_BATCH_ALL || (opt->batch == HPM_RECON_BATCH_EXACT && !jacobi);
        for (int i = 0; i < n_views; i += batched ? group : 1) {
            const int r = batched ? run_group(i, std::min(n_views, i + group), mode, texture_level)
                                  : run(i, mode, texture_level);
            if (r) return r;
        }
        return HPM_OK;
    };
    // device time of the non-PatchMatch stages, when profiling is on (hpm_profile)
    auto timed = [&](int kind, auto&& fn) -> int {
        TimedLaunch* t = nullptr;
        int r = record_start(kind, t);
        if (r) return r;
        r = fn();
        if (t) cudaEventRecord(t->stop, stream);
        return r;
    };
    auto confidence = [&](int depth_kind) -> int {
        return timed(HPM_STAGE_CONFIDENCE, [&]() {
            return consistency_scan(0, n_views, src_off, src_ids, depth_kind, nullptr, nullptr, 0, nullptr, nullptr);
        });
    };
    // A view's prior depends only on its own maps and the confidences computed
    // before the pass, so all support points are taken first and the host
    // triangulations run on worker threads while the GPU works through the
    // views in order (view i's PatchMatch overlaps the triangulation of later
    // views).  The results are those of one view at a time.
    auto prior_passes = [&](int level) -> int {
        for (int hpm_scale = max_hpm_scale; hpm_scale >= level; --hpm_scale) {
            int r = confidence(HPM_MAP_DEPTH);
            if (r) return r;
            ++pass;
            std::vector<std::vector<int32_t>> xy(n_views);
            std::vector<int> sup_w(n_views), sup_h(n_views), dist(n_views);
            for (int i = 0; i < n_views; ++i) {
                dist[i] = hpm_scale - num_downscale[i] - 1;
                if (dist[i] < 0 || dist[i] > 2)
                    return fail(HPM_E_STATE, "view %d: prior scale distance %d is outside 0..2", i, dist[i]);
                if (!views[i].maps[HPM_MAP_DEPTH].ptr) return fail(HPM_E_STATE, "view %d lacks a depth map", i);
                r = timed(HPM_STAGE_PRIOR, [&]() { return support_points(i, dist[i], xy[i], sup_w[i], sup_h[i]); });
                if (r) return r;
            }
            std::vector<std::future<std::vector<hpm_triangle>>> tris(n_views);
            // two cores stay with the thread that feeds the GPU, so that it is not preempted by the workers
            const unsigned hc = std::thread::hardware_concurrency();
            const int workers = (int)std::max(1u, std::min(16u, hc > 3 ? hc - 2 : 1u));
            std::atomic<int> next{ 0 };
            std::vector<std::promise<std::vector<hpm_triangle>>> done(n_views);
            for (int i = 0; i < n_views; ++i) tris[i] = done[i].get_future();
            std::vector<std::thread> pool;
            for (int w = 0; w < std::min(workers, n_views); ++w)
                pool.emplace_back([&]() {
                    for (int i = next++; i < n_views; i = next++) {
                        std::vector<hpm_triangle> t;
                        delaunay_triangulate(xy[i].data(), (int)xy[i].size() / 2, sup_w[i], sup_h[i], t);
                        done[i].set_value(std::move(t));
                    }
                });
            if (opt->batch == HPM_RECON_SEQUENTIAL) {
                for (int i = 0; i < n_views && !r; ++i) {
                    const std::vector<hpm_triangle> t = tris[i].get();
                    r = timed(HPM_STAGE_PRIOR, [&]() {
                        return prior_from_triangles(i, dist[i], t.data(), (int)t.size(), sup_w[i], sup_h[i]);
                    });
                    if (!r) r = run(i, HPM_MODE_PRIOR, level);
                }
            } else {
                // a group's priors are built, then its batch runs while later triangulations continue
                // (four groups unless batch_views says otherwise, so the host triangulations overlap the GPU)
                const int pgroup = opt->batch_views > 0 ? opt->batch_views : std::max(1, (n_views + 3) / 4);
                for (int g = 0; g < n_views && !r; g += pgroup) {
                    const int end = std::min(n_views, g + pgroup);
                    for (int i = g; i < end && !r; ++i) {
                        const std::vector<hpm_triangle> t = tris[i].get();
                        r = timed(HPM_STAGE_PRIOR, [&]() {
                            return prior_from_triangles(i, dist[i], t.data(), (int)t.size(), sup_w[i], sup_h[i]);
                        });
                    }
                    if (!r) r = run_group(g, end, HPM_MODE_PRIOR, level);
                }
            }
            for (auto& th : pool) th.join();
            if (r) return r;
        }
        return HPM_OK;
    };
    auto geom_passes = [&](int level) -> int {
        for (int it = 0; it < geom_iterations; ++it) {
            uint32_t mode = HPM_MODE_GEOM;
            if (it > 0) {
                mode |= HPM_MODE_MULTIGEOM | HPM_MODE_MAND;
                int r = confidence(HPM_MAP_DEPTH_GEOM);
                if (r) return r;
            }
            ++pass;
            int r = run_pass(mode, level);
            if (r) return r;
        }
        return HPM_OK;
    };

    bool first = true;
    while (max_num_downscale >= 0) {
        for (int i = 0; i < n_views; ++i) {
            if (num_downscale[i] >= 0) {
                cur_max_side[i] = (int)(initial_max_side[i] / std::pow(2.0, num_downscale[i]));
                num_downscale[i]--;
            }
        }
        // PrepareScaleImages (main.cpp:107-161) + InuputInitialization's camera scaling (HPM.cpp:668-676)
        for (int i = 0; i < n_views; ++i) {
            ViewState& v = views[i];
            int w = v.orig_w, h = v.orig_h;
            const int target = cur_max_side[i];
            if (std::max(w, h) > target) {
                const float factor = std::min((float)target / w, (float)target / h);
                w = std::max(1, (int)std::round(v.orig_w * factor));
                h = std::max(1, (int)std::round(v.orig_h * factor));
            }
            hpm_camera c = cams[i];
            const float sx = w / (float)v.orig_w, sy = h / (float)v.orig_h;
            c.K[0] *= sx; c.K[2] *= sx; c.K[4] *= sy; c.K[5] *= sy;
            rc = timed(HPM_STAGE_LEVEL, [&]() { return prepare_level_image(i, w, h, c); });
            if (rc) return rc;
        }
        const int level = max_num_downscale;
        if (first) {
            first = false;
            ++pass;
            if ((rc = run_pass(0, level))) return rc;
            if ((rc = prior_passes(level))) return rc;
            if ((rc = geom_passes(level))) return rc;
        } else {
            for (int i = 0; i < n_views; ++i) {
                int applied = 0;
                if ((rc = timed(HPM_STAGE_JBU, [&]() { return jbu_view(i, &applied); }))) return rc;
            }
            ++pass;
            if ((rc = run_pass(HPM_MODE_HIERARCHY, level))) return rc;
            if ((rc = prior_passes(level))) return rc;
            if ((rc = geom_passes(level))) return rc;
        }
        --max_num_downscale;
    }
    n_points = 0;
    if (opt->fuse) {
        size_t total = 0;
        for (int i = 0; i < n_views; ++i) total += (size_t)views[i].w * views[i].h;
        cudaError_t e = cudaSuccess;
        if (total + 1 > points_cap || !points) {
            if (points) cudaFree(points);
            points = nullptr;
            points_cap = 0;
            e = cudaMalloc((void**)&points, (total + 1) * sizeof(hpm_point));
            if (e == cudaSuccess) points_cap = total + 1;
        }
        if (e != cudaSuccess) return cuda_fail(e, "alloc points");
        int64_t n = 0;
        rc = timed(HPM_STAGE_FUSION, [&]() {
            return consistency_scan(1, n_views, src_off, src_ids, HPM_MAP_DEPTH_GEOM, nullptr, points, (int64_t)total,
                                    &n, nullptr);
        });
        if (rc) return rc;
        n_points = n;
    }
    if (n_points_out) *n_points_out = n_points;
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "reconstruction");
    return HPM_OK;
}

}  // namespace hpm
