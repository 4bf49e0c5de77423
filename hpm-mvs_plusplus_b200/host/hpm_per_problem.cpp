// The reference's main loop run problem by problem through the HPM class,
// with every stage's results handed to the next through the .dmb files of the
// dense folder, as main.cpp:1183-1359 does (ProcessProblem main.cpp:237-634,
// JointBilateralUpsampling main.cpp:636-657, ConfidenceEvaluation
// main.cpp:959-1109, RunFusion main.cpp:823-957).  It draws the same random
// streams as hpm_reconstruct (hpm_run_seed with the same pass numbering), so
// the two produce the same maps; the command-line driver runs it with
// --per-problem.
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "formats.hpp"
#include "hpm_class.hpp"

namespace hpm_host {

namespace {

void check(hpm_ctx* ctx, int rc, const char* what) {
    if (rc != HPM_OK) throw std::runtime_error(std::string(what) + ": " + hpm_last_error(ctx));
}

std::string result_folder(const std::string& folder, int id) { return folder + "/HPM_MVS_plusplus/2333_" + id8(id); }

std::vector<float> download(hpm_ctx* ctx, int view, int kind, int& w, int& h) {
    check(ctx, hpm_get_map(ctx, view, kind, nullptr, 0, &w, &h), "hpm_get_map");
    std::vector<float> m((size_t)w * h * (kind == HPM_MAP_NORMAL ? 3 : 1));
    check(ctx, hpm_get_map(ctx, view, kind, m.data(), m.size(), &w, &h), "hpm_get_map");
    return m;
}

void write_map(hpm_ctx* ctx, int view, int kind, const std::string& path) {
    int w, h;
    const std::vector<float> m = download(ctx, view, kind, w, h);
    if (!write_dmb(path, m.data(), w, h, kind == HPM_MAP_NORMAL ? 3 : 1)) throw std::runtime_error("cannot write " + path);
}

void read_map(hpm_ctx* ctx, int view, int kind, const std::string& path) {
    std::vector<float> m;
    int w, h, c;
    if (!read_dmb(path, m, w, h, c)) throw std::runtime_error("cannot read " + path);
    check(ctx, hpm_set_map(ctx, view, kind, m.data(), w, h), "hpm_set_map");
}

// ProcessProblem (main.cpp:237-634) for one problem and pass.
void process_problem(const std::string& folder, const std::vector<PyramidProblem>& problems, int idx, bool geom,
                     bool prior, bool hierarchy, bool mand, int image_scale, bool multi_geometry, int distance,
                     uint64_t seed) {
    HPM hpm;
    if (geom) hpm.SetGeomConsistencyParams(multi_geometry);
    if (hierarchy) hpm.SetHierarchyParams();
    hpm.InuputInitialization(folder, problems, idx);
    hpm.CudaSpaceInitialization(folder, problems[idx]);
    hpm.SetMandConsistencyParams(mand);
    hpm.set_texture_level(image_scale);
    if (mand || prior) hpm.CudaConfidenceInitialization(folder, problems, idx);
    const int id = problems[idx].ref_image_id;
    const std::string dir = result_folder(folder, id);
    hpm_ctx* ctx = HPM::context();
    if (prior) {
        hpm.SetPlanarPriorParams();
        read_map(ctx, id, HPM_MAP_DEPTH, dir + "/depths.dmb");
        read_map(ctx, id, HPM_MAP_NORMAL, dir + "/normals.dmb");
        read_map(ctx, id, HPM_MAP_COST, dir + "/costs.dmb");
        hpm.BuildPlanarPrior(distance);
    }
    hpm.RunPatchMatch(seed);
    write_map(ctx, id, geom ? HPM_MAP_DEPTH_GEOM : HPM_MAP_DEPTH, dir + (geom ? "/depths_geom.dmb" : "/depths.dmb"));
    write_map(ctx, id, HPM_MAP_NORMAL, dir + "/normals.dmb");
    write_map(ctx, id, HPM_MAP_COST, dir + "/costs.dmb");
    if (!prior && !mand)
        write_map(ctx, id, HPM_MAP_TEXTURE0 + image_scale, dir + "/texture" + std::to_string(image_scale) + ".dmb");
}

// ConfidenceEvaluation (main.cpp:959-1109): every view's depth map of the given
// kind and its normals from the files, confidence.dmb back out.
void confidence_evaluation(const std::string& folder, const std::vector<PyramidProblem>& problems,
                           const std::vector<int32_t>& src_off, const std::vector<int32_t>& src_ids, bool geom) {
    hpm_ctx* ctx = HPM::context();
    const int n = (int)problems.size();
    const int kind = geom ? HPM_MAP_DEPTH_GEOM : HPM_MAP_DEPTH;
    for (int i = 0; i < n; ++i) {
        const std::string dir = result_folder(folder, i);
        read_map(ctx, i, kind, dir + (geom ? "/depths_geom.dmb" : "/depths.dmb"));
        read_map(ctx, i, HPM_MAP_NORMAL, dir + "/normals.dmb");
    }
    check(ctx, hpm_confidence_eval(ctx, n, src_off.data(), src_ids.data(), kind, nullptr), "hpm_confidence_eval");
    for (int i = 0; i < n; ++i) write_map(ctx, i, HPM_MAP_CONF, result_folder(folder, i) + "/confidence.dmb");
}

}  // namespace

int64_t run_per_problem(const std::string& folder, const std::vector<Problem>& pairs, int scale, uint64_t seed,
                        int level_max_side, const std::vector<int32_t>& src_off, const std::vector<int32_t>& src_ids) {
    hpm_ctx* ctx = HPM::context();
    const int n = (int)pairs.size();
    std::vector<PyramidProblem> problems(n);
    for (int i = 0; i < n; ++i) static_cast<Problem&>(problems[i]) = pairs[i];
    // ComputeMultiScaleSettings (main.cpp:202-235), image sizes from the decoded images
    const int size_bound = level_max_side > 0 ? level_max_side : 1000;
    std::vector<int> initial_max_side(n), num_downscale(n);
    int max_num_downscale = -1;
    for (int i = 0; i < n; ++i) {
        int w = 0, h = 0;
        HPM::original_size(folder, i, &w, &h);
        const int original = std::max(w, h);
        initial_max_side[i] = std::max(1, (original + scale / 2) / scale);
        int k = 0, side = initial_max_side[i];
        while (side > size_bound) { side /= 2; ++k; }
        num_downscale[i] = k;
        max_num_downscale = std::max(max_num_downscale, k);
    }
    mkdir((folder + "/HPM_MVS_plusplus").c_str(), 0755);
    for (int i = 0; i < n; ++i) mkdir(result_folder(folder, i).c_str(), 0755);
    const int max_hpm_scale = max_num_downscale;
    int pass = 0;
    bool first = true;
    while (max_num_downscale >= 0) {
        for (int i = 0; i < n; ++i)
            if (num_downscale[i] >= 0) {
                problems[i].cur_max_side = (int)(initial_max_side[i] / std::pow(2.0, num_downscale[i]));
                problems[i].num_downscale = --num_downscale[i];
            }
        const int level = max_num_downscale;
        if (first) {
            first = false;
            ++pass;
            for (int i = 0; i < n; ++i)
                process_problem(folder, problems, i, false, false, false, false, level, false, 0,
                                hpm_run_seed(seed, pass, i));
        } else {
            // JointBilateralUpsampling (main.cpp:636-657): the coarser depths_geom.dmb to this level's depths.dmb
            for (int i = 0; i < n; ++i) {
                HPM view;  // puts view i at this level's size
                std::vector<PyramidProblem> one(problems);
                one[i].src_image_ids.clear();
                view.InuputInitialization(folder, one, i);
                const std::string dir = result_folder(folder, i);
                read_map(ctx, i, HPM_MAP_DEPTH_GEOM, dir + "/depths_geom.dmb");
                int applied = 0;
                check(ctx, hpm_jbu(ctx, i, &applied), "hpm_jbu");
                if (applied) write_map(ctx, i, HPM_MAP_DEPTH, dir + "/depths.dmb");
            }
            ++pass;
            for (int i = 0; i < n; ++i)
                process_problem(folder, problems, i, false, false, true, false, level, false, 0,
                                hpm_run_seed(seed, pass, i));
        }
        for (int hpm_scale = max_hpm_scale; hpm_scale >= level; --hpm_scale) {
            confidence_evaluation(folder, problems, src_off, src_ids, false);
            ++pass;
            for (int i = 0; i < n; ++i) {
                const int distance = hpm_scale - num_downscale[i] - 1;
                if (distance < 0 || distance > 2) throw std::runtime_error("prior scale distance outside 0..2");
                process_problem(folder, problems, i, false, true, false, false, level, false, distance,
                                hpm_run_seed(seed, pass, i));
            }
        }
        for (int it = 0; it < 3; ++it) {
            if (it > 0) confidence_evaluation(folder, problems, src_off, src_ids, true);
            ++pass;
            for (int i = 0; i < n; ++i)
                process_problem(folder, problems, i, true, false, false, it > 0, level, it > 0, 0,
                                hpm_run_seed(seed, pass, i));
        }
        --max_num_downscale;
    }
    // the fusion inputs from the files
    for (int i = 0; i < n; ++i) {
        const std::string dir = result_folder(folder, i);
        read_map(ctx, i, HPM_MAP_DEPTH_GEOM, dir + "/depths_geom.dmb");
        read_map(ctx, i, HPM_MAP_NORMAL, dir + "/normals.dmb");
    }
    return 0;
}

}  // namespace hpm_host
