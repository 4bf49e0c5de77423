#include "hpm_class.hpp"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <map>
#include <stdexcept>

#include "hpm_host.h"

namespace hpm_host {

namespace {

hpm_ctx* g_ctx = nullptr;

struct Uploaded {
    int w = 0, h = 0;          // original size
    int level_w = 0, level_h = 0;
};
std::map<int, Uploaded> g_views;  // per image id

void check(int rc, const char* what) {
    if (rc != HPM_OK) throw std::runtime_error(std::string(what) + ": " + hpm_last_error(g_ctx));
}

std::string result_folder(const std::string& dense_folder, int id) {
    return dense_folder + "/HPM_MVS_plusplus/2333_" + id8(id);
}

void load_map(const std::string& path, int view, int kind) {
    std::vector<float> m;
    int w, h, c;
    if (!read_dmb(path, m, w, h, c)) throw std::runtime_error("cannot read " + path);
    check(hpm_set_map(g_ctx, view, kind, m.data(), w, h), "hpm_set_map");
}

std::vector<float> download(int view, int kind) {
    int w = 0, h = 0;
    check(hpm_get_map(g_ctx, view, kind, nullptr, 0, &w, &h), "hpm_get_map");
    std::vector<float> m((size_t)w * h * (kind == HPM_MAP_NORMAL ? 3 : 1));
    check(hpm_get_map(g_ctx, view, kind, m.data(), m.size(), &w, &h), "hpm_get_map");
    return m;
}

void upload_original(const std::string& dense_folder, int id) {
    Uploaded& u = g_views[id];
    if (u.w != 0) return;
    const std::string path = dense_folder + "/images/" + id8(id) + ".jpg";
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot read " + path);
    std::vector<uint8_t> bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    uint8_t* bgr = nullptr;
    if (hpm_decode_image(bytes.data(), bytes.size(), &bgr, &u.w, &u.h) != 0)
        throw std::runtime_error(path + ": " + hpm_image_error());
    const int rc = hpm_set_image(g_ctx, id, bgr, u.w, u.h);
    const int rs = hpm_synchronize(g_ctx);
    hpm_free_image(bgr);
    check(rc, "hpm_set_image");
    check(rs, "hpm_synchronize");
}

// Uploads image `id` once, then (re)builds its level at `target` longest side
// (PrepareScaleImages, main.cpp:107-161; camera scaling of HPM.cpp:668-676).
void prepare_view(const std::string& dense_folder, int id, int target, hpm_camera* cam_out) {
    upload_original(dense_folder, id);
    Uploaded& u = g_views[id];
    hpm_camera cam;
    if (!read_camera(dense_folder + "/cams/" + id8(id) + "_cam.txt", &cam))
        throw std::runtime_error("cannot read the camera of image " + std::to_string(id));
    int w = u.w, h = u.h;
    if (target > 0 && std::max(w, h) > target) {
        const float factor = std::min((float)target / u.w, (float)target / u.h);
        w = std::max(1, (int)std::round(u.w * factor));
        h = std::max(1, (int)std::round(u.h * factor));
    }
    const float sx = w / (float)u.w, sy = h / (float)u.h;
    cam.K[0] *= sx; cam.K[2] *= sx; cam.K[4] *= sy; cam.K[5] *= sy;
    cam.width = w;
    cam.height = h;
    if (u.level_w != w || u.level_h != h) {
        check(hpm_prepare_level(g_ctx, id, w, h, &cam), "hpm_prepare_level");
        u.level_w = w;
        u.level_h = h;
    }
    if (cam_out) *cam_out = cam;
}

}  // namespace

void HPM::original_size(const std::string& dense_folder, int id, int* w, int* h) {
    context();
    upload_original(dense_folder, id);
    *w = g_views[id].w;
    *h = g_views[id].h;
}

hpm_ctx* HPM::context() {
    if (!g_ctx && hpm_create(0, &g_ctx) != HPM_OK) throw std::runtime_error("hpm_create failed (no CUDA device?)");
    return g_ctx;
}

void HPM::release_context() {
    if (g_ctx) hpm_destroy(g_ctx);
    g_ctx = nullptr;
    g_views.clear();
}

HPM::HPM() {
    context();
    params_.max_iterations = 3;  // RunPatchMatch hard-codes 3 (HPM.cu:3013)
    params_.patch_size = 11;
    params_.radius_increment = 2;
    params_.sigma_spatial = 5.0f;
    params_.sigma_color = 3.0f;
    params_.top_k = 4;
}

HPM::~HPM() = default;

void HPM::SetGeomConsistencyParams(bool multi_geometry) {
    mode_ |= HPM_MODE_GEOM;
    if (multi_geometry) mode_ |= HPM_MODE_MULTIGEOM;
}
void HPM::SetPlanarPriorParams() { mode_ |= HPM_MODE_PRIOR; }
void HPM::SetHierarchyParams() { mode_ |= HPM_MODE_HIERARCHY; }
void HPM::SetMandConsistencyParams(bool flag) {
    if (flag) mode_ |= HPM_MODE_MAND;
    else mode_ &= ~(uint32_t)HPM_MODE_MAND;
}

void HPM::InuputInitialization(const std::string& dense_folder, const std::vector<PyramidProblem>& problems,
                               const int idx) {
    const PyramidProblem& pb = problems[idx];
    ref_ = pb.ref_image_id;
    srcs_ = pb.src_image_ids;
    hpm_camera cam;
    prepare_view(dense_folder, ref_, pb.cur_max_side, &cam);
    for (int s : srcs_) prepare_view(dense_folder, s, problems[s].cur_max_side, nullptr);
    width_ = cam.width;
    height_ = cam.height;
    params_.depth_min = cam.depth_min * 0.6f;
    params_.depth_max = cam.depth_max * 1.2f;
    params_.num_images = (int)srcs_.size() + 1;
    if (mode_ & HPM_MODE_GEOM) {  // HPM.cpp:688-737: depths(_geom).dmb of the reference and its sources
        const int kind = (mode_ & HPM_MODE_MULTIGEOM) ? HPM_MAP_DEPTH_GEOM : HPM_MAP_DEPTH;
        const char* suffix = (mode_ & HPM_MODE_MULTIGEOM) ? "/depths_geom.dmb" : "/depths.dmb";
        load_map(result_folder(dense_folder, ref_) + suffix, ref_, kind);
        for (int s : srcs_) load_map(result_folder(dense_folder, s) + suffix, s, kind);
    }
}

void HPM::CudaSpaceInitialization(const std::string& dense_folder, const PyramidProblem& problem) {
    const std::string dir = result_folder(dense_folder, problem.ref_image_id);
    if ((mode_ & HPM_MODE_GEOM) && !(mode_ & HPM_MODE_PRIOR)) {  // hypotheses reload (HPM.cpp:813-846)
        load_map(dir + "/normals.dmb", ref_, HPM_MAP_NORMAL);
        load_map(dir + "/costs.dmb", ref_, HPM_MAP_COST);
    }
    if (mode_ & HPM_MODE_HIERARCHY) {  // the upsampled depths and the coarser level's normals and costs (HPM.cpp:848-906)
        load_map(dir + "/depths.dmb", ref_, HPM_MAP_DEPTH);
        load_map(dir + "/normals.dmb", ref_, HPM_MAP_NORMAL);
        load_map(dir + "/costs.dmb", ref_, HPM_MAP_COST);
    }
}

void HPM::CudaConfidenceInitialization(const std::string& dense_folder, const std::vector<PyramidProblem>& problems,
                                       const int idx) {
    load_map(result_folder(dense_folder, problems[idx].ref_image_id) + "/confidence.dmb", ref_, HPM_MAP_CONF);
}

void HPM::CudaCannyInitialization(const Map<int>& canny) {
    std::vector<uint8_t> e(canny.data.size());
    for (size_t i = 0; i < e.size(); ++i) e[i] = canny.data[i] ? 255 : 0;
    check(hpm_set_canny(g_ctx, ref_, e.data(), canny.cols, canny.rows), "hpm_set_canny");
}

void HPM::CudaHypothesesReload(const Map<float>& depths, const Map<float>& costs, const Map<float>& normals) {
    check(hpm_set_map(g_ctx, ref_, HPM_MAP_DEPTH, depths.data.data(), depths.cols, depths.rows), "hpm_set_map");
    check(hpm_set_map(g_ctx, ref_, HPM_MAP_COST, costs.data.data(), costs.cols, costs.rows), "hpm_set_map");
    check(hpm_set_map(g_ctx, ref_, HPM_MAP_NORMAL, normals.data.data(), normals.cols, normals.rows), "hpm_set_map");
}

void HPM::CudaPlanarPriorInitialization(const std::vector<Plane4>& plane_params, const Map<float>& masks) {
    std::vector<float> planes((size_t)masks.rows * masks.cols * 4, 0.0f);
    std::vector<uint8_t> m((size_t)masks.rows * masks.cols, 0);
    for (size_t i = 0; i < m.size(); ++i) {
        const int label = (int)masks.data[i];
        if (label > 0 && label <= (int)plane_params.size()) {
            const Plane4& p = plane_params[label - 1];
            planes[4 * i] = p.x; planes[4 * i + 1] = p.y; planes[4 * i + 2] = p.z; planes[4 * i + 3] = p.w;
            m[i] = 1;
        }
    }
    check(hpm_set_prior(g_ctx, ref_, planes.data(), m.data(), masks.cols, masks.rows), "hpm_set_prior");
}

void HPM::BuildPlanarPrior(int distance) {
    check(hpm_build_prior(g_ctx, ref_, distance, nullptr, nullptr), "hpm_build_prior");
}

void HPM::RunPatchMatch(uint64_t seed) {
    params_.mode = mode_;
    params_.scaled_cols = params_.scaled_rows = 0;
    check(hpm_run_patchmatch(g_ctx, ref_, srcs_.data(), (int)srcs_.size(), &params_, texture_level_, seed),
          "hpm_run_patchmatch");
    depth_ = download(ref_, (mode_ & HPM_MODE_GEOM) ? HPM_MAP_DEPTH_GEOM : HPM_MAP_DEPTH);
    normal_ = download(ref_, HPM_MAP_NORMAL);
    cost_ = download(ref_, HPM_MAP_COST);
    if (!(mode_ & (HPM_MODE_PRIOR | HPM_MODE_MAND))) texture_ = download(ref_, HPM_MAP_TEXTURE0 + texture_level_);
}

Plane4 HPM::GetPlaneHypothesis(const int index) const {
    return Plane4{ normal_[3 * (size_t)index], normal_[3 * (size_t)index + 1], normal_[3 * (size_t)index + 2],
                   depth_[index] };
}

float HPM::GetCost(const int index) const { return cost_[index]; }

float HPM::GetTexture(const int index) const { return texture_.empty() ? 0.0f : texture_[index]; }

Map<uint8_t> HPM::GetReferenceImage() const {
    Map<uint8_t> img(height_, width_, 3);
    check(hpm_get_level(g_ctx, ref_, img.data.data(), nullptr, nullptr), "hpm_get_level");
    return img;
}

}  // namespace hpm_host
