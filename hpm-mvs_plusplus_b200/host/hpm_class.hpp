// The reference's host-side `HPM` class (HPM.h:57-140) rebuilt on the C ABI
// of libhpm_cuda.so, with its method names and call order, for callers written
// against it (ProcessProblem, main.cpp:237-634).  cv::Mat_ arguments become the
// small row-major `Map` below; all views share one process-wide context, so
// images uploaded for one problem stay resident for the next.
//
// Per problem the caller does what ProcessProblem does:
//   HPM hpm;                                   // one per problem
//   hpm.SetGeomConsistencyParams(multi);       // geometric runs
//   hpm.SetHierarchyParams();                  // hierarchy run
//   hpm.InuputInitialization(folder, problems, idx);
//   hpm.CudaSpaceInitialization(folder, problems[idx]);
//   hpm.SetMandConsistencyParams(mand);
//   hpm.CudaConfidenceInitialization(folder, problems, idx);  // prior / mandatory
//   hpm.SetPlanarPriorParams(); hpm.BuildPlanarPrior(distance); hpm.CudaHypothesesReload(...);  // prior
//   hpm.RunPatchMatch(seed);
//   ... GetPlaneHypothesis(i), GetCost(i), GetTexture(i)
// The differences: the random stream of a run is keyed by an explicit seed
// (the reference seeds from clock64(), HPM.cu:579), and the planar prior is
// built on the GPU (BuildPlanarPrior) where the reference's caller assembles it
// from support points, cv::Subdiv2D and host loops (main.cpp:349-597).
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "formats.hpp"
#include "hpm_capi.h"

namespace hpm_host {

template <class T>
struct Map {  // row-major, `channels` values per pixel
    int rows = 0, cols = 0, channels = 1;
    std::vector<T> data;
    Map() = default;
    Map(int r, int c, int ch = 1) : rows(r), cols(c), channels(ch), data((size_t)r * c * ch) {}
    T& operator()(int r, int c, int ch = 0) { return data[((size_t)r * cols + c) * channels + ch]; }
    const T& operator()(int r, int c, int ch = 0) const { return data[((size_t)r * cols + c) * channels + ch]; }
};

struct Plane4 {
    float x, y, z, w;
};

// What the reference keeps in Problem for the pyramid (main.h:49-58).
struct PyramidProblem : Problem {
    int cur_max_side = 0;  // longest side of this level's images
    int num_downscale = 0;
};

class HPM {
public:
    HPM();
    ~HPM();

    // The process-wide context; created on first use on device 0.
    static hpm_ctx* context();
    static void release_context();
    // Size of images/%08d.jpg of `id` (decoded and uploaded on first use).
    static void original_size(const std::string& dense_folder, int id, int* w, int* h);

    void InuputInitialization(const std::string& dense_folder, const std::vector<PyramidProblem>& problems,
                              const int idx);
    void CudaSpaceInitialization(const std::string& dense_folder, const PyramidProblem& problem);
    void RunPatchMatch(uint64_t seed);
    void SetGeomConsistencyParams(bool multi_geometry);
    void SetPlanarPriorParams();
    void SetHierarchyParams();
    void SetMandConsistencyParams(bool flag);

    int GetReferenceImageWidth() const { return width_; }
    int GetReferenceImageHeight() const { return height_; }
    Map<uint8_t> GetReferenceImage() const;  // BGR level image
    Plane4 GetPlaneHypothesis(const int index) const;
    float GetCost(const int index) const;
    float GetTexture(const int index) const;
    float GetMinDepth() const { return params_.depth_min; }
    float GetMaxDepth() const { return params_.depth_max; }

    void CudaPlanarPriorInitialization(const std::vector<Plane4>& plane_params, const Map<float>& masks);
    void CudaHypothesesReload(const Map<float>& depths, const Map<float>& costs, const Map<float>& normals);
    void CudaConfidenceInitialization(const std::string& dense_folder, const std::vector<PyramidProblem>& problems,
                                      const int idx);
    void CudaCannyInitialization(const Map<int>& canny);
    void TextureInformationInitialization() {}
    // Support points, Delaunay triangulation, raster and plane fits of the
    // prior at scale distance 0, 1 or 2 (main.cpp:349-597), on the context.
    void BuildPlanarPrior(int distance);
    void CudaPlanarPriorRelease() {}
    void CudaSpaceRelease(bool) {}
    void ReleaseProblemHostMemory() {}

    void set_texture_level(int level) { texture_level_ = level; }

private:
    int ref_ = 0;
    std::vector<int> srcs_;
    int width_ = 0, height_ = 0;
    hpm_params params_{};
    uint32_t mode_ = 0;
    int texture_level_ = 0;
    // results of the last RunPatchMatch (world normal + depth, cost, texture)
    std::vector<float> depth_, normal_, cost_, texture_;
};

}  // namespace hpm_host
