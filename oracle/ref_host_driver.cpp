// CHECKER ONLY: runs two host stages of the reference's own main.cpp,
// ConfidenceEvaluation (main.cpp:959-1109) and RunFusion / RunFusion_Sky_Strict
// (main.cpp:659-957), and one member of HPM.cpp, the prior's support-point
// selection HPM::GetSupportPoints_Classify_Check (HPM.cpp:1026-1073), compiled
// from their sources by oracle/ref_host.mk against
// the OpenCV stand-ins of oracle/ref_shim_host.  They read a dense folder the
// caller writes: cams/%08d_cam.txt, images/%08d.jpg.raw (see cv::imread below)
// and HPM_MVS_plusplus/2333_%08d/{depths,depths_geom,normals}.dmb, and write
// confidence.dmb or HPM_MVS_plusplus.ply and fused.ply there.  Used by
// tests/test_ref_host.py.
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "main.h"  // the standard headers first, so that only HPM's members open up below
#define private public
#include "HPM.h"
#undef private

void ConfidenceEvaluation(std::string& dense_folder, const std::vector<Problem>& problems, bool geom_consistency);
void RunFusion(std::string& dense_folder, const std::vector<Problem>& problems, bool geom_consistency);
void RunFusion_Sky_Strict(std::string& dense_folder, const std::vector<Problem>& problems, bool geom_consistency);

namespace cv {

// The image as the caller stored it beside the named path: <path>.raw holds
// int32 rows, cols, channels, then rows*cols*channels bytes (BGR for 3).
Mat imread(const std::string& path, int flags) {
    Mat m;
    FILE* f = std::fopen((path + ".raw").c_str(), "rb");
    if (!f) return m;
    int32_t hdr[3] = {0, 0, 0};
    if (std::fread(hdr, sizeof(int32_t), 3, f) == 3 && hdr[0] > 0 && hdr[1] > 0 && (hdr[2] == 1 || hdr[2] == 3)) {
        m.create(hdr[0], hdr[1], hdr[2] == 3 ? CV_8UC3 : CV_8UC1);
        const size_t n = (size_t)hdr[0] * hdr[1] * hdr[2];
        if (std::fread(m.data, 1, n, f) != n) m.release();
        if (!m.empty() && flags == IMREAD_COLOR && hdr[2] == 1) {
            Mat c(hdr[0], hdr[1], CV_8UC3);
            for (size_t i = 0; i < (size_t)hdr[0] * hdr[1]; ++i)
                c.data[3 * i] = c.data[3 * i + 1] = c.data[3 * i + 2] = m.data[i];
            m = c;
        }
    }
    std::fclose(f);
    return m;
}

// RescaleImageAndCamera (HPM.cpp:186-207) resizes only when the image and the
// depth map differ in size; the caller stores images at the maps' size.
void resize(const Mat& src, Mat& dst, Size dsize, double, double, int) {
    if (src.rows != dsize.height || src.cols != dsize.width)
        throw std::runtime_error("checker: images must be stored at the depth maps' size");
    dst = src.clone();
}

}  // namespace cv

static std::vector<Problem> make_problems(int n, const int* src_off, const int* src_ids) {
    std::vector<Problem> problems(n);
    for (int i = 0; i < n; ++i) {
        problems[i].ref_image_id = i;
        problems[i].src_image_ids.assign(src_ids + src_off[i], src_ids + src_off[i + 1]);
    }
    return problems;
}

// src_off: n + 1 offsets into src_ids (the pair.txt sources of each view).
extern "C" __attribute__((visibility("default"))) int ref_host_confidence(const char* dense_folder, int n,
                                                                          const int* src_off, const int* src_ids,
                                                                          int geom) {
    try {
        std::string folder(dense_folder);
        ConfidenceEvaluation(folder, make_problems(n, src_off, src_ids), geom != 0);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_host_confidence: %s\n", e.what());
        return -1;
    }
}

// sky != 0: RunFusion_Sky_Strict (masks/%08d.jpg.raw beside the images)
extern "C" __attribute__((visibility("default"))) int ref_host_fusion(const char* dense_folder, int n,
                                                                      const int* src_off, const int* src_ids,
                                                                      int geom, int sky) {
    try {
        std::string folder(dense_folder);
        if (sky) RunFusion_Sky_Strict(folder, make_problems(n, src_off, src_ids), geom != 0);
        else RunFusion(folder, make_problems(n, src_off, src_ids), geom != 0);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_host_fusion: %s\n", e.what());
        return -1;
    }
}

// HPM::GetSupportPoints_Classify_Check on maps of (width*factor) x
// (height*factor) pixels of a reference camera of width x height.  The HPM
// object is never destroyed: its destructor releases CUDA resources.
extern "C" __attribute__((visibility("default"))) int ref_host_support_points(
    const Camera* cam, const float* costs, const float* confidences, const float* texture, int map_w, int map_h,
    float factor, int* out_xy, int max_points) {
    try {
        static HPM* hpm = new HPM();
        hpm->cameras.assign(1, *cam);
        cv::Mat_<float> c(cv::Mat(map_h, map_w, CV_32FC1, const_cast<float*>(costs)));
        cv::Mat_<float> q(cv::Mat(map_h, map_w, CV_32FC1, const_cast<float*>(confidences)));
        cv::Mat_<float> t(cv::Mat(map_h, map_w, CV_32FC1, const_cast<float*>(texture)));
        std::vector<cv::Point> pts;
        hpm->GetSupportPoints_Classify_Check(pts, c, q, t, factor);
        const int n = (int)pts.size();
        for (int i = 0; i < n && i < max_points; ++i) {
            out_xy[2 * i] = pts[i].x;
            out_xy[2 * i + 1] = pts[i].y;
        }
        return n;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_host_support_points: %s\n", e.what());
        return -1;
    }
}
