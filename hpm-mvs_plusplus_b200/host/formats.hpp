// On-disk formats of HPM-MVS++ used by the command-line driver: the dense
// folder's cams/%08d_cam.txt and pair.txt, the per-view .dmb maps and the two
// point-cloud PLY files.  Plain C++17; no OpenCV.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "hpm_capi.h"

namespace hpm_host {

struct Problem {  // one line pair of pair.txt (main.cpp:171-200)
    int ref_image_id = 0;
    std::vector<int> src_image_ids;
};

// pair.txt: count, then per view its id and "n  id score  id score ...";
// sources with score <= 0 are dropped, as GenerateSampleList does.
std::vector<Problem> read_pair(const std::string& path);

// cams/%08d_cam.txt (ReadCamera, HPM.cpp:159-184): extrinsic 3x4 (+ last row),
// intrinsic 3x3, then "depth_min interval depth_num depth_max".  Width and
// height are not in the file; the caller sets them from the image.
bool read_camera(const std::string& path, hpm_camera* cam);

// .dmb (HPM.cpp:291-407): int32 type = 1, h, w, channels, then h*w*channels
// floats, row-major.
bool write_dmb(const std::string& path, const float* data, int w, int h, int channels);
bool read_dmb(const std::string& path, std::vector<float>& data, int& w, int& h, int& channels);

// HPM_MVS_plusplus.ply (ExportPointCloud, HPM.cpp:433-482): x y z float and
// red green blue uchar, taken from the BGR colour floats; non-finite
// coordinates are written as the origin.
bool write_points_ply(const std::string& path, const hpm_point* pts, size_t n);

// fused.ply (ExportFusedPointCloud, HPM.cpp:410-431): points with finite
// coordinates and a non-zero normal, x y z, the unit normal, red green blue.
bool write_fused_ply(const std::string& path, const hpm_point* pts, size_t n, size_t* written);

// "%08d"
std::string id8(int id);

}  // namespace hpm_host
