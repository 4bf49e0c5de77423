#include "formats.hpp"
#include "hpm_host.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace hpm_host {

std::string id8(int id) {
    char buf[32];
    std::snprintf(buf, sizeof(buf), "%08d", id);
    return buf;
}

std::vector<Problem> read_pair(const std::string& path) {
    std::vector<Problem> out;
    std::ifstream f(path);
    if (!f) return out;
    int n = 0;
    if (!(f >> n) || n < 0) return out;
    for (int i = 0; i < n; ++i) {
        Problem p;
        int k = 0;
        if (!(f >> p.ref_image_id >> k)) return {};
        for (int j = 0; j < k; ++j) {
            int id = 0;
            float score = 0.f;
            if (!(f >> id >> score)) return {};
            if (score <= 0.0f) continue;
            p.src_image_ids.push_back(id);
        }
        out.push_back(std::move(p));
    }
    return out;
}

bool read_camera(const std::string& path, hpm_camera* cam) {
    std::ifstream f(path);
    if (!f) return false;
    std::memset(cam, 0, sizeof(*cam));
    std::string word;
    f >> word;  // "extrinsic"
    for (int i = 0; i < 3; ++i) f >> cam->R[3 * i + 0] >> cam->R[3 * i + 1] >> cam->R[3 * i + 2] >> cam->t[i];
    float last_row[4];
    f >> last_row[0] >> last_row[1] >> last_row[2] >> last_row[3];
    f >> word;  // "intrinsic"
    for (int i = 0; i < 3; ++i) f >> cam->K[3 * i + 0] >> cam->K[3 * i + 1] >> cam->K[3 * i + 2];
    float interval = 0.f, depth_num = 0.f;
    f >> cam->depth_min >> interval >> depth_num >> cam->depth_max;
    return !f.fail();
}

bool write_dmb(const std::string& path, const float* data, int w, int h, int channels) {
    FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) return false;
    const int32_t hdr[4] = { 1, h, w, channels };
    bool ok = std::fwrite(hdr, sizeof(int32_t), 4, fp) == 4;
    const size_t n = (size_t)w * h * channels;
    ok = ok && std::fwrite(data, sizeof(float), n, fp) == n;
    return std::fclose(fp) == 0 && ok;
}

bool read_dmb(const std::string& path, std::vector<float>& data, int& w, int& h, int& channels) {
    FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) return false;
    int32_t hdr[4] = { -1, 0, 0, 0 };
    bool ok = std::fread(hdr, sizeof(int32_t), 4, fp) == 4 && hdr[0] == 1 && hdr[1] > 0 && hdr[2] > 0 && hdr[3] > 0;
    if (ok) {
        h = hdr[1]; w = hdr[2]; channels = hdr[3];
        data.resize((size_t)w * h * channels);
        ok = std::fread(data.data(), sizeof(float), data.size(), fp) == data.size();
    }
    std::fclose(fp);
    return ok;
}

bool write_points_ply(const std::string& path, const hpm_point* pts, size_t n) {
    FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) return false;
    std::fprintf(fp, "ply\nformat binary_little_endian 1.0\nelement vertex %zu\n", n);
    std::fprintf(fp, "property float x\nproperty float y\nproperty float z\n");
    std::fprintf(fp, "property uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n");
    bool ok = true;
    for (size_t i = 0; i < n && ok; ++i) {
        float X[3] = { pts[i].coord[0], pts[i].coord[1], pts[i].coord[2] };
        const bool finite = X[0] < FLT_MAX && X[0] > -FLT_MAX && X[1] < FLT_MAX && X[1] > -FLT_MAX && X[2] < FLT_MAX &&
                            X[2] >= -FLT_MAX;
        if (!finite) X[0] = X[1] = X[2] = 0.0f;
        // colour floats are B, G, R; the file stores R, G, B as (char)(int)
        const char rgb[3] = { (char)(int)pts[i].color[2], (char)(int)pts[i].color[1], (char)(int)pts[i].color[0] };
        ok = std::fwrite(X, sizeof(float), 3, fp) == 3 && std::fwrite(rgb, 1, 3, fp) == 3;
    }
    return std::fclose(fp) == 0 && ok;
}

bool write_fused_ply(const std::string& path, const hpm_point* pts, size_t n, size_t* written) {
    auto valid = [](const hpm_point& p) {
        const double nn = (double)p.normal[0] * p.normal[0] + (double)p.normal[1] * p.normal[1] +
                          (double)p.normal[2] * p.normal[2];
        return std::isfinite(p.coord[0]) && std::isfinite(p.coord[1]) && std::isfinite(p.coord[2]) &&
               std::isfinite(nn) && nn > 1e-20;
    };
    size_t count = 0;
    for (size_t i = 0; i < n; ++i) count += valid(pts[i]);
    const std::string tmp = path + ".tmp";
    FILE* fp = std::fopen(tmp.c_str(), "wb");
    if (!fp) return false;
    std::fprintf(fp, "ply\nformat binary_little_endian 1.0\nelement vertex %zu\n", count);
    std::fprintf(fp, "property float x\nproperty float y\nproperty float z\n");
    std::fprintf(fp, "property float nx\nproperty float ny\nproperty float nz\n");
    std::fprintf(fp, "property uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n");
    auto channel = [](float v) -> unsigned char {
        return std::isfinite(v) ? (unsigned char)std::max(0.0f, std::min(255.0f, v)) : 0;
    };
    bool ok = true;
    for (size_t i = 0; i < n && ok; ++i) {
        const hpm_point& p = pts[i];
        if (!valid(p)) continue;
        const double len = std::sqrt((double)p.normal[0] * p.normal[0] + (double)p.normal[1] * p.normal[1] +
                                     (double)p.normal[2] * p.normal[2]);
        const float v[6] = { p.coord[0], p.coord[1], p.coord[2], (float)(p.normal[0] / len), (float)(p.normal[1] / len),
                             (float)(p.normal[2] / len) };
        const unsigned char rgb[3] = { channel(p.color[2]), channel(p.color[1]), channel(p.color[0]) };
        ok = std::fwrite(v, sizeof(float), 6, fp) == 6 && std::fwrite(rgb, 1, 3, fp) == 3;
    }
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) return false;
    if (written) *written = count;
    return true;
}

}  // namespace hpm_host

extern "C" int hpm_write_ply(const char* path, const hpm_point* pts, size_t n, int fused, size_t* written) {
    if (!path || (!pts && n)) return -1;
    if (fused) return hpm_host::write_fused_ply(path, pts, n, written) ? 0 : -1;
    if (written) *written = n;
    return hpm_host::write_points_ply(path, pts, n) ? 0 : -1;
}
