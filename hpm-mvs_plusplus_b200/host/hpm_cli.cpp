// HPM-MVS_plusplus command-line driver on libhpm_cuda.so: the same command
// line, inputs and outputs as the reference's main (main.cpp:1143-1364).
//
//   HPM-MVS_plusplus dense_folder [--initial-image-scale N] [--show-medium-result]
//                    [--mask] [--fusion-only | --fuse]
//
// Reads dense_folder/pair.txt, cams/%08d_cam.txt and images/%08d.jpg (PNG or
// JPEG content), runs the whole schedule resident on the GPU, and writes
// HPM_MVS_plusplus/2333_%08d/{depths.dmb, depths_geom.dmb, normals.dmb} for
// every view (plus costs.dmb and confidence.dmb with --show-medium-result),
// HPM_MVS_plusplus/HPM_MVS_plusplus.ply and HPM_MVS_plusplus/fused.ply.
// --mask fuses with the sky masks masks/%08d.jpg (RunFusion_Sky_Strict);
// the environment variable HPM_SEED (decimal) fixes the random streams;
// --fusion-only skips the reconstruction and fuses the existing
// depths_geom.dmb / normals.dmb; --per-problem runs the reference's main loop
// problem by problem through the HPM class, with .dmb files between the
// stages (same results as the default resident schedule).  HPM_LEVEL_MAX_SIDE
// (default 1000) is the pyramid bound of main.cpp:205, for small test inputs.
#include <sys/stat.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "formats.hpp"
#include "hpm_capi.h"
#include "hpm_class.hpp"
#include "hpm_host.h"

using namespace hpm_host;

namespace hpm_host {
int64_t run_per_problem(const std::string& folder, const std::vector<Problem>& pairs, int scale, uint64_t seed,
                        int level_max_side, const std::vector<int32_t>& src_off, const std::vector<int32_t>& src_ids);
}

namespace {

struct Image {
    std::vector<uint8_t> bgr;
    int w = 0, h = 0;
};

bool load_image(const std::string& path, Image& img) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    std::vector<uint8_t> bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    uint8_t* data = nullptr;
    if (hpm_decode_image(bytes.data(), bytes.size(), &data, &img.w, &img.h) != 0) {
        std::cerr << path << ": " << hpm_image_error() << std::endl;
        return false;
    }
    img.bgr.assign(data, data + (size_t)img.w * img.h * 3);
    hpm_free_image(data);
    return true;
}

void check(hpm_ctx* ctx, int rc, const char* what) {
    if (rc != HPM_OK) throw std::runtime_error(std::string(what) + ": " + (ctx ? hpm_last_error(ctx) : "no context"));
}

std::vector<float> get_map(hpm_ctx* ctx, int view, int kind, int& w, int& h) {
    check(ctx, hpm_get_map(ctx, view, kind, nullptr, 0, &w, &h), "hpm_get_map");
    std::vector<float> m((size_t)w * h * (kind == HPM_MAP_NORMAL ? 3 : 1));
    check(ctx, hpm_get_map(ctx, view, kind, m.data(), m.size(), &w, &h), "hpm_get_map");
    return m;
}

// camera scaled to a w x h map of an image of the original size (RescaleImageAndCamera, HPM.cpp:186-207)
hpm_camera scaled_camera(hpm_camera c, int orig_w, int orig_h, int w, int h) {
    if (w != orig_w || h != orig_h) {
        const float sx = w / static_cast<float>(orig_w), sy = h / static_cast<float>(orig_h);
        c.K[0] *= sx; c.K[2] *= sx; c.K[4] *= sy; c.K[5] *= sy;
    }
    c.width = w;
    c.height = h;
    return c;
}

}  // namespace

int main(int argc, char** argv) {
    const auto t0 = std::chrono::steady_clock::now();
    if (argc < 2) {
        std::cout << "USAGE: HPM-MVS_plusplus dense_folder [--initial-image-scale N] "
                     "[--show-medium-result] [--mask] [--fusion-only/--fuse]\n"
                     "  --initial-image-scale N: downscale width and height by N before pyramid processing "
                     "(default 4)\n"
                     "  --show-medium-result: also keep costs.dmb and confidence.dmb; depth/normal maps are always "
                     "kept."
                  << std::endl;
        return -1;
    }
    const std::string folder = argv[1];
    bool mask_flag = false, fuse_only = false, show_medium = false, per_problem = false;
    int scale = 4;
    try {
        for (int a = 2; a < argc;) {
            const std::string opt(argv[a++]);
            if (opt == "--mask") mask_flag = true;
            else if (opt == "--fusion-only" || opt == "--fuse") fuse_only = true;
            else if (opt == "--show-medium-result") show_medium = true;
            else if (opt == "--per-problem") per_problem = true;
            else if (opt == "--initial-image-scale" && a < argc) {
                const std::string v(argv[a++]);
                size_t parsed = 0;
                scale = std::stoi(v, &parsed);
                if (parsed != v.size() || scale < 1)
                    throw std::invalid_argument("--initial-image-scale must be a positive integer (1 = original resolution)");
            } else {
                throw std::invalid_argument("unknown or incomplete option: " + opt);
            }
        }
    } catch (const std::exception& e) {
        std::cerr << e.what() << std::endl;
        return EXIT_FAILURE;
    }

    hpm_ctx* ctx = nullptr;
    try {
        const std::vector<Problem> problems = read_pair(folder + "/pair.txt");
        if (problems.empty()) throw std::runtime_error("cannot read " + folder + "/pair.txt");
        const int n = (int)problems.size();
        if (n > HPM_MAX_VIEWS - 1) throw std::runtime_error("too many views for one context");
        std::vector<int32_t> src_off(1, 0), src_ids;
        for (int i = 0; i < n; ++i) {
            if (problems[i].ref_image_id != i)
                throw std::runtime_error("pair.txt lists image " + std::to_string(problems[i].ref_image_id) +
                                         " at position " + std::to_string(i) +
                                         "; images must be numbered 0..n-1 in order, as the reference assumes");
            for (int s : problems[i].src_image_ids) {
                if (s < 0 || s >= n) throw std::runtime_error("pair.txt: source id out of range");
                src_ids.push_back(s);
            }
            src_off.push_back((int32_t)src_ids.size());
        }
        std::cout << "There are " << n << " problems needed to be processed!" << std::endl;
        if (per_problem) ctx = HPM::context();
        else check(ctx, hpm_create(0, &ctx), "hpm_create");
        std::vector<hpm_camera> cams(n);
        std::vector<Image> images(n);
        for (int i = 0; i < n; ++i) {
            const std::string img_path = folder + "/images/" + id8(i) + ".jpg";
            if (!load_image(img_path, images[i])) throw std::runtime_error("cannot read " + img_path);
            if (!read_camera(folder + "/cams/" + id8(i) + "_cam.txt", &cams[i]))
                throw std::runtime_error("cannot read " + folder + "/cams/" + id8(i) + "_cam.txt");
            cams[i].width = images[i].w;
            cams[i].height = images[i].h;
            if (!per_problem)
                check(ctx, hpm_set_image(ctx, i, images[i].bgr.data(), images[i].w, images[i].h), "hpm_set_image");
        }
        const std::string out_folder = folder + "/HPM_MVS_plusplus";
        mkdir(out_folder.c_str(), 0755);

        if (fuse_only) {
            std::cout << "Fuse-only mode: skip MVS pipeline, run fusion with existing files." << std::endl;
            for (int i = 0; i < n; ++i) {
                const std::string dir = out_folder + "/2333_" + id8(i);
                std::vector<float> depth, normal;
                int w, h, c, wn, hn, cn;
                if (!read_dmb(dir + "/depths_geom.dmb", depth, w, h, c) || c != 1)
                    throw std::runtime_error("cannot read " + dir + "/depths_geom.dmb");
                if (!read_dmb(dir + "/normals.dmb", normal, wn, hn, cn) || cn != 3 || wn != w || hn != h)
                    throw std::runtime_error("cannot read " + dir + "/normals.dmb");
                const hpm_camera sc = scaled_camera(cams[i], images[i].w, images[i].h, w, h);
                check(ctx, hpm_prepare_level(ctx, i, w, h, &sc), "hpm_prepare_level");
                check(ctx, hpm_set_map(ctx, i, HPM_MAP_DEPTH_GEOM, depth.data(), w, h), "hpm_set_map");
                check(ctx, hpm_set_map(ctx, i, HPM_MAP_NORMAL, normal.data(), w, h), "hpm_set_map");
            }
        } else {
            std::cout << "Initial image scale: 1/" << scale << std::endl;
            hpm_recon_options opt{};
            opt.initial_image_scale = scale;
            opt.geom_iterations = 3;
            opt.fuse = 0;
            opt.level_max_side = 0;
            // the reference seeds from the clock (HPM.cu:579); HPM_SEED fixes the streams for reproducible runs
            opt.seed = (uint64_t)std::chrono::steady_clock::now().time_since_epoch().count();
            if (const char* env = std::getenv("HPM_SEED")) opt.seed = std::strtoull(env, nullptr, 10);
            if (const char* env = std::getenv("HPM_LEVEL_MAX_SIDE")) opt.level_max_side = std::atoi(env);
            if (per_problem) {
                run_per_problem(folder, problems, scale, opt.seed, opt.level_max_side, src_off, src_ids);
                if (!show_medium)  // RemoveIntermediateResults (main.cpp:1111-1141)
                    for (int i = 0; i < n; ++i) {
                        const std::string dir = out_folder + "/2333_" + id8(i);
                        std::remove((dir + "/costs.dmb").c_str());
                        std::remove((dir + "/confidence.dmb").c_str());
                        for (int k = 0; k < 8; ++k) std::remove((dir + "/texture" + std::to_string(k) + ".dmb").c_str());
                    }
            } else {
                int64_t unused = 0;
                check(ctx, hpm_reconstruct(ctx, n, cams.data(), src_off.data(), src_ids.data(), &opt, &unused),
                      "hpm_reconstruct");
            }
            for (int i = 0; i < n && !per_problem; ++i) {
                const std::string dir = out_folder + "/2333_" + id8(i);
                mkdir(dir.c_str(), 0755);
                int w, h;
                struct Out { int kind; const char* name; bool medium; };
                const Out outs[] = { { HPM_MAP_DEPTH, "depths.dmb", false }, { HPM_MAP_DEPTH_GEOM, "depths_geom.dmb", false },
                                     { HPM_MAP_NORMAL, "normals.dmb", false }, { HPM_MAP_COST, "costs.dmb", true },
                                     { HPM_MAP_CONF, "confidence.dmb", true } };
                for (const Out& o : outs) {
                    if (o.medium && !show_medium) continue;
                    const std::vector<float> m = get_map(ctx, i, o.kind, w, h);
                    if (!write_dmb(dir + "/" + o.name, m.data(), w, h, o.kind == HPM_MAP_NORMAL ? 3 : 1))
                        throw std::runtime_error("cannot write " + dir + "/" + o.name);
                }
            }
        }

        // fusion (RunFusion / RunFusion_Sky_Strict), with the masks resized to the map size on the GPU
        std::vector<std::vector<uint8_t>> masks;
        std::vector<const uint8_t*> mask_ptrs;
        if (mask_flag) {
            const int scratch_view = HPM_MAX_VIEWS - 1;
            for (int i = 0; i < n; ++i) {
                Image m;
                const std::string path = folder + "/masks/" + id8(i) + ".jpg";
                if (!load_image(path, m)) throw std::runtime_error("cannot read " + path);
                int w, h;
                (void)get_map(ctx, i, HPM_MAP_DEPTH_GEOM, w, h);
                check(ctx, hpm_set_image(ctx, scratch_view, m.bgr.data(), m.w, m.h), "hpm_set_image");
                const hpm_camera sc = scaled_camera(cams[i], m.w, m.h, w, h);
                check(ctx, hpm_prepare_level(ctx, scratch_view, w, h, &sc), "hpm_prepare_level");
                masks.emplace_back((size_t)w * h * 3);
                check(ctx, hpm_get_level(ctx, scratch_view, masks.back().data(), nullptr, nullptr), "hpm_get_level");
            }
            for (auto& m : masks) mask_ptrs.push_back(m.data());
        }
        int64_t n_points = 0;
        check(ctx, hpm_fuse(ctx, n, src_off.data(), src_ids.data(), HPM_MAP_DEPTH_GEOM,
                            mask_flag ? mask_ptrs.data() : nullptr, nullptr, 0, &n_points),
              "hpm_fuse");
        std::vector<hpm_point> pts((size_t)n_points);
        if (n_points > 0) check(ctx, hpm_get_points(ctx, pts.data(), n_points, nullptr), "hpm_get_points");
        if (!write_points_ply(out_folder + "/HPM_MVS_plusplus.ply", pts.data(), pts.size()))
            throw std::runtime_error("cannot write HPM_MVS_plusplus.ply");
        size_t fused = 0;
        if (!write_fused_ply(out_folder + "/fused.ply", pts.data(), pts.size(), &fused))
            throw std::runtime_error("cannot write fused.ply");
        std::cout << "Saved " << pts.size() << " points to " << out_folder << "/HPM_MVS_plusplus.ply and " << fused
                  << " with unit normals to " << out_folder << "/fused.ply" << std::endl;
    } catch (const std::exception& e) {
        std::cerr << e.what() << std::endl;
        if (per_problem) HPM::release_context();
        else if (ctx) hpm_destroy(ctx);
        return EXIT_FAILURE;
    }
    if (per_problem) HPM::release_context();
    else hpm_destroy(ctx);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::cout << "Total execution time: " << secs << " seconds" << std::endl;
    return 0;
}
