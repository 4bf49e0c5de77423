// Planar prior of a view (ProcessProblem's prior branch, main.cpp:349-597,
// with HPM.cpp:964-984, 1026-1206, 1433-1453) on the GPU:
//   support points per 5x5 block      k_support_blocks (block order kept)
//   Delaunay triangulation            host, delaunay.cpp
//   triangle raster, later wins       k_raster (atomicMax of the label)
//   3-point plane fits in double      k_plane_fit
//   prior depth and mask              k_prior_pixels / k_prior_small
//   distance > 0: float downsampling (k_resize_f32), prior JBU, reload
// Float arithmetic follows the host code of the reference (IEEE, no implicit
// contraction); the raster mixes float and double exactly as main.cpp:398-402.
#include "aux_kernels.cuh"
#include "ctx.hpp"

#include <algorithm>
#include <cmath>
#include <vector>

namespace hpm {

int delaunay_triangulate(const int32_t* xy, int n, int width, int height, std::vector<hpm_triangle>& out);

// cv::resize INTER_LINEAR of one float channel (the oracle's ora_resize_linear_f32):
// coordinates in double, each two-tap sum evaluated exactly and rounded once.
__global__ void k_resize_f32(const float* __restrict__ src, int sw, int sh, float* __restrict__ dst, int dw, int dh) {
    const int dx = blockIdx.x * blockDim.x + threadIdx.x;
    const int dy = blockIdx.y * blockDim.y + threadIdx.y;
    if (dx >= dw || dy >= dh) return;
    const double sxs = 1.0 / ((double)dw / sw), sys = 1.0 / ((double)dh / sh);
    const double fxd = (dx + 0.5) * sxs - 0.5;
    int sx = (int)floor(fxd);
    float fx = (float)(fxd - sx);
    if (sx < 0) { fx = 0; sx = 0; }
    if (sx >= sw - 1) { fx = 0; sx = sw - 1; }
    const int sx1 = sx + 1 < sw ? sx + 1 : sw - 1;
    const double fyd = (dy + 0.5) * sys - 0.5;
    int sy = (int)floor(fyd);
    float fy = (float)(fyd - sy);
    if (sy < 0) { fy = 0; sy = 0; }
    if (sy >= sh - 1) { fy = 0; sy = sh - 1; }
    const int sy1 = sy + 1 < sh ? sy + 1 : sh - 1;
    const float a0 = 1.0f - fx, a1 = fx, b0 = 1.0f - fy, b1 = fy;
    const float r0 = (float)((double)src[(size_t)sy * sw + sx] * a0 + (double)src[(size_t)sy * sw + sx1] * a1);
    const float r1 = (float)((double)src[(size_t)sy1 * sw + sx] * a0 + (double)src[(size_t)sy1 * sw + sx1] * a1);
    dst[(size_t)dy * dw + dx] = (float)((double)r0 * b0 + (double)r1 * b1);
}

// GetSupportPoints_Classify_Check (HPM.cpp:1026-1073): one thread per 5x5 block,
// blocks enumerated column-major as the reference loops (col outer, row inner).
// Slot 2b holds the "texture" point, 2b+1 the "no texture" point, (-1,-1) if none.
__global__ void k_support_blocks(const float* __restrict__ costs, const float* __restrict__ conf, int map_w,
                                 int width, int height, int2* __restrict__ slots) {
    const int nbr = (height + 4) / 5, nbc = (width + 4) / 5;
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbr * nbc) return;
    const int col = (b / nbr) * 5, row = (b % nbr) * 5;
    float min_nt = 2.0f, min_t = 2.0f;
    int2 pnt = make_int2(0, 0), pt = make_int2(0, 0);
    const int cb = min(width, col + 5), rb = min(height, row + 5);
    for (int c = col; c < cb; ++c)
        for (int r = row; r < rb; ++r) {
            const float pc = costs[(size_t)r * map_w + c];
            const float cf = conf[(size_t)r * map_w + c];
            if (pc < 2.0f) {
                const float f_nt = pc - cf;
                const float f_t = (float)(pc + 0.2 - cf);
                if (min_nt > f_nt) { pnt = make_int2(c, r); min_nt = f_nt; }
                if (min_t > f_t) { pt = make_int2(c, r); min_t = f_t; }
            }
        }
    slots[2 * b] = min_t < 0.1 ? pt : make_int2(-1, -1);
    slots[2 * b + 1] = min_nt < 0.1 ? pnt : make_int2(-1, -1);
}

// Barycentric stepping raster of main.cpp:391-404; labels idx+1, the later
// triangle wins, so the label is the maximum over the triangles covering a pixel.
// The positions visited are those of the reference's loops,
//   for (float p = 0; p < 1.0; p += step) for (float q = 0; q < 1.0 - p; q += step),
// step = 1 / (longest edge): about L^2 / 2 of them for a triangle with longest
// edge L, from a few for the triangles between neighbouring support points to
// hundreds of thousands for the ones spanning textureless regions.  Small
// triangles take one warp each (rows p_k to lanes k mod 32); large ones a block
// each, with the float sequence 0, step, 2 step, ... (the same for p and q)
// tabulated once in shared memory.
__device__ __forceinline__ float raster_step(const hpm_triangle& T) {
    const double d01 = (double)(T.x1 - T.x2) * (T.x1 - T.x2) + (double)(T.y1 - T.y2) * (T.y1 - T.y2);
    const double d02 = (double)(T.x1 - T.x3) * (T.x1 - T.x3) + (double)(T.y1 - T.y3) * (T.y1 - T.y3);
    const double d12 = (double)(T.x2 - T.x3) * (T.x2 - T.x3) + (double)(T.y2 - T.y3) * (T.y2 - T.y3);
    const float L01 = (float)sqrt(d01), L02 = (float)sqrt(d02), L12 = (float)sqrt(d12);
    const float mx = fmaxf(L01, fmaxf(L02, L12));
    return (float)(1.0 / mx);
}

__device__ __forceinline__ void raster_point(const hpm_triangle& T, float p, float q, int width, int lab,
                                             int* __restrict__ label) {
    const int x = (int)((double)(p * T.x1 + q * T.x2) + (1.0 - p - q) * T.x3);
    const int y = (int)((double)(p * T.y1 + q * T.y2) + (1.0 - p - q) * T.y3);
    atomicMax(&label[(size_t)y * width + x], lab);
}

__global__ void k_raster(const hpm_triangle* __restrict__ tris, const int32_t* __restrict__ small, int n_small,
                         int width, int* __restrict__ label) {
    const int w = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (w >= n_small) return;
    const int t = small[w];
    const hpm_triangle T = tris[t];
    const float step = raster_step(T);
    int k = 0;
    for (float p = 0; p < 1.0; p += step, ++k) {
        if ((k & 31) != lane) continue;
        for (float q = 0; q < 1.0 - p; q += step) raster_point(T, p, q, width, t + 1, label);
    }
}

constexpr int kRasterSeq = 8192;  // longest tabulated step sequence (longest edge up to 8190 px)

__global__ void k_raster_big(const hpm_triangle* __restrict__ tris, const int32_t* __restrict__ big, int width,
                             int* __restrict__ label) {
    __shared__ float seq[kRasterSeq];
    __shared__ int len;
    const int t = big[blockIdx.x];
    const hpm_triangle T = tris[t];
    const float step = raster_step(T);
    if (threadIdx.x == 0) {
        int k = 0;
        for (float v = 0; v < 1.0 && k < kRasterSeq; v += step) seq[k++] = v;
        len = k;
    }
    __syncthreads();
    for (int k = 0; k < len; ++k) {
        const float p = seq[k];
        for (int m = threadIdx.x; m < len && seq[m] < 1.0 - p; m += blockDim.x)
            raster_point(T, p, seq[m], width, t + 1, label);
    }
}

// 3-point plane in the camera frame (HPM.cpp:1099-1167): the unit-normal null
// vector of [X Y Z 1] from 3x3 cofactors in double, sign such that w >= 0.
__global__ void k_plane_fit(const hpm_triangle* __restrict__ tris, int n, const float* __restrict__ depths, int width,
                            hpm_camera cam, float factor, int use_factor, float4* __restrict__ planes) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const hpm_triangle T = tris[t];
    const int xs[3] = { T.x1, T.x2, T.x3 }, ys[3] = { T.y1, T.y2, T.y3 };
    double a[3][4];
    for (int k = 0; k < 3; ++k) {
        const float d = depths[(size_t)ys[k] * width + xs[k]];
        float X, Y;
        if (!use_factor) {
            X = d * (xs[k] - cam.K[2]) / cam.K[0];
            Y = d * (ys[k] - cam.K[5]) / cam.K[4];
        } else {
            X = d * (xs[k] - cam.K[2] * factor) / (cam.K[0] * factor);
            Y = d * (ys[k] - cam.K[5] * factor) / (cam.K[4] * factor);
        }
        a[k][0] = X; a[k][1] = Y; a[k][2] = d; a[k][3] = 1.0;
    }
    double v[4];
    for (int k = 0; k < 4; ++k) {
        int ci[3], m = 0;
        for (int q = 0; q < 4; ++q) if (q != k) ci[m++] = q;
        const double det = a[0][ci[0]] * (a[1][ci[1]] * a[2][ci[2]] - a[1][ci[2]] * a[2][ci[1]]) -
                           a[0][ci[1]] * (a[1][ci[0]] * a[2][ci[2]] - a[1][ci[2]] * a[2][ci[0]]) +
                           a[0][ci[2]] * (a[1][ci[0]] * a[2][ci[1]] - a[1][ci[1]] * a[2][ci[0]]);
        v[k] = (k % 2 == 0) ? det : -det;
    }
    double nrm = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (v[3] < 0) nrm = -nrm;
    planes[t] = make_float4((float)(v[0] / nrm), (float)(v[1] / nrm), (float)(v[2] / nrm), (float)(v[3] / nrm));
}

// distance 0 (main.cpp:411-424 + HPM.cpp:964-984): prior plane and mask per pixel.
__global__ void k_prior_pixels(const int* __restrict__ label, const float4* __restrict__ planes, int W, int H,
                               hpm_camera cam, float dmin, float dmax, float4* __restrict__ prior,
                               uint8_t* __restrict__ mask, float* __restrict__ prior_depth) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const size_t c = (size_t)y * W + x;
    const int lab = label[c];
    float4 pl = make_float4(0.f, 0.f, 0.f, 0.f);
    uint8_t m = 0;
    float pd = 0.0f;
    if (lab > 0) {
        const float4 P = planes[lab - 1];
        const float d = -P.w * cam.K[0] / ((x - cam.K[2]) * P.x + (cam.K[0] / cam.K[4]) * (y - cam.K[5]) * P.y + cam.K[0] * P.z);
        if (d <= dmax && d >= dmin) { pl = P; m = 1; pd = d; }
    }
    prior[c] = pl;
    mask[c] = m;
    if (prior_depth) prior_depth[c] = pd;
}

// distance > 0 (main.cpp:516-535): prior depth and world normal at the reduced size.
__global__ void k_prior_small(const int* __restrict__ label, const float4* __restrict__ planes, int w, int h,
                              hpm_camera cam, float factor, float dmin, float dmax, float* __restrict__ pdepth,
                              float* __restrict__ pnormal) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t c = (size_t)y * w + x;
    const int lab = label[c];
    float d0 = 0.f, n0 = 0.f, n1 = 0.f, n2 = 0.f;
    if (lab > 0) {
        const float4 P = planes[lab - 1];
        const float d = -P.w * (cam.K[0] * factor) /
                        ((x - cam.K[2] * factor) * P.x + (cam.K[0] / cam.K[4]) * (y - cam.K[5] * factor) * P.y +
                         cam.K[0] * factor * P.z);
        if (d <= dmax * 1.2f && d >= dmin * 0.6f) {
            d0 = d;
            n0 = cam.R[0] * P.x + cam.R[3] * P.y + cam.R[6] * P.z;
            n1 = cam.R[1] * P.x + cam.R[4] * P.y + cam.R[7] * P.z;
            n2 = cam.R[2] * P.x + cam.R[5] * P.y + cam.R[8] * P.z;
        }
    }
    pdepth[c] = d0;
    pnormal[3 * c] = n0;
    pnormal[3 * c + 1] = n1;
    pnormal[3 * c + 2] = n2;
}

// main.cpp:548-570 + HPM.cpp:1433-1453: upsampled prior -> camera-frame planes.
__global__ void k_prior_reload(const float* __restrict__ udepth, const float* __restrict__ unormal, int W, int H,
                               hpm_camera cam, float dmin, float dmax, float4* __restrict__ prior,
                               uint8_t* __restrict__ mask) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const size_t c = (size_t)y * W + x;
    const float d = udepth[c];
    float4 pl = make_float4(0.f, 0.f, 0.f, 0.f);
    uint8_t m = 0;
    if (d <= dmax && d >= dmin) {
        const float a = unormal[3 * c], b = unormal[3 * c + 1], e = unormal[3 * c + 2];
        pl.x = cam.R[0] * a + cam.R[1] * b + cam.R[2] * e;
        pl.y = cam.R[3] * a + cam.R[4] * b + cam.R[5] * e;
        pl.z = cam.R[6] * a + cam.R[7] * b + cam.R[8] * e;
        const float X0 = d * (x - cam.K[2]) / (cam.K[0]);
        const float X1 = d * (y - cam.K[5]) / (cam.K[4]);
        pl.w = -(pl.x * X0 + pl.y * X1 + pl.z * d);
        m = 1;
    }
    prior[c] = pl;
    mask[c] = m;
}

template <class T>
static cudaError_t ensure_p(T*& p, size_t& cap, size_t n) {
    if (n <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) cap = n;
    return e;
}

// Downsampled depth, cost and confidence of a view for prior distance > 0
// (cv::resize INTER_LINEAR, main.cpp:444-454) into prior_small.
int Ctx::prior_downsample(int view, int distance, int& hw, int& hh) {
    ViewState& v = views[view];
    const int W = v.w, H = v.h;
    const float f = 1.0f / (distance * 2);
    hw = (int)std::round(W * f);
    hh = (int)std::round(H * f);
    cudaError_t e = ensure_p(prior_small, prior_small_cap, (size_t)hw * hh * 3);
    if (e != cudaSuccess) return cuda_fail(e, "alloc prior buffers");
    float* dd = prior_small;
    float* dc = dd + (size_t)hw * hh;
    float* df = dc + (size_t)hw * hh;
    dim3 b(32, 8), g((hw + 31) / 32, (hh + 7) / 8);
    k_resize_f32<<<g, b, 0, stream>>>(v.maps[HPM_MAP_DEPTH].ptr, W, H, dd, hw, hh);
    k_resize_f32<<<g, b, 0, stream>>>(v.maps[HPM_MAP_COST].ptr, W, H, dc, hw, hh);
    k_resize_f32<<<g, b, 0, stream>>>(v.maps[HPM_MAP_CONF].ptr, W, H, df, hw, hh);
    launches += 3;
    return HPM_OK;
}

int Ctx::support_points(int view, int distance, std::vector<int32_t>& xy, int& sup_w, int& sup_h) {
    cudaSetDevice(device);
    ViewState& v = views[view];
    const int W = v.w, H = v.h;
    const DevMap& dm = v.maps[HPM_MAP_DEPTH];
    const DevMap& cm = v.maps[HPM_MAP_COST];
    const DevMap& fm = v.maps[HPM_MAP_CONF];
    if (!dm.ptr || !cm.ptr || !fm.ptr || dm.w != W || dm.h != H || cm.w != W || cm.h != H || fm.w != W || fm.h != H)
        return fail(HPM_E_STATE, "view %d lacks depth/cost/confidence maps of its size", view);
    const float* costs = cm.ptr;
    const float* conf = fm.ptr;
    int map_w = W, width = W, height = H;
    cudaError_t e;
    if (distance > 0) {
        int hw = 0, hh = 0;
        int rc = prior_downsample(view, distance, hw, hh);
        if (rc) return rc;
        const float f = 1.0f / (distance * 2);
        costs = prior_small + (size_t)hw * hh;
        conf = costs + (size_t)hw * hh;
        map_w = hw;
        width = (int)(W * f);   // GetReferenceImageWidth() * hpm_factor, truncated (HPM.cpp:1030-1031)
        height = (int)(H * f);
        sup_w = hw;
        sup_h = hh;
    } else {
        sup_w = W;
        sup_h = H;
    }
    const int nb = ((width + 4) / 5) * ((height + 4) / 5);
    e = ensure_p(scratch, scratch_cap, (size_t)nb * 16 + 256);
    if (e != cudaSuccess) return cuda_fail(e, "alloc support slots");
    int2* slots = reinterpret_cast<int2*>(scratch);
    k_support_blocks<<<(nb + 127) / 128, 128, 0, stream>>>(costs, conf, map_w, width, height, slots);
    ++launches;
    std::vector<int2> hs((size_t)nb * 2);
    e = cudaMemcpyAsync(hs.data(), slots, sizeof(int2) * hs.size(), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "download support points");
    xy.clear();
    for (const int2& s : hs)
        if (s.x >= 0) { xy.push_back(s.x); xy.push_back(s.y); }
    return HPM_OK;
}

int Ctx::prior_from_triangles(int view, int distance, const hpm_triangle* tris, int n_tris, int sup_w, int sup_h) {
    cudaSetDevice(device);
    ViewState& v = views[view];
    const int W = v.w, H = v.h;
    // triangles with all vertices inside the (reduced) image rectangle, in order (main.cpp:389-390)
    std::vector<hpm_triangle> acc;
    acc.reserve(n_tris);
    for (int t = 0; t < n_tris; ++t) {
        const hpm_triangle& T = tris[t];
        const int xs[3] = { T.x1, T.x2, T.x3 }, ys[3] = { T.y1, T.y2, T.y3 };
        bool in = true;
        for (int k = 0; k < 3; ++k) in = in && xs[k] >= 0 && xs[k] < sup_w && ys[k] >= 0 && ys[k] < sup_h;
        if (in) acc.push_back(T);
    }
    const int na = (int)acc.size();
    const size_t nsmall = (size_t)sup_w * sup_h;
    // triangles (24 bytes each) then the float4 planes at a 256-byte aligned offset
    const size_t planes_off = ((size_t)std::max(na, 1) * sizeof(hpm_triangle) + 255) & ~size_t(255);
    const size_t lists_off = planes_off + (((size_t)std::max(na, 1) * 16 + 255) & ~size_t(255));
    // raster work lists: triangles whose longest edge is at most kSmallEdge go one per warp,
    // the others one per block (same float step as the kernel: double lengths, float max)
    const float kSmallEdge = 64.0f;
    std::vector<int32_t> lists((size_t)std::max(na, 1));
    int n_small = 0, n_big = 0;
    for (int t = 0; t < na; ++t) {
        const hpm_triangle& T = acc[t];
        const double d01 = (double)(T.x1 - T.x2) * (T.x1 - T.x2) + (double)(T.y1 - T.y2) * (T.y1 - T.y2);
        const double d02 = (double)(T.x1 - T.x3) * (T.x1 - T.x3) + (double)(T.y1 - T.y3) * (T.y1 - T.y3);
        const double d12 = (double)(T.x2 - T.x3) * (T.x2 - T.x3) + (double)(T.y2 - T.y3) * (T.y2 - T.y3);
        const float mx = std::max((float)std::sqrt(d01), std::max((float)std::sqrt(d02), (float)std::sqrt(d12)));
        // (edges beyond the block kernel's table stay on the warp path, slow but exact)
        if (mx <= kSmallEdge || mx > (float)(kRasterSeq - 8)) lists[n_small++] = t;
        else lists[na - 1 - n_big++] = t;
    }
    cudaError_t e = ensure_p(prior_tris, prior_tris_cap, lists_off + (size_t)std::max(na, 1) * 4);
    if (e != cudaSuccess) return cuda_fail(e, "alloc triangles");
    hpm_triangle* d_tris = reinterpret_cast<hpm_triangle*>(prior_tris);
    float4* d_planes = reinterpret_cast<float4*>(prior_tris + planes_off);
    e = ensure_p(prior_label, prior_label_cap, nsmall);
    if (e != cudaSuccess) return cuda_fail(e, "alloc labels");
    int32_t* d_lists = reinterpret_cast<int32_t*>(prior_tris + lists_off);
    if (na > 0) {
        e = cudaMemcpyAsync(d_tris, acc.data(), sizeof(hpm_triangle) * na, cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_lists, lists.data(), sizeof(int32_t) * na, cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return cuda_fail(e, "upload triangles");
    }
    cudaMemsetAsync(prior_label, 0, sizeof(int) * nsmall, stream);
    e = ensure_p(v.prior, v.prior_cap, (size_t)W * H);
    if (e == cudaSuccess) e = ensure_p(v.pmask, v.pmask_cap, (size_t)W * H);
    if (e != cudaSuccess) return cuda_fail(e, "alloc prior");
    const hpm_camera& cam = v.cam;
    const float dmin = cam.depth_min * 0.6f, dmax = cam.depth_max * 1.2f;  // params range (HPM.cpp:685-686)
    if (na > 0) {
        if (n_small > 0) {
            k_raster<<<(int)(((size_t)n_small * 32 + 255) / 256), 256, 0, stream>>>(d_tris, d_lists, n_small, sup_w,
                                                                                    prior_label);
            ++launches;
        }
        if (n_big > 0) {
            k_raster_big<<<n_big, 256, 0, stream>>>(d_tris, d_lists + (na - n_big), sup_w, prior_label);
            ++launches;
        }
    }
    if (distance == 0) {
        if (na > 0) {
            k_plane_fit<<<(na + 127) / 128, 128, 0, stream>>>(d_tris, na, v.maps[HPM_MAP_DEPTH].ptr, W, cam, 1.0f, 0,
                                                              d_planes);
            ++launches;
        }
        dim3 b(32, 8), g((W + 31) / 32, (H + 7) / 8);
        k_prior_pixels<<<g, b, 0, stream>>>(prior_label, d_planes, W, H, cam, dmin, dmax, v.prior, v.pmask, nullptr);
        ++launches;
    } else {
        const float f = 1.0f / (distance * 2);
        int hw = 0, hh = 0;
        int rc = prior_downsample(view, distance, hw, hh);
        if (rc) return rc;
        if (hw != sup_w || hh != sup_h) return fail(HPM_E_INVALID, "prior size %dx%d != %dx%d", sup_w, sup_h, hw, hh);
        float* dd = prior_small;  // downsampled depth
        e = ensure_p(prior_work, prior_work_cap, nsmall * 4 + (size_t)W * H * 4 + 64);
        if (e != cudaSuccess) return cuda_fail(e, "alloc prior work");
        float* pdepth = prior_work;
        float* pnormal = pdepth + nsmall;
        float* udepth = pnormal + 3 * nsmall;
        float* unormal_ = nullptr;
        e = ensure_p(prior_unormal, prior_unormal_cap, (size_t)W * H * 3);
        if (e != cudaSuccess) return cuda_fail(e, "alloc prior normals");
        unormal_ = prior_unormal;
        if (na > 0) {
            k_plane_fit<<<(na + 127) / 128, 128, 0, stream>>>(d_tris, na, dd, sup_w, cam, f, 1, d_planes);
            ++launches;
        }
        dim3 bs(32, 8), gs((sup_w + 31) / 32, (sup_h + 7) / 8);
        k_prior_small<<<gs, bs, 0, stream>>>(prior_label, d_planes, sup_w, sup_h, cam, f, dmin, dmax, pdepth, pnormal);
        ++launches;
        const int scale = std::max(H / sup_h, W / sup_w);
        if (scale == 1) {
            // JointBilateralUpsampling_prior returns early; the outputs stay zero (HPM.cpp:1328-1331)
            cudaMemsetAsync(udepth, 0, sizeof(float) * W * H, stream);
            cudaMemsetAsync(unormal_, 0, sizeof(float) * W * H * 3, stream);
        } else {
            e = launch_jbu_prior(v.gray, W, H, pdepth, pnormal, sup_w, sup_h, udepth, unormal_, stream);
            if (e != cudaSuccess) return cuda_fail(e, "prior JBU");
            ++launches;
        }
        dim3 b(32, 8), g((W + 31) / 32, (H + 7) / 8);
        k_prior_reload<<<g, b, 0, stream>>>(udepth, unormal_, W, H, cam, dmin, dmax, v.prior, v.pmask);
        ++launches;
    }
    v.prior_w = W;
    v.prior_h = H;
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "prior kernels");
    return HPM_OK;
}

int Ctx::build_prior(int view, int distance, int* n_points, int* n_triangles) {
    if (view < 0 || view >= HPM_MAX_VIEWS || views[view].w == 0) return fail(HPM_E_STATE, "view %d not set", view);
    if (distance < 0 || distance > 2) return fail(HPM_E_INVALID, "prior scale distance must be 0, 1 or 2");
    const DevMap& dm = views[view].maps[HPM_MAP_DEPTH];
    if (!dm.ptr || dm.w != views[view].w || dm.h != views[view].h)
        return fail(HPM_E_STATE, "view %d lacks a depth map of its size", view);
    std::vector<int32_t> xy;
    int sw = 0, sh = 0;
    int rc = support_points(view, distance, xy, sw, sh);
    if (rc) return rc;
    std::vector<hpm_triangle> tris;
    delaunay_triangulate(xy.data(), (int)xy.size() / 2, sw, sh, tris);
    if (n_points) *n_points = (int)xy.size() / 2;
    if (n_triangles) *n_triangles = (int)tris.size();
    return prior_from_triangles(view, distance, tris.data(), (int)tris.size(), sw, sh);
}

}  // namespace hpm
