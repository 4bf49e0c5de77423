// CHECKER ONLY: drives the reference's own CUDA code (HPM.cu of HPM-MVS++,
// compiled from its sources by oracle/ref_build.mk with the reference's flags)
// on in-memory inputs.  It fills the members of an `HPM` object the way
// HPM::CudaSpaceInitialization and friends do (HPM.cpp:741-984: one float
// cudaArray per view with linear filtering and wrap addressing, per-pixel
// buffers) and calls HPM::RunPatchMatch() (HPM.cu:2987-3035) unchanged.
// Random draws come from oracle/ref_shim/ref_rng.h.  Used by
// tests/test_ref_build.py and the reference-CUDA timing of bench.py.
#define private public
#include "HPM.h"
#undef private

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

extern __device__ unsigned long long g_ref_seed;
extern __device__ unsigned int g_ref_view;

// HPM.cpp is not compiled (it needs OpenCV I/O); the three symbols of it that
// HPM.cu links against are supplied here.
void CudaSafeCall(const cudaError_t error, const std::string& file, const int line) {
    if (error != cudaSuccess) fprintf(stderr, "reference CUDA error %s at %s:%d\n", cudaGetErrorString(error), file.c_str(), line);
}

HPM::HPM() {
    num_images = 0;
    plane_hypotheses_host = scaled_plane_hypotheses_host = prior_planes_host = nullptr;
    costs_host = pre_costs_host = confidences_host = texture_host = nullptr;
    plane_masks_host = nullptr;
    cameras_cuda = nullptr;
    texture_objects_cuda = texture_depths_cuda = nullptr;
    plane_hypotheses_cuda = scaled_plane_hypotheses_cuda = prior_planes_cuda = nullptr;
    costs_cuda = pre_costs_cuda = depths_cuda = confidences_cuda = texture_cuda = nullptr;
    rand_states_cuda = nullptr;
    selected_views_cuda = plane_masks_cuda = Canny_cuda = nullptr;
    memset(&params, 0, sizeof(params));
}

HPM::~HPM() {
    for (int i = 0; i < num_images; ++i) {
        cudaDestroyTextureObject(texture_objects_host.images[i]);
        cudaFreeArray(cuArray[i]);
        if (params.geom_consistency) {
            cudaDestroyTextureObject(texture_depths_host.images[i]);
            cudaFreeArray(cuDepthArray[i]);
        }
    }
    delete[] plane_hypotheses_host;
    delete[] scaled_plane_hypotheses_host;
    delete[] prior_planes_host;
    delete[] costs_host;
    delete[] pre_costs_host;
    delete[] confidences_host;
    delete[] texture_host;
    delete[] plane_masks_host;
    void* dev[] = {cameras_cuda, texture_objects_cuda, texture_depths_cuda, plane_hypotheses_cuda,
                   scaled_plane_hypotheses_cuda, prior_planes_cuda, costs_cuda, pre_costs_cuda, depths_cuda,
                   confidences_cuda, texture_cuda, rand_states_cuda, selected_views_cuda, plane_masks_cuda, Canny_cuda};
    for (void* d : dev) cudaFree(d);
}

// plain-C mirror of the PatchMatchParams fields the reference reads
struct RefParams {
    int max_iterations, patch_size, num_images, radius_increment;
    float sigma_spatial, sigma_color;
    int top_k;
    float depth_min, depth_max;
    int scaled_cols, scaled_rows;
    unsigned int mode;  // hpm_types.h HPM_MODE_* bits
};

static void make_texture(const float* host, int w, int h, cudaArray** arr, cudaTextureObject_t* tex,
                         cudaTextureAddressMode mode = cudaAddressModeWrap) {
    cudaChannelFormatDesc fd = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    cudaMallocArray(arr, &fd, w, h);
    cudaMemcpy2DToArray(*arr, 0, 0, host, sizeof(float) * w, sizeof(float) * w, h, cudaMemcpyHostToDevice);
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = *arr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = mode;
    td.addressMode[1] = mode;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaCreateTextureObject(tex, &rd, &td, nullptr);
}

static void fill_params(PatchMatchParams& p, const RefParams* rp, int num_images) {
    p.max_iterations = rp->max_iterations;
    p.patch_size = rp->patch_size;
    p.num_images = num_images;
    p.radius_increment = rp->radius_increment;
    p.sigma_spatial = rp->sigma_spatial;
    p.sigma_color = rp->sigma_color;
    p.top_k = rp->top_k;
    p.depth_min = rp->depth_min;
    p.depth_max = rp->depth_max;
    p.scaled_cols = (float)rp->scaled_cols;
    p.scaled_rows = (float)rp->scaled_rows;
    p.geom_consistency = rp->mode & 1u;
    p.prior_consistency = rp->mode & 2u;
    p.multi_geometry = rp->mode & 4u;
    p.hierarchy = rp->mode & 8u;
    p.upsample = rp->mode & 16u;
    p.mand_consistency = rp->mode & 32u;
}

__global__ void RandomInitialization(cudaTextureObjects* texture_objects, Camera* cameras, float4* plane_hypotheses,
                                     float4* scaled_plane_hypotheses, float* costs, float* pre_costs,
                                     curandState* rand_states, unsigned int* selected_views, float4* prior_planes,
                                     unsigned int* plane_masks, const PatchMatchParams params, float* confidences,
                                     unsigned int* Canny, float* texture);

__global__ void BlackPixelUpdate(cudaTextureObjects* texture_objects, cudaTextureObjects* texture_depths,
                                 Camera* cameras, float4* plane_hypotheses, float* costs, float* pre_costs,
                                 curandState* rand_states, unsigned int* selected_views, float4* prior_planes,
                                 unsigned int* plane_masks, const PatchMatchParams params, const int iter,
                                 float* confidences, unsigned int* Canny);
__global__ void RedPixelUpdate(cudaTextureObjects* texture_objects, cudaTextureObjects* texture_depths,
                               Camera* cameras, float4* plane_hypotheses, float* costs, float* pre_costs,
                               curandState* rand_states, unsigned int* selected_views, float4* prior_planes,
                               unsigned int* plane_masks, const PatchMatchParams params, const int iter,
                               float* confidences, unsigned int* Canny);

// One view's run on an HPM object filled as CudaSpaceInitialization and friends
// fill it.  n_half < 0: HPM::RunPatchMatch unchanged.  n_half >= 0: the
// RandomInitialization kernel followed by the first n_half half-sweeps
// (Black, Red, Black, ...), launched as RunPatchMatch launches them
// (HPM.cu:2987-3021), with the planes left in the camera frame and the view
// masks returned in `selected`.
static int run_ref(const float* const* images, const Camera* cams, int num_images, const RefParams* rp, float* planes,
                   float* costs, const float* scaled_planes, const float* prior_planes,
                   const unsigned int* plane_masks, float* confidences, const unsigned int* canny, float* texture,
                   const float* const* depth_maps, unsigned long long seed, unsigned int view, float* elapsed_ms,
                   int n_half, unsigned int* selected) {
    const bool init_only = n_half >= 0;
    (void)cudaGetLastError();
    HPM hpm;
    const int W = cams[0].width, H = cams[0].height;
    const size_t n = (size_t)W * H;
    PatchMatchParams& p = hpm.params;
    fill_params(p, rp, num_images);
    hpm.num_images = num_images;
    hpm.cameras.assign(cams, cams + num_images);
    for (int i = 0; i < num_images; ++i)
        make_texture(images[i], cams[i].width, cams[i].height, &hpm.cuArray[i], &hpm.texture_objects_host.images[i]);
    cudaMalloc((void**)&hpm.texture_objects_cuda, sizeof(cudaTextureObjects));
    cudaMemcpy(hpm.texture_objects_cuda, &hpm.texture_objects_host, sizeof(cudaTextureObjects), cudaMemcpyHostToDevice);
    cudaMalloc((void**)&hpm.cameras_cuda, sizeof(Camera) * num_images);
    cudaMemcpy(hpm.cameras_cuda, cams, sizeof(Camera) * num_images, cudaMemcpyHostToDevice);
    hpm.plane_hypotheses_host = new float4[n];
    memcpy(hpm.plane_hypotheses_host, planes, sizeof(float4) * n);
    cudaMalloc((void**)&hpm.plane_hypotheses_cuda, sizeof(float4) * n);
    cudaMemcpy(hpm.plane_hypotheses_cuda, planes, sizeof(float4) * n, cudaMemcpyHostToDevice);
    hpm.costs_host = new float[n];
    cudaMalloc((void**)&hpm.costs_cuda, sizeof(float) * n);
    cudaMemcpy(hpm.costs_cuda, costs, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMalloc((void**)&hpm.pre_costs_cuda, sizeof(float) * n);
    cudaMalloc((void**)&hpm.rand_states_cuda, sizeof(curandState) * n);
    cudaMalloc((void**)&hpm.selected_views_cuda, sizeof(unsigned int) * n);
    cudaMemset(hpm.selected_views_cuda, 0, sizeof(unsigned int) * n);
    cudaMalloc((void**)&hpm.depths_cuda, sizeof(float) * n);
    if (p.geom_consistency) {
        for (int i = 0; i < num_images; ++i)
            make_texture(depth_maps[i], cams[i].width, cams[i].height, &hpm.cuDepthArray[i],
                         &hpm.texture_depths_host.images[i]);
        cudaMalloc((void**)&hpm.texture_depths_cuda, sizeof(cudaTextureObjects));
        cudaMemcpy(hpm.texture_depths_cuda, &hpm.texture_depths_host, sizeof(cudaTextureObjects), cudaMemcpyHostToDevice);
    }
    if (p.hierarchy) {
        const size_t ns = (size_t)rp->scaled_cols * rp->scaled_rows;
        hpm.scaled_plane_hypotheses_host = new float4[ns];
        hpm.pre_costs_host = new float[n];
        cudaMalloc((void**)&hpm.scaled_plane_hypotheses_cuda, sizeof(float4) * ns);
        cudaMemcpy(hpm.scaled_plane_hypotheses_cuda, scaled_planes, sizeof(float4) * ns, cudaMemcpyHostToDevice);
    }
    if (p.prior_consistency) {
        hpm.prior_planes_host = new float4[n];
        hpm.plane_masks_host = new unsigned int[n];
        cudaMalloc((void**)&hpm.prior_planes_cuda, sizeof(float4) * n);
        cudaMemcpy(hpm.prior_planes_cuda, prior_planes, sizeof(float4) * n, cudaMemcpyHostToDevice);
        cudaMalloc((void**)&hpm.plane_masks_cuda, sizeof(unsigned int) * n);
        cudaMemcpy(hpm.plane_masks_cuda, plane_masks, sizeof(unsigned int) * n, cudaMemcpyHostToDevice);
    }
    cudaMalloc((void**)&hpm.confidences_cuda, sizeof(float) * n);
    cudaMemcpy(hpm.confidences_cuda, confidences, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMalloc((void**)&hpm.Canny_cuda, sizeof(unsigned int) * n);
    cudaMemcpy(hpm.Canny_cuda, canny, sizeof(unsigned int) * n, cudaMemcpyHostToDevice);
    hpm.texture_host = new float[n];
    cudaMalloc((void**)&hpm.texture_cuda, sizeof(float) * n);
    cudaMemcpyToSymbol(g_ref_seed, &seed, sizeof(seed));
    cudaMemcpyToSymbol(g_ref_view, &view, sizeof(view));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a);
    if (init_only) {
        const dim3 grid((W + 15) / 16, (H + 15) / 16, 1), block(16, 16, 1);
        RandomInitialization<<<grid, block>>>(hpm.texture_objects_cuda, hpm.cameras_cuda, hpm.plane_hypotheses_cuda,
                                              hpm.scaled_plane_hypotheses_cuda, hpm.costs_cuda, hpm.pre_costs_cuda,
                                              hpm.rand_states_cuda, hpm.selected_views_cuda, hpm.prior_planes_cuda,
                                              hpm.plane_masks_cuda, hpm.params, hpm.confidences_cuda, hpm.Canny_cuda,
                                              hpm.texture_cuda);
        const dim3 cgrid((W + 31) / 32, ((H / 2) + 15) / 16, 1), cblock(32, 16, 1);
        for (int h = 0; h < n_half; ++h) {
            if (h % 2 == 0)
                BlackPixelUpdate<<<cgrid, cblock>>>(hpm.texture_objects_cuda, hpm.texture_depths_cuda,
                                                    hpm.cameras_cuda, hpm.plane_hypotheses_cuda, hpm.costs_cuda,
                                                    hpm.pre_costs_cuda, hpm.rand_states_cuda,
                                                    hpm.selected_views_cuda, hpm.prior_planes_cuda,
                                                    hpm.plane_masks_cuda, hpm.params, h / 2, hpm.confidences_cuda,
                                                    hpm.Canny_cuda);
            else
                RedPixelUpdate<<<cgrid, cblock>>>(hpm.texture_objects_cuda, hpm.texture_depths_cuda,
                                                  hpm.cameras_cuda, hpm.plane_hypotheses_cuda, hpm.costs_cuda,
                                                  hpm.pre_costs_cuda, hpm.rand_states_cuda, hpm.selected_views_cuda,
                                                  hpm.prior_planes_cuda, hpm.plane_masks_cuda, hpm.params, h / 2,
                                                  hpm.confidences_cuda, hpm.Canny_cuda);
        }
    } else {
        hpm.RunPatchMatch();
    }
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (elapsed_ms) *elapsed_ms = ms;
    if (init_only) {
        cudaMemcpy(planes, hpm.plane_hypotheses_cuda, sizeof(float4) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(costs, hpm.costs_cuda, sizeof(float) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(selected, hpm.selected_views_cuda, sizeof(unsigned int) * n, cudaMemcpyDeviceToHost);
        if (!p.mand_consistency && !p.prior_consistency)
            cudaMemcpy(texture, hpm.texture_cuda, sizeof(float) * n, cudaMemcpyDeviceToHost);
    } else {
        memcpy(planes, hpm.plane_hypotheses_host, sizeof(float4) * n);
        memcpy(costs, hpm.costs_host, sizeof(float) * n);
        if (!p.mand_consistency && !p.prior_consistency) memcpy(texture, hpm.texture_host, sizeof(float) * n);
    }
    cudaMemcpy(confidences, hpm.confidences_cuda, sizeof(float) * n, cudaMemcpyDeviceToHost);
    const cudaError_t err = cudaDeviceSynchronize();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return err == cudaSuccess ? 0 : (int)err;
}

extern "C" int ref_run_patchmatch(const float* const* images, const Camera* cams, int num_images, const RefParams* rp,
                                  float* planes, float* costs, const float* scaled_planes, const float* prior_planes,
                                  const unsigned int* plane_masks, float* confidences, const unsigned int* canny,
                                  float* texture, const float* const* depth_maps, unsigned long long seed,
                                  unsigned int view, float* elapsed_ms) {
    return run_ref(images, cams, num_images, rp, planes, costs, scaled_planes, prior_planes, plane_masks, confidences,
                   canny, texture, depth_maps, seed, view, elapsed_ms, -1, nullptr);
}

// The reference's RandomInitialization (HPM.cu:567-763) and its first n_half
// half-sweeps (HPM.cu:2793-2827): same arguments as ref_run_patchmatch plus
// the per-pixel view masks.
extern "C" int ref_random_init(const float* const* images, const Camera* cams, int num_images, const RefParams* rp,
                               float* planes, float* costs, const float* scaled_planes, const float* prior_planes,
                               const unsigned int* plane_masks, float* confidences, const unsigned int* canny,
                               float* texture, const float* const* depth_maps, unsigned long long seed,
                               unsigned int view, int n_half, unsigned int* selected) {
    if (!selected || n_half < 0 || n_half > 6) return -1;
    return run_ref(images, cams, num_images, rp, planes, costs, scaled_planes, prior_planes, plane_masks, confidences,
                   canny, texture, depth_maps, seed, view, nullptr, n_half, selected);
}

// ---------------------------------------------------------------------------
// Per-function probes: the reference's own __device__ functions (HPM.cu,
// linked through -rdc) evaluated at given (pixel, hypothesis) pairs, for the
// golden vectors that pin the oracle function by function.
__device__ void ComputeMultiViewCostVector(const cudaTextureObject_t* images, const Camera* cameras, const int2 p,
                                           const float4 plane_hypothesis, float* cost_vector,
                                           const PatchMatchParams params);
__device__ float ComputeMultiViewInitialCostandSelectedViews(const cudaTextureObject_t* images, const Camera* cameras,
                                                             const int2 p, const float4 plane_hypothesis,
                                                             unsigned int* selected_views,
                                                             const PatchMatchParams params);
__device__ float ComputeGeomConsistencyCost(const cudaTextureObject_t depth_image, const Camera ref_camera,
                                            const Camera src_camera, const float4 plane_hypothesis, const int2 p);
__device__ float ComputeDepthfromPlaneHypothesis(const Camera camera, const float4 plane_hypothesis, const int2 p);
__device__ float ComputeTexture(const unsigned int* Canny, const Camera* cameras, const int2 p);

// One thread per probe; cost_vec and geom hold 32 entries per probe (sources in order).
__global__ void k_ref_probe(const cudaTextureObjects* tex, const cudaTextureObjects* dtex, const Camera* cams,
                            const PatchMatchParams p, const unsigned int* canny, const int2* pix, const float4* planes,
                            int n, float* cost_vec, float* init_cost, unsigned int* sel, float* depth, float* geom,
                            float* texture) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int2 q = pix[i];
    const float4 pl = planes[i];
    float cv[32];
    ComputeMultiViewCostVector(tex->images, cams, q, pl, cv, p);
    for (int j = 0; j < p.num_images - 1; ++j) cost_vec[32 * i + j] = cv[j];
    unsigned int s = 0;
    init_cost[i] = ComputeMultiViewInitialCostandSelectedViews(tex->images, cams, q, pl, &s, p);
    sel[i] = s;
    depth[i] = ComputeDepthfromPlaneHypothesis(cams[0], pl, q);
    for (int j = 1; j < p.num_images; ++j)
        geom[32 * i + j - 1] = ComputeGeomConsistencyCost(dtex->images[j], cams[0], cams[j], pl, q);
    texture[i] = ComputeTexture(canny, cams, q);
}

// images / depth_maps: num_images float maps of each camera's size; canny: the
// reference's width*height; pix: n int2 inside the reference image; planes: n
// float4 (camera frame).  address_mode 0 = clamp, 1 = wrap (the reference's
// HPM.cpp:759-768).
extern "C" int ref_probe(const float* const* images, const float* const* depth_maps, const Camera* cams,
                         int num_images, const RefParams* rp, const unsigned int* canny, const int* pix,
                         const float* planes, int n, int address_mode, float* cost_vec, float* init_cost,
                         unsigned int* sel, float* depth, float* geom, float* texture) {
    (void)cudaGetLastError();
    if (num_images < 2 || num_images > 33 || n <= 0) return -1;
    const int W = cams[0].width, H = cams[0].height;
    for (int i = 0; i < n; ++i)
        if (pix[2 * i] < 0 || pix[2 * i] >= W || pix[2 * i + 1] < 0 || pix[2 * i + 1] >= H) return -2;
    const cudaTextureAddressMode mode = address_mode ? cudaAddressModeWrap : cudaAddressModeClamp;
    cudaTextureObjects th, dh;
    memset(&th, 0, sizeof(th));
    memset(&dh, 0, sizeof(dh));
    std::vector<cudaArray*> arrs(2 * num_images, nullptr);
    for (int i = 0; i < num_images; ++i) {
        make_texture(images[i], cams[i].width, cams[i].height, &arrs[i], &th.images[i], mode);
        make_texture(depth_maps[i], cams[i].width, cams[i].height, &arrs[num_images + i], &dh.images[i], mode);
    }
    PatchMatchParams p;
    memset(&p, 0, sizeof(p));
    fill_params(p, rp, num_images);
    const size_t wh = (size_t)W * H;
    cudaTextureObjects *dt = nullptr, *dd = nullptr;
    Camera* dc = nullptr;
    unsigned int *dcanny = nullptr, *dsel = nullptr;
    int2* dpix = nullptr;
    float4* dpl = nullptr;
    float *dcv = nullptr, *dic = nullptr, *ddep = nullptr, *dgeom = nullptr, *dtexo = nullptr;
    cudaMalloc((void**)&dt, sizeof(th));
    cudaMalloc((void**)&dd, sizeof(dh));
    cudaMalloc((void**)&dc, sizeof(Camera) * num_images);
    cudaMalloc((void**)&dcanny, sizeof(unsigned int) * wh);
    cudaMalloc((void**)&dpix, sizeof(int2) * n);
    cudaMalloc((void**)&dpl, sizeof(float4) * n);
    cudaMalloc((void**)&dcv, sizeof(float) * 32 * n);
    cudaMalloc((void**)&dic, sizeof(float) * n);
    cudaMalloc((void**)&dsel, sizeof(unsigned int) * n);
    cudaMalloc((void**)&ddep, sizeof(float) * n);
    cudaMalloc((void**)&dgeom, sizeof(float) * 32 * n);
    cudaMalloc((void**)&dtexo, sizeof(float) * n);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) {
        cudaMemcpy(dt, &th, sizeof(th), cudaMemcpyHostToDevice);
        cudaMemcpy(dd, &dh, sizeof(dh), cudaMemcpyHostToDevice);
        cudaMemcpy(dc, cams, sizeof(Camera) * num_images, cudaMemcpyHostToDevice);
        cudaMemcpy(dcanny, canny, sizeof(unsigned int) * wh, cudaMemcpyHostToDevice);
        cudaMemcpy(dpix, pix, sizeof(int2) * n, cudaMemcpyHostToDevice);
        cudaMemcpy(dpl, planes, sizeof(float4) * n, cudaMemcpyHostToDevice);
        cudaMemset(dcv, 0, sizeof(float) * 32 * n);
        cudaMemset(dgeom, 0, sizeof(float) * 32 * n);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) {
        k_ref_probe<<<(n + 127) / 128, 128>>>(dt, dd, dc, p, dcanny, dpix, dpl, n, dcv, dic, dsel, ddep, dgeom, dtexo);
        err = cudaDeviceSynchronize();
    }
    if (err == cudaSuccess) {
        cudaMemcpy(cost_vec, dcv, sizeof(float) * 32 * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(init_cost, dic, sizeof(float) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(sel, dsel, sizeof(unsigned int) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(depth, ddep, sizeof(float) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(geom, dgeom, sizeof(float) * 32 * n, cudaMemcpyDeviceToHost);
        err = cudaMemcpy(texture, dtexo, sizeof(float) * n, cudaMemcpyDeviceToHost);
    }
    void* bufs[] = {dt, dd, dc, dcanny, dpix, dpl, dcv, dic, dsel, ddep, dgeom, dtexo};
    for (void* b : bufs) cudaFree(b);
    for (int i = 0; i < num_images; ++i) {
        cudaDestroyTextureObject(th.images[i]);
        cudaDestroyTextureObject(dh.images[i]);
    }
    for (cudaArray* a : arrs) cudaFreeArray(a);
    return err == cudaSuccess ? 0 : (int)err;
}

// ---------------------------------------------------------------------------
// JBU probes: the reference's own JBU_cu and JBU_cu_prior kernels (HPM.cu:
// 3037-3197) launched the way JBU::CudaRun does (16x16 blocks), on textures
// made the way JBUAddImageToTextureFloatGray makes them (HPM.cpp:1213-1239:
// float, linear filtering, wrap addressing).  Raw kernel output: the host-side
// NaN fallback of RunJBU (HPM.cpp:1296-1302) is left to the caller.
__global__ void JBU_cu(JBUParameters* jp, JBUTexObj* jt, float* depth);
__global__ void JBU_cu_prior(JBUParameters* jp, JBUTexObj* jt, float* depth, float4* normal,
                             float4* normal_origin_cuda);

// image: W*H grey levels; src_depth: sw*sh; src_normal: sw*sh*3 (prior kernel)
// or null (plain kernel); out_depth: W*H; out_normal: W*H*3 when src_normal is set.
extern "C" int ref_jbu(const float* image, int W, int H, const float* src_depth, const float* src_normal, int sw,
                       int sh, float* out_depth, float* out_normal) {
    (void)cudaGetLastError();
    if (W <= 0 || H <= 0 || sw <= 0 || sh <= 0) return -1;
    const int scale = std::max(H / sh, W / sw);
    if (scale == 1) return -2;  // RunJBU returns without upsampling (HPM.cpp:1272-1275)
    JBUParameters jp;
    jp.height = H;
    jp.width = W;
    jp.s_height = sh;
    jp.s_width = sw;
    jp.Imagescale = scale;
    JBUTexObj jt;
    memset(&jt, 0, sizeof(jt));
    cudaArray* arrs[2] = {nullptr, nullptr};
    make_texture(image, W, H, &arrs[0], &jt.imgs[0]);
    make_texture(src_depth, sw, sh, &arrs[1], &jt.imgs[1]);
    const size_t n = (size_t)W * H, ns = (size_t)sw * sh;
    JBUParameters* djp = nullptr;
    JBUTexObj* djt = nullptr;
    float* dd = nullptr;
    float4 *dn = nullptr, *dno = nullptr;
    cudaMalloc((void**)&djp, sizeof(jp));
    cudaMalloc((void**)&djt, sizeof(jt));
    cudaMalloc((void**)&dd, sizeof(float) * n);
    if (src_normal) {
        cudaMalloc((void**)&dn, sizeof(float4) * n);
        cudaMalloc((void**)&dno, sizeof(float4) * ns);
    }
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) {
        cudaMemcpy(djp, &jp, sizeof(jp), cudaMemcpyHostToDevice);
        cudaMemcpy(djt, &jt, sizeof(jt), cudaMemcpyHostToDevice);
        if (src_normal) {
            // normal_origin_host: (normal, depth) per coarse pixel (HPM.cpp:1334-1343)
            std::vector<float4> no(ns);
            for (size_t i = 0; i < ns; ++i)
                no[i] = make_float4(src_normal[3 * i], src_normal[3 * i + 1], src_normal[3 * i + 2], src_depth[i]);
            cudaMemcpy(dno, no.data(), sizeof(float4) * ns, cudaMemcpyHostToDevice);
        }
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) {
        const dim3 grid((W + 15) / 16, (H + 15) / 16, 1), block(16, 16, 1);
        if (src_normal) JBU_cu_prior<<<grid, block>>>(djp, djt, dd, dn, dno);
        else JBU_cu<<<grid, block>>>(djp, djt, dd);
        err = cudaDeviceSynchronize();
    }
    if (err == cudaSuccess) {
        err = cudaMemcpy(out_depth, dd, sizeof(float) * n, cudaMemcpyDeviceToHost);
        if (err == cudaSuccess && src_normal) {
            std::vector<float4> on(n);
            err = cudaMemcpy(on.data(), dn, sizeof(float4) * n, cudaMemcpyDeviceToHost);
            for (size_t i = 0; i < n; ++i) {
                out_normal[3 * i] = on[i].x;
                out_normal[3 * i + 1] = on[i].y;
                out_normal[3 * i + 2] = on[i].z;
            }
        }
    }
    void* bufs[] = {djp, djt, dd, dn, dno};
    for (void* b : bufs) cudaFree(b);
    for (int i = 0; i < 2; ++i) {
        cudaDestroyTextureObject(jt.imgs[i]);
        cudaFreeArray(arrs[i]);
    }
    return err == cudaSuccess ? 0 : (int)err;
}
