// Measurement entry points of the C ABI: the context's stream, per-launch
// profiling, and an FP32 FMA throughput probe used as the compute roof of the
// PatchMatch kernels (which issue no tensor-core work).
#include "ctx.hpp"

#include <algorithm>

using hpm::Ctx;

namespace {

// Eight independent FMA chains per thread; the result is stored only when a
// impossible value appears, so the compiler keeps every FMA.
__global__ void k_fma_peak(float* out, int iters, float a, float b) {
    float x0 = threadIdx.x * 1e-3f, x1 = x0 + 0.1f, x2 = x0 + 0.2f, x3 = x0 + 0.3f;
    float x4 = x0 + 0.4f, x5 = x0 + 0.5f, x6 = x0 + 0.6f, x7 = x0 + 0.7f;
    for (int i = 0; i < iters; ++i) {
        x0 = __fmaf_rn(x0, a, b); x1 = __fmaf_rn(x1, a, b); x2 = __fmaf_rn(x2, a, b); x3 = __fmaf_rn(x3, a, b);
        x4 = __fmaf_rn(x4, a, b); x5 = __fmaf_rn(x5, a, b); x6 = __fmaf_rn(x6, a, b); x7 = __fmaf_rn(x7, a, b);
    }
    const float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == -1234.5f) out[blockIdx.x] = s;
}

__device__ __forceinline__ unsigned tex_probe_hash(unsigned x) {
    x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
    return x;
}

// Linear-filtered fetches in the access pattern of the half-sweep: a warp's
// lanes are 32 pixels of one checkerboard colour (x = x0 + lane, y alternating
// between two rows), each fetching its 6 x 6 stride-2 patch at fractional
// positions, six independent fetches in flight per thread.  With jitter > 0
// every lane's patch is moved by its own offset, uniform in [-jitter, jitter]
// pixels per axis and redrawn for every column of six fetches: the lanes of a
// warp then sample apart, as they do when neighbouring pixels hold different
// planes.  Coordinates outside the texture are clamped by the texture unit.
__global__ void k_tex_peak(cudaTextureObject_t tex, int w, int h, int iters, float jitter, float* out) {
    const int lane = threadIdx.x & 31, warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const float px = 8.0f + (float)((warp * 32) % (w - 48)) + (float)lane;
    const float py = 8.0f + (float)((warp * 7) % (h - 24)) + (float)(lane & 1);
    float acc = 0.f;
    for (int it = 0; it < iters; ++it) {
        const float fx = 0.25f + 0.0625f * (it & 7), fy = 0.375f + 0.03125f * (it & 15);
        const int i = it % 6;
        float jx = 0.f, jy = 0.f;
        if (jitter > 0.f) {
            const unsigned hv = tex_probe_hash((unsigned)(warp * 131 + lane) * 977u + (unsigned)(it / 6) * 7919u);
            jx = jitter * ((float)(hv & 0xffffu) * (2.0f / 65535.0f) - 1.0f);
            jy = jitter * ((float)(hv >> 16) * (2.0f / 65535.0f) - 1.0f);
        }
        float v[6];
#pragma unroll
        for (int k = 0; k < 6; ++k)
            v[k] = tex2D<float>(tex, px + jx - 5.0f + 2.0f * i + fx, py + jy - 5.0f + 2.0f * k + fy);
        acc += ((v[0] + v[1]) + (v[2] + v[3])) + (v[4] + v[5]);
    }
    if (acc == -1234.5f) out[blockIdx.x] = acc;
}

}  // namespace

extern "C" {

int hpm_get_stream(hpm_ctx* ctx, void** stream) {
    if (!ctx || !stream) return HPM_E_INVALID;
    *stream = (void*)reinterpret_cast<Ctx*>(ctx)->stream;
    return HPM_OK;
}

int hpm_profile_enable(hpm_ctx* ctx, int flags) {
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (flags & ~(HPM_PROFILE_TIMING | HPM_PROFILE_COUNT)) return c->fail(HPM_E_INVALID, "unknown profile flags %d", flags);
    cudaSetDevice(c->device);
    if ((flags & HPM_PROFILE_COUNT) && !c->prof_hyp) {
        cudaError_t e = cudaMalloc((void**)&c->prof_hyp, 3 * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMemsetAsync(c->prof_hyp, 0, 3 * sizeof(unsigned long long), c->stream);
        if (e != cudaSuccess) return c->cuda_fail(e, "profile counters");
    }
    c->prof_flags = flags;
    return HPM_OK;
}

int hpm_profile_read(hpm_ctx* ctx, hpm_profile* out) {
    if (!ctx || !out) return HPM_E_INVALID;
    return reinterpret_cast<Ctx*>(ctx)->profile_read(out);
}

int hpm_measure_fp32_peak(int device, double* tflops) {
    if (!tflops) return HPM_E_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return HPM_E_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return HPM_E_CUDA;
    const int threads = 256, blocks = sms * 8, iters = 1 << 16;
    float* out = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaMalloc((void**)&out, sizeof(float) * blocks);
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    double best = 0.0;
    for (int rep = 0; rep < 6 && e == cudaSuccess; ++rep) {
        cudaEventRecord(a);
        k_fma_peak<<<blocks, threads>>>(out, iters, 0.99999f, 1e-5f);
        cudaEventRecord(b);
        e = cudaEventSynchronize(b);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
        if (e == cudaSuccess && rep > 0 && ms > 0.f)
            best = std::max(best, 2.0 * 8.0 * iters * (double)blocks * threads / (ms * 1e-3) / 1e12);
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (out) cudaFree(out);
    if (e != cudaSuccess) { cudaGetLastError(); return HPM_E_CUDA; }
    *tflops = best;
    return HPM_OK;
}

int hpm_measure_tex_peak(int device, int format, double* gsamples) {
    return hpm_measure_tex_rate(device, format, 0.0f, gsamples);
}

int hpm_measure_tex_rate(int device, int format, float jitter, double* gsamples) {
    if (!gsamples || (format != HPM_TEX_F32 && format != HPM_TEX_F16 && format != HPM_TEX_U8)) return HPM_E_INVALID;
    if (!(jitter >= 0.0f && jitter <= 64.0f)) return HPM_E_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return HPM_E_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return HPM_E_CUDA;
    const int w = 1024, h = 256, threads = 128, blocks = sms * 12, iters = 1 << 12;
    const cudaChannelFormatDesc fd =
        format == HPM_TEX_F16 ? cudaCreateChannelDesc(16, 0, 0, 0, cudaChannelFormatKindFloat)
                              : (format == HPM_TEX_U8 ? cudaCreateChannelDesc(8, 0, 0, 0, cudaChannelFormatKindUnsigned)
                                                      : cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat));
    const size_t texel = format == HPM_TEX_F32 ? 4 : (format == HPM_TEX_F16 ? 2 : 1);
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
    float* out = nullptr;
    void* stage = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaMallocArray(&arr, &fd, w, h);
    if (e == cudaSuccess) e = cudaMalloc(&stage, (size_t)w * h * texel);
    if (e == cudaSuccess) e = cudaMemset(stage, 0x3c, (size_t)w * h * texel);  // any finite texel value
    if (e == cudaSuccess) e = cudaMemcpy2DToArray(arr, 0, 0, stage, w * texel, w * texel, h, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) {
        cudaResourceDesc rd{};
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = arr;
        cudaTextureDesc td{};
        td.addressMode[0] = td.addressMode[1] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = format == HPM_TEX_U8 ? cudaReadModeNormalizedFloat : cudaReadModeElementType;
        e = cudaCreateTextureObject(&tex, &rd, &td, nullptr);
    }
    if (e == cudaSuccess) e = cudaMalloc((void**)&out, sizeof(float) * blocks);
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    double best = 0.0;
    for (int rep = 0; rep < 5 && e == cudaSuccess; ++rep) {
        cudaEventRecord(a);
        k_tex_peak<<<blocks, threads>>>(tex, w, h, iters, jitter, out);
        cudaEventRecord(b);
        e = cudaEventSynchronize(b);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
        if (e == cudaSuccess && rep > 0 && ms > 0.f)
            best = std::max(best, 6.0 * iters * (double)blocks * threads / (ms * 1e-3) / 1e9);
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (tex) cudaDestroyTextureObject(tex);
    if (arr) cudaFreeArray(arr);
    if (stage) cudaFree(stage);
    if (out) cudaFree(out);
    if (e != cudaSuccess) { cudaGetLastError(); return HPM_E_CUDA; }
    *gsamples = best;
    return HPM_OK;
}

}  // extern "C"
