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
        cudaError_t e = cudaMalloc((void**)&c->prof_hyp, 2 * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMemsetAsync(c->prof_hyp, 0, 2 * sizeof(unsigned long long), c->stream);
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

}  // extern "C"
