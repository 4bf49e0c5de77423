// hpm_eval_costs_noalloc: the fixed-hypothesis cost evaluation of
// hpm_eval_costs with its device staging in a fixed, file-scope array instead
// of memory the context allocates.
//
// Some callers cannot let a library call cudaMalloc or cudaFree while they run:
// both can synchronise the whole device, stalling work the caller has in flight
// on other streams, and both can fail in a process whose device memory is
// already handed out to another allocator under a fixed budget.  A caller that
// evaluates costs in such a loop (a plane refiner, a test harness driving the
// cost many times) uses this entry point: once its views are resident, it
// allocates nothing.
//
// Limits and sharing:
//   - the staging array holds kNoAllocBytes (4 MiB) on every GPU that loads the
//     library, until the process exits; a call needs n * (24 + 4 * n_src) bytes
//     plus alignment and is rejected with HPM_E_INVALID when that does not fit
//     (65,536 hypotheses with 10 sources);
//   - all calls on a device share the array and it keeps the last call's
//     contents; every output slot is written before it is read back, so nothing
//     has to be cleared.  Calls that overlap on the GPU (two contexts of one
//     device used from two threads) race on the array and must be serialised
//     by the caller;
//   - the first call on a device looks the array's device address up
//     (cudaGetSymbolAddress with that device current); make that first call
//     before any stream capture.
#include "ctx.hpp"

#include <mutex>

namespace {

constexpr size_t kNoAllocBytes = size_t(4) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_staging[kNoAllocBytes];

std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_addr[kMaxDevices] = {};

// Device address of the staging array on the current device `device`.  In host
// code the array's name is only a host-side stand-in, never a device pointer.
cudaError_t staging_address(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_staging);
        if (e != cudaSuccess) return e;
        g_noalloc_addr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_addr[device];
    return cudaSuccess;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

extern "C" int hpm_eval_costs_noalloc(hpm_ctx* ctx, int ref, const int32_t* srcs, int n_src,
                                      const hpm_params* params, int n, const int32_t* px, const float* planes,
                                      float* out) {
    using hpm::Ctx;
    if (!ctx) return HPM_E_INVALID;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return c->cuda_fail(e, "hpm_eval_costs_noalloc: set device");
    if (n < 0 || (n > 0 && (!px || !planes || !out)))
        return c->fail(HPM_E_INVALID, "hpm_eval_costs_noalloc: bad arguments");
    hpm::RunArgs a;
    int rc = c->fill_run_args(ref, srcs, n_src, params, a);
    if (rc) return rc;
    if (n == 0) return HPM_OK;
    for (int k = 0; k < n; ++k)
        if (px[2 * k] < 0 || px[2 * k] >= a.W || px[2 * k + 1] < 0 || px[2 * k + 1] >= a.H)
            return c->fail(HPM_E_INVALID, "pixel %d outside the reference image", k);
    const size_t planes_bytes = align256((size_t)n * 16);
    const size_t px_bytes = align256((size_t)n * 8);
    const size_t out_bytes = align256((size_t)n * n_src * 4);
    if (planes_bytes + px_bytes + out_bytes > kNoAllocBytes)
        return c->fail(HPM_E_INVALID,
                       "hpm_eval_costs_noalloc: %d hypotheses x %d sources need %zu bytes of staging, more than its "
                       "fixed %zu; use hpm_eval_costs or fewer hypotheses per call",
                       n, n_src, planes_bytes + px_bytes + out_bytes, kNoAllocBytes);
    unsigned char* base = nullptr;
    if ((e = staging_address(c->device, &base)) != cudaSuccess)
        return c->cuda_fail(e, "hpm_eval_costs_noalloc: staging address");
    float4* d_planes = reinterpret_cast<float4*>(base);
    int32_t* d_px = reinterpret_cast<int32_t*>(base + planes_bytes);
    float* d_out = reinterpret_cast<float*>(base + planes_bytes + px_bytes);
    e = cudaMemcpyAsync(d_planes, planes, (size_t)n * 16, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_px, px, (size_t)n * 8, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "hpm_eval_costs_noalloc: upload hypotheses");
    if ((e = hpm::launch_eval_costs(a, n, d_px, d_planes, d_out, c->stream)) != cudaSuccess)
        return c->cuda_fail(e, "hpm_eval_costs_noalloc: launch");
    ++c->launches;
    e = cudaMemcpyAsync(out, d_out, (size_t)n * n_src * 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return c->cuda_fail(e, "hpm_eval_costs_noalloc: download costs");
    return HPM_OK;
}
