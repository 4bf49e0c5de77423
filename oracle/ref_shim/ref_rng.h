// CHECKER ONLY: force-included ahead of the reference's HPM.cu.  It routes the
// reference's curand_init / curand_uniform / clock64 seeding to the counter-based
// stream of include/hpm_philox.h (key = run seed, counter = (draw/4, x, y, view)),
// reusing each pixel's 48-byte curandState as storage, so the reference kernels
// draw exactly the uniforms the CUDA path and the CPU oracle draw.
#pragma once
#include <cfloat>
#include <curand_kernel.h>
#include "hpm_philox.h"

struct RefRngState {
    unsigned long long seed;
    unsigned int x, y, draw;
};
static_assert(sizeof(RefRngState) <= sizeof(curandState), "state fits");

__device__ unsigned long long g_ref_seed;
__device__ unsigned int g_ref_view;

__device__ __forceinline__ unsigned long long hpm_ref_clock_seed() { return g_ref_seed; }

__device__ __forceinline__ void hpm_ref_curand_init(unsigned long long seed, unsigned long long subsequence,
                                                    unsigned long long offset, curandState* state) {
    RefRngState* s = reinterpret_cast<RefRngState*>(state);
    s->seed = seed;
    s->y = (unsigned int)subsequence;  // curand_init(clock64(), p.y, p.x, ...) (HPM.cu:579)
    s->x = (unsigned int)offset;
    s->draw = 0;
}

__device__ __forceinline__ float hpm_ref_curand_uniform(curandState* state) {
    RefRngState* s = reinterpret_cast<RefRngState*>(state);
    const unsigned int bits = hpm_rng_bits(s->seed, g_ref_view, s->x, s->y, s->draw);
    s->draw++;
    return hpm_bits_to_uniform(bits);
}

#define clock64() hpm_ref_clock_seed()
#define curand_init(seed, subsequence, offset, state) hpm_ref_curand_init(seed, subsequence, offset, state)
#define curand_uniform(state) hpm_ref_curand_uniform(state)
