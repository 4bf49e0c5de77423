/*
 * Counter-based random numbers for the PatchMatch hot path.
 *
 * HPM-MVS++ draws from one curand XORWOW stream per pixel, seeded with
 * curand_init(clock64(), p.y, p.x, &state) (HPM.cu:579), so two runs of the
 * reference never agree.  This project replaces that stream with
 * Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy
 * as 1, 2, 3", SC'11): a stateless bijection of a 128-bit counter under a
 * 64-bit key.  A pixel's stream is the counter (draw/4, x, y, view) under the
 * run's seed; draw k of that pixel returns word k%4 of the block.  The only
 * per-pixel state is the 32-bit draw index, which persists across the init and
 * red/black launches exactly like the curandState it replaces.
 *
 * hpm_uniform() maps 24 random bits to (0, 1], the same half-open range as
 * curand_uniform.  The CUDA kernels and the CPU oracle include this one
 * definition, so both see bit-identical uniforms.
 */
#ifndef HPM_PHILOX_H
#define HPM_PHILOX_H

#include <stdint.h>

#if defined(__CUDACC__)
#define HPM_HD __host__ __device__ __forceinline__
#else
#define HPM_HD static inline
#endif

#define HPM_PHILOX_M0 0xD2511F53u
#define HPM_PHILOX_M1 0xCD9E8D57u
#define HPM_PHILOX_W0 0x9E3779B9u
#define HPM_PHILOX_W1 0xBB67AE85u

typedef struct hpm_u32x4 { uint32_t v[4]; } hpm_u32x4;

HPM_HD uint32_t hpm_mulhi32(uint32_t a, uint32_t b)
{
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
#endif
}

/* Ten Philox rounds over counter c under key (k0, k1). */
HPM_HD hpm_u32x4 hpm_philox4x32_10(hpm_u32x4 c, uint32_t k0, uint32_t k1)
{
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = hpm_mulhi32(HPM_PHILOX_M0, c.v[0]);
        const uint32_t lo0 = HPM_PHILOX_M0 * c.v[0];
        const uint32_t hi1 = hpm_mulhi32(HPM_PHILOX_M1, c.v[2]);
        const uint32_t lo1 = HPM_PHILOX_M1 * c.v[2];
        hpm_u32x4 n;
        n.v[0] = hi1 ^ c.v[1] ^ k0;
        n.v[1] = lo1;
        n.v[2] = hi0 ^ c.v[3] ^ k1;
        n.v[3] = lo0;
        c = n;
        k0 += HPM_PHILOX_W0;
        k1 += HPM_PHILOX_W1;
    }
    return c;
}

/* Raw 32-bit draw number `draw` of pixel (x, y) of view `view`. */
HPM_HD uint32_t hpm_rng_bits(uint64_t seed, uint32_t view, uint32_t x, uint32_t y, uint32_t draw)
{
    hpm_u32x4 c;
    c.v[0] = draw >> 2;
    c.v[1] = x;
    c.v[2] = y;
    c.v[3] = view;
    const hpm_u32x4 r = hpm_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    return r.v[draw & 3u];
}

/* Uniform float in (0, 1]: (k + 1) / 2^24 for the top 24 bits k; exact in fp32. */
HPM_HD float hpm_bits_to_uniform(uint32_t bits)
{
    return (float)((bits >> 8) + 1u) * (1.0f / 16777216.0f);
}

#endif /* HPM_PHILOX_H */
