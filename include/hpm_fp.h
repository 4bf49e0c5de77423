/*
 * Floating-point conventions of the plain FP32 path, shared by the CUDA
 * kernels and the CPU oracle so both evaluate the same operation sequence.
 *
 * HPM-MVS++ builds its kernels with --use_fast_math (CMakeLists.txt:10), which
 * leaves the rounding of exp/sin/cos, division and multiply-add contraction to
 * the compiler.  This project pins them instead:
 *   - every +, -, *, / and sqrt is an IEEE fp32 operation (kernels built with
 *     -fmad=false -prec-div=true -prec-sqrt=true, oracle with -ffp-contract=off);
 *   - a multiply-add is fused only where the code calls hpm_fma;
 *   - exp, sin and cos of floats are the functions below, written only with
 *     IEEE operations and fmaf, so CPU and GPU produce identical bits;
 *   - a reciprocal near a known one (the perspective divide over a patch) is
 *     refined by hpm_recip_near, again bit-identical on both sides.
 * Accuracy: hpm_expf and hpm_sinf/hpm_cosf are within about 2 ulp of the exact
 * functions, hpm_recip_near within 1 ulp when |x/x0 - 1| < 2^-8.
 */
#ifndef HPM_FP_H
#define HPM_FP_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define HPM_FP_HD __host__ __device__ __forceinline__
#else
#define HPM_FP_HD static inline
#endif

HPM_FP_HD float hpm_fma(float a, float b, float c) { return fmaf(a, b, c); }

HPM_FP_HD float hpm_pow2i(int n) /* 2^n for -126 <= n <= 127, exact */
{
    const uint32_t bits = (uint32_t)(n + 127) << 23;
    float f;
#if defined(__CUDA_ARCH__)
    f = __uint_as_float(bits);
#else
    memcpy(&f, &bits, sizeof(f));
#endif
    return f;
}

/* e^x: Cody-Waite reduction x = n ln2 + r (|r| <= ln2/2, ln2 split in a
 * 16-bit-exact head and a tail) and a degree-7 Taylor polynomial of e^r in
 * Horner form; scaling by 2^n in two exact steps so results that underflow
 * into the denormal range round once. */
HPM_FP_HD float hpm_expf(float x)
{
    if (x != x) return x;
    if (x > 88.72283935546875f) return INFINITY;
    if (x < -103.97208404541015625f) return 0.0f;
    const float kLog2e = 1.44269502162933349609375f;
    const float kLn2Hi = 0.693145751953125f;          /* 16 significant bits */
    const float kLn2Lo = 1.428606765330187045e-06f;   /* ln2 - kLn2Hi */
    const float n = rintf(x * kLog2e);
    float r = hpm_fma(-n, kLn2Hi, x);
    r = hpm_fma(-n, kLn2Lo, r);
    float p = 1.0f / 5040.0f;
    p = hpm_fma(p, r, 1.0f / 720.0f);
    p = hpm_fma(p, r, 1.0f / 120.0f);
    p = hpm_fma(p, r, 1.0f / 24.0f);
    p = hpm_fma(p, r, 1.0f / 6.0f);
    p = hpm_fma(p, r, 0.5f);
    p = hpm_fma(p, r, 1.0f);
    p = hpm_fma(p, r, 1.0f);
    const int ni = (int)n;
    const int n1 = ni / 2;
    const int n2 = ni - n1;
    return (p * hpm_pow2i(n1)) * hpm_pow2i(n2);
}

/* sin and cos by Taylor polynomials on |x| <= pi/4 (truncation below 2e-9);
 * outside that range (never reached by the perturbation angles of the hot
 * path, |x| < 0.2) the double-precision functions are rounded once. */
HPM_FP_HD float hpm_sinf(float x)
{
    if (!(fabsf(x) <= 0.78539816339744830962f)) return (float)sin((double)x);
    const float x2 = x * x;
    float p = 1.0f / 362880.0f;
    p = hpm_fma(p, x2, -1.0f / 5040.0f);
    p = hpm_fma(p, x2, 1.0f / 120.0f);
    p = hpm_fma(p, x2, -1.0f / 6.0f);
    return hpm_fma(x * x2, p, x);
}

HPM_FP_HD float hpm_cosf(float x)
{
    if (!(fabsf(x) <= 0.78539816339744830962f)) return (float)cos((double)x);
    const float x2 = x * x;
    float p = -1.0f / 3628800.0f;
    p = hpm_fma(p, x2, 1.0f / 40320.0f);
    p = hpm_fma(p, x2, -1.0f / 720.0f);
    p = hpm_fma(p, x2, 1.0f / 24.0f);
    p = hpm_fma(p, x2, -0.5f);
    return hpm_fma(x2, p, 1.0f);
}

/* 1/x from r0 = 1/x0 of a nearby x0 by two Newton steps (fused). */
HPM_FP_HD float hpm_recip_near(float x, float r0)
{
    float e = hpm_fma(-x, r0, 1.0f);
    float r = hpm_fma(r0, e, r0);
    e = hpm_fma(-x, r, 1.0f);
    return hpm_fma(r, e, r);
}

#endif /* HPM_FP_H */
