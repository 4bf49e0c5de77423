// Device-side building blocks of the PatchMatch hot path (sm_100a): camera and
// plane geometry, random plane generation on the counter-based stream, the
// geometric-consistency cost and the edge-density term.  The formulas restate
// HPM-MVS++'s device helpers (HPM.cu:114-564) under the rounding conventions of
// include/hpm_fp.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include "hpm_types.h"
#include "hpm_philox.h"
#include "hpm_fp.h"
#include "hpm_geometry.h"

namespace hpm {

constexpr int kPatchSamples = 36;   // 11x11 window, stride 2 (HPM.h:34-36)
constexpr int kPatchRadius = 5;
constexpr int kPatchStep = 2;
constexpr int kMarsagliaMaxTries = 4096;

struct PixelRng {
    uint64_t seed;
    uint32_t view, x, y, draw;
    uint32_t block_id;  // draw >> 2 of the cached block, or 0xffffffff
    uint32_t w[4];
    __device__ __forceinline__ void init(uint64_t s, uint32_t v, uint32_t px, uint32_t py, uint32_t d) {
        seed = s; view = v; x = px; y = py; draw = d; block_id = 0xffffffffu;
    }
    __device__ __forceinline__ float uniform() {
        const uint32_t b = draw >> 2;
        if (b != block_id) {
            hpm_u32x4 c;
            c.v[0] = b; c.v[1] = x; c.v[2] = y; c.v[3] = view;
            const hpm_u32x4 r = hpm_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
            w[0] = r.v[0]; w[1] = r.v[1]; w[2] = r.v[2]; w[3] = r.v[3];
            block_id = b;
        }
        const uint32_t bits = w[draw & 3u];
        ++draw;
        return hpm_bits_to_uniform(bits);
    }
};

// ---------------- camera / plane helpers (HPM.cu:114-157, 322-340, 497-537) ----------------

__device__ __forceinline__ float4 rotate_to_world(const hpm_camera& c, float4 p) {
    float4 r;
    r.x = c.R[0] * p.x + c.R[3] * p.y + c.R[6] * p.z;
    r.y = c.R[1] * p.x + c.R[4] * p.y + c.R[7] * p.z;
    r.z = c.R[2] * p.x + c.R[5] * p.y + c.R[8] * p.z;
    r.w = p.w;
    return r;
}

__device__ __forceinline__ float4 rotate_to_cam(const hpm_camera& c, float4 p) {
    float4 r;
    r.x = c.R[0] * p.x + c.R[1] * p.y + c.R[2] * p.z;
    r.y = c.R[3] * p.x + c.R[4] * p.y + c.R[5] * p.z;
    r.z = c.R[6] * p.x + c.R[7] * p.y + c.R[8] * p.z;
    r.w = p.w;
    return r;
}

__device__ __forceinline__ float distance_to_origin(const hpm_camera& c, int px, int py, float depth, float4 n) {
    const float X0 = depth * (px - c.K[2]) / c.K[0];
    const float X1 = depth * (py - c.K[5]) / c.K[4];
    return -(n.x * X0 + n.y * X1 + n.z * depth);
}

__device__ __forceinline__ float depth_from_plane(const hpm_camera& c, float4 pl, int px, int py) {
    return -pl.w * c.K[0] / ((px - c.K[2]) * pl.x + (c.K[0] / c.K[4]) * (py - c.K[5]) * pl.y + c.K[0] * pl.z);
}

__device__ __forceinline__ float4 view_direction(const hpm_camera& c, int px, int py, float depth) {
    const float X0 = depth * (px - c.K[2]) / c.K[0];
    const float X1 = depth * (py - c.K[5]) / c.K[4];
    const float X2 = depth;
    const float norm = sqrtf(X0 * X0 + X1 * X1 + X2 * X2);
    return make_float4(X0 / norm, X1 / norm, X2 / norm, 0.0f);
}

__device__ __forceinline__ void normalize3(float4& v) {
    const float inv = 1.0f / sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    v.x *= inv; v.y *= inv; v.z *= inv;
}

__device__ __forceinline__ float4 random_normal(const hpm_camera& c, int px, int py, PixelRng& rng, float depth) {
    float q1 = 1.0f, q2 = 1.0f, s = 2.0f;
    int tries = 0;
    while (s >= 1.0f && tries < kMarsagliaMaxTries) {
        q1 = 2.0f * rng.uniform() - 1.0f;
        q2 = 2.0f * rng.uniform() - 1.0f;
        s = q1 * q1 + q2 * q2;
        ++tries;
    }
    if (s >= 1.0f) { q1 = 0.0f; q2 = 0.0f; s = 0.0f; }
    const float sq = sqrtf(1.0f - s);
    float4 n = make_float4(2.0f * q1 * sq, 2.0f * q2 * sq, 1.0f - 2.0f * s, 0.0f);
    const float4 vd = view_direction(c, px, py, depth);
    if (n.x * vd.x + n.y * vd.y + n.z * vd.z > 0.0f) { n.x = -n.x; n.y = -n.y; n.z = -n.z; }
    normalize3(n);
    return n;
}

__device__ __forceinline__ float4 perturbed_normal(const hpm_camera& c, int px, int py, float4 normal,
                                                   PixelRng& rng, float perturbation) {
    const float4 vd = view_direction(c, px, py, 1.0f);
    const float a1 = (rng.uniform() - 0.5f) * perturbation;
    const float a2 = (rng.uniform() - 0.5f) * perturbation;
    const float a3 = (rng.uniform() - 0.5f) * perturbation;
    const float s1 = hpm_sinf(a1), s2 = hpm_sinf(a2), s3 = hpm_sinf(a3);
    const float c1 = hpm_cosf(a1), c2 = hpm_cosf(a2), c3 = hpm_cosf(a3);
    const float R0 = c2 * c3, R1 = c3 * s1 * s2 - c1 * s3, R2 = s1 * s3 + c1 * c3 * s2;
    const float R3 = c2 * s3, R4 = c1 * c3 + s1 * s2 * s3, R5 = c1 * s2 * s3 - c3 * s1;
    const float R6 = -s2, R7 = c2 * s1, R8 = c1 * c2;
    float4 np;
    np.x = R0 * normal.x + R1 * normal.y + R2 * normal.z;
    np.y = R3 * normal.x + R4 * normal.y + R5 * normal.z;
    np.z = R6 * normal.x + R7 * normal.y + R8 * normal.z;
    np.w = normal.w;
    if (np.x * vd.x + np.y * vd.y + np.z * vd.z >= 0.0f) np = normal;
    normalize3(np);
    return np;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ComputeGeomConsistencyCost (HPM.cu:539-564): the pixel's 3D point at the
// hypothesis depth carried into source j, the source depth read there (a
// clamped point fetch at (int)x, (int)y) and carried back; the cost is the
// reprojection distance, at most 3.  The two transfers use the per-view bases
// of hpm_view_transfer (include/hpm_geometry.h).
__device__ __forceinline__ float geom_cost(const float* __restrict__ sdepth, int sw, int sh, const float* Gf,
                                           const float* gf, const float* Gb, const float* gb, float depth, int px,
                                           int py) {
    const float max_cost = 3.0f;
    float sx, sy;
    hpm_transfer(Gf, gf, (float)px, (float)py, depth, &sx, &sy);
    const int ix = clampi(__float2int_rz(sx), 0, sw - 1);
    const int iy = clampi(__float2int_rz(sy), 0, sh - 1);
    const float d = __ldg(sdepth + (size_t)iy * sw + ix);
    if (d == 0.0f) return max_cost;
    float bx, by;
    hpm_transfer(Gb, gb, sx, sy, d, &bx, &by);
    const float dx = px - bx, dy = py - by;
    return fminf(max_cost, sqrtf(dx * dx + dy * dy));
}

// Edge-density texture term (HPM.cu:349-373); the ratio is evaluated in double
// as in the reference (double literals).
__device__ __forceinline__ float texture_term(const uint8_t* __restrict__ canny, int W, int H, int px, int py) {
    int total = 0, edges = 0;
#pragma unroll
    for (int i = -5; i < 6; i += 2)
#pragma unroll
        for (int j = -5; j < 6; j += 2) {
            const int x = px + j, y = py + i;
            if (x >= 0 && x < W && y >= 0 && y < H) {
                ++total;
                if (__ldg(canny + (size_t)y * W + x) >= 1) ++edges;
            }
        }
    const float frac = edges * 1.0f / total;
    return (float)(((double)frac + 0.00005) / ((double)frac + 0.0001));
}

}  // namespace hpm
