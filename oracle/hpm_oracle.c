/*
 * CPU ORACLE -- test infrastructure only (see hpm_oracle.h).
 *
 * Restates the PatchMatch kernels of HPM-MVS++ (HPM.cu) as CPU loops.  The
 * red/black half-sweeps read only opposite-colour neighbours and write only the
 * pixel itself (offsets +-5/+-6 and steps of 2 keep the colour parity), so a
 * plain loop over the pixels of one colour reproduces the GPU launch exactly;
 * OpenMP only splits that loop.
 *
 * Arithmetic follows the reference expression by expression in float (compile
 * without -ffast-math and with -ffp-contract=off); where the reference mixes in
 * double literals the double promotion is kept.
 */
#include "hpm_oracle.h"
#include "hpm_philox.h"
#include "hpm_fp.h"
#include "hpm_geometry.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct { float x, y, z, w; } f4;
typedef struct { float x, y; } f2;

static int g_tex_model = 0;
void ora_set_texture_model(int model) { g_tex_model = model; }
int ora_get_texture_model(void) { return g_tex_model; }

/* Shifted moments in the NCC (the precision form): the reference patch is
 * accumulated relative to its centre texel and the source patch relative to
 * its first sample, so flat patches keep their variance instead of losing it
 * to E[x^2] - E[x]^2 cancellation.  Off (shift 0) gives the plain arithmetic
 * bit for bit. */
static int g_ncc_shift = 0;
void ora_set_ncc_shift(int on) { g_ncc_shift = on != 0; }

/* float -> int conversion with the semantics of the GPU's cvt.rzi.s32.f32:
 * truncation toward zero, NaN -> 0, saturation at the int range. */
static inline int f2i_rz(float v)
{
    if (v != v) return 0;
    if (v >= 2147483647.0f) return 2147483647;
    if (v <= -2147483648.0f) return (-2147483647 - 1);
    return (int)v;
}

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

static inline f4 load4(const float *p, int idx)
{
    f4 r = { p[4 * idx], p[4 * idx + 1], p[4 * idx + 2], p[4 * idx + 3] };
    return r;
}
static inline void store4(float *p, int idx, f4 v)
{
    p[4 * idx] = v.x; p[4 * idx + 1] = v.y; p[4 * idx + 2] = v.z; p[4 * idx + 3] = v.w;
}

/* Linear-filtered fetch with unnormalised coordinates and clamp addressing
 * (tex2D on a cudaFilterModeLinear float texture, HPM.cu:409).
 *
 * Model 0 is the filter as measured on B200 (sm_100a): xB = x - 0.5, i =
 * floor(xB), and the fractional weights alpha, beta rounded half-up to 8
 * fractional bits; the cross weight alpha*beta is itself rounded half-up to 8
 * bits and the other three weights are derived from it so each row and column
 * still sums exactly.  NaN coordinates read as 0.  Model 1 is the separable
 * form of the CUDA Programming Guide ("Texture Fetching": 9-bit fixed-point
 * alpha and beta, products in float). */
float ora_tex2d(const float *img, int width, int height, float x, float y)
{
    if (x != x) x = 0.0f;
    if (y != y) y = 0.0f;
    double xb = (double)x - 0.5;
    double yb = (double)y - 0.5;
    const double lim = 1.0e9;
    if (xb > lim) xb = lim;
    if (xb < -lim) xb = -lim;
    if (yb > lim) yb = lim;
    if (yb < -lim) yb = -lim;
    const long long ix = (long long)floor(xb * 256.0 + 0.5);
    const long long iy = (long long)floor(yb * 256.0 + 0.5);
    const long long i0 = ix >> 8, j0 = iy >> 8; /* arithmetic shift = floor division */
    const int ai = (int)(ix & 255), bi = (int)(iy & 255);
    const int x0 = (int)(i0 < 0 ? 0 : (i0 > width - 1 ? width - 1 : i0));
    const int x1 = (int)(i0 + 1 < 0 ? 0 : (i0 + 1 > width - 1 ? width - 1 : i0 + 1));
    const int y0 = (int)(j0 < 0 ? 0 : (j0 > height - 1 ? height - 1 : j0));
    const int y1 = (int)(j0 + 1 < 0 ? 0 : (j0 + 1 > height - 1 ? height - 1 : j0 + 1));
    const float t00 = img[y0 * width + x0], t10 = img[y0 * width + x1];
    const float t01 = img[y1 * width + x0], t11 = img[y1 * width + x1];
    const float a = (float)ai * (1.0f / 256.0f);
    const float b = (float)bi * (1.0f / 256.0f);
    if (g_tex_model == 1)
        return (1.0f - a) * (1.0f - b) * t00 + a * (1.0f - b) * t10 + (1.0f - a) * b * t01 + a * b * t11;
    const float w11 = (float)((ai * bi + 128) >> 8) * (1.0f / 256.0f);
    const float w10 = a - w11, w01 = b - w11, w00 = 1.0f - a - b + w11;
    return w00 * t00 + w10 * t10 + w01 * t01 + w11 * t11;
}

/* Texel fetch at an integer position (tex2D at x + 0.5, y + 0.5), clamped. */
static inline float texel(const float *img, int width, int height, int x, int y)
{
    return img[clampi(y, 0, height - 1) * width + clampi(x, 0, width - 1)];
}

/* ---------------- camera / plane helpers (HPM.cu:114-157, 251-340, 497-537) ---------------- */

static void get_3d_point(const hpm_camera *c, int px, int py, float depth, float X[3])
{
    X[0] = depth * (px - c->K[2]) / c->K[0];
    X[1] = depth * (py - c->K[5]) / c->K[4];
    X[2] = depth;
}

static f4 view_direction(const hpm_camera *c, int px, int py, float depth)
{
    float X[3];
    get_3d_point(c, px, py, depth, X);
    const float norm = sqrtf(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
    f4 v = { X[0] / norm, X[1] / norm, X[2] / norm, 0.0f };
    return v;
}

static float distance_to_origin(const hpm_camera *c, int px, int py, float depth, f4 n)
{
    float X[3];
    get_3d_point(c, px, py, depth, X);
    return -(n.x * X[0] + n.y * X[1] + n.z * X[2]);
}

static float depth_from_plane(const hpm_camera *c, f4 pl, int px, int py)
{
    return -pl.w * c->K[0] / ((px - c->K[2]) * pl.x + (c->K[0] / c->K[4]) * (py - c->K[5]) * pl.y + c->K[0] * pl.z);
}

static void normalize3(f4 *v)
{
    const float n2 = v->x * v->x + v->y * v->y + v->z * v->z;
    const float inv = 1.0f / sqrtf(n2);
    v->x *= inv; v->y *= inv; v->z *= inv;
}

static f4 rotate_to_world(const hpm_camera *c, f4 p) /* TransformNormal, HPM.cu:322-330 */
{
    f4 r;
    r.x = c->R[0] * p.x + c->R[3] * p.y + c->R[6] * p.z;
    r.y = c->R[1] * p.x + c->R[4] * p.y + c->R[7] * p.z;
    r.z = c->R[2] * p.x + c->R[5] * p.y + c->R[8] * p.z;
    r.w = p.w;
    return r;
}

static f4 rotate_to_cam(const hpm_camera *c, f4 p) /* TransformNormal2RefCam, HPM.cu:332-340 */
{
    f4 r;
    r.x = c->R[0] * p.x + c->R[1] * p.y + c->R[2] * p.z;
    r.y = c->R[3] * p.x + c->R[4] * p.y + c->R[5] * p.z;
    r.z = c->R[6] * p.x + c->R[7] * p.y + c->R[8] * p.z;
    r.w = p.w;
    return r;
}

static inline f2 corresponding_point(const float H[9], int x, int y)
{
    const float px = H[0] * x + H[1] * y + H[2];
    const float py = H[3] * x + H[4] * y + H[5];
    const float pz = H[6] * x + H[7] * y + H[8];
    f2 r = { px / pz, py / pz };
    return r;
}

/* ---------------- random planes (HPM.cu:159-230) ---------------- */

typedef struct { uint64_t seed; uint32_t view, x, y; uint32_t *draw; } rng_t;

static inline float rng_uniform(rng_t *r)
{
    const uint32_t bits = hpm_rng_bits(r->seed, r->view, r->x, r->y, *r->draw);
    (*r->draw)++;
    return hpm_bits_to_uniform(bits);
}

#define MARSAGLIA_MAX_TRIES 4096

static f4 random_normal(const hpm_camera *c, int px, int py, rng_t *rng, float depth)
{
    f4 n;
    float q1 = 1.0f, q2 = 1.0f, s = 2.0f;
    int tries = 0;
    while (s >= 1.0f && tries < MARSAGLIA_MAX_TRIES) {
        q1 = 2.0f * rng_uniform(rng) - 1.0f;
        q2 = 2.0f * rng_uniform(rng) - 1.0f;
        s = q1 * q1 + q2 * q2;
        ++tries;
    }
    if (s >= 1.0f) { q1 = 0.0f; q2 = 0.0f; s = 0.0f; }
    const float sq = sqrtf(1.0f - s);
    n.x = 2.0f * q1 * sq;
    n.y = 2.0f * q2 * sq;
    n.z = 1.0f - 2.0f * s;
    n.w = 0.0f;
    const f4 vd = view_direction(c, px, py, depth);
    const float dot = n.x * vd.x + n.y * vd.y + n.z * vd.z;
    if (dot > 0.0f) { n.x = -n.x; n.y = -n.y; n.z = -n.z; }
    normalize3(&n);
    return n;
}

static f4 perturbed_normal(const hpm_camera *c, int px, int py, f4 normal, rng_t *rng, float perturbation)
{
    const f4 vd = view_direction(c, px, py, 1.0f);
    const float a1 = (rng_uniform(rng) - 0.5f) * perturbation;
    const float a2 = (rng_uniform(rng) - 0.5f) * perturbation;
    const float a3 = (rng_uniform(rng) - 0.5f) * perturbation;
    const float s1 = hpm_sinf(a1), s2 = hpm_sinf(a2), s3 = hpm_sinf(a3);
    const float c1 = hpm_cosf(a1), c2 = hpm_cosf(a2), c3 = hpm_cosf(a3);
    float R[9];
    R[0] = c2 * c3;
    R[1] = c3 * s1 * s2 - c1 * s3;
    R[2] = s1 * s3 + c1 * c3 * s2;
    R[3] = c2 * s3;
    R[4] = c1 * c3 + s1 * s2 * s3;
    R[5] = c1 * s2 * s3 - c3 * s1;
    R[6] = -s2;
    R[7] = c2 * s1;
    R[8] = c1 * c2;
    f4 np;
    np.x = R[0] * normal.x + R[1] * normal.y + R[2] * normal.z;
    np.y = R[3] * normal.x + R[4] * normal.y + R[5] * normal.z;
    np.z = R[6] * normal.x + R[7] * normal.y + R[8] * normal.z;
    np.w = normal.w;
    if (np.x * vd.x + np.y * vd.y + np.z * vd.z >= 0.0f) np = normal;
    normalize3(&np);
    return np;
}

static f4 random_plane(const hpm_camera *c, int px, int py, rng_t *rng, float dmin, float dmax)
{
    const float depth = rng_uniform(rng) * (dmax - dmin) + dmin;
    f4 pl = random_normal(c, px, py, rng, depth);
    pl.w = distance_to_origin(c, px, py, depth, pl);
    return pl;
}

/* ---------------- costs ---------------- */

float ora_bilateral_ncc(const float *ref, const hpm_camera *rc, const float *src, const hpm_camera *sc,
                        int px, int py, const float plane[4], const hpm_params *prm)
{
    /* HPM.cu:375-448.  The reference patch statistics (view independent) are
     * formed first, then the source moments; both follow include/hpm_fp.h. */
    const float cost_max = 2.0f;
    const int rw = rc->width, rh = rc->height, sw = sc->width, sh = sc->height;
    const float center = texel(ref, rw, rh, px, py);
    const float two_ss = 2.0f * prm->sigma_spatial * prm->sigma_spatial;
    const float two_sc = 2.0f * prm->sigma_color * prm->sigma_color;
    const float cs = g_ncc_shift ? center : 0.0f;
    float pw[36], pwr[36];
    float s_r = 0.f, s_rr = 0.f, s_w = 0.f;
    for (int i = 0; i < 6; ++i) {
        float r_r = 0.f, r_rr = 0.f, r_w = 0.f;
        const int dx = -5 + 2 * i;
        for (int j = 0; j < 6; ++j) {
            const int dy = -5 + 2 * j;
            const float r = texel(ref, rw, rh, px + dx, py + dy);
            const float sd = sqrtf((float)(dx * dx + dy * dy));
            const float w = hpm_expf(-sd / two_ss - fabsf(r - center) / two_sc);
            const float rs = r - cs;
            const float wr = w * rs;
            pw[i * 6 + j] = w;
            pwr[i * 6 + j] = wr;
            r_r += wr;
            r_rr = hpm_fma(wr, rs, r_rr);
            r_w += w;
        }
        s_r += r_r; s_rr += r_rr; s_w += r_w;
    }
    const float inv_w = 1.0f / s_w;
    const float mean_r = s_r * inv_w;
    const float var_r = s_rr * inv_w - mean_r * mean_r;
    const float kMinVar = 1e-5f;
    if (var_r < kMinVar) return cost_max;

    /* homography factored as H = A - b m^T (include/hpm_geometry.h) */
    float A[9], bv[3], kinv[4], m[3], H[9];
    hpm_view_basis(rc, sc, A, bv);
    hpm_ref_kinv(rc, kinv);
    hpm_plane_m(kinv, plane[0], plane[1], plane[2], plane[3], m);
    hpm_homography(A, bv, m, H);
    float iz_c;
    {
        const float fx = (float)px, fy = (float)py;
        const float cx = hpm_fma(H[0], fx, hpm_fma(H[1], fy, H[2]));
        const float cy = hpm_fma(H[3], fx, hpm_fma(H[4], fy, H[5]));
        const float cz = hpm_fma(H[6], fx, hpm_fma(H[7], fy, H[8]));
        iz_c = 1.0f / cz;
        const float ux = cx * iz_c, uy = cy * iz_c;
        if (ux >= sw || ux < 0.0f || uy >= sh || uy < 0.0f) return cost_max;
    }
    float s_s = 0.f, s_ss = 0.f, s_rs = 0.f;
    float vshift = 0.0f;
    for (int i = 0; i < 6; ++i) {
        const float x = (float)(px - 5 + 2 * i);
        float r_s = 0.f, r_ss = 0.f, r_rs = 0.f;
        for (int k = 0; k < 6; ++k) {
            const float y = (float)(py - 5 + 2 * k);
            const float qx = hpm_fma(H[0], x, hpm_fma(H[1], y, H[2]));
            const float qy = hpm_fma(H[3], x, hpm_fma(H[4], y, H[5]));
            const float qz = hpm_fma(H[6], x, hpm_fma(H[7], y, H[8]));
            const float iz = hpm_recip_near(qz, iz_c);
            const float v0 = ora_tex2d(src, sw, sh, hpm_fma(qx, iz, 0.5f), hpm_fma(qy, iz, 0.5f));
            if (g_ncc_shift && i == 0 && k == 0) vshift = v0;
            const float v = v0 - vshift;
            const float ws = pw[i * 6 + k] * v;
            r_s += ws;
            r_ss = hpm_fma(ws, v, r_ss);
            r_rs = hpm_fma(pwr[i * 6 + k], v, r_rs);
        }
        s_s += r_s; s_ss += r_ss; s_rs += r_rs;
    }
    s_s *= inv_w; s_ss *= inv_w; s_rs *= inv_w;
    const float var_s = s_ss - s_s * s_s;
    if (var_s < kMinVar) return cost_max;
    const float cov = s_rs - mean_r * s_s;
    const float vrs = sqrtf(var_r * var_s);
    float c = 1.0f - cov / vrs;
    /* max(0, min(2, c)) with fminf/fmaxf NaN semantics (the non-NaN operand wins) */
    c = fminf(cost_max, c);
    c = fmaxf(0.0f, c);
    return c;
}

double ora_bilateral_ncc64(const float *ref, const hpm_camera *rc, const float *src, const hpm_camera *sc,
                        int px, int py, const float plane[4], const hpm_params *prm)
{
    /* ora_bilateral_ncc with the same weights and the same float sample
     * positions and filtered samples, but every moment accumulated and the
     * NCC formed in double: the reference the precision form's accumulation
     * errors are measured against. */
    const float cost_max = 2.0f;
    const int rw = rc->width, rh = rc->height, sw = sc->width, sh = sc->height;
    const float center = texel(ref, rw, rh, px, py);
    const float two_ss = 2.0f * prm->sigma_spatial * prm->sigma_spatial;
    const float two_sc = 2.0f * prm->sigma_color * prm->sigma_color;
    double pw[36];
    double s_r = 0, s_w = 0;
    for (int i = 0; i < 6; ++i) {
        const int dx = -5 + 2 * i;
        for (int j = 0; j < 6; ++j) {
            const int dy = -5 + 2 * j;
            const float r = texel(ref, rw, rh, px + dx, py + dy);
            const float sd = sqrtf((float)(dx * dx + dy * dy));
            const float w = hpm_expf(-sd / two_ss - fabsf(r - center) / two_sc);
            pw[i * 6 + j] = w;
            s_r += (double)w * r;
            s_w += w;
        }
    }
    const double mean_r = s_r / s_w;
    double var_r = 0;
    for (int i = 0; i < 36; ++i) {
        const int dx = -5 + 2 * (i / 6), dy = -5 + 2 * (i % 6);
        const double d = (double)texel(ref, rw, rh, px + dx, py + dy) - mean_r;
        var_r += pw[i] * d * d;
    }
    var_r /= s_w;
    const float kMinVar = 1e-5f;
    if (var_r < kMinVar) return cost_max;

    /* homography factored as H = A - b m^T (include/hpm_geometry.h) */
    float A[9], bv[3], kinv[4], m[3], H[9];
    hpm_view_basis(rc, sc, A, bv);
    hpm_ref_kinv(rc, kinv);
    hpm_plane_m(kinv, plane[0], plane[1], plane[2], plane[3], m);
    hpm_homography(A, bv, m, H);
    float iz_c;
    {
        const float fx = (float)px, fy = (float)py;
        const float cx = hpm_fma(H[0], fx, hpm_fma(H[1], fy, H[2]));
        const float cy = hpm_fma(H[3], fx, hpm_fma(H[4], fy, H[5]));
        const float cz = hpm_fma(H[6], fx, hpm_fma(H[7], fy, H[8]));
        iz_c = 1.0f / cz;
        const float ux = cx * iz_c, uy = cy * iz_c;
        if (ux >= sw || ux < 0.0f || uy >= sh || uy < 0.0f) return cost_max;
    }
    double vals[36];
    for (int i = 0; i < 6; ++i) {
        const float x = (float)(px - 5 + 2 * i);
        for (int k = 0; k < 6; ++k) {
            const float y = (float)(py - 5 + 2 * k);
            const float qx = hpm_fma(H[0], x, hpm_fma(H[1], y, H[2]));
            const float qy = hpm_fma(H[3], x, hpm_fma(H[4], y, H[5]));
            const float qz = hpm_fma(H[6], x, hpm_fma(H[7], y, H[8]));
            const float iz = hpm_recip_near(qz, iz_c);
            vals[i * 6 + k] = ora_tex2d(src, sw, sh, hpm_fma(qx, iz, 0.5f), hpm_fma(qy, iz, 0.5f));
        }
    }
    /* two-pass moments in double */
    double mean_s = 0;
    for (int i = 0; i < 36; ++i) mean_s += pw[i] * vals[i];
    mean_s /= s_w;
    double var_s = 0, cov = 0;
    for (int i = 0; i < 36; ++i) {
        const int dx = -5 + 2 * (i / 6), dy = -5 + 2 * (i % 6);
        const double dr = (double)texel(ref, rw, rh, px + dx, py + dy) - mean_r;
        const double ds = vals[i] - mean_s;
        var_s += pw[i] * ds * ds;
        cov += pw[i] * dr * ds;
    }
    var_s /= s_w;
    cov /= s_w;
    if (var_s < kMinVar) return cost_max;
    double c = 1.0 - cov / sqrt(var_r * var_s);
    c = c < 0.0 ? 0.0 : (c > 2.0 ? 2.0 : c);
    return c;
}

void ora_eval_costs(const float *const *images, const hpm_camera *cams, int num_images,
                    const hpm_params *params, int n, const int32_t *px, const float *planes, float *out)
{
    const int S = num_images - 1;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < S; ++j)
            out[(size_t)k * S + j] = ora_bilateral_ncc(images[0], &cams[0], images[j + 1], &cams[j + 1],
                                                      px[2 * k], px[2 * k + 1], planes + 4 * (size_t)k, params);
}

static void cost_vector(const float *const *images, const hpm_camera *cams, int num_images,
                        const hpm_params *prm, int px, int py, f4 pl, float *out)
{
    const float p4[4] = { pl.x, pl.y, pl.z, pl.w };
    for (int i = 1; i < num_images; ++i)
        out[i - 1] = ora_bilateral_ncc(images[0], &cams[0], images[i], &cams[i], px, py, p4, prm);
}

float ora_initial_cost(const float *const *images, const hpm_camera *cams, int num_images,
                       const hpm_params *prm, int px, int py, const float plane[4], uint32_t *selected)
{
    const float cost_max = 2.0f;
    float cv[32], sorted[32];
    int count = 0, valid = 0;
    const f4 pl = { plane[0], plane[1], plane[2], plane[3] };
    cost_vector(images, cams, num_images, prm, px, py, pl, cv);
    for (int i = 0; i < num_images - 1; ++i) {
        sorted[i] = cv[i];
        ++count;
        if (cv[i] < cost_max) ++valid;
    }
    /* insertion sort (HPM.cu:15-24) */
    for (int i = 1; i < count; ++i) {
        const float t = sorted[i];
        int j;
        for (j = i; j >= 1 && t < sorted[j - 1]; --j) sorted[j] = sorted[j - 1];
        sorted[j] = t;
    }
    *selected = 0;
    const int top_k = valid < prm->top_k ? valid : prm->top_k;
    if (top_k > 0) {
        float cost = 0.0f;
        for (int i = 0; i < top_k; ++i) cost += sorted[i];
        const float thr = sorted[top_k - 1];
        for (int i = 0; i < num_images - 1; ++i)
            if (cv[i] <= thr) *selected |= (1u << i);
        return cost / top_k;
    }
    return cost_max;
}

/* ComputeGeomConsistencyCost (HPM.cu:539-564) as the point transfer of
 * hpm_view_transfer / hpm_transfer (include/hpm_geometry.h): forward into the
 * source at the hypothesis depth, a clamped point read of the source depth at
 * the truncated position, back into the reference. */
float ora_geom_cost(const float *src_depth, const hpm_camera *rc, const hpm_camera *sc,
                    const float plane[4], int px, int py)
{
    const float max_cost = 3.0f;
    const f4 pl = { plane[0], plane[1], plane[2], plane[3] };
    const float depth = depth_from_plane(rc, pl, px, py);
    float Gf[9], gf[3], Gb[9], gb[3];
    hpm_view_transfer(rc, sc, Gf, gf);
    hpm_view_transfer(sc, rc, Gb, gb);
    float sx, sy;
    hpm_transfer(Gf, gf, (float)px, (float)py, depth, &sx, &sy);
    const float d = texel(src_depth, sc->width, sc->height, f2i_rz(sx), f2i_rz(sy));
    if (d == 0.0f) return max_cost;
    float bx, by;
    hpm_transfer(Gb, gb, sx, sy, d, &bx, &by);
    const float dx = px - bx, dy = py - by;
    const float e = sqrtf(dx * dx + dy * dy);
    return (e < max_cost) ? e : max_cost; /* fminf: NaN -> 3 */
}

float ora_depth_from_plane(const hpm_camera *c, const float plane[4], int px, int py)
{
    const f4 pl = { plane[0], plane[1], plane[2], plane[3] };
    return depth_from_plane(c, pl, px, py);
}

float ora_texture(const uint8_t *canny, int width, int height, int px, int py)
{
    int total = 0, edges = 0;
    for (int i = -5; i < 6; i += 2)
        for (int j = -5; j < 6; j += 2) {
            const int x = px + j, y = py + i;
            if (x >= 0 && x < width && y >= 0 && y < height) {
                ++total;
                if (canny[y * width + x] >= 1) ++edges;
            }
        }
    const float frac = edges * 1.0f / total;
    return (float)(((double)frac + 0.00005) / ((double)frac + 0.0001));
}

/* ---------------- RandomInitialization (HPM.cu:567-763) ---------------- */

static float spatial_gauss(float x1, float y1, float x2, float y2, float sigma) /* HPM.cu:142-146 */
{
    const float dx = x1 - x2, dy = y1 - y2;
    const float dis = dx * dx + dy * dy - 0.0f;
    return (float)exp(-1.0 * dis / (2 * sigma * sigma));
}

static float range_gauss(float x, float sigma) /* HPM.cu:148-152 */
{
    const float xp = x - 0.0f;
    return (float)exp(-1.0 * (xp * xp) / (2 * sigma * sigma));
}

static void init_pixel(const float *const *images, const hpm_camera *cams, int num_images,
                       const hpm_params *prm, ora_state *st, uint64_t seed, uint32_t view_id,
                       int px, int py)
{
    const hpm_camera *c0 = &cams[0];
    const int W = c0->width, H = c0->height;
    const int center = py * W + px;
    const uint32_t mode = prm->mode;
    const int geom = (mode & HPM_MODE_GEOM) != 0, prior = (mode & HPM_MODE_PRIOR) != 0;
    const int hier = (mode & HPM_MODE_HIERARCHY) != 0, ups = (mode & HPM_MODE_UPSAMPLE) != 0;
    const int mand = (mode & HPM_MODE_MAND) != 0;
    st->rng_draw[center] = 0;
    rng_t rng = { seed, view_id, (uint32_t)px, (uint32_t)py, &st->rng_draw[center] };

    if (!prior && !mand) st->texture[center] = ora_texture(st->canny, W, H, px, py);

    float tmp[4];
    if (!geom && !hier && !prior) {
        const f4 pl = random_plane(c0, px, py, &rng, prm->depth_min, prm->depth_max);
        store4(st->planes, center, pl);
        tmp[0] = pl.x; tmp[1] = pl.y; tmp[2] = pl.z; tmp[3] = pl.w;
        st->costs[center] = ora_initial_cost(images, cams, num_images, prm, px, py, tmp, &st->selected_views[center]);
    } else if (prior) {
        if (st->plane_masks[center] > 0) {
            if (st->confidences[center] > 0.3) {
                f4 pl = load4(st->planes, center);
                const float depth = pl.w;
                pl.w = distance_to_origin(c0, px, py, depth, pl);
                store4(st->planes, center, pl);
                st->costs[center] = 0.1f;
            } else if (st->costs[center] > 0.1f) {
                const float perturbation = 0.02f;
                const f4 prior_pl = load4(st->prior_planes, center);
                float dp = prior_pl.w;
                const float dmin_p = (1 - 3 * perturbation) * dp;
                const float dmax_p = (1 + 3 * perturbation) * dp;
                dp = rng_uniform(&rng) * (dmax_p - dmin_p) + dmin_p;
                f4 pp = perturbed_normal(c0, px, py, prior_pl, &rng, (float)(3 * perturbation * M_PI));
                pp.w = dp;
                store4(st->planes, center, pp);
                tmp[0] = pp.x; tmp[1] = pp.y; tmp[2] = pp.z; tmp[3] = pp.w;
                st->costs[center] = ora_initial_cost(images, cams, num_images, prm, px, py, tmp, &st->selected_views[center]);
            } else {
                f4 pl = load4(st->planes, center);
                const float depth = pl.w;
                pl.w = distance_to_origin(c0, px, py, depth, pl);
                store4(st->planes, center, pl);
                tmp[0] = pl.x; tmp[1] = pl.y; tmp[2] = pl.z; tmp[3] = pl.w;
                st->costs[center] = ora_initial_cost(images, cams, num_images, prm, px, py, tmp, &st->selected_views[center]);
            }
        } else {
            f4 pl = load4(st->planes, center);
            const float depth = pl.w;
            pl.w = distance_to_origin(c0, px, py, depth, pl);
            store4(st->planes, center, pl);
            if (st->confidences[center] > 0.3) st->costs[center] = 0.1f;
        }
    } else if (ups) {
        const float scale = (float)(1.0 * prm->scaled_cols / W);
        const float sigmad = 0.50f, sigmar = 25.5f;
        const float sc_f = (float)prm->scaled_cols, sr_f = (float)prm->scaled_rows;
        const float ia = W / sc_f, ib = H / sr_f;
        const int image_scale = (int)(ia > ib ? ia : ib);
        const int win = image_scale * image_scale + 1;
        const int nn = win / 2;
        const float o_y = py * scale, o_x = px * scale;
        const float ref_pix = texel(images[0], W, H, px, py);
        float nf = 0.0f;
        f4 nt = { 0, 0, 0, 0 };
        for (int j = -nn; j <= nn; ++j) {
            int r_y = f2i_rz(o_y + j);
            r_y = (r_y > 0 ? (r_y < sr_f ? r_y : prm->scaled_rows - 1) : 0);
            const int r_ys = py + j;
            for (int i = -nn; i <= nn; ++i) {
                int r_x = f2i_rz(o_x + i);
                r_x = (r_x > 0 ? (r_x < sc_f ? r_x : prm->scaled_cols - 1) : 0);
                const int s_center = (int)(r_y * sc_f + r_x);
                f4 sn = load4(st->scaled_planes, s_center);
                const float nb = texel(images[0], W, H, px + i, r_ys);
                const float sg = spatial_gauss(o_x, o_y, (float)r_x, (float)r_y, sigmad);
                const float rg = range_gauss(fabsf(ref_pix - nb), sigmar);
                const float tg = sg * rg;
                nf += tg;
                sn.x = sn.x * tg; sn.y = sn.y * tg; sn.z = sn.z * tg;
                nt.x = nt.x + sn.x; nt.y = nt.y + sn.y; nt.z = nt.z + sn.z;
            }
        }
        nt.x = nt.x / nf; nt.y = nt.y / nf; nt.z = nt.z / nf;
        normalize3(&nt);
        /* the pre-cost plane: zero normal and the upsampled depth as w (HPM.cu:689) */
        f4 cur = load4(st->planes, center);
        tmp[0] = 0.0f; tmp[1] = 0.0f; tmp[2] = 0.0f; tmp[3] = cur.w;
        st->costs[center] = ora_initial_cost(images, cams, num_images, prm, px, py, tmp, &st->selected_views[center]);
        st->pre_costs[center] = st->costs[center];
        f4 pl = rotate_to_cam(c0, nt);
        const float depth = cur.w;
        pl.w = distance_to_origin(c0, px, py, depth, pl);
        store4(st->planes, center, pl);
        tmp[0] = pl.x; tmp[1] = pl.y; tmp[2] = pl.z; tmp[3] = pl.w;
        st->costs[center] = ora_initial_cost(images, cams, num_images, prm, px, py, tmp, &st->selected_views[center]);
    } else {
        if (mand && !(st->confidences[center] >= 0.3)) {
            const float t = ora_texture(st->canny, W, H, px, py);
            if (t > 0.5) st->confidences[center] = 0.1f;
        }
        f4 pl = hier ? load4(st->scaled_planes, center) : load4(st->planes, center);
        pl = rotate_to_cam(c0, pl);
        const float depth = pl.w;
        pl.w = distance_to_origin(c0, px, py, depth, pl);
        store4(st->planes, center, pl);
        tmp[0] = pl.x; tmp[1] = pl.y; tmp[2] = pl.z; tmp[3] = pl.w;
        st->costs[center] = ora_initial_cost(images, cams, num_images, prm, px, py, tmp, &st->selected_views[center]);
    }
}

void ora_random_init(const float *const *images, const hpm_camera *cams, int num_images,
                     const hpm_params *params, ora_state *st, uint64_t seed, uint32_t view_id)
{
    const int W = cams[0].width, H = cams[0].height;
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
            init_pixel(images, cams, num_images, params, st, seed, view_id, x, y);
}

/* ---------------- checkerboard propagation (HPM.cu:843-1873, 1875-2791) ---------------- */

/* Direction order of the reference (HPM.cu:1379):
 * 0 left_up, 1 up_far, 2 right_up, 3 down_far, 4 right_down, 5 left_far, 6 left_down, 7 right_far. */

static int far_search(const float *costs, int W, int H, int px, int py, int dx, int dy, int keep_max, int *pos)
{
    /* first candidate at 5 px, then 4 more every 2 px while inside the image */
    int x = px + 5 * dx, y = py + 5 * dy;
    if (x < 0 || x >= W || y < 0 || y >= H) return 0;
    int best = y * W + x;
    float bc = costs[best];
    for (int i = 1; i < 5; ++i) {
        const int xi = px + (5 + 2 * i) * dx, yi = py + (5 + 2 * i) * dy;
        if (xi < 0 || xi >= W || yi < 0 || yi >= H) break;
        const int q = yi * W + xi;
        if (keep_max ? (bc < costs[q]) : (costs[q] < bc)) { bc = costs[q]; best = q; }
    }
    *pos = best;
    return 1;
}

/* Diagonal "V" paths: start offset (sx, sy); even steps move along axis a by
 * (ax, ay), odd steps along (bx, by); 7 steps, stop at the first step outside. */
static void v_path_scan(const float *costs, int W, int H, int x, int y, int ax, int ay, int bx, int by,
                        float *bc, int *best)
{
    for (int i = 0; i < 7; ++i) {
        if (i % 2 == 0) { x += ax; y += ay; } else { x += bx; y += by; }
        if (x >= 0 && x < W && y < H && y >= 0) {
            const int q = y * W + x;
            if (costs[q] < *bc) { *bc = costs[q]; *best = q; }
        } else break;
    }
}

static int judge_extend(int iter, int ext_iter, const float *row, int S, int flag)
{
    if (!flag) return 0;
    const int it = 3 - ext_iter;
    const float good_thr = (float)(0.8 * exp(-iter * iter * it / 90.0));
    const float bad_thr = 1.2f;
    int good = 0, bad = 0;
    for (int i = 0; i < S; ++i) {
        if (row[i] < good_thr) ++good;
        if (row[i] > bad_thr) ++bad;
    }
    return !(good >= 1 && bad <= 2);
}

static float prior_score(float final_cost, float depth_now, float depth_prior, f4 prior_pl, f4 pl,
                         float texture, float two_dss, float two_ass)
{
    const float gamma = 0.5f, beta = 0.18f;
    const float dd = depth_now - depth_prior;
    const float nd = fabsf(prior_pl.x - pl.x) + fabsf(prior_pl.y - pl.y) + fabsf(prior_pl.z - pl.z);
    const float prior = (float)(gamma * (1.2 - 0.2 * texture) + (double)(hpm_expf(-dd * dd / two_dss) * hpm_expf(-nd * nd / two_ass)));
    return (float)(exp(-final_cost * final_cost / beta * (1 + 0.2 * texture)) * (double)prior);
}

static void refinement(const float *const *images, const float *const *depths, const hpm_camera *cams,
                       int num_images, const hpm_params *prm, const ora_state *st, f4 *plane, float *depth,
                       float *cost, rng_t *rng, const float *vw, float weight_norm, float *restricted_cost,
                       int px, int py, float texture)
{
    const hpm_camera *c0 = &cams[0];
    const int center = py * c0->width + px;
    const int S = num_images - 1;
    const int prior = (prm->mode & HPM_MODE_PRIOR) != 0;
    const int geom = (prm->mode & HPM_MODE_GEOM) != 0;
    const float perturbation = 0.02f;
    const float gamma = 0.5f, beta = 0.18f;
    const float depth_sigma = (prm->depth_max - prm->depth_min) / 64.0f;
    const float two_dss = 2 * depth_sigma * depth_sigma;
    const float angle_sigma = (float)(M_PI * (5.0f / 180.0f));
    const float two_ass = 2 * angle_sigma * angle_sigma;
    float depth_prior = 0.0f;
    float depth_rand;
    f4 plane_rand;
    const int use_prior = prior && st->plane_masks[center] > 0;
    if (use_prior) {
        const f4 pp = load4(st->prior_planes, center);
        depth_prior = depth_from_plane(c0, pp, px, py);
        depth_rand = rng_uniform(rng) * 6 * depth_sigma + (depth_prior - 3 * depth_sigma);
        plane_rand = perturbed_normal(c0, px, py, pp, rng, angle_sigma);
    } else {
        depth_rand = rng_uniform(rng) * (prm->depth_max - prm->depth_min) + prm->depth_min;
        plane_rand = random_normal(c0, px, py, rng, *depth);
    }
    const float dmin_p = (1 - perturbation) * *depth;
    const float dmax_p = (1 + perturbation) * *depth;
    const float depth_perturbed = rng_uniform(rng) * (dmax_p - dmin_p) + dmin_p;
    const f4 plane_perturbed = perturbed_normal(c0, px, py, *plane, rng, (float)(perturbation * M_PI));

    const float depths5[5] = { depth_rand, *depth, depth_rand, *depth, depth_perturbed };
    const f4 normals5[5] = { *plane, plane_rand, plane_rand, plane_perturbed, *plane };
    (void)gamma; (void)beta;
    for (int i = 0; i < 5; ++i) {
        float cv[32];
        f4 t = normals5[i];
        t.w = distance_to_origin(c0, px, py, depths5[i], t);
        cost_vector(images, cams, num_images, prm, px, py, t, cv);
        float tc = 0.0f;
        const float t4[4] = { t.x, t.y, t.z, t.w };
        for (int j = 0; j < S; ++j)
            if (vw[j] > 0) {
                if (geom) tc += vw[j] * (cv[j] + 0.2f * ora_geom_cost(depths[j + 1], c0, &cams[j + 1], t4, px, py));
                else tc += vw[j] * cv[j];
            }
        tc /= weight_norm;
        const float depth_before = depth_from_plane(c0, t, px, py);
        if (use_prior) {
            const f4 pp = load4(st->prior_planes, center);
            const float rt = prior_score(tc, depths5[i], depth_prior, pp, t, texture, two_dss, two_ass);
            if (depth_before >= prm->depth_min && depth_before <= prm->depth_max && rt > *restricted_cost) {
                *depth = depth_before; *plane = t; *cost = tc; *restricted_cost = rt;
            }
        } else {
            if (depth_before >= prm->depth_min && depth_before <= prm->depth_max && tc < *cost) {
                *depth = depth_before; *plane = t; *cost = tc;
            }
        }
    }
}

static int find_min_index(const float *c, int n) /* HPM.cu:41-52: ties -> last */
{
    float m = c[0]; int idx = 0;
    for (int i = 1; i < n; ++i) if (c[i] <= m) { m = c[i]; idx = i; }
    return idx;
}

static int find_max_index(const float *c, int n) /* HPM.cu:54-65: ties -> last */
{
    float m = c[0]; int idx = 0;
    for (int i = 1; i < n; ++i) if (c[i] >= m) { m = c[i]; idx = i; }
    return idx;
}

/* Shared part of both propagation variants: direction search, extension,
 * joint view selection, final costs.  Returns via the out-parameters. */
typedef struct {
    float cost_array[8][32];
    int flag[8];
    int positions[8];
    float view_weights[32];
    uint32_t temp_selected;
    int num_selected;
    float weight_norm;
    float final_costs[8];
} sweep_ctx;

static void propagate_common(const float *const *images, const float *const *depths, const hpm_camera *cams,
                             int num_images, const hpm_params *prm, ora_state *st, int iter, int px, int py,
                             rng_t *rng, sweep_ctx *s)
{
    const hpm_camera *c0 = &cams[0];
    const int W = c0->width, H = c0->height;
    const int center = py * W + px;
    const int S = num_images - 1;
    const int geom = (prm->mode & HPM_MODE_GEOM) != 0;
    const float *costs = st->costs;

    memset(s->cost_array, 0, sizeof(s->cost_array));
    s->cost_array[0][0] = 2.0f; /* `float cost_array[8][32] = { 2.0f }` (HPM.cu:1378) */
    for (int i = 0; i < 8; ++i) s->flag[i] = 0;
    int pos[8];
    pos[0] = center - 5 - 6 * W; pos[2] = center + 6 - 5 * W; pos[4] = center + 5 + 6 * W; pos[6] = center - 6 + 5 * W;
    pos[5] = center - 5; pos[7] = center + 5; pos[1] = center - 5 * W; pos[3] = center + 5 * W;

    /* far directions (HPM.cu:1385-1475) */
    if (far_search(costs, W, H, px, py, 0, -1, 0, &pos[1])) s->flag[1] = 1;
    if (s->flag[1]) cost_vector(images, cams, num_images, prm, px, py, load4(st->planes, pos[1]), s->cost_array[1]);
    if (far_search(costs, W, H, px, py, 0, 1, 0, &pos[3])) s->flag[3] = 1;
    if (s->flag[3]) cost_vector(images, cams, num_images, prm, px, py, load4(st->planes, pos[3]), s->cost_array[3]);
    if (far_search(costs, W, H, px, py, -1, 0, 0, &pos[5])) s->flag[5] = 1;
    if (s->flag[5]) cost_vector(images, cams, num_images, prm, px, py, load4(st->planes, pos[5]), s->cost_array[5]);
    if (far_search(costs, W, H, px, py, 1, 0, 1, &pos[7])) s->flag[7] = 1;
    if (s->flag[7]) cost_vector(images, cams, num_images, prm, px, py, load4(st->planes, pos[7]), s->cost_array[7]);

    /* V paths (HPM.cu:1478-1608) */
    if (px > 4 && py > 5) {
        s->flag[0] = 1;
        float bc = costs[pos[0]]; int best = pos[0];
        v_path_scan(costs, W, H, px - 5, py - 6, -2, 0, 0, -2, &bc, &best);
        pos[0] = best;
        cost_vector(images, cams, num_images, prm, px, py, load4(st->planes, pos[0]), s->cost_array[0]);
    }
    if (px < W - 6 && py > 4) {
        s->flag[2] = 1;
        float bc = costs[pos[2]]; int best = pos[2];
        v_path_scan(costs, W, H, px + 6, py - 5, 0, -2, 2, 0, &bc, &best);
        pos[2] = best;
        cost_vector(images, cams, num_images, prm, px, py, load4(st->planes, pos[2]), s->cost_array[2]);
    }
    if (px < W - 5 && py < H - 6) {
        s->flag[4] = 1;
        float bc = costs[pos[4]]; int best = pos[4];
        v_path_scan(costs, W, H, px + 5, py + 6, 2, 0, 0, 2, &bc, &best);
        pos[4] = best;
        cost_vector(images, cams, num_images, prm, px, py, load4(st->planes, pos[4]), s->cost_array[4]);
    }
    if (px > 5 && py < H - 5) {
        s->flag[6] = 1;
        float bc = costs[pos[6]]; int best = pos[6];
        v_path_scan(costs, W, H, px - 6, py + 5, 0, 2, -2, 0, &bc, &best);
        pos[6] = best;
        cost_vector(images, cams, num_images, prm, px, py, load4(st->planes, pos[6]), s->cost_array[6]);
    }

    /* Extended propagation: `symbol_eight_orientations[10] = { true }` enables
     * only orientation 0 (left_up) (HPM.cu:1609-1680, 1063-1126). */
    for (int it = 0; it < 3; ++it) {
        if (!judge_extend(iter, it, s->cost_array[0], S, s->flag[0])) break;
        if (px > 4 + 8 * it && py > 5 + 8 * it) {
            const int sx = px - 5 - 8 * it, sy = py - 6 - 8 * it;
            int best = sy * W + sx;
            float bc = costs[best];
            v_path_scan(costs, W, H, sx, sy, -2, 0, 0, -2, &bc, &best);
            if (bc > costs[pos[0]]) {
                best = pos[0]; /* previous choice is strictly better: keep its row */
            } else {
                cost_vector(images, cams, num_images, prm, px, py, load4(st->planes, best), s->cost_array[0]);
            }
            pos[0] = best;
        }
        /* else: flag[0] is set (JudgeExtend checked it) -> position and row unchanged */
    }
    for (int i = 0; i < 8; ++i) s->positions[i] = pos[i];

    /* Multi-hypothesis joint view selection (HPM.cu:1686-1751) */
    float priors[32];
    for (int j = 0; j < 32; ++j) { priors[j] = 0.0f; s->view_weights[j] = 0.0f; }
    const int nbr[4] = { center - W * 5, center + W * 5, center - 5, center + 5 };
    for (int i = 0; i < 4; ++i)
        if (s->flag[2 * i + 1])
            for (int j = 0; j < S; ++j) {
                if ((st->selected_views[nbr[i]] >> j) & 1u) priors[j] += 0.9f;
                else priors[j] += 0.1f;
            }
    float probs[32];
    for (int j = 0; j < 32; ++j) probs[j] = 0.0f;
    const float cost_thr = (float)(0.8 * hpm_expf((float)(iter * iter) / (-90.0f)));
    for (int i = 0; i < S; ++i) {
        float count = 0; int count_false = 0; float tmpw = 0;
        for (int j = 0; j < 8; ++j) {
            const float c = s->cost_array[j][i];
            if (c < cost_thr) { tmpw += hpm_expf(c * c / (-0.18f)); count++; }
            if (c > 1.2f) count_false++;
        }
        if (count > 2 && count_false < 3) probs[i] = tmpw / count;
        else if (count_false < 3) probs[i] = hpm_expf(cost_thr * cost_thr / (-0.32f));
        probs[i] = probs[i] * priors[i];
    }
    /* TransformPDFToCDF (HPM.cu:98-112) */
    {
        float sum = 0.0f;
        for (int i = 0; i < S; ++i) sum += probs[i];
        const float inv = 1.0f / sum;
        float cum = 0.0f;
        for (int i = 0; i < S; ++i) { cum += probs[i] * inv; probs[i] = cum; }
    }
    for (int smp = 0; smp < 15; ++smp) {
        const float rp = rng_uniform(rng) - FLT_EPSILON;
        for (int id = 0; id < S; ++id)
            if (probs[id] > rp) { s->view_weights[id] += 1.0f; break; }
    }
    s->temp_selected = 0; s->num_selected = 0; s->weight_norm = 0;
    for (int i = 0; i < S; ++i)
        if (s->view_weights[i] > 0) {
            s->temp_selected |= (1u << i);
            s->weight_norm += s->view_weights[i];
            s->num_selected++;
        }
    for (int i = 0; i < 8; ++i) {
        float fc = 0.0f;
        const f4 pl = load4(st->planes, s->positions[i]);
        const float p4[4] = { pl.x, pl.y, pl.z, pl.w };
        for (int j = 0; j < S; ++j)
            if (s->view_weights[j] > 0) {
                if (geom) {
                    if (s->flag[i])
                        fc += s->view_weights[j] * (s->cost_array[i][j] + 0.2f * ora_geom_cost(depths[j + 1], c0, &cams[j + 1], p4, px, py));
                    else
                        fc += s->view_weights[j] * (s->cost_array[i][j] + 0.1f * 3.0f);
                } else fc += s->view_weights[j] * s->cost_array[i][j];
            }
        s->final_costs[i] = fc / s->weight_norm;
    }
}

static float current_cost(const float *const *images, const float *const *depths, const hpm_camera *cams,
                          int num_images, const hpm_params *prm, int px, int py, f4 pl, const float *vw,
                          float weight_norm)
{
    const int S = num_images - 1;
    const int geom = (prm->mode & HPM_MODE_GEOM) != 0;
    float cv[32];
    cost_vector(images, cams, num_images, prm, px, py, pl, cv);
    const float p4[4] = { pl.x, pl.y, pl.z, pl.w };
    float c = 0.0f;
    for (int i = 0; i < S; ++i) {
        if (geom) c += vw[i] * (cv[i] + 0.2f * ora_geom_cost(depths[i + 1], &cams[0], &cams[i + 1], p4, px, py));
        else c += vw[i] * cv[i];
    }
    return c / weight_norm;
}

/* CheckerboardPropagation (HPM.cu:1347-1873) */
static void propagate_pixel(const float *const *images, const float *const *depths, const hpm_camera *cams,
                            int num_images, const hpm_params *prm, ora_state *st, int iter, int px, int py,
                            uint64_t seed, uint32_t view_id)
{
    const hpm_camera *c0 = &cams[0];
    const int W = c0->width;
    const int center = py * W + px;
    const int prior = (prm->mode & HPM_MODE_PRIOR) != 0;
    const int hier = (prm->mode & HPM_MODE_HIERARCHY) != 0;
    if (prior) {
        if (st->confidences[center] > 0.3) return;
        if (st->plane_masks[center] == 0) return;
    }
    rng_t rng = { seed, view_id, (uint32_t)px, (uint32_t)py, &st->rng_draw[center] };
    sweep_ctx s;
    propagate_common(images, depths, cams, num_images, prm, st, iter, px, py, &rng, &s);
    const int min_idx = find_min_index(s.final_costs, 8);

    float cost_now = current_cost(images, depths, cams, num_images, prm, px, py, load4(st->planes, center),
                                  s.view_weights, s.weight_norm);
    st->costs[center] = cost_now;
    float depth_now = depth_from_plane(c0, load4(st->planes, center), px, py);
    float restricted_cost = 0.0f;
    float texture = 0.0f;
    f4 prior_pick = load4(st->planes, center);
    int has_pick = 0;
    if (prior) {
        const float depth_sigma = (prm->depth_max - prm->depth_min) / 64.0f;
        const float two_dss = 2 * depth_sigma * depth_sigma;
        const float angle_sigma = (float)(M_PI * (5.0f / 180.0f));
        const float two_ass = 2 * angle_sigma * angle_sigma;
        const f4 pp = load4(st->prior_planes, center);
        const float depth_prior = depth_from_plane(c0, pp, px, py);
        texture = ora_texture(st->canny, W, c0->height, px, py);
        if (st->plane_masks[center] > 0) {
            float rfc[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };
            for (int i = 0; i < 8; ++i)
                if (s.flag[i]) {
                    const f4 pl = load4(st->planes, s.positions[i]);
                    const float dn = depth_from_plane(c0, pl, px, py);
                    rfc[i] = prior_score(s.final_costs[i], dn, depth_prior, pp, pl, texture, two_dss, two_ass);
                }
            const int max_idx = find_max_index(rfc, 8);
            const f4 cur = load4(st->planes, center);
            const float dn = depth_from_plane(c0, cur, px, py);
            const float rnow = prior_score(cost_now, dn, depth_prior, pp, cur, texture, two_dss, two_ass);
            if (s.flag[max_idx]) {
                const f4 pl = load4(st->planes, s.positions[max_idx]);
                const float db = depth_from_plane(c0, pl, px, py);
                prior_pick = pl;
                has_pick = 1;
                if (db >= prm->depth_min && db <= prm->depth_max && rfc[max_idx] > rnow) {
                    /* no depth_now = db: HPM.cu:1815 declares a second depth_now in this
                     * block, so the assignment at HPM.cu:1825 never reaches the depth the
                     * refinement receives (the pre-acceptance depth) */
                    store4(st->planes, center, pl);
                    st->costs[center] = s.final_costs[max_idx];
                    restricted_cost = rfc[max_idx];
                    st->selected_views[center] = s.temp_selected;
                }
            }
        } else if (s.flag[min_idx]) {
            const f4 pl = load4(st->planes, s.positions[min_idx]);
            const float db = depth_from_plane(c0, pl, px, py);
            if (db >= prm->depth_min && db <= prm->depth_max && s.final_costs[min_idx] < cost_now) {
                depth_now = db;
                store4(st->planes, center, pl);
                st->costs[center] = s.final_costs[min_idx];
            }
        }
    }

    /* plane_hypotheses_now (HPM.cu:1844) is assigned only when the neighbour is
     * accepted.  The reference as compiled holds the minimum-cost neighbour's
     * plane in it whenever that direction is valid, accepted or not (its
     * half-sweep golden vectors, tests/golden/ref_init.npz).  Prior mode never
     * assigns it; there the compiled reference holds the maximum-score
     * neighbour's plane when that direction is valid.  Elsewhere (an invalid
     * direction) it starts as the pixel's current plane. */
    f4 plane_now = load4(st->planes, center);
    if (prior && has_pick) plane_now = prior_pick;
    if (!prior && s.flag[min_idx]) {
        const f4 pl = load4(st->planes, s.positions[min_idx]);
        const float db = depth_from_plane(c0, pl, px, py);
        plane_now = pl;
        if (db >= prm->depth_min && db <= prm->depth_max && s.final_costs[min_idx] < cost_now) {
            depth_now = db; plane_now = pl; cost_now = s.final_costs[min_idx];
            st->selected_views[center] = s.temp_selected;
        }
        if (st->costs[center] != st->costs[center]) {
            depth_now = db; plane_now = pl; cost_now = s.final_costs[min_idx];
            st->selected_views[center] = s.temp_selected;
        }
    }
    refinement(images, depths, cams, num_images, prm, st, &plane_now, &depth_now, &cost_now, &rng,
               s.view_weights, s.weight_norm, &restricted_cost, px, py, texture);
    if (hier) {
        if (cost_now < st->pre_costs[center] - 0.1f) {
            st->costs[center] = cost_now;
            store4(st->planes, center, plane_now);
        }
    } else {
        st->costs[center] = cost_now;
        store4(st->planes, center, plane_now);
    }
}

/* CheckerboardPropagation_MandatoryConsistency (HPM.cu:1875-2791) */
static void propagate_pixel_mand(const float *const *images, const float *const *depths, const hpm_camera *cams,
                                 int num_images, const hpm_params *prm, ora_state *st, int iter, int px, int py,
                                 uint64_t seed, uint32_t view_id)
{
    const hpm_camera *c0 = &cams[0];
    const int W = c0->width;
    const int center = py * W + px;
    rng_t rng = { seed, view_id, (uint32_t)px, (uint32_t)py, &st->rng_draw[center] };
    sweep_ctx s;
    const int reliable = st->confidences[center] >= 0.3;
    propagate_common(images, depths, cams, num_images, prm, st, iter, px, py, &rng, &s);

    if (reliable) {
        const int min_idx = find_min_index(s.final_costs, 8);
        float cost_now = current_cost(images, depths, cams, num_images, prm, px, py, load4(st->planes, center),
                                      s.view_weights, s.weight_norm);
        st->costs[center] = cost_now;
        float depth_now = depth_from_plane(c0, load4(st->planes, center), px, py);
        f4 plane_now = load4(st->planes, center); /* HPM.cu:2299: read as at HPM.cu:1844 */
        if (s.flag[min_idx]) {
            const f4 pl = load4(st->planes, s.positions[min_idx]);
            const float db = depth_from_plane(c0, pl, px, py);
            plane_now = pl;
            if (db >= prm->depth_min && db <= prm->depth_max && s.final_costs[min_idx] < cost_now) {
                depth_now = db; plane_now = pl; cost_now = s.final_costs[min_idx];
                st->selected_views[center] = s.temp_selected;
            }
            if (st->costs[center] != st->costs[center]) {
                plane_now = pl; cost_now = s.final_costs[min_idx];
                st->selected_views[center] = s.temp_selected;
            }
        }
        refinement(images, depths, cams, num_images, prm, st, &plane_now, &depth_now, &cost_now, &rng,
                   s.view_weights, s.weight_norm, NULL, px, py, 0.0f);
        st->costs[center] = cost_now;
        store4(st->planes, center, plane_now);
        return;
    }

    const float beta = 0.18f;
    float rfc[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };
    const float mmc = s.num_selected * 0.5f;
    for (int i = 0; i < 8; ++i) {
        if (s.flag[i]) {
            const float cp = st->confidences[s.positions[i]];
            const float gce = hpm_expf(-s.final_costs[i] * s.final_costs[i] / beta);
            const float dm = (0.0f > mmc - cp) ? 0.0f : (mmc - cp);
            const float mce = (float)(0.5f + exp(-dm * dm / (mmc * mmc * 1.0)));
            if (cp > 0) rfc[i] = (3.0f > mce ? 3.0f : mce) * gce;
            else rfc[i] = mce * gce;
            if (cp > 0) {
                const double e = (double)hpm_expf(-cp * 2);
                s.final_costs[i] = (float)(s.final_costs[i] * (e < 0.35 ? e : 0.35));
            }
        }
    }
    const int max_idx = find_max_index(rfc, 8);
    float cost_now = current_cost(images, depths, cams, num_images, prm, px, py, load4(st->planes, center),
                                  s.view_weights, s.weight_norm);
    st->costs[center] = cost_now;
    const float cc = st->confidences[center];
    const float gce = hpm_expf(-cost_now * cost_now / beta);
    const float dm = (0.0f > mmc - cc) ? 0.0f : (mmc - cc);
    const float mce = (float)(0.5f + exp(-dm * dm / (mmc * mmc * 1.0)));
    float rnow;
    if (cc > 0) rnow = (3.0f > mce ? 3.0f : mce) * gce;
    else rnow = mce * gce;
    if (cc < 0.3) cost_now = (float)(cost_now * exp(0.2 + cc * 2));
    else cost_now = cost_now * hpm_expf(-cc * 2);

    /* HPM.cu:2761: the maximum-score neighbour's plane whenever that direction
     * is valid, as at HPM.cu:1844; the pixel's current plane otherwise */
    f4 plane_now = load4(st->planes, center);
    if (s.flag[max_idx]) {
        const int pm = s.positions[max_idx];
        const f4 pl = load4(st->planes, pm);
        plane_now = pl;
        const float db = depth_from_plane(c0, pl, px, py);
        if (db >= prm->depth_min && db <= prm->depth_max && rfc[max_idx] > rnow) {
            plane_now = pl; cost_now = s.final_costs[max_idx];
            st->selected_views[center] = s.temp_selected;
            st->confidences[center] = (float)(0.5 * st->confidences[pm]);
        }
        if (st->costs[center] != st->costs[center]) {
            plane_now = pl; cost_now = s.final_costs[max_idx];
            st->selected_views[center] = s.temp_selected;
            st->confidences[center] = (float)(0.5 * st->confidences[pm]);
        }
    }
    st->costs[center] = cost_now;
    store4(st->planes, center, plane_now);
}

/* Rows covered by the checkerboard grid of RunPatchMatch (HPM.cu:3004-3011):
 * blocks of 16 row pairs over floor(H/2) pairs. */
static int covered_row_pairs(int H)
{
    const int pairs = H / 2;
    return ((pairs + 15) / 16) * 16;
}

void ora_half_sweep(const float *const *images, const float *const *depths, const hpm_camera *cams,
                    int num_images, const hpm_params *params, ora_state *st, int color, int iter,
                    uint64_t seed, uint32_t view_id)
{
    const int W = cams[0].width, H = cams[0].height;
    const int cover = covered_row_pairs(H);
    const int mand = (params->mode & HPM_MODE_MAND) != 0;
#pragma omp parallel for schedule(dynamic, 2)
    for (int y = 0; y < H; ++y) {
        if (y / 2 >= cover) continue;
        for (int x = 0; x < W; ++x) {
            if (((x + y) & 1) != color) continue;
            if (mand) propagate_pixel_mand(images, depths, cams, num_images, params, st, iter, x, y, seed, view_id);
            else propagate_pixel(images, depths, cams, num_images, params, st, iter, x, y, seed, view_id);
        }
    }
}

void ora_export(const hpm_camera *c, float *planes)
{
    const int W = c->width, H = c->height;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const int k = y * W + x;
            f4 pl = load4(planes, k);
            pl.w = depth_from_plane(c, pl, x, y);
            pl = rotate_to_world(c, pl);
            store4(planes, k, pl);
        }
}

void ora_run_patchmatch(const float *const *images, const float *const *depths, const hpm_camera *cams,
                        int num_images, const hpm_params *params, ora_state *st, uint64_t seed, uint32_t view_id)
{
    ora_random_init(images, cams, num_images, params, st, seed, view_id);
    for (int i = 0; i < params->max_iterations; ++i) {
        ora_half_sweep(images, depths, cams, num_images, params, st, 0, i, seed, view_id);
        ora_half_sweep(images, depths, cams, num_images, params, st, 1, i, seed, view_id);
    }
    ora_export(&cams[0], st->planes);
}

/* ---------------- JBU (HPM.cu:3037-3197, HPM.cpp:1266-1392) ---------------- */

static void jbu_pixel(const float *image, int W, int H, const float *sdepth, const float *snormal,
                      int sw, int sh, int px, int py, float *od, float *on)
{
    const float scale = (float)(1.0 * sw / W);
    const float sigmad = 0.50f, sigmar = 25.5f;
    const int a = H / sh, b = W / sw;
    const int image_scale = a > b ? a : b;
    const int win = image_scale * image_scale + 1;
    const int nn = win / 2;
    const float o_y = py * scale, o_x = px * scale;
    const float ref_pix = texel(image, W, H, px, py);
    float nf = 0.0f, val = 0.0f;
    float n0 = 0.0f, n1 = 0.0f, n2 = 0.0f;
    for (int j = -nn; j <= nn; ++j) {
        int r_y = f2i_rz(o_y + j);
        r_y = (r_y > 0 ? (r_y < sh ? r_y : sh - 1) : 0);
        int r_ys = py + j;
        if (!snormal) r_ys = (r_ys > 0 ? (r_ys < H ? r_ys : H - 1) : 0);
        for (int i = -nn; i <= nn; ++i) {
            int r_x = f2i_rz(o_x + i);
            r_x = (r_x > 0 ? (r_x < sw ? r_x : sw - 1) : 0);
            const float sp = sdepth[r_y * sw + r_x];
            int r_xs = px + i;
            if (!snormal) r_xs = (r_xs > 0 ? (r_xs < W ? r_xs : W - 1) : 0);
            const float nb = texel(image, W, H, r_xs, r_ys);
            const float sg = spatial_gauss(o_x, o_y, (float)r_x, (float)r_y, sigmad);
            const float rg = range_gauss(fabsf(ref_pix - nb), sigmar);
            const float tg = sg * rg;
            nf += tg;
            val += sp * tg;
            if (snormal) {
                const float *sn = snormal + 3 * (size_t)(r_y * sw + r_x);
                n0 = n0 + sn[0] * tg; n1 = n1 + sn[1] * tg; n2 = n2 + sn[2] * tg;
            }
        }
    }
    *od = val / nf;
    if (snormal) {
        f4 n = { n0 / nf, n1 / nf, n2 / nf, 0.0f };
        normalize3(&n);
        on[0] = n.x; on[1] = n.y; on[2] = n.z;
    }
}

void ora_jbu(const float *image, int W, int H, const float *sdepth, int sw, int sh, float *out)
{
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            float d;
            jbu_pixel(image, W, H, sdepth, NULL, sw, sh, x, y, &d, NULL);
            if (d != d) {
                /* RunJBU falls back to src_depthmap(j/2, i/2) (HPM.cpp:1297-1300); clamp keeps
                 * the read inside the coarse map when the scale exceeds 2 */
                d = sdepth[clampi(y / 2, 0, sh - 1) * sw + clampi(x / 2, 0, sw - 1)];
            }
            out[y * W + x] = d;
        }
}

void ora_jbu_prior(const float *image, int W, int H, const float *sdepth, const float *snormal,
                   int sw, int sh, float *od, float *on)
{
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            /* the NaN fallback of HPM.cpp:1362-1368 is overwritten by 1369-1372 */
            jbu_pixel(image, W, H, sdepth, snormal, sw, sh, x, y, &od[y * W + x], &on[3 * (size_t)(y * W + x)]);
        }
}

/* Philox4x32-10 of include/hpm_philox.h, exported for the known-answer tests. */
void ora_philox(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4])
{
    hpm_u32x4 c;
    for (int i = 0; i < 4; ++i) c.v[i] = ctr[i];
    const hpm_u32x4 r = hpm_philox4x32_10(c, k0, k1);
    for (int i = 0; i < 4; ++i) out[i] = r.v[i];
}

float ora_uniform(uint64_t seed, uint32_t view, uint32_t x, uint32_t y, uint32_t draw)
{
    return hpm_bits_to_uniform(hpm_rng_bits(seed, view, x, y, draw));
}
