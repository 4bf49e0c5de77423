/*
 * Plane-induced homography of the bilateral NCC (ComputeHomography, HPM.cu:251-311),
 * factored so that its per-view and per-hypothesis parts are computed once.
 *
 * The reference forms, for every (pixel, hypothesis, source view),
 *     H = Ks' (R_rel - t_rel n^T / d) Kr^-1
 * with Ks' = [[fx_s, 0, cx_s], [0, fy_s, cy_s], [0, 0, K8_s]] and
 * Kr^-1 = [[1/fx_r, 0, -cx_r/fx_r], [0, 1/fy_r, -cy_r/fy_r], [0, 0, 1]]
 * written out element by element (HPM.cu:281-310, the skew entries of K are
 * not used).  The same matrix is
 *     H = A - b m^T,   A = Ks' R_rel Kr^-1,  b = Ks' t_rel  (per source view)
 *                      m = Kr^-T n / d                      (per hypothesis)
 * so the work per (hypothesis, view) is nine multiply-adds and the per-view
 * basis is formed once on the host in double precision and rounded to float.
 * The CUDA path and the CPU oracle both evaluate it with these functions, so
 * they agree bit for bit; against the reference's float expression the
 * difference is rounding only.
 */
#ifndef HPM_GEOMETRY_H
#define HPM_GEOMETRY_H

#include "hpm_fp.h"
#include "hpm_types.h"

/* Per-view basis (A, b) of source `sc` relative to reference `rc`; host only. */
static inline void hpm_view_basis(const hpm_camera *rc, const hpm_camera *sc, float A[9], float b[3])
{
    double rC[3], sC[3], Rrel[9], tr[3], M[9];
    for (int k = 0; k < 3; ++k) {
        rC[k] = -((double)rc->R[0 + k] * rc->t[0] + (double)rc->R[3 + k] * rc->t[1] + (double)rc->R[6 + k] * rc->t[2]);
        sC[k] = -((double)sc->R[0 + k] * sc->t[0] + (double)sc->R[3 + k] * sc->t[1] + (double)sc->R[6 + k] * sc->t[2]);
    }
    for (int r = 0; r < 3; ++r) {
        for (int k = 0; k < 3; ++k)
            Rrel[3 * r + k] = (double)sc->R[3 * r + 0] * rc->R[3 * k + 0] + (double)sc->R[3 * r + 1] * rc->R[3 * k + 1] +
                              (double)sc->R[3 * r + 2] * rc->R[3 * k + 2];
        tr[r] = (double)sc->R[3 * r + 0] * (rC[0] - sC[0]) + (double)sc->R[3 * r + 1] * (rC[1] - sC[1]) +
                (double)sc->R[3 * r + 2] * (rC[2] - sC[2]);
    }
    const double fx = rc->K[0], fy = rc->K[4], cx = rc->K[2], cy = rc->K[5];
    for (int r = 0; r < 3; ++r) { /* M = R_rel Kr^-1 */
        M[3 * r + 0] = Rrel[3 * r + 0] / fx;
        M[3 * r + 1] = Rrel[3 * r + 1] / fy;
        M[3 * r + 2] = -Rrel[3 * r + 0] * cx / fx - Rrel[3 * r + 1] * cy / fy + Rrel[3 * r + 2];
    }
    for (int k = 0; k < 3; ++k) { /* A = Ks' M */
        A[0 + k] = (float)((double)sc->K[0] * M[0 + k] + (double)sc->K[2] * M[6 + k]);
        A[3 + k] = (float)((double)sc->K[4] * M[3 + k] + (double)sc->K[5] * M[6 + k]);
        A[6 + k] = (float)((double)sc->K[8] * M[6 + k]);
    }
    b[0] = (float)((double)sc->K[0] * tr[0] + (double)sc->K[2] * tr[2]);
    b[1] = (float)((double)sc->K[4] * tr[1] + (double)sc->K[5] * tr[2]);
    b[2] = (float)((double)sc->K[8] * tr[2]);
}

/* Point transfer of the geometric consistency cost (ComputeGeomConsistencyCost,
 * HPM.cu:539-564, through Get3DPointonWorld_cu and ProjectonCamera_cu,
 * HPM.cu:501-537): pixel u = (x, y, 1) of camera `from` at depth d lands at
 *     q = G u d + g,   pixel = (q_x / q_z, q_y / q_z)
 * in camera `to`, with G = K_to R_rel Kinv_from and g = K_to t_rel.  As in the
 * reference, the back-projection uses (x - cx) / fx, (y - cy) / fy (no skew)
 * and the projection all nine entries of K_to.  Host only; double, rounded. */
static inline void hpm_view_transfer(const hpm_camera *from, const hpm_camera *to, float G[9], float g[3])
{
    double fC[3], tC[3], Rrel[9], tr[3], M[9];
    for (int k = 0; k < 3; ++k) {
        fC[k] = -((double)from->R[0 + k] * from->t[0] + (double)from->R[3 + k] * from->t[1] +
                  (double)from->R[6 + k] * from->t[2]);
        tC[k] = -((double)to->R[0 + k] * to->t[0] + (double)to->R[3 + k] * to->t[1] + (double)to->R[6 + k] * to->t[2]);
    }
    for (int r = 0; r < 3; ++r) {
        for (int k = 0; k < 3; ++k)
            Rrel[3 * r + k] = (double)to->R[3 * r + 0] * from->R[3 * k + 0] +
                              (double)to->R[3 * r + 1] * from->R[3 * k + 1] +
                              (double)to->R[3 * r + 2] * from->R[3 * k + 2];
        tr[r] = (double)to->R[3 * r + 0] * (fC[0] - tC[0]) + (double)to->R[3 * r + 1] * (fC[1] - tC[1]) +
                (double)to->R[3 * r + 2] * (fC[2] - tC[2]);
    }
    const double fx = from->K[0], fy = from->K[4], cx = from->K[2], cy = from->K[5];
    for (int r = 0; r < 3; ++r) { /* M = R_rel Kinv_from */
        M[3 * r + 0] = Rrel[3 * r + 0] / fx;
        M[3 * r + 1] = Rrel[3 * r + 1] / fy;
        M[3 * r + 2] = -Rrel[3 * r + 0] * cx / fx - Rrel[3 * r + 1] * cy / fy + Rrel[3 * r + 2];
    }
    for (int r = 0; r < 3; ++r) {
        for (int k = 0; k < 3; ++k)
            G[3 * r + k] = (float)((double)to->K[3 * r + 0] * M[k] + (double)to->K[3 * r + 1] * M[3 + k] +
                                   (double)to->K[3 * r + 2] * M[6 + k]);
        g[r] = (float)((double)to->K[3 * r + 0] * tr[0] + (double)to->K[3 * r + 1] * tr[1] +
                       (double)to->K[3 * r + 2] * tr[2]);
    }
}

/* Transfer of pixel (x, y) at depth d with (G, g) of hpm_view_transfer. */
HPM_FP_HD void hpm_transfer(const float G[9], const float g[3], float x, float y, float d, float *ox, float *oy)
{
    const float ax = hpm_fma(G[0], x, hpm_fma(G[1], y, G[2]));
    const float ay = hpm_fma(G[3], x, hpm_fma(G[4], y, G[5]));
    const float az = hpm_fma(G[6], x, hpm_fma(G[7], y, G[8]));
    const float qz = hpm_fma(az, d, g[2]);
    *ox = hpm_fma(ax, d, g[0]) / qz;
    *oy = hpm_fma(ay, d, g[1]) / qz;
}

/* Entries of Kr^-1 the hypothesis term needs: 1/fx, 1/fy, cx/fx, cy/fy; host only. */
static inline void hpm_ref_kinv(const hpm_camera *rc, float kinv[4])
{
    kinv[0] = (float)(1.0 / rc->K[0]);
    kinv[1] = (float)(1.0 / rc->K[4]);
    kinv[2] = (float)((double)rc->K[2] / rc->K[0]);
    kinv[3] = (float)((double)rc->K[5] / rc->K[4]);
}

/* m = Kr^-T n / d of the hypothesis (n, d) (camera frame, d = plane offset). */
HPM_FP_HD void hpm_plane_m(const float kinv[4], float nx, float ny, float nz, float d, float m[3])
{
    const float id = 1.0f / d;
    m[0] = (nx * kinv[0]) * id;
    m[1] = (ny * kinv[1]) * id;
    float t = hpm_fma(-nx, kinv[2], nz);
    t = hpm_fma(-ny, kinv[3], t);
    m[2] = t * id;
}

/* H = A - b m^T. */
HPM_FP_HD void hpm_homography(const float A[9], const float b[3], const float m[3], float H[9])
{
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) H[3 * r + k] = hpm_fma(-b[r], m[k], A[3 * r + k]);
}

#endif /* HPM_GEOMETRY_H */
