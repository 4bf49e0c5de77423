/*
 * CPU ORACLE -- test infrastructure only (see hpm_oracle.h).
 *
 * FP64 restatement of the differentiable form of the bilateral NCC
 * (ComputeBilateralNCC, HPM.cu:375-448, with the homography of HPM.cu:251-311)
 * and its gradient with respect to the pixel's plane parameters
 * theta = (depth, nx, ny), camera frame, nz = -sqrt(1 - nx^2 - ny^2).
 *
 * The differentiable form samples the source image with exact bilinear
 * interpolation (texel centres at integers, replicated border) where the
 * reference uses the texture unit's 8-bit weights; everything else is the
 * reference's cost: 36 samples of an 11x11 window at stride 2, bilateral
 * weights exp(-|d|/(2 sigma_s^2) - |I - I_c|/(2 sigma_c^2)), cost
 * 1 - cov / sqrt(var_r var_s) clamped to [0, 2], and 2 (zero gradient) for an
 * out-of-image centre or a variance below 1e-5.
 */
#include "hpm_oracle.h"

#include <math.h>
#include <string.h>

static double texel64(const float *img, int w, int h, int x, int y)
{
    x = x < 0 ? 0 : (x >= w ? w - 1 : x);
    y = y < 0 ? 0 : (y >= h ? h - 1 : y);
    return img[(size_t)y * w + x];
}

/* exact bilinear sample at (X, Y) and its partial derivatives; the position is
   clamped to [-2, size + 1] first (NaN to -2), where every tap already reads the
   edge texel, so the integer conversion below stays in range */
static double bilinear64(const float *img, int w, int h, double X, double Y, double *dX, double *dY)
{
    X = X >= -2.0 ? (X <= w + 1.0 ? X : w + 1.0) : -2.0;
    Y = Y >= -2.0 ? (Y <= h + 1.0 ? Y : h + 1.0) : -2.0;
    const double fx = floor(X), fy = floor(Y);
    const int x0 = (int)fx, y0 = (int)fy;
    const double ax = X - fx, ay = Y - fy;
    const double i00 = texel64(img, w, h, x0, y0), i10 = texel64(img, w, h, x0 + 1, y0);
    const double i01 = texel64(img, w, h, x0, y0 + 1), i11 = texel64(img, w, h, x0 + 1, y0 + 1);
    *dX = (1 - ay) * (i10 - i00) + ay * (i11 - i01);
    *dY = (1 - ax) * (i01 - i00) + ax * (i11 - i10);
    return (1 - ay) * ((1 - ax) * i00 + ax * i10) + ay * ((1 - ax) * i01 + ax * i11);
}

static void basis64(const hpm_camera *rc, const hpm_camera *sc, double A[9], double b[3])
{
    double rC[3], sC[3], Rrel[9], tr[3], M[9];
    for (int k = 0; k < 3; ++k) {
        rC[k] = -((double)rc->R[0 + k] * rc->t[0] + (double)rc->R[3 + k] * rc->t[1] + (double)rc->R[6 + k] * rc->t[2]);
        sC[k] = -((double)sc->R[0 + k] * sc->t[0] + (double)sc->R[3 + k] * sc->t[1] + (double)sc->R[6 + k] * sc->t[2]);
    }
    for (int r = 0; r < 3; ++r) {
        for (int k = 0; k < 3; ++k)
            Rrel[3 * r + k] = (double)sc->R[3 * r] * rc->R[3 * k] + (double)sc->R[3 * r + 1] * rc->R[3 * k + 1] +
                              (double)sc->R[3 * r + 2] * rc->R[3 * k + 2];
        tr[r] = (double)sc->R[3 * r] * (rC[0] - sC[0]) + (double)sc->R[3 * r + 1] * (rC[1] - sC[1]) +
                (double)sc->R[3 * r + 2] * (rC[2] - sC[2]);
    }
    const double fx = rc->K[0], fy = rc->K[4], cx = rc->K[2], cy = rc->K[5];
    for (int r = 0; r < 3; ++r) {
        M[3 * r + 0] = Rrel[3 * r + 0] / fx;
        M[3 * r + 1] = Rrel[3 * r + 1] / fy;
        M[3 * r + 2] = -Rrel[3 * r + 0] * cx / fx - Rrel[3 * r + 1] * cy / fy + Rrel[3 * r + 2];
    }
    for (int k = 0; k < 3; ++k) {
        A[0 + k] = (double)sc->K[0] * M[0 + k] + (double)sc->K[2] * M[6 + k];
        A[3 + k] = (double)sc->K[4] * M[3 + k] + (double)sc->K[5] * M[6 + k];
        A[6 + k] = (double)sc->K[8] * M[6 + k];
    }
    b[0] = (double)sc->K[0] * tr[0] + (double)sc->K[2] * tr[2];
    b[1] = (double)sc->K[4] * tr[1] + (double)sc->K[5] * tr[2];
    b[2] = (double)sc->K[8] * tr[2];
}

double ora_cost_grad64(const float *ref, const hpm_camera *rc, const float *src, const hpm_camera *sc,
                       const hpm_params *prm, int px, int py, const double theta[3], double grad[3])
{
    const int rw = rc->width, rh = rc->height, sw = sc->width, sh = sc->height;
    if (grad) grad[0] = grad[1] = grad[2] = 0.0;
    /* reference patch and bilateral weights (view independent) */
    const double center = texel64(ref, rw, rh, px, py);
    const double two_ss = 2.0 * prm->sigma_spatial * prm->sigma_spatial;
    const double two_sc = 2.0 * prm->sigma_color * prm->sigma_color;
    double wk[36], rk[36], W = 0, Sr = 0, Srr = 0;
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            const int dx = -5 + 2 * i, dy = -5 + 2 * j, k = i * 6 + j;
            rk[k] = texel64(ref, rw, rh, px + dx, py + dy);
            wk[k] = exp(-sqrt((double)(dx * dx + dy * dy)) / two_ss - fabs(rk[k] - center) / two_sc);
            W += wk[k]; Sr += wk[k] * rk[k]; Srr += wk[k] * rk[k] * rk[k];
        }
    const double mean_r = Sr / W, var_r = Srr / W - mean_r * mean_r;
    if (var_r < 1e-5) return 2.0;
    /* plane from theta */
    const double nx = theta[1], ny = theta[2];
    const double nn = 1.0 - nx * nx - ny * ny;
    if (nn <= 0.0) return 2.0;
    const double nz = -sqrt(nn);
    const double fx = rc->K[0], fy = rc->K[4], cx = rc->K[2], cy = rc->K[5];
    const double ray[3] = { (px - cx) / fx, (py - cy) / fy, 1.0 };
    const double nr = nx * ray[0] + ny * ray[1] + nz * ray[2];
    const double w = -theta[0] * nr;
    const double t[3] = { nx / fx, ny / fy, nz - nx * cx / fx - ny * cy / fy };
    const double m[3] = { t[0] / w, t[1] / w, t[2] / w };
    double A[9], b[3], H[9];
    basis64(rc, sc, A, b);
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) H[3 * r + k] = A[3 * r + k] - b[r] * m[k];
    {
        const double qx = H[0] * px + H[1] * py + H[2], qy = H[3] * px + H[4] * py + H[5];
        const double qz = H[6] * px + H[7] * py + H[8];
        const double X = qx / qz, Y = qy / qz;
        if (X >= sw || X < 0.0 || Y >= sh || Y < 0.0) return 2.0;
    }
    double v[36], gX[36], gY[36], Xs[36], Ys[36], qzs[36];
    double Ss = 0, Sss = 0, Srs = 0;
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            const int k = i * 6 + j;
            const double ux = px - 5 + 2 * i, uy = py - 5 + 2 * j;
            const double qx = H[0] * ux + H[1] * uy + H[2], qy = H[3] * ux + H[4] * uy + H[5];
            const double qz = H[6] * ux + H[7] * uy + H[8];
            Xs[k] = qx / qz; Ys[k] = qy / qz; qzs[k] = qz;
            v[k] = bilinear64(src, sw, sh, Xs[k], Ys[k], &gX[k], &gY[k]);
            Ss += wk[k] * v[k]; Sss += wk[k] * v[k] * v[k]; Srs += wk[k] * rk[k] * v[k];
        }
    Ss /= W; Sss /= W; Srs /= W;
    const double var_s = Sss - Ss * Ss;
    if (var_s < 1e-5) return 2.0;
    const double cov = Srs - mean_r * Ss;
    const double sig = sqrt(var_r * var_s);
    const double c = 1.0 - cov / sig;
    if (c < 0.0) return 0.0;
    if (c > 2.0) return 2.0;
    if (!grad) return c;
    /* dc/dm */
    double dm[3] = { 0, 0, 0 };
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            const int k = i * 6 + j;
            const double dcdv = wk[k] / W * (-(rk[k] - mean_r) / sig + cov * (v[k] - Ss) / (sig * var_s));
            const double g0 = gX[k] / qzs[k], g1 = gY[k] / qzs[k], g2 = -(gX[k] * Xs[k] + gY[k] * Ys[k]) / qzs[k];
            const double gb = g0 * b[0] + g1 * b[1] + g2 * b[2];
            const double u[3] = { (double)(px - 5 + 2 * i), (double)(py - 5 + 2 * j), 1.0 };
            for (int a = 0; a < 3; ++a) dm[a] += dcdv * (-gb) * u[a];
        }
    /* m = t / w: explicit normal part and the offset */
    const double dw = -(dm[0] * m[0] + dm[1] * m[1] + dm[2] * m[2]) / w;
    double dn[3] = { (dm[0] / fx - dm[2] * cx / fx) / w, (dm[1] / fy - dm[2] * cy / fy) / w, dm[2] / w };
    /* w = -depth (n . ray) */
    for (int a = 0; a < 3; ++a) dn[a] += dw * (-theta[0] * ray[a]);
    grad[0] = dw * (-nr);
    /* nz(nx, ny) */
    grad[1] = dn[0] + dn[2] * (-nx / nz);
    grad[2] = dn[1] + dn[2] * (-ny / nz);
    return c;
}
