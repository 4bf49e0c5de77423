/*
 * CPU ORACLE -- test infrastructure only (see hpm_oracle.h).
 *
 * Host stages of HPM-MVS++ restated in C: ConfidenceEvaluation and RunFusion
 * (main.cpp:659-1109), support points (HPM.cpp:1026-1073), the triangle raster
 * and planar-prior fit (main.cpp:384-597, HPM.cpp:1099-1206), and OpenCV's
 * INTER_LINEAR resize of float maps used by the prior downsampling
 * (main.cpp:452-454).
 *
 * These loops run on the host in the reference (compiled by g++ without
 * -ffast-math).  In those translation units the CUDA headers bring <math.h>'s
 * overloads into the global namespace, so `exp(float)`, `fabs(float)` and
 * `sqrt(float)` are the float functions while `pow(float, int)` promotes to
 * double (checked by compiling main.cpp's includes, oracle/ref_host.mk).  The
 * restatement rounds where the reference rounds: the float exp is the double
 * exp rounded to float.
 */
#include "hpm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { float x, y, z; } f3;
typedef struct { float x, y; } f2;

static f3 world_point(int x, int y, float depth, const hpm_camera *c) /* HPM.cpp:221-245 */
{
    f3 X, T, C, R;
    X.x = depth * (x - c->K[2]) / c->K[0];
    X.y = depth * (y - c->K[5]) / c->K[4];
    X.z = depth;
    T.x = c->R[0] * X.x + c->R[3] * X.y + c->R[6] * X.z;
    T.y = c->R[1] * X.x + c->R[4] * X.y + c->R[7] * X.z;
    T.z = c->R[2] * X.x + c->R[5] * X.y + c->R[8] * X.z;
    C.x = -(c->R[0] * c->t[0] + c->R[3] * c->t[1] + c->R[6] * c->t[2]);
    C.y = -(c->R[1] * c->t[0] + c->R[4] * c->t[1] + c->R[7] * c->t[2]);
    C.z = -(c->R[2] * c->t[0] + c->R[5] * c->t[1] + c->R[8] * c->t[2]);
    R.x = T.x + C.x; R.y = T.y + C.y; R.z = T.z + C.z;
    return R;
}

static void project_cam(f3 X, const hpm_camera *c, f2 *pt, float *depth) /* HPM.cpp:269-279 */
{
    f3 T;
    T.x = c->R[0] * X.x + c->R[1] * X.y + c->R[2] * X.z + c->t[0];
    T.y = c->R[3] * X.x + c->R[4] * X.y + c->R[5] * X.z + c->t[1];
    T.z = c->R[6] * X.x + c->R[7] * X.y + c->R[8] * X.z + c->t[2];
    *depth = c->K[6] * T.x + c->K[7] * T.y + c->K[8] * T.z;
    pt->x = (c->K[0] * T.x + c->K[1] * T.y + c->K[2] * T.z) / *depth;
    pt->y = (c->K[3] * T.x + c->K[4] * T.y + c->K[5] * T.z) / *depth;
}

static float angle_between(const float *a, const float *b) /* HPM.cpp:281-290 */
{
    /* acosf evaluated as the double acos rounded once (include/hpm_fp.h), so CPU
     * and GPU agree bit for bit; it differs from a libm acosf by at most 1 ulp */
    const float dot = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    const float ang = (float)acos((double)dot);
    if (ang != ang) return 0.0f;
    return ang;
}

static int f2i_trunc(float v) /* int(point.y + 0.5f): truncation toward zero */
{
    if (v != v) return -2147483647 - 1; /* x86 cvttss2si gives INT_MIN for NaN */
    if (v >= 2147483647.0f || v <= -2147483648.0f) return -2147483647 - 1;
    return (int)v;
}

/* Shared scan of ConfidenceEvaluation / RunFusion.  kind 0 = confidence
 * (depth-range checks, writes conf maps), 1 = fusion (emits points). */
static int64_t consistency_scan(int kind, int num_views, const hpm_camera *cams, const float *const *depths,
                                const float *const *normals, const uint8_t *const *colors,
                                const uint8_t *const *sky, const int32_t *src_off, const int32_t *src_ids,
                                float *const *conf_out, hpm_point *out, int64_t max_points, int64_t *n_total)
{
    uint8_t **masks = (uint8_t **)calloc((size_t)num_views, sizeof(uint8_t *));
    float **cons = NULL;
    for (int i = 0; i < num_views; ++i)
        masks[i] = (uint8_t *)calloc((size_t)cams[i].width * cams[i].height, 1);
    if (kind == 0) {
        cons = (float **)calloc((size_t)num_views, sizeof(float *));
        for (int i = 0; i < num_views; ++i)
            cons[i] = (float *)calloc((size_t)cams[i].width * cams[i].height, sizeof(float));
    }
    int64_t count = 0;
    for (int i = 0; i < num_views; ++i) {
        const hpm_camera *ci = &cams[i];
        const int cols = ci->width, rows = ci->height;
        const int n_ngb = src_off[i + 1] - src_off[i];
        const int32_t *ngb = src_ids + src_off[i];
        int used_x[HPM_MAX_VIEWS], used_y[HPM_MAX_VIEWS];
        /* used_list lives for the whole view scan, not per pixel (main.cpp:737, 883, 1018) */
        for (int j = 0; j < n_ngb; ++j) { used_x[j] = -1; used_y[j] = -1; }
        for (int r = 0; r < rows; ++r) {
            for (int c = 0; c < cols; ++c) {
                if (masks[i][r * cols + c] == 1) continue;
                const float ref_depth = depths[i][r * cols + c];
                const float *ref_normal = normals[i] + 3 * (size_t)(r * cols + c);
                if (ref_depth <= 0.0) continue;
                if (kind == 0 && (ref_depth < ci->depth_min || ref_depth > ci->depth_max)) continue;
                const f3 X = world_point(c, r, ref_depth, ci);
                int n_cons = 0;
                float dyn = 0.0f;
                for (int j = 0; j < n_ngb; ++j) {
                    const int sid = ngb[j];
                    const hpm_camera *cs = &cams[sid];
                    const int scols = cs->width, srows = cs->height;
                    f2 pt; float pd;
                    project_cam(X, cs, &pt, &pd);
                    const int sr = f2i_trunc(pt.y + 0.5f);
                    const int sc = f2i_trunc(pt.x + 0.5f);
                    if (sc >= 0 && sc < scols && sr >= 0 && sr < srows) {
                        if (masks[sid][sr * scols + sc] == 1) continue;
                        const float sdepth = depths[sid][sr * scols + sc];
                        const float *snormal = normals[sid] + 3 * (size_t)(sr * scols + sc);
                        if (sdepth <= 0.0) continue;
                        if (kind == 0 && (sdepth < ci->depth_min || sdepth > ci->depth_max)) continue;
                        const f3 tX = world_point(sc, sr, sdepth, cs);
                        f2 tp;
                        project_cam(tX, ci, &tp, &pd);
                        const float dx = c - tp.x, dy = r - tp.y;
                        const float reproj = (float)sqrt(pow((double)dx, 2) + pow((double)dy, 2));
                        const float rel = (float)(fabs((double)(pd - ref_depth)) / ref_depth);
                        const float ang = angle_between(ref_normal, snormal);
                        if (reproj < 2.0f && rel < 0.01f && ang < 0.174533f) {
                            used_x[j] = sc; used_y[j] = sr;
                            const float idx = reproj + 200 * rel + ang * 10;
                            dyn = dyn + (float)exp((double)(-idx)); /* float exp, float sum */
                            n_cons++;
                        }
                    }
                }
                if (n_cons >= 1 && (dyn > 0.3 * n_cons)) {
                    if (kind == 0) {
                        cons[i][r * cols + c] = dyn;
                    } else {
                        const uint8_t *col = colors[i] + 3 * (size_t)(r * cols + c);
                        int keep = 1;
                        if (sky) {
                            const uint8_t *sm = sky[i] + 3 * (size_t)(r * cols + c);
                            keep = (sm[0] != 234 && sm[1] != 235 && sm[2] != 55);
                        }
                        if (keep) {
                            if (count < max_points && out) {
                                hpm_point *p = &out[count];
                                p->coord[0] = X.x; p->coord[1] = X.y; p->coord[2] = X.z;
                                p->normal[0] = ref_normal[0]; p->normal[1] = ref_normal[1]; p->normal[2] = ref_normal[2];
                                p->color[0] = (float)col[0]; p->color[1] = (float)col[1]; p->color[2] = (float)col[2];
                            }
                            count++;
                        }
                    }
                    for (int j = 0; j < n_ngb; ++j) {
                        if (used_x[j] == -1) continue;
                        const int sid = ngb[j];
                        masks[sid][used_y[j] * cams[sid].width + used_x[j]] = 1;
                        if (kind == 0) cons[sid][used_y[j] * cams[sid].width + used_x[j]] = dyn;
                    }
                }
            }
        }
        if (kind == 0)  /* confidence.dmb of view i is written right after its scan (main.cpp:1091-1095) */
            memcpy(conf_out[i], cons[i], sizeof(float) * (size_t)cols * rows);
    }
    for (int i = 0; i < num_views; ++i) {
        free(masks[i]);
        if (cons) free(cons[i]);
    }
    free(masks);
    free(cons);
    if (n_total) *n_total = count;
    return count < max_points ? count : max_points;
}

void ora_confidence_eval(int num_views, const hpm_camera *cams, const float *const *depths,
                         const float *const *normals, const int32_t *src_off, const int32_t *src_ids,
                         float *const *conf_out)
{
    consistency_scan(0, num_views, cams, depths, normals, NULL, NULL, src_off, src_ids, conf_out, NULL, 0, NULL);
}

int64_t ora_fusion(int num_views, const hpm_camera *cams, const float *const *depths,
                   const float *const *normals, const uint8_t *const *colors, const uint8_t *const *sky_masks,
                   const int32_t *src_off, const int32_t *src_ids, hpm_point *out, int64_t max_points,
                   int64_t *n_total)
{
    return consistency_scan(1, num_views, cams, depths, normals, colors, sky_masks, src_off, src_ids, NULL, out,
                            max_points, n_total);
}

int32_t ora_support_points(const float *costs, const float *conf, const float *texture, int tex_w,
                           int width, int height, int32_t *out_xy, int32_t max_points)
{
    /* `texture_flag` is computed but never used by the reference (HPM.cpp:1041-1048) */
    (void)texture; (void)tex_w;
    const int step = 5;
    int32_t n = 0;
    for (int col = 0; col < width; col += step) {
        for (int row = 0; row < height; row += step) {
            float min_nt = 2.0f, min_t = 2.0f;
            int pnt_x = 0, pnt_y = 0, pt_x = 0, pt_y = 0;
            const int cb = width < col + step ? width : col + step;
            const int rb = height < row + step ? height : row + step;
            for (int c = col; c < cb; ++c)
                for (int r = row; r < rb; ++r) {
                    const float pc = costs[r * width + c];
                    const float cf = conf[r * width + c];
                    if (pc < 2.0f) {
                        const float f_nt = pc - cf;
                        const float f_t = (float)(pc + 0.2 - cf);
                        if (min_nt > f_nt) { pnt_x = c; pnt_y = r; min_nt = f_nt; }
                        if (min_t > f_t) { pt_x = c; pt_y = r; min_t = f_t; }
                    }
                }
            if (min_t < 0.1) {
                if (n < max_points) { out_xy[2 * n] = pt_x; out_xy[2 * n + 1] = pt_y; }
                ++n;
            }
            if (min_nt < 0.1) {
                if (n < max_points) { out_xy[2 * n] = pnt_x; out_xy[2 * n + 1] = pnt_y; }
                ++n;
            }
        }
    }
    return n;
}

/* 3-point plane through camera-frame points: unit-normal null vector of the
 * 3x4 system [X Y Z 1] (cv::SVD::solveZ, HPM.cpp:1120/1155), computed from
 * cofactors in double precision; normalised by |n| with w >= 0. */
static void plane_fit(const double P[3][3], float out[4])
{
    const double a[3][4] = {
        { P[0][0], P[0][1], P[0][2], 1.0 },
        { P[1][0], P[1][1], P[1][2], 1.0 },
        { P[2][0], P[2][1], P[2][2], 1.0 } };
    double v[4];
    for (int k = 0; k < 4; ++k) {
        int cidx[3], m = 0;
        for (int q = 0; q < 4; ++q) if (q != k) cidx[m++] = q;
        const double det =
            a[0][cidx[0]] * (a[1][cidx[1]] * a[2][cidx[2]] - a[1][cidx[2]] * a[2][cidx[1]]) -
            a[0][cidx[1]] * (a[1][cidx[0]] * a[2][cidx[2]] - a[1][cidx[2]] * a[2][cidx[0]]) +
            a[0][cidx[2]] * (a[1][cidx[0]] * a[2][cidx[1]] - a[1][cidx[1]] * a[2][cidx[0]]);
        v[k] = (k % 2 == 0) ? det : -det;
    }
    double nrm = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (v[3] < 0) nrm = -nrm;
    out[0] = (float)(v[0] / nrm);
    out[1] = (float)(v[1] / nrm);
    out[2] = (float)(v[2] / nrm);
    out[3] = (float)(v[3] / nrm);
}

int32_t ora_planar_prior(const hpm_triangle *tris, int32_t n_tris, const float *depths, int width, int height,
                         const hpm_camera *c, float factor, float depth_min, float depth_max, int mode,
                         float *mask, float *planes_out, float *prior_depth, float *prior_normal)
{
    memset(mask, 0, sizeof(float) * (size_t)width * height);
    memset(prior_depth, 0, sizeof(float) * (size_t)width * height);
    if (prior_normal) memset(prior_normal, 0, sizeof(float) * 3 * (size_t)width * height);
    uint32_t idx = 0;
    for (int t = 0; t < n_tris; ++t) {
        const hpm_triangle *T = &tris[t];
        const int xs[3] = { T->x1, T->x2, T->x3 }, ys[3] = { T->y1, T->y2, T->y3 };
        int inside = 1;
        for (int k = 0; k < 3; ++k)
            if (!(xs[k] >= 0 && xs[k] < width && ys[k] >= 0 && ys[k] < height)) inside = 0;
        if (!inside) continue;
        const float L01 = (float)sqrt(pow((double)(T->x1 - T->x2), 2) + pow((double)(T->y1 - T->y2), 2));
        const float L02 = (float)sqrt(pow((double)(T->x1 - T->x3), 2) + pow((double)(T->y1 - T->y3), 2));
        const float L12 = (float)sqrt(pow((double)(T->x2 - T->x3), 2) + pow((double)(T->y2 - T->y3), 2));
        float mx = L01 > L02 ? L01 : L02;
        mx = mx > L12 ? mx : L12;
        const float step = (float)(1.0 / mx);
        for (float p = 0; p < 1.0; p += step)
            for (float q = 0; q < 1.0 - p; q += step) {
                const int x = (int)((double)(p * T->x1 + q * T->x2) + (1.0 - p - q) * T->x3);
                const int y = (int)((double)(p * T->y1 + q * T->y2) + (1.0 - p - q) * T->y3);
                mask[y * width + x] = (float)(idx + 1.0);
            }
        double P[3][3];
        for (int k = 0; k < 3; ++k) {
            const float d = depths[ys[k] * width + xs[k]];
            float X, Y;
            if (mode == 0) {
                X = d * (xs[k] - c->K[2]) / c->K[0];
                Y = d * (ys[k] - c->K[5]) / c->K[4];
            } else {
                X = d * (xs[k] - c->K[2] * factor) / (c->K[0] * factor);
                Y = d * (ys[k] - c->K[5] * factor) / (c->K[4] * factor);
            }
            P[k][0] = X; P[k][1] = Y; P[k][2] = d;
        }
        plane_fit(P, planes_out + 4 * (size_t)idx);
        idx++;
    }
    for (int i = 0; i < width; ++i)
        for (int j = 0; j < height; ++j) {
            const int k = j * width + i;
            if (mask[k] > 0) {
                const float *pl = planes_out + 4 * (size_t)((int)mask[k] - 1);
                float d;
                if (mode == 0) {
                    d = -pl[3] * c->K[0] / ((i - c->K[2]) * pl[0] + (c->K[0] / c->K[4]) * (j - c->K[5]) * pl[1] + c->K[0] * pl[2]);
                    if (d <= depth_max && d >= depth_min) prior_depth[k] = d;
                    else mask[k] = 0;
                } else {
                    d = -pl[3] * (c->K[0] * factor) / ((i - c->K[2] * factor) * pl[0] + (c->K[0] / c->K[4]) * (j - c->K[5] * factor) * pl[1] + c->K[0] * factor * pl[2]);
                    if (d <= depth_max * 1.2f && d >= depth_min * 0.6f) {
                        prior_depth[k] = d;
                        /* TransformNormal (HPM.cpp:1179-1187): camera -> world */
                        prior_normal[3 * k + 0] = c->R[0] * pl[0] + c->R[3] * pl[1] + c->R[6] * pl[2];
                        prior_normal[3 * k + 1] = c->R[1] * pl[0] + c->R[4] * pl[1] + c->R[7] * pl[2];
                        prior_normal[3 * k + 2] = c->R[2] * pl[0] + c->R[5] * pl[1] + c->R[8] * pl[2];
                    } else mask[k] = 0;
                }
            }
        }
    return (int32_t)idx;
}

/* cv::resize(..., INTER_LINEAR) for one float channel: half-pixel centres, taps
 * clamped at the borders.  The source coordinate is formed in double, and each
 * pass output is the two-tap sum evaluated exactly and rounded once; this agrees
 * with OpenCV 4.x to within 1 ulp (its SIMD kernels round differently). */
void ora_resize_linear_f32(const float *src, int sw, int sh, float *dst, int dw, int dh)
{
    const double sx_scale = 1.0 / ((double)dw / sw), sy_scale = 1.0 / ((double)dh / sh);
    int *xo = (int *)malloc(sizeof(int) * 2 * (size_t)dw);
    float *xa = (float *)malloc(sizeof(float) * 2 * (size_t)dw);
    for (int dx = 0; dx < dw; ++dx) {
        const double fxd = (dx + 0.5) * sx_scale - 0.5;
        int sx = (int)floor(fxd);
        float fx = (float)(fxd - sx);
        if (sx < 0) { fx = 0; sx = 0; }
        if (sx >= sw - 1) { fx = 0; sx = sw - 1; }
        xo[2 * dx] = sx; xo[2 * dx + 1] = sx + 1 < sw ? sx + 1 : sw - 1;
        xa[2 * dx] = 1.0f - fx; xa[2 * dx + 1] = fx;
    }
    float *r0 = (float *)malloc(sizeof(float) * (size_t)dw);
    float *r1 = (float *)malloc(sizeof(float) * (size_t)dw);
    for (int dy = 0; dy < dh; ++dy) {
        const double fyd = (dy + 0.5) * sy_scale - 0.5;
        int sy = (int)floor(fyd);
        float fy = (float)(fyd - sy);
        if (sy < 0) { fy = 0; sy = 0; }
        if (sy >= sh - 1) { fy = 0; sy = sh - 1; }
        const int sy1 = sy + 1 < sh ? sy + 1 : sh - 1;
        for (int dx = 0; dx < dw; ++dx) {
            r0[dx] = (float)((double)src[sy * sw + xo[2 * dx]] * xa[2 * dx] + (double)src[sy * sw + xo[2 * dx + 1]] * xa[2 * dx + 1]);
            r1[dx] = (float)((double)src[sy1 * sw + xo[2 * dx]] * xa[2 * dx] + (double)src[sy1 * sw + xo[2 * dx + 1]] * xa[2 * dx + 1]);
        }
        const float b0 = 1.0f - fy, b1 = fy;
        for (int dx = 0; dx < dw; ++dx) dst[dy * dw + dx] = (float)((double)r0[dx] * b0 + (double)r1[dx] * b1);
    }
    free(xo); free(xa); free(r0); free(r1);
}

void ora_prior_reload(const float *udepth, const float *unormal, int W, int H, const hpm_camera *c, float dmin,
                      float dmax, float *prior, uint8_t *mask)
{
    /* main.cpp:548-570 with TransformNormal2RefCam (HPM.cpp:1189-1197) and
     * GetDistance2Origin (HPM.cpp:1199-1206) */
    for (int j = 0; j < H; ++j)
        for (int i = 0; i < W; ++i) {
            const size_t k = (size_t)j * W + i;
            const float d = udepth[k];
            float *pl = prior + 4 * k;
            pl[0] = pl[1] = pl[2] = pl[3] = 0.0f;
            mask[k] = 0;
            if (d <= dmax && d >= dmin) {
                const float a = unormal[3 * k], b = unormal[3 * k + 1], e = unormal[3 * k + 2];
                pl[0] = c->R[0] * a + c->R[1] * b + c->R[2] * e;
                pl[1] = c->R[3] * a + c->R[4] * b + c->R[5] * e;
                pl[2] = c->R[6] * a + c->R[7] * b + c->R[8] * e;
                const float X0 = d * (i - c->K[2]) / (c->K[0]);
                const float X1 = d * (j - c->K[5]) / (c->K[4]);
                pl[3] = -(pl[0] * X0 + pl[1] * X1 + pl[2] * d);
                mask[k] = 1;
            }
        }
}
