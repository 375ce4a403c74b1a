/*
 * CPU oracle for the Fourier-slice path.  TEST INFRASTRUCTURE ONLY: the
 * product never links or calls this file.  Only tests/, the smoke check and
 * the CPU-baseline legs of bench.py load it, as the checker.
 *
 * It restates, in plain C float32 arithmetic, the reference algorithm of
 * torch-fourier-slice / torch-image-interpolation (teamtomo monorepo,
 * packages/primitives/...):
 *
 *   extract   torch_fourier_slice/slice_extraction/_extract_central_slices_rfft_3d.py:84-222
 *             (+ _determine_near_zero_conjugate_mask :9-81)
 *   insert    torch_fourier_slice/slice_insertion/_insert_central_slices_rfft_3d.py:9-106,
 *             _insert_into_3d_dft :213-286, _insert_into_3d_dft_linear :289-406
 *             (the Friedel mirror is applied per corner, exactly as the reference
 *             does it, not as the x=0 plane post-pass the CUDA path uses)
 *   coords    torch_fourier_slice/_dft_utils.py:37-72
 *   grid      torch_fourier_slice/_grids/_central_slice_fftfreq_grid.py:6-32 and
 *             torch_grid_utils/fftfreq_grid.py:180-224 (fftfreq = f32(k) * f32(1/n))
 *   sampling  torch_image_interpolation/image_interpolation_3d.py:11-101 with
 *             F.grid_sample(trilinear, padding 'border', align_corners=True),
 *             including the array -> grid -> array coordinate round trip of
 *             torch_image_interpolation/grid_sample_utils.py:6-26
 *   gradients autograd of the extraction: d/dvolume is the trilinear scatter of
 *             the (conjugated where the conjugate mask is set) upstream
 *             gradient; d/drotation chains grid_sample's grid gradient through
 *             the coordinate scaling, the conjugate flip, the matmul and the
 *             xyz<->zyx flip; elements zeroed by rot_tolerance get zero gradient.
 *
 * Arithmetic order follows the reference on CPU: the rotation is
 * ((r0*q0 + r1*q1) + r2*q2) with every product rounded (torch's CPU matmul for
 * these shapes uses no fused multiply-add), and every other expression is
 * evaluated left to right in float32.  Build with -ffp-contract=off.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* fftfreq value of row `i` of an fftshifted axis of length n. */
static float shifted_freq(int64_t i, int64_t n, float inv_n) {
    int64_t k = (i - n / 2 + n) % n;
    int64_t kk = (k < (n + 1) / 2) ? k : k - n;
    return (float)kk * inv_n;
}

/* float32 copy of the caller's matrix with optional tolerance zeroing (xyz
 * layout, before the flip) and the xyz -> zyx flip. */
static void prep_rotation(const float *r, int zyx, int has_rot_tol, float rot_tol,
                          float out[9]) {
    float m[9];
    for (int k = 0; k < 9; k++) {
        float v = r[k];
        if (has_rot_tol && fabsf(v) < rot_tol) v = 0.0f;
        m[k] = v;
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            out[i * 3 + j] = zyx ? m[i * 3 + j] : m[(2 - i) * 3 + (2 - j)];
}

static void rotate(const float m[9], const float q[3], float p[3]) {
    for (int i = 0; i < 3; i++) {
        float a = m[i * 3 + 0] * q[0];
        float b = m[i * 3 + 1] * q[1];
        float c = m[i * 3 + 2] * q[2];
        float s = a + b;
        p[i] = s + c;
    }
}

typedef struct {
    float s0, s1, sx;     /* (d-1), (h-1), (wr-1) of the image shape */
    float iw0, iw1;       /* 1 - 1/d, 1 - 1/h */
} coord_scale;

static coord_scale make_scale(int64_t d, int64_t h, int64_t w) {
    coord_scale s;
    float fd = (float)d, fh = (float)h, fwr = (float)(w / 2 + 1);
    float dd = 1.0f / fd, dh = 1.0f / fh;
    s.iw0 = 1.0f - dd;
    s.iw1 = 1.0f - dh;
    s.s0 = fd - 1.0f;
    s.s1 = fh - 1.0f;
    s.sx = fwr - 1.0f;
    return s;
}

static void to_dft_coords(const coord_scale *s, const float p[3], float c[3]) {
    float t0 = p[0] + 0.5f;
    t0 = t0 / s->iw0;
    c[0] = t0 * s->s0;
    float t1 = p[1] + 0.5f;
    t1 = t1 / s->iw1;
    c[1] = t1 * s->s1;
    float t2 = p[2] * 2.0f;
    c[2] = t2 * s->sx;
}

/* array coordinate -> grid_sample coordinate -> unnormalised source index,
 * clipped to [0, n-1] (padding_mode='border', align_corners=True).  *grad_ok:
 * the clip passes a coordinate gradient, i.e. the unclipped index lies
 * strictly inside (0, n-1) — on the border itself grid_sample's backward
 * treats the point as clipped and gives that axis zero gradient. */
static float roundtrip_index(float c, int64_t n, int *grad_ok) {
    float fn = (float)n;
    float half = 0.5f * fn - 0.5f;
    float g = c / half - 1.0f;
    float ix = ((g + 1.0f) / 2.0f) * (fn - 1.0f);
    *grad_ok = ix > 0.0f && ix < fn - 1.0f;
    if (ix < 0.0f) ix = 0.0f;
    if (ix > fn - 1.0f) ix = fn - 1.0f;
    return ix;
}

static int inside3(const float c[3], int64_t D, int64_t H, int64_t W) {
    return c[0] >= 0.0f && c[0] <= (float)(D - 1) && c[1] >= 0.0f && c[1] <= (float)(H - 1) &&
           c[2] >= 0.0f && c[2] <= (float)(W - 1);
}

/* grid_sample trilinear corner set: indices and weights in the order
 * tnw, tne, tsw, tse, bnw, bne, bsw, bse (t/b = z0/z1, n/s = y0/y1, w/e = x0/x1). */
typedef struct {
    int64_t z[8], y[8], x[8];
    float w[8];
    /* d w / d(ix, iy, iz) for each corner */
    float gx[8], gy[8], gz[8];
    float ix, iy, iz;
    int ok_x, ok_y, ok_z; /* the coordinate gradient passes the border clip */
} tri_corners;

static void grid_sample_corners(const float c[3], int64_t D, int64_t H, int64_t W,
                                tri_corners *t) {
    float iz = roundtrip_index(c[0], D, &t->ok_z);
    float iy = roundtrip_index(c[1], H, &t->ok_y);
    float ix = roundtrip_index(c[2], W, &t->ok_x);
    float x0 = floorf(ix), y0 = floorf(iy), z0 = floorf(iz);
    float x1 = x0 + 1.0f, y1 = y0 + 1.0f, z1 = z0 + 1.0f;
    float ax0 = x1 - ix, ax1 = ix - x0;
    float ay0 = y1 - iy, ay1 = iy - y0;
    float az0 = z1 - iz, az1 = iz - z0;
    t->ix = ix; t->iy = iy; t->iz = iz;
    for (int k = 0; k < 8; k++) {
        int bz = (k >> 2) & 1, by = (k >> 1) & 1, bx = k & 1;
        float wx = bx ? ax1 : ax0, wy = by ? ay1 : ay0, wz = bz ? az1 : az0;
        float sx = bx ? 1.0f : -1.0f, sy = by ? 1.0f : -1.0f, sz = bz ? 1.0f : -1.0f;
        t->x[k] = (int64_t)(bx ? x1 : x0);
        t->y[k] = (int64_t)(by ? y1 : y0);
        t->z[k] = (int64_t)(bz ? z1 : z0);
        t->w[k] = wx * wy * wz;
        t->gx[k] = sx * wy * wz;
        t->gy[k] = sy * wx * wz;
        t->gz[k] = sz * wx * wy;
    }
}

static int in_bounds(int64_t z, int64_t y, int64_t x, int64_t D, int64_t H, int64_t W) {
    return z >= 0 && z < D && y >= 0 && y < H && x >= 0 && x < W;
}

typedef struct {
    int has_fmax;
    float fmax;
    int zyx;
    float x_tol, x_tol10;
    int has_rot_tol;
    float rot_tol;
} extract_opts;

/* Per-point extraction geometry: returns 0 when the pixel is outside the
 * fftfreq_max disc, otherwise fills conj flag, rotated+flipped frequency and
 * array coordinate. */
static int extract_point(const float m[9], int64_t iy, int64_t ix, int64_t img_h,
                         float inv_h, float inv_w, const extract_opts *o, const coord_scale *s,
                         int *conj, float q[3], float c[3]) {
    q[0] = 0.0f;
    q[1] = shifted_freq(iy, img_h, inv_h);
    q[2] = (float)ix * inv_w;
    if (o->has_fmax) {
        float a = q[0] * q[0], b = q[1] * q[1], cc = q[2] * q[2];
        float nrm = sqrtf((a + b) + cc);
        if (!(nrm <= o->fmax)) return 0;
    }
    float p[3];
    rotate(m, q, p);
    int cj = p[2] < -o->x_tol;
    if (fabsf(p[2]) < o->x_tol) {
        float r11 = m[8], r12 = m[7];
        if (fabsf(r11) <= o->x_tol10) cj = cj || (r12 < 0.0f);
        else cj = cj || (r11 < 0.0f);
    }
    if (cj) { p[0] = -p[0]; p[1] = -p[1]; p[2] = -p[2]; }
    *conj = cj;
    to_dft_coords(s, p, c);
    return 1;
}

int orc_extract(const float *vol, int64_t D, int64_t H, int64_t W, const float *rot, int64_t n,
                int64_t img_d, int64_t img_h, int64_t img_w, int has_fmax, float fmax, int zyx,
                float x_tol, float x_tol10, int has_rot_tol, float rot_tol, float *out,
                uint8_t *conj_out, float *coords_out, int nthreads) {
    int64_t wr = img_w / 2 + 1, P = img_h * wr;
    float inv_h = (float)(1.0 / (double)img_h), inv_w = (float)(1.0 / (double)img_w);
    extract_opts o = {has_fmax, fmax, zyx, x_tol, x_tol10, has_rot_tol, rot_tol};
    coord_scale s = make_scale(img_d, img_h, img_w);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
    for (int64_t b = 0; b < n; b++) {
        float m[9];
        prep_rotation(rot + b * 9, zyx, has_rot_tol, rot_tol, m);
        for (int64_t iy = 0; iy < img_h; iy++)
            for (int64_t ix = 0; ix < wr; ix++) {
                int64_t o_idx = b * P + iy * wr + ix;
                float q[3], c[3];
                int cj = 0;
                float re = 0.0f, im = 0.0f;
                int valid = extract_point(m, iy, ix, img_h, inv_h, inv_w, &o, &s, &cj, q, c);
                if (conj_out) conj_out[o_idx] = (uint8_t)(valid ? (cj ? 1 : 0) : 0);
                if (coords_out) {
                    coords_out[o_idx * 3 + 0] = valid ? c[0] : 0.0f;
                    coords_out[o_idx * 3 + 1] = valid ? c[1] : 0.0f;
                    coords_out[o_idx * 3 + 2] = valid ? c[2] : 0.0f;
                }
                if (valid && inside3(c, D, H, W)) {
                    tri_corners t;
                    grid_sample_corners(c, D, H, W, &t);
                    for (int k = 0; k < 8; k++) {
                        if (!in_bounds(t.z[k], t.y[k], t.x[k], D, H, W)) continue;
                        const float *v = vol + ((t.z[k] * H + t.y[k]) * W + t.x[k]) * 2;
                        re += v[0] * t.w[k];
                        im += v[1] * t.w[k];
                    }
                    if (cj) im = -im;
                }
                out[o_idx * 2 + 0] = re;
                out[o_idx * 2 + 1] = im;
            }
    }
    return 0;
}

/* Gradient of the extraction.  `grad` is the upstream gradient of the slices
 * (n, img_h, wr) complex64 in PyTorch's convention (dL = Re(conj(G) ds)).
 * dvol (D,H,W complex, accumulated, may be NULL) receives d/dvolume; drot (n,9,
 * may be NULL) receives d/d(rotation) in the caller's (xyz unless zyx) layout
 * with tolerance-zeroed elements set to zero.  Sums run in double. */
int orc_extract_grad(const float *vol, int64_t D, int64_t H, int64_t W, const float *rot,
                     int64_t n, int64_t img_d, int64_t img_h, int64_t img_w, int has_fmax,
                     float fmax, int zyx, float x_tol, float x_tol10, int has_rot_tol,
                     float rot_tol, const float *grad, float *dvol, double *drot, int nthreads) {
    int64_t wr = img_w / 2 + 1, P = img_h * wr;
    float inv_h = (float)(1.0 / (double)img_h), inv_w = (float)(1.0 / (double)img_w);
    extract_opts o = {has_fmax, fmax, zyx, x_tol, x_tol10, has_rot_tol, rot_tol};
    coord_scale s = make_scale(img_d, img_h, img_w);
    /* d c_i / d p_i, in double */
    double dcdp[3] = {(double)s.s0 / (double)s.iw0, (double)s.s1 / (double)s.iw1,
                      2.0 * (double)s.sx};
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
    for (int64_t b = 0; b < n; b++) {
        float m[9];
        prep_rotation(rot + b * 9, zyx, has_rot_tol, rot_tol, m);
        double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int64_t iy = 0; iy < img_h; iy++)
            for (int64_t ix = 0; ix < wr; ix++) {
                int64_t o_idx = b * P + iy * wr + ix;
                float q[3], c[3];
                int cj = 0;
                if (!extract_point(m, iy, ix, img_h, inv_h, inv_w, &o, &s, &cj, q, c)) continue;
                if (!inside3(c, D, H, W)) continue;
                float gre = grad[o_idx * 2 + 0], gim = grad[o_idx * 2 + 1];
                if (cj) gim = -gim; /* G' = conj(G) where the sample was conjugated */
                tri_corners t;
                grid_sample_corners(c, D, H, W, &t);
                double dz = 0, dy = 0, dx = 0;
                for (int k = 0; k < 8; k++) {
                    if (!in_bounds(t.z[k], t.y[k], t.x[k], D, H, W)) continue;
                    int64_t vi = (t.z[k] * H + t.y[k]) * W + t.x[k];
                    if (dvol) {
#ifdef _OPENMP
#pragma omp atomic
#endif
                        dvol[vi * 2 + 0] += gre * t.w[k];
#ifdef _OPENMP
#pragma omp atomic
#endif
                        dvol[vi * 2 + 1] += gim * t.w[k];
                    }
                    if (drot) {
                        /* Re(conj(G') * V) */
                        double rv = (double)gre * vol[vi * 2 + 0] + (double)gim * vol[vi * 2 + 1];
                        dz += rv * t.gz[k];
                        dy += rv * t.gy[k];
                        dx += rv * t.gx[k];
                    }
                }
                if (drot) {
                    /* the clip of padding_mode='border' passes no gradient along an
                     * axis whose source index lies on the border (0 or n-1) */
                    double sg = cj ? -1.0 : 1.0;
                    double dp[3] = {dz * dcdp[0] * sg * t.ok_z, dy * dcdp[1] * sg * t.ok_y,
                                    dx * dcdp[2] * sg * t.ok_x};
                    for (int i = 0; i < 3; i++)
                        for (int j = 0; j < 3; j++) acc[i * 3 + j] += dp[i] * (double)q[j];
                }
            }
        if (drot) {
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) {
                    /* undo the xyz -> zyx flip */
                    int si = zyx ? i : 2 - i, sj = zyx ? j : 2 - j;
                    double g = acc[i * 3 + j];
                    if (has_rot_tol && fabsf(rot[b * 9 + si * 3 + sj]) < rot_tol) g = 0.0;
                    drot[b * 9 + si * 3 + sj] = g;
                }
        }
    }
    return 0;
}

/* Per-pixel geometry under the extraction (mode 0) or insertion (mode 1) rule:
 * flags bit0 pixel kept (fftfreq_max; insertion also drops the x==0, y<0
 * source pixels), bit1 conjugate redirect, bit2 inside the volume (extraction:
 * sample_image_3d's inside test; insertion: _insert_into_3d_dft's bounds
 * filter, the same test); coords are the redirected array coordinates.
 * Insertion applies no rot_tolerance and the strict x' < 0 rule
 * (_insert_central_slices_rfft_3d.py:78-80). */
int orc_slice_geometry(const float *rot, int64_t n, int64_t img_d, int64_t img_h, int64_t img_w,
                       int64_t D, int64_t H, int64_t W, int has_fmax, float fmax, int zyx,
                       float x_tol, float x_tol10, int has_rot_tol, float rot_tol, int mode,
                       uint8_t *flags, float *coords) {
    int64_t wr = img_w / 2 + 1, P = img_h * wr;
    float inv_h = (float)(1.0 / (double)img_h), inv_w = (float)(1.0 / (double)img_w);
    coord_scale s = make_scale(img_d, img_h, img_w);
    for (int64_t b = 0; b < n; b++) {
        float m[9];
        prep_rotation(rot + b * 9, zyx, mode == 0 ? has_rot_tol : 0, rot_tol, m);
        for (int64_t iy = 0; iy < img_h; iy++)
            for (int64_t ix = 0; ix < wr; ix++) {
                int64_t o = b * P + iy * wr + ix;
                float q[3] = {0.0f, shifted_freq(iy, img_h, inv_h), (float)ix * inv_w};
                float c[3] = {0.0f, 0.0f, 0.0f};
                uint8_t f = 0;
                int valid = 1;
                if (has_fmax) {
                    float a = q[0] * q[0], bb = q[1] * q[1], cc = q[2] * q[2];
                    float nrm = sqrtf((a + bb) + cc);
                    valid = nrm <= fmax;
                }
                if (mode == 1 && q[2] == 0.0f && q[1] < 0.0f) valid = 0;
                if (valid) {
                    float p[3];
                    int cj;
                    rotate(m, q, p);
                    if (mode == 0) {
                        cj = p[2] < -x_tol;
                        if (fabsf(p[2]) < x_tol) {
                            float r11 = m[8], r12 = m[7];
                            cj = (fabsf(r11) <= x_tol10) ? (r12 < 0.0f) : (r11 < 0.0f);
                        }
                    } else {
                        cj = p[2] < 0.0f;
                    }
                    if (cj) { p[0] = -p[0]; p[1] = -p[1]; p[2] = -p[2]; }
                    to_dft_coords(&s, p, c);
                    f = (uint8_t)(1 | (cj ? 2 : 0) | (inside3(c, D, H, W) ? 4 : 0));
                }
                flags[o] = f;
                coords[o * 3 + 0] = c[0];
                coords[o * 3 + 1] = c[1];
                coords[o * 3 + 2] = c[2];
            }
    }
    return 0;
}

/* Insertion.  Follows _insert_central_slices_rfft_3d.py:9-106 and
 * _insert_into_3d_dft_linear :289-406 literally, including the per-corner
 * Friedel mirror on the x=0 plane.  Accumulates into vol / wts.
 * REAL is float (complex64 data, float32 weights) or double (complex128 data,
 * float64 weights; coordinates and weights are still computed in float32). */
#define DEFINE_INSERT(NAME, REAL)                                                            \
    int NAME(const REAL *img, int64_t n, int64_t vd, int64_t vh, int64_t vw, const float *rot, \
             int has_fmax, float fmax, int zyx, REAL *vol, REAL *wts, int mirror, int nthreads) { \
        int64_t wr = vw / 2 + 1, P = vh * wr;                                               \
        int64_t D = vd, H = vh, W = wr;                                                     \
        float inv_h = (float)(1.0 / (double)vh), inv_w = (float)(1.0 / (double)vw);          \
        coord_scale s = make_scale(vd, vh, vw);                                             \
        float ub0 = (float)D - 1.0f, ub1 = (float)H - 1.0f, ub2 = (float)W - 1.0f;           \
        (void)nthreads;                                                                     \
        for (int64_t b = 0; b < n; b++) {                                                   \
            float m[9];                                                                     \
            prep_rotation(rot + b * 9, zyx, 0, 0.0f, m);                                    \
            for (int64_t iy = 0; iy < vh; iy++)                                             \
                for (int64_t ix = 0; ix < wr; ix++) {                                       \
                    float q[3] = {0.0f, shifted_freq(iy, vh, inv_h), (float)ix * inv_w};    \
                    if (has_fmax) {                                                         \
                        float a = q[0] * q[0], bb = q[1] * q[1], cc = q[2] * q[2];          \
                        float nrm = sqrtf((a + bb) + cc);                                   \
                        if (!(nrm <= fmax)) continue;                                       \
                    }                                                                       \
                    if (q[2] == 0.0f && q[1] < 0.0f) continue; /* Friedel-redundant */      \
                    const REAL *dv = img + (b * P + iy * wr + ix) * 2;                      \
                    REAL dre = dv[0], dim = dv[1];                                          \
                    float p[3], c[3];                                                       \
                    rotate(m, q, p);                                                        \
                    if (p[2] < 0.0f) {                                                      \
                        p[0] = -p[0]; p[1] = -p[1]; p[2] = -p[2];                           \
                        dim = -dim;                                                         \
                    }                                                                       \
                    to_dft_coords(&s, p, c);                                                \
                    if (!(c[0] >= 0.0f && c[0] <= ub0 && c[1] >= 0.0f && c[1] <= ub1 &&      \
                          c[2] >= 0.0f && c[2] <= ub2))                                     \
                        continue;                                                           \
                    float z0 = floorf(c[0]), y0 = floorf(c[1]), x0 = floorf(c[2]);          \
                    float z1 = ceilf(c[0]), y1 = ceilf(c[1]), x1 = ceilf(c[2]);             \
                    float tz = c[0] - z0, ty = c[1] - y0, tx = c[2] - x0;                   \
                    for (int k = 0; k < 8; k++) {                                           \
                        int bz = (k >> 2) & 1, by = (k >> 1) & 1, bx = k & 1;               \
                        float fz = bz ? tz : (1.0f - tz);                                   \
                        float fy = by ? ty : (1.0f - ty);                                   \
                        float fx = bx ? tx : (1.0f - tx);                                   \
                        float w = (fz * fy) * fx;                                           \
                        int64_t zi = (int64_t)(bz ? z1 : z0), yi = (int64_t)(by ? y1 : y0);  \
                        int64_t xi = (int64_t)(bx ? x1 : x0);                               \
                        int64_t vi = (zi * H + yi) * W + xi;                                \
                        REAL rw = (REAL)w;                                                  \
                        vol[vi * 2 + 0] += dre * rw;                                        \
                        vol[vi * 2 + 1] += dim * rw;                                        \
                        wts[vi] += rw;                                                      \
                        if (mirror && xi == 0 && !(zi == D / 2 && yi == H / 2)) {           \
                            int64_t zm = (D - zi) % D, ym = (H - yi) % H;                   \
                            int64_t mi = (zm * H + ym) * W;                                 \
                            vol[mi * 2 + 0] += dre * rw;                                    \
                            vol[mi * 2 + 1] += (-dim) * rw;                                 \
                            wts[mi] += rw;                                                  \
                        }                                                                   \
                    }                                                                       \
                }                                                                           \
        }                                                                                   \
        return 0;                                                                           \
    }

DEFINE_INSERT(orc_insert_c64, float)
DEFINE_INSERT(orc_insert_c128, double)

/* Multi-threaded variant of the complex64 insertion used only for CPU
 * baseline timing: slices are split over threads and the accumulation uses
 * atomic adds (memory stays one volume however many threads run). */
int orc_insert_c64_mt(const float *img, int64_t n, int64_t vd, int64_t vh, int64_t vw,
                      const float *rot, int has_fmax, float fmax, int zyx, float *vol,
                      float *wts, int mirror, int nthreads) {
    int64_t wr = vw / 2 + 1, P = vh * wr;
    int64_t D = vd, H = vh, W = wr;
    float inv_h = (float)(1.0 / (double)vh), inv_w = (float)(1.0 / (double)vw);
    coord_scale s = make_scale(vd, vh, vw);
    float ub0 = (float)D - 1.0f, ub1 = (float)H - 1.0f, ub2 = (float)W - 1.0f;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int64_t b = 0; b < n; b++) {
        float m[9];
        prep_rotation(rot + b * 9, zyx, 0, 0.0f, m);
        for (int64_t iy = 0; iy < vh; iy++)
            for (int64_t ix = 0; ix < wr; ix++) {
                float q[3] = {0.0f, shifted_freq(iy, vh, inv_h), (float)ix * inv_w};
                if (has_fmax) {
                    float a = q[0] * q[0], bb = q[1] * q[1], cc = q[2] * q[2];
                    if (!(sqrtf((a + bb) + cc) <= fmax)) continue;
                }
                if (q[2] == 0.0f && q[1] < 0.0f) continue;
                const float *dv = img + (b * P + iy * wr + ix) * 2;
                float dre = dv[0], dim = dv[1];
                float p[3], c[3];
                rotate(m, q, p);
                if (p[2] < 0.0f) { p[0] = -p[0]; p[1] = -p[1]; p[2] = -p[2]; dim = -dim; }
                to_dft_coords(&s, p, c);
                if (!(c[0] >= 0.0f && c[0] <= ub0 && c[1] >= 0.0f && c[1] <= ub1 && c[2] >= 0.0f &&
                      c[2] <= ub2))
                    continue;
                float z0 = floorf(c[0]), y0 = floorf(c[1]), x0 = floorf(c[2]);
                float z1 = ceilf(c[0]), y1 = ceilf(c[1]), x1 = ceilf(c[2]);
                float tz = c[0] - z0, ty = c[1] - y0, tx = c[2] - x0;
                for (int k = 0; k < 8; k++) {
                    int bz = (k >> 2) & 1, by = (k >> 1) & 1, bx = k & 1;
                    float w = ((bz ? tz : 1.0f - tz) * (by ? ty : 1.0f - ty)) * (bx ? tx : 1.0f - tx);
                    int64_t zi = (int64_t)(bz ? z1 : z0), yi = (int64_t)(by ? y1 : y0);
                    int64_t xi = (int64_t)(bx ? x1 : x0);
                    int64_t vi = (zi * H + yi) * W + xi;
                    float a = dre * w, bi = dim * w;
#ifdef _OPENMP
#pragma omp atomic
#endif
                    vol[vi * 2 + 0] += a;
#ifdef _OPENMP
#pragma omp atomic
#endif
                    vol[vi * 2 + 1] += bi;
#ifdef _OPENMP
#pragma omp atomic
#endif
                    wts[vi] += w;
                    if (mirror && xi == 0 && !(zi == D / 2 && yi == H / 2)) {
                        int64_t mi = (((D - zi) % D) * H + (H - yi) % H) * W;
#ifdef _OPENMP
#pragma omp atomic
#endif
                        vol[mi * 2 + 0] += a;
#ifdef _OPENMP
#pragma omp atomic
#endif
                        vol[mi * 2 + 1] -= bi;
#ifdef _OPENMP
#pragma omp atomic
#endif
                        wts[mi] += w;
                    }
                }
            }
    }
    return 0;
}
