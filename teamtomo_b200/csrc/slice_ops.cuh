// Per-point operations shared by the single-volume and the batched kernels:
// grid_sample-style trilinear sampling of an rfft volume, the insertion splat,
// and the in-kernel CTF.
#pragma once
#include <cuda_runtime.h>

#include "slice_common.cuh"

namespace tt {

// ---------------------------------------------------------------- sampling

// grid_sample's source index of array coordinate c on an axis of n samples:
// c -> grid coordinate c / (0.5 n - 0.5) - 1 (grid_sample_utils.py:6-26) ->
// ((g + 1) / 2) * (n - 1) (align_corners=True), clipped to [0, n-1].
// grad_ok: the border clip passes a coordinate gradient — grid_sample's
// backward treats an index on the border itself (0 or n-1) as clipped.
__device__ __forceinline__ float source_index(float c, float half, float nm1, bool& grad_ok) {
    const float gc = __fsub_rn(__fdiv_rn(c, half), 1.0f);
    const float ix = __fmul_rn(__fmul_rn(__fadd_rn(gc, 1.0f), 0.5f), nm1);
    grad_ok = ix > 0.0f && ix < nm1;
    return fminf(fmaxf(ix, 0.0f), nm1);
}

struct Corners {
    int z0, y0, x0;
    float ax0, ax1, ay0, ay1, az0, az1;  // per-axis weights of the low/high corner
    bool zin, yin, xin;                  // high corner inside the array
    bool gz, gy, gx;                     // the axis passes a coordinate gradient (not on the border)
};

// grid_sample source indices (z, y, x) of an inside array coordinate c, in
// [0, n-1], and whether each axis passes a coordinate gradient.
struct SourceIdx {
    float z, y, x;
    bool gz, gy, gx;
};

__device__ __forceinline__ SourceIdx source_indices(const SliceGeom& g, const float c[3]) {
    SourceIdx si;
    si.z = source_index(c[0], 0.5f * (float)g.D - 0.5f, g.ub0, si.gz);
    si.y = source_index(c[1], 0.5f * (float)g.H - 0.5f, g.ub1, si.gy);
    si.x = source_index(c[2], 0.5f * (float)g.W - 0.5f, g.ub2, si.gx);
    return si;
}

// Trilinear corner set of source indices (iz, iy, ix); gz, gy, gx are left
// false (make_corners sets them).
__device__ __forceinline__ Corners corners_at(const SliceGeom& g, float iz, float iy, float ix) {
    Corners k;
    k.gz = k.gy = k.gx = false;
    const float fz = floorf(iz), fy = floorf(iy), fx = floorf(ix);
    k.z0 = (int)fz;
    k.y0 = (int)fy;
    k.x0 = (int)fx;
    k.az0 = (fz + 1.0f) - iz;
    k.az1 = iz - fz;
    k.ay0 = (fy + 1.0f) - iy;
    k.ay1 = iy - fy;
    k.ax0 = (fx + 1.0f) - ix;
    k.ax1 = ix - fx;
    k.zin = k.z0 + 1 < g.D;
    k.yin = k.y0 + 1 < g.H;
    k.xin = k.x0 + 1 < g.W;
    return k;
}

// grid_sample trilinear corner set of an inside array coordinate c (the
// round trip decides the cell at integer kinks, where the derivative jumps).
__device__ __forceinline__ Corners make_corners(const SliceGeom& g, const float c[3]) {
    const SourceIdx si = source_indices(g, c);
    Corners k = corners_at(g, si.z, si.y, si.x);
    k.gz = si.gz;
    k.gy = si.gy;
    k.gx = si.gx;
    return k;
}

// Geometry of one extraction pixel: false when the pixel is outside
// fftfreq_max or its point outside the volume.
__device__ __forceinline__ bool extract_geometry(const SliceGeom& g, const float* m, int iy, int ix, float& qy,
                                                 float& qx, bool& cj, float c[3]) {
    qy = shifted_freq(iy, g.img_h, g.inv_h);
    qx = __fmul_rn((float)ix, g.inv_w);
    if (!in_fmax(g, qy, qx)) return false;
    float p[3];
    rotate_slice_point(m, qy, qx, p);
    cj = extract_conj(g, m, p[2]);
    if (cj) {
        p[0] = -p[0];
        p[1] = -p[1];
        p[2] = -p[2];
    }
    to_dft_coords(g, p, c);
    return inside_volume(g, c);
}

// The part of the extraction geometry that depends only on the slice row:
// its frequency qy, qy^2 for the fftfreq_max test, and the rotation's products
// m[i][1] * qy, each rounded as rotate_slice_point rounds it.  The slice
// kernels walk a row of tiles with a fixed row per thread, so these are formed
// once per thread instead of once per pixel.
struct SliceRow {
    float qy, qy2, my[3];
};

__device__ __forceinline__ SliceRow slice_row_geom(const SliceGeom& g, const float* m, int iy) {
    SliceRow r;
    r.qy = shifted_freq(iy, g.img_h, g.inv_h);
    r.qy2 = __fmul_rn(r.qy, r.qy);
#pragma unroll
    for (int i = 0; i < 3; i++) r.my[i] = __fmul_rn(m[i * 3 + 1], r.qy);
    return r;
}

// extract_geometry with the row part precomputed: the same operations and
// roundings, so the same flags and coordinates bit for bit.
__device__ __forceinline__ bool extract_geometry_row(const SliceGeom& g, const float* m, const SliceRow& row, int ix,
                                                     float& qx, bool& cj, float c[3]) {
    qx = __fmul_rn((float)ix, g.inv_w);
    if (g.has_fmax && !(__fsqrt_rn(__fadd_rn(row.qy2, __fmul_rn(qx, qx))) <= g.fmax)) return false;
    float p[3];
#pragma unroll
    for (int i = 0; i < 3; i++) p[i] = __fadd_rn(row.my[i], __fmul_rn(m[i * 3 + 2], qx));
    cj = extract_conj(g, m, p[2]);
    if (cj) {
        p[0] = -p[0];
        p[1] = -p[1];
        p[2] = -p[2];
    }
    to_dft_coords(g, p, c);
    return inside_volume(g, c);
}

// Element type of the bricked copy (brick_index addressing): one complex64 voxel.
struct VoxBrick2 {
    float x, y;
};

// The two x-corners (x0, x0 + 1) of volume row (z, y) (fftshifted
// coordinates): v0 when lo, v1 when hi (hi implies lo), zero otherwise.
// Plain layout: two 8-byte gathers.
__device__ __forceinline__ void load_xrow(const float2* __restrict__ vol, const SliceGeom& g, int z, int y, int x0,
                                          bool lo, bool hi, float2& v0, float2& v1) {
    const int64_t base = vox_index(g, z, y, x0);
    v0 = lo ? __ldg(vol + base) : make_float2(0.0f, 0.0f);
    v1 = hi ? __ldg(vol + base + 1) : make_float2(0.0f, 0.0f);
}

// x-paired layout (entry = (V[x], V[x + 1])): one 16-byte gather.
__device__ __forceinline__ void load_xrow(const float4* __restrict__ vol, const SliceGeom& g, int z, int y, int x0,
                                          bool lo, bool hi, float2& v0, float2& v1) {
    const float4 q = lo ? __ldg(vol + vox_index(g, z, y, x0)) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    v0 = make_float2(q.x, q.y);
    v1 = hi ? make_float2(q.z, q.w) : make_float2(0.0f, 0.0f);
}

// The four x-rows (z0 + bz, y0 + by) of a trilinear corner set k, addressed
// for layout VT: row (bz, by) gives v0 = V[.., x0] when lo and v1 =
// V[.., x0 + 1] when hi (hi implies lo), zero otherwise.
template <typename VT>
struct XRows {
    const VT* vol;
    int z0, y0, x0;
    __device__ __forceinline__ XRows(const VT* v, const SliceGeom&, const Corners& k)
        : vol(v), z0(k.z0), y0(k.y0), x0(k.x0) {}
    __device__ __forceinline__ void load(const SliceGeom& g, int bz, int by, bool lo, bool hi, float2& v0,
                                         float2& v1) const {
        load_xrow(vol, g, z0 + bz, y0 + by, x0, lo, hi, v0, v1);
    }
};

// Bricked layout (always fftshifted): the corner (z0, y0, x0) is addressed
// once; its +1 neighbours are the next slot of the brick along an even
// coordinate and the first slot of the next brick along an odd one (x: 1 or
// 7 slots, y: 2 or one brick row - 2, z: 4 or one brick plane - 4).  32-bit
// slot offsets: bricked copies hold fewer than 2^31 slots.
template <>
struct XRows<VoxBrick2> {
    const float2* p;
    uint32_t base, dz, dy, dx;
    __device__ __forceinline__ XRows(const VoxBrick2* v, const SliceGeom& g, const Corners& k)
        : p(reinterpret_cast<const float2*>(v)) {
        const uint32_t bh = (uint32_t)(g.H + 1) >> 1, bw = (uint32_t)(g.W + 1) >> 1;
        base = ((((uint32_t)k.z0 >> 1) * bh + ((uint32_t)k.y0 >> 1)) * bw + ((uint32_t)k.x0 >> 1)) * 8u +
               (((uint32_t)k.z0 & 1u) << 2) + (((uint32_t)k.y0 & 1u) << 1) + ((uint32_t)k.x0 & 1u);
        dx = (k.x0 & 1) ? 7u : 1u;
        dy = (k.y0 & 1) ? bw * 8u - 2u : 2u;
        dz = (k.z0 & 1) ? bh * bw * 8u - 4u : 4u;
    }
    __device__ __forceinline__ void load(const SliceGeom&, int bz, int by, bool lo, bool hi, float2& v0,
                                         float2& v1) const {
        const uint32_t i = base + (bz ? dz : 0u) + (by ? dy : 0u);
        v0 = lo ? __ldg(p + i) : make_float2(0.0f, 0.0f);
        v1 = hi ? __ldg(p + (i + dx)) : make_float2(0.0f, 0.0f);
    }
};

// Trilinear sample of the complex volume at corner set k; VT is float2 (plain
// layout), float4 (x-paired) or VoxBrick2 (bricked), with the same values and
// FMA order.
template <typename VT>
__device__ __forceinline__ float2 sample_trilinear(const VT* __restrict__ vol, const SliceGeom& g,
                                                   const Corners& k) {
    float2 r = make_float2(0.0f, 0.0f);
    const XRows<VT> rows(vol, g, k);
#pragma unroll
    for (int bz = 0; bz < 2; bz++) {
        if (bz && !k.zin) continue;
        const float wz = bz ? k.az1 : k.az0;
#pragma unroll
        for (int by = 0; by < 2; by++) {
            if (by && !k.yin) continue;
            const float wzy = (by ? k.ay1 : k.ay0) * wz;
            float2 v0, v1;
            rows.load(g, bz, by, true, k.xin, v0, v1);
            const float w0 = k.ax0 * wzy;
            r.x = fmaf(v0.x, w0, r.x);
            r.y = fmaf(v0.y, w0, r.y);
            if (k.xin) {
                const float w1 = k.ax1 * wzy;
                r.x = fmaf(v1.x, w1, r.x);
                r.y = fmaf(v1.y, w1, r.y);
            }
        }
    }
    return r;
}

// --------------------------------------------------------------------- CTF

// Per-image constants of the 2D CTF -sin(chi) of torch-ctf's calculate_ctf_2d
// (ctf_2d.py:12-131, ctf_utils.py:46-86, ctf_aberrations.py:42-81):
//   chi = k1 * s^2 * df(direction) + k2 * s^4 - phase_shift - atan(A / sqrt(1 - A^2))
//   k1 = -pi * lambda, k2 = pi / 2 * Cs * lambda^3 (Angstrom), s in cycles/Angstrom,
//   df = defocus - astig + 2 * (u . a)^2, u the unit frequency direction
//   (with float32 epsilon in its norm), a = sqrt(astig) * (sin theta, cos theta) (yx).
struct CtfConst {
    double k1, k2, phase;        // Angstrom units; phase includes the amplitude-contrast term
    double defocus, astig;       // micrometres (the astigmatism adjustment is done in um)
    double ay, ax;               // astigmatism vector sqrt(astig) * (sin, cos)
    double inv_px;               // 1 / pixel size (1/Angstrom)
};

// Constants of one image from its tt_ctf_params (double precision, once per image).
__host__ __device__ inline CtfConst make_ctf_const(const tt_ctf_params& p) {
    const double h = 6.62607015e-34, c = 299792458.0, m0 = 9.1093837015e-31, e = 1.602176634e-19;
    const double volts = (double)p.voltage_kv * 1e3;
    const double ev = e * volts;
    const double lambda = h * c / sqrt(ev * (2.0 * m0 * c * c + ev)) * 1e10;  // Angstrom
    const double pi = 3.14159265358979323846;
    const double cs = (double)p.spherical_aberration_mm * 1e7;
    const double ac = (double)p.amplitude_contrast;
    CtfConst k;
    k.k1 = -pi * lambda;
    k.k2 = pi / 2.0 * cs * lambda * lambda * lambda;
    k.phase = (double)p.phase_shift_deg * pi / 180.0 + atan(ac / sqrt(1.0 - ac * ac));
    k.defocus = p.defocus_um;
    k.astig = p.astigmatism_um;
    const double th = (double)p.astigmatism_angle_deg * pi / 180.0;
    const double sa = sqrt((double)(p.astigmatism_um > 0 ? p.astigmatism_um : 0.0f));
    k.ay = sa * sin(th);
    k.ax = sa * cos(th);
    k.inv_px = 1.0 / (double)p.pixel_size_a;
    return k;
}

// CTF at slice frequency (qy, qx) in cycles/pixel.  The phase reaches hundreds
// of radians at high frequency, so it is evaluated in double.
__device__ __forceinline__ float ctf_value(const CtfConst& k, float qy, float qx) {
    const double y = (double)qy * k.inv_px, x = (double)qx * k.inv_px;
    const double s2 = y * y + x * x;
    const double inv = 1.0 / sqrt(s2 + 1.1920928955078125e-07);  // torch.finfo(float32).eps
    const double dot = (y * inv) * k.ay + (x * inv) * k.ax;
    const double df = (k.defocus - k.astig + 2.0 * dot * dot) * 1e4;  // um -> Angstrom
    const double chi = k.k1 * s2 * df + k.k2 * s2 * s2 - k.phase;
    // the phase is reduced to [-pi, pi] in double (error ~1e-12 at a few
    // thousand radians); the float sine of the reduced phase is then accurate
    // to ~1e-7, as the float result, at a fraction of a double sine's cost
    const double two_pi = 6.283185307179586;
    const double red = chi - two_pi * rint(chi * (1.0 / two_pi));
    return -sinf((float)red);
}

// ---------------------------------------------------------------- insertion

template <typename R>
struct Acc;
template <>
struct Acc<float> {
    using T = float4;
    using C = float2;
};
template <>
struct Acc<double> {
    using T = double4;
    using C = double2;
};

__device__ __forceinline__ void acc_add(float4* a, float re, float im, float w) {
    atomicAdd(a, make_float4(re, im, w, 0.0f));
}
__device__ __forceinline__ void acc_add(double4* a, double re, double im, double w) {
    atomicAdd(&a->x, re);
    atomicAdd(&a->y, im);
    atomicAdd(&a->z, w);
}

__device__ __forceinline__ float2 load_slice(const float2* p) { return __ldcs(p); }
__device__ __forceinline__ double2 load_slice(const double2* p) { return __ldcs(p); }

// Float accumulation target: one (re, im, w, 0) vector reduction per corner.
template <typename R>
struct FloatSplat {
    typename Acc<R>::T* acc;
    __device__ __forceinline__ void operator()(int64_t vi, R dre, R dim, R w, R wscale) const {
        acc_add(acc + vi, dre * w, dim * w, w * wscale);
    }
};

// Source pixels the insertion skips: outside fftfreq_max, and the
// Friedel-redundant half of the x = 0 column (x == 0, y < 0).
__device__ __forceinline__ bool insert_pixel_kept(const SliceGeom& g, float qy, float qx) {
    return in_fmax(g, qy, qx) && !(qx == 0.0f && qy < 0.0f);
}

// Floor / ceil cell of an insertion point and its fractional offsets.
struct InsertCell {
    int iz0, iy0, ix0, iz1, iy1, ix1;
    float tz, ty, tx;
};

// Insertion geometry of slice frequency (qy, qx): rotation, the strict x' < 0
// redirect (cj), array coordinates c and the whole-point bounds test.
__device__ __forceinline__ bool insert_coords(const SliceGeom& g, const float* m, float qy, float qx, bool& cj,
                                              float c[3]) {
    float p[3];
    rotate_slice_point(m, qy, qx, p);
    cj = p[2] < 0.0f;
    if (cj) {
        p[0] = -p[0];
        p[1] = -p[1];
        p[2] = -p[2];
    }
    to_dft_coords(g, p, c);
    return inside_volume(g, c);
}

// insert_coords with the row part of the geometry precomputed (slice_row_geom):
// the same operations and roundings.
__device__ __forceinline__ bool insert_coords_row(const SliceGeom& g, const float* m, const SliceRow& row, float qx,
                                                  bool& cj, float c[3]) {
    float p[3];
#pragma unroll
    for (int i = 0; i < 3; i++) p[i] = __fadd_rn(row.my[i], __fmul_rn(m[i * 3 + 2], qx));
    cj = p[2] < 0.0f;
    if (cj) {
        p[0] = -p[0];
        p[1] = -p[1];
        p[2] = -p[2];
    }
    to_dft_coords(g, p, c);
    return inside_volume(g, c);
}

// Floor / ceil cell of inside array coordinates c.
__device__ __forceinline__ void cell_at(const float c[3], InsertCell& k) {
    const float z0 = floorf(c[0]), y0 = floorf(c[1]), x0 = floorf(c[2]);
    k.tz = c[0] - z0;
    k.ty = c[1] - y0;
    k.tx = c[2] - x0;
    k.iz0 = (int)z0;
    k.iy0 = (int)y0;
    k.ix0 = (int)x0;
    k.iz1 = (int)ceilf(c[0]);
    k.iy1 = (int)ceilf(c[1]);
    k.ix1 = (int)ceilf(c[2]);
}

// z-phase of an insertion tile: the accumulator of a large volume is filled
// in nphase passes, pass k taking the tiles whose centre point (after the
// x' < 0 redirect) lies in the k-th z-slab, so each pass reduces into about
// 1/nphase of the accumulator and more of its lines stay in L2.  Only the
// order of the work changes: every tile belongs to exactly one pass.
// (cy, cx): the tile's centre pixel.
__device__ __forceinline__ int insert_tile_phase(const SliceGeom& g, const float* m, int cy, int cx, int nphase) {
    const float qy = shifted_freq(cy, g.img_h, g.inv_h);
    const float qx = __fmul_rn((float)cx, g.inv_w);
    float p[3];
    rotate_slice_point(m, qy, qx, p);
    const float z = p[2] < 0.0f ? -p[0] : p[0];
    const int ph = (int)floorf((z + 0.5f) * (float)nphase);
    return ph < 0 ? 0 : (ph >= nphase ? nphase - 1 : ph);
}

// Insertion geometry and cell of slice frequency (qy, qx); false when the
// point is outside the volume.
__device__ __forceinline__ bool insert_cell(const SliceGeom& g, const float* m, float qy, float qx, bool& cj,
                                            InsertCell& k) {
    float c[3];
    if (!insert_coords(g, m, qy, qx, cj, c)) return false;
    cell_at(c, k);
    return true;
}

// Weight of corner `corner` (bit 2: z, bit 1: y, bit 0: x high) with the
// reference's float32 products, left to right.
__device__ __forceinline__ float insert_corner_weight(const InsertCell& k, int corner) {
    const int bz = (corner >> 2) & 1, by = (corner >> 1) & 1, bx = corner & 1;
    const float fz = bz ? k.tz : 1.0f - k.tz;
    const float fy = by ? k.ty : 1.0f - k.ty;
    const float fx = bx ? k.tx : 1.0f - k.tx;
    return (fz * fy) * fx;
}

__device__ __forceinline__ void insert_corner_zyx(const InsertCell& k, int corner, int& z, int& y, int& x) {
    z = (corner & 4) ? k.iz1 : k.iz0;
    y = (corner & 2) ? k.iy1 : k.iy0;
    x = (corner & 1) ? k.ix1 : k.ix0;
}

// Splat of one source pixel, following _insert_central_slices_rfft_3d.py:30-85
// and _insert_into_3d_dft_linear :289-346: each of the eight corners receives
// (data * w, w) through sink(voxel, re, im, w, weight scale).  With a CTF
// (ctf != nullptr) the data are weighted by the CTF and the interpolation
// weights by its square.
template <typename R, typename Sink>
__device__ __forceinline__ void insert_point_to(const typename Acc<R>::C* __restrict__ img, const float* m,
                                                const Sink& sink, const SliceGeom& g, int64_t s, int iy, int ix,
                                                const CtfConst* ctf = nullptr) {
    const float qy = shifted_freq(iy, g.img_h, g.inv_h);
    const float qx = __fmul_rn((float)ix, g.inv_w);
    if (!insert_pixel_kept(g, qy, qx)) return;
    // issued before the geometry so the load overlaps it
    const typename Acc<R>::C d = load_slice(img + (s * g.slice_rows + slice_row(g, iy)) * (int64_t)g.wr + ix);
    bool cj;
    InsertCell k;
    if (!insert_cell(g, m, qy, qx, cj, k)) return;
    R dre = d.x, dim = d.y, wscale = (R)1;
    if (ctf) {
        const float cv = ctf_value(*ctf, qy, qx);
        dre *= (R)cv;
        dim *= (R)cv;
        wscale = (R)(cv * cv);
    }
    if (cj) dim = -dim;
#pragma unroll
    for (int corner = 0; corner < 8; corner++) {
        const float w = insert_corner_weight(k, corner);
        if (w == 0.0f) continue;  // adds nothing (ceil == floor or zero fraction)
        int z, y, x;
        insert_corner_zyx(k, corner, z, y, x);
        sink(vox_index(g, z, y, x), dre, dim, (R)w, wscale);
    }
}

// Slot of voxel (z, y, x) (fftshifted) in a 2 x 2 x 2-bricked accumulator:
// bricks of 8 float4 slots (one 128-byte line) in (z, y, x) brick order, x
// fastest inside a brick; dims padded to even.
__device__ __forceinline__ int64_t accumulator_slot(const SliceGeom& g, int z, int y, int x) {
    const int64_t bh = (g.H + 1) >> 1, bw = (g.W + 1) >> 1;
    return ((((int64_t)(z >> 1) * bh + (y >> 1)) * bw + (x >> 1)) << 3) + ((z & 1) << 2) + ((y & 1) << 1) +
           (x & 1);
}

// The value a float splat adds for source pixel (iy, ix) of slice s: the
// (CTF-weighted, redirect-conjugated) data, the weight scale and the array
// coordinates c, with c[0] = -1 where the pixel adds nothing (no pixel,
// outside fftfreq_max, the redundant half of the x = 0 column, or a point
// outside the volume).
__device__ __forceinline__ void splat_source(const float2* __restrict__ img, const float* m, const SliceGeom& g,
                                             int64_t s, bool has_pixel, int iy, int ix, const CtfConst* ctf,
                                             float& dre, float& dim, float& wscale, float c[3]) {
    dre = 0.f;
    dim = 0.f;
    wscale = 1.f;
    c[0] = -1.f;
    c[1] = 0.f;
    c[2] = 0.f;
    if (!has_pixel) return;
    const float qy = shifted_freq(iy, g.img_h, g.inv_h);
    const float qx = __fmul_rn((float)ix, g.inv_w);
    if (!insert_pixel_kept(g, qy, qx)) return;
    const float2 d = load_slice(img + (s * g.slice_rows + slice_row(g, iy)) * (int64_t)g.wr + ix);
    bool cj;
    float ci[3];
    if (!insert_coords(g, m, qy, qx, cj, ci)) return;
    dre = d.x;
    dim = cj ? -d.y : d.y;
    if (ctf) {
        const float cv = ctf_value(*ctf, qy, qx);
        dre *= cv;
        dim *= cv;
        wscale = cv * cv;
    }
    c[0] = ci[0];
    c[1] = ci[1];
    c[2] = ci[2];
}

// Float splat of one source pixel with x-paired lanes into the plain
// accumulator: lanes 2j and 2j+1 reduce the x-low and the x-high corner of
// the same pixel in the same instruction (adjacent voxels, usually one
// 32-byte L2 sector), serving pixels j and j + 16 in two rounds.  Only the
// pixel's value (and CTF weight) and its three array coordinates move by warp
// shuffles; each lane rebuilds the floor / ceil cell from them.  Same pixels,
// corners, weights ((fz * fy) * fx), CTF weighting and values as
// insert_point.  Must be called by all 32 lanes of the warp (has_pixel false
// where the tile overhangs the slice).
__device__ __forceinline__ void insert_point_paired(const float2* __restrict__ img, const float* m,
                                                    float4* __restrict__ acc, const SliceGeom& g, int64_t s,
                                                    bool has_pixel, int iy, int ix, const CtfConst* ctf = nullptr) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, bx = lane & 1;
    float dre, dim, wscale, c[3];
    splat_source(img, m, g, s, has_pixel, iy, ix, ctf, dre, dim, wscale, c);
#pragma unroll
    for (int half = 0; half < 2; half++) {
        const int src = (lane >> 1) + 16 * half;
        // every lane runs every shuffle (full mask; ctf is the same for the warp)
        const float sre = __shfl_sync(full, dre, src), sim = __shfl_sync(full, dim, src);
        const float sws = ctf ? __shfl_sync(full, wscale, src) : 1.0f;
        float sc[3];
#pragma unroll
        for (int a = 0; a < 3; a++) sc[a] = __shfl_sync(full, c[a], src);
        if (sc[0] < 0.0f) continue;
        InsertCell k;
        cell_at(sc, k);
        const int x = bx ? k.ix1 : k.ix0;
        const float fx = bx ? k.tx : 1.0f - k.tx;
#pragma unroll
        for (int zy = 0; zy < 4; zy++) {
            const int bz = zy >> 1, by = zy & 1;
            const float w = ((bz ? k.tz : 1.0f - k.tz) * (by ? k.ty : 1.0f - k.ty)) * fx;
            if (w != 0.0f) {
                const int z = bz ? k.iz1 : k.iz0, y = by ? k.iy1 : k.iy0;
                acc_add(acc + vox_index(g, z, y, x), sre * w, sim * w, w * sws);
            }
        }
    }
}

// Float splat of one source pixel into the 2 x 2 x 2-bricked accumulator
// (accumulator_slot) with lane octets: lanes 8j..8j+7 reduce the eight
// corners of one pixel in the same instruction (corner = lane & 7: bit 2 z,
// bit 1 y, bit 0 x high), four neighbouring pixels of the warp per
// instruction in eight rounds.  A cell's corners fall on (1.5)^3 128-byte
// lines on average, which the L2 takes as one request each, against 1.5 lines
// for each of the four x-paired rows (256^3 x 4096: 3.65 vs 3.82 ms).  Same
// pixels, corners, weights and values as insert_point_paired; all 32 lanes
// call it.
__device__ __forceinline__ void insert_point_octet(const float2* __restrict__ img, const float* m,
                                                   float4* __restrict__ acc, const SliceGeom& g, int64_t s,
                                                   bool has_pixel, int iy, int ix, const CtfConst* ctf = nullptr) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, corner = lane & 7;
    const int bz = corner >> 2, by = (corner >> 1) & 1, bx = corner & 1;
    float dre, dim, wscale, c[3];
    splat_source(img, m, g, s, has_pixel, iy, ix, ctf, dre, dim, wscale, c);
#pragma unroll
    for (int r = 0; r < 8; r++) {
        const int src = 4 * r + (lane >> 3);
        const float sre = __shfl_sync(full, dre, src), sim = __shfl_sync(full, dim, src);
        const float sws = ctf ? __shfl_sync(full, wscale, src) : 1.0f;
        float sc[3];
#pragma unroll
        for (int a = 0; a < 3; a++) sc[a] = __shfl_sync(full, c[a], src);
        if (sc[0] < 0.0f) continue;
        InsertCell k;
        cell_at(sc, k);
        const float w = ((bz ? k.tz : 1.0f - k.tz) * (by ? k.ty : 1.0f - k.ty)) * (bx ? k.tx : 1.0f - k.tx);
        if (w != 0.0f) {
            const int z = bz ? k.iz1 : k.iz0, y = by ? k.iy1 : k.iy0, x = bx ? k.ix1 : k.ix0;
            acc_add(acc + accumulator_slot(g, z, y, x), sre * w, sim * w, w * sws);
        }
    }
}

// dL/dacc at voxel (z, y, x) for upstream dL/dvolume G: the adjoint of the
// Friedel completion, G[v] + conj(G[m v]) on the x = 0 plane unless v is DC.
template <typename R>
__device__ __forceinline__ typename Acc<R>::C completed_grad(const typename Acc<R>::C* __restrict__ gvol,
                                                            const SliceGeom& g, int z, int y, int x) {
    typename Acc<R>::C a = gvol[vox_index(g, z, y, x)];
    if (x == 0 && !(z == g.D / 2 && y == g.H / 2)) {
        const typename Acc<R>::C b = gvol[vox_index(g, (g.D - z) % g.D, (g.H - y) % g.H, 0)];
        a.x += b.x;
        a.y -= b.y;
    }
    return a;
}

// Splat into the float (re, im, w, 0) accumulator.
template <typename R>
__device__ __forceinline__ void insert_point(const typename Acc<R>::C* __restrict__ img, const float* m,
                                             typename Acc<R>::T* __restrict__ acc, const SliceGeom& g, int64_t s,
                                             int iy, int ix, const CtfConst* ctf = nullptr) {
    insert_point_to<R>(img, m, FloatSplat<R>{acc}, g, s, iy, ix, ctf);
}

}  // namespace tt
