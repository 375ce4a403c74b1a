// Device-side geometry shared by every Fourier-slice kernel.
//
// The arithmetic mirrors the reference's float32 CPU evaluation order so that
// the conjugate / inside / Friedel masks come out bit-identical:
//   * slice frequencies: f32(k) * f32(1/n)  (torch.fft.fftfreq / rfftfreq)
//   * rotation:          ((r0*q0 + r1*q1) + r2*q2), each product rounded, no FMA
//                        (torch CPU matmul for (...,1,3,3) @ (b,3,1))
//   * array coordinates: ((p + 0.5) / (1 - 1/n)) * (n - 1) for z and y,
//                        (p * 2) * (w/2 + 1 - 1) for x
//                        (torch_fourier_slice/_dft_utils.py:37-72)
// __fmul_rn / __fadd_rn / __fdiv_rn keep nvcc from contracting into FMAs.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/teamtomo_b200.h"

namespace tt {

// Launch-constant geometry of one batch of central slices.
struct SliceGeom {
    int n;          // number of slices
    int img_h, wr;  // slice grid rows and rfft columns (h, w/2+1)
    float inv_h, inv_w;            // f32(1/h), f32(1/w)
    float iw0, iw1, s0, s1, sx;    // coordinate scaling of the image/volume shape
    int D, H, W;                   // rfft volume dims (d, h, w/2+1)
    float ub0, ub1, ub2;           // D-1, H-1, W-1 as float
    int has_fmax;
    float fmax;
    int zyx;
    float x_tol, x_tol10;
    int has_rot_tol;
    float rot_tol;
    int rot_f64;                   // rotation matrices are float64
    int vol_unshifted;             // volume is the plain rfftn output (no fftshift of z, y)
    int slice_unshifted;           // slices are stored ifftshifted along rows (irfft-ready)
    int vol_layout;                // TT_VOLUME_PLAIN / _XPAIRS / _BRICKS (tt_slice_params.volume_layout)
    int slice_rows;                // storage rows per slice of the insertion's images
                                   // (img_h; channels * img_h for channel-interleaved stacks)
    float dcdp0, dcdp1, dcdp2;     // d(array coord)/d(frequency) per axis
};

__host__ inline SliceGeom make_geom(const tt_slice_params& p) {
    SliceGeom g;
    g.n = (int)p.n;
    g.img_h = (int)p.img_h;
    g.wr = (int)(p.img_w / 2 + 1);
    g.inv_h = (float)(1.0 / (double)p.img_h);
    g.inv_w = (float)(1.0 / (double)p.img_w);
    float fd = (float)p.img_d, fh = (float)p.img_h, fwr = (float)(p.img_w / 2 + 1);
    // host float32 arithmetic: same rounding as the device
    volatile float dd = 1.0f / fd, dh = 1.0f / fh;
    g.iw0 = 1.0f - dd;
    g.iw1 = 1.0f - dh;
    g.s0 = fd - 1.0f;
    g.s1 = fh - 1.0f;
    g.sx = fwr - 1.0f;
    g.D = (int)p.vol_d;
    g.H = (int)p.vol_h;
    g.W = (int)p.vol_w;
    g.ub0 = (float)(p.vol_d - 1);
    g.ub1 = (float)(p.vol_h - 1);
    g.ub2 = (float)(p.vol_w - 1);
    g.has_fmax = p.has_fftfreq_max;
    g.fmax = p.fftfreq_max;
    g.zyx = p.zyx_matrices;
    g.x_tol = p.x_tolerance;
    g.x_tol10 = p.x_tolerance10;
    g.has_rot_tol = p.has_rot_tolerance;
    g.rot_tol = p.rot_tolerance;
    g.rot_f64 = p.rotation_f64;
    g.vol_unshifted = p.volume_unshifted;
    g.slice_unshifted = p.slices_unshifted;
    g.vol_layout = p.volume_layout;
    g.slice_rows = (int)p.img_h;
    g.dcdp0 = g.s0 / g.iw0;
    g.dcdp1 = g.s1 / g.iw1;
    g.dcdp2 = 2.0f * g.sx;
    return g;
}

// Frequency of row i of an fftshifted axis of length n (torch.fft.fftshift
// rolls by n//2, so row i holds unshifted index (i - n//2) mod n).
__device__ __forceinline__ float shifted_freq(int i, int n, float inv_n) {
    int k = i - n / 2;
    if (k < 0) k += n;
    int kk = (k < (n + 1) / 2) ? k : k - n;
    return __fmul_rn((float)kk, inv_n);
}

// Rotation prep for one slice: float32 cast, optional tolerance zeroing of the
// caller's (xyz) matrix, then the xyz -> zyx flip (both axes reversed).
// Thread t < 9 produces element t of the zyx matrix.
__device__ __forceinline__ float prep_rotation_elem(const void* rot, int rot_f64, int64_t slice,
                                                    int t, const SliceGeom& g, bool apply_tol) {
    int src = g.zyx ? t : 8 - t;
    float v = rot_f64 ? __double2float_rn(((const double*)rot)[slice * 9 + src])
                      : ((const float*)rot)[slice * 9 + src];
    if (apply_tol && g.has_rot_tol && fabsf(v) < g.rot_tol) v = 0.0f;
    return v;
}

// p = M q for q = (0, qy, qx): ((m0*0 + m1*qy) + m2*qx).  The zero term only
// affects the sign of a zero result, which no mask or coordinate depends on.
__device__ __forceinline__ void rotate_slice_point(const float* m, float qy, float qx, float p[3]) {
#pragma unroll
    for (int i = 0; i < 3; i++) p[i] = __fadd_rn(__fmul_rn(m[i * 3 + 1], qy), __fmul_rn(m[i * 3 + 2], qx));
}

__device__ __forceinline__ void to_dft_coords(const SliceGeom& g, const float p[3], float c[3]) {
    c[0] = __fmul_rn(__fdiv_rn(__fadd_rn(p[0], 0.5f), g.iw0), g.s0);
    c[1] = __fmul_rn(__fdiv_rn(__fadd_rn(p[1], 0.5f), g.iw1), g.s1);
    c[2] = __fmul_rn(__fmul_rn(p[2], 2.0f), g.sx);
}

// fftfreq_max disc test of the slice grid (|f| <= fmax, f32 sqrt).
__device__ __forceinline__ bool in_fmax(const SliceGeom& g, float qy, float qx) {
    if (!g.has_fmax) return true;
    float nrm = __fsqrt_rn(__fadd_rn(__fmul_rn(qy, qy), __fmul_rn(qx, qx)));
    return nrm <= g.fmax;
}

// Extraction conjugate rule (_extract_central_slices_rfft_3d.py:193-201 and
// _determine_near_zero_conjugate_mask :9-81).
__device__ __forceinline__ bool extract_conj(const SliceGeom& g, const float* m, float px) {
    bool cj = px < -g.x_tol;
    if (fabsf(px) < g.x_tol) {
        float r11 = m[8], r12 = m[7];
        cj = (fabsf(r11) <= g.x_tol10) ? (r12 < 0.0f) : (r11 < 0.0f);
    }
    return cj;
}

__device__ __forceinline__ bool inside_volume(const SliceGeom& g, const float c[3]) {
    return c[0] >= 0.0f && c[0] <= g.ub0 && c[1] >= 0.0f && c[1] <= g.ub1 && c[2] >= 0.0f &&
           c[2] <= g.ub2;
}

// Linear index of volume voxel (z, y, x) given in fftshifted coordinates.
__device__ __forceinline__ int64_t vox_index(const SliceGeom& g, int z, int y, int x) {
    if (g.vol_unshifted) {
        z -= g.D / 2;
        if (z < 0) z += g.D;
        y -= g.H / 2;
        if (y < 0) y += g.H;
    }
    return ((int64_t)z * g.H + y) * g.W + x;
}

// Storage row of slice row iy (fftshifted order) for the slice layout in use.
__device__ __forceinline__ int slice_row(const SliceGeom& g, int iy) {
    if (!g.slice_unshifted) return iy;
    int r = iy - g.img_h / 2;
    return r < 0 ? r + g.img_h : r;
}

// Slice pixels are processed in 8 (x) x 32 (y) tiles of 256 threads; each warp
// takes an 8 x 4 patch so that its 32 points, and their volume corners, stay
// close together (fewer cache lines per warp-wide gather or reduction).
constexpr int kTileX = 8, kTileY = 32, kTileThreads = kTileX * kTileY;

__host__ __device__ inline int tiles_x_of(int wr) { return (wr + kTileX - 1) / kTileX; }
__host__ __device__ inline int tiles_per_slice(int img_h, int wr) {
    return tiles_x_of(wr) * ((img_h + kTileY - 1) / kTileY);
}

// Pixel (iy, ix) of this thread in tile `tile` of a slice; false when the
// tile overhangs the slice.
__device__ __forceinline__ bool tile_pixel(const SliceGeom& g, int tile, int& iy, int& ix) {
    const int tx_tiles = tiles_x_of(g.wr);
    const int ty = tile / tx_tiles, tx = tile - ty * tx_tiles;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    ix = tx * kTileX + (lane & 7);
    iy = ty * kTileY + warp * 4 + (lane >> 3);
    return ix < g.wr && iy < g.img_h;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Warp totals of eight values per lane by recursive halving (9 shuffles
// instead of 8 x 5): at each step a lane keeps half of its values and adds
// the partner's copy of that half.  Lane l returns the total of value l >> 2.
__device__ __forceinline__ float warp_reduce8(const float v[8]) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
    float a[4], b[2];
#pragma unroll
    for (int i = 0; i < 4; i++)
        a[i] = (h16 ? v[i + 4] : v[i]) + __shfl_xor_sync(full, h16 ? v[i] : v[i + 4], 16);
#pragma unroll
    for (int i = 0; i < 2; i++)
        b[i] = (h8 ? a[i + 2] : a[i]) + __shfl_xor_sync(full, h8 ? a[i] : a[i + 2], 8);
    float c = (h4 ? b[1] : b[0]) + __shfl_xor_sync(full, h4 ? b[0] : b[1], 4);
    c += __shfl_xor_sync(full, c, 2);
    c += __shfl_xor_sync(full, c, 1);
    return c;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace tt
