// Central-slice extraction from an fftshifted rfft volume, and its backward.
//
// Forward (extract_central_slices_rfft_3d, _extract_central_slices_rfft_3d.py:84-222):
// one thread per slice pixel of an 8 x 32 tile, one block per row of tiles of
// a slice.  The pixel's
// frequency is generated in registers, rotated with the reference's float32
// operation order, redirected into the stored half (conjugate rule with the
// x-tolerance tie-break), scaled to array coordinates and sampled trilinearly
// with grid_sample's semantics: padding_mode='border', align_corners=True, the
// array -> grid -> array round trip of the coordinate (it decides the cell at
// integer kinks, where the trilinear derivative jumps), zero outside [0, n-1].
//
// Backward: the same per-pixel geometry, recomputed rather than stored.
//   d/dvolume  = trilinear scatter of G' (G conjugated where the sample was)
//   d/drotation: per pixel Re(conj(G') dV/dc) chained through the coordinate
//                scale, the conjugate flip and the rotation, reduced per slice.
// Per-block partial sums of the rotation gradient go to the caller's
// workspace and are reduced in a fixed order by a second kernel, so the
// rotation gradient is deterministic.
#include <cuda_runtime.h>

#include <mutex>
#include <type_traits>

#include "capi_util.cuh"
#include "fixed_point.cuh"
#include "slice_common.cuh"
#include "slice_grad.cuh"
#include "slice_ops.cuh"

namespace tt {

constexpr int kExtractThreads = kTileThreads;

__device__ __forceinline__ void load_rotation(float* sm, const void* rot, int64_t s,
                                              const SliceGeom& g, bool apply_tol) {
    if (threadIdx.x < 9) sm[threadIdx.x] = prep_rotation_elem(rot, g.rot_f64, s, threadIdx.x, g, apply_tol);
}

// VT: float2 (plain volume), float4 (x-paired copy, tt_pack_volume_xpairs) or
// VoxBrick2 (bricked copy, tt_pack_volume_bricks).
// One block per (slice, row of tiles), eight resident blocks (32 registers):
// the gathers are latency-bound at six (64 % warps active); full occupancy
// takes 8.5 % off the launch, the row loop another 1 %.
// From the bricked copy the row of tiles is unrolled by four at six resident
// blocks (40 registers), so one thread's gathers of neighbouring tiles
// overlap: 256^3 x 4096 1.30 vs 1.32-1.35 ms, 128^3 0.386 vs 0.394 ms.
template <typename VT, int UNR = std::is_same<VT, VoxBrick2>::value ? 4 : 1>
__global__ void __launch_bounds__(kExtractThreads, UNR > 1 ? 6 : 8)
extract_fwd_kernel(const VT* __restrict__ vol, const void* __restrict__ rot,
                   float2* __restrict__ out, SliceGeom g, int tiles) {
    __shared__ float m[9];
    const int tx_tiles = tiles_x_of(g.wr);
    const int rows = tiles / tx_tiles;
    const int64_t s = blockIdx.x / rows;
    const int ty = blockIdx.x - (int)(s * rows);
    load_rotation(m, rot, s, g, true);
    __syncthreads();
    // this thread's pixels share one slice row across the row of tiles
    const int lane = threadIdx.x & 31;
    const int iy = ty * kTileY + (threadIdx.x >> 5) * 4 + (lane >> 3);
    if (iy >= g.img_h) return;
    const SliceRow row = slice_row_geom(g, m, iy);
    float2* orow = out + (s * g.img_h + slice_row(g, iy)) * (int64_t)g.wr;
#pragma unroll UNR
    for (int tx = 0; tx < tx_tiles; tx++) {
        const int ix = tx * kTileX + (lane & 7);
        if (ix >= g.wr) continue;
        float qx, c[3];
        bool cj = false;
        float2 r = make_float2(0.0f, 0.0f);
        if (extract_geometry_row(g, m, row, ix, qx, cj, c)) {
            r = sample_trilinear(vol, g, make_corners(g, c));
            if (cj) r.y = -r.y;
        }
        // streaming store: the slices are written once and should not evict the volume from L2
        __stcs(orow + ix, r);
    }
}

// Backward of one slice pixel; the pixel's 6 contributions to d/dR_zyx are
// added to acc.  Called by every lane of the warp (has_pixel false where the tile
// overhangs the slice): the float d/dvolume scatter pairs lanes across the warp.
template <bool WANT_DV, bool WANT_DR, bool FIXED, typename VT>
__device__ __forceinline__ void bwd_point(const VT* __restrict__ vol, const float* m,
                                          const float2* __restrict__ grad, const DvTarget<FIXED>& dv,
                                          const SliceGeom& g, int64_t s, bool has_pixel, int iy, int ix,
                                          float acc[6]) {
    float qy = 0.f, qx = 0.f, c[3];
    bool cj = false;
    const bool valid = has_pixel && extract_geometry(g, m, iy, ix, qy, qx, cj, c);
    Corners k{};
    SourceIdx si{};
    float2 gv = make_float2(0.f, 0.f);
    if (valid) {
        si = source_indices(g, c);
        k = corners_at(g, si.z, si.y, si.x);
        k.gz = si.gz;
        k.gy = si.gy;
        k.gx = si.gx;
        gv = __ldcs(grad + (s * g.img_h + slice_row(g, iy)) * (int64_t)g.wr + ix);
        if (cj) gv.y = -gv.y;  // G' = conj(G) where the sample was conjugated
    }
    // the rotation gradient first: its corner values are dead before the
    // scatter's shuffles and reductions, which then run without spills
    // (256^3 x 4096: 3.21 vs 3.52 ms with the scatter first)
    if (WANT_DR && valid) {
        float2 v[2][2][2];
        load_corners(vol, g, k, v);
        drot_terms(v, k, gv, cj, g, qy, qx, acc);
    }
    if (WANT_DV) {
        if (FIXED) {
            scatter_dv_fixed_paired(dv.fixed, dv.scale, g, si, gv, valid);
        } else {
            scatter_dv_paired(dv.dvol, g, si, gv, valid);
        }
    }
}

// Sample, residual and loss term of one pixel (mse_point); returns G'.
template <typename VT>
__device__ __forceinline__ float2 mse_residual(const VT* __restrict__ vol, const SliceGeom& g, const Corners& k,
                                               float2 t, bool cj, float scale, double& loss, float acc[6], float qy,
                                               float qx, bool want_dr) {
    float2 v[2][2][2];
    load_corners(vol, g, k, v);
    float2 sv = make_float2(0.f, 0.f);
#pragma unroll
    for (int bz = 0; bz < 2; bz++) {
        const float wz = bz ? k.az1 : k.az0;
#pragma unroll
        for (int by = 0; by < 2; by++) {
            const float wzy = (by ? k.ay1 : k.ay0) * wz;
            const float w0 = k.ax0 * wzy, w1 = k.ax1 * wzy;
            sv.x = fmaf(v[bz][by][0].x, w0, sv.x);
            sv.y = fmaf(v[bz][by][0].y, w0, sv.y);
            sv.x = fmaf(v[bz][by][1].x, w1, sv.x);
            sv.y = fmaf(v[bz][by][1].y, w1, sv.y);
        }
    }
    if (cj) sv.y = -sv.y;
    const float rx = sv.x - t.x, ry = sv.y - t.y;
    loss += (double)rx * rx + (double)ry * ry;
    float2 gv = make_float2(rx * scale, ry * scale);
    if (cj) gv.y = -gv.y;
    if (want_dr) drot_terms(v, k, gv, cj, g, qy, qx, acc);
    return gv;
}

// Fused extraction + squared-error loss + backward of one pixel: the sample S
// is rebuilt from the corner values the rotation gradient needs anyway (same
// operation order as extract_fwd_kernel), r = S - T, the loss term |r|^2, and
// G = scale * r (scale = 2 / M for the mean) feeds the two gradients.  Pixels
// whose sample is zero (outside fftfreq_max or the volume) add |T|^2 and no
// gradient.
// Called by every lane of the warp (the d/dvolume scatter pairs lanes).
template <bool WANT_DV, bool WANT_DR, typename VT>
__device__ __forceinline__ void mse_point(const VT* __restrict__ vol, const float* m,
                                          const float2* __restrict__ target, const DvTarget<false>& dv,
                                          const SliceGeom& g, int64_t s, bool has_pixel, int iy, int ix, float scale,
                                          float acc[6], double& loss) {
    float qy = 0.f, qx = 0.f, c[3];
    bool cj = false;
    bool valid = false;
    float2 gv = make_float2(0.f, 0.f);
    Corners k{};
    SourceIdx si{};
    if (has_pixel) {
        const float2 t = __ldcs(target + (s * g.img_h + slice_row(g, iy)) * (int64_t)g.wr + ix);
        valid = extract_geometry(g, m, iy, ix, qy, qx, cj, c);
        if (!valid) {
            loss += (double)t.x * t.x + (double)t.y * t.y;
        } else {
            si = source_indices(g, c);
            k = corners_at(g, si.z, si.y, si.x);
            k.gz = si.gz;
            k.gy = si.gy;
            k.gx = si.gx;
            gv = mse_residual(vol, g, k, t, cj, scale, loss, acc, qy, qx, WANT_DR);
        }
    }
    if (WANT_DV) scatter_dv_paired(dv.dvol, g, si, gv, valid);
}

// One block per (slice, row of tiles): the rotation is loaded and the
// rotation-gradient partials reduced once per row.  WANT_DR: the row's sums of
// the 6 non-zero entries of d/dR_zyx (per thread over its pixels, warp totals
// in float, then the eight warps in double, in a fixed order) go to
// part[(s * rows + row) * 6 + k], one slot per row of tiles.  FIXED:
// the volume gradient goes to the
// fixed-point words `fixed` at the scale set by *absmax and n.  Resident
// blocks: 6 for the rotation gradient alone (39 registers), 5 with the volume
// gradient (6 would spill into the L1 pipe that bounds it), 4 in fixed point.
template <bool WANT_DV, bool WANT_DR, bool FIXED, typename VT>
__global__ void __launch_bounds__(kExtractThreads, FIXED ? 4 : (WANT_DV ? 5 : 6))
extract_bwd_kernel(const VT* __restrict__ vol, const void* __restrict__ rot,
                   const float2* __restrict__ grad, float2* __restrict__ dvol,
                   unsigned long long* __restrict__ fixed, const uint32_t* __restrict__ absmax,
                   float* __restrict__ part, SliceGeom g, int tiles) {
    __shared__ float m[9];
    __shared__ double red[kExtractThreads / 32][6];
    const int tx_tiles = tiles_x_of(g.wr);
    const int rows = tiles / tx_tiles;
    const int64_t s = blockIdx.x / rows;
    const int ty = blockIdx.x - (int)(s * rows);
    load_rotation(m, rot, s, g, true);
    __syncthreads();
    float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    DvTarget<FIXED> dv{dvol, fixed, 0.0};
    if (FIXED) dv.scale = fixed_data_scale(*absmax, ceil_log2(g.n));
    for (int tx = 0; tx < tx_tiles; tx++) {  // every lane runs every tile (the paired scatter shuffles)
        int iy, ix;
        const bool has_pixel = tile_pixel(g, ty * tx_tiles + tx, iy, ix);
        bwd_point<WANT_DV, WANT_DR, FIXED, VT>(vol, m, grad, dv, g, s, has_pixel, iy, ix, acc);
    }
    if (WANT_DR) {
        // warp totals in float (fixed order), then the warps in double
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const float v8[8] = {acc[0], acc[1], acc[2], acc[3], acc[4], acc[5], 0.f, 0.f};
        const float t = warp_reduce8(v8);
        if ((lane & 3) == 0 && (lane >> 2) < 6) red[warp][lane >> 2] = (double)t;
        __syncthreads();
        if (threadIdx.x < 6) {
            double v = 0.0;
#pragma unroll
            for (int w = 0; w < kExtractThreads / 32; w++) v += red[w][threadIdx.x];
            part[((int64_t)s * rows + ty) * 6 + threadIdx.x] = (float)v;
        }
    }
}

// Fused extraction + mean squared error + backward: one block per (slice, row
// of tiles).  The row's partials of the loss (double) go to
// loss_part[s * rows + row] and, with WANT_DR, those of d/dR_zyx to
// part[(s * rows + row) * 6 + k]: one slot per row of tiles.
// Five resident blocks (48 registers); four for the rotation gradient alone,
// which spills at 48 (256^3 x 4096: 1.95 vs 2.19 ms at five).
template <bool WANT_DV, bool WANT_DR, typename VT>
__global__ void __launch_bounds__(kExtractThreads, (WANT_DR && !WANT_DV) ? 4 : 5)
slice_mse_kernel(const VT* __restrict__ vol, const void* __restrict__ rot, const float2* __restrict__ target,
                 float2* __restrict__ dvol, float* __restrict__ part, double* __restrict__ loss_part, float scale,
                 SliceGeom g, int tiles) {
    __shared__ float m[9];
    __shared__ double red[kExtractThreads / 32][7];
    const int tx_tiles = tiles_x_of(g.wr);
    const int rows = tiles / tx_tiles;
    const int64_t s = blockIdx.x / rows;
    const int ty = blockIdx.x - (int)(s * rows);
    load_rotation(m, rot, s, g, true);
    __syncthreads();
    float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    double loss = 0.0;
    const DvTarget<false> dv{dvol, nullptr, 0.0};
    for (int tx = 0; tx < tx_tiles; tx++) {  // every lane runs every tile (the paired scatter shuffles)
        int iy, ix;
        const bool has_pixel = tile_pixel(g, ty * tx_tiles + tx, iy, ix);
        mse_point<WANT_DV, WANT_DR, VT>(vol, m, target, dv, g, s, has_pixel, iy, ix, scale, acc, loss);
    }
    // rotation-gradient warp totals in float (fixed order), the loss in double
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float v8[8] = {acc[0], acc[1], acc[2], acc[3], acc[4], acc[5], 0.f, 0.f};
    const float t = warp_reduce8(v8);
    if ((lane & 3) == 0 && (lane >> 2) < 6) red[warp][lane >> 2] = (double)t;
    const double lw = warp_sum_d(loss);
    if (lane == 0) red[warp][6] = lw;
    __syncthreads();
    if (threadIdx.x < 7) {
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < kExtractThreads / 32; w++) v += red[w][threadIdx.x];
        const int64_t b0 = (int64_t)s * rows + ty;
        if (threadIdx.x == 6)
            loss_part[b0] = v;
        else if (WANT_DR)
            part[b0 * 6 + threadIdx.x] = (float)v;
    }
}

// loss = inv_m * sum of the block partials, summed in a fixed order by one block.
__global__ void __launch_bounds__(1024) mse_loss_finish_kernel(const double* __restrict__ loss_part, int64_t count,
                                                               double inv_m, float* __restrict__ loss) {
    __shared__ double red[32];
    double v = 0.0;
    for (int64_t i = threadIdx.x; i < count; i += blockDim.x) v += loss_part[i];
    v = warp_sum_d(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        v = warp_sum_d(v);
        if (threadIdx.x == 0) *loss = (float)(v * inv_m);
    }
}

// Sums the per-block partials of each slice in a fixed order and writes the
// caller-layout gradient: undo the xyz->zyx flip, zero the tolerance-zeroed
// elements, cast to the rotation dtype.  One thread per (slice, element).
__global__ void drot_finish_kernel(const float* __restrict__ part, const void* __restrict__ rot,
                                   void* __restrict__ drot, SliceGeom g, int parts) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)g.n * 9) return;
    const int64_t s = idx / 9;
    const int t = (int)(idx - s * 9);
    const int a = t / 3, b = t % 3;
    const int i = g.zyx ? a : 2 - a, j = g.zyx ? b : 2 - b;
    double v = 0.0;
    if (j != 0) {
        const float* ps = part + (int64_t)s * parts * 6 + i * 2 + (j - 1);
        for (int k = 0; k < parts; k++) v += (double)ps[(int64_t)k * 6];
    }
    float r = g.rot_f64 ? __double2float_rn(((const double*)rot)[idx]) : ((const float*)rot)[idx];
    if (g.has_rot_tol && fabsf(r) < g.rot_tol) v = 0.0;
    if (g.rot_f64)
        ((double*)drot)[idx] = (double)(float)v;
    else
        ((float*)drot)[idx] = (float)v;
}

// Per-pixel geometry of the extraction (mode 0) or insertion (mode 1) rule,
// exported for bit-exact checks of the index / mask logic.
// flags: bit0 inside fftfreq_max (and, for insertion, not the Friedel-
// redundant x==0,y<0 source pixel), bit1 conjugated, bit2 inside the volume.
__global__ void slice_geometry_kernel(const void* __restrict__ rot, uint8_t* __restrict__ flags,
                                      float* __restrict__ coords, SliceGeom g, int tiles, int mode) {
    __shared__ float m[9];
    const int64_t s = blockIdx.x / tiles;
    const int tile = blockIdx.x - (int)(s * tiles);
    load_rotation(m, rot, s, g, mode == 0);
    __syncthreads();
    int iy, ix;
    if (!tile_pixel(g, tile, iy, ix)) return;
    const float qy = shifted_freq(iy, g.img_h, g.inv_h);
    const float qx = __fmul_rn((float)ix, g.inv_w);
    const int64_t o = (s * g.img_h + iy) * (int64_t)g.wr + ix;
    uint8_t f = 0;
    float c[3] = {0.f, 0.f, 0.f};
    bool valid = in_fmax(g, qy, qx);
    if (mode == 1 && qx == 0.0f && qy < 0.0f) valid = false;
    if (valid) {
        float p[3];
        rotate_slice_point(m, qy, qx, p);
        const bool cj = mode == 0 ? extract_conj(g, m, p[2]) : (p[2] < 0.0f);
        if (cj) {
            p[0] = -p[0];
            p[1] = -p[1];
            p[2] = -p[2];
        }
        to_dft_coords(g, p, c);
        f = 1 | (cj ? 2 : 0) | (inside_volume(g, c) ? 4 : 0);
    }
    flags[o] = f;
    coords[o * 3 + 0] = c[0];
    coords[o * 3 + 1] = c[1];
    coords[o * 3 + 2] = c[2];
}

static int extract_tiles(const SliceGeom& g) { return tiles_per_slice(g.img_h, g.wr); }

// grad_volume += the fixed-point volume gradient, converted back once.
__global__ void dv_fixed_add_kernel(const long long* __restrict__ fixed, float2* __restrict__ dvol,
                                    const uint32_t* __restrict__ absmax, int slices_log2, int64_t voxels) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= voxels) return;
    const double inv = 1.0 / fixed_data_scale(*absmax, slices_log2);
    const longlong2 q = reinterpret_cast<const longlong2*>(fixed)[i];
    float2 o = dvol[i];
    o.x += (float)((double)q.x * inv);
    o.y += (float)((double)q.y * inv);
    dvol[i] = o;
}

// Rotation-gradient partials: `parts` slots of 6 floats per slice (one per
// row of tiles for the single-channel kernels, one per tile for the
// multichannel ones).
static size_t partial_bytes(int64_t n, int parts) { return (size_t)(n * parts * 6) * sizeof(float); }

// Rows of tiles per slice: the single-channel kernels' blocks and partial slots.
static int tile_rows(int img_h) { return (img_h + kTileY - 1) / kTileY; }

int launch_drot_finish(const float* part, const void* rot, void* drot, const SliceGeom& g, int parts,
                       cudaStream_t st) {
    const int64_t total = (int64_t)g.n * 9;
    drot_finish_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(part, rot, drot, g, parts);
    return check_launch("drot_finish_kernel");
}

// Fixed-point volume gradient of the deterministic mode: 256-byte header
// (absmax word) + 2 words per voxel, ahead of the rotation partials.
static size_t fixed_dv_bytes(const tt_slice_params* p) {
    return p->deterministic ? kFixedHeaderBytes + (size_t)(p->vol_d * p->vol_h * p->vol_w) * 16 : 0;
}

// Launches the backward and the rotation-gradient reduction; `part` holds
// 6 floats per row of tiles when grad_rotation is set; `fixed` (deterministic
// volume gradient) is the zeroed header + accumulator of fixed_dv_bytes.
template <typename VT>
static int launch_backward_t(const VT* v, const void* rot, const float2* gr, float2* dv, void* grad_rotation,
                             float* part, const SliceGeom& g, cudaStream_t st, void* fixed) {
    const int tiles = extract_tiles(g);
    const unsigned blocks = (unsigned)((int64_t)g.n * (tiles / tiles_x_of(g.wr)));  // one block per row of tiles
    uint32_t* absmax = (uint32_t*)fixed;
    unsigned long long* facc = fixed ? (unsigned long long*)((char*)fixed + kFixedHeaderBytes) : nullptr;
    if (dv && fixed) {
        if (int e = launch_fixed_absmax(gr, 0, (int64_t)g.n * g.img_h * g.wr * 2, absmax, st)) return e;
        if (grad_rotation)
            extract_bwd_kernel<true, true, true, VT><<<blocks, kExtractThreads, 0, st>>>(v, rot, gr, dv, facc, absmax,
                                                                                    part, g, tiles);
        else
            extract_bwd_kernel<true, false, true, VT><<<blocks, kExtractThreads, 0, st>>>(v, rot, gr, dv, facc, absmax,
                                                                                     part, g, tiles);
        if (int e = check_launch("extract_bwd_kernel")) return e;
        const int64_t vox = (int64_t)g.D * g.H * g.W;
        dv_fixed_add_kernel<<<(unsigned)((vox + 255) / 256), 256, 0, st>>>((const long long*)facc, dv, absmax,
                                                                           ceil_log2(g.n), vox);
    } else if (dv && grad_rotation) {
        extract_bwd_kernel<true, true, false, VT><<<blocks, kExtractThreads, 0, st>>>(v, rot, gr, dv, nullptr, nullptr,
                                                                                 part, g, tiles);
    } else if (dv) {
        extract_bwd_kernel<true, false, false, VT><<<blocks, kExtractThreads, 0, st>>>(v, rot, gr, dv, nullptr, nullptr,
                                                                                  part, g, tiles);
    } else {
        extract_bwd_kernel<false, true, false, VT><<<blocks, kExtractThreads, 0, st>>>(v, rot, gr, dv, nullptr, nullptr,
                                                                                  part, g, tiles);
    }
    if (int e = check_launch("extract_bwd_kernel")) return e;
    if (grad_rotation)
        if (int e = launch_drot_finish(part, rot, grad_rotation, g, tile_rows(g.img_h), st)) return e;
    return TT_OK;
}

// `v` is the plain complex64 volume or the copy g.vol_layout names.
static int launch_backward(const void* v, const void* rot, const float2* gr, float2* dv, void* grad_rotation,
                           float* part, const SliceGeom& g, cudaStream_t st, void* fixed = nullptr) {
    switch (g.vol_layout) {
        case TT_VOLUME_XPAIRS:
            return launch_backward_t((const float4*)v, rot, gr, dv, grad_rotation, part, g, st, fixed);
        case TT_VOLUME_BRICKS:
            return launch_backward_t((const VoxBrick2*)v, rot, gr, dv, grad_rotation, part, g, st, fixed);
        default:
            return launch_backward_t((const float2*)v, rot, gr, dv, grad_rotation, part, g, st, fixed);
    }
}

// Bricked copy: voxel (z, y, x), in fftshifted (z, y) order whatever the
// source's, sits in 2 x 2 x 2 brick ((z/2 * ceil(H/2) + y/2) * ceil(W/2) + x/2)
// at slot (z&1)*4 + (y&1)*2 + (x&1): eight complex64 voxels, 64 bytes, two
// x-adjacent bricks per 128-byte line.  One thread per destination slot (a
// warp writes four whole bricks, 256 contiguous bytes), reading the source
// voxel (an unshifted source remapped by vox_index) or zero for the slots
// past an odd dimension.  Grid-stride over the slots.
__global__ void pack_bricks_kernel(const float2* __restrict__ vol, float2* __restrict__ bricks, SliceGeom g,
                                   int64_t slots) {
    const int bh = (g.H + 1) >> 1, bw = (g.W + 1) >> 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < slots;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = i >> 3;
        const int s = (int)(i & 7);
        const int bx = (int)(b % bw);
        const int64_t bzy = b / bw;
        const int by = (int)(bzy % bh), bz = (int)(bzy / bh);
        const int z = 2 * bz + (s >> 2), y = 2 * by + ((s >> 1) & 1), x = 2 * bx + (s & 1);
        bricks[i] = (z < g.D && y < g.H && x < g.W) ? vol[vox_index(g, z, y, x)] : make_float2(0.0f, 0.0f);
    }
}

// x-paired copy: xp[r * W + x] = (vol[r * W + x], vol[r * W + x + 1]), zero
// past the last column.  Threads run along x (coalesced), rows in a grid-stride loop.
__global__ void pack_xpairs_kernel(const float2* __restrict__ vol, float4* __restrict__ xp, int64_t rows, int W) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= W) return;
    for (int64_t r = (int64_t)blockIdx.y * blockDim.y + threadIdx.y; r < rows; r += (int64_t)gridDim.y * blockDim.y) {
        const int64_t i = r * W + x;
        const float2 a = vol[i];
        const float2 b = x + 1 < W ? vol[i + 1] : make_float2(0.0f, 0.0f);
        xp[i] = make_float4(a.x, a.y, b.x, b.y);
    }
}

template <typename VT>
static int launch_mse(const VT* v, const void* rot, const float2* t, float2* dv, void* grad_rotation, float* part,
                      double* loss_part, float scale, const SliceGeom& g, int tiles, unsigned nb, cudaStream_t st) {
    if (dv && grad_rotation)
        slice_mse_kernel<true, true, VT><<<nb, kExtractThreads, 0, st>>>(v, rot, t, dv, part, loss_part, scale, g,
                                                                        tiles);
    else if (dv)
        slice_mse_kernel<true, false, VT><<<nb, kExtractThreads, 0, st>>>(v, rot, t, dv, part, loss_part, scale, g,
                                                                         tiles);
    else if (grad_rotation)
        slice_mse_kernel<false, true, VT><<<nb, kExtractThreads, 0, st>>>(v, rot, t, dv, part, loss_part, scale, g,
                                                                         tiles);
    else
        slice_mse_kernel<false, false, VT><<<nb, kExtractThreads, 0, st>>>(v, rot, t, dv, part, loss_part, scale, g,
                                                                          tiles);
    return check_launch("slice_mse_kernel");
}

}  // namespace tt

using namespace tt;

// Loss partials (double) and rotation-gradient partials, one slot per row of tiles.
static size_t mse_workspace_bytes(int64_t n, int rows) {
    return (size_t)(n * rows) * sizeof(double) + partial_bytes(n, rows);
}

extern "C" size_t tt_central_slice_mse_workspace_bytes(const tt_slice_params* p) {
    if (!p || p->n <= 0 || p->img_h < 1 || p->img_w < 1) return 0;
    return mse_workspace_bytes(p->n, tile_rows((int)p->img_h));
}

extern "C" int tt_central_slice_mse(const void* volume_rfft, const void* rotation_matrices, const void* targets,
                                    float* loss, void* grad_volume, void* grad_rotation, void* workspace,
                                    size_t workspace_bytes, const tt_slice_params* p, void* stream) {
    if (int e = validate_params(p, true)) return e;
    if (p->deterministic)
        return fail(TT_ERR_INVALID, "central_slice_mse: no deterministic mode (the gradient scale is known only "
                                    "after the loss); use the extraction backward");
    if (p->n == 0) return fail(TT_ERR_INVALID, "central_slice_mse: no slices (the mean is undefined)");
    if (!volume_rfft || !rotation_matrices || !targets || !loss)
        return fail(TT_ERR_INVALID, "central_slice_mse: NULL pointer argument");
    SliceGeom g = make_geom(*p);
    const int tiles = extract_tiles(g);
    const int rows = tile_rows(g.img_h);
    const int64_t blocks = (int64_t)g.n * rows;  // one block (and one partial slot) per row of tiles
    if ((int64_t)g.n * tiles > 0x7fffffffLL) return fail(TT_ERR_INVALID, "central_slice_mse: too many blocks");
    const size_t need = mse_workspace_bytes(g.n, rows);
    if (!workspace || workspace_bytes < need)
        return fail(TT_ERR_WORKSPACE, "central_slice_mse: workspace of %zu bytes needed, got %zu", need,
                    workspace_bytes);
    double* loss_part = (double*)workspace;
    float* part = (float*)((char*)workspace + (size_t)blocks * sizeof(double));
    const double m = (double)g.n * g.img_h * g.wr;
    const float scale = (float)(2.0 / m);
    const float2* t = (const float2*)targets;
    float2* dv = (float2*)grad_volume;
    cudaStream_t st = as_stream(stream);
    const unsigned nb = (unsigned)((int64_t)g.n * (tiles / tiles_x_of(g.wr)));  // one block per row of tiles
    int e;
    switch (g.vol_layout) {
        case TT_VOLUME_XPAIRS:
            e = launch_mse((const float4*)volume_rfft, rotation_matrices, t, dv, grad_rotation, part, loss_part,
                           scale, g, tiles, nb, st);
            break;
        case TT_VOLUME_BRICKS:
            e = launch_mse((const VoxBrick2*)volume_rfft, rotation_matrices, t, dv, grad_rotation, part, loss_part,
                           scale, g, tiles, nb, st);
            break;
        default:
            e = launch_mse((const float2*)volume_rfft, rotation_matrices, t, dv, grad_rotation, part, loss_part,
                           scale, g, tiles, nb, st);
    }
    if (e) return e;
    mse_loss_finish_kernel<<<1, 1024, 0, st>>>(loss_part, blocks, 1.0 / m, loss);
    if (int e = check_launch("mse_loss_finish_kernel")) return e;
    if (grad_rotation) return launch_drot_finish(part, rotation_matrices, grad_rotation, g, rows, st);
    return TT_OK;
}

extern "C" int tt_extract_central_slices_rfft_3d(const void* volume_rfft, const void* rotation_matrices,
                                                 void* slices_out, const tt_slice_params* p, void* stream) {
    if (int e = validate_params(p, true)) return e;
    if (p->n == 0) return TT_OK;
    if (!volume_rfft || !rotation_matrices || !slices_out)
        return fail(TT_ERR_INVALID, "extract: NULL pointer argument");
    SliceGeom g = make_geom(*p);
    const int tiles = extract_tiles(g);
    const int64_t blocks = (int64_t)g.n * tiles;
    if (blocks > 0x7fffffffLL) return fail(TT_ERR_INVALID, "extract: too many blocks");
    const unsigned nb = (unsigned)((int64_t)g.n * (tiles / tiles_x_of(g.wr)));  // one block per row of tiles
    cudaStream_t st = as_stream(stream);
    switch (g.vol_layout) {
        case TT_VOLUME_XPAIRS:
            extract_fwd_kernel<<<nb, kExtractThreads, 0, st>>>((const float4*)volume_rfft, rotation_matrices,
                                                               (float2*)slices_out, g, tiles);
            break;
        case TT_VOLUME_BRICKS:
            extract_fwd_kernel<<<nb, kExtractThreads, 0, st>>>((const VoxBrick2*)volume_rfft, rotation_matrices,
                                                               (float2*)slices_out, g, tiles);
            break;
        default:
            extract_fwd_kernel<<<nb, kExtractThreads, 0, st>>>((const float2*)volume_rfft, rotation_matrices,
                                                               (float2*)slices_out, g, tiles);
    }
    return check_launch("extract_fwd_kernel");
}

extern "C" size_t tt_volume_xpairs_bytes(const tt_slice_params* p) {
    if (!p || p->vol_d < 1 || p->vol_h < 1 || p->vol_w < 1) return 0;
    return (size_t)(p->vol_d * p->vol_h * p->vol_w) * sizeof(float4);
}

extern "C" int tt_pack_volume_xpairs(const void* volume_rfft, void* xpairs, const tt_slice_params* p,
                                     void* stream) {
    if (int e = validate_params(p, true)) return e;
    if (!volume_rfft || !xpairs) return fail(TT_ERR_INVALID, "pack_volume_xpairs: NULL pointer argument");
    if ((reinterpret_cast<uintptr_t>(xpairs) & 15) != 0)
        return fail(TT_ERR_INVALID, "pack_volume_xpairs: the x-paired copy must be 16-byte aligned");
    if ((reinterpret_cast<uintptr_t>(volume_rfft) & 7) != 0)
        return fail(TT_ERR_INVALID, "pack_volume_xpairs: the volume must be 8-byte aligned");
    const int64_t rows = p->vol_d * p->vol_h;
    const int W = (int)p->vol_w;
    const dim3 block(32, 8);
    const int64_t gy = (rows + block.y - 1) / block.y;
    const dim3 grid((unsigned)((W + 31) / 32), (unsigned)(gy < 65535 ? gy : 65535));
    pack_xpairs_kernel<<<grid, block, 0, as_stream(stream)>>>((const float2*)volume_rfft, (float4*)xpairs, rows, W);
    return check_launch("pack_xpairs_kernel");
}

extern "C" size_t tt_volume_bricks_bytes(const tt_slice_params* p) {
    if (!p || p->vol_d < 1 || p->vol_h < 1 || p->vol_w < 1) return 0;
    return (size_t)(((p->vol_d + 1) / 2) * ((p->vol_h + 1) / 2) * ((p->vol_w + 1) / 2)) * 64;
}

extern "C" int tt_pack_volume_bricks(const void* volume_rfft, void* bricks, const tt_slice_params* p,
                                     void* stream) {
    if (int e = validate_params(p, true)) return e;
    if (!volume_rfft || !bricks) return fail(TT_ERR_INVALID, "pack_volume_bricks: NULL pointer argument");
    if ((reinterpret_cast<uintptr_t>(bricks) & 15) != 0)
        return fail(TT_ERR_INVALID, "pack_volume_bricks: the bricked copy must be 16-byte aligned");
    if ((reinterpret_cast<uintptr_t>(volume_rfft) & 7) != 0)
        return fail(TT_ERR_INVALID, "pack_volume_bricks: the volume must be 8-byte aligned");
    if (!bricks_fit(p)) return fail(TT_ERR_INVALID, "pack_volume_bricks: the copy must hold fewer than 2^31 slots");
    const SliceGeom g = make_geom(*p);
    const int64_t slots = (int64_t)(tt_volume_bricks_bytes(p) / sizeof(float2));
    const int64_t want = (slots + 255) / 256;
    const unsigned grid = (unsigned)(want < 148 * 64 ? want : 148 * 64);
    pack_bricks_kernel<<<grid, 256, 0, as_stream(stream)>>>((const float2*)volume_rfft, (float2*)bricks, g, slots);
    return check_launch("pack_bricks_kernel");
}

extern "C" int tt_slice_geometry(const void* rotation_matrices, int32_t mode, uint8_t* flags, float* coords,
                                 const tt_slice_params* p, void* stream) {
    if (int e = validate_params(p, true)) return e;
    if (p->n == 0) return TT_OK;
    if (!rotation_matrices || !flags || !coords) return fail(TT_ERR_INVALID, "slice_geometry: NULL pointer argument");
    if (mode != 0 && mode != 1) return fail(TT_ERR_INVALID, "slice_geometry: mode must be 0 or 1");
    SliceGeom g = make_geom(*p);
    const int tiles = extract_tiles(g);
    const int64_t blocks = (int64_t)g.n * tiles;
    if (blocks > 0x7fffffffLL) return fail(TT_ERR_INVALID, "slice_geometry: too many blocks");
    slice_geometry_kernel<<<(unsigned)blocks, kExtractThreads, 0, as_stream(stream)>>>(rotation_matrices, flags,
                                                                                     coords, g, tiles, mode);
    return check_launch("slice_geometry_kernel");
}

extern "C" size_t tt_extract_backward_workspace_bytes(const tt_slice_params* p) {
    if (!p || p->n <= 0 || p->img_h < 1 || p->img_w < 1) return 0;
    // one slot of partials per tile: the multichannel backward (one block per
    // tile) takes this workspace too; the single-channel kernels use one slot
    // per row of tiles of it
    return fixed_dv_bytes(p) + partial_bytes(p->n, tiles_per_slice((int)p->img_h, (int)(p->img_w / 2 + 1)));
}

extern "C" int tt_extract_central_slices_rfft_3d_backward(
    const void* volume_rfft, const void* rotation_matrices, const void* grad_slices, void* grad_volume,
    void* grad_rotation, void* workspace, size_t workspace_bytes, const tt_slice_params* p, void* stream) {
    if (int e = validate_params(p, true)) return e;
    if (p->n == 0) return TT_OK;
    if (!volume_rfft || !rotation_matrices || !grad_slices)
        return fail(TT_ERR_INVALID, "extract backward: NULL pointer argument");
    if (!grad_volume && !grad_rotation) return TT_OK;
    SliceGeom g = make_geom(*p);
    const int tiles = extract_tiles(g);
    if ((int64_t)g.n * tiles > 0x7fffffffLL) return fail(TT_ERR_INVALID, "extract backward: too many blocks");
    const size_t fixed = grad_volume ? fixed_dv_bytes(p) : 0;
    if (grad_rotation || fixed) {
        const size_t need = fixed + (grad_rotation ? partial_bytes(g.n, tile_rows(g.img_h)) : 0);
        if (!workspace || workspace_bytes < need)
            return fail(TT_ERR_WORKSPACE, "extract backward: workspace of %zu bytes needed, got %zu", need,
                        workspace_bytes);
    }
    cudaStream_t st = as_stream(stream);
    if (fixed) {
        cudaError_t e = cudaMemsetAsync(workspace, 0, fixed, st);
        if (e != cudaSuccess) return fail(TT_ERR_CUDA, "extract backward: memset: %s", cudaGetErrorString(e));
    }
    return launch_backward(volume_rfft, rotation_matrices, (const float2*)grad_slices, (float2*)grad_volume,
                           grad_rotation, (float*)((char*)workspace + fixed), g, st, fixed ? workspace : nullptr);
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the extraction backward.
//
// Some callers cannot allocate device memory at the time they run this
// backward: a host application or plugin framework that owns every device
// allocation and only lends the library the buffers of one call, or a caller
// working inside a fixed, pre-reserved memory budget that must never grow.
// For them the rotation-gradient partial sums live in a fixed scratch array
// compiled into this library instead of a caller-provided workspace.
//
// * The array is TT_NOALLOC_SCRATCH_BYTES (4 MiB) of device memory per GPU that
//   loads the library, held until the process exits.
// * Host code cannot pass the array's name to a kernel (it is only a host-side
//   stand-in for the device symbol), so the first call on each device looks up
//   its device address with cudaGetSymbolAddress while that device is current
//   and keeps it.  Make that first call before any stream capture.
// * Every call shares the one array.  Calls whose kernels overlap on the GPU
//   (different streams, or different host threads on the same device) race on
//   it and must be serialised by the caller.  Each call fully overwrites the
//   part it reads, so nothing has to be cleared between calls.
// * No cudaMalloc, cudaFree or allocating library routine is called.
// ---------------------------------------------------------------------------

static __device__ __align__(256) float g_noalloc_scratch[TT_NOALLOC_SCRATCH_BYTES / sizeof(float)];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
float* g_noalloc_ptr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device (looked up once).
int noalloc_scratch(float** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return tt::fail(TT_ERR_CUDA, "noalloc backward: cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return tt::fail(TT_ERR_INVALID, "noalloc backward: device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        float* ptr = nullptr;
        e = cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return tt::fail(TT_ERR_CUDA, "noalloc backward: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        g_noalloc_ptr[dev] = ptr;
    }
    *out = g_noalloc_ptr[dev];
    return TT_OK;
}
}  // namespace

extern "C" int tt_extract_central_slices_rfft_3d_backward_noalloc(const void* volume_rfft,
                                                                  const void* rotation_matrices,
                                                                  const void* grad_slices, void* grad_volume,
                                                                  void* grad_rotation, const tt_slice_params* p,
                                                                  void* stream) {
    if (int e = validate_params(p, true)) return e;
    if (p->n == 0) return TT_OK;
    if (!volume_rfft || !rotation_matrices || !grad_slices)
        return fail(TT_ERR_INVALID, "noalloc backward: NULL pointer argument");
    if (!grad_volume && !grad_rotation) return TT_OK;
    if (p->deterministic && grad_volume)
        return fail(TT_ERR_INVALID, "noalloc backward: the deterministic volume gradient needs a workspace "
                                    "(tt_extract_central_slices_rfft_3d_backward)");
    SliceGeom g = make_geom(*p);
    const int tiles = extract_tiles(g);
    if ((int64_t)g.n * tiles > 0x7fffffffLL) return fail(TT_ERR_INVALID, "noalloc backward: too many blocks");
    cudaStream_t st = as_stream(stream);
    const void* v = volume_rfft;
    const float2* gr = (const float2*)grad_slices;
    float2* dv = (float2*)grad_volume;
    // the scratch holds 6 partial sums of the rotation gradient per row of tiles
    if (!grad_rotation)  // the volume gradient alone needs no scratch
        return launch_backward(v, rotation_matrices, gr, dv, nullptr, nullptr, g, st);
    const size_t need = partial_bytes(g.n, tile_rows(g.img_h));
    if (need > (size_t)TT_NOALLOC_SCRATCH_BYTES)
        return fail(TT_ERR_INVALID,
                    "noalloc backward: %lld slices of %lld x %lld need %zu bytes of scratch, more than the "
                    "%u-byte built-in array; split the slices into smaller calls or use "
                    "tt_extract_central_slices_rfft_3d_backward with a workspace",
                    (long long)p->n, (long long)p->img_h, (long long)(p->img_w / 2 + 1), need,
                    (unsigned)TT_NOALLOC_SCRATCH_BYTES);
    float* part = nullptr;
    if (int e = noalloc_scratch(&part)) return e;
    return launch_backward(v, rotation_matrices, gr, dv, grad_rotation, part, g, st);
}
