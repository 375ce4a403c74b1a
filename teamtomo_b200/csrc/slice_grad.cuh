// Per-pixel pieces of the extraction backward shared by the single- and the
// multi-channel kernels: the d/dvolume scatter target, the corner loads and the
// rotation-gradient terms.
#pragma once
#include <cuda_runtime.h>

#include "fixed_point.cuh"
#include "slice_common.cuh"
#include "slice_ops.cuh"

namespace tt {

// Volume-gradient target: float2 atomics, or (FIXED, the deterministic mode)
// two 64-bit fixed-point words per voxel at scale `scale`.
template <bool FIXED>
struct DvTarget {
    float2* dvol;
    unsigned long long* fixed;
    double scale;
    __device__ __forceinline__ void add(int64_t vi, float2 gv, float w) const {
        if (FIXED) {
            fixed_add(fixed + 2 * vi, (double)gv.x * (double)w * scale);
            fixed_add(fixed + 2 * vi + 1, (double)gv.y * (double)w * scale);
        } else {
            atomicAdd(dvol + vi, make_float2(gv.x * w, gv.y * w));
        }
    }
};

// d/dvolume scatter of G' over the grid_sample corners of one pixel.
template <bool FIXED>
__device__ __forceinline__ void scatter_dv(const DvTarget<FIXED>& dv, const SliceGeom& g, const Corners& k,
                                           float2 gv) {
#pragma unroll
    for (int bz = 0; bz < 2; bz++) {
        if (bz && !k.zin) continue;
        const float wz = bz ? k.az1 : k.az0;
#pragma unroll
        for (int by = 0; by < 2; by++) {
            if (by && !k.yin) continue;
            const float wzy = (by ? k.ay1 : k.ay0) * wz;
            const int64_t base = vox_index(g, k.z0 + bz, k.y0 + by, k.x0);
#pragma unroll
            for (int bx = 0; bx < 2; bx++) {
                if (bx && !k.xin) continue;
                const float w = (bx ? k.ax1 : k.ax0) * wzy;
                if (w != 0.0f) dv.add(base + bx, gv, w);
            }
        }
    }
}

// d/dvolume scatter with x-paired lanes: lanes 2j and 2j+1 reduce the x-low
// and the x-high corner of the same pixel in the same instruction.  The two
// corners are adjacent voxels, usually in one 32-byte L2 sector, so a warp's
// reduction touches fewer sectors than with one pixel per lane (each pair of
// lanes serves pixels j and j + 16 in two rounds).  Only the pixel's G' and
// its three source indices move by warp shuffles (5 per round; shuffles share
// the L1 data pipe that limits the backward); each lane rebuilds the corner
// set from the indices with the same arithmetic, so corners, weights and
// values are those of scatter_dv.  Must be called by all 32 lanes of the warp
// (valid = false for lanes without a pixel).
__device__ __forceinline__ void scatter_dv_paired(float2* __restrict__ dvol, const SliceGeom& g, const SourceIdx& si,
                                                  float2 gv, bool valid) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, bx = lane & 1;
#pragma unroll
    for (int half = 0; half < 2; half++) {
        const int src = (lane >> 1) + 16 * half;
        const float sgx = __shfl_sync(full, gv.x, src), sgy = __shfl_sync(full, gv.y, src);
        const float siz = __shfl_sync(full, valid ? si.z : -1.0f, src);  // < 0: no pixel
        const float siy = __shfl_sync(full, si.y, src), six = __shfl_sync(full, si.x, src);
        if (siz < 0.0f) continue;
        const Corners k = corners_at(g, siz, siy, six);
        if (bx && !k.xin) continue;
        const float wx = bx ? k.ax1 : k.ax0;
#pragma unroll
        for (int zy = 0; zy < 4; zy++) {
            const int bz = zy >> 1, by = zy & 1;
            if ((bz && !k.zin) || (by && !k.yin)) continue;
            const float w = wx * ((by ? k.ay1 : k.ay0) * (bz ? k.az1 : k.az0));
            if (w != 0.0f)
                atomicAdd(dvol + vox_index(g, k.z0 + bz, k.y0 + by, k.x0) + bx, make_float2(sgx * w, sgy * w));
        }
    }
}

// Fixed-point d/dvolume scatter with lane pairs: lanes 2j and 2j+1 take the
// same pixel (pixels j and j + 16 in two rounds) and add the re and the im
// word of each corner in the same instruction — one 16-byte voxel slot, one
// L2 sector, where scatter_dv spends two.  Same corners, weights and rounded
// integers as scatter_dv (integer sums do not depend on who adds them).  Must
// be called by all 32 lanes of the warp (valid = false for lanes without a pixel).
__device__ __forceinline__ void scatter_dv_fixed_paired(unsigned long long* __restrict__ fixed, double scale,
                                                        const SliceGeom& g, const SourceIdx& si, float2 gv,
                                                        bool valid) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, odd = lane & 1;
#pragma unroll
    for (int half = 0; half < 2; half++) {
        const int src = (lane >> 1) + 16 * half;
        const float sgx = __shfl_sync(full, gv.x, src), sgy = __shfl_sync(full, gv.y, src);
        const float siz = __shfl_sync(full, valid ? si.z : -1.0f, src);  // < 0: no pixel
        const float siy = __shfl_sync(full, si.y, src), six = __shfl_sync(full, si.x, src);
        if (siz < 0.0f) continue;
        const Corners k = corners_at(g, siz, siy, six);
        const double sv = (double)(odd ? sgy : sgx);
#pragma unroll
        for (int zy = 0; zy < 4; zy++) {
            const int bz = zy >> 1, by = zy & 1;
            if ((bz && !k.zin) || (by && !k.yin)) continue;
            const float wzy = (by ? k.ay1 : k.ay0) * (bz ? k.az1 : k.az0);
            const int64_t base = vox_index(g, k.z0 + bz, k.y0 + by, k.x0);
#pragma unroll
            for (int bx = 0; bx < 2; bx++) {
                if (bx && !k.xin) continue;
                const float w = (bx ? k.ax1 : k.ax0) * wzy;
                if (w != 0.0f) fixed_add(fixed + 2 * (base + bx) + odd, sv * (double)w * scale);
            }
        }
    }
}

// The eight corner values of a pixel; corners past the last index read as
// zero, as in grid_sample.  VT: float2 (plain layout), float4 (x-paired) or
// VoxBrick2 (bricked).
template <typename VT>
__device__ __forceinline__ void load_corners(const VT* __restrict__ vol, const SliceGeom& g, const Corners& k,
                                             float2 v[2][2][2]) {
    const XRows<VT> rows(vol, g, k);
#pragma unroll
    for (int bz = 0; bz < 2; bz++)
#pragma unroll
        for (int by = 0; by < 2; by++) {
            const bool row_ok = (!bz || k.zin) && (!by || k.yin);
            rows.load(g, row_ok ? bz : 0, row_ok ? by : 0, row_ok, row_ok && k.xin, v[bz][by][0], v[bz][by][1]);
        }
}

// Adds the pixel's 6 contributions to d/dR_zyx (rows z, y, x x columns y, x —
// column 0 multiplies the zero z frequency of a central slice) to acc, from
// its corner values: the trilinear gradient from differences of neighbouring
// voxels (subtracting first keeps it accurate where the volume varies
// slowly), then Re(conj(G') dV/dc) chained through dc/dp and the redirect sign.
__device__ __forceinline__ void drot_terms(const float2 v[2][2][2], const Corners& k, float2 gv, bool cj,
                                           const SliceGeom& g, float qy, float qx, float acc[6]) {
    float2 gz = make_float2(0.f, 0.f), gy = gz, gx = gz;
    const float wzs[2] = {k.az0, k.az1}, wys[2] = {k.ay0, k.ay1}, wxs[2] = {k.ax0, k.ax1};
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 2; b++) {
            const float wyx = wys[a] * wxs[b], wzx = wzs[a] * wxs[b], wzy = wzs[a] * wys[b];
            gz.x = fmaf(wyx, v[1][a][b].x - v[0][a][b].x, gz.x);
            gz.y = fmaf(wyx, v[1][a][b].y - v[0][a][b].y, gz.y);
            gy.x = fmaf(wzx, v[a][1][b].x - v[a][0][b].x, gy.x);
            gy.y = fmaf(wzx, v[a][1][b].y - v[a][0][b].y, gy.y);
            gx.x = fmaf(wzy, v[a][b][1].x - v[a][b][0].x, gx.x);
            gx.y = fmaf(wzy, v[a][b][1].y - v[a][b][0].y, gx.y);
        }
    const float sg = cj ? -1.f : 1.f;
    // an axis whose source index is on the border gets no gradient (grid_sample's clip)
    const float p0 = k.gz ? fmaf(gv.x, gz.x, gv.y * gz.y) * g.dcdp0 * sg : 0.0f;
    const float p1 = k.gy ? fmaf(gv.x, gy.x, gv.y * gy.y) * g.dcdp1 * sg : 0.0f;
    const float p2 = k.gx ? fmaf(gv.x, gx.x, gv.y * gx.y) * g.dcdp2 * sg : 0.0f;
    acc[0] += p0 * qy;
    acc[1] += p0 * qx;
    acc[2] += p1 * qy;
    acc[3] += p1 * qx;
    acc[4] += p2 * qy;
    acc[5] += p2 * qx;
}

// Launch of the fixed-order d/drotation reduction (extract.cu).
int launch_drot_finish(const float* part, const void* rot, void* drot, const SliceGeom& g, int tiles,
                       cudaStream_t st);

}  // namespace tt
