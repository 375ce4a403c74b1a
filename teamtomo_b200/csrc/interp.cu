// Generic 3D interpolation primitives of torch_image_interpolation
// (image_interpolation_3d.py:11-101 sample_image_3d, :104-275 insert_into_image_3d).
//
// sample: one thread per coordinate.  Trilinear follows grid_sample with
//   padding_mode='border', align_corners=True: the 8 corners of the clamped
//   coordinate, corners past the last index contribute nothing, and samples
//   whose coordinate is outside [0, n-1] on any axis are zero.  Nearest rounds
//   half to even (nearbyint).
// insert: one thread per value.  Coordinates are float32 (the reference casts
//   with .float()); points outside [0, n-1] on any axis are dropped; trilinear
//   splats with floor/ceil corners and float32 (1-t)/t weight products cast to
//   the weight dtype; nearest adds the value and a weight of 1 at rint(c).
// Element types: float32, float64, complex64, complex128 (dtype codes 0-3).
#include <cuda_runtime.h>

#include "capi_util.cuh"

namespace tt {

template <typename T>
__device__ __forceinline__ void atomic_add_real(T* p, T v) {
    atomicAdd(p, v);
}

// One sample of the (C, D, H, W) image at (cz, cy, cx) into o[0 .. C*E).
template <typename T, int E>
__device__ __forceinline__ void sample_point(const T* __restrict__ img, int64_t C, int D, int H, int W, T cz, T cy,
                                             T cx, T* __restrict__ o, int nearest) {
    const bool inside = cz >= (T)0 && cz <= (T)(D - 1) && cy >= (T)0 && cy <= (T)(H - 1) && cx >= (T)0 &&
                        cx <= (T)(W - 1);
    const int64_t plane = (int64_t)D * H * W;
    if (!inside) {
        for (int64_t k = 0; k < C * E; k++) o[k] = (T)0;
        return;
    }
    if (nearest) {
        const int z = (int)nearbyint((double)cz), y = (int)nearbyint((double)cy), x = (int)nearbyint((double)cx);
        const int64_t vi = ((int64_t)z * H + y) * W + x;
        for (int64_t ch = 0; ch < C; ch++)
#pragma unroll
            for (int e = 0; e < E; e++) o[ch * E + e] = img[(ch * plane + vi) * E + e];
        return;
    }
    const T fz = floor(cz), fy = floor(cy), fx = floor(cx);
    const int z0 = (int)fz, y0 = (int)fy, x0 = (int)fx;
    const T az[2] = {(fz + (T)1) - cz, cz - fz};
    const T ay[2] = {(fy + (T)1) - cy, cy - fy};
    const T ax[2] = {(fx + (T)1) - cx, cx - fx};
    for (int64_t ch = 0; ch < C; ch++) {
        T acc[E];
#pragma unroll
        for (int e = 0; e < E; e++) acc[e] = (T)0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int bz = (k >> 2) & 1, by = (k >> 1) & 1, bx = k & 1;
            const int z = z0 + bz, y = y0 + by, x = x0 + bx;
            if (z >= D || y >= H || x >= W) continue;
            const T wgt = ax[bx] * ay[by] * az[bz];
            const int64_t vi = ch * plane + ((int64_t)z * H + y) * W + x;
#pragma unroll
            for (int e = 0; e < E; e++) acc[e] += img[vi * E + e] * wgt;
        }
#pragma unroll
        for (int e = 0; e < E; e++) o[ch * E + e] = acc[e];
    }
}

template <typename T, int E>
__global__ void sample3d_kernel(const T* __restrict__ img, int64_t C, int D, int H, int W,
                                const T* __restrict__ coords, int64_t n, T* __restrict__ out, int nearest) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    sample_point<T, E>(img, C, D, H, W, coords[i * 3 + 0], coords[i * 3 + 1], coords[i * 3 + 2], out + i * C * E,
                       nearest);
}

// Backward of sample3d_kernel: d/dimage (ACCUMULATED, atomics) and
// d/dcoordinates (overwritten), PyTorch's complex-gradient convention.
// Trilinear: the same corners and weights; the coordinate gradient per axis is
// Re(conj(G) dS/dc) summed over the channels, zero where grid_sample's border
// clip stops it (a source index of exactly 0 or n-1 on that axis).  Nearest:
// the gradient goes to the sampled voxel; coordinates get none.
template <typename T>
__device__ __forceinline__ bool coord_grad_passes(T c, int n) {
    // grid_sample's round trip of the coordinate: c -> c / (0.5 n - 0.5) - 1 -> ((g + 1) / 2) (n - 1)
    const T half = (T)0.5 * (T)n - (T)0.5;
    const T raw = ((c / half - (T)1 + (T)1) * (T)0.5) * (T)(n - 1);
    return raw > (T)0 && raw < (T)(n - 1);
}

template <typename T, int E>
__global__ void sample3d_bwd_kernel(const T* __restrict__ img, int64_t C, int D, int H, int W,
                                    const T* __restrict__ coords, int64_t n, const T* __restrict__ grad,
                                    T* __restrict__ gimg, T* __restrict__ gcoord, int nearest) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const T cz = coords[i * 3 + 0], cy = coords[i * 3 + 1], cx = coords[i * 3 + 2];
    const T* gi = grad + i * C * E;
    T dz = (T)0, dy = (T)0, dx = (T)0;
    const bool inside = cz >= (T)0 && cz <= (T)(D - 1) && cy >= (T)0 && cy <= (T)(H - 1) && cx >= (T)0 &&
                        cx <= (T)(W - 1);
    const int64_t plane = (int64_t)D * H * W;
    if (inside && nearest) {
        if (gimg) {
            const int z = (int)nearbyint((double)cz), y = (int)nearbyint((double)cy), x = (int)nearbyint((double)cx);
            const int64_t vi = ((int64_t)z * H + y) * W + x;
            for (int64_t ch = 0; ch < C; ch++)
#pragma unroll
                for (int e = 0; e < E; e++) atomicAdd(gimg + (ch * plane + vi) * E + e, gi[ch * E + e]);
        }
    } else if (inside) {
        const T fz = floor(cz), fy = floor(cy), fx = floor(cx);
        const int z0 = (int)fz, y0 = (int)fy, x0 = (int)fx;
        const T az[2] = {(fz + (T)1) - cz, cz - fz};
        const T ay[2] = {(fy + (T)1) - cy, cy - fy};
        const T ax[2] = {(fx + (T)1) - cx, cx - fx};
        const T sgn[2] = {(T)-1, (T)1};
        for (int64_t ch = 0; ch < C; ch++) {
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int bz = (k >> 2) & 1, by = (k >> 1) & 1, bx = k & 1;
                const int z = z0 + bz, y = y0 + by, x = x0 + bx;
                if (z >= D || y >= H || x >= W) continue;
                const int64_t vi = ch * plane + ((int64_t)z * H + y) * W + x;
                if (gimg) {
                    const T wgt = ax[bx] * ay[by] * az[bz];
#pragma unroll
                    for (int e = 0; e < E; e++) atomicAdd(gimg + vi * E + e, gi[ch * E + e] * wgt);
                }
                if (gcoord) {
                    T gv = (T)0;  // Re(conj(G) v)
#pragma unroll
                    for (int e = 0; e < E; e++) gv += gi[ch * E + e] * img[vi * E + e];
                    dz += gv * sgn[bz] * ay[by] * ax[bx];
                    dy += gv * az[bz] * sgn[by] * ax[bx];
                    dx += gv * az[bz] * ay[by] * sgn[bx];
                }
            }
        }
        if (!coord_grad_passes(cz, D)) dz = (T)0;
        if (!coord_grad_passes(cy, H)) dy = (T)0;
        if (!coord_grad_passes(cx, W)) dx = (T)0;
    }
    if (gcoord) {
        gcoord[i * 3 + 0] = dz;
        gcoord[i * 3 + 1] = dy;
        gcoord[i * 3 + 2] = dx;
    }
}

// affine_transform_image_3d (torch_transform_image/transforms_3d.py:10-40):
// output voxel (z, y, x) of matrix m samples the image at M_m (z, y, x, 1),
// M in zyx order, computed in float32 with the reference's operation order
// (((m0 z + m1 y) + m2 x) + m3 1, each product rounded) so that nearest
// sampling picks the same voxels.  One thread per (matrix, output voxel).
template <typename T, int E>
__global__ void affine3d_kernel(const T* __restrict__ img, int64_t C, int D, int H, int W,
                                const float* __restrict__ mats, int64_t nm, int od, int oh, int ow,
                                T* __restrict__ out, int nearest) {
    const int64_t vox = (int64_t)od * oh * ow;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nm * vox) return;
    const int64_t mi = idx / vox, r = idx - mi * vox;
    const float z = (float)(r / ((int64_t)oh * ow)), y = (float)((r / ow) % oh), x = (float)(r % ow);
    const float* M = mats + mi * 16;
    float c[3];
#pragma unroll
    for (int i = 0; i < 3; i++)
        c[i] = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(M[i * 4 + 0], z), __fmul_rn(M[i * 4 + 1], y)),
                                   __fmul_rn(M[i * 4 + 2], x)),
                         __fmul_rn(M[i * 4 + 3], 1.0f));
    sample_point<T, E>(img, C, D, H, W, (T)c[0], (T)c[1], (T)c[2], out + idx * C * E, nearest);
}

template <typename T, int E, typename WT>
__global__ void insert3d_kernel(const T* __restrict__ vals, const float* __restrict__ coords, int64_t n,
                                T* __restrict__ img, int64_t C, int D, int H, int W, WT* __restrict__ wts,
                                int nearest) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float cz = coords[i * 3 + 0], cy = coords[i * 3 + 1], cx = coords[i * 3 + 2];
    if (!(cz >= 0.0f && cz <= (float)D - 1.0f && cy >= 0.0f && cy <= (float)H - 1.0f && cx >= 0.0f &&
          cx <= (float)W - 1.0f))
        return;
    const int64_t plane = (int64_t)D * H * W;
    const T* v = vals + i * C * E;
    if (nearest) {
        const int64_t vi = ((int64_t)rintf(cz) * H + (int64_t)rintf(cy)) * W + (int64_t)rintf(cx);
        for (int64_t ch = 0; ch < C; ch++)
#pragma unroll
            for (int e = 0; e < E; e++) atomic_add_real(img + (ch * plane + vi) * E + e, v[ch * E + e]);
        atomic_add_real(wts + vi, (WT)1);
        return;
    }
    const float z0 = floorf(cz), y0 = floorf(cy), x0 = floorf(cx);
    const int iz[2] = {(int)z0, (int)ceilf(cz)}, iy[2] = {(int)y0, (int)ceilf(cy)}, ix[2] = {(int)x0, (int)ceilf(cx)};
    const float tz = cz - z0, ty = cy - y0, tx = cx - x0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int bz = (k >> 2) & 1, by = (k >> 1) & 1, bx = k & 1;
        const float w = ((bz ? tz : 1.0f - tz) * (by ? ty : 1.0f - ty)) * (bx ? tx : 1.0f - tx);
        if (w == 0.0f) continue;
        const int64_t vi = ((int64_t)iz[bz] * H + iy[by]) * W + ix[bx];
        const WT ww = (WT)w;
        const T wv = (T)ww;
        for (int64_t ch = 0; ch < C; ch++)
#pragma unroll
            for (int e = 0; e < E; e++) atomic_add_real(img + (ch * plane + vi) * E + e, v[ch * E + e] * wv);
        atomic_add_real(wts + vi, ww);
    }
}

// Backward of insert3d_kernel w.r.t. the values: each point gathers the
// upstream image gradient at the voxels it was added to, with the same float32
// weights (grad_values (n, channels) overwritten; zero for dropped points).
template <typename T, int E>
__global__ void insert3d_bwd_kernel(const T* __restrict__ gimg, const float* __restrict__ coords, int64_t n,
                                    int64_t C, int D, int H, int W, T* __restrict__ gvals, int nearest) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float cz = coords[i * 3 + 0], cy = coords[i * 3 + 1], cx = coords[i * 3 + 2];
    T* o = gvals + i * C * E;
    for (int64_t k = 0; k < C * E; k++) o[k] = (T)0;
    if (!(cz >= 0.0f && cz <= (float)D - 1.0f && cy >= 0.0f && cy <= (float)H - 1.0f && cx >= 0.0f &&
          cx <= (float)W - 1.0f))
        return;
    const int64_t plane = (int64_t)D * H * W;
    if (nearest) {
        const int64_t vi = ((int64_t)rintf(cz) * H + (int64_t)rintf(cy)) * W + (int64_t)rintf(cx);
        for (int64_t ch = 0; ch < C; ch++)
#pragma unroll
            for (int e = 0; e < E; e++) o[ch * E + e] = gimg[(ch * plane + vi) * E + e];
        return;
    }
    const float z0 = floorf(cz), y0 = floorf(cy), x0 = floorf(cx);
    const int iz[2] = {(int)z0, (int)ceilf(cz)}, iy[2] = {(int)y0, (int)ceilf(cy)}, ix[2] = {(int)x0, (int)ceilf(cx)};
    const float tz = cz - z0, ty = cy - y0, tx = cx - x0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int bz = (k >> 2) & 1, by = (k >> 1) & 1, bx = k & 1;
        const float w = ((bz ? tz : 1.0f - tz) * (by ? ty : 1.0f - ty)) * (bx ? tx : 1.0f - tx);
        if (w == 0.0f) continue;
        const int64_t vi = ((int64_t)iz[bz] * H + iy[by]) * W + ix[bx];
        for (int64_t ch = 0; ch < C; ch++)
#pragma unroll
            for (int e = 0; e < E; e++) o[ch * E + e] += gimg[(ch * plane + vi) * E + e] * (T)w;
    }
}

inline unsigned nblocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace tt

using namespace tt;

extern "C" int tt_sample_image_3d(const void* image, int32_t dtype, int64_t channels, int64_t d, int64_t h,
                                  int64_t w, const void* coordinates, int64_t n, void* out, int32_t nearest,
                                  void* stream) {
    if (n == 0) return TT_OK;
    if (!image || !coordinates || !out || channels < 1 || d < 1 || h < 1 || w < 1 || n < 0)
        return fail(TT_ERR_INVALID, "sample_image_3d: bad arguments");
    cudaStream_t st = as_stream(stream);
    const unsigned b = nblocks(n, 256);
    switch (dtype) {
        case 0:
            sample3d_kernel<float, 1><<<b, 256, 0, st>>>((const float*)image, channels, (int)d, (int)h, (int)w,
                                                          (const float*)coordinates, n, (float*)out, nearest);
            break;
        case 1:
            sample3d_kernel<double, 1><<<b, 256, 0, st>>>((const double*)image, channels, (int)d, (int)h, (int)w,
                                                           (const double*)coordinates, n, (double*)out, nearest);
            break;
        case 2:
            sample3d_kernel<float, 2><<<b, 256, 0, st>>>((const float*)image, channels, (int)d, (int)h, (int)w,
                                                          (const float*)coordinates, n, (float*)out, nearest);
            break;
        case 3:
            sample3d_kernel<double, 2><<<b, 256, 0, st>>>((const double*)image, channels, (int)d, (int)h, (int)w,
                                                           (const double*)coordinates, n, (double*)out, nearest);
            break;
        default:
            return fail(TT_ERR_INVALID, "sample_image_3d: unknown dtype code %d", dtype);
    }
    return check_launch("sample3d_kernel");
}

extern "C" int tt_insert_into_image_3d(const void* values, int32_t dtype, const float* coordinates, int64_t n,
                                       void* image, int64_t channels, int64_t d, int64_t h, int64_t w,
                                       void* weights, int32_t weights_f64, int32_t nearest, void* stream) {
    if (n == 0) return TT_OK;
    if (!values || !coordinates || !image || !weights || channels < 1 || d < 1 || h < 1 || w < 1 || n < 0)
        return fail(TT_ERR_INVALID, "insert_into_image_3d: bad arguments");
    cudaStream_t st = as_stream(stream);
    const unsigned b = nblocks(n, 256);
#define TT_INSERT_CASE(T, E)                                                                                  \
    if (weights_f64)                                                                                          \
        insert3d_kernel<T, E, double><<<b, 256, 0, st>>>((const T*)values, coordinates, n, (T*)image, channels, \
                                                         (int)d, (int)h, (int)w, (double*)weights, nearest);  \
    else                                                                                                      \
        insert3d_kernel<T, E, float><<<b, 256, 0, st>>>((const T*)values, coordinates, n, (T*)image, channels,  \
                                                        (int)d, (int)h, (int)w, (float*)weights, nearest);
    switch (dtype) {
        case 0: TT_INSERT_CASE(float, 1) break;
        case 1: TT_INSERT_CASE(double, 1) break;
        case 2: TT_INSERT_CASE(float, 2) break;
        case 3: TT_INSERT_CASE(double, 2) break;
        default:
            return fail(TT_ERR_INVALID, "insert_into_image_3d: unknown dtype code %d", dtype);
    }
#undef TT_INSERT_CASE
    return check_launch("insert3d_kernel");
}

extern "C" int tt_affine_transform_image_3d(const void* image, int32_t dtype, int64_t channels, int64_t d, int64_t h,
                                            int64_t w, const float* matrices_zyx, int64_t n_matrices, int64_t od,
                                            int64_t oh, int64_t ow, int32_t nearest, void* out, void* stream) {
    if (n_matrices == 0 || od * oh * ow == 0) return TT_OK;
    if (!image || !matrices_zyx || !out || channels < 1 || d < 1 || h < 1 || w < 1 || n_matrices < 0 || od < 0 ||
        oh < 0 || ow < 0)
        return fail(TT_ERR_INVALID, "affine_transform_image_3d: bad arguments");
    if (dtype < 0 || dtype > 3) return fail(TT_ERR_INVALID, "affine_transform_image_3d: dtype must be 0-3");
    const int64_t total = n_matrices * od * oh * ow;
    const unsigned b = nblocks(total, 256);
    cudaStream_t st = as_stream(stream);
    switch (dtype) {
        case 0:
            affine3d_kernel<float, 1><<<b, 256, 0, st>>>((const float*)image, channels, (int)d, (int)h, (int)w,
                                                         matrices_zyx, n_matrices, (int)od, (int)oh, (int)ow,
                                                         (float*)out, nearest);
            break;
        case 1:
            affine3d_kernel<double, 1><<<b, 256, 0, st>>>((const double*)image, channels, (int)d, (int)h, (int)w,
                                                          matrices_zyx, n_matrices, (int)od, (int)oh, (int)ow,
                                                          (double*)out, nearest);
            break;
        case 2:
            affine3d_kernel<float, 2><<<b, 256, 0, st>>>((const float*)image, channels, (int)d, (int)h, (int)w,
                                                         matrices_zyx, n_matrices, (int)od, (int)oh, (int)ow,
                                                         (float*)out, nearest);
            break;
        default:
            affine3d_kernel<double, 2><<<b, 256, 0, st>>>((const double*)image, channels, (int)d, (int)h, (int)w,
                                                          matrices_zyx, n_matrices, (int)od, (int)oh, (int)ow,
                                                          (double*)out, nearest);
    }
    return check_launch("affine3d_kernel");
}

extern "C" int tt_sample_image_3d_backward(const void* image, int32_t dtype, int64_t channels, int64_t d, int64_t h,
                                           int64_t w, const void* coordinates, int64_t n, const void* grad_out,
                                           void* grad_image, void* grad_coordinates, int32_t nearest, void* stream) {
    if (n == 0) return TT_OK;
    if (!image || !coordinates || !grad_out || channels < 1 || d < 1 || h < 1 || w < 1 || n < 0)
        return fail(TT_ERR_INVALID, "sample_image_3d backward: bad arguments");
    if (dtype < 0 || dtype > 3) return fail(TT_ERR_INVALID, "sample_image_3d backward: dtype must be 0-3");
    if (!grad_image && !grad_coordinates) return TT_OK;
    const unsigned b = nblocks(n, 256);
    cudaStream_t st = as_stream(stream);
    switch (dtype) {
        case 0:
            sample3d_bwd_kernel<float, 1><<<b, 256, 0, st>>>((const float*)image, channels, (int)d, (int)h, (int)w,
                                                             (const float*)coordinates, n, (const float*)grad_out,
                                                             (float*)grad_image, (float*)grad_coordinates, nearest);
            break;
        case 1:
            sample3d_bwd_kernel<double, 1><<<b, 256, 0, st>>>((const double*)image, channels, (int)d, (int)h,
                                                              (int)w, (const double*)coordinates, n,
                                                              (const double*)grad_out, (double*)grad_image,
                                                              (double*)grad_coordinates, nearest);
            break;
        case 2:
            sample3d_bwd_kernel<float, 2><<<b, 256, 0, st>>>((const float*)image, channels, (int)d, (int)h, (int)w,
                                                             (const float*)coordinates, n, (const float*)grad_out,
                                                             (float*)grad_image, (float*)grad_coordinates, nearest);
            break;
        default:
            sample3d_bwd_kernel<double, 2><<<b, 256, 0, st>>>((const double*)image, channels, (int)d, (int)h,
                                                              (int)w, (const double*)coordinates, n,
                                                              (const double*)grad_out, (double*)grad_image,
                                                              (double*)grad_coordinates, nearest);
    }
    return check_launch("sample3d_bwd_kernel");
}

extern "C" int tt_insert_into_image_3d_backward(const void* grad_image, int32_t dtype, const float* coordinates,
                                                int64_t n, int64_t channels, int64_t d, int64_t h, int64_t w,
                                                int32_t nearest, void* grad_values, void* stream) {
    if (n == 0) return TT_OK;
    if (!grad_image || !coordinates || !grad_values || channels < 1 || d < 1 || h < 1 || w < 1 || n < 0)
        return fail(TT_ERR_INVALID, "insert_into_image_3d backward: bad arguments");
    if (dtype < 0 || dtype > 3) return fail(TT_ERR_INVALID, "insert_into_image_3d backward: dtype must be 0-3");
    const unsigned b = nblocks(n, 256);
    cudaStream_t st = as_stream(stream);
    switch (dtype) {
        case 0:
            insert3d_bwd_kernel<float, 1><<<b, 256, 0, st>>>((const float*)grad_image, coordinates, n, channels,
                                                             (int)d, (int)h, (int)w, (float*)grad_values, nearest);
            break;
        case 1:
            insert3d_bwd_kernel<double, 1><<<b, 256, 0, st>>>((const double*)grad_image, coordinates, n, channels,
                                                              (int)d, (int)h, (int)w, (double*)grad_values, nearest);
            break;
        case 2:
            insert3d_bwd_kernel<float, 2><<<b, 256, 0, st>>>((const float*)grad_image, coordinates, n, channels,
                                                             (int)d, (int)h, (int)w, (float*)grad_values, nearest);
            break;
        default:
            insert3d_bwd_kernel<double, 2><<<b, 256, 0, st>>>((const double*)grad_image, coordinates, n, channels,
                                                              (int)d, (int)h, (int)w, (double*)grad_values, nearest);
    }
    return check_launch("insert3d_bwd_kernel");
}
