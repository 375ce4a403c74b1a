// Central-slice insertion into an fftshifted rfft volume plus its weight
// volume (insert_central_slices_rfft_3d, _insert_central_slices_rfft_3d.py:9-106,
// _insert_into_3d_dft :213-286, _insert_into_3d_dft_linear :289-406).
//
// Splat stage: one thread per source pixel.  Pixels outside fftfreq_max and
// the Friedel-redundant half of the x=0 column (x == 0 and y < 0) are skipped;
// the rotated frequency is redirected (conjugating the data) when x' < 0;
// points with any array coordinate outside [0, n-1] are dropped whole; the
// eight floor/ceil corners receive data*w and w with the reference's float32
// weights ((1-t) and t products, left to right).
//
// Mirror stage: the reference also inserts conj(data)*w at ((d-z)%d, (h-y)%h, 0)
// for every corner that lands on the x=0 plane except the DC voxel.  Summed
// over all points that equals, per plane voxel v with partner m(v),
//   out[v] = acc[v] + conj(acc[m(v)])   unless m(v) is the DC voxel,
// which one pass over the plane applies after the last splat (m is an
// involution, so each thread owns the pair {v, m(v)}).
#include <cuda_runtime.h>

#include "capi_util.cuh"
#include "slice_common.cuh"

namespace tt {

constexpr int kInsertThreads = 256;

template <typename R>
struct cplx;
template <>
struct cplx<float> {
    using T = float2;
};
template <>
struct cplx<double> {
    using T = double2;
};

__device__ __forceinline__ void accumulate(float2* vol, float* w, int64_t i, float re, float im, float wt) {
    atomicAdd(vol + i, make_float2(re, im));
    atomicAdd(w + i, wt);
}
__device__ __forceinline__ void accumulate(double2* vol, double* w, int64_t i, double re, double im, double wt) {
    atomicAdd(&vol[i].x, re);
    atomicAdd(&vol[i].y, im);
    atomicAdd(w + i, wt);
}

template <typename R>
__global__ void __launch_bounds__(kInsertThreads)
insert_splat_kernel(const typename cplx<R>::T* __restrict__ img, const void* __restrict__ rot,
                    typename cplx<R>::T* __restrict__ vol, R* __restrict__ wts, SliceGeom g, int tiles) {
    __shared__ float m[9];
    const int64_t s = blockIdx.x / tiles;
    const int tile = blockIdx.x - (int)(s * tiles);
    if (threadIdx.x < 9) m[threadIdx.x] = prep_rotation_elem(rot, g.rot_f64, s, threadIdx.x, g, false);
    __syncthreads();
    const int P = g.img_h * g.wr;
    const int pix = tile * kInsertThreads + threadIdx.x;
    if (pix >= P) return;
    const int iy = pix / g.wr, ix = pix - iy * g.wr;
    const float qy = shifted_freq(iy, g.img_h, g.inv_h);
    const float qx = __fmul_rn((float)ix, g.inv_w);
    if (!in_fmax(g, qy, qx)) return;
    if (qx == 0.0f && qy < 0.0f) return;  // Friedel-redundant source pixel
    float p[3], c[3];
    rotate_slice_point(m, qy, qx, p);
    const typename cplx<R>::T d = img[(s * g.img_h + slice_row(g, iy)) * (int64_t)g.wr + ix];
    R dre = d.x, dim = d.y;
    if (p[2] < 0.0f) {
        p[0] = -p[0];
        p[1] = -p[1];
        p[2] = -p[2];
        dim = -dim;
    }
    to_dft_coords(g, p, c);
    if (!inside_volume(g, c)) return;
    const float z0 = floorf(c[0]), y0 = floorf(c[1]), x0 = floorf(c[2]);
    const float tz = c[0] - z0, ty = c[1] - y0, tx = c[2] - x0;
    const int iz0 = (int)z0, iy0 = (int)y0, ix0 = (int)x0;
    const int iz1 = (int)ceilf(c[0]), iy1 = (int)ceilf(c[1]), ix1 = (int)ceilf(c[2]);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int bz = (k >> 2) & 1, by = (k >> 1) & 1, bx = k & 1;
        const float fz = bz ? tz : 1.0f - tz;
        const float fy = by ? ty : 1.0f - ty;
        const float fx = bx ? tx : 1.0f - tx;
        const float w = (fz * fy) * fx;
        if (w == 0.0f) continue;  // adds nothing (ceil == floor or zero fraction)
        const int64_t vi = vox_index(g, bz ? iz1 : iz0, by ? iy1 : iy0, bx ? ix1 : ix0);
        const R rw = (R)w;
        accumulate(vol, wts, vi, dre * rw, dim * rw, rw);
    }
}

// Friedel completion of the x=0 plane (see file comment).  `vol` holds
// `channels` volumes of (d, h, w) complex; `wts` one (d, h, w) weight volume.
template <typename R>
__global__ void mirror_x0_kernel(typename cplx<R>::T* __restrict__ vol, R* __restrict__ wts, int64_t channels,
                                 int d, int h, int w) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)d * h) return;
    const int z = (int)(idx / h), y = (int)(idx - (int64_t)z * h);
    const int zm = (d - z) % d, ym = (h - y) % h;
    const int64_t u = (int64_t)zm * h + ym;
    if (u < idx) return;  // the pair is owned by its lower index
    const bool v_dc = (z == d / 2) && (y == h / 2);
    const bool u_dc = (zm == d / 2) && (ym == h / 2);
    const int64_t plane = (int64_t)d * h * w;
    for (int64_t ch = 0; ch < channels; ch++) {
        typename cplx<R>::T* base = vol + ch * plane;
        const typename cplx<R>::T a = base[idx * w];
        if (u == idx) {
            if (!u_dc) {
                typename cplx<R>::T o;
                o.x = a.x + a.x;
                o.y = a.y - a.y;
                base[idx * w] = o;
            }
        } else {
            const typename cplx<R>::T b = base[u * w];
            typename cplx<R>::T oa = a, ob = b;
            if (!u_dc) {
                oa.x = a.x + b.x;
                oa.y = a.y - b.y;
            }
            if (!v_dc) {
                ob.x = b.x + a.x;
                ob.y = b.y - a.y;
            }
            base[idx * w] = oa;
            base[u * w] = ob;
        }
    }
    if (wts) {
        const R a = wts[idx * w];
        if (u == idx) {
            if (!u_dc) wts[idx * w] = a + a;
        } else {
            const R b = wts[u * w];
            if (!u_dc) wts[idx * w] = a + b;
            if (!v_dc) wts[u * w] = b + a;
        }
    }
}

}  // namespace tt

using namespace tt;

extern "C" int tt_insert_central_slices_rfft_3d(const void* image_rfft, int32_t complex128,
                                                const void* rotation_matrices, void* volume_rfft, void* weights,
                                                const tt_slice_params* p, void* stream) {
    if (int e = validate_params(p)) return e;
    if (p->n == 0) return TT_OK;
    if (!image_rfft || !rotation_matrices || !volume_rfft || !weights)
        return fail(TT_ERR_INVALID, "insert: NULL pointer argument");
    if (p->vol_d != p->img_d || p->vol_h != p->img_h || p->vol_w != p->img_w / 2 + 1)
        return fail(TT_ERR_INVALID, "insert: volume dims (%lld, %lld, %lld) are not the rfft of volume_shape",
                    (long long)p->vol_d, (long long)p->vol_h, (long long)p->vol_w);
    SliceGeom g = make_geom(*p);
    const int P = g.img_h * g.wr;
    const int tiles = (P + kInsertThreads - 1) / kInsertThreads;
    const int64_t blocks = (int64_t)g.n * tiles;
    if (blocks > 0x7fffffffLL) return fail(TT_ERR_INVALID, "insert: too many blocks");
    cudaStream_t st = as_stream(stream);
    if (complex128)
        insert_splat_kernel<double><<<(unsigned)blocks, kInsertThreads, 0, st>>>(
            (const double2*)image_rfft, rotation_matrices, (double2*)volume_rfft, (double*)weights, g, tiles);
    else
        insert_splat_kernel<float><<<(unsigned)blocks, kInsertThreads, 0, st>>>(
            (const float2*)image_rfft, rotation_matrices, (float2*)volume_rfft, (float*)weights, g, tiles);
    return check_launch("insert_splat_kernel");
}

extern "C" int tt_friedel_mirror_x0(void* volume_rfft, void* weights, int32_t complex128, int64_t channels,
                                    int64_t d, int64_t h, int64_t w_rfft, void* stream) {
    if (!volume_rfft) return fail(TT_ERR_INVALID, "mirror: NULL volume");
    if (channels < 1 || d < 1 || h < 1 || w_rfft < 1) return fail(TT_ERR_INVALID, "mirror: bad dims");
    const int64_t total = d * h;
    const unsigned blocks = (unsigned)((total + 255) / 256);
    cudaStream_t st = as_stream(stream);
    if (complex128)
        mirror_x0_kernel<double><<<blocks, 256, 0, st>>>((double2*)volume_rfft, (double*)weights, channels, (int)d,
                                                         (int)h, (int)w_rfft);
    else
        mirror_x0_kernel<float><<<blocks, 256, 0, st>>>((float2*)volume_rfft, (float*)weights, channels, (int)d,
                                                        (int)h, (int)w_rfft);
    return check_launch("mirror_x0_kernel");
}
