// Deterministic insertion through 64-bit fixed-point accumulators, and the
// absmax pre-pass that sets their scale (the scale rule is in fixed_point.cuh).
//
// The splat is the one of insert.cu (same pixels, redirect, bounds and float32
// corner weights); only the accumulation differs.  The finalize stage does the
// Friedel completion of the x=0 plane on the integers, exactly, and converts
// each sum back once.
#include <cuda_runtime.h>

#include "capi_util.cuh"
#include "fixed_point.cuh"
#include "slice_common.cuh"
#include "slice_ops.cuh"

namespace tt {

// Grid-stride max of |x| as float32 bit patterns; one atomicMax per warp.
template <bool F64>
__global__ void absmax_kernel(const void* __restrict__ data, int64_t count, uint32_t* __restrict__ out) {
    uint32_t m = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (F64) {
        const double* x = (const double*)data;
        for (int64_t j = i; j < count; j += stride)
            m = max(m, __float_as_uint(__double2float_ru(fabs(__ldcs(x + j)))));
    } else {
        const float* x = (const float*)data;
        const int64_t n4 = ((uintptr_t)x & 15) == 0 ? count / 4 : 0;
        const float4* x4 = (const float4*)x;
        for (int64_t j = i; j < n4; j += stride) {
            const float4 v = __ldcs(x4 + j);
            m = max(m, max(max(__float_as_uint(fabsf(v.x)), __float_as_uint(fabsf(v.y))),
                           max(__float_as_uint(fabsf(v.z)), __float_as_uint(fabsf(v.w)))));
        }
        for (int64_t j = n4 * 4 + i; j < count; j += stride) m = max(m, __float_as_uint(fabsf(x[j])));
    }
    m = __reduce_max_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

int launch_fixed_absmax(const void* data, int is_f64, int64_t count, uint32_t* absmax, cudaStream_t st) {
    if (count <= 0) return TT_OK;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t want = (count + 1023) / 1024;
    const int64_t cap = (int64_t)sms * 8;
    const unsigned blocks = (unsigned)(want < cap ? want : cap);
    if (is_f64)
        absmax_kernel<true><<<blocks, 256, 0, st>>>(data, count, absmax);
    else
        absmax_kernel<false><<<blocks, 256, 0, st>>>(data, count, absmax);
    return check_launch("absmax_kernel");
}

// Fixed-point splat of one complex64 source pixel with lane pairs: lanes 2j
// and 2j+1 take the same pixel (pixels j and j + 16 in two rounds); per row of
// the cell they add (re | im) of the x-low corner, (w | w) of the two corners
// and (re | im) of the x-high corner, so an instruction's two words share a
// 32-byte voxel slot or lie in adjacent ones: 4 sector operations per row
// where one word per lane takes 6.  Same corners, weights ((fz * fy) * fx) and
// rounded integers as the FixedSplat path.  Must be called by all 32 lanes of
// the warp (has_pixel false where the tile overhangs the slice).
__device__ __forceinline__ void insert_point_fixed_paired(const float2* __restrict__ img, const float* m,
                                                          unsigned long long* __restrict__ acc, double sd, double sw,
                                                          const SliceGeom& g, int64_t s, bool has_pixel, int iy,
                                                          int ix) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, odd = lane & 1;
    float dre = 0.f, dim = 0.f;
    float c[3] = {-1.f, 0.f, 0.f};  // c[0] < 0: no point
    if (has_pixel) {
        const float qy = shifted_freq(iy, g.img_h, g.inv_h);
        const float qx = __fmul_rn((float)ix, g.inv_w);
        if (insert_pixel_kept(g, qy, qx)) {
            const float2 d = load_slice(img + (s * g.slice_rows + slice_row(g, iy)) * (int64_t)g.wr + ix);
            bool cj;
            float ci[3];
            if (insert_coords(g, m, qy, qx, cj, ci)) {
                dre = d.x;
                dim = cj ? -d.y : d.y;
                c[0] = ci[0];
                c[1] = ci[1];
                c[2] = ci[2];
            }
        }
    }
#pragma unroll
    for (int half = 0; half < 2; half++) {
        const int src = (lane >> 1) + 16 * half;
        const float sre = __shfl_sync(full, dre, src), sim = __shfl_sync(full, dim, src);
        float sc[3];
#pragma unroll
        for (int a = 0; a < 3; a++) sc[a] = __shfl_sync(full, c[a], src);
        if (sc[0] < 0.0f) continue;
        InsertCell k;
        cell_at(sc, k);
        const double sv = (double)(odd ? sim : sre);
#pragma unroll
        for (int zy = 0; zy < 4; zy++) {
            const int bz = zy >> 1, by = zy & 1;
            const float wzy = (bz ? k.tz : 1.0f - k.tz) * (by ? k.ty : 1.0f - k.ty);
            const float w0 = wzy * (1.0f - k.tx), w1 = wzy * k.tx;
            const int z = bz ? k.iz1 : k.iz0, y = by ? k.iy1 : k.iy0;
            const int64_t v0 = vox_index(g, z, y, k.ix0), v1 = vox_index(g, z, y, k.ix1);
            if (w0 != 0.0f) fixed_add(acc + v0 * 4 + odd, sv * (double)w0 * sd);
            const float wc = odd ? w1 : w0;
            if (wc != 0.0f) fixed_add(acc + (odd ? v1 : v0) * 4 + 2, (double)wc * 1.0 * sw);
            if (w1 != 0.0f) fixed_add(acc + v1 * 4 + odd, sv * (double)w1 * sd);
        }
    }
}

// One block per (slice, row of tiles), as insert_accumulate_kernel, in
// z-phases for accumulators larger than the L2 (integer sums: bit-identical
// in any order).
template <typename R>
__global__ void __launch_bounds__(kTileThreads)
insert_fixed_kernel(const typename Acc<R>::C* __restrict__ img, const void* __restrict__ rot,
                    unsigned long long* __restrict__ acc, const uint32_t* __restrict__ absmax, int slices_log2,
                    SliceGeom g, int phase, int nphase) {
    __shared__ float m[9];
    const int tx_tiles = tiles_x_of(g.wr);
    const int rows = (g.img_h + kTileY - 1) / kTileY;
    const int64_t s = blockIdx.x / rows;
    const int ty = blockIdx.x - (int)(s * rows);
    if (threadIdx.x < 9) m[threadIdx.x] = prep_rotation_elem(rot, g.rot_f64, s, threadIdx.x, g, false);
    __syncthreads();
    const FixedSplat sink{acc, fixed_data_scale(*absmax, slices_log2), fixed_weight_scale(slices_log2)};
    for (int tx = 0; tx < tx_tiles; tx++) {
        if (nphase > 1 && insert_tile_phase(g, m, min(ty * kTileY + kTileY / 2, g.img_h - 1),
                                            min(tx * kTileX + kTileX / 2, g.wr - 1), nphase) != phase)
            continue;
        int iy, ix;
        const bool has_pixel = tile_pixel(g, ty * tx_tiles + tx, iy, ix);
        if constexpr (sizeof(R) == 4)
            insert_point_fixed_paired(img, m, acc, sink.sd, sink.sw, g, s, has_pixel, iy, ix);  // every lane
        else if (has_pixel)
            insert_point_to<R>(img, m, sink, g, s, iy, ix);
    }
}

// Fixed-point accumulator -> (volume, weights), with the Friedel completion of
// the x=0 plane (out[v] = acc[v] + conj(acc[m(v)]) unless m(v) is DC) done on
// the integers.  Weights come from channel 0.
template <typename R>
__global__ void insert_fixed_finalize_kernel(const long long* __restrict__ acc, typename Acc<R>::C* __restrict__ vol,
                                             R* __restrict__ wts, const uint32_t* __restrict__ absmax,
                                             int slices_log2, int64_t channels, int d, int h, int w) {
    const int64_t per = (int64_t)d * h * w;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= channels * per) return;
    const int64_t ch = idx / per, r = idx - ch * per;
    const longlong4 a = reinterpret_cast<const longlong4*>(acc)[idx];
    unsigned long long re = (unsigned long long)a.x, im = (unsigned long long)a.y, wt = (unsigned long long)a.z;
    const int x = (int)(r % w);
    if (x == 0) {
        const int64_t zy = r / w;
        const int z = (int)(zy / h), y = (int)(zy % h);
        const int zm = (d - z) % d, ym = (h - y) % h;
        if (!(zm == d / 2 && ym == h / 2)) {
            const longlong4 b = reinterpret_cast<const longlong4*>(acc)[ch * per + ((int64_t)zm * h + ym) * w];
            re += (unsigned long long)b.x;
            im -= (unsigned long long)b.y;
            wt += (unsigned long long)b.z;
        }
    }
    const double inv_d = 1.0 / fixed_data_scale(*absmax, slices_log2);
    const double inv_w = 1.0 / fixed_weight_scale(slices_log2);
    typename Acc<R>::C o;
    o.x = (R)((double)(long long)re * inv_d);
    o.y = (R)((double)(long long)im * inv_d);
    vol[idx] = o;
    if (ch == 0 && wts) wts[r] = (R)((double)(long long)wt * inv_w);
}

static int check_fixed_insert_params(const tt_slice_params* p) {
    if (int e = validate_params(p)) return e;
    if (p->vol_d != p->img_d || p->vol_h != p->img_h || p->vol_w != p->img_w / 2 + 1)
        return fail(TT_ERR_INVALID, "insert: volume dims (%lld, %lld, %lld) are not the rfft of volume_shape",
                    (long long)p->vol_d, (long long)p->vol_h, (long long)p->vol_w);
    return TT_OK;
}

int insert_phases(size_t acc_bytes);  // insert.cu

int launch_insert_fixed(const void* image_rfft, int32_t complex128, const void* rot, void* acc,
                        const uint32_t* absmax, int64_t max_slices, const tt_slice_params* p, cudaStream_t st) {
    SliceGeom g = make_geom(*p);
    const int64_t items = (int64_t)g.n * ((g.img_h + kTileY - 1) / kTileY);
    if (items > 0x7fffffffLL) return fail(TT_ERR_INVALID, "insert: too many blocks");
    const int l = ceil_log2(max_slices);
    const int nphase = insert_phases((size_t)((int64_t)g.D * g.H * g.W) * 4 * sizeof(long long));
    for (int ph = 0; ph < nphase; ph++) {
        if (complex128)
            insert_fixed_kernel<double><<<(unsigned)items, kTileThreads, 0, st>>>(
                (const double2*)image_rfft, rot, (unsigned long long*)acc, absmax, l, g, ph, nphase);
        else
            insert_fixed_kernel<float><<<(unsigned)items, kTileThreads, 0, st>>>(
                (const float2*)image_rfft, rot, (unsigned long long*)acc, absmax, l, g, ph, nphase);
        if (int e = check_launch("insert_fixed_kernel")) return e;
    }
    return TT_OK;
}

int launch_insert_fixed_finalize(const void* acc, int32_t complex128, int64_t channels, int64_t d, int64_t h,
                                 int64_t w, const uint32_t* absmax, int64_t max_slices, void* volume, void* weights,
                                 cudaStream_t st) {
    const int64_t total = channels * d * h * w;
    const unsigned blocks = (unsigned)((total + 255) / 256);
    const int l = ceil_log2(max_slices);
    if (complex128)
        insert_fixed_finalize_kernel<double><<<blocks, 256, 0, st>>>((const long long*)acc, (double2*)volume,
                                                                     (double*)weights, absmax, l, channels, (int)d,
                                                                     (int)h, (int)w);
    else
        insert_fixed_finalize_kernel<float><<<blocks, 256, 0, st>>>((const long long*)acc, (float2*)volume,
                                                                    (float*)weights, absmax, l, channels, (int)d,
                                                                    (int)h, (int)w);
    return check_launch("insert_fixed_finalize_kernel");
}

// One-shot deterministic insertion over a workspace of
// [256-byte header: absmax word][fixed-point accumulator].
int insert_deterministic(const void* image_rfft, int32_t complex128, const void* rot, void* volume, void* weights,
                         void* workspace, const tt_slice_params* p, cudaStream_t st) {
    const size_t acc_bytes = tt_insert_fixed_accumulator_bytes(1, p->vol_d, p->vol_h, p->vol_w);
    cudaError_t e = cudaMemsetAsync(workspace, 0, kFixedHeaderBytes + acc_bytes, st);
    if (e != cudaSuccess) return fail(TT_ERR_CUDA, "insert: memset: %s", cudaGetErrorString(e));
    uint32_t* absmax = (uint32_t*)workspace;
    void* acc = (char*)workspace + kFixedHeaderBytes;
    const int64_t n = p->n > 0 ? p->n : 1;
    if (p->n > 0) {
        const int64_t count = p->n * p->img_h * (p->img_w / 2 + 1) * 2;
        if (int r = launch_fixed_absmax(image_rfft, complex128, count, absmax, st)) return r;
        if (int r = launch_insert_fixed(image_rfft, complex128, rot, acc, absmax, n, p, st)) return r;
    }
    return launch_insert_fixed_finalize(acc, complex128, 1, p->vol_d, p->vol_h, p->vol_w, absmax, n, volume, weights,
                                        st);
}

}  // namespace tt

using namespace tt;

extern "C" size_t tt_insert_fixed_accumulator_bytes(int64_t channels, int64_t d, int64_t h, int64_t w_rfft) {
    if (channels < 1 || d < 1 || h < 1 || w_rfft < 1) return 0;
    return (size_t)(channels * d * h * w_rfft) * 4 * sizeof(long long);
}

extern "C" int tt_fixed_absmax(const void* data, int32_t is_f64, int64_t count, uint32_t* absmax_bits,
                               void* stream) {
    if (count < 0) return fail(TT_ERR_INVALID, "fixed_absmax: count must be >= 0");
    if (count == 0) return TT_OK;
    if (!data || !absmax_bits) return fail(TT_ERR_INVALID, "fixed_absmax: NULL pointer argument");
    return launch_fixed_absmax(data, is_f64, count, absmax_bits, as_stream(stream));
}

extern "C" int tt_insert_fixed_accumulate(const void* image_rfft, int32_t complex128, const void* rotation_matrices,
                                          void* accumulator, const uint32_t* absmax_bits, int64_t max_slices,
                                          const tt_slice_params* p, void* stream) {
    if (int e = check_fixed_insert_params(p)) return e;
    if (max_slices < p->n || max_slices < 1)
        return fail(TT_ERR_INVALID, "insert_fixed_accumulate: max_slices (%lld) below the %lld slices of this call",
                    (long long)max_slices, (long long)p->n);
    if (p->n == 0) return TT_OK;
    if (!image_rfft || !rotation_matrices || !accumulator || !absmax_bits)
        return fail(TT_ERR_INVALID, "insert_fixed_accumulate: NULL pointer argument");
    return launch_insert_fixed(image_rfft, complex128, rotation_matrices, accumulator, absmax_bits, max_slices, p,
                               as_stream(stream));
}

extern "C" int tt_insert_fixed_finalize(const void* accumulator, int32_t complex128, int64_t channels, int64_t d,
                                        int64_t h, int64_t w_rfft, const uint32_t* absmax_bits, int64_t max_slices,
                                        void* volume_rfft, void* weights, void* stream) {
    if (!accumulator || !volume_rfft || !absmax_bits)
        return fail(TT_ERR_INVALID, "insert_fixed_finalize: NULL pointer argument");
    if (channels < 1 || d < 1 || h < 1 || w_rfft < 1) return fail(TT_ERR_INVALID, "insert_fixed_finalize: bad dims");
    if (max_slices < 1) return fail(TT_ERR_INVALID, "insert_fixed_finalize: max_slices must be >= 1");
    return launch_insert_fixed_finalize(accumulator, complex128, channels, d, h, w_rfft, absmax_bits, max_slices,
                                        volume_rfft, weights, as_stream(stream));
}
