// Elementwise kernels around the FFTs of the real-space wrappers
// project_3d_to_2d (torch_fourier_slice/project.py:48-92) and
// backproject_2d_to_3d (torch_fourier_slice/backproject.py:48-92).
// Each replaces a chain of pad / multiply / fftshift / divide / crop passes by
// one read and one write, folding every shift into the index arithmetic.
//
// Shift conventions (torch.fft): fftshift(x)[i] = x[(i - n/2) mod n],
// ifftshift(x)[i] = x[(i + n/2) mod n], n/2 rounded down.
#include <cuda_runtime.h>

#include "capi_util.cuh"

namespace tt {

// i mod n for i in (-n, 2n), the range every shift here produces.
__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// f32(k) * f32(1/n) for unshifted index k of an axis of length n.
__device__ __forceinline__ float fftfreq_at(int k, int n, float inv_n) {
    const int kk = (k < (n + 1) / 2) ? k : k - n;
    return __fmul_rn((float)kk, inv_n);
}

// Frequency at fftshifted position a of an axis of length n.
__device__ __forceinline__ float shifted_fftfreq(int a, int n, float inv_n) {
    return fftfreq_at(wrap(a - n / 2, n), n, inv_n);
}

// sinc(|f|)^2 from the squared frequency norm's two leading terms (f0^2 +
// f1^2, rounded as the reference sums them) and the third frequency, on the
// fftshifted norm grid (fftfreq_grid(rfft=False, fftshift=True, norm=True)).
__device__ __forceinline__ float sinc2_from(float f01, float f2) {
    const float r = __fsqrt_rn(__fadd_rn(f01, __fmul_rn(f2, f2)));
    if (r == 0.0f) return 1.0f;
    const float px = __fmul_rn(3.14159265358979323846f, r);
    const float s = __fdiv_rn(sinpif(r), px);
    return s * s;
}

// The kernels below run one block per row of their output (the leading
// indices are split once per block in 64-bit arithmetic) and stride the row
// with the block's threads, so each element costs 32-bit index work only and
// consecutive threads write consecutive addresses.
inline int row_threads(int64_t row_len) {
    const int64_t t = (row_len + 31) / 32 * 32;
    return (int)(t < 32 ? 32 : (t > 256 ? 256 : t));
}

// out (n^3, FFT order) = fftshift(pad(vol, p) * sinc^2); row = (i, j).
template <typename T>
__global__ void project_prepare_kernel(const T* __restrict__ vol, T* __restrict__ out, int d, int p, int n,
                                       float inv_n) {
    const int64_t row = blockIdx.x;
    const int i = (int)(row / n), j = (int)(row - (int64_t)i * n);
    const int a0 = wrap(i - n / 2, n), a1 = wrap(j - n / 2, n);
    const int v0 = a0 - p, v1 = a1 - p;
    T* o = out + row * n;
    if (!(v0 >= 0 && v0 < d && v1 >= 0 && v1 < d)) {
        for (int k = threadIdx.x; k < n; k += blockDim.x) o[k] = (T)0;
        return;
    }
    const float f0 = shifted_fftfreq(a0, n, inv_n), f1 = shifted_fftfreq(a1, n, inv_n);
    const float f01 = __fadd_rn(__fmul_rn(f0, f0), __fmul_rn(f1, f1));
    const T* src = vol + ((int64_t)v0 * d + v1) * d;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int a2 = wrap(k - n / 2, n), v2 = a2 - p;
        o[k] = (v2 >= 0 && v2 < d) ? src[v2] * (T)sinc2_from(f01, shifted_fftfreq(a2, n, inv_n)) : (T)0;
    }
}

// out (m, h-2p, w-2p) = crop(ifftshift(images, (-2,-1)), p), images (m, h, w); row = (b, i).
template <typename T>
__global__ void recentre_crop_2d_kernel(const T* __restrict__ img, T* __restrict__ out, int h, int w, int p) {
    const int ch = h - 2 * p, cw = w - 2 * p;
    const int64_t row = blockIdx.x;
    const int64_t b = row / ch;
    const int i = (int)(row - b * ch);
    const T* src = img + (b * h + wrap(i + p + h / 2, h)) * (int64_t)w;
    T* o = out + row * cw;
    for (int j = threadIdx.x; j < cw; j += blockDim.x) o[j] = src[wrap(j + p + w / 2, w)];
}

// out (m, n, n) = fftshift(pad(images, p), (-2,-1)), images (m, d, d); row = (b, i).
template <typename T>
__global__ void pad_fftshift_2d_kernel(const T* __restrict__ img, T* __restrict__ out, int d, int p, int n) {
    const int64_t row = blockIdx.x;
    const int64_t b = row / n;
    const int i = (int)(row - b * n);
    const int a0 = wrap(i - n / 2, n) - p;
    T* o = out + row * n;
    if (a0 < 0 || a0 >= d) {
        for (int j = threadIdx.x; j < n; j += blockDim.x) o[j] = (T)0;
        return;
    }
    const T* src = img + (b * d + a0) * (int64_t)d;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int a1 = wrap(j - n / 2, n) - p;
        o[j] = (a1 >= 0 && a1 < d) ? src[a1] : (T)0;
    }
}

template <typename R>
struct C2;
template <>
struct C2<float> {
    using T = float2;
    using A = float4;
};
template <>
struct C2<double> {
    using T = double2;
    using A = double4;
};

// Backprojection normalisation of `channels` insertion accumulators
// ((re, im, w, 0) slots of fftshifted rfft volumes (d, h, w); every channel
// carries the same weights): Friedel completion of the x=0 plane, division by
// max(weights, 1), written ifftshifted along (d, h) for the 3D irfft.
// Row = (channel, i, j) of the output.
template <typename R>
__global__ void normalize_unshift_kernel(const typename C2<R>::A* __restrict__ acc,
                                         typename C2<R>::T* __restrict__ out, int d, int h, int w) {
    const int64_t row = blockIdx.x;
    const int64_t dh = (int64_t)d * h, per = dh * w;
    const int64_t ch = row / dh;
    const int rr = (int)(row - ch * dh);
    const int i = rr / h, j = rr - i * h;
    const int z = wrap(i + d / 2, d), y = wrap(j + h / 2, h);  // source (shifted) voxel row
    const int64_t src = ((int64_t)z * h + y) * w;
    const typename C2<R>::A* a_ch = acc + ch * per;
    typename C2<R>::T* o = out + row * w;
    for (int k = threadIdx.x; k < w; k += blockDim.x) {
        // the interpolation weights live in channel 0 (the channels share them)
        const typename C2<R>::A a = a_ch[src + k];
        R re = a.x, im = a.y, wt = acc[src + k].z;
        if (k == 0) {
            const int zm = (d - z) % d, ym = (h - y) % h;
            const bool m_dc = (zm == d / 2) && (ym == h / 2);
            if (!m_dc) {
                const int64_t msrc = ((int64_t)zm * h + ym) * w;
                const typename C2<R>::A u = a_ch[msrc];
                re += u.x;
                im -= u.y;
                wt += acc[msrc].z;
            }
        }
        const R den = wt < (R)1 ? (R)1 : wt;
        typename C2<R>::T v;
        v.x = re / den;
        v.y = im / den;
        o[k] = v;
    }
}

// out (n0-2p, n1-2p, n2-2p) = crop(ifftshift(vol) / sinc^2, p), vol (n0, n1, n2)
// real; the sinc^2 grid is that of the (n0, n1, n2) array.  Row = (i, j) of the output.
template <typename T>
__global__ void backproject_finish_kernel(const T* __restrict__ vol, T* __restrict__ out, int n0, int n1, int n2,
                                          int p, float i0, float i1, float i2) {
    const int c1 = n1 - 2 * p, c2 = n2 - 2 * p;
    const int64_t row = blockIdx.x;
    const int ci = (int)(row / c1), cj = (int)(row - (int64_t)ci * c1);
    const int i = ci + p, j = cj + p;
    const T* src = vol + ((int64_t)wrap(i + n0 / 2, n0) * n1 + wrap(j + n1 / 2, n1)) * n2;
    const float f0 = shifted_fftfreq(i, n0, i0), f1 = shifted_fftfreq(j, n1, i1);
    const float f01 = __fadd_rn(__fmul_rn(f0, f0), __fmul_rn(f1, f1));
    T* o = out + row * c2;
    for (int ck = threadIdx.x; ck < c2; ck += blockDim.x) {
        const int k = ck + p;
        o[ck] = src[wrap(k + n2 / 2, n2)] / (T)sinc2_from(f01, shifted_fftfreq(k, n2, i2));
    }
}

}  // namespace tt

using namespace tt;

extern "C" int tt_project_prepare(const void* volume, int32_t is_f64, int64_t d, int64_t pad, void* out,
                                  void* stream) {
    if (!volume || !out || d < 1 || pad < 0) return fail(TT_ERR_INVALID, "project_prepare: bad arguments");
    const int64_t n = d + 2 * pad;
    if (n > (1 << 15)) return fail(TT_ERR_INVALID, "project_prepare: padded box above 32768");
    const float inv_n = (float)(1.0 / (double)n);
    const unsigned rows = (unsigned)(n * n);
    const int th = row_threads(n);
    if (is_f64)
        project_prepare_kernel<double><<<rows, th, 0, as_stream(stream)>>>((const double*)volume, (double*)out,
                                                                           (int)d, (int)pad, (int)n, inv_n);
    else
        project_prepare_kernel<float><<<rows, th, 0, as_stream(stream)>>>((const float*)volume, (float*)out,
                                                                          (int)d, (int)pad, (int)n, inv_n);
    return check_launch("project_prepare_kernel");
}

extern "C" int tt_recentre_crop_2d(const void* images, int32_t is_f64, int64_t m, int64_t h, int64_t w, int64_t pad,
                                   void* out, void* stream) {
    if (!images || !out || m < 0 || h < 1 || w < 1 || pad < 0 || 2 * pad >= h || 2 * pad >= w)
        return fail(TT_ERR_INVALID, "recentre_crop_2d: bad arguments");
    if (m == 0) return TT_OK;
    const int64_t rows = m * (h - 2 * pad);
    if (h > (1 << 30) || w > (1 << 30) || rows > 0x7fffffffLL)
        return fail(TT_ERR_INVALID, "recentre_crop_2d: too many rows");
    const int th = row_threads(w - 2 * pad);
    if (is_f64)
        recentre_crop_2d_kernel<double><<<(unsigned)rows, th, 0, as_stream(stream)>>>(
            (const double*)images, (double*)out, (int)h, (int)w, (int)pad);
    else
        recentre_crop_2d_kernel<float><<<(unsigned)rows, th, 0, as_stream(stream)>>>(
            (const float*)images, (float*)out, (int)h, (int)w, (int)pad);
    return check_launch("recentre_crop_2d_kernel");
}

extern "C" int tt_pad_fftshift_2d(const void* images, int32_t is_f64, int64_t m, int64_t d, int64_t pad, void* out,
                                  void* stream) {
    if (!images || !out || m < 0 || d < 1 || pad < 0) return fail(TT_ERR_INVALID, "pad_fftshift_2d: bad arguments");
    if (m == 0) return TT_OK;
    const int64_t n = d + 2 * pad, rows = m * n;
    if (n > (1 << 30) || rows > 0x7fffffffLL) return fail(TT_ERR_INVALID, "pad_fftshift_2d: too many rows");
    const int th = row_threads(n);
    if (is_f64)
        pad_fftshift_2d_kernel<double><<<(unsigned)rows, th, 0, as_stream(stream)>>>(
            (const double*)images, (double*)out, (int)d, (int)pad, (int)n);
    else
        pad_fftshift_2d_kernel<float><<<(unsigned)rows, th, 0, as_stream(stream)>>>(
            (const float*)images, (float*)out, (int)d, (int)pad, (int)n);
    return check_launch("pad_fftshift_2d_kernel");
}

extern "C" int tt_backproject_normalize(const void* accumulator, int32_t complex128, int64_t channels, int64_t d,
                                        int64_t h, int64_t w_rfft, void* out, void* stream) {
    if (!accumulator || !out || channels < 1 || d < 1 || h < 1 || w_rfft < 1)
        return fail(TT_ERR_INVALID, "backproject_normalize: bad arguments");
    if (accumulator == out) return fail(TT_ERR_INVALID, "backproject_normalize: out must not alias the input");
    const int64_t rows = channels * d * h;
    if (d > (1 << 30) || h > (1 << 30) || w_rfft > (1 << 30) || rows > 0x7fffffffLL)
        return fail(TT_ERR_INVALID, "backproject_normalize: too many rows");
    const int th = row_threads(w_rfft);
    if (complex128)
        normalize_unshift_kernel<double><<<(unsigned)rows, th, 0, as_stream(stream)>>>(
            (const double4*)accumulator, (double2*)out, (int)d, (int)h, (int)w_rfft);
    else
        normalize_unshift_kernel<float><<<(unsigned)rows, th, 0, as_stream(stream)>>>(
            (const float4*)accumulator, (float2*)out, (int)d, (int)h, (int)w_rfft);
    return check_launch("normalize_unshift_kernel");
}

extern "C" int tt_backproject_finish(const void* volume, int32_t is_f64, int64_t channels, int64_t n0, int64_t n1,
                                     int64_t n2, int64_t pad, void* out, void* stream) {
    if (!volume || !out || channels < 1 || n0 < 1 || n1 < 1 || n2 < 1 || pad < 0 || 2 * pad >= n0 ||
        2 * pad >= n1 || 2 * pad >= n2)
        return fail(TT_ERR_INVALID, "backproject_finish: bad arguments");
    if (n0 > (1 << 15) || n1 > (1 << 15) || n2 > (1 << 15))
        return fail(TT_ERR_INVALID, "backproject_finish: box above 32768");
    const int64_t per = (n0 - 2 * pad) * (n1 - 2 * pad) * (n2 - 2 * pad), in = n0 * n1 * n2;
    const unsigned rows = (unsigned)((n0 - 2 * pad) * (n1 - 2 * pad));
    const int th = row_threads(n2 - 2 * pad);
    const float i0 = (float)(1.0 / (double)n0), i1 = (float)(1.0 / (double)n1), i2 = (float)(1.0 / (double)n2);
    for (int64_t ch = 0; ch < channels; ch++) {
        if (is_f64)
            backproject_finish_kernel<double><<<rows, th, 0, as_stream(stream)>>>(
                (const double*)volume + ch * in, (double*)out + ch * per, (int)n0, (int)n1, (int)n2, (int)pad, i0,
                i1, i2);
        else
            backproject_finish_kernel<float><<<rows, th, 0, as_stream(stream)>>>(
                (const float*)volume + ch * in, (float*)out + ch * per, (int)n0, (int)n1, (int)n2, (int)pad, i0, i1,
                i2);
        if (int e = check_launch("backproject_finish_kernel")) return e;
    }
    return TT_OK;
}
