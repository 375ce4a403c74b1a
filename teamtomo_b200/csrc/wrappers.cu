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

__device__ __forceinline__ int64_t wrap(int64_t i, int64_t n) {
    i %= n;
    return i < 0 ? i + n : i;
}

// f32(k) * f32(1/n) for unshifted index k of an axis of length n.
__device__ __forceinline__ float fftfreq_at(int64_t k, int64_t n, float inv_n) {
    int64_t kk = (k < (n + 1) / 2) ? k : k - n;
    return __fmul_rn((float)kk, inv_n);
}

// sinc(|f|)^2 at position a of the fftshifted norm grid of an (n0, n1, n2)
// array (fftfreq_grid(rfft=False, fftshift=True, norm=True)).
__device__ __forceinline__ float sinc2_at(int64_t a0, int64_t a1, int64_t a2, int64_t n0, int64_t n1, int64_t n2,
                                          float i0, float i1, float i2) {
    const float f0 = fftfreq_at(wrap(a0 - n0 / 2, n0), n0, i0);
    const float f1 = fftfreq_at(wrap(a1 - n1 / 2, n1), n1, i1);
    const float f2 = fftfreq_at(wrap(a2 - n2 / 2, n2), n2, i2);
    const float r = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(f0, f0), __fmul_rn(f1, f1)), __fmul_rn(f2, f2)));
    if (r == 0.0f) return 1.0f;
    const float px = __fmul_rn(3.14159265358979323846f, r);
    const float s = __fdiv_rn(sinpif(r), px);
    return s * s;
}

// out (n^3, FFT order) = fftshift(pad(vol, p) * sinc^2)
template <typename T>
__global__ void project_prepare_kernel(const T* __restrict__ vol, T* __restrict__ out, int64_t d, int64_t p,
                                       int64_t n, float inv_n) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n * n * n) return;
    const int64_t i = idx / (n * n), j = (idx / n) % n, k = idx % n;
    const int64_t a0 = wrap(i - n / 2, n), a1 = wrap(j - n / 2, n), a2 = wrap(k - n / 2, n);
    const int64_t v0 = a0 - p, v1 = a1 - p, v2 = a2 - p;
    T v = 0;
    if (v0 >= 0 && v0 < d && v1 >= 0 && v1 < d && v2 >= 0 && v2 < d)
        v = vol[(v0 * d + v1) * d + v2] * (T)sinc2_at(a0, a1, a2, n, n, n, inv_n, inv_n, inv_n);
    out[idx] = v;
}

// out (m, h-2p, w-2p) = crop(ifftshift(images, (-2,-1)), p), images (m, h, w)
template <typename T>
__global__ void recentre_crop_2d_kernel(const T* __restrict__ img, T* __restrict__ out, int64_t m, int64_t h,
                                        int64_t w, int64_t p) {
    const int64_t ch = h - 2 * p, cw = w - 2 * p;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= m * ch * cw) return;
    const int64_t b = idx / (ch * cw), i = (idx / cw) % ch, j = idx % cw;
    const int64_t si = wrap(i + p + h / 2, h), sj = wrap(j + p + w / 2, w);
    out[idx] = img[(b * h + si) * w + sj];
}

// out (m, n, n) = fftshift(pad(images, p), (-2,-1)), images (m, d, d)
template <typename T>
__global__ void pad_fftshift_2d_kernel(const T* __restrict__ img, T* __restrict__ out, int64_t m, int64_t d,
                                       int64_t p, int64_t n) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= m * n * n) return;
    const int64_t b = idx / (n * n), i = (idx / n) % n, j = idx % n;
    const int64_t a0 = wrap(i - n / 2, n) - p, a1 = wrap(j - n / 2, n) - p;
    T v = 0;
    if (a0 >= 0 && a0 < d && a1 >= 0 && a1 < d) v = img[(b * d + a0) * d + a1];
    out[idx] = v;
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
template <typename R>
__global__ void normalize_unshift_kernel(const typename C2<R>::A* __restrict__ acc,
                                         typename C2<R>::T* __restrict__ out, int64_t channels, int64_t d,
                                         int64_t h, int64_t w) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t per = d * h * w;
    if (idx >= channels * per) return;
    const int64_t ch = idx / per, r = idx % per;
    const int64_t i = r / (h * w), j = (r / w) % h, k = r % w;
    const int64_t z = wrap(i + d / 2, d), y = wrap(j + h / 2, h);  // source (shifted) voxel
    const int64_t src = (z * h + y) * w + k;
    // the interpolation weights live in channel 0 (the channels share them)
    const typename C2<R>::A a = acc[ch * per + src];
    R re = a.x, im = a.y, wt = acc[src].z;
    if (k == 0) {
        const int64_t zm = (d - z) % d, ym = (h - y) % h;
        const bool m_dc = (zm == d / 2) && (ym == h / 2);
        if (!m_dc) {
            const int64_t msrc = (zm * h + ym) * w;
            const typename C2<R>::A u = acc[ch * per + msrc];
            re += u.x;
            im -= u.y;
            wt += acc[msrc].z;
        }
    }
    const R den = wt < (R)1 ? (R)1 : wt;
    typename C2<R>::T v;
    v.x = re / den;
    v.y = im / den;
    out[idx] = v;
}

// out (n0-2p, n1-2p, n2-2p) = crop(ifftshift(vol) / sinc^2, p), vol (n0, n1, n2)
// real; the sinc^2 grid is that of the (n0, n1, n2) array.
template <typename T>
__global__ void backproject_finish_kernel(const T* __restrict__ vol, T* __restrict__ out, int64_t n0, int64_t n1,
                                          int64_t n2, int64_t p) {
    const int64_t c0 = n0 - 2 * p, c1 = n1 - 2 * p, c2 = n2 - 2 * p;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= c0 * c1 * c2) return;
    const int64_t i = idx / (c1 * c2) + p, j = (idx / c2) % c1 + p, k = idx % c2 + p;
    const int64_t s = (wrap(i + n0 / 2, n0) * n1 + wrap(j + n1 / 2, n1)) * n2 + wrap(k + n2 / 2, n2);
    const float i0 = (float)(1.0 / (double)n0), i1 = (float)(1.0 / (double)n1), i2 = (float)(1.0 / (double)n2);
    out[idx] = vol[s] / (T)sinc2_at(i, j, k, n0, n1, n2, i0, i1, i2);
}

inline unsigned blocks_for(int64_t total, int threads) { return (unsigned)((total + threads - 1) / threads); }

}  // namespace tt

using namespace tt;

extern "C" int tt_project_prepare(const void* volume, int32_t is_f64, int64_t d, int64_t pad, void* out,
                                  void* stream) {
    if (!volume || !out || d < 1 || pad < 0) return fail(TT_ERR_INVALID, "project_prepare: bad arguments");
    const int64_t n = d + 2 * pad, total = n * n * n;
    const float inv_n = (float)(1.0 / (double)n);
    if (is_f64)
        project_prepare_kernel<double><<<blocks_for(total, 256), 256, 0, as_stream(stream)>>>(
            (const double*)volume, (double*)out, d, pad, n, inv_n);
    else
        project_prepare_kernel<float><<<blocks_for(total, 256), 256, 0, as_stream(stream)>>>(
            (const float*)volume, (float*)out, d, pad, n, inv_n);
    return check_launch("project_prepare_kernel");
}

extern "C" int tt_recentre_crop_2d(const void* images, int32_t is_f64, int64_t m, int64_t h, int64_t w, int64_t pad,
                                   void* out, void* stream) {
    if (!images || !out || m < 0 || h < 1 || w < 1 || pad < 0 || 2 * pad >= h || 2 * pad >= w)
        return fail(TT_ERR_INVALID, "recentre_crop_2d: bad arguments");
    if (m == 0) return TT_OK;
    const int64_t total = m * (h - 2 * pad) * (w - 2 * pad);
    if (is_f64)
        recentre_crop_2d_kernel<double><<<blocks_for(total, 256), 256, 0, as_stream(stream)>>>(
            (const double*)images, (double*)out, m, h, w, pad);
    else
        recentre_crop_2d_kernel<float><<<blocks_for(total, 256), 256, 0, as_stream(stream)>>>(
            (const float*)images, (float*)out, m, h, w, pad);
    return check_launch("recentre_crop_2d_kernel");
}

extern "C" int tt_pad_fftshift_2d(const void* images, int32_t is_f64, int64_t m, int64_t d, int64_t pad, void* out,
                                  void* stream) {
    if (!images || !out || m < 0 || d < 1 || pad < 0) return fail(TT_ERR_INVALID, "pad_fftshift_2d: bad arguments");
    if (m == 0) return TT_OK;
    const int64_t n = d + 2 * pad, total = m * n * n;
    if (is_f64)
        pad_fftshift_2d_kernel<double><<<blocks_for(total, 256), 256, 0, as_stream(stream)>>>(
            (const double*)images, (double*)out, m, d, pad, n);
    else
        pad_fftshift_2d_kernel<float><<<blocks_for(total, 256), 256, 0, as_stream(stream)>>>(
            (const float*)images, (float*)out, m, d, pad, n);
    return check_launch("pad_fftshift_2d_kernel");
}

extern "C" int tt_backproject_normalize(const void* accumulator, int32_t complex128, int64_t channels, int64_t d,
                                        int64_t h, int64_t w_rfft, void* out, void* stream) {
    if (!accumulator || !out || channels < 1 || d < 1 || h < 1 || w_rfft < 1)
        return fail(TT_ERR_INVALID, "backproject_normalize: bad arguments");
    if (accumulator == out) return fail(TT_ERR_INVALID, "backproject_normalize: out must not alias the input");
    const int64_t total = channels * d * h * w_rfft;
    if (complex128)
        normalize_unshift_kernel<double><<<blocks_for(total, 256), 256, 0, as_stream(stream)>>>(
            (const double4*)accumulator, (double2*)out, channels, d, h, w_rfft);
    else
        normalize_unshift_kernel<float><<<blocks_for(total, 256), 256, 0, as_stream(stream)>>>(
            (const float4*)accumulator, (float2*)out, channels, d, h, w_rfft);
    return check_launch("normalize_unshift_kernel");
}

extern "C" int tt_backproject_finish(const void* volume, int32_t is_f64, int64_t channels, int64_t n0, int64_t n1,
                                     int64_t n2, int64_t pad, void* out, void* stream) {
    if (!volume || !out || channels < 1 || n0 < 1 || n1 < 1 || n2 < 1 || pad < 0 || 2 * pad >= n0 ||
        2 * pad >= n1 || 2 * pad >= n2)
        return fail(TT_ERR_INVALID, "backproject_finish: bad arguments");
    const int64_t per = (n0 - 2 * pad) * (n1 - 2 * pad) * (n2 - 2 * pad), in = n0 * n1 * n2;
    for (int64_t ch = 0; ch < channels; ch++) {
        if (is_f64)
            backproject_finish_kernel<double><<<blocks_for(per, 256), 256, 0, as_stream(stream)>>>(
                (const double*)volume + ch * in, (double*)out + ch * per, n0, n1, n2, pad);
        else
            backproject_finish_kernel<float><<<blocks_for(per, 256), 256, 0, as_stream(stream)>>>(
                (const float*)volume + ch * in, (float*)out + ch * per, n0, n1, n2, pad);
        if (int e = check_launch("backproject_finish_kernel")) return e;
    }
    return TT_OK;
}
