// Central lines through the rfft of a 2D image
// (extract_central_slices_rfft_2d, _extract_central_slices_rfft_2d.py:9-84),
// the 2D counterpart of the central-slice extraction, and its backward.
//
// Line sample k has frequency (0, qx), qx = f32(k) * f32(1/w); the 2x2 matrix
// (flipped to act on yx unless yx_matrices) maps it to p = (m01 qx, m11 qx)
// (the zero y term drops out exactly); p is negated (and the sample later
// conjugated) when p_x < 0; array coordinates follow _dft_utils.py:37-72 for an
// (h, w) image: y ((p_y + 0.5) / (1 - 1/h)) (h - 1), x (p_x 2) (w/2); the
// sample is grid_sample's bilinear with padding 'border', align_corners and
// the array -> grid -> array round trip, zero outside [0, N-1].
// fftfreq_max zeroes samples with qx > fftfreq_max.
//
// One thread per (line, sample); the backward reduces each line's 2x2
// gradient in a block per line, in a fixed order.
#include <cuda_runtime.h>

#include "capi_util.cuh"
#include "slice_ops.cuh"

namespace tt {

struct LineGeom {
    int n;              // lines
    int wr;             // samples per line, w/2 + 1
    float inv_w;        // f32(1/w)
    float iw0, s0, sx;  // 1 - 1/h, h - 1, w/2 (coordinate scaling of the image shape)
    int H, W;           // rfft image dims (h, w/2+1)
    float ub0, ub1;     // H - 1, W - 1
    int has_fmax;
    float fmax;
    int yx;             // matrices act on yx column vectors
    int rot_f64;
};

static LineGeom make_line_geom(int64_t n, int64_t h, int64_t w, int64_t H, int64_t W, int has_fmax, float fmax,
                               int yx, int rot_f64) {
    LineGeom g;
    g.n = (int)n;
    g.wr = (int)(w / 2 + 1);
    g.inv_w = (float)(1.0 / (double)w);
    volatile float dh = 1.0f / (float)h;
    g.iw0 = 1.0f - dh;
    g.s0 = (float)h - 1.0f;
    g.sx = (float)(w / 2 + 1) - 1.0f;
    g.H = (int)H;
    g.W = (int)W;
    g.ub0 = (float)(H - 1);
    g.ub1 = (float)(W - 1);
    g.has_fmax = has_fmax;
    g.fmax = fmax;
    g.yx = yx;
    g.rot_f64 = rot_f64;
    return g;
}

// Element (i, j) of line s's matrix acting on yx vectors, rounded to float32.
__device__ __forceinline__ float line_rot(const void* rot, const LineGeom& g, int64_t s, int i, int j) {
    const int src = g.yx ? i * 2 + j : (1 - i) * 2 + (1 - j);
    return g.rot_f64 ? __double2float_rn(((const double*)rot)[s * 4 + src]) : ((const float*)rot)[s * 4 + src];
}

struct LineSample {
    bool in;              // a non-zero sample
    bool cj;              // redirected (conjugated)
    float qx;
    int y0, x0;
    bool yin, xin;        // high corner inside the image
    bool gy, gx;          // the axis passes a coordinate gradient (not on the border)
    float ay0, ay1, ax0, ax1;
};

__device__ __forceinline__ LineSample line_sample(const LineGeom& g, float m01, float m11, int k) {
    LineSample t;
    t.qx = __fmul_rn((float)k, g.inv_w);
    t.in = false;
    t.cj = false;
    if (g.has_fmax && !(t.qx <= g.fmax)) return t;
    float py = __fmul_rn(m01, t.qx), px = __fmul_rn(m11, t.qx);
    t.cj = px < 0.0f;
    if (t.cj) {
        py = -py;
        px = -px;
    }
    const float cy = __fmul_rn(__fdiv_rn(__fadd_rn(py, 0.5f), g.iw0), g.s0);
    const float cx = __fmul_rn(__fmul_rn(px, 2.0f), g.sx);
    if (!(cy >= 0.0f && cy <= g.ub0 && cx >= 0.0f && cx <= g.ub1)) return t;
    const float iy = source_index(cy, 0.5f * (float)g.H - 0.5f, g.ub0, t.gy);
    const float ix = source_index(cx, 0.5f * (float)g.W - 0.5f, g.ub1, t.gx);
    const float fy = floorf(iy), fx = floorf(ix);
    t.y0 = (int)fy;
    t.x0 = (int)fx;
    t.ay0 = (fy + 1.0f) - iy;
    t.ay1 = iy - fy;
    t.ax0 = (fx + 1.0f) - ix;
    t.ax1 = ix - fx;
    t.yin = t.y0 + 1 < g.H;
    t.xin = t.x0 + 1 < g.W;
    t.in = true;
    return t;
}

__device__ __forceinline__ void line_corners(const float2* __restrict__ img, const LineGeom& g, const LineSample& t,
                                             float2 v[2][2]) {
#pragma unroll
    for (int by = 0; by < 2; by++)
#pragma unroll
        for (int bx = 0; bx < 2; bx++) {
            const bool ok = (!by || t.yin) && (!bx || t.xin);
            v[by][bx] = ok ? __ldg(img + (int64_t)(t.y0 + by) * g.W + t.x0 + bx) : make_float2(0.f, 0.f);
        }
}

__global__ void line_extract_kernel(const float2* __restrict__ img, const void* __restrict__ rot,
                                    float2* __restrict__ out, LineGeom g) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)g.n * g.wr) return;
    const int64_t s = idx / g.wr;
    const int k = (int)(idx - s * g.wr);
    const LineSample t = line_sample(g, line_rot(rot, g, s, 0, 1), line_rot(rot, g, s, 1, 1), k);
    float2 r = make_float2(0.f, 0.f);
    if (t.in) {
        float2 v[2][2];
        line_corners(img, g, t, v);
#pragma unroll
        for (int by = 0; by < 2; by++) {
            const float wy = by ? t.ay1 : t.ay0;
            const float w0 = t.ax0 * wy, w1 = t.ax1 * wy;
            r.x = fmaf(v[by][0].x, w0, r.x);
            r.y = fmaf(v[by][0].y, w0, r.y);
            r.x = fmaf(v[by][1].x, w1, r.x);
            r.y = fmaf(v[by][1].y, w1, r.y);
        }
        if (t.cj) r.y = -r.y;
    }
    out[idx] = r;
}

// One block per line: d/dimage scattered with float2 atomics; the line's
// d/dM (column 1 of the yx matrix; column 0 multiplies the zero y frequency)
// reduced in double in a fixed order and written in the caller's layout.
constexpr int kLineThreads = 128;

template <bool WANT_DI, bool WANT_DR>
__global__ void __launch_bounds__(kLineThreads)
line_backward_kernel(const float2* __restrict__ img, const void* __restrict__ rot, const float2* __restrict__ grad,
                     float2* __restrict__ dimg, void* __restrict__ drot, LineGeom g) {
    __shared__ double red[kLineThreads / 32][2];
    const int64_t s = blockIdx.x;
    const float m01 = line_rot(rot, g, s, 0, 1), m11 = line_rot(rot, g, s, 1, 1);
    double a0 = 0.0, a1 = 0.0;
    const float dcdp0 = g.s0 / g.iw0, dcdp1 = 2.0f * g.sx;
    for (int k = threadIdx.x; k < g.wr; k += kLineThreads) {
        const LineSample t = line_sample(g, m01, m11, k);
        if (!t.in) continue;
        float2 gv = grad[s * g.wr + k];
        if (t.cj) gv.y = -gv.y;
        if (WANT_DI) {
#pragma unroll
            for (int by = 0; by < 2; by++) {
                if (by && !t.yin) continue;
                const float wy = by ? t.ay1 : t.ay0;
#pragma unroll
                for (int bx = 0; bx < 2; bx++) {
                    if (bx && !t.xin) continue;
                    const float w = (bx ? t.ax1 : t.ax0) * wy;
                    if (w != 0.0f)
                        atomicAdd(dimg + (int64_t)(t.y0 + by) * g.W + t.x0 + bx, make_float2(gv.x * w, gv.y * w));
                }
            }
        }
        if (WANT_DR) {
            float2 v[2][2];
            line_corners(img, g, t, v);
            float2 dy = make_float2(0.f, 0.f), dx = dy;
#pragma unroll
            for (int b = 0; b < 2; b++) {
                const float wx = b ? t.ax1 : t.ax0, wy = b ? t.ay1 : t.ay0;
                dy.x = fmaf(wx, v[1][b].x - v[0][b].x, dy.x);
                dy.y = fmaf(wx, v[1][b].y - v[0][b].y, dy.y);
                dx.x = fmaf(wy, v[b][1].x - v[b][0].x, dx.x);
                dx.y = fmaf(wy, v[b][1].y - v[b][0].y, dx.y);
            }
            const float sg = t.cj ? -1.f : 1.f;
            if (t.gy) a0 += (double)(fmaf(gv.x, dy.x, gv.y * dy.y) * dcdp0 * sg * t.qx);
            if (t.gx) a1 += (double)(fmaf(gv.x, dx.x, gv.y * dx.y) * dcdp1 * sg * t.qx);
        }
    }
    if (!WANT_DR) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    a0 = warp_sum_d(a0);
    a1 = warp_sum_d(a1);
    if (lane == 0) {
        red[warp][0] = a0;
        red[warp][1] = a1;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        // element (i, j) of the caller's matrix: yx element (i', j') with the flip undone
        const int i = threadIdx.x >> 1, j = threadIdx.x & 1;
        const int iy = g.yx ? i : 1 - i, jy = g.yx ? j : 1 - j;
        double v = 0.0;
        if (jy == 1)
            for (int w = 0; w < kLineThreads / 32; w++) v += red[w][iy];
        if (g.rot_f64)
            ((double*)drot)[s * 4 + threadIdx.x] = (double)(float)v;
        else
            ((float*)drot)[s * 4 + threadIdx.x] = (float)v;
    }
}

static int check_line_args(int64_t n, int64_t h, int64_t w, int64_t H, int64_t W) {
    if (n < 0 || h < 1 || w < 1 || H < 1 || W < 1) return fail(TT_ERR_INVALID, "lines: bad shape");
    if (n > (1LL << 31) - 1 || (int64_t)n * (w / 2 + 1) > (1LL << 40) || H * W >= (1LL << 31))
        return fail(TT_ERR_INVALID, "lines: too large");
    return TT_OK;
}

}  // namespace tt

using namespace tt;

extern "C" int tt_extract_central_lines_rfft_2d(const void* image_rfft, int64_t img_h, int64_t img_w_rfft,
                                                const void* rotation_matrices, int32_t rotation_f64, int64_t n,
                                                int64_t h, int64_t w, int32_t has_fftfreq_max, float fftfreq_max,
                                                int32_t yx_matrices, void* lines_out, void* stream) {
    if (int e = check_line_args(n, h, w, img_h, img_w_rfft)) return e;
    if (n == 0) return TT_OK;
    if (!image_rfft || !rotation_matrices || !lines_out) return fail(TT_ERR_INVALID, "lines: NULL pointer argument");
    const LineGeom g = make_line_geom(n, h, w, img_h, img_w_rfft, has_fftfreq_max, fftfreq_max, yx_matrices,
                                      rotation_f64);
    const int64_t total = n * g.wr;
    line_extract_kernel<<<(unsigned)((total + 255) / 256), 256, 0, as_stream(stream)>>>(
        (const float2*)image_rfft, rotation_matrices, (float2*)lines_out, g);
    return check_launch("line_extract_kernel");
}

extern "C" int tt_extract_central_lines_rfft_2d_backward(const void* image_rfft, int64_t img_h, int64_t img_w_rfft,
                                                         const void* rotation_matrices, int32_t rotation_f64,
                                                         int64_t n, int64_t h, int64_t w, int32_t has_fftfreq_max,
                                                         float fftfreq_max, int32_t yx_matrices,
                                                         const void* grad_lines, void* grad_image,
                                                         void* grad_rotation, void* stream) {
    if (int e = check_line_args(n, h, w, img_h, img_w_rfft)) return e;
    if (n == 0 || (!grad_image && !grad_rotation)) return TT_OK;
    if (!image_rfft || !rotation_matrices || !grad_lines)
        return fail(TT_ERR_INVALID, "lines backward: NULL pointer argument");
    const LineGeom g = make_line_geom(n, h, w, img_h, img_w_rfft, has_fftfreq_max, fftfreq_max, yx_matrices,
                                      rotation_f64);
    cudaStream_t st = as_stream(stream);
    const float2* im = (const float2*)image_rfft;
    const float2* gr = (const float2*)grad_lines;
    float2* di = (float2*)grad_image;
    if (di && grad_rotation)
        line_backward_kernel<true, true><<<(unsigned)n, kLineThreads, 0, st>>>(im, rotation_matrices, gr, di,
                                                                              grad_rotation, g);
    else if (di)
        line_backward_kernel<true, false><<<(unsigned)n, kLineThreads, 0, st>>>(im, rotation_matrices, gr, di,
                                                                               grad_rotation, g);
    else
        line_backward_kernel<false, true><<<(unsigned)n, kLineThreads, 0, st>>>(im, rotation_matrices, gr, di,
                                                                               grad_rotation, g);
    return check_launch("line_backward_kernel");
}
