// Multichannel central slices (extract_central_slices_rfft_3d_multichannel,
// _extract_central_slices_rfft_3d.py:225-367, and
// insert_central_slices_rfft_3d_multichannel, _insert_central_slices_rfft_3d.py:109-210):
// c volumes share one set of rotations, so each pixel's geometry (rotation,
// redirect, coordinates, corners and weights) is computed once and applied to
// every channel.  Layouts: volumes (c, d, h, w/2+1), slices (n, c, h, w/2+1)
// (the reference's (..., c, h, w) order), insertion accumulators
// (c, d, h, w/2+1) float4 slots with the weights in channel 0.
#include <cuda_runtime.h>

#include "capi_util.cuh"
#include "slice_common.cuh"
#include "slice_grad.cuh"
#include "slice_ops.cuh"

namespace tt {

__device__ __forceinline__ int64_t chan_pixel(const SliceGeom& g, int64_t s, int ch, int channels, int iy, int ix) {
    return (((int64_t)s * channels + ch) * g.img_h + slice_row(g, iy)) * g.wr + ix;
}

// Extraction: one thread per slice pixel, all channels; eight resident blocks
// (32 registers) for the gathers.  VT: float2 (plain volumes) or VoxBrick2
// (the channels' bricked copies back to back); vstride in VT elements.
template <typename VT>
__global__ void __launch_bounds__(kTileThreads, 8)
extract_multi_fwd_kernel(const VT* __restrict__ vol, int64_t vstride, int channels,
                         const void* __restrict__ rot, float2* __restrict__ out, SliceGeom g, int tiles) {
    __shared__ float m[9];
    const int64_t s = blockIdx.x / tiles;
    const int tile = blockIdx.x - (int)(s * tiles);
    if (threadIdx.x < 9) m[threadIdx.x] = prep_rotation_elem(rot, g.rot_f64, s, threadIdx.x, g, true);
    __syncthreads();
    int iy, ix;
    if (!tile_pixel(g, tile, iy, ix)) return;
    float qy, qx, c[3];
    bool cj = false;
    const bool in = extract_geometry(g, m, iy, ix, qy, qx, cj, c);
    Corners k;
    if (in) k = make_corners(g, c);
    for (int ch = 0; ch < channels; ch++) {
        float2 r = make_float2(0.0f, 0.0f);
        if (in) {
            r = sample_trilinear(vol + ch * vstride, g, k);
            if (cj) r.y = -r.y;
        }
        __stcs(out + chan_pixel(g, s, ch, channels, iy, ix), r);
    }
}

// Backward: d/dvolume per channel, d/drotation summed over the channels
// (block partials reduced as in the single-channel kernel).  The gathers read
// vol (VT as in the forward, channel stride vstride); d/dvolume is plain
// complex64 with channel stride dstride.
template <bool WANT_DV, bool WANT_DR, typename VT>
__global__ void __launch_bounds__(kTileThreads)
extract_multi_bwd_kernel(const VT* __restrict__ vol, int64_t vstride, int64_t dstride, int channels,
                         const void* __restrict__ rot, const float2* __restrict__ grad,
                         float2* __restrict__ dvol, float* __restrict__ part, SliceGeom g, int tiles) {
    __shared__ float m[9];
    __shared__ double red[kTileThreads / 32][6];
    const int64_t s = blockIdx.x / tiles;
    const int tile = blockIdx.x - (int)(s * tiles);
    if (threadIdx.x < 9) m[threadIdx.x] = prep_rotation_elem(rot, g.rot_f64, s, threadIdx.x, g, true);
    __syncthreads();
    float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int iy, ix;
    if (tile_pixel(g, tile, iy, ix)) {
        float qy, qx, c[3];
        bool cj = false;
        if (extract_geometry(g, m, iy, ix, qy, qx, cj, c)) {
            const Corners k = make_corners(g, c);
            for (int ch = 0; ch < channels; ch++) {
                float2 gv = __ldcs(grad + chan_pixel(g, s, ch, channels, iy, ix));
                if (cj) gv.y = -gv.y;
                if (WANT_DV) scatter_dv(DvTarget<false>{dvol + ch * dstride, nullptr, 0.0}, g, k, gv);
                if (WANT_DR) {
                    float2 v[2][2][2];
                    load_corners(vol + ch * vstride, g, k, v);
                    drot_terms(v, k, gv, cj, g, qy, qx, acc);
                }
            }
        }
    }
    if (WANT_DR) {
        // warp totals in float by recursive halving (fixed order), the warps in double
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const float v8[8] = {acc[0], acc[1], acc[2], acc[3], acc[4], acc[5], 0.f, 0.f};
        const float t = warp_reduce8(v8);
        if ((lane & 3) == 0 && (lane >> 2) < 6) red[warp][lane >> 2] = (double)t;
        __syncthreads();
        if (threadIdx.x < 6) {
            double v = 0.0;
#pragma unroll
            for (int w = 0; w < kTileThreads / 32; w++) v += red[w][threadIdx.x];
            part[((int64_t)s * tiles + tile) * 6 + threadIdx.x] = (float)v;
        }
    }
}

// Insertion backward of all channels: gather adjoint per channel with the
// shared geometry.
__global__ void __launch_bounds__(kTileThreads)
insert_multi_bwd_kernel(const float2* __restrict__ gvol, int64_t vstride, int channels,
                        const void* __restrict__ rot, float2* __restrict__ gimg, SliceGeom g, int tiles) {
    __shared__ float m[9];
    const int64_t s = blockIdx.x / tiles;
    const int tile = blockIdx.x - (int)(s * tiles);
    if (threadIdx.x < 9) m[threadIdx.x] = prep_rotation_elem(rot, g.rot_f64, s, threadIdx.x, g, false);
    __syncthreads();
    int iy, ix;
    if (!tile_pixel(g, tile, iy, ix)) return;
    const float qy = shifted_freq(iy, g.img_h, g.inv_h);
    const float qx = __fmul_rn((float)ix, g.inv_w);
    bool cj = false;
    InsertCell k;
    const bool kept = insert_pixel_kept(g, qy, qx) && insert_cell(g, m, qy, qx, cj, k);
    for (int ch = 0; ch < channels; ch++) {
        float2 out = make_float2(0.0f, 0.0f);
        if (kept) {
#pragma unroll
            for (int corner = 0; corner < 8; corner++) {
                const float w = insert_corner_weight(k, corner);
                if (w == 0.0f) continue;
                int z, y, x;
                insert_corner_zyx(k, corner, z, y, x);
                const float2 gv = completed_grad<float>(gvol + ch * vstride, g, z, y, x);
                out.x += w * gv.x;
                out.y += w * gv.y;
            }
            if (cj) out.y = -out.y;
        }
        __stcs(gimg + chan_pixel(g, s, ch, channels, iy, ix), out);
    }
}

static int multi_blocks(const SliceGeom& g, int& tiles, int64_t& blocks, const char* what) {
    tiles = tiles_per_slice(g.img_h, g.wr);
    blocks = (int64_t)g.n * tiles;
    if (blocks > 0x7fffffffLL) return fail(TT_ERR_INVALID, "%s: too many blocks", what);
    return TT_OK;
}

static int check_channels(int64_t channels, const char* what) {
    if (channels < 1 || channels > 4096) return fail(TT_ERR_INVALID, "%s: channels must be in [1, 4096]", what);
    return TT_OK;
}

// Multichannel extraction volumes: plain, or the channels' bricked copies back
// to back (vstride = one copy's slots); the x-paired copy is not taken.
static int multi_volume_stride(const tt_slice_params* p, int64_t& vstride, const char* what) {
    if (p->volume_layout == TT_VOLUME_XPAIRS)
        return fail(TT_ERR_INVALID, "%s: volume_layout: plain or bricked volumes only", what);
    vstride = p->volume_layout == TT_VOLUME_BRICKS
                  ? ((p->vol_d + 1) / 2) * ((p->vol_h + 1) / 2) * ((p->vol_w + 1) / 2) * 8
                  : p->vol_d * p->vol_h * p->vol_w;
    return TT_OK;
}

template <typename VT>
static void launch_multi_bwd(const VT* v, int64_t vstride, int64_t dstride, int c, const void* rot,
                             const float2* gr, float2* dv, bool want_dr, float* part, const SliceGeom& g, int tiles,
                             unsigned nb, cudaStream_t st) {
    if (dv && want_dr)
        extract_multi_bwd_kernel<true, true, VT><<<nb, kTileThreads, 0, st>>>(v, vstride, dstride, c, rot, gr, dv,
                                                                            part, g, tiles);
    else if (dv)
        extract_multi_bwd_kernel<true, false, VT><<<nb, kTileThreads, 0, st>>>(v, vstride, dstride, c, rot, gr, dv,
                                                                             part, g, tiles);
    else
        extract_multi_bwd_kernel<false, true, VT><<<nb, kTileThreads, 0, st>>>(v, vstride, dstride, c, rot, gr,
                                                                              dv, part, g, tiles);
}

}  // namespace tt

using namespace tt;

extern "C" int tt_extract_central_slices_rfft_3d_multichannel(const void* volume_rfft, int64_t channels,
                                                              const void* rotation_matrices, void* slices_out,
                                                              const tt_slice_params* p, void* stream) {
    if (int e = validate_params(p, true)) return e;
    if (int e = check_channels(channels, "extract multichannel")) return e;
    int64_t vstride;
    if (int e = multi_volume_stride(p, vstride, "extract multichannel")) return e;
    if (p->n == 0) return TT_OK;
    if (!volume_rfft || !rotation_matrices || !slices_out)
        return fail(TT_ERR_INVALID, "extract multichannel: NULL pointer argument");
    SliceGeom g = make_geom(*p);
    int tiles;
    int64_t blocks;
    if (int e = multi_blocks(g, tiles, blocks, "extract multichannel")) return e;
    if (p->volume_layout == TT_VOLUME_BRICKS)
        extract_multi_fwd_kernel<<<(unsigned)blocks, kTileThreads, 0, as_stream(stream)>>>(
            (const VoxBrick2*)volume_rfft, vstride, (int)channels, rotation_matrices, (float2*)slices_out, g, tiles);
    else
        extract_multi_fwd_kernel<<<(unsigned)blocks, kTileThreads, 0, as_stream(stream)>>>(
            (const float2*)volume_rfft, vstride, (int)channels, rotation_matrices, (float2*)slices_out, g, tiles);
    return check_launch("extract_multi_fwd_kernel");
}

extern "C" int tt_extract_central_slices_rfft_3d_multichannel_backward(
    const void* volume_rfft, int64_t channels, const void* rotation_matrices, const void* grad_slices,
    void* grad_volume, void* grad_rotation, void* workspace, size_t workspace_bytes, const tt_slice_params* p,
    void* stream) {
    if (int e = validate_params(p, true)) return e;
    if (int e = check_channels(channels, "extract multichannel backward")) return e;
    int64_t vstride;
    if (int e = multi_volume_stride(p, vstride, "extract multichannel backward")) return e;
    if (p->deterministic)
        return fail(TT_ERR_INVALID, "extract multichannel backward: no deterministic mode; run the channels "
                                    "through tt_extract_central_slices_rfft_3d_backward");
    if (p->n == 0) return TT_OK;
    if (!volume_rfft || !rotation_matrices || !grad_slices)
        return fail(TT_ERR_INVALID, "extract multichannel backward: NULL pointer argument");
    if (!grad_volume && !grad_rotation) return TT_OK;
    SliceGeom g = make_geom(*p);
    int tiles;
    int64_t blocks;
    if (int e = multi_blocks(g, tiles, blocks, "extract multichannel backward")) return e;
    const size_t need = (size_t)(g.n * tiles * 6) * sizeof(float);
    if (grad_rotation && (!workspace || workspace_bytes < need))
        return fail(TT_ERR_WORKSPACE, "extract multichannel backward: workspace of %zu bytes needed, got %zu",
                    need, workspace_bytes);
    const int64_t dstride = p->vol_d * p->vol_h * p->vol_w;
    cudaStream_t st = as_stream(stream);
    const float2* gr = (const float2*)grad_slices;
    float2* dv = (float2*)grad_volume;
    float* part = (float*)workspace;
    const unsigned nb = (unsigned)blocks;
    const int c = (int)channels;
    const bool want_dr = grad_rotation != nullptr;
    if (p->volume_layout == TT_VOLUME_BRICKS)
        launch_multi_bwd((const VoxBrick2*)volume_rfft, vstride, dstride, c, rotation_matrices, gr, dv, want_dr,
                         part, g, tiles, nb, st);
    else
        launch_multi_bwd((const float2*)volume_rfft, vstride, dstride, c, rotation_matrices, gr, dv, want_dr, part,
                         g, tiles, nb, st);
    if (int e = check_launch("extract_multi_bwd_kernel")) return e;
    if (grad_rotation) return launch_drot_finish(part, rotation_matrices, grad_rotation, g, tiles, st);
    return TT_OK;
}

namespace tt {
int launch_insert_accumulate_channels(const float2* img, int64_t channels, const void* rot, float4* acc,
                                      const tt_slice_params* p, cudaStream_t st);  // insert.cu
}  // namespace tt

extern "C" int tt_insert_accumulate_multichannel(const void* image_rfft, int64_t channels,
                                                 const void* rotation_matrices, void* accumulator,
                                                 const tt_slice_params* p, void* stream) {
    if (int e = validate_params(p)) return e;
    if (int e = check_channels(channels, "insert multichannel")) return e;
    if (p->vol_d != p->img_d || p->vol_h != p->img_h || p->vol_w != p->img_w / 2 + 1)
        return fail(TT_ERR_INVALID, "insert multichannel: volume dims are not the rfft of volume_shape");
    if (p->deterministic)
        return fail(TT_ERR_INVALID, "insert multichannel: the deterministic mode accumulates per channel through "
                                    "tt_insert_fixed_accumulate");
    if (p->n == 0) return TT_OK;
    if (!image_rfft || !rotation_matrices || !accumulator)
        return fail(TT_ERR_INVALID, "insert multichannel: NULL pointer argument");
    if (channels * p->img_h > 0x7fffffffLL) return fail(TT_ERR_INVALID, "insert multichannel: too many rows");
    return launch_insert_accumulate_channels((const float2*)image_rfft, channels, rotation_matrices,
                                             (float4*)accumulator, p, as_stream(stream));
}

extern "C" int tt_insert_central_slices_rfft_3d_multichannel_backward(const void* grad_volume, int64_t channels,
                                                                      const void* rotation_matrices,
                                                                      void* grad_image, const tt_slice_params* p,
                                                                      void* stream) {
    if (int e = validate_params(p)) return e;
    if (int e = check_channels(channels, "insert multichannel backward")) return e;
    if (p->vol_d != p->img_d || p->vol_h != p->img_h || p->vol_w != p->img_w / 2 + 1)
        return fail(TT_ERR_INVALID, "insert multichannel backward: volume dims are not the rfft of volume_shape");
    if (p->n == 0) return TT_OK;
    if (!grad_volume || !rotation_matrices || !grad_image)
        return fail(TT_ERR_INVALID, "insert multichannel backward: NULL pointer argument");
    SliceGeom g = make_geom(*p);
    int tiles;
    int64_t blocks;
    if (int e = multi_blocks(g, tiles, blocks, "insert multichannel backward")) return e;
    const int64_t vstride = p->vol_d * p->vol_h * p->vol_w;
    insert_multi_bwd_kernel<<<(unsigned)blocks, kTileThreads, 0, as_stream(stream)>>>(
        (const float2*)grad_volume, vstride, (int)channels, rotation_matrices, (float2*)grad_image, g, tiles);
    return check_launch("insert_multi_bwd_kernel");
}
