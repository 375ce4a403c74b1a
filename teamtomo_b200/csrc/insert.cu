// Central-slice insertion into an fftshifted rfft volume plus its weight
// volume (insert_central_slices_rfft_3d, _insert_central_slices_rfft_3d.py:9-106,
// _insert_into_3d_dft :213-286, _insert_into_3d_dft_linear :289-406).
//
// Accumulate stage: one thread per source pixel, 8 x 32 pixel tiles per block
// (warp = 8 x 4 patch, so a warp's corners stay close in the volume).  Pixels
// outside fftfreq_max and the Friedel-redundant half of the x=0 column
// (x == 0 and y < 0) are skipped; the rotated frequency is redirected
// (conjugating the data) when x' < 0; points with any array coordinate outside
// [0, n-1] are dropped whole; the eight floor/ceil corners receive data*w and w
// with the reference's float32 weights ((1-t) and t products, left to right).
// Data and weight of a voxel share one 16-byte accumulator slot
// (re, im, w, 0) so each corner costs one vector reduction in L2 instead of
// two; complex128 uses a 32-byte (re, im, w, 0) double slot.  In the float
// kernel, lane pairs reduce the x-low and x-high corners of one pixel in the
// same instruction (insert_point_paired): the two voxels usually share an L2
// sector, so a warp's reductions touch fewer sectors (-15 % time at 256^3).
//
// The one-shot entry point (tt_insert_central_slices_rfft_3d) accumulates
// large float volumes into a 2 x 2 x 2-bricked accumulator instead
// (accumulator_slot: the eight corners of an even-aligned cell share one
// 128-byte line; a cell touches 3.4 lines on average instead of 4.5), with
// the eight corners of a pixel reduced by eight lanes in one instruction
// (insert_point_octet), split by insert_finalize_bricked_kernel.
//
// Finalize stage: the reference also inserts conj(data)*w at ((d-z)%d, (h-y)%h, 0)
// for every corner that lands on the x=0 plane except the DC voxel.  Summed
// over all points that equals, per plane voxel v with partner m(v),
//   out[v] = acc[v] + conj(acc[m(v)])   unless m(v) is the DC voxel,
// applied while splitting the accumulator into the volume and weight arrays.
#include <cuda_runtime.h>

#include <type_traits>

#include "capi_util.cuh"
#include "fixed_point.cuh"
#include "slice_common.cuh"
#include "slice_ops.cuh"

namespace tt {

// One block per (slice, row of tiles): the block loads the rotation once and
// walks the row, skipping the tiles of other z-phases (a few instructions
// each, so extra phases cost almost nothing).
template <typename R, bool BRICKED = false>
__global__ void __launch_bounds__(kTileThreads)
insert_accumulate_kernel(const typename Acc<R>::C* __restrict__ img, const void* __restrict__ rot,
                         typename Acc<R>::T* __restrict__ acc, SliceGeom g, int phase, int nphase) {
    __shared__ float m[9];
    const int tx_tiles = tiles_x_of(g.wr);
    const int rows = (g.img_h + kTileY - 1) / kTileY;
    const int64_t s = blockIdx.x / rows;
    const int ty = blockIdx.x - (int)(s * rows);
    if (threadIdx.x < 9) m[threadIdx.x] = prep_rotation_elem(rot, g.rot_f64, s, threadIdx.x, g, false);
    __syncthreads();
    for (int tx = 0; tx < tx_tiles; tx++) {
        // the same answer in every thread: the whole block skips the tile
        if (nphase > 1 && insert_tile_phase(g, m, min(ty * kTileY + kTileY / 2, g.img_h - 1),
                                            min(tx * kTileX + kTileX / 2, g.wr - 1), nphase) != phase)
            continue;
        int iy, ix;
        const bool has_pixel = tile_pixel(g, ty * tx_tiles + tx, iy, ix);
        if constexpr (std::is_same<R, float>::value && BRICKED)
            insert_point_octet(img, m, acc, g, s, has_pixel, iy, ix);  // every lane takes part
        else if constexpr (std::is_same<R, float>::value)
            insert_point_paired(img, m, acc, g, s, has_pixel, iy, ix);  // every lane takes part
        else if (has_pixel)
            insert_point<R>(img, m, acc, g, s, iy, ix);
    }
}

// Accumulator -> (volume, weights) with the Friedel completion of the x=0
// plane.  `channels` accumulators of (d, h, w); the weights come from channel 0
// (every channel carries the same weights).
template <typename R>
__global__ void insert_finalize_kernel(const typename Acc<R>::T* __restrict__ acc,
                                       typename Acc<R>::C* __restrict__ vol, R* __restrict__ wts, int64_t channels,
                                       int d, int h, int w) {
    const int64_t per = (int64_t)d * h * w;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= channels * per) return;
    const int64_t ch = idx / per, r = idx - ch * per;
    const typename Acc<R>::T a = acc[idx];
    R re = a.x, im = a.y, wt = a.z;
    const int x = (int)(r % w);
    if (x == 0) {
        const int64_t zy = r / w;
        const int z = (int)(zy / h), y = (int)(zy % h);
        const int zm = (d - z) % d, ym = (h - y) % h;
        if (!(zm == d / 2 && ym == h / 2)) {
            const typename Acc<R>::T b = acc[ch * per + ((int64_t)zm * h + ym) * w];
            re += b.x;
            im -= b.y;
            wt += b.z;
        }
    }
    typename Acc<R>::C o;
    o.x = re;
    o.y = im;
    vol[idx] = o;
    if (ch == 0 && wts) wts[r] = wt;
}

// Bricked float accumulator (accumulator_slot) -> (volume, weights) with the
// Friedel completion of the x=0 plane.  One block per (z, y) pair of brick
// rows: it reads that brick row's contiguous slots (coalesced float4 loads)
// and writes the four voxel rows it covers (runs of two x per brick).
__global__ void insert_finalize_bricked_kernel(const float4* __restrict__ acc, float2* __restrict__ vol,
                                               float* __restrict__ wts, SliceGeom g) {
    const int bh = (g.H + 1) >> 1, bw = (g.W + 1) >> 1;
    const int bz = blockIdx.x / bh, by = blockIdx.x - bz * bh;
    const float4* row = acc + (int64_t)blockIdx.x * bw * 8;
    for (int t = threadIdx.x; t < bw * 8; t += blockDim.x) {
        const int z = 2 * bz + ((t >> 2) & 1), y = 2 * by + ((t >> 1) & 1), x = 2 * (t >> 3) + (t & 1);
        if (z >= g.D || y >= g.H || x >= g.W) continue;
        const float4 a = row[t];
        float re = a.x, im = a.y, wt = a.z;
        if (x == 0) {
            const int zm = (g.D - z) % g.D, ym = (g.H - y) % g.H;
            if (!(zm == g.D / 2 && ym == g.H / 2)) {
                const float4 b = acc[accumulator_slot(g, zm, ym, 0)];
                re += b.x;
                im -= b.y;
                wt += b.z;
            }
        }
        const int64_t o = ((int64_t)z * g.H + y) * g.W + x;
        vol[o] = make_float2(re, im);
        if (wts) wts[o] = wt;
    }
}

// Friedel completion of the x=0 plane of already split volumes, in place
// (kept for callers that accumulate into (volume, weights) themselves).
template <typename R>
__global__ void mirror_x0_kernel(typename Acc<R>::C* __restrict__ vol, R* __restrict__ wts, int64_t channels,
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
        typename Acc<R>::C* base = vol + ch * plane;
        const typename Acc<R>::C a = base[idx * w];
        if (u == idx) {
            if (!u_dc) {
                typename Acc<R>::C o;
                o.x = a.x + a.x;
                o.y = a.y - a.y;
                base[idx * w] = o;
            }
        } else {
            const typename Acc<R>::C b = base[u * w];
            typename Acc<R>::C oa = a, ob = b;
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

// Backward of the insertion w.r.t. the slices, the adjoint of the splat and of
// the Friedel completion.  The completion adds conj(acc[m u]) to out[u] unless
// m u is DC; m is its own inverse, so acc[v] reaches out[m v] unless v is DC
// (for odd boxes m(DC) is not DC):
//   dL/dacc[v] = G[v] + conj(G[m v])  on the x = 0 plane, v not DC
// and each kept source pixel gathers sum_k w_k dL/dacc[corner k] with the
// splat's own float32 weights, conjugated where the point was redirected.
// One thread per slice pixel, one block per row of tiles (the row part of the
// geometry formed once per thread); every pixel is written (zero when
// dropped).  float: eight resident blocks (32 registers) for the gathers.
template <typename R, bool BRICKED = false>
__global__ void __launch_bounds__(kTileThreads, sizeof(R) == 4 ? (BRICKED ? 6 : 8) : 1)
insert_bwd_kernel(const typename Acc<R>::C* __restrict__ gvol, const void* __restrict__ rot,
                  typename Acc<R>::C* __restrict__ gimg, SliceGeom g, int tiles) {
    __shared__ float m[9];
    // one block per (slice, row of tiles); this thread's slice row is fixed
    const int tx_tiles = tiles_x_of(g.wr);
    const int rows = tiles / tx_tiles;
    const int64_t s = blockIdx.x / rows;
    const int ty = blockIdx.x - (int)(s * rows);
    if (threadIdx.x < 9) m[threadIdx.x] = prep_rotation_elem(rot, g.rot_f64, s, threadIdx.x, g, false);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int iy = ty * kTileY + (threadIdx.x >> 5) * 4 + (lane >> 3);
    if (iy >= g.img_h) return;
    const SliceRow row = slice_row_geom(g, m, iy);
    typename Acc<R>::C* orow = gimg + (s * g.img_h + slice_row(g, iy)) * (int64_t)g.wr;
    for (int tx = 0; tx < tx_tiles; tx++) {
        const int ix = tx * kTileX + (lane & 7);
        if (ix >= g.wr) continue;
        typename Acc<R>::C out;
        out.x = 0;
        out.y = 0;
        const float qx = __fmul_rn((float)ix, g.inv_w);
        bool cj;
        float c[3];
        const bool kept = (!g.has_fmax || __fsqrt_rn(__fadd_rn(row.qy2, __fmul_rn(qx, qx))) <= g.fmax) &&
                          !(qx == 0.0f && row.qy < 0.0f);
        if (kept && insert_coords_row(g, m, row, qx, cj, c)) {
            InsertCell k;
            cell_at(c, k);
            if constexpr (BRICKED) {
                // the x-rows of the cell from the bricked copy (corner addressed
                // once, neighbours by parity steps); corners of zero weight are
                // not read; same corner order, weights and sums as below
                Corners kk{};
                kk.z0 = k.iz0;
                kk.y0 = k.iy0;
                kk.x0 = k.ix0;
                const XRows<VoxBrick2> xr(reinterpret_cast<const VoxBrick2*>(gvol), g, kk);
                const bool hx = k.tx != 0.0f;
#pragma unroll
                for (int bz = 0; bz < 2; bz++) {
                    if (bz && k.tz == 0.0f) continue;
#pragma unroll
                    for (int by = 0; by < 2; by++) {
                        if (by && k.ty == 0.0f) continue;
                        float2 v0, v1;
                        xr.load(g, bz, by, true, hx, v0, v1);
                        const int z = bz ? k.iz1 : k.iz0, y = by ? k.iy1 : k.iy0;
                        if (k.ix0 == 0 && !(z == g.D / 2 && y == g.H / 2)) {
                            const float2 b = gvol[accumulator_slot(g, (g.D - z) % g.D, (g.H - y) % g.H, 0)];
                            v0.x += b.x;
                            v0.y -= b.y;
                        }
                        const float fzy = (bz ? k.tz : 1.0f - k.tz) * (by ? k.ty : 1.0f - k.ty);
                        const float w0 = fzy * (1.0f - k.tx);
                        out.x += w0 * v0.x;
                        out.y += w0 * v0.y;
                        if (hx) {
                            const float w1 = fzy * k.tx;
                            out.x += w1 * v1.x;
                            out.y += w1 * v1.y;
                        }
                    }
                }
            } else {
#pragma unroll
                for (int corner = 0; corner < 8; corner++) {
                    const float w = insert_corner_weight(k, corner);
                    if (w == 0.0f) continue;
                    int z, y, x;
                    insert_corner_zyx(k, corner, z, y, x);
                    const typename Acc<R>::C gv = completed_grad<R>(gvol, g, z, y, x);
                    out.x += (R)w * gv.x;
                    out.y += (R)w * gv.y;
                }
            }
            if (cj) out.y = -out.y;
        }
        __stcs(orow + ix, out);
    }
}

int insert_deterministic(const void* image_rfft, int32_t complex128, const void* rot, void* volume, void* weights,
                         void* workspace, const tt_slice_params* p, cudaStream_t st);

static int check_insert_params(const tt_slice_params* p) {
    if (int e = validate_params(p)) return e;
    if (p->vol_d != p->img_d || p->vol_h != p->img_h || p->vol_w != p->img_w / 2 + 1)
        return fail(TT_ERR_INVALID, "insert: volume dims (%lld, %lld, %lld) are not the rfft of volume_shape",
                    (long long)p->vol_d, (long long)p->vol_h, (long long)p->vol_w);
    return TT_OK;
}

// Number of z-phases for an accumulator of acc_bytes: one per 1.1 x the L2
// (at most 16).  Measured on a B200 (126 MB L2, 4096 slices): 320^3 (264 MB)
// 7.70 -> 6.12 ms with 2 phases (6.05 with 3); 256^3 (135 MB) 3.79 ms with 1
// phase, 3.81 with 2.
int insert_phases(size_t acc_bytes) {
    int dev = 0, l2 = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev) != cudaSuccess ||
        l2 <= 0) {
        cudaGetLastError();  // a failed query only costs the phasing
        return 1;
    }
    const int k = (int)ceil((double)acc_bytes / (1.1 * (double)l2));
    return k < 1 ? 1 : (k > 16 ? 16 : k);
}

// Bytes of the 2 x 2 x 2-bricked float accumulator of p's volume.
size_t bricked_accumulator_bytes(const tt_slice_params* p) {
    return (size_t)(((p->vol_d + 1) / 2) * ((p->vol_h + 1) / 2) * ((p->vol_w + 1) / 2)) * 8 * sizeof(float4);
}

// The one-shot float insertion accumulates into the bricked layout from this
// accumulator size up.  Measured on a B200: 3.86 vs 3.93 ms at 256^3 x 4096
// slices, 3.21 vs 3.31 ms at 320^3 x 2048, equal at 128^3, and 0.130 vs
// 0.102 ms at 64^3 x 1000 (where the brick-row finalize's small blocks cost
// more than the splat saves).
constexpr size_t kBrickedAccumulatorMinBytes = 64u << 20;

bool insert_bricked(const tt_slice_params* p) {
    return !p->volume_unshifted && bricked_accumulator_bytes(p) >= kBrickedAccumulatorMinBytes;
}

int launch_insert_accumulate(const void* image_rfft, int32_t complex128, const void* rot, void* acc,
                             const tt_slice_params* p, cudaStream_t st) {
    SliceGeom g = make_geom(*p);
    const int64_t items = (int64_t)g.n * ((g.img_h + kTileY - 1) / kTileY);
    if (items > 0x7fffffffLL) return fail(TT_ERR_INVALID, "insert: too many blocks");
    const size_t acc_bytes = (size_t)((int64_t)g.D * g.H * g.W) * (complex128 ? sizeof(double4) : sizeof(float4));
    const int nphase = insert_phases(acc_bytes);
    for (int ph = 0; ph < nphase; ph++) {
        if (complex128)
            insert_accumulate_kernel<double><<<(unsigned)items, kTileThreads, 0, st>>>(
                (const double2*)image_rfft, rot, (double4*)acc, g, ph, nphase);
        else
            insert_accumulate_kernel<float><<<(unsigned)items, kTileThreads, 0, st>>>(
                (const float2*)image_rfft, rot, (float4*)acc, g, ph, nphase);
        if (int e = check_launch("insert_accumulate_kernel")) return e;
    }
    return TT_OK;
}

// Channel-interleaved images (n, c, h, w/2+1) into c float accumulators: the
// single-channel splat once per channel (storage rows per slice: c * h), so
// each pass reduces into one accumulator with the paired lanes and z-phases
// of the single-channel path.  Splatting all channels from one geometry pass
// reduced into c accumulators at once and was slower: 2.85 vs 1.97 ms for 2
// channels, 6.52 vs 3.93 ms for 4 (256^3, 1024 slices).  Every channel gets
// the weights; readers take them from channel 0.
int launch_insert_accumulate_channels(const float2* img, int64_t channels, const void* rot, float4* acc,
                                      const tt_slice_params* p, cudaStream_t st) {
    SliceGeom g = make_geom(*p);
    g.slice_rows = (int)(channels * g.img_h);
    const int64_t items = (int64_t)g.n * ((g.img_h + kTileY - 1) / kTileY);
    if (items > 0x7fffffffLL) return fail(TT_ERR_INVALID, "insert multichannel: too many blocks");
    const int64_t vox = (int64_t)g.D * g.H * g.W;
    const int nphase = insert_phases((size_t)vox * sizeof(float4));
    for (int64_t ch = 0; ch < channels; ch++)
        for (int ph = 0; ph < nphase; ph++) {
            insert_accumulate_kernel<float><<<(unsigned)items, kTileThreads, 0, st>>>(
                img + ch * (int64_t)g.img_h * g.wr, rot, acc + ch * vox, g, ph, nphase);
            if (int e = check_launch("insert_accumulate_kernel")) return e;
        }
    return TT_OK;
}

int launch_insert_finalize(const void* acc, int32_t complex128, int64_t channels, int64_t d, int64_t h, int64_t w,
                           void* volume, void* weights, cudaStream_t st) {
    const int64_t total = channels * d * h * w;
    const unsigned blocks = (unsigned)((total + 255) / 256);
    if (complex128)
        insert_finalize_kernel<double><<<blocks, 256, 0, st>>>((const double4*)acc, (double2*)volume,
                                                               (double*)weights, channels, (int)d, (int)h, (int)w);
    else
        insert_finalize_kernel<float><<<blocks, 256, 0, st>>>((const float4*)acc, (float2*)volume, (float*)weights,
                                                              channels, (int)d, (int)h, (int)w);
    return check_launch("insert_finalize_kernel");
}

}  // namespace tt

using namespace tt;

extern "C" size_t tt_insert_accumulator_bytes(int32_t complex128, int64_t channels, int64_t d, int64_t h,
                                              int64_t w_rfft) {
    if (channels < 1 || d < 1 || h < 1 || w_rfft < 1) return 0;
    return (size_t)(channels * d * h * w_rfft) * (complex128 ? sizeof(double4) : sizeof(float4));
}

extern "C" size_t tt_insert_workspace_bytes(int32_t complex128, const tt_slice_params* p) {
    if (!p) return 0;
    if (p->deterministic) return kFixedHeaderBytes + tt_insert_fixed_accumulator_bytes(1, p->vol_d, p->vol_h, p->vol_w);
    if (!complex128 && insert_bricked(p)) return bricked_accumulator_bytes(p);  // dims padded to even
    return tt_insert_accumulator_bytes(complex128, 1, p->vol_d, p->vol_h, p->vol_w);
}

extern "C" int tt_insert_accumulate(const void* image_rfft, int32_t complex128, const void* rotation_matrices,
                                    void* accumulator, const tt_slice_params* p, void* stream) {
    if (int e = check_insert_params(p)) return e;
    if (p->deterministic)
        return fail(TT_ERR_INVALID, "insert_accumulate: the deterministic mode accumulates through "
                                    "tt_insert_fixed_accumulate");
    if (p->n == 0) return TT_OK;
    if (!image_rfft || !rotation_matrices || !accumulator)
        return fail(TT_ERR_INVALID, "insert_accumulate: NULL pointer argument");
    return launch_insert_accumulate(image_rfft, complex128, rotation_matrices, accumulator, p, as_stream(stream));
}

// The batched insertion's policy: bricked from 64 MB of accumulator while the
// accumulator fits one z-phase.  Measured on a B200 (batched launch, CTF,
// best tile shape): 256^3 x 4096 3.77 vs 3.84 ms, 200^3 2.38 vs 2.37 ms (below
// 64 MB), 320^3 x 10000 (two z-phases) 16.1 vs 15.0 ms.
extern "C" int32_t tt_insert_accumulator_layout(const tt_slice_params* p) {
    if (!p || p->deterministic || !insert_bricked(p)) return TT_VOLUME_PLAIN;
    return insert_phases(bricked_accumulator_bytes(p)) == 1 ? TT_VOLUME_BRICKS : TT_VOLUME_PLAIN;
}

extern "C" size_t tt_insert_bricked_accumulator_bytes(int64_t d, int64_t h, int64_t w_rfft) {
    if (d < 1 || h < 1 || w_rfft < 1) return 0;
    return (size_t)(((d + 1) / 2) * ((h + 1) / 2) * ((w_rfft + 1) / 2)) * 8 * sizeof(float4);
}

extern "C" int tt_insert_finalize_bricked(const void* accumulator, int64_t d, int64_t h, int64_t w_rfft,
                                          void* volume_rfft, void* weights, void* stream) {
    if (!accumulator || !volume_rfft) return fail(TT_ERR_INVALID, "insert_finalize_bricked: NULL pointer argument");
    if (d < 1 || h < 1 || w_rfft < 1 || d > 0x7fffffff || h > 0x7fffffff || w_rfft > 0x7fffffff)
        return fail(TT_ERR_INVALID, "insert_finalize_bricked: bad dims");
    const int64_t rows = ((d + 1) / 2) * ((h + 1) / 2);
    if (rows > 0x7fffffffLL) return fail(TT_ERR_INVALID, "insert_finalize_bricked: too many brick rows");
    SliceGeom g{};  // the finalize reads only the volume dims
    g.D = (int)d;
    g.H = (int)h;
    g.W = (int)w_rfft;
    insert_finalize_bricked_kernel<<<(unsigned)rows, 256, 0, as_stream(stream)>>>(
        (const float4*)accumulator, (float2*)volume_rfft, (float*)weights, g);
    return check_launch("insert_finalize_bricked_kernel");
}

extern "C" int tt_insert_finalize(const void* accumulator, int32_t complex128, int64_t channels, int64_t d, int64_t h,
                                  int64_t w_rfft, void* volume_rfft, void* weights, void* stream) {
    if (!accumulator || !volume_rfft) return fail(TT_ERR_INVALID, "insert_finalize: NULL pointer argument");
    if (channels < 1 || d < 1 || h < 1 || w_rfft < 1) return fail(TT_ERR_INVALID, "insert_finalize: bad dims");
    return launch_insert_finalize(accumulator, complex128, channels, d, h, w_rfft, volume_rfft, weights,
                                  as_stream(stream));
}

extern "C" int tt_insert_central_slices_rfft_3d(const void* image_rfft, int32_t complex128,
                                                const void* rotation_matrices, void* volume_rfft, void* weights,
                                                void* workspace, size_t workspace_bytes, const tt_slice_params* p,
                                                void* stream) {
    if (int e = check_insert_params(p)) return e;
    if (!volume_rfft || !weights || (p->n > 0 && (!image_rfft || !rotation_matrices)))
        return fail(TT_ERR_INVALID, "insert: NULL pointer argument");
    const size_t need = tt_insert_workspace_bytes(complex128, p);
    if (!workspace || workspace_bytes < need)
        return fail(TT_ERR_WORKSPACE, "insert: workspace of %zu bytes needed, got %zu", need, workspace_bytes);
    cudaStream_t st = as_stream(stream);
    if (p->deterministic)
        return insert_deterministic(image_rfft, complex128, rotation_matrices, volume_rfft, weights, workspace, p, st);
    cudaError_t e = cudaMemsetAsync(workspace, 0, need, st);
    if (e != cudaSuccess) return fail(TT_ERR_CUDA, "insert: memset: %s", cudaGetErrorString(e));
    if (!complex128 && insert_bricked(p)) {
        // float: the 2 x 2 x 2-bricked accumulator (fewer 128-byte lines per splatted cell)
        SliceGeom g = make_geom(*p);
        if (p->n > 0) {
            const int64_t items = (int64_t)g.n * ((g.img_h + kTileY - 1) / kTileY);
            if (items > 0x7fffffffLL) return fail(TT_ERR_INVALID, "insert: too many blocks");
            const int nphase = insert_phases(bricked_accumulator_bytes(p));
            for (int ph = 0; ph < nphase; ph++) {
                insert_accumulate_kernel<float, true><<<(unsigned)items, kTileThreads, 0, st>>>(
                    (const float2*)image_rfft, rotation_matrices, (float4*)workspace, g, ph, nphase);
                if (int r = check_launch("insert_accumulate_kernel")) return r;
            }
        }
        const unsigned rows = (unsigned)(((g.D + 1) / 2) * ((g.H + 1) / 2));
        insert_finalize_bricked_kernel<<<rows, 256, 0, st>>>((const float4*)workspace, (float2*)volume_rfft,
                                                             (float*)weights, g);
        return check_launch("insert_finalize_bricked_kernel");
    }
    if (p->n > 0)
        if (int r = launch_insert_accumulate(image_rfft, complex128, rotation_matrices, workspace, p, st)) return r;
    return launch_insert_finalize(workspace, complex128, 1, p->vol_d, p->vol_h, p->vol_w, volume_rfft, weights, st);
}

extern "C" int tt_insert_central_slices_rfft_3d_backward(const void* grad_volume, int32_t complex128,
                                                         const void* rotation_matrices, void* grad_image,
                                                         const tt_slice_params* p, void* stream) {
    if (!p) return fail(TT_ERR_INVALID, "insert backward: NULL params");
    // grad_volume plain, or (complex64, fftshifted) its bricked copy (tt_pack_volume_bricks)
    const bool bricked = p->volume_layout == TT_VOLUME_BRICKS;
    if (bricked && (complex128 || p->volume_unshifted))
        return fail(TT_ERR_INVALID, "insert backward: a bricked gradient volume is complex64 and fftshifted");
    if (p->volume_layout == TT_VOLUME_XPAIRS)
        return fail(TT_ERR_INVALID, "insert backward: the gradient volume is plain or bricked");
    if (int e = validate_params(p, true)) return e;
    if (p->vol_d != p->img_d || p->vol_h != p->img_h || p->vol_w != p->img_w / 2 + 1)
        return fail(TT_ERR_INVALID, "insert: volume dims (%lld, %lld, %lld) are not the rfft of volume_shape",
                    (long long)p->vol_d, (long long)p->vol_h, (long long)p->vol_w);
    if (p->n == 0) return TT_OK;
    if (!grad_volume || !rotation_matrices || !grad_image)
        return fail(TT_ERR_INVALID, "insert backward: NULL pointer argument");
    SliceGeom g = make_geom(*p);
    const int tiles = tiles_per_slice(g.img_h, g.wr);
    if ((int64_t)g.n * tiles > 0x7fffffffLL) return fail(TT_ERR_INVALID, "insert backward: too many blocks");
    const int64_t items = (int64_t)g.n * (tiles / tiles_x_of(g.wr));  // one block per row of tiles
    cudaStream_t st = as_stream(stream);
    if (complex128)
        insert_bwd_kernel<double><<<(unsigned)items, kTileThreads, 0, st>>>((const double2*)grad_volume,
                                                                           rotation_matrices, (double2*)grad_image,
                                                                           g, tiles);
    else if (bricked)
        insert_bwd_kernel<float, true><<<(unsigned)items, kTileThreads, 0, st>>>(
            (const float2*)grad_volume, rotation_matrices, (float2*)grad_image, g, tiles);
    else
        insert_bwd_kernel<float><<<(unsigned)items, kTileThreads, 0, st>>>((const float2*)grad_volume,
                                                                          rotation_matrices, (float2*)grad_image, g,
                                                                          tiles);
    return check_launch("insert_bwd_kernel");
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
