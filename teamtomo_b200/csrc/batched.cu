// Batched central-slice extraction / insertion over many volumes of uneven
// box sizes, each with its own set of rotations and an optional per-image
// CTF, in ONE persistent launch.
//
// Work queue over (volume, slice, row of tiles) items: the items of all
// volumes form one global list; each block takes the next item from an atomic
// counter, finds its volume by binary search over the per-volume item
// offsets, loads the slice's rotation (and computes its CTF constants), and
// walks the row of pixel tiles.  The items of a volume are equal work and
// small (one row of tiles), so the queue balances uneven box sizes and slice
// counts without any host-side scheduling and without a long tail.  The
// extraction gathers from each volume's plain rfft or, when every volume of
// the call is given as its bricked copy (volume_layout 2,
// tt_pack_volume_bricks), from the bricked copies.
//
// The per-volume descriptors travel as a __grid_constant__ kernel parameter
// (no host-to-device copy, so the launch captures into a CUDA graph as-is);
// the only device state is the queue counter in the caller's workspace,
// zeroed by a memset issued on the same stream before the launch.
//
// Three tile shapes (8x32, 16x16, 32x8 pixels per 256-thread block) are
// compiled; the host-side autotuner picks one per box size.
#include <cuda_runtime.h>

#include <mutex>

#include "capi_util.cuh"
#include "slice_common.cuh"
#include "slice_ops.cuh"

namespace tt {

constexpr int kMaxBatch = TT_MAX_BATCH_VOLUMES;

struct BatchVolumeDev {
    SliceGeom g;
    const float2* vol;
    float2* slices;
    float4* acc;
    const void* rot;
    const tt_ctf_params* ctf;
    int tiles;
};

struct BatchParams {
    int nvol;
    int64_t item_offset[kMaxBatch + 1];  // work items (slice, row of tiles) before each volume
    BatchVolumeDev v[kMaxBatch];
};

template <int TX>
__host__ inline int tiles_t(int img_h, int wr) {
    constexpr int TY = 256 / TX;
    return ((wr + TX - 1) / TX) * ((img_h + TY - 1) / TY);
}

// The extraction instantiations keep six blocks resident (40 registers, no
// spills): 389K CTF slices of 32 volumes in 63.9 / 71.7 ms (8 x 32 / 16 x 16
// tiles) against 65.8 / 74.7 ms at five (47 registers) and 72.8 / 83.1 ms at
// four.  The insertion's keep five (44 registers; equal times).
template <int TX, bool INSERT, typename VT>
__global__ void __launch_bounds__(256, INSERT ? 5 : 6)
batched_slices_kernel(const __grid_constant__ BatchParams bp, unsigned long long* __restrict__ queue,
                      int64_t total, int phase, int nphase) {
    constexpr int TY = 256 / TX, RPW = 32 / TX;
    __shared__ float m[9];
    __shared__ CtfConst cc;
    __shared__ int64_t cur;
    __shared__ int vsel;
    const int lane = threadIdx.x & 31;
    // volume of item gi: item_offset[lo] <= gi < item_offset[lo + 1]
    auto volume_of = [&](int64_t gi) {
        int lo = 0, hi = bp.nvol;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (bp.item_offset[mid] <= gi) lo = mid;
            else hi = mid;
        }
        return lo;
    };
    if (threadIdx.x == 0) {
        cur = (int64_t)atomicAdd(queue, 1ULL);
        vsel = volume_of(cur);
    }
    for (;;) {
        __syncthreads();  // this item's cur / vsel are visible; m / cc of the previous one are no longer read
        const int64_t gi = cur;
        if (gi >= total) return;
        const BatchVolumeDev& bv = bp.v[vsel];
        const int txt = (bv.g.wr + TX - 1) / TX, tyt = (bv.g.img_h + TY - 1) / TY;
        const int64_t local = gi - bp.item_offset[vsel];
        const int64_t s = local / tyt;  // item = (slice, row of tiles)
        const int ty = (int)(local - s * tyt);
        if (threadIdx.x < 9) m[threadIdx.x] = prep_rotation_elem(bv.rot, bv.g.rot_f64, s, threadIdx.x, bv.g, !INSERT);
        if (threadIdx.x == 0 && bv.ctf) cc = make_ctf_const(bv.ctf[s]);
        // the next item is taken now and published after this one's pixels, so
        // the queue's round trip overlaps the work
        unsigned long long next = 0;
        if (threadIdx.x == 0) next = atomicAdd(queue, 1ULL);
        __syncthreads();  // every thread has read cur / vsel and sees m / cc
        const CtfConst* ccp = bv.ctf ? &cc : nullptr;
        const int iy = ty * TY + (threadIdx.x >> 5) * RPW + lane / TX;
        if constexpr (!INSERT) {
            // extraction: the row part of the geometry formed once for the row of tiles
            if (iy < bv.g.img_h) {
                const SliceRow row = slice_row_geom(bv.g, m, iy);
                float2* orow = bv.slices + (s * bv.g.img_h + slice_row(bv.g, iy)) * (int64_t)bv.g.wr;
                const VT* vol = reinterpret_cast<const VT*>(bv.vol);
                for (int tx = 0; tx < txt; tx++) {
                    const int ix = tx * TX + (lane % TX);
                    if (ix >= bv.g.wr) continue;
                    float qx, c[3];
                    bool cj = false;
                    float2 r = make_float2(0.0f, 0.0f);
                    if (extract_geometry_row(bv.g, m, row, ix, qx, cj, c)) {
                        r = sample_trilinear(vol, bv.g, make_corners(bv.g, c));
                        if (cj) r.y = -r.y;
                        if (ccp) {
                            const float cv = ctf_value(*ccp, row.qy, qx);
                            r.x *= cv;
                            r.y *= cv;
                        }
                    }
                    __stcs(orow + ix, r);
                }
            }
        } else {
            for (int tx = 0; tx < txt; tx++) {
                // z-phased filling of large accumulators (the same answer in every thread)
                if (nphase > 1 && insert_tile_phase(bv.g, m, min(ty * TY + TY / 2, bv.g.img_h - 1),
                                                    min(tx * TX + TX / 2, bv.g.wr - 1), nphase) != phase)
                    continue;
                const int ix = tx * TX + (lane % TX);
                const bool has_pixel = ix < bv.g.wr && iy < bv.g.img_h;
                // every lane takes part: lane octets (bricked accumulator) or lane pairs share a pixel
                if (bv.g.vol_layout == TT_VOLUME_BRICKS)
                    insert_point_octet(bv.slices, m, bv.acc, bv.g, s, has_pixel, iy, ix, ccp);
                else
                    insert_point_paired(bv.slices, m, bv.acc, bv.g, s, has_pixel, iy, ix, ccp);
            }
        }
        if (threadIdx.x == 0) {
            cur = (int64_t)next;
            vsel = volume_of((int64_t)next);
        }
    }
}

template <int TX>
static int tiles_for_shape(const SliceGeom& g) {
    return tiles_t<TX>(g.img_h, g.wr);
}

int insert_phases(size_t acc_bytes);                     // insert.cu
size_t bricked_accumulator_bytes(const tt_slice_params* p);  // insert.cu

template <int TX, bool INSERT, typename VT>
static int launch_batched(BatchParams& bp, const size_t* acc_bytes, unsigned long long* queue, cudaStream_t st) {
    constexpr int TY = 256 / TX;
    bp.item_offset[0] = 0;
    for (int v = 0; v < bp.nvol; v++) {
        bp.v[v].tiles = tiles_for_shape<TX>(bp.v[v].g);
        const int64_t rows = (bp.v[v].g.img_h + TY - 1) / TY;
        bp.item_offset[v + 1] = bp.item_offset[v] + (int64_t)bp.v[v].g.n * rows;
    }
    const int64_t total = bp.item_offset[bp.nvol];
    if (total == 0) return TT_OK;
    int dev = 0, sms = 148, occ = 1;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batched_slices_kernel<TX, INSERT, VT>, 256, 0) !=
            cudaSuccess ||
        occ < 1)
        occ = 1;
    int64_t blocks = (int64_t)sms * occ;
    if (blocks > total) blocks = total;
    // insertion into large accumulators runs in z-phases (insert_phases), one queue pass each
    int nphase = 1;
    if (INSERT)
        for (int v = 0; v < bp.nvol; v++) {
            const int k = insert_phases(acc_bytes[v]);
            nphase = k > nphase ? k : nphase;
        }
    for (int ph = 0; ph < nphase; ph++) {
        if (ph > 0) {
            cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st);
            if (e != cudaSuccess) return fail(TT_ERR_CUDA, "batched: memset: %s", cudaGetErrorString(e));
        }
        batched_slices_kernel<TX, INSERT, VT><<<(unsigned)blocks, 256, 0, st>>>(bp, queue, total, ph, nphase);
        if (int e = check_launch("batched_slices_kernel")) return e;
    }
    return TT_OK;
}

static int run_batched(const tt_batch_volume* volumes, int32_t n_volumes, int32_t tile_shape, void* workspace,
                       size_t workspace_bytes, void* stream, bool insert) {
    const char* what = insert ? "insert_batched" : "extract_batched";
    if (!volumes || n_volumes < 0) return fail(TT_ERR_INVALID, "%s: bad volume list", what);
    if (n_volumes > kMaxBatch)
        return fail(TT_ERR_INVALID, "%s: %d volumes, at most %d per call", what, n_volumes, kMaxBatch);
    if (tile_shape < 0 || tile_shape > 2) return fail(TT_ERR_INVALID, "%s: tile_shape must be 0, 1 or 2", what);
    if (!workspace || workspace_bytes < sizeof(unsigned long long))
        return fail(TT_ERR_WORKSPACE, "%s: workspace of %zu bytes needed", what, sizeof(unsigned long long));
    static BatchParams bp;  // large; filled under the lock below
    static size_t acc_bytes[kMaxBatch];
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    bp.nvol = n_volumes;
    int layout = -1;  // every volume of an extraction batch gathers from the same layout
    int64_t slices = 0;
    for (int v = 0; v < n_volumes; v++) {
        const tt_batch_volume& x = volumes[v];
        if (int e = validate_params(&x.params, true)) return e;
        if (!insert && x.params.volume_layout == TT_VOLUME_XPAIRS)
            return fail(TT_ERR_INVALID, "%s: volume %d: the batched extraction takes plain or bricked volumes", what,
                        v);
        if (!insert && x.params.n > 0) {
            if (layout >= 0 && x.params.volume_layout != layout)
                return fail(TT_ERR_INVALID, "%s: volume %d: all volumes of one call share one volume_layout", what,
                            v);
            layout = x.params.volume_layout;
        }
        if (x.params.deterministic)
            return fail(TT_ERR_INVALID, "%s: volume %d: the batched launch has no deterministic mode", what, v);
        if (x.params.n > 0) {
            if (!x.rotation_matrices || !x.slices) return fail(TT_ERR_INVALID, "%s: volume %d: NULL pointer", what, v);
            if (insert) {
                if (!x.accumulator) return fail(TT_ERR_INVALID, "%s: volume %d: NULL accumulator", what, v);
                if (x.params.volume_layout != TT_VOLUME_PLAIN &&
                    (x.params.volume_layout != TT_VOLUME_BRICKS || x.params.volume_unshifted))
                    return fail(TT_ERR_INVALID,
                                "%s: volume %d: the accumulator is plain or (fftshifted volumes) bricked", what, v);
                if (x.params.vol_d != x.params.img_d || x.params.vol_h != x.params.img_h ||
                    x.params.vol_w != x.params.img_w / 2 + 1)
                    return fail(TT_ERR_INVALID, "%s: volume %d: dims are not the rfft of volume_shape", what, v);
            } else if (!x.volume_rfft) {
                return fail(TT_ERR_INVALID, "%s: volume %d: NULL volume", what, v);
            }
        }
        BatchVolumeDev& d = bp.v[v];
        d.g = make_geom(x.params);
        d.vol = (const float2*)x.volume_rfft;
        d.slices = (float2*)x.slices;
        d.acc = (float4*)x.accumulator;
        d.rot = x.rotation_matrices;
        d.ctf = x.ctf;
        acc_bytes[v] = x.params.volume_layout == TT_VOLUME_BRICKS
                           ? bricked_accumulator_bytes(&x.params)
                           : (size_t)(x.params.vol_d * x.params.vol_h * x.params.vol_w) * sizeof(float4);
        slices += x.params.n;
    }
    if (slices == 0) return TT_OK;
    cudaStream_t st = as_stream(stream);
    unsigned long long* queue = (unsigned long long*)workspace;
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return fail(TT_ERR_CUDA, "%s: memset: %s", what, cudaGetErrorString(e));
    if (insert) {
        if (tile_shape == 0) return launch_batched<8, true, float2>(bp, acc_bytes, queue, st);
        if (tile_shape == 1) return launch_batched<16, true, float2>(bp, acc_bytes, queue, st);
        return launch_batched<32, true, float2>(bp, acc_bytes, queue, st);
    }
    if (layout == TT_VOLUME_BRICKS) {
        if (tile_shape == 0) return launch_batched<8, false, VoxBrick2>(bp, acc_bytes, queue, st);
        if (tile_shape == 1) return launch_batched<16, false, VoxBrick2>(bp, acc_bytes, queue, st);
        return launch_batched<32, false, VoxBrick2>(bp, acc_bytes, queue, st);
    }
    if (tile_shape == 0) return launch_batched<8, false, float2>(bp, acc_bytes, queue, st);
    if (tile_shape == 1) return launch_batched<16, false, float2>(bp, acc_bytes, queue, st);
    return launch_batched<32, false, float2>(bp, acc_bytes, queue, st);
}

}  // namespace tt

using namespace tt;

extern "C" size_t tt_batch_workspace_bytes(void) { return 256; }

extern "C" int tt_extract_central_slices_rfft_3d_batched(const tt_batch_volume* volumes, int32_t n_volumes,
                                                         int32_t tile_shape, void* workspace, size_t workspace_bytes,
                                                         void* stream) {
    return run_batched(volumes, n_volumes, tile_shape, workspace, workspace_bytes, stream, false);
}

extern "C" int tt_insert_central_slices_rfft_3d_batched(const tt_batch_volume* volumes, int32_t n_volumes,
                                                        int32_t tile_shape, void* workspace, size_t workspace_bytes,
                                                        void* stream) {
    return run_batched(volumes, n_volumes, tile_shape, workspace, workspace_bytes, stream, true);
}
