// Batched central-slice extraction / insertion over many volumes of uneven
// box sizes, each with its own set of rotations and an optional per-image
// CTF, in ONE persistent launch.
//
// Work queue: the slices of all volumes form one global list; each block
// takes the next slice from an atomic counter, finds its volume by binary
// search over the per-volume slice offsets, loads the rotation (and computes
// the slice's CTF constants) once, and walks the slice's pixel tiles.  Every
// slice of a volume is equal work, so the queue balances uneven box sizes
// and slice counts without any host-side scheduling.
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
    int64_t slice_offset[kMaxBatch + 1];
    BatchVolumeDev v[kMaxBatch];
};

// Pixel of this thread in tile `tile` for TX-wide tiles of 256 pixels
// (each warp covers TX x 32/TX pixels).
template <int TX>
__device__ __forceinline__ bool tile_pixel_t(const SliceGeom& g, int tile, int& iy, int& ix) {
    constexpr int TY = 256 / TX, RPW = 32 / TX;
    const int txt = (g.wr + TX - 1) / TX;
    const int ty = tile / txt, tx = tile - ty * txt;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    ix = tx * TX + (lane % TX);
    iy = ty * TY + warp * RPW + lane / TX;
    return ix < g.wr && iy < g.img_h;
}

template <int TX>
__host__ inline int tiles_t(int img_h, int wr) {
    constexpr int TY = 256 / TX;
    return ((wr + TX - 1) / TX) * ((img_h + TY - 1) / TY);
}

template <int TX, bool INSERT>
__global__ void __launch_bounds__(256)
batched_slices_kernel(const __grid_constant__ BatchParams bp, unsigned long long* __restrict__ queue,
                      int64_t total, int phase, int nphase) {
    __shared__ float m[9];
    __shared__ CtfConst cc;
    __shared__ int64_t cur;
    __shared__ int vsel;
    for (;;) {
        __syncthreads();  // m / cc / cur of the previous slice are no longer read
        if (threadIdx.x == 0) {
            const int64_t gs = (int64_t)atomicAdd(queue, 1ULL);
            int lo = 0, hi = bp.nvol;  // slice_offset[lo] <= gs < slice_offset[lo + 1]
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (bp.slice_offset[mid] <= gs) lo = mid;
                else hi = mid;
            }
            cur = gs;
            vsel = lo;
        }
        __syncthreads();
        const int64_t gs = cur;
        if (gs >= total) return;
        const BatchVolumeDev& bv = bp.v[vsel];
        const int64_t s = gs - bp.slice_offset[vsel];
        if (threadIdx.x < 9) m[threadIdx.x] = prep_rotation_elem(bv.rot, bv.g.rot_f64, s, threadIdx.x, bv.g, !INSERT);
        if (threadIdx.x == 0 && bv.ctf) cc = make_ctf_const(bv.ctf[s]);
        __syncthreads();
        const CtfConst* ccp = bv.ctf ? &cc : nullptr;
        for (int tile = 0; tile < bv.tiles; tile++) {
            int iy, ix;
            const bool has_pixel = tile_pixel_t<TX>(bv.g, tile, iy, ix);
            if (INSERT) {
                // z-phased filling of large accumulators (the same answer in every thread)
                if (nphase > 1) {
                    constexpr int TY = 256 / TX;
                    const int txt = (bv.g.wr + TX - 1) / TX;
                    const int ty = tile / txt, tx = tile - ty * txt;
                    if (insert_tile_phase(bv.g, m, min(ty * TY + TY / 2, bv.g.img_h - 1),
                                          min(tx * TX + TX / 2, bv.g.wr - 1), nphase) != phase)
                        continue;
                }
                // every lane takes part: lane pairs share a pixel's x-corners
                insert_point_paired(bv.slices, m, bv.acc, bv.g, s, has_pixel, iy, ix, ccp);
            } else {
                if (!has_pixel) continue;
                float qy, qx, c[3];
                bool cj = false;
                float2 r = make_float2(0.0f, 0.0f);
                if (extract_geometry(bv.g, m, iy, ix, qy, qx, cj, c)) {
                    r = sample_trilinear(bv.vol, bv.g, make_corners(bv.g, c));
                    if (cj) r.y = -r.y;
                    if (ccp) {
                        const float cv = ctf_value(*ccp, qy, qx);
                        r.x *= cv;
                        r.y *= cv;
                    }
                }
                __stcs(bv.slices + (s * bv.g.img_h + slice_row(bv.g, iy)) * (int64_t)bv.g.wr + ix, r);
            }
        }
    }
}

template <int TX>
static int tiles_for_shape(const SliceGeom& g) {
    return tiles_t<TX>(g.img_h, g.wr);
}

int insert_phases(size_t acc_bytes);  // insert.cu

template <int TX, bool INSERT>
static int launch_batched(BatchParams& bp, unsigned long long* queue, int64_t total, cudaStream_t st) {
    for (int v = 0; v < bp.nvol; v++) bp.v[v].tiles = tiles_for_shape<TX>(bp.v[v].g);
    int dev = 0, sms = 148, occ = 1;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batched_slices_kernel<TX, INSERT>, 256, 0) !=
            cudaSuccess ||
        occ < 1)
        occ = 1;
    int64_t blocks = (int64_t)sms * occ;
    if (blocks > total) blocks = total;
    // insertion into large accumulators runs in z-phases (insert_phases), one queue pass each
    int nphase = 1;
    if (INSERT)
        for (int v = 0; v < bp.nvol; v++) {
            const int k = insert_phases((size_t)((int64_t)bp.v[v].g.D * bp.v[v].g.H * bp.v[v].g.W) * sizeof(float4));
            nphase = k > nphase ? k : nphase;
        }
    for (int ph = 0; ph < nphase; ph++) {
        if (ph > 0) {
            cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st);
            if (e != cudaSuccess) return fail(TT_ERR_CUDA, "batched: memset: %s", cudaGetErrorString(e));
        }
        batched_slices_kernel<TX, INSERT><<<(unsigned)blocks, 256, 0, st>>>(bp, queue, total, ph, nphase);
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
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    bp.nvol = n_volumes;
    bp.slice_offset[0] = 0;
    for (int v = 0; v < n_volumes; v++) {
        const tt_batch_volume& x = volumes[v];
        if (int e = validate_params(&x.params)) return e;
        if (x.params.deterministic)
            return fail(TT_ERR_INVALID, "%s: volume %d: the batched launch has no deterministic mode", what, v);
        if (x.params.n > 0) {
            if (!x.rotation_matrices || !x.slices) return fail(TT_ERR_INVALID, "%s: volume %d: NULL pointer", what, v);
            if (insert) {
                if (!x.accumulator) return fail(TT_ERR_INVALID, "%s: volume %d: NULL accumulator", what, v);
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
        bp.slice_offset[v + 1] = bp.slice_offset[v] + x.params.n;
    }
    const int64_t total = bp.slice_offset[n_volumes];
    if (total == 0) return TT_OK;
    cudaStream_t st = as_stream(stream);
    unsigned long long* queue = (unsigned long long*)workspace;
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return fail(TT_ERR_CUDA, "%s: memset: %s", what, cudaGetErrorString(e));
    if (insert) {
        if (tile_shape == 0) return launch_batched<8, true>(bp, queue, total, st);
        if (tile_shape == 1) return launch_batched<16, true>(bp, queue, total, st);
        return launch_batched<32, true>(bp, queue, total, st);
    }
    if (tile_shape == 0) return launch_batched<8, false>(bp, queue, total, st);
    if (tile_shape == 1) return launch_batched<16, false>(bp, queue, total, st);
    return launch_batched<32, false>(bp, queue, total, st);
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
