// Measurement probe: the L2's float4 reduction rate for a scatter over a
// buffer of a given size, the ceiling the insertion splat is measured against.
//
// The insertion adds one (re, im, w, 0) float4 per trilinear corner with a
// vector reduction; its time is set by how many of those the L2 retires per
// second, not by HBM bytes.  This kernel issues the same instruction in a
// controlled pattern: groups of `lanes` lanes of a warp (1, 2, 4 or 8) add to
// adjacent 16-byte slots of one 128-byte line, each group's line drawn by a
// hash of the group index over the whole buffer.  Eight lanes per line over a
// buffer larger than the L2 is the pattern of a lane-octet splat into a
// bricked accumulator without the locality of neighbouring pixels; over a
// buffer that fits the L2 it is the same pattern with every line resident.
#include <cuda_runtime.h>

#include "capi_util.cuh"

namespace tt {

__device__ __forceinline__ unsigned long long probe_mix(unsigned long long x) {
    // splitmix64 finaliser
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebULL;
    x ^= x >> 31;
    return x;
}

__global__ void __launch_bounds__(256) l2_reduction_probe_kernel(float4* __restrict__ buf, unsigned long long lines,
                                                                 long long groups, int lanes,
                                                                 unsigned long long seed) {
    const int lane = threadIdx.x & 31;
    const int per_warp = 32 / lanes;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long w = warp; w * per_warp < groups; w += warps) {
        const long long gi = w * per_warp + lane / lanes;
        if (gi < groups) {
            // multiply-shift range reduction of the hash's high word (no 64-bit division:
            // the probe must not be bound by its own index arithmetic)
            const unsigned long long h = probe_mix((unsigned long long)gi ^ seed) >> 32;
            const unsigned long long line = (h * lines) >> 32;
            atomicAdd(buf + line * 8 + (lane % lanes), make_float4(1.0f, 1.0f, 1.0f, 0.0f));
        }
    }
}

}  // namespace tt

using namespace tt;

extern "C" int tt_probe_l2_reductions(void* buffer, size_t bytes, int64_t reductions, int32_t lanes_per_line,
                                      uint64_t seed, void* stream) {
    if (!buffer) return fail(TT_ERR_INVALID, "probe_l2_reductions: NULL buffer");
    if ((reinterpret_cast<uintptr_t>(buffer) & 127) != 0)
        return fail(TT_ERR_INVALID, "probe_l2_reductions: the buffer must be 128-byte aligned");
    if (bytes < 128 || bytes % 128 != 0 || bytes / 128 > 0xffffffffULL)
        return fail(TT_ERR_INVALID, "probe_l2_reductions: bytes must be a positive multiple of 128 below 512 GiB");
    if (lanes_per_line != 1 && lanes_per_line != 2 && lanes_per_line != 4 && lanes_per_line != 8)
        return fail(TT_ERR_INVALID, "probe_l2_reductions: lanes_per_line must be 1, 2, 4 or 8");
    if (reductions < 0) return fail(TT_ERR_INVALID, "probe_l2_reductions: negative count");
    const long long groups = reductions / lanes_per_line;
    if (groups == 0) return TT_OK;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    l2_reduction_probe_kernel<<<(unsigned)(sms * 8), 256, 0, as_stream(stream)>>>(
        (float4*)buffer, (unsigned long long)(bytes / 128), groups, lanes_per_line, (unsigned long long)seed);
    return check_launch("l2_reduction_probe_kernel");
}
