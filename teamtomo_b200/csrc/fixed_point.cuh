// 64-bit fixed-point accumulation for the deterministic scatters.
//
// Floating-point atomics add in whatever order the memory system serves them,
// so a float accumulator differs in its last bits from launch to launch.  In
// the deterministic mode each contribution is rounded once to an integer at a
// power-of-two scale and added with 64-bit integer atomics; integer addition is
// associative, so the sums do not depend on the order, on how the slices are
// split into calls, or (with an integer all-reduce) on the number of GPUs.
//
// Scale.  The points of one slice lie on a plane lattice of spacing >= 1/2
// voxel.  A voxel takes contributions from points inside the 2 x 2 x 2 cell
// around it; a plane meets that cell in a region of area <= 4 sqrt(2), which
// holds at most 48 lattice points at spacing 1/2 (12 at spacing 1); the
// conjugate redirect adds at most one more sheet and the Friedel completion
// doubles the total: at most 192 < 2^8 contributions per slice, each at most
// |data| (interpolation weights and squared CTF values are at most 1).  With
// |data| < 2^E and at most 2^L slices every sum stays below 2^(E + 8 + L),
// so data are scaled by 2^(62 - 8 - L - E) and weights by 2^(62 - 8 - L).
#pragma once
#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

namespace tt {

constexpr int kFixedHeadroomBits = 8;
constexpr size_t kFixedHeaderBytes = 256;  // workspace prefix holding the absmax word

__host__ __device__ inline int ceil_log2(int64_t n) {
    int l = 0;
    while (l < 62 && ((int64_t)1 << l) < n) l++;
    return l;
}

// Scale of the data of a fixed-point accumulator (see above); absmax_bits is
// the float32 bit pattern of a bound on |re|, |im|.
__device__ __forceinline__ double fixed_data_scale(uint32_t absmax_bits, int slices_log2) {
    const float a = __uint_as_float(absmax_bits);
    int e = 0;
    if (a > 0.0f && a <= FLT_MAX) frexpf(a, &e);  // a = m 2^e, 0.5 <= m < 1, so a < 2^e
    return ldexp(1.0, 62 - kFixedHeadroomBits - slices_log2 - e);
}

__device__ __forceinline__ double fixed_weight_scale(int slices_log2) {
    return ldexp(1.0, 62 - kFixedHeadroomBits - slices_log2);
}

__device__ __forceinline__ void fixed_add(unsigned long long* a, double v) {
    const long long q = __double2ll_rn(v);
    if (q) atomicAdd(a, (unsigned long long)q);  // two's complement: signed sum
}

// Insertion splat target: 4 words (re, im, w, pad) per voxel.
struct FixedSplat {
    unsigned long long* acc;
    double sd, sw;  // data and weight scales
    template <typename R>
    __device__ __forceinline__ void operator()(int64_t vi, R dre, R dim, R w, R wscale) const {
        unsigned long long* a = acc + vi * 4;
        // float products are exact in double, so each term is rounded once
        fixed_add(a + 0, (double)dre * (double)w * sd);
        fixed_add(a + 1, (double)dim * (double)w * sd);
        fixed_add(a + 2, (double)w * (double)wscale * sw);
    }
};

// Launches of fixed_point.cu.
int launch_fixed_absmax(const void* data, int is_f64, int64_t count, uint32_t* absmax, cudaStream_t st);

}  // namespace tt
