// Status / error-text plumbing shared by the extern "C" entry points.
#pragma once
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include <string>

#include "../../include/teamtomo_b200.h"

namespace tt {

std::string& last_error_slot();

inline int fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
inline int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    last_error_slot() = buf;
    return code;
}

// Checks the launch that was just issued.
inline int check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(TT_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return TT_OK;
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Whether the bricked copy of the volume (8 slots per 2 x 2 x 2 brick) has
// fewer than 2^31 slots, the range of its 32-bit slot offsets.
inline bool bricks_fit(const tt_slice_params* p) {
    return ((p->vol_d + 1) / 2) * ((p->vol_h + 1) / 2) * ((p->vol_w + 1) / 2) * 8 < (1LL << 31);
}

// Validates the common slice parameters; vol_w must be the rfft width of a
// real dimension and all sizes must fit the int32 index arithmetic used on
// the per-slice grid.
inline int validate_params(const tt_slice_params* p, bool allow_layouts = false) {
    if (!p) return fail(TT_ERR_INVALID, "params is NULL");
    if (p->n < 0) return fail(TT_ERR_INVALID, "n must be >= 0 (got %lld)", (long long)p->n);
    if (p->img_d < 1 || p->img_h < 1 || p->img_w < 1)
        return fail(TT_ERR_INVALID, "image shape must be positive");
    if (p->vol_d < 1 || p->vol_h < 1 || p->vol_w < 1)
        return fail(TT_ERR_INVALID, "volume shape must be positive");
    const long long lim = 1LL << 30;
    if ((long long)p->img_h * (p->img_w / 2 + 1) >= lim || p->vol_d * p->vol_h * p->vol_w >= lim * 4)
        return fail(TT_ERR_INVALID, "slice or volume too large");
    if (p->n > (1LL << 31) - 1) return fail(TT_ERR_INVALID, "too many slices");
    if (p->deterministic != 0 && p->deterministic != 1) return fail(TT_ERR_INVALID, "deterministic must be 0 or 1");
    if (p->volume_layout < TT_VOLUME_PLAIN || p->volume_layout > TT_VOLUME_BRICKS)
        return fail(TT_ERR_INVALID, "volume_layout must be 0 (plain), 1 (x-paired) or 2 (bricked)");
    if (p->volume_layout != TT_VOLUME_PLAIN && !allow_layouts)
        return fail(TT_ERR_INVALID, "volume_layout: this entry point takes the plain volume layout");
    if (p->volume_layout == TT_VOLUME_BRICKS && !bricks_fit(p))
        return fail(TT_ERR_INVALID, "volume_layout: a bricked copy must hold fewer than 2^31 voxel slots");
    return TT_OK;
}

}  // namespace tt
