/*
 * teamtomo_b200 — C ABI of the B200 Fourier-slice kernels.
 *
 * Every entry point takes raw device pointers (C-contiguous, CUDA memory of
 * the current device), sizes in a parameter struct, and a CUDA stream handle
 * (cudaStream_t passed as void*, NULL = legacy default stream).  Launches are
 * asynchronous on that stream; no entry point synchronises the host, and none
 * allocates device memory: scratch space is passed in by the caller
 * (see the *_workspace_bytes queries).  The return value is a status code
 * (TT_OK on success); tt_last_error() gives the message of the last failure
 * on the calling thread.
 *
 * Complex arrays are interleaved (re, im): complex64 = 2 x float32,
 * complex128 = 2 x float64.  "fftshifted rfft" volumes have shape
 * (d, h, w/2+1) with the zero frequency at (d/2, h/2, 0), the layout the
 * reference functions consume and produce.
 *
 * Reference interfaces replaced (teamtomo monorepo, packages/primitives/…):
 *   torch-fourier-slice/src/torch_fourier_slice/slice_extraction/_extract_central_slices_rfft_3d.py
 *   torch-fourier-slice/src/torch_fourier_slice/slice_insertion/_insert_central_slices_rfft_3d.py
 *   torch-fourier-slice/src/torch_fourier_slice/project.py, backproject.py
 *   torch-image-interpolation/src/torch_image_interpolation/image_interpolation_3d.py
 * The reference is pure Python over PyTorch; these entry points are what its
 * torch ops (grid_sample, index_put_, bmm, boolean indexing) are replaced by.
 */
#ifndef TEAMTOMO_B200_H
#define TEAMTOMO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    TT_OK = 0,
    TT_ERR_INVALID = 1,   /* bad shape, size, flag or NULL pointer */
    TT_ERR_CUDA = 2,      /* a CUDA launch or runtime call failed */
    TT_ERR_WORKSPACE = 3  /* workspace missing or too small */
};

/* Layouts of the volume the extraction gathers read (tt_slice_params.volume_layout). */
enum tt_volume_layout {
    TT_VOLUME_PLAIN = 0,   /* the complex64 rfft volume itself */
    TT_VOLUME_XPAIRS = 1,  /* x-paired copy, tt_pack_volume_xpairs */
    TT_VOLUME_BRICKS = 2   /* 2 x 2 x 2 bricked copy, tt_pack_volume_bricks */
};

/* Geometry of one batch of central slices through one rfft volume. */
typedef struct tt_slice_params {
    int64_t n;                     /* number of slices (rotation matrices) */
    int64_t img_d, img_h, img_w;   /* real-space shape defining the slice grid and the
                                      frequency->array scaling: image_shape for extraction,
                                      volume_shape for insertion */
    int64_t vol_d, vol_h, vol_w;   /* dims of the rfft volume array, (d, h, w/2+1) */
    int32_t has_fftfreq_max;       /* 1: keep only |f| <= fftfreq_max */
    float fftfreq_max;
    int32_t zyx_matrices;          /* 0: matrices act on xyz column vectors (default) */
    float x_tolerance;             /* extraction: conjugate tie-break tolerance (f32) */
    float x_tolerance10;           /* f32(x_tolerance * 10), computed in double first */
    int32_t has_rot_tolerance;     /* extraction: zero |R_ij| < rot_tolerance */
    float rot_tolerance;
    int32_t rotation_f64;          /* rotation matrices are float64 (else float32) */
    int32_t volume_unshifted;      /* volume is plain rfftn output (z, y not fftshifted) */
    int32_t slices_unshifted;      /* slices stored ifftshifted along rows (irfft-ready) */
    int32_t deterministic;         /* 1: insertion and the volume gradient accumulate in 64-bit
                                      fixed point, bit-identical for any launch order (the
                                      workspace queries grow accordingly) */
    int32_t volume_layout;         /* layout of volume_rfft (tt_volume_layout): TT_VOLUME_PLAIN,
                                      TT_VOLUME_XPAIRS (the copy of tt_pack_volume_xpairs) or
                                      TT_VOLUME_BRICKS (tt_pack_volume_bricks); the copies are
                                      taken by the extraction forward, backward and
                                      tt_central_slice_mse only, other entry points refuse them.
                                      Occupies the struct's former tail padding: 0 keeps the
                                      plain layout, so zero-initialised structs are unchanged. */
} tt_slice_params;

/* Per-image contrast transfer function, the scalar arguments of torch-ctf's
 * calculate_ctf_2d (torch_ctf/ctf_2d.py:12-131) without the Zernike / beam
 * tilt / anisotropic-magnification extras. */
typedef struct tt_ctf_params {
    float defocus_um;              /* (defocus_u + defocus_v) / 2, positive is underfocus */
    float astigmatism_um;          /* (defocus_u - defocus_v) / 2 */
    float astigmatism_angle_deg;   /* 0 places defocus_u along y */
    float voltage_kv;
    float spherical_aberration_mm;
    float amplitude_contrast;      /* fraction in [0, 1) */
    float phase_shift_deg;
    float pixel_size_a;            /* Angstrom per pixel */
} tt_ctf_params;

/* Library version (major*10000 + minor*100 + patch) and last error text. */
int tt_version(void);
const char *tt_last_error(void);

/* Central-slice extraction (trilinear gather with the reference's Hermitian
 * redirect).  volume_rfft: complex64 (vol_d, vol_h, vol_w); rotation_matrices:
 * (n, 3, 3) float32 or float64; slices_out: complex64 (n, img_h, img_w/2+1),
 * fully written (zeros outside fftfreq_max / outside the volume).
 * Replaces extract_central_slices_rfft_3d,
 * _extract_central_slices_rfft_3d.py:84-222 (+ :9-81). */
int tt_extract_central_slices_rfft_3d(const void *volume_rfft, const void *rotation_matrices,
                                      void *slices_out, const tt_slice_params *p, void *stream);

/* Per-pixel geometry of the slice grid under the extraction (mode 0) or the
 * insertion (mode 1) rule, for bit-exact checks of the index and mask logic:
 * flags (n, img_h, img_w/2+1) uint8 — bit0 pixel kept (inside fftfreq_max and,
 * for insertion, not the Friedel-redundant x==0, y<0 source pixel), bit1
 * conjugate redirect, bit2 inside the volume; coords (n, img_h, img_w/2+1, 3)
 * float32 zyx array coordinates after the redirect (0 for dropped pixels).
 * Exposes the intermediate values of _extract_central_slices_rfft_3d.py:183-209
 * and _insert_central_slices_rfft_3d.py:30-85, which the reference keeps internal. */
int tt_slice_geometry(const void *rotation_matrices, int32_t mode, uint8_t *flags, float *coords,
                      const tt_slice_params *p, void *stream);

/* x-paired copy of an rfft volume for the extraction gathers: entry (z, y, x)
 * holds the complex64 pair (V[z, y, x], V[z, y, x + 1]) as four floats, the
 * second zero in the last column, in the (z, y) order of the source (fftshifted,
 * or plain when p->volume_unshifted).  A pixel's eight trilinear corners are
 * then four 16-byte loads instead of eight 8-byte ones, which lowers the L1
 * wavefronts of the scattered gathers.  Pass the copy as volume_rfft with
 * p->volume_layout = TT_VOLUME_XPAIRS; results are bit-identical to the plain layout.
 * tt_volume_xpairs_bytes: p->vol_d * vol_h * vol_w * 16.  The source is
 * complex64 (vol_d, vol_h, vol_w); xpairs must be 16-byte aligned.  The
 * reference has no such layout (it samples with grid_sample on the volume). */
size_t tt_volume_xpairs_bytes(const tt_slice_params *p);
int tt_pack_volume_xpairs(const void *volume_rfft, void *xpairs, const tt_slice_params *p, void *stream);

/* Bricked copy of an rfft volume for the extraction gathers: 2 x 2 x 2 voxel
 * bricks of 64 bytes in (z, y, x) brick order, voxels (z, y, x) inside a
 * brick, always in fftshifted (z, y) order (a p->volume_unshifted source is
 * shifted while packing).  Voxel (z, y, x) sits at complex64 index
 *   ((z/2 * ceil(vol_h/2) + y/2) * ceil(vol_w/2) + x/2) * 8 + (z%2)*4 + (y%2)*2 + x%2,
 * slots past an odd dimension are zero.  A 128-byte line then holds a
 * 4 x 2 x 2 block of voxels instead of 16 voxels of one row, so the
 * trilinear corners of a warp's 8 x 4 pixels touch fewer lines.  Pass the
 * copy as volume_rfft with p->volume_layout = TT_VOLUME_BRICKS; results are
 * bit-identical to the plain layout.  tt_volume_bricks_bytes:
 * ceil(vol_d/2) * ceil(vol_h/2) * ceil(vol_w/2) * 64.  The source is complex64
 * (vol_d, vol_h, vol_w), 8-byte aligned; bricks must be 16-byte aligned and
 * hold fewer than 2^31 slots (boxes up to about 2000^3).  The
 * reference has no such layout (it samples with grid_sample on the volume). */
size_t tt_volume_bricks_bytes(const tt_slice_params *p);
int tt_pack_volume_bricks(const void *volume_rfft, void *bricks, const tt_slice_params *p, void *stream);

/* Bytes of workspace tt_extract_central_slices_rfft_3d_backward needs when a
 * rotation gradient or (p->deterministic) a volume gradient is requested
 * (otherwise 0 is also accepted). */
size_t tt_extract_backward_workspace_bytes(const tt_slice_params *p);

/* Backward of the extraction.  grad_slices: complex64 (n, img_h, img_w/2+1),
 * PyTorch's convention for complex gradients (dL = Re(conj(G) dS)).
 * grad_volume (nullable): complex64 (vol_d, vol_h, vol_w), ACCUMULATED into.
 * grad_rotation (nullable): (n, 3, 3) in the rotation dtype, overwritten; the
 * elements zeroed by rot_tolerance get zero gradient.  The rotation gradient
 * is reduced deterministically through the caller's workspace; with
 * p->deterministic the volume gradient is accumulated in 64-bit fixed point
 * there too (scale from the grads' max |re|, |im| and n) and then added in.
 * Replaces the autograd graph of extract_central_slices_rfft_3d
 * (grid_sampler_3d_backward + the coordinate chain of _dft_utils.py:61-67). */
int tt_extract_central_slices_rfft_3d_backward(const void *volume_rfft,
                                               const void *rotation_matrices,
                                               const void *grad_slices, void *grad_volume,
                                               void *grad_rotation, void *workspace,
                                               size_t workspace_bytes,
                                               const tt_slice_params *p, void *stream);

/* Fused extraction + mean squared error + backward, for fitting a volume
 * and/or orientations to target slices:
 *   *loss = mean over the n * img_h * (img_w/2+1) complex elements of
 *           |extract(volume_rfft, R) - targets|^2            (device float)
 * and, for the loss itself as the objective (upstream gradient 1),
 * grad_volume (nullable, ACCUMULATED into) and grad_rotation (nullable, (n,3,3)
 * in the rotation dtype, overwritten) — the gradients
 * tt_extract_central_slices_rfft_3d_backward computes for G = 2 (S - T) / M,
 * without writing S or reading G: the sample is rebuilt from the corner
 * values the rotation gradient loads anyway.  The loss and the rotation
 * gradient are reduced in a fixed order.  targets: complex64 (n, img_h, img_w/2+1).
 * Workspace: tt_central_slice_mse_workspace_bytes.  No deterministic mode.
 * The reference has no fused loss; this replaces extract_central_slices_rfft_3d
 * + a torch MSE + its autograd backward. */
size_t tt_central_slice_mse_workspace_bytes(const tt_slice_params *p);
int tt_central_slice_mse(const void *volume_rfft, const void *rotation_matrices, const void *targets,
                         float *loss, void *grad_volume, void *grad_rotation, void *workspace,
                         size_t workspace_bytes, const tt_slice_params *p, void *stream);

/* Size of the built-in scratch array used by
 * tt_extract_central_slices_rfft_3d_backward_noalloc (per GPU, for the life of
 * the process). */
#define TT_NOALLOC_SCRATCH_BYTES (4u << 20)

/* Same computation as tt_extract_central_slices_rfft_3d_backward, for callers
 * that cannot allocate device memory (a host or plugin framework that owns
 * all device allocations and only hands over the buffers of the call, or a
 * fixed memory budget that must not grow): it takes no workspace and calls no
 * allocator; the rotation-gradient partial sums go to a 4 MiB array built
 * into the library instead.
 *  - Limit: when grad_rotation is requested, n * ceil(img_h / 32) * 24 bytes
 *    (the partial sums of each row of 8 x 32 pixel tiles) must not exceed
 *    TT_NOALLOC_SCRATCH_BYTES (at a 256^3 box that is 21845 slices per call);
 *    larger calls fail with TT_ERR_INVALID and a message.
 *  - The first call on each device looks up the array's device address
 *    (cudaGetSymbolAddress) with that device current; make it before any
 *    stream capture.
 *  - All calls share the array: calls that overlap on the GPU race and must be
 *    serialised by the caller.  Each call writes every slot it reads, so
 *    nothing needs clearing between calls.
 *  - The deterministic (fixed-point) volume gradient needs a workspace: a
 *    call with p->deterministic and a grad_volume fails with TT_ERR_INVALID.
 * This entry point has no counterpart in the reference. */
int tt_extract_central_slices_rfft_3d_backward_noalloc(const void *volume_rfft,
                                                       const void *rotation_matrices,
                                                       const void *grad_slices,
                                                       void *grad_volume, void *grad_rotation,
                                                       const tt_slice_params *p, void *stream);

/* Central-slice insertion: trilinear scatter of the slices and of the
 * interpolation weights with the reference's strict x<0 conjugate redirect,
 * the x=0/y<0 source-pixel exclusion and whole-point bounds rejection, then
 * the Friedel completion of the x=0 plane.  volume_rfft (vol_d, vol_h, vol_w)
 * and weights (same dims) are OVERWRITTEN.  complex128 = 1: image/volume
 * complex128 and weights float64 (coordinates and weights still computed in
 * float32, as the reference does); else complex64 / float32.  The workspace
 * holds the accumulator (tt_insert_accumulator_bytes(complex128, 1, ...)).
 * Replaces insert_central_slices_rfft_3d, _insert_central_slices_rfft_3d.py:9-106, :213-406. */
int tt_insert_central_slices_rfft_3d(const void *image_rfft, int32_t complex128,
                                     const void *rotation_matrices, void *volume_rfft,
                                     void *weights, void *workspace, size_t workspace_bytes,
                                     const tt_slice_params *p, void *stream);

/* Backward of the insertion w.r.t. the slices: grad_image (n, img_h, img_w/2+1)
 * is OVERWRITTEN with dL/dslices for upstream grad_volume (vol dims), both
 * complex64 (complex128 = 0) or complex128, in PyTorch's complex-gradient
 * convention.  The adjoint of the splat (the same float32 corner weights,
 * gathered; conjugated where the point was redirected; zero for dropped
 * pixels) and of the Friedel completion of the x=0 plane.  The weights output
 * does not depend on the slices, so its gradient contributes nothing.
 * complex64 with p->volume_layout = TT_VOLUME_BRICKS: grad_volume is the
 * bricked copy of an fftshifted gradient volume (tt_pack_volume_bricks); the
 * gathers then read fewer lines (256^3 x 4096: 1.23 vs 1.76 ms), results
 * bit-identical.
 * Replaces the autograd graph of insert_central_slices_rfft_3d w.r.t. image_rfft
 * (index_put_ backward of _insert_central_slices_rfft_3d.py:213-406). */
int tt_insert_central_slices_rfft_3d_backward(const void *grad_volume, int32_t complex128,
                                              const void *rotation_matrices, void *grad_image,
                                              const tt_slice_params *p, void *stream);

/* Bytes of an insertion accumulator for `channels` volumes of (d, h, w_rfft):
 * one (re, im, w, pad) slot per voxel, 16 bytes (complex64) or 32 (complex128). */
size_t tt_insert_accumulator_bytes(int32_t complex128, int64_t channels, int64_t d, int64_t h,
                                   int64_t w_rfft);

/* Two-stage insertion for accumulating many batches into one volume:
 * tt_insert_accumulate adds the splat of n slices into a caller-zeroed
 * accumulator (no Friedel completion); call it any number of times, then
 * tt_insert_finalize once to write volume (channels, d, h, w_rfft) and
 * weights (d, h, w_rfft, may be NULL) with the x=0 plane completed. */
int tt_insert_accumulate(const void *image_rfft, int32_t complex128, const void *rotation_matrices,
                         void *accumulator, const tt_slice_params *p, void *stream);
int tt_insert_finalize(const void *accumulator, int32_t complex128, int64_t channels, int64_t d,
                       int64_t h, int64_t w_rfft, void *volume_rfft, void *weights, void *stream);

/* Accumulator layout for p's volume in the batched float insertion:
 * TT_VOLUME_BRICKS from 64 MB of accumulator up while it fits one z-phase
 * (about 1.1 x the L2; fftshifted volumes), else TT_VOLUME_PLAIN (the
 * one-shot tt_insert_central_slices_rfft_3d bricks every accumulator from
 * 64 MB up, whatever its phases).  A bricked accumulator holds 2 x 2 x 2 voxel bricks of 8
 * (re, im, w, pad) float32 slots (one 128-byte line) in (z, y, x) brick
 * order, x fastest inside a brick, dims rounded up to even
 * (tt_insert_bricked_accumulator_bytes); the splat reduces the eight
 * corners of a pixel in one instruction.  The batched insertion takes one
 * per volume (params.volume_layout = TT_VOLUME_BRICKS), finished by
 * tt_insert_finalize_bricked.  No counterpart in the reference (its
 * index_put_ accumulates into the output volume directly). */
int32_t tt_insert_accumulator_layout(const tt_slice_params *p);
size_t tt_insert_bricked_accumulator_bytes(int64_t d, int64_t h, int64_t w_rfft);
/* Bricked accumulator -> volume (d, h, w_rfft) complex64 and weights (may be
 * NULL) with the Friedel completion of the x=0 plane, as tt_insert_finalize. */
int tt_insert_finalize_bricked(const void *accumulator, int64_t d, int64_t h, int64_t w_rfft,
                               void *volume_rfft, void *weights, void *stream);

/* Friedel completion of the x=0 plane, equal to the reference's per-corner
 * mirror insertion (_insert_central_slices_rfft_3d.py:350-404):
 * out[v] = acc[v] + conj(acc[m(v)]) unless m(v) is the DC voxel, with
 * m(z, y) = ((d - z) % d, (h - y) % h), and the same for the weights.
 * channels volumes of (d, h, w_rfft) share one weight volume (weights may be
 * NULL).  In place. */
int tt_friedel_mirror_x0(void *volume_rfft, void *weights, int32_t complex128, int64_t channels,
                         int64_t d, int64_t h, int64_t w_rfft, void *stream);

/* ---- deterministic scatters (64-bit fixed point) ----------------------
 * Every contribution data*w is rounded to a 64-bit integer at a power-of-two
 * scale and added with integer atomics, which are associative: the sums are
 * identical for any launch order, any split of the slices into calls and,
 * summing accumulators with an integer all-reduce, any number of GPUs.  The
 * scale follows from a bound on |data| (the float32 bit pattern of max |re|,
 * |im| -- see tt_fixed_absmax) and on the number of slices ever added to the
 * accumulator (max_slices): data scale 2^(54 - ceil(log2 max_slices) - E)
 * with |data| < 2^E, weight scale 2^(54 - ceil(log2 max_slices)), which keeps
 * every sum below 2^62 (a voxel receives at most 256 contributions of at most
 * |data| per slice, Friedel completion included).  All calls that add into
 * one accumulator must use the same absmax value and max_slices.  Non-finite
 * data are not supported in this mode.
 * One-shot use: set tt_slice_params.deterministic = 1 on
 * tt_insert_central_slices_rfft_3d (workspace: tt_insert_workspace_bytes) or
 * on tt_extract_central_slices_rfft_3d_backward (volume gradient; workspace:
 * tt_extract_backward_workspace_bytes).  The reference accumulates with
 * float atomics (index_put_ with accumulate=True) and has no such mode. */

/* Bytes of workspace tt_insert_central_slices_rfft_3d needs for p
 * (p->deterministic selects the fixed-point layout). */
size_t tt_insert_workspace_bytes(int32_t complex128, const tt_slice_params *p);

/* *absmax_bits = max(*absmax_bits, bits of max |x| over count float32 (is_f64 = 0)
 * or float64 (is_f64 = 1, rounded up to float32) values).  Non-negative
 * float32 values order like their bit patterns, so the caller zeroes the word
 * once and may run this over several buffers (or all-reduce it with MAX). */
int tt_fixed_absmax(const void *data, int32_t is_f64, int64_t count, uint32_t *absmax_bits,
                    void *stream);

/* Bytes of a fixed-point insertion accumulator: 4 int64 (re, im, w, pad) per voxel. */
size_t tt_insert_fixed_accumulator_bytes(int64_t channels, int64_t d, int64_t h, int64_t w_rfft);

/* Two-stage deterministic insertion: adds the splat of n slices into a
 * caller-zeroed fixed-point accumulator, at the scale given by *absmax_bits
 * (device memory) and max_slices. */
int tt_insert_fixed_accumulate(const void *image_rfft, int32_t complex128,
                               const void *rotation_matrices, void *accumulator,
                               const uint32_t *absmax_bits, int64_t max_slices,
                               const tt_slice_params *p, void *stream);

/* Fixed-point accumulator -> volume (channels, d, h, w_rfft) and weights
 * (d, h, w_rfft, may be NULL), Friedel completion of the x=0 plane done in
 * integers, then one conversion back at the same scale. */
int tt_insert_fixed_finalize(const void *accumulator, int32_t complex128, int64_t channels,
                             int64_t d, int64_t h, int64_t w_rfft, const uint32_t *absmax_bits,
                             int64_t max_slices, void *volume_rfft, void *weights, void *stream);

/* ---- central lines of 2D images -----------------------------------------
 * image_rfft: complex64 (img_h, img_w_rfft), fftshifted along h (the rfft of an
 * (h, w) image); rotation_matrices (n, 2, 2) float32 or float64 (rotation_f64),
 * acting on xy column vectors unless yx_matrices; lines_out complex64
 * (n, w/2+1), fully written (zeros beyond fftfreq_max / outside the image).
 * Replaces extract_central_slices_rfft_2d (_extract_central_slices_rfft_2d.py:9-84);
 * the reference raises for any fftfreq_max (its mask is taken over the (w, 2)
 * coordinate grid), here it zeroes the samples with frequency > fftfreq_max. */
int tt_extract_central_lines_rfft_2d(const void *image_rfft, int64_t img_h, int64_t img_w_rfft,
                                     const void *rotation_matrices, int32_t rotation_f64, int64_t n,
                                     int64_t h, int64_t w, int32_t has_fftfreq_max, float fftfreq_max,
                                     int32_t yx_matrices, void *lines_out, void *stream);
/* Backward: grad_image (img_h, img_w_rfft) ACCUMULATED into (nullable),
 * grad_rotation (n, 2, 2) in the rotation dtype, overwritten (nullable);
 * grad_lines in PyTorch's complex-gradient convention. */
int tt_extract_central_lines_rfft_2d_backward(const void *image_rfft, int64_t img_h, int64_t img_w_rfft,
                                              const void *rotation_matrices, int32_t rotation_f64,
                                              int64_t n, int64_t h, int64_t w, int32_t has_fftfreq_max,
                                              float fftfreq_max, int32_t yx_matrices,
                                              const void *grad_lines, void *grad_image,
                                              void *grad_rotation, void *stream);

/* ---- multichannel slices (c volumes, one set of rotations) -------------
 * Each pixel's geometry is computed once and applied to every channel.
 * Volumes (channels, vol_d, vol_h, vol_w) complex64; slices
 * (n, channels, img_h, img_w/2+1) complex64 — the reference's (..., c, h, w)
 * layout.  Replace the per-channel loops of
 * extract_central_slices_rfft_3d_multichannel (_extract_central_slices_rfft_3d.py:225-367)
 * and insert_central_slices_rfft_3d_multichannel (_insert_central_slices_rfft_3d.py:109-210).
 * The two extraction entry points also take p->volume_layout =
 * TT_VOLUME_BRICKS: volume_rfft is then the channels' bricked copies
 * (tt_pack_volume_bricks of each channel) back to back, each
 * tt_volume_bricks_bytes long; grad_volume stays plain.  They refuse
 * TT_VOLUME_XPAIRS. */
int tt_extract_central_slices_rfft_3d_multichannel(const void *volume_rfft, int64_t channels,
                                                   const void *rotation_matrices, void *slices_out,
                                                   const tt_slice_params *p, void *stream);
/* grad_volume (channels, ...) ACCUMULATED into; grad_rotation summed over the
 * channels (workspace: tt_extract_backward_workspace_bytes with
 * p->deterministic = 0; no deterministic mode here). */
int tt_extract_central_slices_rfft_3d_multichannel_backward(
    const void *volume_rfft, int64_t channels, const void *rotation_matrices,
    const void *grad_slices, void *grad_volume, void *grad_rotation, void *workspace,
    size_t workspace_bytes, const tt_slice_params *p, void *stream);
/* Splat of (n, channels, h, w/2+1) complex64 slices into `channels` caller-zeroed
 * float accumulators (tt_insert_accumulator_bytes(0, channels, ...)), one
 * channel after the other; every channel's slots also receive the
 * interpolation weights, and tt_insert_finalize reads them from channel 0. */
int tt_insert_accumulate_multichannel(const void *image_rfft, int64_t channels,
                                      const void *rotation_matrices, void *accumulator,
                                      const tt_slice_params *p, void *stream);
/* Backward of the multichannel insertion w.r.t. the slices (per channel as
 * tt_insert_central_slices_rfft_3d_backward), complex64; grad_image overwritten. */
int tt_insert_central_slices_rfft_3d_multichannel_backward(const void *grad_volume, int64_t channels,
                                                           const void *rotation_matrices,
                                                           void *grad_image,
                                                           const tt_slice_params *p, void *stream);

/* ---- batched, CTF-weighted slices over many volumes -------------------
 * Many volumes of uneven box size, each with its own rotations and optional
 * per-image CTF, in ONE persistent launch whose blocks take slices from a
 * work queue.  The call issues a memset of the workspace (the queue counter)
 * and the launch on `stream`; it copies nothing and is capturable into a
 * CUDA graph.  complex64 only.  tile_shape: 0 = 8x32, 1 = 16x16, 2 = 32x8
 * pixels per block (chosen per box size by the Python autotuner).
 * The reference has no batched entry point: these run its per-volume
 * extract / insert semantics for each volume of the list. */
#define TT_MAX_BATCH_VOLUMES 96

typedef struct tt_batch_volume {
    tt_slice_params params;          /* geometry of this volume's slices (params.n = its slice count) */
    const void *volume_rfft;         /* extraction: complex64 source volume */
    void *slices;                    /* extraction: complex64 output (n, h, w/2+1); insertion: input */
    void *accumulator;               /* insertion: (re, im, w, pad) float32 slots, zeroed by the caller;
                                        bricked when params.volume_layout = TT_VOLUME_BRICKS
                                        (tt_insert_accumulator_layout) */
    const void *rotation_matrices;   /* (n, 3, 3) float32 or float64 */
    const tt_ctf_params *ctf;        /* device array of n CTFs, or NULL for none.  Extraction
                                        multiplies each slice by its CTF; insertion weights the
                                        data by the CTF and the interpolation weights by CTF^2 */
} tt_batch_volume;

size_t tt_batch_workspace_bytes(void);
int tt_extract_central_slices_rfft_3d_batched(const tt_batch_volume *volumes, int32_t n_volumes,
                                              int32_t tile_shape, void *workspace,
                                              size_t workspace_bytes, void *stream);
/* Accumulates into each volume's accumulator; finish each volume with
 * tt_insert_finalize, or tt_insert_finalize_bricked for a bricked one
 * (Friedel completion, volume + weights). */
int tt_insert_central_slices_rfft_3d_batched(const tt_batch_volume *volumes, int32_t n_volumes,
                                             int32_t tile_shape, void *workspace,
                                             size_t workspace_bytes, void *stream);

/* ---- measurement probe ------------------------------------------------
 * `reductions` float4 additions into `buffer` (`bytes`: a positive multiple
 * of 128 below 512 GiB, 128-byte aligned) in groups of `lanes_per_line` (1, 2, 4 or 8)
 * lanes of a warp on adjacent 16-byte slots of one 128-byte line, each
 * group's line drawn by a hash of its index and `seed`: the L2's float4
 * reduction rate for a scatter over a buffer of that size, the ceiling the
 * insertion splat is measured against.  The buffer's contents are
 * incremented (no other meaning).  No counterpart in the reference. */
int tt_probe_l2_reductions(void *buffer, size_t bytes, int64_t reductions, int32_t lanes_per_line,
                           uint64_t seed, void *stream);

/* ---- generic 3D interpolation (torch_image_interpolation) -------------
 * dtype codes: 0 float32, 1 float64, 2 complex64, 3 complex128.  Images are
 * (channels, d, h, w) of that dtype. */

/* Samples at n zyx coordinates (n, 3) of the image's real dtype into out
 * (n, channels): trilinear (grid_sample, padding 'border', align_corners) or
 * nearest (nearbyint); zero where any coordinate is outside [0, dim-1].
 * Replaces sample_image_3d, image_interpolation_3d.py:11-101. */
int tt_sample_image_3d(const void *image, int32_t dtype, int64_t channels, int64_t d, int64_t h,
                       int64_t w, const void *coordinates, int64_t n, void *out, int32_t nearest,
                       void *stream);

/* Backward of tt_sample_image_3d for upstream grad_out (n, channels):
 * grad_image (channels, d, h, w) ACCUMULATED into (nullable), grad_coordinates
 * (n, 3) overwritten (nullable), in PyTorch's complex-gradient convention;
 * coordinate gradients follow grid_sample's backward (zero on the border of
 * an axis and outside; none for nearest).  Replaces the autograd graph of
 * sample_image_3d (grid_sample backward). */
int tt_sample_image_3d_backward(const void *image, int32_t dtype, int64_t channels, int64_t d,
                                int64_t h, int64_t w, const void *coordinates, int64_t n,
                                const void *grad_out, void *grad_image, void *grad_coordinates,
                                int32_t nearest, void *stream);

/* Splats values (n, channels) at float32 coordinates (n, 3) into image and
 * weights (d, h, w; float32, or float64 when weights_f64), ACCUMULATED into:
 * trilinear (floor/ceil corners, float32 weights) or nearest (rint, weight 1);
 * points with any coordinate outside [0, dim-1] are dropped.
 * Replaces insert_into_image_3d, image_interpolation_3d.py:104-275. */
int tt_insert_into_image_3d(const void *values, int32_t dtype, const float *coordinates, int64_t n,
                            void *image, int64_t channels, int64_t d, int64_t h, int64_t w,
                            void *weights, int32_t weights_f64, int32_t nearest, void *stream);

/* Affine resampling: out (n_matrices, od, oh, ow, channels) of the image's
 * dtype = image sampled at M (z, y, x, 1) for every output voxel (z, y, x),
 * matrices_zyx (n_matrices, 4, 4) float32 already in zyx order; coordinates in
 * float32 with the reference's operation order, then trilinear / nearest as
 * tt_sample_image_3d.  Replaces affine_transform_image_3d
 * (torch_transform_image/transforms_3d.py:10-40: coordinate_grid, matmul,
 * sample_image_3d) without materialising the coordinate grid. */
int tt_affine_transform_image_3d(const void *image, int32_t dtype, int64_t channels, int64_t d,
                                 int64_t h, int64_t w, const float *matrices_zyx, int64_t n_matrices,
                                 int64_t od, int64_t oh, int64_t ow, int32_t nearest, void *out,
                                 void *stream);

/* Backward of tt_insert_into_image_3d w.r.t. the values: grad_values
 * (n, channels) of the image's dtype, overwritten, = the upstream image
 * gradient gathered with the insertion's own weights (zero for dropped points).
 * Replaces the index_put_ backward of insert_into_image_3d. */
int tt_insert_into_image_3d_backward(const void *grad_image, int32_t dtype, const float *coordinates,
                                     int64_t n, int64_t channels, int64_t d, int64_t h, int64_t w,
                                     int32_t nearest, void *grad_values, void *stream);

/* ---- elementwise passes around the FFTs of the real-space wrappers ------
 * is_f64 selects float64 (else float32) real data; complex128 likewise. */

/* out (n^3, n = d + 2*pad) = fftshift(pad(volume, pad) * sinc(|f|)^2), the FFT
 * input of project_3d_to_2d (project.py:48-69).  volume (d, d, d). */
int tt_project_prepare(const void *volume, int32_t is_f64, int64_t d, int64_t pad, void *out,
                       void *stream);

/* out (m, h-2*pad, w-2*pad) = crop(ifftshift(images, (-2, -1)), pad) for
 * images (m, h, w) (project.py:87-92; w = h-1 for odd padded sizes, because
 * the reference's irfftn runs without an output size). */
int tt_recentre_crop_2d(const void *images, int32_t is_f64, int64_t m, int64_t h, int64_t w,
                        int64_t pad, void *out, void *stream);

/* out (m, n, n) = fftshift(pad(images, pad), (-2, -1)), images (m, d, d),
 * n = d + 2*pad (backproject.py:48-59). */
int tt_pad_fftshift_2d(const void *images, int32_t is_f64, int64_t m, int64_t d, int64_t pad,
                       void *out, void *stream);

/* Friedel completion + division by max(weights, 1) + ifftshift along (d, h)
 * of `channels` insertion accumulators (tt_insert_accumulate, not finalized;
 * the weights are read from channel 0) into complex volumes out
 * (channels, d, h, w_rfft) (backproject.py:66-79). */
int tt_backproject_normalize(const void *accumulator, int32_t complex128, int64_t channels,
                             int64_t d, int64_t h, int64_t w_rfft, void *out, void *stream);

/* out (channels, n0-2*pad, n1-2*pad, n2-2*pad) = crop(ifftshift(volume) /
 * sinc(|f|)^2) of the irfft output volumes (channels, n0, n1, n2), the sinc
 * grid being that of the (n0, n1, n2) array (backproject.py:80-92). */
int tt_backproject_finish(const void *volume, int32_t is_f64, int64_t channels, int64_t n0,
                          int64_t n1, int64_t n2, int64_t pad, void *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* TEAMTOMO_B200_H */
