/*
 * rang_wgridder.h — C ABI of the B200 (sm_100a) w-gridder.
 *
 * Part 1 is the reference's C ABI for the exact gridder, symbol for symbol:
 * rang-core `core/src/ffi_wgridder.rs`. Every array is a HOST array owned by
 * the caller and borrowed for the call; the library copies it to the GPU,
 * runs the CUDA pipeline and copies the outputs back. Status codes are the
 * reference's: 0 success; 1 invalid arguments (the message is kept per thread
 * for rang_core_wgridder_last_error); 2 an internal failure (a CUDA error, no
 * device memory; the message is kept likewise). Outputs are zeroed by the
 * callee. `info` receives 14 doubles: kernel_index, supp, nu, nv, nplanes,
 * nvis, wmin_d, wmax_d, nm1min, nm1max, nshift, dw, wmin, ofactor
 * (core/src/wgridder.rs:469-511).
 *
 * Part 2 extends the ABI for callers whose data already lives on the GPU
 * (the PyTorch autograd wrapper, FISTA): a persistent plan on device
 * pointers, the reference's `Prepared` (core/src/wgridder.rs:3170-3499).
 */
#ifndef RANG_WGRIDDER_H
#define RANG_WGRIDDER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* core/src/ffi_wgridder.rs:22-42 (#[repr(C)] WgridderOptions), same layout. */
typedef struct WgridderOptions {
  size_t nx, ny;
  double pixsize_x, pixsize_y, epsilon, center_x, center_y, sigma_min, sigma_max;
  int32_t do_wgridding, divide_by_n, flip_u, flip_v, flip_w, allow_nshift;
  int64_t kernel_index; /* < 0: the cost model chooses */
  size_t nu, nv;
} WgridderOptions;

/* Kinds of the _ex entry points (ffi_wgridder.rs:297-310). */
#define WGRIDDER_VIS_UNIT 0
#define WGRIDDER_VIS_C64 1
#define WGRIDDER_VIS_C128 2
#define WGRIDDER_WGT_NONE 0
#define WGRIDDER_WGT_F32 1
#define WGRIDDER_WGT_F64 2
#define WGRIDDER_WGT_F32_PRODUCT 3

/* ---------------------------------------------------------------- part 1 */

/* ffi_wgridder.rs:155 — visibilities (nrow * nchan interleaved complex
 * doubles) to the dirty image (nx * ny doubles, first axis l); wgt and mask
 * may be null. */
int32_t rang_core_wgridder_vis2dirty_f64(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                         const double* uvw, const double* freq, const double* vis,
                                         const double* wgt, const uint8_t* mask, double* dirty,
                                         double* info);
/* ffi_wgridder.rs:191 — as above in single precision. */
int32_t rang_core_wgridder_vis2dirty_f32(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                         const double* uvw, const double* freq, const float* vis,
                                         const float* wgt, const uint8_t* mask, float* dirty,
                                         double* info);
/* ffi_wgridder.rs:228 — the image to visibilities (written). */
int32_t rang_core_wgridder_dirty2vis_f64(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                         const double* uvw, const double* freq, const double* dirty,
                                         const double* wgt, const uint8_t* mask, double* vis,
                                         double* info);
/* ffi_wgridder.rs:264 — as above in single precision. */
int32_t rang_core_wgridder_dirty2vis_f32(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                         const double* uvw, const double* freq, const float* dirty,
                                         const float* wgt, const uint8_t* mask, float* vis,
                                         double* info);
/* ffi_wgridder.rs:454 — data of kind vis_kind, weights of kind wgt_kind read
 * in place; dirty and/or psf (either may be null, not both). With a PSF both
 * images use the plan of wgt * mask != 0. */
int32_t rang_core_wgridder_vis2dirty_ex_f64(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                            const double* uvw, const double* freq, const void* vis,
                                            int32_t vis_kind, const void* wgt, int32_t wgt_kind,
                                            const uint8_t* mask, double* dirty, double* psf,
                                            double* info);
/* ffi_wgridder.rs:496 */
int32_t rang_core_wgridder_vis2dirty_ex_f32(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                            const double* uvw, const double* freq, const void* vis,
                                            int32_t vis_kind, const void* wgt, int32_t wgt_kind,
                                            const uint8_t* mask, float* dirty, float* psf,
                                            double* info);
/* ffi_wgridder.rs:542 — with WGRIDDER_WGT_F32_PRODUCT the weight is the
 * float product wgt[i] * wgt2[i]. */
int32_t rang_core_wgridder_vis2dirty_ex2_f64(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                             const double* uvw, const double* freq, const void* vis,
                                             int32_t vis_kind, const void* wgt, const void* wgt2,
                                             int32_t wgt_kind, const uint8_t* mask, double* dirty,
                                             double* psf, double* info);
/* ffi_wgridder.rs:573 */
int32_t rang_core_wgridder_vis2dirty_ex2_f32(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                             const double* uvw, const double* freq, const void* vis,
                                             int32_t vis_kind, const void* wgt, const void* wgt2,
                                             int32_t wgt_kind, const uint8_t* mask, float* dirty,
                                             float* psf, double* info);
/* ffi_wgridder.rs:668 */
int32_t rang_core_wgridder_dirty2vis_ex_f64(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                            const double* uvw, const double* freq, const double* dirty,
                                            const void* wgt, int32_t wgt_kind, const uint8_t* mask,
                                            double* vis, double* info);
/* ffi_wgridder.rs:695 */
int32_t rang_core_wgridder_dirty2vis_ex_f32(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                            const double* uvw, const double* freq, const float* dirty,
                                            const void* wgt, int32_t wgt_kind, const uint8_t* mask,
                                            float* vis, double* info);
/* ffi_wgridder.rs:722 — row `index` of the kernel table into out[7] (W,
 * ofactor, epsilon, beta, e0, ndim, singleprec); 1 past the end. */
int32_t rang_core_wgridder_kernel_row(size_t index, double* out);
/* ffi_wgridder.rs:749 — this thread's last failure message into buf (at most
 * len bytes, not terminated); returns its full length. */
size_t rang_core_wgridder_last_error(uint8_t* buf, size_t len);

/* ---------------------------------------------------------------- part 2 */

/* A persistent plan on DEVICE pointers (no counterpart symbol in the
 * reference; it is the reference's Prepared, wgridder.rs:3170-3222, whose
 * active set is wgt * mask != 0, or |vis|^2 wgt mask != 0 with with_vis).
 * `uvw_dev` (nrow * 3 doubles) is copied; `freq` is a HOST array; the
 * activity arrays are read during the call only. `single` selects float
 * working precision. `stream` is a cudaStream_t (null: the legacy stream).
 * The plan's buffers live on `stream`'s device; destroy the plan before the
 * stream. */
typedef struct RangWgridPlan RangWgridPlan;
int32_t rang_b200_wgridder_plan_create(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                       const double* uvw_dev, const double* freq, const void* vis_dev,
                                       int32_t vis_kind, const void* wgt_dev, const void* wgt2_dev,
                                       int32_t wgt_kind, const uint8_t* mask_dev, int32_t with_vis,
                                       int32_t single, void* stream, RangWgridPlan** plan,
                                       double* info);
/* vis2dirty with the plan into image_dev (nx * ny, the plan's precision):
 * weights as in the _ex2 entry points. `flags`: bit 0 (1) grids unit
 * visibilities (the PSF) instead of vis_dev; bit 1 (2) tells that vis_dev,
 * wgt_dev and wgt2_dev are the arrays the plan was created with, unchanged
 * since, so the plan's scan already holds their largest value and the pass
 * over the data that finds it is skipped (a plan checks the pointers; the
 * caller vouches for the contents). Asynchronous on `stream`. */
int32_t rang_b200_wgridder_plan_grid(RangWgridPlan* plan, const void* vis_dev, int32_t vis_kind,
                                     const void* wgt_dev, const void* wgt2_dev, int32_t wgt_kind,
                                     int32_t flags, void* image_dev, void* stream);
/* dirty2vis with the plan: image_dev (nx * ny) to vis_dev (nrow * nchan
 * interleaved complex, overwritten; inactive visibilities zero), times the
 * weights. Asynchronous on `stream`. */
int32_t rang_b200_wgridder_plan_degrid(RangWgridPlan* plan, const void* image_dev, const void* wgt_dev,
                                       int32_t wgt_kind, void* vis_dev, void* stream);
/* Waits for `stream` and reports a failure the kernels detected (status 2)
 * or 0. */
int32_t rang_b200_wgridder_plan_status(RangWgridPlan* plan, void* stream);
/* The plan's 14 info doubles. */
int32_t rang_b200_wgridder_plan_info(const RangWgridPlan* plan, double* info);
void rang_b200_wgridder_plan_destroy(RangWgridPlan* plan);

/* Prepared::residual / residual_sorted (wgridder.rs:3232-3278): the residual
 * image of `data_dev` against the image `model_dev` (nx * ny in the plan's
 * precision; null: the data alone) into image_dev, gridded with the weights
 * (kinds as for plan_grid), and sum w |d - A model|^2 into *misfit_dev (one
 * double on the device; null: not formed). The prediction is degridded
 * without weights. sorted = 0: data and weights are nrow * nchan; 1: they
 * hold the plan's active visibilities in its sorted order
 * (rang_b200_wgridder_plan_sorted). The values live in the plan's stored
 * work space (sorted order), so no visibility-sized buffer is allocated per
 * call, and nothing waits for the device: the call is asynchronous on
 * `stream`. Passes of one plan must run in stream order (they share that
 * work space). */
int32_t rang_b200_wgridder_plan_residual(RangWgridPlan* plan, const void* data_dev, int32_t vis_kind,
                                         const void* wgt_dev, const void* wgt2_dev, int32_t wgt_kind,
                                         const void* model_dev, int32_t sorted, void* image_dev, double* misfit_dev,
                                         void* stream);
/* The Gram operator A^H W A of the plan (the reference's gram_apply,
 * clean_certified.rs:233-236) on x_dev (nx * ny) into image_dev, W the
 * weights (sorted as for plan_residual), and x^T A^H W A x = sum w |A x|^2
 * into *xgx_dev (null: not formed). Asynchronous on `stream`. */
int32_t rang_b200_wgridder_plan_gram(RangWgridPlan* plan, const void* x_dev, const void* wgt_dev,
                                     const void* wgt2_dev, int32_t wgt_kind, int32_t sorted, void* image_dev,
                                     double* xgx_dev, void* stream);
/* Prepared::sorted (wgridder.rs:3287-3302): dense_dev (nrow * nchan elements
 * of elem_bytes = 1, 4, 8 or 16) at the active visibilities, in the plan's
 * sorted order, into out_dev (plan_active elements). */
int32_t rang_b200_wgridder_plan_sorted(const RangWgridPlan* plan, const void* dense_dev, int32_t elem_bytes,
                                       void* out_dev, void* stream);
/* Prepared::active: the number of active visibilities. */
int32_t rang_b200_wgridder_plan_active(const RangWgridPlan* plan, size_t* active);
/* Prepared::memory (wgridder.rs:3397-3430): device bytes held per buffer
 * into bytes[0, n); returns the number of buffers (names from
 * plan_memory_name), or -1 for a null plan. */
int32_t rang_b200_wgridder_plan_memory(const RangWgridPlan* plan, size_t* bytes, int32_t n);
const char* rang_b200_wgridder_plan_memory_name(int32_t index);
/* Prepared::release_grids (wgridder.rs:3432-3440): frees the stored values
 * that residual and Gram passes keep; the next pass allocates them again. */
void rang_b200_wgridder_plan_release_work(RangWgridPlan* plan);
/* No counterpart in the reference (whose buffers are host memory freed at
 * the end of each call). The library keeps released device buffers of 64 MB
 * or more for the next request of the same size, so that repeated calls of
 * one shape allocate nothing; the device memory they hold (and what the
 * stream-ordered pool keeps) is not available to other allocators in the
 * process, such as PyTorch's. rang_b200_wgridder_cached_bytes reports the
 * bytes held on the current device; rang_b200_wgridder_release_cached
 * returns them, and the pool's unused memory, to the device (status 0, 2 on
 * a CUDA error), after the work already queued that uses them. */
size_t rang_b200_wgridder_cached_bytes(void);
int32_t rang_b200_wgridder_release_cached(void);
/* `plan` and `gridding_footprint` (wgridder.rs:3527-3588) on HOST arrays:
 * the kernel and grid a call would choose (info, 14 doubles; the activity as
 * for rang_b200_wgridder_binning, with_vis when vis_kind is not 0), without
 * binning or gridding, and in *footprint (may be null) the device bytes of
 * a gridding pass's work space for `nout` images. */
int32_t rang_b200_wgridder_plan_only(const WgridderOptions* opts, size_t nrow, size_t nchan, const double* uvw,
                                     const double* freq, const void* vis, int32_t vis_kind, const void* wgt,
                                     const void* wgt2, int32_t wgt_kind, const uint8_t* mask, int32_t single,
                                     int32_t nout, double* info, size_t* footprint);

/* The visibility binning of a call on HOST arrays, for parity tests: per
 * visibility (row-major) iu0, iv0 (-1 when inactive) and the bin key
 * tile * max(nplanes, 1) + first plane (0xffffffff when inactive), and the
 * active visibilities in the reference's layout order, (tile, first plane,
 * row, channel) (`sorted`, nrow * nchan entries of room; `nsorted` receives
 * the active count). Arguments as rang_core_wgridder_vis2dirty_ex2_*;
 * with_vis selects the activity |vis|^2 wgt mask != 0. */
int32_t rang_b200_wgridder_binning(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                   const double* uvw, const double* freq, const void* vis,
                                   int32_t vis_kind, const void* wgt, const void* wgt2, int32_t wgt_kind,
                                   const uint8_t* mask, int32_t with_vis, int32_t single, int64_t* iu0,
                                   int64_t* iv0, uint32_t* key, uint32_t* sorted, size_t* nsorted,
                                   double* info);

/* The visibility binning of rang_b200_wgridder_plan_create (scan, kernel and
 * grid choice, counting sort by uv tile and first w-plane) without any
 * device allocation. It has no counterpart in the reference. It is for
 * callers that cannot call cudaMalloc: an application whose device memory is
 * all handed out by its own allocator under a fixed budget, or a path that
 * must not take the CUDA allocator's locks or wait on it. Every temporary
 * lives in one 16 MiB array that the library holds on each GPU that loads it
 * (NOALLOC_SCRATCH_BYTES); a call whose bin counters and scan do not fit in
 * it fails with status 1 and says how many bytes it needed. The first call on
 * a device looks up that array's device address (cudaGetSymbolAddress).
 * Every call reads the scan's count back to the host and waits for `stream`
 * before it returns, so no call can be made inside a stream capture. All calls
 * share the array, so calls whose GPU work overlaps race: run them on one
 * stream, or wait for one before starting another. The call clears what must
 * start at zero.
 * Inputs: uvw_dev (nrow * 3 doubles) and the optional weights wgt_dev
 * (WGRIDDER_WGT_NONE, _F32 or _F64) and mask_dev (nrow * nchan) are device
 * arrays; freq is a host array; the active set is wgt * mask != 0 (as for
 * degridding). Outputs, device arrays of nrow * nchan entries: key_dev, per
 * visibility (row-major) tile * max(nplanes, 1) + first plane, 0xffffffff
 * when inactive; sorted_dev, the active visibilities' linear indices in
 * (tile, first plane) order, *nsorted of them; info, the plan's 14
 * doubles. */
int32_t rang_b200_wgridder_bin_noalloc(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                       const double* uvw_dev, const double* freq, const void* wgt_dev,
                                       int32_t wgt_kind, const uint8_t* mask_dev, int32_t single, void* stream,
                                       uint32_t* key_dev, uint32_t* sorted_dev, size_t* nsorted, double* info);

/* Instrumentation (no counterpart in the reference, whose timing report is
 * RANG_WGRIDDER_TIMING on stderr, wgridder.rs:1773-1812). The launch count
 * is the number of this library's own CUDA kernels launched so far (cuFFT's
 * are not counted). While profiling is on, every stage of the pipeline is
 * bracketed by CUDA events on its stream; profile_read waits for them and
 * returns per stage the launches and the summed device milliseconds since the
 * previous read, in the order of stage_name(0 .. n-1). */
int64_t rang_b200_wgridder_launch_count(void);
/* How single-precision gridding forms its sums (no counterpart in the
 * reference, whose RANG_WGRIDDER_SIMD selects CPU instruction sets,
 * wgridder.rs:1593-1627): 3 (the default) exact integer products of 23-bit
 * fixed-point factors on the integer tensor cores, summed in an int64
 * fixed-point grid, so that results are bit-identical from call to call and
 * do not depend on the visibilities' order; 1 split-precision 3 x TF32 and
 * 2 split-precision 3 x BF16 tensor-core products with FP32 accumulation
 * (their results depend on the order of the sorted visibilities, which the
 * binning leaves free); 0 plain FP32 CUDA-core products, each rounded into
 * the fixed-point grid (order-independent). Process-wide;
 * RANG_WGRIDDER_GPU_METHOD=int8|fp32|tf32x3|bf16x3 sets the initial value.
 * Other values select 3. Returns the previous method. */
int32_t rang_b200_wgridder_set_method(int32_t method);
void rang_b200_wgridder_profile(int32_t on);
int32_t rang_b200_wgridder_profile_read(int64_t* launches, double* ms, int32_t n);
const char* rang_b200_wgridder_stage_name(int32_t index);

#ifdef __cplusplus
}
#endif

#endif /* RANG_WGRIDDER_H */
