// The device-resident plan of a gridder call: scan, kernel choice, the
// visibility binning by (uv tile, first w-plane), and the task list of the
// gridding and degridding kernels. A plan is built once per set of
// coordinates, weights and mask and can then grid and degrid any number of
// times (the reference's `Prepared`, core/src/wgridder.rs:3170-3499).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <utility>
#include <vector>

#include "wgrid_common.h"
#include "wgrid_device.cuh"
#include "wgrid_setup.h"

namespace wg {

// A gridding task: visibilities [k0, k1) of the sorted order, all in one uv
// tile, with first planes in [plo, phi].
struct Task {
  uint32_t tile, k0, k1;
  uint16_t plo, phi;
};

// Failures inside a library call that are not the caller's arguments
// (CUDA errors, device memory) map to status 2.
struct DeviceError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void check_cuda(cudaError_t e, const char* what);

constexpr size_t CACHED_MIN = (size_t)64 << 20;
// Bytes of cached buffers free for reuse on device `dev`.
size_t cached_free_bytes(int dev);
// Returns the cached buffers of device `dev` to the pool.
void flush_cache(int dev);

// Device memory taken from the stream-ordered pool and returned on release.
// Buffers of CACHED_MIN bytes or more are kept on release in a cache by
// exact size and handed to the next request of that size on the device,
// after the releasing stream's work (an event the new stream waits on):
// repeated calls of one shape then take no allocation. The pool's own reuse
// of such sizes measured 2 to 200 ms per call on B200 (the host waits in
// cudaMallocAsync). A failed allocation empties the cache and retries.
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(size_t bytes, cudaStream_t s) { alloc(bytes, s); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_), s_(o.s_) { o.p_ = nullptr; }
  DevBuf& operator=(DevBuf&& o) noexcept;
  ~DevBuf() { release(); }
  void alloc(size_t bytes, cudaStream_t s);
  void release();
  template <class U>
  U* as() const { return reinterpret_cast<U*>(p_); }
  void* get() const { return p_; }
  size_t size() const { return n_; }

 private:
  void* p_ = nullptr;
  size_t n_ = 0;
  cudaStream_t s_ = nullptr;
};

// How a gridding pass forms each visibility's value.
enum ValueMode : int { VALUE_DATA = 0, VALUE_UNIT = 1 };

template <class T>
class Plan {
 public:
  // Scan the active set (`with_vis`: |vis|^2 wgt mask != 0, else wgt mask
  // != 0), choose kernel and grid, and bin the active visibilities. `uvw`
  // and the arrays of `act` are device pointers; `freq` is on the host.
  // With `row_chunks` > 1 the rows are split into that many equal ranges and
  // the sorted order is chunk-major (each range's visibilities contiguous,
  // binned among themselves), so that gridding can start on the rows that
  // have arrived and degridding can hand out finished rows early.
  // `layout` LAYOUT_NONE stops after the kernel and grid choice (the
  // reference's `plan` and `gridding_footprint`): such a plan reports `info`
  // and `footprint` but cannot grid. LAYOUT_STREAMED defers the binning to
  // degrid_streamed, which bins each row chunk just before degridding it.
  enum Layout : int { LAYOUT_NONE = 0, LAYOUT_FULL = 1, LAYOUT_STREAMED = 2 };
  Plan(const WgridderOptions& o, size_t nrow, size_t nchan, const double* uvw_dev, const double* freq_host,
       const Inputs& act, bool with_vis, cudaStream_t s, int row_chunks = 1, int layout = LAYOUT_FULL);

  // dirty2vis of a LAYOUT_STREAMED plan, its only pass: the image's planes
  // are transformed, then row chunk c is binned (count, offsets after the
  // earlier chunks' on the device, placement) and degridded before chunk
  // c + 1 is binned, so done[c] is recorded long before the whole binning
  // would end. The results equal degrid's bit for bit. Plans the streamed
  // form does not serve (double precision, supports above 8, one chunk,
  // plane groups) are binned whole and degridded as by degrid.
  void degrid_streamed(const T* image, const Inputs& wts, T* vis, cudaStream_t s, cudaEvent_t* done);

  bool empty() const { return nvis_ == 0; }
  const PlanInfo& info() const { return info_; }
  size_t nvis() const { return nvis_; }
  const Geom<T>& geom() const { return g_; }

  // vis2dirty into `image` (nx * ny, device): `data` gives the data and the
  // weights; VALUE_UNIT grids unit visibilities (the PSF). With `ready`
  // (one event per row chunk), gridding waits for every ready[c]: the grid's
  // fixed-point scale needs the largest value of all the data. `scanned`:
  // `data` is the input this plan scanned (the same arrays, unchanged since),
  // whose value bound the scan already took; otherwise one pass over `data`
  // takes it.
  // `bound`, when given, is the device value bound (fast::ValueBound) of
  // `data`, formed by the caller's kernels.
  void grid(const Inputs& data, ValueMode mode, T* image, cudaStream_t s, const cudaEvent_t* ready = nullptr,
            bool scanned = false, const void* bound = nullptr);
  // dirty2vis of `image` into `vis` (nrow * nchan interleaved complex,
  // device, overwritten; inactive visibilities zero), times the weights of
  // `wts`. With `done` (one event per row chunk), done[c] is recorded once
  // the rows of chunk c are final.
  void degrid(const T* image, const Inputs& wts, T* vis, cudaStream_t s, cudaEvent_t* done = nullptr);

  // The residual image of `data` against the image `model` (null: the data
  // alone), gridded with the weights of `data`, and the weighted misfit
  // sum w |d - A model|^2 into `misfit` (one device double; null: not
  // formed): the reference's Prepared::residual and residual_sorted
  // (wgridder.rs:3232-3395). The prediction is degridded without weights.
  // With `sorted_data`, the data and weights hold the active visibilities in
  // the plan's sorted order (`gather_sorted`) instead of nrow * nchan.
  // Asynchronous on `s`: nothing waits for the device.
  void residual(const Inputs& data, bool sorted_data, const T* model, T* image, double* misfit, cudaStream_t s);
  // A^H W A x into `image`, with W the weights of `wts` (sorted as for
  // `residual`), and x^T A^H W A x = sum w |A x|^2 into `xgx` (null: not
  // formed): the prediction, weighted, is gridded from the stored values.
  void gram(const T* x, const Inputs& wts, bool sorted_wts, T* image, double* xgx, cudaStream_t s);
  // `dense` (nrow * nchan elements of `elem_bytes`: 1, 4, 8 or 16) at the
  // active visibilities in the sorted order (the reference's Prepared::sorted).
  void gather_sorted(const void* dense, int elem_bytes, void* out, cudaStream_t s) const;
  // Device bytes held, by buffer (the reference's Prepared::memory), in the
  // order of memory_names().
  std::vector<std::pair<const char*, size_t>> memory() const;
  static std::vector<const char*> memory_names();
  // Frees the values the residual and Gram passes keep between calls; the
  // next pass allocates them again.
  void release_work();
  // Device bytes of a gridding pass's work space for `nout` images (the
  // reference's gridding_footprint): the fixed-point and transform planes of
  // one plane group, and the image accumulator.
  size_t footprint(int nout) const;

  // Rows per chunk when `nrow` rows are asked to be split `row_chunks` ways.
  static size_t chunk_rows(size_t nrow, int row_chunks) {
    const size_t k = std::max<size_t>(1, std::min<size_t>((size_t)std::max(row_chunks, 1), std::max<size_t>(nrow, 1)));
    return std::max<size_t>(1, (nrow + k - 1) / k);
  }
  // Row chunks of the sorted order: chunk c holds rows [row_begin(c), row_begin(c + 1)).
  int chunks() const { return nchunk_; }
  size_t row_begin(int c) const { return std::min(nrow_, (size_t)c * rows_per_chunk_); }
  // Scans another active set and tells whether its count and |w| range equal
  // this plan's (then the kernel, grid and planes would be the same).
  bool same_scan(const Inputs& act, bool with_vis, cudaStream_t s) const;

  // Waits for `s` and returns the inconsistencies the kernels flagged (0: none).
  int kernel_errors(cudaStream_t s) const;

  // For the tests: per visibility (row-major) the reference's bin key
  // tile * nbuckets + first plane (0xffffffff inactive), and the sorted order.
  void export_binning(uint32_t* key_host, uint32_t* sorted_host, cudaStream_t s) const;
  // Per visibility iu0, iv0 (int64) from the device arithmetic, for the tests.
  void export_pixels(const Inputs& act, bool with_vis, int64_t* iu0_host, int64_t* iv0_host, cudaStream_t s) const;

 private:
  void build_layout(const Inputs& act, bool with_vis, const uint32_t* bits, cudaStream_t s);
  // Per row the binning's coordinates and sign (double4, nrow_ of them).
  void row_coords(DevBuf& out, cudaStream_t s) const;
  // Degridding into `vis` (by visibility index), or, with `fused` (a
  // fast::DegridOut), into the stored values by sorted position.
  void degrid_to(const T* image, const Inputs& wts, T* vis, const void* fused, cudaStream_t s, cudaEvent_t* done);
  // The residual (gram false) or Gram (true) values, gridded into `image`.
  void values_pass(bool gram, const Inputs& data, bool sorted_data, const T* model, T* image, double* sum,
                   cudaStream_t s);
  // The single-precision tensor-core kernels serve the pass (the degridder
  // writes the stored values in sorted order, the integer gridder reads them).
  bool fused_values() const;
  // Bytes of one gridding plane group and of the fixed part, and the group.
  void grid_sizes(size_t& plane_bytes, size_t& fixed, size_t& group) const;
  void corrections(cudaStream_t s);
  int touched_rows(double umax, double wmax) const;
  size_t plane_group(size_t plane_bytes, size_t fixed) const;

  WgridderOptions o_;
  size_t nrow_, nchan_, n_;
  size_t nvis_ = 0;
  double r_l_ = 0, r_m_ = 0;
  Geom<T> g_;
  PlanInfo info_{};
  EsKernel* kernel_ = nullptr;
  DevBuf uvw_, foc_;
  DevBuf key_;      // u32 per visibility: bin or 0xffffffff
  DevBuf starts_;   // u32 per bin + 1: exclusive offsets
  DevBuf sorted_;   // u32 per active visibility: linear index
  DevBuf rec_;      // single precision: a 32-byte record per active visibility, in sorted order
  DevBuf bound_;    // the scan's largest |vis| |wgt| and |wgt|
  DevBuf scale_;    // the fixed-point scales of the current gridding pass
  DevBuf tasks_;    // Task, at most max_tasks_
  DevBuf ntasks_;   // u32: tasks in use
  DevBuf corr_;     // double per pixel: the global correction
  DevBuf err_;      // int: kernel-detected inconsistencies
  DevBuf stored_;   // residual / Gram values by sorted position (single precision, tensor-core path)
  DevBuf work_;     // residual / Gram values by visibility index (the other paths)
  DevBuf partials_; // FP64 per-block partial sums of the misfit
  DevBuf res_bound_;  // the largest |value| of a residual or Gram pass
  size_t nbins_ = 0, ntiles_ = 0, max_tasks_ = 0;
  int nchunk_ = 1;
  size_t rows_per_chunk_ = 0;
  std::vector<uint64_t> chunk_sorted_;  // nchunk_ + 1 offsets into the sorted order
  std::vector<uint32_t> chunk_tasks_;   // nchunk_ + 1 offsets into the task list
  unsigned long long scan_[4] = {0, 0, 0, 0};  // count, finite count, |w| min and max bits
  bool foc_finite_ = true;  // every channel's f / c finite
  bool streamed_ = false;   // LAYOUT_STREAMED, not yet binned
  DevBuf bits_;             // LAYOUT_STREAMED: the scan's active set, one bit per visibility
  // The arrays of the scan whose value maxima bound_ holds (with the
  // visibilities when scan_vis_), to tell whether a gridding pass's data
  // need their own bound.
  mutable Inputs scan_in_{};
  mutable bool scan_vis_ = false;
  bool bound_of(const Inputs& data, ValueMode mode) const;
  // Grid rows (u) that footprints can touch: storage rows [0, urows_) and
  // [nu - urows_, nu); 0 means all rows (the v transforms run on these only).
  int urows_ = 0;
};

// How single-precision gridding forms its sums: exact integer products of
// 23-bit fixed-point factors on the integer tensor cores (default; results
// independent of the visibilities' order), split-precision 3 x TF32 or
// 3 x BF16 tensor-core products, or plain FP32 CUDA-core products (each term
// rounded into the fixed-point grid, also order-independent). The float
// tensor-core methods sum blocks of visibilities inside the tensor core, so
// their results depend on the sorted order, which the counting sort's
// atomics leave free. Double precision always uses FP64 CUDA-core products
// rounded into the fixed-point grid. The environment variable
// RANG_WGRIDDER_GPU_METHOD (int8 | fp32 | tf32x3 | bf16x3) sets the default.
enum GridMethod : int { GRID_FP32 = 0, GRID_TF32X3 = 1, GRID_BF16X3 = 2, GRID_INT8 = 3 };
int grid_method();
void set_grid_method(int method);

// The largest shared-memory tile window (planes) per CTA.
int max_window_planes(int L, size_t cell_bytes);

// Stages of the pipeline, for the launch counter and the event profiler.
enum Stage : int {
  ST_SCAN = 0, ST_BIN_COUNT, ST_PREFIX, ST_BIN_SCATTER, ST_TASKS, ST_CORR, ST_GRID, ST_FFT, ST_PROJECT,
  ST_CORRECT_INPUT, ST_PLACE, ST_DEGRID, ST_FIXED, ST_OTHER, N_STAGES
};
extern const char* const STAGE_NAMES[N_STAGES];

// Brackets the launches of one stage on `s`: counts them and, while the
// profiler is on, records a CUDA event pair around them.
class StageTimer {
 public:
  StageTimer(Stage st, cudaStream_t s, int launches = 1);
  ~StageTimer();

 private:
  Stage st_;
  cudaStream_t s_;
  cudaEvent_t a_ = nullptr, b_ = nullptr;
};

void profile_enable(bool on);
// This thread's last-error message of the C ABI.
std::string* last_error_slot();
// Totals per stage since the last read (waits for the recorded events).
void profile_read(long long* launches, double* ms);
long long launch_count();

}  // namespace wg
