// The C ABI of include/rang_wgridder.h.
//
// Part 1 restates the reference's `core/src/ffi_wgridder.rs` entry points
// (argument checks, messages, status codes) on top of the CUDA pipeline: the
// host arrays are copied to the device on a per-thread stream, planned,
// gridded or degridded there, and the outputs copied back. Part 2 exposes the
// device-resident plan.
#include <cstring>
#include <functional>
#include <map>
#include <algorithm>
#include <vector>
#include <cstdlib>
#include <memory>
#include <mutex>
#include <string>

#include "rang_weights.h"
#include "wgrid_plan.h"

// The imaging-weight pipeline (wgrid_weights.cu).
namespace wg {
void weight_grid_shape(size_t width, size_t height, double super_weight, size_t* w, size_t* h);
size_t padded_size(size_t trimmed, double padding);
void stokes_i(const StokesIInputs& in, StokesIOutputs& out, cudaStream_t s);
void imaging_weights(const ImagingWeightInputs& in, ImagingWeightOutputs& out, cudaStream_t s);
int32_t status_guarded(const std::function<void()>& f);
cudaStream_t stream_of(void* stream);
}  // namespace wg

using namespace wg;

namespace {

thread_local std::string g_last_error;

template <class F>
int32_t guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const InvalidArgument& e) {
    g_last_error = e.what();
    return 1;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return 2;
  } catch (...) {
    g_last_error = "internal failure in the gridder";
    return 2;
  }
}

// Keeps freed device memory in the stream-ordered pool (set once per device),
// so a call does not pay for cudaMalloc of the previous call's buffers again.
void configure_pool(int dev) {
  static std::mutex mu;
  static std::map<int, bool> done;
  std::lock_guard<std::mutex> lock(mu);
  if (done[dev]) return;
  cudaMemPool_t pool;
  check_cuda(cudaDeviceGetDefaultMemPool(&pool, dev), "memory pool");
  uint64_t keep = UINT64_MAX;
  check_cuda(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "memory pool");
  done[dev] = true;
}

// The library's own stream for host-array calls: one per thread and device.
cudaStream_t call_stream() {
  static thread_local std::map<int, cudaStream_t> streams;
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "no CUDA device");
  auto it = streams.find(dev);
  if (it != streams.end()) return it->second;
  configure_pool(dev);
  cudaStream_t s;
  check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
  streams[dev] = s;
  return s;
}

// A second per-thread stream for the host <-> device copies of the pipelined calls.
cudaStream_t copy_stream() {
  static thread_local std::map<int, cudaStream_t> streams;
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "no CUDA device");
  auto it = streams.find(dev);
  if (it != streams.end()) return it->second;
  cudaStream_t s;
  check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
  streams[dev] = s;
  return s;
}

// Row chunks of a host call whose visibilities take `bytes`: the copies of
// one chunk overlap the gridding or degridding of another. Small calls are
// not split. RANG_WGRIDDER_ROW_CHUNKS overrides (1: no pipelining).
int host_row_chunks(size_t bytes) {
  const char* e = std::getenv("RANG_WGRIDDER_ROW_CHUNKS");
  const int env = e ? std::atoi(e) : 0;
  if (env > 0) return std::min(env, 64);
  return bytes >= ((size_t)256 << 20) ? 8 : 1;
}

// Events without timing, destroyed with the holder.
struct Events {
  std::vector<cudaEvent_t> e;
  explicit Events(int n) : e((size_t)n, nullptr) {
    for (auto& x : e) check_cuda(cudaEventCreateWithFlags(&x, cudaEventDisableTiming), "event");
  }
  ~Events() {
    for (auto x : e)
      if (x) cudaEventDestroy(x);
  }
  Events(const Events&) = delete;
  Events& operator=(const Events&) = delete;
};

size_t vis_bytes(int kind, const void* p) {  // ffi_wgridder.rs:319-336
  switch (kind) {
    case VIS_UNIT:
      return 0;
    case VIS_C64:
      if (p) return 8;
      break;
    case VIS_C128:
      if (p) return 16;
      break;
  }
  throw InvalidArgument("invalid visibility array or kind");
}

size_t wgt_bytes(int kind, const void* p, const void* p2) {  // ffi_wgridder.rs:344-371
  switch (kind) {
    case WGT_NONE:
      return 0;
    case WGT_F32:
      if (p) return 4;
      break;
    case WGT_F64:
      if (p) return 8;
      break;
    case WGT_F32_PRODUCT:
      if (p && p2) return 4;
      break;
  }
  throw InvalidArgument("invalid weight array or kind");
}

DevBuf upload(const void* host, size_t bytes, cudaStream_t s) {
  DevBuf b;
  if (host && bytes) {
    b.alloc(bytes, s);
    check_cuda(cudaMemcpyAsync(b.get(), host, bytes, cudaMemcpyHostToDevice, s), "copy to device");
  }
  return b;
}

struct Uploaded {
  DevBuf uvw, vis, wgt, wgt2, mask;
  Inputs in;
};

Uploaded upload_inputs(size_t nrow, size_t nchan, const double* uvw, const void* vis, int vis_kind,
                       const void* wgt, const void* wgt2, int wgt_kind, const uint8_t* mask, cudaStream_t s) {
  size_t n = nrow * nchan;
  size_t vb = vis_bytes(vis_kind, vis), wb = wgt_bytes(wgt_kind, wgt, wgt2);
  Uploaded u;
  u.uvw = upload(uvw, nrow * 3 * sizeof(double), s);
  u.vis = upload(vis_kind == VIS_UNIT ? nullptr : vis, n * vb, s);
  u.wgt = upload(wgt_kind == WGT_NONE ? nullptr : wgt, n * wb, s);
  u.wgt2 = upload(wgt_kind == WGT_F32_PRODUCT ? wgt2 : nullptr, n * 4, s);
  u.mask = upload(mask, n, s);
  u.in.vis = u.vis.get();
  u.in.vis_kind = vis_kind;
  u.in.wgt = u.wgt.get();
  u.in.wgt2 = u.wgt2.get();
  u.in.wgt_kind = wgt_kind;
  u.in.mask = u.mask.as<uint8_t>();
  return u;
}

template <class T>
void finish(Plan<T>& plan, cudaStream_t s) {
  check_cuda(cudaStreamSynchronize(s), "gridder");
  if (plan.kernel_errors(s)) throw DeviceError("a visibility fell outside its uv tile (internal inconsistency)");
}

// vis2dirty of host data with the visibility copy overlapped: coordinates,
// weights and mask go first and are planned on with the active set they
// give (weight * mask != 0) while the visibilities follow in row chunks on a
// second stream; each chunk is gridded as soon as it is on the device. The
// reference's active set also drops visibilities that are exactly zero, so
// the plan stands only if a scan of the full active set finds the same count
// and |w| range (then kernel, grid and planes are the same, and the extra
// visibilities, all zero, add nothing); otherwise the call is planned and
// gridded again on the full active set.
template <class T>
void host_vis2dirty_pipelined(const WgridderOptions* o, size_t nrow, size_t nchan, const double* uvw,
                              const double* freq, const void* vis, int vis_kind, const void* wgt, const void* wgt2,
                              int wgt_kind, const uint8_t* mask, T* dirty, double* info, int chunks) {
  const size_t npix = o->nx * o->ny, vb = vis_bytes(vis_kind, vis), rowb = nchan * vb;
  cudaStream_t s = call_stream(), sc = copy_stream();
  Uploaded u = upload_inputs(nrow, nchan, uvw, nullptr, VIS_UNIT, wgt, wgt2, wgt_kind, mask, s);
  // The plan's row chunks: rows [c * rpc, (c + 1) * rpc).
  const size_t rpc = Plan<T>::chunk_rows(nrow, chunks);
  const int nchunk = (int)((std::max<size_t>(nrow, 1) + rpc - 1) / rpc);
  Events ready(nchunk);
  DevBuf visd(nrow * rowb, sc);
  for (int c = 0; c < nchunk; c++) {
    const size_t r0 = (size_t)c * rpc, r1 = std::min(nrow, r0 + rpc);
    check_cuda(cudaMemcpyAsync(visd.as<unsigned char>() + r0 * rowb, static_cast<const unsigned char*>(vis) + r0 * rowb,
                               (r1 - r0) * rowb, cudaMemcpyHostToDevice, sc),
               "copy to device");
    check_cuda(cudaEventRecord(ready.e[c], sc), "record");
  }
  Plan<T> plan(*o, nrow, nchan, u.uvw.as<double>(), freq, u.in, false, s, chunks);
  std::memset(dirty, 0, npix * sizeof(T));
  Inputs data = u.in;
  data.vis = visd.get();
  data.vis_kind = vis_kind;
  if (plan.empty()) {  // nothing passes the weights and mask: nothing is active
    check_cuda(cudaStreamSynchronize(sc), "copy");
    std::memcpy(info, plan.info().v, sizeof(plan.info().v));
    return;
  }
  DevBuf img(npix * sizeof(T), s);
  if (plan.chunks() == nchunk) {
    plan.grid(data, VALUE_DATA, img.as<T>(), s, ready.e.data());
  } else {  // the plan kept one chunk (too many bins): wait for all rows
    check_cuda(cudaStreamWaitEvent(s, ready.e[nchunk - 1], 0), "wait");
    plan.grid(data, VALUE_DATA, img.as<T>(), s);
  }
  if (plan.same_scan(data, true, s)) {
    std::memcpy(info, plan.info().v, sizeof(plan.info().v));
    check_cuda(cudaMemcpyAsync(dirty, img.get(), npix * sizeof(T), cudaMemcpyDeviceToHost, s), "copy to host");
    finish(plan, s);
    return;
  }
  Plan<T> exact(*o, nrow, nchan, u.uvw.as<double>(), freq, data, true, s);
  std::memcpy(info, exact.info().v, sizeof(exact.info().v));
  if (exact.empty()) return;
  exact.grid(data, VALUE_DATA, img.as<T>(), s, nullptr, true);
  check_cuda(cudaMemcpyAsync(dirty, img.get(), npix * sizeof(T), cudaMemcpyDeviceToHost, s), "copy to host");
  finish(exact, s);
}

// vis2dirty_multi (wgridder.rs:2436-2496) on host arrays.
template <class T>
void host_vis2dirty(const WgridderOptions* o, size_t nrow, size_t nchan, const double* uvw, const double* freq,
                    const void* vis, int vis_kind, const void* wgt, const void* wgt2, int wgt_kind,
                    const uint8_t* mask, T* dirty, T* psf, double* info) {
  if (!o) throw InvalidArgument("null options");
  if (!uvw || !freq || !info || (!dirty && !psf)) throw InvalidArgument("null array");
  vis_bytes(vis_kind, vis);
  wgt_bytes(wgt_kind, wgt, wgt2);
  check_common(*o, nrow, nchan);
  f_over_c(freq, nchan);  // the frequency checks, before any device work
  size_t npix = o->nx * o->ny;
  cudaStream_t s = call_stream();
  const size_t vb = vis_bytes(vis_kind, vis);
  const int chunks = host_row_chunks(nrow * nchan * vb);
  if (dirty && !psf && vb && chunks > 1) {
    host_vis2dirty_pipelined<T>(o, nrow, nchan, uvw, freq, vis, vis_kind, wgt, wgt2, wgt_kind, mask, dirty, info,
                                chunks);
    return;
  }
  Uploaded u = upload_inputs(nrow, nchan, uvw, vis, vis_kind, wgt, wgt2, wgt_kind, mask, s);
  Plan<T> plan(*o, nrow, nchan, u.uvw.as<double>(), freq, u.in, psf == nullptr, s);
  if (dirty) std::memset(dirty, 0, npix * sizeof(T));
  if (psf) std::memset(psf, 0, npix * sizeof(T));
  std::memcpy(info, plan.info().v, sizeof(plan.info().v));
  if (plan.empty()) return;
  DevBuf img(npix * sizeof(T), s);
  if (dirty) {
    plan.grid(u.in, VALUE_DATA, img.as<T>(), s, nullptr, true);
    check_cuda(cudaMemcpyAsync(dirty, img.get(), npix * sizeof(T), cudaMemcpyDeviceToHost, s), "copy to host");
  }
  if (psf) {
    plan.grid(u.in, VALUE_UNIT, img.as<T>(), s, nullptr, true);
    check_cuda(cudaMemcpyAsync(psf, img.get(), npix * sizeof(T), cudaMemcpyDeviceToHost, s), "copy to host");
  }
  finish(plan, s);
}

// dirty2vis_multi (wgridder.rs:2998-3041) on host arrays.
template <class T>
void host_dirty2vis(const WgridderOptions* o, size_t nrow, size_t nchan, const double* uvw, const double* freq,
                    const T* dirty, const void* wgt, int wgt_kind, const uint8_t* mask, T* vis, double* info) {
  if (!o) throw InvalidArgument("null options");
  if (!uvw || !freq || !vis || !dirty || !info) throw InvalidArgument("null array");
  wgt_bytes(wgt_kind, wgt, nullptr);
  check_common(*o, nrow, nchan);
  f_over_c(freq, nchan);
  size_t n = nrow * nchan, npix = o->nx * o->ny;
  cudaStream_t s = call_stream();
  Uploaded u = upload_inputs(nrow, nchan, uvw, nullptr, VIS_UNIT, wgt, nullptr, wgt_kind, mask, s);
  // Row chunks are binned one at a time, each just before it is degridded.
  const int chunks = host_row_chunks(n * 2 * sizeof(T));
  Plan<T> plan(*o, nrow, nchan, u.uvw.as<double>(), freq, u.in, false, s, chunks,
               chunks > 1 ? Plan<T>::LAYOUT_STREAMED : Plan<T>::LAYOUT_FULL);
  std::memcpy(info, plan.info().v, sizeof(plan.info().v));
  if (plan.empty()) {
    std::memset(vis, 0, n * 2 * sizeof(T));
    return;
  }
  DevBuf img = upload(dirty, npix * sizeof(T), s);
  DevBuf out(n * 2 * sizeof(T), s);
  if (plan.chunks() == 1) {
    plan.degrid(img.as<T>(), u.in, out.as<T>(), s);
    check_cuda(cudaMemcpyAsync(vis, out.get(), n * 2 * sizeof(T), cudaMemcpyDeviceToHost, s), "copy to host");
    finish(plan, s);
    return;
  }
  // Each row chunk's visibilities go back while the next chunk is degridded.
  cudaStream_t sc = copy_stream();
  Events done(plan.chunks());
  plan.degrid_streamed(img.as<T>(), u.in, out.as<T>(), s, done.e.data());
  const size_t rowb = nchan * 2 * sizeof(T);
  for (int c = 0; c < plan.chunks(); c++) {
    const size_t r0 = plan.row_begin(c), r1 = plan.row_begin(c + 1);
    check_cuda(cudaStreamWaitEvent(sc, done.e[c], 0), "wait");
    check_cuda(cudaMemcpyAsync(reinterpret_cast<unsigned char*>(vis) + r0 * rowb, out.as<unsigned char>() + r0 * rowb,
                               (r1 - r0) * rowb, cudaMemcpyDeviceToHost, sc),
               "copy to host");
  }
  check_cuda(cudaStreamSynchronize(sc), "copy to host");
  finish(plan, s);
}

}  // namespace

std::string* wg::last_error_slot() { return &g_last_error; }

// The Gram operator's and the solver's entry points (wgrid_gram.cu,
// wgrid_solver.cu) share the status mapping,
// the per-thread message and the per-thread stream.
int32_t wg::status_guarded(const std::function<void()>& f) { return guarded(f); }
cudaStream_t wg::stream_of(void* stream) {
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "no CUDA device");
  configure_pool(dev);
  return (cudaStream_t)stream;  // the caller's stream; null is the legacy default stream
}

struct RangWgridPlan {
  int single = 0;
  std::unique_ptr<Plan<float>> f;
  std::unique_ptr<Plan<double>> d;
};

extern "C" {

int32_t rang_core_wgridder_vis2dirty_f64(const WgridderOptions* opts, size_t nrow, size_t nchan, const double* uvw,
                                         const double* freq, const double* vis, const double* wgt,
                                         const uint8_t* mask, double* dirty, double* info) {
  return guarded([&] {
    if (!vis) throw InvalidArgument("null array");
    host_vis2dirty<double>(opts, nrow, nchan, uvw, freq, vis, VIS_C128, wgt, nullptr, wgt ? WGT_F64 : WGT_NONE,
                           mask, dirty, nullptr, info);
  });
}

int32_t rang_core_wgridder_vis2dirty_f32(const WgridderOptions* opts, size_t nrow, size_t nchan, const double* uvw,
                                         const double* freq, const float* vis, const float* wgt,
                                         const uint8_t* mask, float* dirty, double* info) {
  return guarded([&] {
    if (!vis) throw InvalidArgument("null array");
    host_vis2dirty<float>(opts, nrow, nchan, uvw, freq, vis, VIS_C64, wgt, nullptr, wgt ? WGT_F32 : WGT_NONE, mask,
                          dirty, nullptr, info);
  });
}

int32_t rang_core_wgridder_dirty2vis_f64(const WgridderOptions* opts, size_t nrow, size_t nchan, const double* uvw,
                                         const double* freq, const double* dirty, const double* wgt,
                                         const uint8_t* mask, double* vis, double* info) {
  return guarded([&] {
    host_dirty2vis<double>(opts, nrow, nchan, uvw, freq, dirty, wgt, wgt ? WGT_F64 : WGT_NONE, mask, vis, info);
  });
}

int32_t rang_core_wgridder_dirty2vis_f32(const WgridderOptions* opts, size_t nrow, size_t nchan, const double* uvw,
                                         const double* freq, const float* dirty, const float* wgt,
                                         const uint8_t* mask, float* vis, double* info) {
  return guarded([&] {
    host_dirty2vis<float>(opts, nrow, nchan, uvw, freq, dirty, wgt, wgt ? WGT_F32 : WGT_NONE, mask, vis, info);
  });
}

int32_t rang_core_wgridder_vis2dirty_ex_f64(const WgridderOptions* opts, size_t nrow, size_t nchan, const double* uvw,
                                            const double* freq, const void* vis, int32_t vis_kind, const void* wgt,
                                            int32_t wgt_kind, const uint8_t* mask, double* dirty, double* psf,
                                            double* info) {
  return guarded([&] {
    if (wgt_kind == WGT_F32_PRODUCT) throw InvalidArgument("invalid weight array or kind");
    host_vis2dirty<double>(opts, nrow, nchan, uvw, freq, vis, vis_kind, wgt, nullptr, wgt_kind, mask, dirty, psf,
                           info);
  });
}

int32_t rang_core_wgridder_vis2dirty_ex_f32(const WgridderOptions* opts, size_t nrow, size_t nchan, const double* uvw,
                                            const double* freq, const void* vis, int32_t vis_kind, const void* wgt,
                                            int32_t wgt_kind, const uint8_t* mask, float* dirty, float* psf,
                                            double* info) {
  return guarded([&] {
    if (wgt_kind == WGT_F32_PRODUCT) throw InvalidArgument("invalid weight array or kind");
    host_vis2dirty<float>(opts, nrow, nchan, uvw, freq, vis, vis_kind, wgt, nullptr, wgt_kind, mask, dirty, psf,
                          info);
  });
}

int32_t rang_core_wgridder_vis2dirty_ex2_f64(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                             const double* uvw, const double* freq, const void* vis, int32_t vis_kind,
                                             const void* wgt, const void* wgt2, int32_t wgt_kind, const uint8_t* mask,
                                             double* dirty, double* psf, double* info) {
  return guarded([&] {
    host_vis2dirty<double>(opts, nrow, nchan, uvw, freq, vis, vis_kind, wgt, wgt2, wgt_kind, mask, dirty, psf, info);
  });
}

int32_t rang_core_wgridder_vis2dirty_ex2_f32(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                             const double* uvw, const double* freq, const void* vis, int32_t vis_kind,
                                             const void* wgt, const void* wgt2, int32_t wgt_kind, const uint8_t* mask,
                                             float* dirty, float* psf, double* info) {
  return guarded([&] {
    host_vis2dirty<float>(opts, nrow, nchan, uvw, freq, vis, vis_kind, wgt, wgt2, wgt_kind, mask, dirty, psf, info);
  });
}

int32_t rang_core_wgridder_dirty2vis_ex_f64(const WgridderOptions* opts, size_t nrow, size_t nchan, const double* uvw,
                                            const double* freq, const double* dirty, const void* wgt,
                                            int32_t wgt_kind, const uint8_t* mask, double* vis, double* info) {
  return guarded([&] {
    if (wgt_kind == WGT_F32_PRODUCT) throw InvalidArgument("invalid weight array or kind");
    host_dirty2vis<double>(opts, nrow, nchan, uvw, freq, dirty, wgt, wgt_kind, mask, vis, info);
  });
}

int32_t rang_core_wgridder_dirty2vis_ex_f32(const WgridderOptions* opts, size_t nrow, size_t nchan, const double* uvw,
                                            const double* freq, const float* dirty, const void* wgt,
                                            int32_t wgt_kind, const uint8_t* mask, float* vis, double* info) {
  return guarded([&] {
    if (wgt_kind == WGT_F32_PRODUCT) throw InvalidArgument("invalid weight array or kind");
    host_dirty2vis<float>(opts, nrow, nchan, uvw, freq, dirty, wgt, wgt_kind, mask, vis, info);
  });
}

int32_t rang_core_wgridder_kernel_row(size_t index, double* out) {
  const KernelRow* r = kernel_row(index);
  if (!r || !out) return 1;
  double v[7] = {(double)r->w, r->ofactor, r->epsilon, r->beta, r->e0, (double)r->ndim, (double)r->single};
  std::memcpy(out, v, sizeof(v));
  return 0;
}

// ------------------------------------------------------------------ imaging weights (ffi_weights.rs)

int32_t rang_core_weight_grid_shape(size_t width, size_t height, double super_weight, size_t* shape) {
  if (!shape || !(super_weight > 0.0)) return 1;
  return guarded([&] { wg::weight_grid_shape(width, height, super_weight, &shape[0], &shape[1]); });
}

size_t rang_core_padded_size(size_t trimmed, double padding) {
  try {
    return wg::padded_size(trimmed, padding);
  } catch (...) {
    return 0;
  }
}

int32_t rang_core_stokes_i(const StokesIInputs* inputs, StokesIOutputs* outputs) {
  if (!inputs || !outputs) return 1;
  return guarded([&] { wg::stokes_i(*inputs, *outputs, call_stream()); });
}

int32_t rang_core_imaging_weights(const ImagingWeightInputs* inputs, ImagingWeightOutputs* outputs) {
  if (!inputs || !outputs) return 1;
  return guarded([&] { wg::imaging_weights(*inputs, *outputs, call_stream()); });
}

size_t rang_core_wgridder_last_error(uint8_t* buf, size_t len) {
  if (buf) std::memcpy(buf, g_last_error.data(), std::min(len, g_last_error.size()));
  return g_last_error.size();
}

int32_t rang_b200_wgridder_plan_create(const WgridderOptions* opts, size_t nrow, size_t nchan, const double* uvw_dev,
                                       const double* freq, const void* vis_dev, int32_t vis_kind, const void* wgt_dev,
                                       const void* wgt2_dev, int32_t wgt_kind, const uint8_t* mask_dev,
                                       int32_t with_vis, int32_t single, void* stream, RangWgridPlan** plan,
                                       double* info) {
  return guarded([&] {
    if (!opts || !plan) throw InvalidArgument("null options");
    if ((!uvw_dev && nrow) || !freq || !info) throw InvalidArgument("null array");
    vis_bytes(vis_kind, vis_dev);
    wgt_bytes(wgt_kind, wgt_dev, wgt2_dev);
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "no CUDA device");
    configure_pool(dev);
    Inputs in{vis_dev, vis_kind, wgt_dev, wgt2_dev, wgt_kind, mask_dev};
    cudaStream_t s = (cudaStream_t)stream;
    auto p = std::make_unique<RangWgridPlan>();
    p->single = single ? 1 : 0;
    if (single) {
      p->f = std::make_unique<Plan<float>>(*opts, nrow, nchan, uvw_dev, freq, in, with_vis != 0, s);
      std::memcpy(info, p->f->info().v, sizeof(p->f->info().v));
    } else {
      p->d = std::make_unique<Plan<double>>(*opts, nrow, nchan, uvw_dev, freq, in, with_vis != 0, s);
      std::memcpy(info, p->d->info().v, sizeof(p->d->info().v));
    }
    *plan = p.release();
  });
}

int32_t rang_b200_wgridder_plan_grid(RangWgridPlan* plan, const void* vis_dev, int32_t vis_kind, const void* wgt_dev,
                                     const void* wgt2_dev, int32_t wgt_kind, int32_t flags, void* image_dev,
                                     void* stream) {
  return guarded([&] {
    if (!plan || !image_dev) throw InvalidArgument("null array");
    const bool unit = (flags & 1) != 0, scanned = (flags & 2) != 0;
    if (!unit) vis_bytes(vis_kind, vis_dev);
    wgt_bytes(wgt_kind, wgt_dev, wgt2_dev);
    Inputs in{vis_dev, vis_kind, wgt_dev, wgt2_dev, wgt_kind, nullptr};
    ValueMode m = unit ? VALUE_UNIT : VALUE_DATA;
    if (plan->single)
      plan->f->grid(in, m, (float*)image_dev, (cudaStream_t)stream, nullptr, scanned);
    else
      plan->d->grid(in, m, (double*)image_dev, (cudaStream_t)stream, nullptr, scanned);
  });
}

int32_t rang_b200_wgridder_plan_degrid(RangWgridPlan* plan, const void* image_dev, const void* wgt_dev,
                                       int32_t wgt_kind, void* vis_dev, void* stream) {
  return guarded([&] {
    if (!plan || !image_dev || !vis_dev) throw InvalidArgument("null array");
    wgt_bytes(wgt_kind, wgt_dev, nullptr);
    Inputs in{nullptr, VIS_UNIT, wgt_dev, nullptr, wgt_kind, nullptr};
    if (plan->single)
      plan->f->degrid((const float*)image_dev, in, (float*)vis_dev, (cudaStream_t)stream);
    else
      plan->d->degrid((const double*)image_dev, in, (double*)vis_dev, (cudaStream_t)stream);
  });
}

int32_t rang_b200_wgridder_plan_status(RangWgridPlan* plan, void* stream) {
  return guarded([&] {
    if (!plan) throw InvalidArgument("null plan");
    int e = plan->single ? plan->f->kernel_errors((cudaStream_t)stream) : plan->d->kernel_errors((cudaStream_t)stream);
    if (e) throw DeviceError("a visibility fell outside its uv tile (internal inconsistency)");
  });
}

int32_t rang_b200_wgridder_plan_info(const RangWgridPlan* plan, double* info) {
  if (!plan || !info) return 1;
  const PlanInfo& pi = plan->single ? plan->f->info() : plan->d->info();
  std::memcpy(info, pi.v, sizeof(pi.v));
  return 0;
}

void rang_b200_wgridder_plan_destroy(RangWgridPlan* plan) { delete plan; }

int32_t rang_b200_wgridder_plan_residual(RangWgridPlan* plan, const void* data_dev, int32_t vis_kind,
                                         const void* wgt_dev, const void* wgt2_dev, int32_t wgt_kind,
                                         const void* model_dev, int32_t sorted, void* image_dev, double* misfit_dev,
                                         void* stream) {
  return guarded([&] {
    if (!plan || !image_dev) throw InvalidArgument("null array");
    if (vis_kind == VIS_UNIT) throw InvalidArgument("the residual needs data");
    vis_bytes(vis_kind, data_dev);
    wgt_bytes(wgt_kind, wgt_dev, wgt2_dev);
    Inputs in{data_dev, vis_kind, wgt_dev, wgt2_dev, wgt_kind, nullptr};
    if (plan->single)
      plan->f->residual(in, sorted != 0, (const float*)model_dev, (float*)image_dev, misfit_dev, (cudaStream_t)stream);
    else
      plan->d->residual(in, sorted != 0, (const double*)model_dev, (double*)image_dev, misfit_dev,
                        (cudaStream_t)stream);
  });
}

int32_t rang_b200_wgridder_plan_gram(RangWgridPlan* plan, const void* x_dev, const void* wgt_dev,
                                     const void* wgt2_dev, int32_t wgt_kind, int32_t sorted, void* image_dev,
                                     double* xgx_dev, void* stream) {
  return guarded([&] {
    if (!plan || !x_dev || !image_dev) throw InvalidArgument("null array");
    wgt_bytes(wgt_kind, wgt_dev, wgt2_dev);
    Inputs in{nullptr, VIS_UNIT, wgt_dev, wgt2_dev, wgt_kind, nullptr};
    if (plan->single)
      plan->f->gram((const float*)x_dev, in, sorted != 0, (float*)image_dev, xgx_dev, (cudaStream_t)stream);
    else
      plan->d->gram((const double*)x_dev, in, sorted != 0, (double*)image_dev, xgx_dev, (cudaStream_t)stream);
  });
}

int32_t rang_b200_wgridder_plan_sorted(const RangWgridPlan* plan, const void* dense_dev, int32_t elem_bytes,
                                       void* out_dev, void* stream) {
  return guarded([&] {
    if (!plan || !dense_dev || !out_dev) throw InvalidArgument("null array");
    if (plan->single)
      plan->f->gather_sorted(dense_dev, elem_bytes, out_dev, (cudaStream_t)stream);
    else
      plan->d->gather_sorted(dense_dev, elem_bytes, out_dev, (cudaStream_t)stream);
  });
}

int32_t rang_b200_wgridder_plan_active(const RangWgridPlan* plan, size_t* active) {
  if (!plan || !active) return 1;
  *active = plan->single ? plan->f->nvis() : plan->d->nvis();
  return 0;
}

int32_t rang_b200_wgridder_plan_memory(const RangWgridPlan* plan, size_t* bytes, int32_t n) {
  if (!plan) return -1;
  const auto m = plan->single ? plan->f->memory() : plan->d->memory();
  for (int32_t i = 0; i < n && i < (int32_t)m.size(); i++) bytes[i] = m[i].second;
  return (int32_t)m.size();
}

const char* rang_b200_wgridder_plan_memory_name(int32_t index) {
  static const auto names = Plan<float>::memory_names();
  return index >= 0 && index < (int32_t)names.size() ? names[index] : nullptr;
}

void rang_b200_wgridder_plan_release_work(RangWgridPlan* plan) {
  if (!plan) return;
  if (plan->single)
    plan->f->release_work();
  else
    plan->d->release_work();
}

size_t rang_b200_wgridder_cached_bytes(void) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  return cached_free_bytes(dev);
}

int32_t rang_b200_wgridder_release_cached(void) {
  return guarded([&] {
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "no CUDA device");
    flush_cache(dev);  // frees in stream order and waits for those frees
    cudaMemPool_t pool;
    check_cuda(cudaDeviceGetDefaultMemPool(&pool, dev), "memory pool");
    check_cuda(cudaMemPoolTrimTo(pool, 0), "memory pool");
  });
}

int32_t rang_b200_wgridder_plan_only(const WgridderOptions* opts, size_t nrow, size_t nchan, const double* uvw,
                                     const double* freq, const void* vis, int32_t vis_kind, const void* wgt,
                                     const void* wgt2, int32_t wgt_kind, const uint8_t* mask, int32_t single,
                                     int32_t nout, double* info, size_t* footprint) {
  return guarded([&] {
    if (!opts) throw InvalidArgument("null options");
    if (!uvw || !freq || !info) throw InvalidArgument("null array");
    vis_bytes(vis_kind, vis);
    wgt_bytes(wgt_kind, wgt, wgt2);
    check_common(*opts, nrow, nchan);
    f_over_c(freq, nchan);
    cudaStream_t s = call_stream();
    Uploaded u = upload_inputs(nrow, nchan, uvw, vis, vis_kind, wgt, wgt2, wgt_kind, mask, s);
    const bool with_vis = vis_kind != VIS_UNIT;
    size_t fp = 0;
    if (single) {
      Plan<float> plan(*opts, nrow, nchan, u.uvw.as<double>(), freq, u.in, with_vis, s, 1, false);
      std::memcpy(info, plan.info().v, sizeof(plan.info().v));
      fp = plan.footprint(nout);
    } else {
      Plan<double> plan(*opts, nrow, nchan, u.uvw.as<double>(), freq, u.in, with_vis, s, 1, false);
      std::memcpy(info, plan.info().v, sizeof(plan.info().v));
      fp = plan.footprint(nout);
    }
    if (footprint) *footprint = fp;
    check_cuda(cudaStreamSynchronize(s), "plan");
  });
}

int32_t rang_b200_wgridder_binning(const WgridderOptions* opts, size_t nrow, size_t nchan, const double* uvw,
                                   const double* freq, const void* vis, int32_t vis_kind, const void* wgt,
                                   const void* wgt2, int32_t wgt_kind, const uint8_t* mask, int32_t with_vis,
                                   int32_t single, int64_t* iu0, int64_t* iv0, uint32_t* key, uint32_t* sorted,
                                   size_t* nsorted, double* info) {
  return guarded([&] {
    if (!opts) throw InvalidArgument("null options");
    if (!uvw || !freq || !info || !iu0 || !iv0 || !key || !sorted || !nsorted) throw InvalidArgument("null array");
    check_common(*opts, nrow, nchan);
    size_t n = nrow * nchan;
    cudaStream_t s = call_stream();
    Uploaded u = upload_inputs(nrow, nchan, uvw, vis, vis_kind, wgt, wgt2, wgt_kind, mask, s);
    auto run = [&](auto& plan) {
      std::memcpy(info, plan.info().v, sizeof(plan.info().v));
      *nsorted = plan.nvis();
      for (size_t i = 0; i < n; i++) {
        iu0[i] = iv0[i] = -1;
        key[i] = 0xffffffffu;
      }
      plan.export_binning(key, sorted, s);
      plan.export_pixels(u.in, with_vis != 0, iu0, iv0, s);
    };
    if (single) {
      Plan<float> plan(*opts, nrow, nchan, u.uvw.as<double>(), freq, u.in, with_vis != 0, s);
      run(plan);
    } else {
      Plan<double> plan(*opts, nrow, nchan, u.uvw.as<double>(), freq, u.in, with_vis != 0, s);
      run(plan);
    }
  });
}

int64_t rang_b200_wgridder_launch_count(void) { return launch_count(); }

int32_t rang_b200_wgridder_set_method(int32_t method) {
  int old = grid_method();
  set_grid_method(method == GRID_FP32     ? GRID_FP32
                  : method == GRID_BF16X3 ? GRID_BF16X3
                  : method == GRID_TF32X3 ? GRID_TF32X3
                                          : GRID_INT8);
  return old;
}

void rang_b200_wgridder_profile(int32_t on) { profile_enable(on != 0); }

int32_t rang_b200_wgridder_profile_read(int64_t* launches, double* ms, int32_t n) {
  long long l[N_STAGES];
  double t[N_STAGES];
  profile_read(l, t);
  for (int i = 0; i < n && i < N_STAGES; i++) {
    if (launches) launches[i] = l[i];
    if (ms) ms[i] = t[i];
  }
  return N_STAGES;
}

const char* rang_b200_wgridder_stage_name(int32_t index) {
  return index >= 0 && index < N_STAGES ? STAGE_NAMES[index] : nullptr;
}

}  // extern "C"
