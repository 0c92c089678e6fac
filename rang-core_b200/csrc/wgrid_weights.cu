// Imaging weights and Stokes I formation on the B200: the reference's port of
// WSClean's weighting (core/src/weights.rs) as CUDA kernels behind its C ABI
// (core/src/ffi_weights.rs).
//
//   grid      every selected (row, channel) sample's float weight added, in
//             double, to its half-plane cell (atomics; warps whose samples
//             share a cell add once), and to the total
//   finish    Briggs / uniform / natural on the host, in the reference's
//             sequential order (the Briggs sum of squares is order-sensitive)
//   rank      the rank filter, one thread per cell, same window loop order
//   lookup    each sample's cell value as a float
//   sums      the header sums (visibility weight sum, total, max, count)
//
// Every per-sample and per-cell value is computed with the reference's
// arithmetic (the file is compiled with --fmad=false), so the results are
// the reference's bit for bit whenever the double sums are exact, which they
// are for float weights unless a cell or the total spans more than 53 bits
// of binary range; the header sums can then differ in the last bits (the
// reference's own Python test allows 1e-12).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "rang_weights.h"
#include "wgrid_plan.h"
#include "wgrid_setup.h"

namespace wg {

namespace {

// WeightGrid's geometry after the super weight (weights.rs:46-57).
struct WGeom {
  int64_t width, height;
  double scale_x, scale_y;
};

// uv_to_xy and within (weights.rs:131-144): the cell of (u, v), or -1.
__device__ __forceinline__ int64_t weight_cell(const WGeom& g, double u, double v) {
  if (v < 0.0) {
    u = -u;
    v = -v;
  }
  const double fx = floor(u * (double)g.width * g.scale_x + (double)(g.width / 2));
  const double fy = floor(v * (double)g.height * g.scale_y);
  // Out-of-range doubles saturate as Rust's `as i64` does.
  const int64_t x = fx >= 9.2e18 ? INT64_MAX : (fx <= -9.2e18 ? INT64_MIN : (fx == fx ? (int64_t)fx : 0));
  const int64_t y = fy >= 9.2e18 ? INT64_MAX : (fy <= -9.2e18 ? INT64_MIN : (fy == fy ? (int64_t)fy : 0));
  if (x >= 0 && x < g.width && y < g.height / 2) return x + y * g.width;
  return -1;
}

__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// grid_rows (weights.rs:158-188) for every (row, channel).
__global__ void k_weight_grid(uint64_t nrow, uint32_t nchan, const double* __restrict__ uvw,
                              const double* __restrict__ wavelength, const float* __restrict__ weights,
                              const uint8_t* __restrict__ selected, WGeom g, double* __restrict__ cells,
                              double* __restrict__ total) {
  const uint64_t n = nrow * nchan;
  const uint64_t nround = (n + 31) & ~31ull;
  double part = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nround;
       i += (uint64_t)gridDim.x * blockDim.x) {
    int64_t cell = -1;
    double w = 0.0;
    if (i < n) {
      const uint64_t row = i / nchan, ch = i - row * nchan;
      if (selected[row]) {
        double um = uvw[3 * row], vm = uvw[3 * row + 1];
        if (vm < 0.0) {
          um = -um;
          vm = -vm;
        }
        const double lambda = wavelength[ch];
        cell = weight_cell(g, um / lambda, vm / lambda);
        if (cell >= 0) w = (double)weights[i];
      }
    }
    part += w;
    // A warp whose samples all fall in one cell (neighbouring channels of one
    // baseline usually do) adds their sum once; otherwise each lane adds.
    const unsigned inside = __ballot_sync(0xffffffffu, cell >= 0);
    if (inside == 0xffffffffu) {
      const unsigned same = __match_any_sync(0xffffffffu, (unsigned long long)cell);
      if (same == 0xffffffffu) {
        const double s = warp_sum_d(w);
        if ((threadIdx.x & 31) == 0) atomicAdd(&cells[cell], s);
        continue;
      }
    }
    if (cell >= 0) atomicAdd(&cells[cell], w);
  }
  part = warp_sum_d(part);
  if ((threadIdx.x & 31) == 0 && part != 0.0) atomicAdd(total, part);
}

// rank_filter (weights.rs:229-269): each non-zero cell above `limit` times
// its window mean is clipped to that value; the mean sums the window's
// non-zero cells in the reference's loop order.
__global__ void k_weight_rank(const double* __restrict__ cells, double* __restrict__ out, int64_t width,
                              int64_t half, double limit, int64_t window) {
  const int64_t ncell = width * half;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncell; c += (int64_t)gridDim.x * blockDim.x) {
    const double w = cells[c];
    double v = w;
    if (w != 0.0) {
      const int64_t y = c / width, x = c - y * width, d = window / 2;
      const int64_t x1 = x >= d ? x - d : 0, y1 = y >= d ? y - d : 0;
      const int64_t x2 = x + d >= width ? width : x + d;
      const int64_t y2 = y + d >= half ? half : y + d;
      int64_t count = 0;
      double sum = 0.0;
      for (int64_t yi = y1; yi < y2; yi++)
        for (int64_t xi = x1; xi < x2; xi++) {
          const double q = cells[yi * width + xi];
          if (q != 0.0) {
            count++;
            sum += q;
          }
        }
      const double mean = sum / (double)count;
      if (w > mean * limit) v = mean * limit;
    }
    out[c] = v;
  }
}

// lookup_rows (weights.rs:283-315): each selected sample's cell as a float.
__global__ void k_weight_lookup(uint64_t nrow, uint32_t nchan, const double* __restrict__ uvw,
                                const double* __restrict__ wavelength, const uint8_t* __restrict__ selected, WGeom g,
                                const double* __restrict__ cells, float* __restrict__ out) {
  const uint64_t n = nrow * nchan;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t row = i / nchan, ch = i - row * nchan;
    float v = 0.0f;
    if (selected[row]) {
      const double lambda = wavelength[ch];
      const int64_t cell = weight_cell(g, uvw[3 * row] / lambda, uvw[3 * row + 1] / lambda);
      if (cell >= 0) v = (float)cells[cell];
    }
    out[i] = v;
  }
}

struct WeightSumsDev {
  double vsum, total;
  unsigned long long max_bits, count;
};

// weight_sums (weights.rs:564-582).
__global__ void k_weight_sums(uint64_t n, const float* __restrict__ weights, const float* __restrict__ imaging,
                              WeightSumsDev* __restrict__ out) {
  double vsum = 0.0, total = 0.0, largest = 0.0;
  unsigned long long count = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float w = weights[i];
    const float cum = w * imaging[i];
    if (cum != 0.0f) {
      vsum += (double)w;
      count++;
    }
    largest = fmax(largest, (double)cum);
    total += (double)cum;
  }
  vsum = warp_sum_d(vsum);
  total = warp_sum_d(total);
  for (int o = 16; o > 0; o >>= 1) {
    largest = fmax(largest, __shfl_xor_sync(0xffffffffu, largest, o));
    count += __shfl_xor_sync(0xffffffffu, count, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (vsum != 0.0) atomicAdd(&out->vsum, vsum);
    if (total != 0.0) atomicAdd(&out->total, total);
    if (count) atomicAdd(&out->count, count);
    // largest >= 0: its bits order as the values do.
    atomicMax(&out->max_bits, (unsigned long long)__double_as_longlong(largest));
  }
}

// Stokes I (weights.rs:522-562), one cell per thread.
__global__ void k_stokes_i(uint64_t ncell, const float* __restrict__ data, const float* __restrict__ weights,
                           const uint8_t* __restrict__ flags, float* __restrict__ vis, float* __restrict__ out) {
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < ncell;
       c += (uint64_t)gridDim.x * blockDim.x) {
    const float* d = data + 8 * c;
    const float xx_re = d[0], xx_im = d[1], yy_re = d[6], yy_im = d[7];
    const float re = (yy_re + xx_re) * 0.5f, im = (yy_im + xx_im) * 0.5f;
    const bool fin = isfinite(re) && isfinite(im);
    vis[2 * c] = fin ? re : 0.0f;
    vis[2 * c + 1] = fin ? im : 0.0f;
    const float* w = weights + 4 * c;
    const uint8_t* f = flags + 4 * c;
    float weight = (f[0] == 0 && isfinite(xx_re) && isfinite(xx_im)) ? w[0] * 4.0f : 0.0f;
    if (f[3] == 0 && isfinite(yy_re) && isfinite(yy_im)) {
      const float yy = w[3] * 4.0f;
      weight = yy < weight ? yy : weight;  // std::min: the second only when strictly smaller
    } else {
      weight = 0.0f;
    }
    out[c] = weight;
  }
}

unsigned grid_blocks(uint64_t n) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 148 * 32)); }

DevBuf upload_bytes(const void* host, size_t bytes, cudaStream_t s) {
  DevBuf b;
  if (bytes) {
    b.alloc(bytes, s);
    check_cuda(cudaMemcpyAsync(b.get(), host, bytes, cudaMemcpyHostToDevice, s), "copy to device");
  }
  return b;
}

}  // namespace

// WeightGrid::shape (weights.rs:102-112): rounded half away from zero, then even.
void weight_grid_shape(size_t width, size_t height, double super_weight, size_t* w, size_t* h) {
  size_t a = (size_t)std::llround((double)width / super_weight);
  size_t b = (size_t)std::llround((double)height / super_weight);
  *w = a + (a % 2);
  *h = b + (b % 2);
}

// padded_size (weights.rs:38-42).
size_t padded_size(size_t trimmed, double padding) {
  size_t p = (size_t)std::ceil((double)trimmed * padding);
  return p + (4 - p % 4) % 4;
}

void stokes_i(const StokesIInputs& in, StokesIOutputs& out, cudaStream_t s) {
  if (!in.data || !in.weights || !in.flags || !out.vis || !out.weight) throw InvalidArgument("null array");
  const size_t n = in.ncell;
  if (n == 0) return;
  DevBuf d = upload_bytes(in.data, n * 8 * sizeof(float), s);
  DevBuf w = upload_bytes(in.weights, n * 4 * sizeof(float), s);
  DevBuf f = upload_bytes(in.flags, n * 4, s);
  DevBuf v(n * 2 * sizeof(float), s), o(n * sizeof(float), s);
  k_stokes_i<<<grid_blocks(n), 256, 0, s>>>(n, d.as<float>(), w.as<float>(), f.as<uint8_t>(), v.as<float>(),
                                            o.as<float>());
  check_cuda(cudaGetLastError(), "stokes i");
  check_cuda(cudaMemcpyAsync(out.vis, v.get(), n * 2 * sizeof(float), cudaMemcpyDeviceToHost, s), "copy to host");
  check_cuda(cudaMemcpyAsync(out.weight, o.get(), n * sizeof(float), cudaMemcpyDeviceToHost, s), "copy to host");
  check_cuda(cudaStreamSynchronize(s), "stokes i");
}

// imaging_weights (weights.rs:465-520 without tapers) and weight_sums
// (:564-582), as the FFI runs them (ffi_weights.rs:166-233).
void imaging_weights(const ImagingWeightInputs& in, ImagingWeightOutputs& out, cudaStream_t s) {
  if (!out.weights) throw InvalidArgument("null output weights");
  if (in.class_ > 2) throw InvalidArgument("weighting class must be 0, 1 or 2");
  if (!in.uvw || !in.wavelength || !in.weights || !in.row_selected) throw InvalidArgument("null array");
  if (in.width == 0 || in.height == 0 || !(in.super_weight > 0.0) || in.pixel_scale_x <= 0.0 ||
      in.pixel_scale_y <= 0.0)
    throw InvalidArgument("positive grid size, scales and super weight required");
  size_t gw, gh;
  weight_grid_shape(in.width, in.height, in.super_weight, &gw, &gh);
  const size_t ncell = gw * (gh / 2), n = in.nrow * in.nchan;
  if (in.nchan > 0xffffffffull) throw InvalidArgument("too many channels");
  WGeom g{(int64_t)gw, (int64_t)gh, in.pixel_scale_x, in.pixel_scale_y};
  DevBuf uvw = upload_bytes(in.uvw, in.nrow * 3 * sizeof(double), s);
  DevBuf wl = upload_bytes(in.wavelength, in.nchan * sizeof(double), s);
  DevBuf wts = upload_bytes(in.weights, n * sizeof(float), s);
  DevBuf sel = upload_bytes(in.row_selected, in.nrow, s);
  DevBuf cells(std::max<size_t>(ncell, 1) * sizeof(double), s), total(sizeof(double), s);
  check_cuda(cudaMemsetAsync(cells.get(), 0, std::max<size_t>(ncell, 1) * sizeof(double), s), "memset");
  check_cuda(cudaMemsetAsync(total.get(), 0, sizeof(double), s), "memset");
  if (n) {
    k_weight_grid<<<grid_blocks(n), 256, 0, s>>>(in.nrow, (uint32_t)in.nchan, uvw.as<double>(), wl.as<double>(),
                                                 wts.as<float>(), sel.as<uint8_t>(), g, cells.as<double>(),
                                                 total.as<double>());
    check_cuda(cudaGetLastError(), "weight grid");
  }
  // finish (weights.rs:190-227), sequentially on the host.
  std::vector<double> host(ncell);
  double tot = 0.0;
  if (ncell) check_cuda(cudaMemcpyAsync(host.data(), cells.get(), ncell * sizeof(double), cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaMemcpyAsync(&tot, total.get(), sizeof(double), cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "weight grid");
  if (in.class_ == 2) {
    double avg_w = 0.0;
    for (double v : host) avg_w += v * v;
    avg_w /= tot;
    const double numerator_sqrt = 5.0 * std::exp(-2.302585092994046 * in.robust);  // -LN_10 * robust
    const double s_sq = numerator_sqrt * numerator_sqrt / avg_w;
    for (double& v : host)
      if (v != 0.0) v = 1.0 / (1.0 + v * s_sq);
  } else if (in.class_ == 1) {
    for (double& v : host)
      if (v != 0.0) v = 1.0 / v;
  } else {
    for (double& v : host)
      if (v != 0.0) v = 1.0;
  }
  if (ncell) check_cuda(cudaMemcpyAsync(cells.get(), host.data(), ncell * sizeof(double), cudaMemcpyHostToDevice, s), "copy");
  if (in.rank_filter_level >= 1.0 && ncell) {
    DevBuf filtered(ncell * sizeof(double), s);
    k_weight_rank<<<grid_blocks(ncell), 256, 0, s>>>(cells.as<double>(), filtered.as<double>(), (int64_t)gw,
                                                     (int64_t)(gh / 2), in.rank_filter_level,
                                                     (int64_t)in.rank_filter_size);
    check_cuda(cudaGetLastError(), "rank filter");
    cells = std::move(filtered);
  }
  DevBuf img(std::max<size_t>(n, 1) * sizeof(float), s);
  if (n) {
    k_weight_lookup<<<grid_blocks(n), 256, 0, s>>>(in.nrow, (uint32_t)in.nchan, uvw.as<double>(), wl.as<double>(),
                                                   sel.as<uint8_t>(), g, cells.as<double>(), img.as<float>());
    check_cuda(cudaGetLastError(), "weight lookup");
    check_cuda(cudaMemcpyAsync(out.weights, img.get(), n * sizeof(float), cudaMemcpyDeviceToHost, s), "copy to host");
  }
  if (out.grid && ncell)
    check_cuda(cudaMemcpyAsync(out.grid, cells.get(), ncell * sizeof(double), cudaMemcpyDeviceToHost, s), "copy to host");
  if (out.sums) {
    DevBuf ws(sizeof(WeightSumsDev), s);
    check_cuda(cudaMemsetAsync(ws.get(), 0, sizeof(WeightSumsDev), s), "memset");
    if (n) {
      k_weight_sums<<<grid_blocks(n), 256, 0, s>>>(n, wts.as<float>(), img.as<float>(), ws.as<WeightSumsDev>());
      check_cuda(cudaGetLastError(), "weight sums");
    }
    WeightSumsDev r{};
    check_cuda(cudaMemcpyAsync(&r, ws.get(), sizeof(r), cudaMemcpyDeviceToHost, s), "copy");
    check_cuda(cudaStreamSynchronize(s), "weight sums");
    double largest;
    std::memcpy(&largest, &r.max_bits, sizeof(largest));
    out.sums[0] = r.vsum;
    out.sums[1] = r.total;
    out.sums[2] = largest;
    out.sums[3] = (double)r.count;
  }
  check_cuda(cudaStreamSynchronize(s), "imaging weights");
}

}  // namespace wg
