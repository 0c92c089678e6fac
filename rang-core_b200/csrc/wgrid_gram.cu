// The w-aware normal operator without visibilities on the B200: the
// reference's GramOperator (core/src/gridder_gram.rs), a sum of Toeplitz
// operators, one per w-node, each applied by FFTs on the 2n grid:
//   G~ m = Re sum_k e_k (K_k * (conj(e_k) m)),  e_k(l) = exp(2 pi i w_k x(l)),
//   K_k(d) = sum_p W_p psi_k(w_p) exp(2 pi i u_p . d),  x = n - 1.
// Setup: the w-expansion psi (a regularised least-squares fit, on the host),
// then per node the weights W_p psi_k(w_p) (a kernel) gridded by this
// library's gridder on the 2n grid without w (unit visibilities 1 - i, whose
// real image is the sum of the even and odd parts of K_k), the even/odd split
// (a kernel) and the real spectrum (cuFFT). Apply: per node the screened,
// zero-padded model, a forward 2-D FFT, the spectrum, the inverse FFT and the
// screened real part added to the output, all on the device.
#include <cufft.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <vector>

#include "rang_gram.h"
#include "wgrid_plan.h"
#include "wgrid_setup.h"

namespace wg {

namespace {

constexpr double GPI = 3.14159265358979323846;
constexpr double GC_LIGHT = 299792458.0;  // wgridder.rs:58
constexpr size_t TABLE_BINS = 8192;       // gridder_gram.rs:37

void check_fft_g(cufftResult r, const char* what) {
  if (r != CUFFT_SUCCESS) throw DeviceError(std::string("cuFFT ") + what + " failed (" + std::to_string((int)r) + ")");
}

}  // namespace

// WExpansion::new (gridder_gram.rs:88-141) and measure_sup (:143-163).
struct WExpansionHost {
  size_t stencil;
  double theta;
  std::vector<double> table;  // (TABLE_BINS + 1) x stencil
  double sup_error = 0.0, lebesgue = 0.0;

  double coefficient(double s, size_t j) const {  // gridder_gram.rs:166-174
    double f = (s + 0.5) * (double)TABLE_BINS;
    size_t b = std::min<size_t>((size_t)f, TABLE_BINS - 1);
    double a = f - (double)b;
    double lo = table[b * stencil + j], hi = table[(b + 1) * stencil + j];
    return lo + a * (hi - lo);
  }

  WExpansionHost(size_t s, double th, double ridge) : stencil(s), theta(th) {
    if (s < 2 || s % 2) throw InvalidArgument("the w stencil must be even and at least 2");
    if (!(th > 0.0 && th < GPI)) throw InvalidArgument("the w phase step must lie in (0, pi)");
    std::vector<double> t(s);
    for (size_t j = 0; j < s; j++) t[j] = (double)j - ((double)s - 1.0) / 2.0;
    const size_t m = 64 * s;
    std::vector<double> xi(m);
    for (size_t i = 0; i < m; i++) xi[i] = std::cos(GPI * ((double)i + 0.5) / (double)m);
    auto kernel = [&](double d) {
      double acc = 0.0;
      for (double x : xi) acc += std::cos(th * x * d);
      return acc / (double)m;
    };
    std::vector<double> l(s * s);
    for (size_t i = 0; i < s; i++) {
      for (size_t j = 0; j < s; j++) l[i * s + j] = kernel(t[i] - t[j]);
      l[i * s + i] *= 1.0 + ridge;
    }
    // Lower Cholesky factor in place (gridder_gram.rs:57-73).
    for (size_t j = 0; j < s; j++) {
      for (size_t k = 0; k < j; k++) {
        double f = l[j * s + k];
        for (size_t i = j; i < s; i++) l[i * s + j] -= l[i * s + k] * f;
      }
      double d = std::sqrt(l[j * s + j]);
      for (size_t i = j; i < s; i++) l[i * s + j] /= d;
    }
    table.assign((TABLE_BINS + 1) * s, 0.0);
    for (size_t b = 0; b <= TABLE_BINS; b++) {
      double sv = -0.5 + (double)b / (double)TABLE_BINS;
      double* row = &table[b * s];
      for (size_t j = 0; j < s; j++) row[j] = kernel(sv - t[j]);
      // Solve L L^T x = c (gridder_gram.rs:75-86).
      for (size_t i = 0; i < s; i++) {
        for (size_t k = 0; k < i; k++) row[i] -= l[i * s + k] * row[k];
        row[i] /= l[i * s + i];
      }
      for (size_t i = s; i-- > 0;) {
        for (size_t k = i + 1; k < s; k++) row[i] -= l[k * s + i] * row[k];
        row[i] /= l[i * s + i];
      }
    }
    for (size_t b = 0; b <= TABLE_BINS; b++) {
      double sum = 0.0;
      for (size_t j = 0; j < s; j++) sum += std::fabs(table[b * s + j]);
      lebesgue = std::max(lebesgue, sum);
    }
    std::vector<double> c(s);
    for (size_t sb = 0; sb <= 256; sb++) {
      double sv = -0.5 + (double)sb / 256.0 + (sb < 256 ? 0.5 / 8192.0 : 0.0);
      for (size_t j = 0; j < s; j++) c[j] = coefficient(sv, j);
      for (size_t xb = 0; xb <= 512; xb++) {
        double x = (double)xb / 512.0;
        double re = std::cos(th * x * sv), im = std::sin(th * x * sv);
        for (size_t j = 0; j < s; j++) {
          re -= c[j] * std::cos(th * x * t[j]);
          im -= c[j] * std::sin(th * x * t[j]);
        }
        sup_error = std::max(sup_error, std::hypot(re, im));
      }
    }
  }
};

namespace {

// nm1 (gridder_gram.rs:176-180).
double nm1(double l, double m) {
  double r2 = l * l + m * m;
  return -r2 / (std::sqrt(std::max(1.0 - r2, 0.0)) + 1.0);
}

// The node-k weights of every visibility (gridder_gram.rs:313-333).
template <class T>
__global__ void k_gram_node_weights(uint64_t nrow, uint32_t nchan, const double* __restrict__ wgt,
                                    const double* __restrict__ abs_w, const double* __restrict__ foc,
                                    const double* __restrict__ table, uint32_t stencil, double wmin, double dw,
                                    uint64_t cells, uint32_t k, T* __restrict__ out,
                                    unsigned long long* __restrict__ active) {
  const uint64_t n = nrow * nchan;
  unsigned long long count = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t row = i / nchan, ch = i - row * nchan;
    const double weight = wgt[i];
    T o = (T)0;
    if (weight != 0.0) {
      const double p = (abs_w[row] * foc[ch] - wmin) / dw;
      const double fl = fmax(floor(p), 0.0);
      uint64_t cell = fl >= 1.8e19 ? ~0ull : (uint64_t)fl;
      cell = cell < cells ? cell : cells;
      if (k >= cell && k < cell + stencil) {
        const double frac = fmin(fmax(p - (double)cell - 0.5, -0.5), 0.5);
        // WExpansion::coefficient (gridder_gram.rs:166-174)
        const double f = (frac + 0.5) * (double)TABLE_BINS;
        uint64_t b = (uint64_t)f;
        b = b < TABLE_BINS - 1 ? b : TABLE_BINS - 1;
        const double a = f - (double)b;
        const uint32_t j = (uint32_t)(k - cell);
        const double lo = table[b * stencil + j], hi = table[(b + 1) * stencil + j];
        o = (T)(weight * (lo + a * (hi - lo)));
        count++;
      }
    }
    out[i] = o;
  }
  for (int s = 16; s > 0; s >>= 1) count += __shfl_down_sync(0xffffffffu, count, s);
  if ((threadIdx.x & 31) == 0 && count) atomicAdd(active, count);
}

// K at d = (i - n, j - n) stored at d mod 2n from the gridded real image:
// the even part is the real part of K, the odd part its imaginary part
// (gridder_gram.rs:354-375); with `no_w` the image is the PSF and K is real.
template <class T>
__global__ void k_gram_kgrid(const T* __restrict__ dirty, int n, int no_w, cplx<T>* __restrict__ kgrid,
                             double* __restrict__ psf_no_w) {
  const int big = 2 * n;
  const uint64_t total = (uint64_t)big * big;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < total; q += (uint64_t)gridDim.x * blockDim.x) {
    const int ki = (int)(q / big), kj = (int)(q - (uint64_t)ki * big);
    const int i = (ki + n) % big, j = (kj + n) % big;
    cplx<T> o{(T)0, (T)0};
    if (i != 0 && j != 0) {
      const T a = dirty[(size_t)i * big + j];
      if (no_w) {
        o = {a, (T)0};
        psf_no_w[(size_t)i * big + j] = (double)a;
      } else {
        const T b = dirty[(size_t)(big - i) * big + (big - j)];
        const T half = (T)0.5;
        o = {(a + b) * half, (a - b) * half};
        psf_no_w[(size_t)i * big + j] += (double)o.re;
      }
    }
    kgrid[q] = o;
  }
}

struct SpecStats {
  unsigned long long re_max_bits, im_max_bits, small;
};

// The real part of the transformed K times `scale` (gridder_gram.rs:647-684).
template <class T>
__global__ void k_gram_real(const cplx<T>* __restrict__ f, uint64_t total, double scale, T* __restrict__ spec,
                            SpecStats* __restrict__ st) {
  double re_max = 0.0, im_max = 0.0;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < total; q += (uint64_t)gridDim.x * blockDim.x) {
    const cplx<T> c = f[q];
    re_max = fmax(re_max, fabs((double)c.re));
    im_max = fmax(im_max, fabs((double)c.im));
    spec[q] = (T)((double)c.re * scale);
  }
  for (int s = 16; s > 0; s >>= 1) {
    re_max = fmax(re_max, __shfl_down_sync(0xffffffffu, re_max, s));
    im_max = fmax(im_max, __shfl_down_sync(0xffffffffu, im_max, s));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&st->re_max_bits, (unsigned long long)__double_as_longlong(re_max));
    atomicMax(&st->im_max_bits, (unsigned long long)__double_as_longlong(im_max));
  }
}

template <class T>
__global__ void k_gram_small(const T* __restrict__ spec, uint64_t total, double floor_v, SpecStats* __restrict__ st) {
  unsigned long long small = 0;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < total; q += (uint64_t)gridDim.x * blockDim.x)
    if (fabs((double)spec[q]) < floor_v) small++;
  for (int s = 16; s > 0; s >>= 1) small += __shfl_down_sync(0xffffffffu, small, s);
  if ((threadIdx.x & 31) == 0 && small) atomicAdd(&st->small, small);
}

// z = m conj(e_k) on the first n rows and columns of the 2n grid, zero elsewhere.
template <class T>
__global__ void k_gram_screen_in(const double* __restrict__ m, const double* __restrict__ x, int n, double wk,
                                 cplx<T>* __restrict__ z) {
  const int big = 2 * n;
  const uint64_t total = (uint64_t)big * big;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < total; q += (uint64_t)gridDim.x * blockDim.x) {
    const int i = (int)(q / big), j = (int)(q - (uint64_t)i * big);
    cplx<T> o{(T)0, (T)0};
    if (i < n && j < n) {
      const double v = m[(size_t)i * n + j];
      if (v != 0.0) {
        double s, c;
        sincos(2.0 * GPI * wk * x[(size_t)i * n + j], &s, &c);
        o = {(T)(v * c), (T)(-v * s)};
      }
    }
    z[q] = o;
  }
}

template <class T>
__global__ void k_gram_spectrum(cplx<T>* __restrict__ z, const T* __restrict__ spec, uint64_t total) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < total; q += (uint64_t)gridDim.x * blockDim.x) {
    const T g = spec[q];
    cplx<T> v = z[q];
    z[q] = {v.re * g, v.im * g};
  }
}

// out += Re(y e_k) on the n x n image.
template <class T>
__global__ void k_gram_screen_out(const cplx<T>* __restrict__ y, const double* __restrict__ x, int n, double wk,
                                  double* __restrict__ out) {
  const int big = 2 * n;
  const uint64_t total = (uint64_t)n * n;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < total; q += (uint64_t)gridDim.x * blockDim.x) {
    const int i = (int)(q / n), j = (int)(q - (uint64_t)i * n);
    double s, c;
    sincos(2.0 * GPI * wk * x[q], &s, &c);
    const cplx<T> v = y[(size_t)i * big + j];
    out[q] += (double)v.re * c - (double)v.im * s;
  }
}

unsigned gblocks(uint64_t n) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 148 * 32)); }

template <class T>
struct FftT;
template <>
struct FftT<float> {
  static constexpr cufftType type = CUFFT_C2C;
  static cufftResult exec(cufftHandle h, cplx<float>* p, int dir) {
    return cufftExecC2C(h, reinterpret_cast<cufftComplex*>(p), reinterpret_cast<cufftComplex*>(p), dir);
  }
};
template <>
struct FftT<double> {
  static constexpr cufftType type = CUFFT_Z2Z;
  static cufftResult exec(cufftHandle h, cplx<double>* p, int dir) {
    return cufftExecZ2Z(h, reinterpret_cast<cufftDoubleComplex*>(p), reinterpret_cast<cufftDoubleComplex*>(p), dir);
  }
};

}  // namespace

// One operator: its spectra, screens' abscissae and statistics.
struct GramOpBase {
  virtual ~GramOpBase() = default;
  virtual void apply(const double* m, double* out, cudaStream_t s) = 0;
  virtual std::unique_ptr<GramOpBase> inverse_filter(double rho, cudaStream_t s) const = 0;
  virtual const double* psf_no_w() const = 0;
  int n = 0;
  double stats[RANG_GRAM_NSTATS] = {0};
};

template <class T>
struct GramOp : GramOpBase {
  double w0 = 0.0, dw = 0.0;
  DevBuf x;                      // n * n doubles: n - 1 per pixel
  std::vector<DevBuf> spectra;   // (2n)^2 T each, row-major, scaled by 1 / (2n)^2
  DevBuf psf;                    // (2n)^2 doubles: sum of Re K_k
  DevBuf work;                   // (2n)^2 cplx<T>
  cufftHandle plan = 0;

  ~GramOp() override {
    if (plan) cufftDestroy(plan);
  }
  void make_plan(cudaStream_t s) {
    const int big = 2 * n;
    check_fft_g(cufftPlan2d(&plan, big, big, FftT<T>::type), "2-D plan");
    check_fft_g(cufftSetStream(plan, s), "stream");
    work.alloc((size_t)big * big * sizeof(cplx<T>), s);
  }

  // The real spectrum of the K grid in `work` (gridder_gram.rs:647-684).
  void push_spectrum(cudaStream_t s, double* hermitian, unsigned long long* small_cells) {
    const int big = 2 * n;
    const uint64_t total = (uint64_t)big * big;
    check_fft_g(cufftSetStream(plan, s), "stream");
    check_fft_g(FftT<T>::exec(plan, work.as<cplx<T>>(), CUFFT_FORWARD), "forward");
    DevBuf spec(total * sizeof(T), s), st(sizeof(SpecStats), s);
    check_cuda(cudaMemsetAsync(st.get(), 0, sizeof(SpecStats), s), "memset");
    const double scale = 1.0 / (double)total;
    k_gram_real<T><<<gblocks(total), 256, 0, s>>>(work.as<cplx<T>>(), total, scale, spec.as<T>(), st.as<SpecStats>());
    check_cuda(cudaGetLastError(), "spectrum");
    SpecStats h{};
    check_cuda(cudaMemcpyAsync(&h, st.get(), sizeof(h), cudaMemcpyDeviceToHost, s), "copy");
    check_cuda(cudaStreamSynchronize(s), "spectrum");
    double re_max, im_max;
    std::memcpy(&re_max, &h.re_max_bits, 8);
    std::memcpy(&im_max, &h.im_max_bits, 8);
    *hermitian = std::max(*hermitian, im_max / std::max(re_max, 1e-300));
    k_gram_small<T><<<gblocks(total), 256, 0, s>>>(spec.as<T>(), total, 1e-7 * re_max * scale, st.as<SpecStats>());
    check_cuda(cudaGetLastError(), "spectrum");
    check_cuda(cudaMemcpyAsync(&h, st.get(), sizeof(h), cudaMemcpyDeviceToHost, s), "copy");
    check_cuda(cudaStreamSynchronize(s), "spectrum");
    *small_cells += h.small;
    spectra.push_back(std::move(spec));
  }

  void apply(const double* m, double* out, cudaStream_t s) override {  // gridder_gram.rs:518-631
    const int big = 2 * n;
    const uint64_t total = (uint64_t)big * big;
    check_cuda(cudaMemsetAsync(out, 0, (size_t)n * n * sizeof(double), s), "memset");
    check_fft_g(cufftSetStream(plan, s), "stream");
    for (size_t k = 0; k < spectra.size(); k++) {
      const double wk = w0 + (double)k * dw;
      k_gram_screen_in<T><<<gblocks(total), 256, 0, s>>>(m, x.as<double>(), n, wk, work.as<cplx<T>>());
      check_fft_g(FftT<T>::exec(plan, work.as<cplx<T>>(), CUFFT_FORWARD), "forward");
      k_gram_spectrum<T><<<gblocks(total), 256, 0, s>>>(work.as<cplx<T>>(), spectra[k].as<T>(), total);
      check_fft_g(FftT<T>::exec(plan, work.as<cplx<T>>(), CUFFT_INVERSE), "inverse");
      k_gram_screen_out<T><<<gblocks((uint64_t)n * n), 256, 0, s>>>(work.as<cplx<T>>(), x.as<double>(), n, wk, out);
    }
    check_cuda(cudaGetLastError(), "gram apply");
  }

  // inverse_filter (gridder_gram.rs:488-511): 1 / norm / (max(K norm, 0) + rho).
  std::unique_ptr<GramOpBase> inverse_filter(double rho, cudaStream_t s) const override {
    if (spectra.size() != 1 || !(rho > 0.0)) throw InvalidArgument("the filter needs a one-node operator and a positive rho");
    const int big = 2 * n;
    const uint64_t total = (uint64_t)big * big;
    std::vector<T> h(total);
    check_cuda(cudaMemcpyAsync(h.data(), spectra[0].get(), total * sizeof(T), cudaMemcpyDeviceToHost, s), "copy");
    check_cuda(cudaStreamSynchronize(s), "copy");
    const double norm = (double)total;
    for (auto& v : h) v = (T)(1.0 / norm / (std::max((double)v * norm, 0.0) + rho));
    auto op = std::make_unique<GramOp<T>>();
    op->n = n;
    std::memcpy(op->stats, stats, sizeof(stats));
    op->x.alloc((size_t)n * n * sizeof(double), s);
    check_cuda(cudaMemsetAsync(op->x.get(), 0, (size_t)n * n * sizeof(double), s), "memset");
    DevBuf spec(total * sizeof(T), s);
    check_cuda(cudaMemcpyAsync(spec.get(), h.data(), total * sizeof(T), cudaMemcpyHostToDevice, s), "copy");
    check_cuda(cudaStreamSynchronize(s), "copy");
    op->spectra.push_back(std::move(spec));
    op->make_plan(s);
    return op;
  }
  const double* psf_no_w() const override { return psf.as<double>(); }
};

template <class T>
std::unique_ptr<GramOpBase> gram_create(const WgridderOptions& opts, size_t nrow, size_t nchan, const double* uvw_dev,
                                        const double* freq, const double* wgt_dev, const WExpansionHost* ex,
                                        double epsilon, cudaStream_t s) {
  const size_t n = opts.nx;
  if (opts.ny != n || n % 2) throw InvalidArgument("the Gram operator needs a square image of even side");
  if (ex && (opts.divide_by_n || opts.center_x != 0.0 || opts.center_y != 0.0))
    throw InvalidArgument("the Gram operator handles divide_by_n = false, no shift");
  if (!uvw_dev || !freq || !wgt_dev || nrow == 0 || nchan == 0) throw InvalidArgument("empty measurement");
  const size_t big = 2 * n;
  const uint64_t total = (uint64_t)big * big;
  auto op = std::make_unique<GramOp<T>>();
  op->n = (int)n;
  // Fold to w >= 0 on the host (gridder_gram.rs:247-260).
  std::vector<double> uvw(nrow * 3);
  check_cuda(cudaMemcpyAsync(uvw.data(), uvw_dev, nrow * 3 * sizeof(double), cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "copy");
  const double fw = opts.flip_w ? -1.0 : 1.0;
  std::vector<double> abs_w(nrow);
  for (size_t r = 0; r < nrow; r++) {
    double* c = &uvw[3 * r];
    const double w = fw * c[2];
    if (w < 0.0) {
      c[0] = -c[0];
      c[1] = -c[1];
      c[2] = -c[2];
    }
    abs_w[r] = std::fabs(w);
  }
  const double fmin = freq[0] / GC_LIGHT, fmax = freq[nchan - 1] / GC_LIGHT;
  double wmin = INFINITY, wmax = 0.0;
  for (double w : abs_w) {
    wmin = std::min(wmin, w * fmin);
    wmax = std::max(wmax, w * fmax);
  }
  // n - 1 per pixel and its range (gridder_gram.rs:262-274).
  const double half = (double)(n / 2);
  std::vector<double> xh(n * n);
  double xmin = 0.0, xmax = -2.0;
  for (size_t i = 0; i < n; i++) {
    const double l = ((double)i - half) * opts.pixsize_x;
    for (size_t j = 0; j < n; j++) {
      const double v = ex ? nm1(l, ((double)j - half) * opts.pixsize_y) : 0.0;
      xh[i * n + j] = v;
      xmin = std::min(xmin, v);
      xmax = std::max(xmax, v);
    }
  }
  op->x.alloc(n * n * sizeof(double), s);
  check_cuda(cudaMemcpyAsync(op->x.get(), xh.data(), n * n * sizeof(double), cudaMemcpyHostToDevice, s), "copy");
  const double x_range = std::max(xmax - xmin, 1e-300);
  size_t stencil = ex ? ex->stencil : 1, planes = 1, cells = 0;
  if (ex) {
    op->dw = ex->theta / (2.0 * GPI * x_range);
    cells = (size_t)std::floor((wmax - wmin) / op->dw);
    planes = cells + stencil;
    op->w0 = wmin - (double)(stencil / 2 - 1) * op->dw;
  }
  // Gridder options on the 2n grid without w (gridder_gram.rs:282-288).
  WgridderOptions g = opts;
  g.nx = big;
  g.ny = big;
  g.do_wgridding = 0;
  g.epsilon = epsilon;
  DevBuf fuvw(nrow * 3 * sizeof(double), s), aw(nrow * sizeof(double), s), foc(nchan * sizeof(double), s);
  std::vector<double> foch(nchan);
  for (size_t c = 0; c < nchan; c++) foch[c] = freq[c] / GC_LIGHT;
  check_cuda(cudaMemcpyAsync(fuvw.get(), uvw.data(), nrow * 3 * sizeof(double), cudaMemcpyHostToDevice, s), "copy");
  check_cuda(cudaMemcpyAsync(aw.get(), abs_w.data(), nrow * sizeof(double), cudaMemcpyHostToDevice, s), "copy");
  check_cuda(cudaMemcpyAsync(foc.get(), foch.data(), nchan * sizeof(double), cudaMemcpyHostToDevice, s), "copy");
  DevBuf table;
  if (ex) {
    table.alloc(ex->table.size() * sizeof(double), s);
    check_cuda(cudaMemcpyAsync(table.get(), ex->table.data(), ex->table.size() * sizeof(double),
                               cudaMemcpyHostToDevice, s),
               "copy");
  }
  const size_t nvis = nrow * nchan;
  // The unit visibility 1 - i: the real image is sum W (cos + sin).
  DevBuf unit;
  if (ex) {
    std::vector<float> one(2 * nvis);
    for (size_t i = 0; i < nvis; i++) {
      one[2 * i] = 1.0f;
      one[2 * i + 1] = -1.0f;
    }
    unit.alloc(nvis * 8, s);
    check_cuda(cudaMemcpyAsync(unit.get(), one.data(), nvis * 8, cudaMemcpyHostToDevice, s), "copy");
    check_cuda(cudaStreamSynchronize(s), "copy");
  }
  DevBuf plane_wgt(nvis * sizeof(T), s), dirty(total * sizeof(T), s), active(8, s);
  check_cuda(cudaMemsetAsync(active.get(), 0, 8, s), "memset");
  op->psf.alloc(total * sizeof(double), s);
  check_cuda(cudaMemsetAsync(op->psf.get(), 0, total * sizeof(double), s), "memset");
  op->make_plan(s);
  double hermitian = 0.0, grid_sec = 0.0, fft_sec = 0.0;
  unsigned long long small = 0;
  std::vector<T> wgt_t;
  for (size_t k = 0; k < planes; k++) {
    auto t0 = std::chrono::steady_clock::now();
    Inputs in;
    in.wgt_kind = sizeof(T) == 4 ? WGT_F32 : WGT_F64;
    if (ex) {
      k_gram_node_weights<T><<<gblocks(nvis), 256, 0, s>>>(nrow, (uint32_t)nchan, wgt_dev, aw.as<double>(),
                                                           foc.as<double>(), table.as<double>(), (uint32_t)stencil, wmin,
                                                           op->dw, cells, (uint32_t)k, plane_wgt.as<T>(),
                                                           active.as<unsigned long long>());
      check_cuda(cudaGetLastError(), "node weights");
      in.vis = unit.get();
      in.vis_kind = VIS_C64;
    } else {
      // no_w (gridder_gram.rs:415-486): the weights as given, the PSF.
      if (sizeof(T) == 8) {
        check_cuda(cudaMemcpyAsync(plane_wgt.get(), wgt_dev, nvis * 8, cudaMemcpyDeviceToDevice, s), "copy");
      } else {
        std::vector<double> wd(nvis);
        check_cuda(cudaMemcpyAsync(wd.data(), wgt_dev, nvis * 8, cudaMemcpyDeviceToHost, s), "copy");
        check_cuda(cudaStreamSynchronize(s), "copy");
        wgt_t.resize(nvis);
        for (size_t i = 0; i < nvis; i++) wgt_t[i] = (T)wd[i];
        check_cuda(cudaMemcpyAsync(plane_wgt.get(), wgt_t.data(), nvis * sizeof(T), cudaMemcpyHostToDevice, s), "copy");
        check_cuda(cudaStreamSynchronize(s), "copy");
      }
    }
    in.wgt = plane_wgt.get();
    {
      Plan<T> p(g, nrow, nchan, ex ? fuvw.as<double>() : uvw_dev, freq, in, ex != nullptr, s);
      if (p.empty())
        check_cuda(cudaMemsetAsync(dirty.get(), 0, total * sizeof(T), s), "memset");
      else
        p.grid(in, ex ? VALUE_DATA : VALUE_UNIT, dirty.as<T>(), s);
      check_cuda(cudaStreamSynchronize(s), "gram grid");
    }
    auto t1 = std::chrono::steady_clock::now();
    k_gram_kgrid<T><<<gblocks(total), 256, 0, s>>>(dirty.as<T>(), (int)n, ex ? 0 : 1,
                                                  op->work.template as<cplx<T>>(), op->psf.template as<double>());
    check_cuda(cudaGetLastError(), "K grid");
    op->push_spectrum(s, &hermitian, &small);
    auto t2 = std::chrono::steady_clock::now();
    grid_sec += std::chrono::duration<double>(t1 - t0).count();
    fft_sec += std::chrono::duration<double>(t2 - t1).count();
  }
  unsigned long long act = 0;
  check_cuda(cudaMemcpyAsync(&act, active.get(), 8, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "gram setup");
  double* st = op->stats;
  st[0] = (double)planes;
  st[1] = ex ? (double)stencil : 0.0;
  st[2] = ex ? ex->theta : 0.0;
  st[3] = ex ? wmin : 0.0;
  st[4] = ex ? wmax : 0.0;
  st[5] = ex ? x_range : 0.0;
  st[6] = ex ? ex->sup_error : 0.0;
  st[7] = ex ? ex->lebesgue : 0.0;
  st[8] = (double)act;
  st[9] = (double)(planes * total * sizeof(T));
  st[10] = grid_sec;
  st[11] = fft_sec;
  st[12] = ex ? (double)small / (double)(planes * total) : 0.0;
  st[13] = ex ? hermitian : 0.0;
  return op;
}

}  // namespace wg

using namespace wg;

struct RangGram {
  std::unique_ptr<GramOpBase> op;
};

namespace wg {
// Status mapping and the per-thread message, shared with the gridder's ABI.
int32_t status_guarded(const std::function<void()>& f);
cudaStream_t stream_of(void* stream);
}  // namespace wg

extern "C" {

int32_t rang_b200_gram_expansion(size_t stencil, double theta, double ridge, double* table, double* sup_error,
                                 double* lebesgue) {
  return status_guarded([&] {
    WExpansionHost ex(stencil, theta, ridge);
    if (table) std::memcpy(table, ex.table.data(), ex.table.size() * sizeof(double));
    if (sup_error) *sup_error = ex.sup_error;
    if (lebesgue) *lebesgue = ex.lebesgue;
  });
}

int32_t rang_b200_gram_create(const WgridderOptions* opts, size_t nrow, size_t nchan, const double* uvw_dev,
                              const double* freq_host, const double* wgt_dev, size_t stencil, double theta,
                              double ridge, double epsilon, int32_t single, int32_t no_w, void* stream,
                              RangGram** out, double* stats) {
  if (!opts || !out) return 1;
  *out = nullptr;
  return status_guarded([&] {
    cudaStream_t s = stream_of(stream);
    std::unique_ptr<WExpansionHost> ex;
    if (!no_w) ex = std::make_unique<WExpansionHost>(stencil, theta, ridge);
    auto g = std::make_unique<RangGram>();
    if (single)
      g->op = gram_create<float>(*opts, nrow, nchan, uvw_dev, freq_host, wgt_dev, ex.get(), epsilon, s);
    else
      g->op = gram_create<double>(*opts, nrow, nchan, uvw_dev, freq_host, wgt_dev, ex.get(), epsilon, s);
    if (stats) std::memcpy(stats, g->op->stats, sizeof(g->op->stats));
    *out = g.release();
  });
}

int32_t rang_b200_gram_apply(RangGram* op, const double* m_dev, double* out_dev, void* stream) {
  if (!op || !m_dev || !out_dev) return 1;
  return status_guarded([&] { op->op->apply(m_dev, out_dev, stream_of(stream)); });
}

int32_t rang_b200_gram_inverse_filter(const RangGram* op, double rho, void* stream, RangGram** out) {
  if (!op || !out) return 1;
  *out = nullptr;
  return status_guarded([&] {
    auto g = std::make_unique<RangGram>();
    g->op = op->op->inverse_filter(rho, stream_of(stream));
    *out = g.release();
  });
}

int32_t rang_b200_gram_psf_no_w(const RangGram* op, double* out_dev, void* stream) {
  if (!op || !out_dev) return 1;
  return status_guarded([&] {
    const size_t big = 2 * (size_t)op->op->n;
    cudaStream_t s = stream_of(stream);
    if (!op->op->psf_no_w()) throw InvalidArgument("no PSF kept by this operator");
    check_cuda(cudaMemcpyAsync(out_dev, op->op->psf_no_w(), big * big * sizeof(double), cudaMemcpyDeviceToDevice, s),
               "copy");
  });
}

int32_t rang_b200_gram_planes(const RangGram* op) { return op ? (int32_t)op->op->stats[0] : 0; }

void rang_b200_gram_destroy(RangGram* op) { delete op; }

}  // extern "C"
