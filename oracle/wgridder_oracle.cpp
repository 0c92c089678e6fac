// CPU ORACLE — test infrastructure only, never shipped or called by the product.
//
// A restatement in C++ (OpenMP) of the reference's exact w-gridder
// `core/src/wgridder.rs` (rang-core, itself a port of ducc0 0.42.0's
// wgridder). Only the tests, the smoke check and the benchmark's CPU-baseline
// leg load it. It follows the reference function by function; every function
// names the reference lines it restates. Floating-point operations are
// written in the reference's order, with `std::fma` exactly where the
// reference uses `mul_add`, and the file is compiled with
// `-ffp-contract=off` so that no other multiply-add is fused. The FFT is this
// file's own mixed-radix Stockham transform (the reference uses rustfft), so
// results agree with the reference to rounding, not bit for bit.
//
// Parity pins (checked by tests/test_oracle.py): the kernel table digest and
// rows, good_size_complex values, the Gauss-Legendre and kernel-approximation
// known answers, DFT agreement at the reference's tolerances, adjointness,
// and the golden DFT vectors under tests/golden/.

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include <omp.h>

namespace {

constexpr double PI = 3.14159265358979323846;
constexpr double C_LIGHT = 299792458.0;  // wgridder.rs:58
constexpr size_t COST_VLEN = 8;          // wgridder.rs:62
constexpr size_t N_INFO = 14;            // wgridder.rs:490
constexpr size_t CHUNK = 2048;           // wgridder.rs:1962

struct KernelRowData {
  int w;
  double ofactor, epsilon, beta, e0;
  int ndim;
  int single;
};

const KernelRowData KERNEL_ROWS[] = {
#include "../rang-core_b200/csrc/kernel_db.inc"
};
constexpr size_t N_KERNEL_ROWS = sizeof(KERNEL_ROWS) / sizeof(KERNEL_ROWS[0]);

thread_local std::string g_last_error;

struct Error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// ---------------------------------------------------------------- kernels

// wgridder.rs:154-181 getAvailableKernels
std::vector<size_t> available_kernels(double epsilon, size_t ndim, bool single,
                                      double ofmin, double ofmax) {
  size_t wlim = single ? 8 : 16;
  double ofc[20];
  size_t idx[20];
  for (int i = 0; i < 20; i++) {
    ofc[i] = ofmax;
    idx[i] = SIZE_MAX;
  }
  for (size_t i = 0; i < N_KERNEL_ROWS; i++) {
    const KernelRowData& r = KERNEL_ROWS[i];
    if ((size_t)r.ndim == ndim && (r.single != 0) == single && (size_t)r.w <= wlim &&
        r.epsilon <= epsilon && r.ofactor <= ofc[r.w] && r.ofactor >= ofmin) {
      ofc[r.w] = r.ofactor;
      idx[r.w] = i;
    }
  }
  std::vector<size_t> res;
  for (int i = 0; i < 20; i++)
    if (idx[i] != SIZE_MAX) res.push_back(idx[i]);
  if (res.empty()) throw Error("no appropriate kernel for this epsilon, sigma range and precision");
  return res;
}

// wgridder.rs:185-222 good_size_cmplx
size_t good_size_complex(size_t n) {
  if (n <= 12) return n;
  size_t best = 2 * n;
  for (size_t f11 = 1; f11 < best; f11 *= 11)
    for (size_t f117 = f11; f117 < best; f117 *= 7)
      for (size_t f1175 = f117; f1175 < best; f1175 *= 5) {
        size_t x = f1175;
        while (x < n) x *= 2;
        for (;;) {
          if (x < n) {
            x *= 3;
          } else if (x > n) {
            if (x < best) best = x;
            if (x & 1) break;
            x >>= 1;
          } else {
            return n;
          }
        }
      }
  return best;
}

// wgridder.rs:225-232 esknew
double es_kernel(double v, double beta, double e0) {
  double tmp = (1.0 - v) * (1.0 + v);
  if (tmp >= 0.0) return std::exp(beta * (std::pow(tmp, e0) - 1.0));
  return 0.0;
}

// wgridder.rs:237-272
void gauss_legendre_symmetric(size_t n, std::vector<double>& x, std::vector<double>& w) {
  size_t m = (n + 1) / 2;
  x.assign(m, 0.0);
  w.assign(m, 0.0);
  for (size_t i = 0; i < m; i++) {
    double z = std::cos(PI * ((double)i + 0.75) / ((double)n + 0.5));
    double pp = 0.0;
    for (int iter = 0; iter < 100; iter++) {
      double p1 = 1.0, p2 = 0.0;
      for (size_t j = 1; j <= n; j++) {
        double p3 = p2;
        p2 = p1;
        p1 = ((double)(2 * j - 1) * z * p2 - (double)(j - 1) * p3) / (double)j;
      }
      pp = (double)n * (z * p1 - p2) / (z * z - 1.0);
      double dz = p1 / pp;
      z -= dz;
      if (std::fabs(dz) <= 1e-16 * std::max(std::fabs(z), 1.0) && iter > 0) break;
    }
    size_t k = m - 1 - i;
    x[k] = z;
    w[k] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
  if (n % 2 == 1) {
    x[0] = 0.0;
    w[0] *= 0.5;
  }
  for (auto& v : w) v *= 2.0;
}

// wgridder.rs:359-412 FunctionApproximator::getCoeffs
std::vector<double> approximate(size_t w, size_t d, double beta, double e0) {
  double lo = -1.0, hi = 1.0;
  std::vector<double> coeff(w * (d + 1), 0.0);
  std::vector<double> chebroot(d + 1);
  for (size_t i = 0; i <= d; i++)
    chebroot[i] = std::cos((double)(2 * i + 1) * PI / (double)(2 * d + 2));
  std::vector<double> cmat((d + 1) * (d + 1), 0.0);
  cmat[0] = 1.0;
  if (d >= 1) cmat[(d + 1) + 1] = 1.0;
  for (size_t j = 2; j <= d; j++) {
    cmat[j * (d + 1)] = -cmat[(j - 2) * (d + 1)];
    for (size_t k = 1; k <= j; k++)
      cmat[j * (d + 1) + k] = 2.0 * cmat[(j - 1) * (d + 1) + k - 1] - cmat[(j - 2) * (d + 1) + k];
  }
  for (size_t i = 0; i < w; i++) {
    double l = -1.0 + 2.0 * (double)i / (double)w;
    double r = -1.0 + 2.0 * (double)(i + 1) / (double)w;
    std::vector<double> y(d + 1);
    for (size_t k = 0; k <= d; k++) {
      double c = chebroot[k];
      double loc = ((c * (r - l) * 0.5 + (r + l) * 0.5) + 1.0) * 0.5 * (hi - lo) + lo;
      y[k] = es_kernel(loc, beta, e0);
    }
    double sum = 0.0;
    for (double v : y) sum += v;
    double avg = sum / (double)(d + 1);
    for (double& v : y) v -= avg;
    std::vector<double> lcf(d + 1, 0.0);
    for (size_t j = 0; j <= d; j++)
      for (size_t k = 0; k <= d; k++)
        lcf[j] += 2.0 / (double)(d + 1) * y[k] *
                  std::cos((double)(j * (2 * k + 1)) * PI / (double)(2 * d + 2));
    lcf[0] *= 0.5;
    std::vector<double> lcf2(d + 1, 0.0);
    for (size_t j = 0; j <= d; j++)
      for (size_t k = 0; k <= d; k++) lcf2[k] += cmat[j * (d + 1) + k] * lcf[j];
    lcf2[0] += avg;
    for (size_t j = 0; j <= d; j++) coeff[i * (d + 1) + j] = lcf2[d - j];
  }
  return coeff;
}

// wgridder.rs:277-356 EsKernel
struct EsKernel {
  size_t index = 0, support = 0, degree = 0;
  double beta = 0, e0 = 0;
  std::vector<double> coeff, corr_x, corr_w;

  explicit EsKernel(size_t idx) {
    if (idx >= N_KERNEL_ROWS) throw Error("kernel index out of range");
    const KernelRowData& row = KERNEL_ROWS[idx];
    index = idx;
    support = (size_t)row.w;
    beta = row.beta * (double)support;
    e0 = row.e0;
    degree = support + 3;
    coeff = approximate(support, degree, beta, e0);
    size_t p = (size_t)(1.5 * (double)support) + 2;
    gauss_legendre_symmetric(2 * p, corr_x, corr_w);
    for (size_t i = 0; i < corr_x.size(); i++) {
      corr_w[i] *= es_kernel(corr_x[i], beta, e0) * (double)support * 0.5;
      corr_x[i] *= PI * (double)support;
    }
  }
  double phi(double v) const { return es_kernel(v, beta, e0); }
  double eval(double v) const {
    if (std::fabs(v) >= 1.0) return 0.0;
    size_t w = support;
    double xrel = (double)w * 0.5 * (v + 1.0);
    size_t nth = std::min((size_t)xrel, w - 1);
    double locx = ((xrel - (double)nth) - 0.5) * 2.0;
    const double* c = &coeff[nth * (degree + 1)];
    double res = c[0];
    for (size_t i = 1; i <= degree; i++) res = res * locx + c[i];
    return res;
  }
  double corfunc(double v) const {
    double tmp = 0.0;
    for (size_t i = 0; i < corr_x.size(); i++) tmp += corr_w[i] * std::cos(corr_x[i] * v);
    return 1.0 / tmp;
  }
  std::vector<double> corfunc_table(size_t n, double dx) const {
    std::vector<double> out(n);
    for (size_t i = 0; i < n; i++) out[i] = corfunc((double)i * dx);
    return out;
  }
};

// ---------------------------------------------------------------- options

struct WgridderOptions {  // ffi_wgridder.rs:24-42
  size_t nx, ny;
  double pixsize_x, pixsize_y, epsilon, center_x, center_y, sigma_min, sigma_max;
  int32_t do_wgridding, divide_by_n, flip_u, flip_v, flip_w, allow_nshift;
  int64_t kernel_index;
  size_t nu, nv;
};

struct Plan {  // wgridder.rs:471-511
  size_t kernel_index = 0, supp = 0, nu = 0, nv = 0, nplanes = 0, nvis = 0;
  double wmin_d = 0, wmax_d = 0, nm1min = 0, nm1max = 0, nshift = 0, dw = 0, wmin = 0,
         ofactor = 0;
  void to_array(double* o) const {
    double a[N_INFO] = {(double)kernel_index, (double)supp, (double)nu, (double)nv,
                        (double)nplanes,      (double)nvis, wmin_d,      wmax_d,
                        nm1min,               nm1max,       nshift,      dw,
                        wmin,                 ofactor};
    std::memcpy(o, a, sizeof(a));
  }
};

template <class T>
struct Traits;
template <>
struct Traits<float> {
  static constexpr bool SINGLE = true;
  static constexpr size_t WMAX = 8;
  static constexpr unsigned LOG2TILE = 5;
};
template <>
struct Traits<double> {
  static constexpr bool SINGLE = false;
  static constexpr size_t WMAX = 16;
  static constexpr unsigned LOG2TILE = 4;
};

// ---------------------------------------------------------------- inputs

enum VisKind { VIS_UNIT = 0, VIS_C64 = 1, VIS_C128 = 2 };
enum WgtKind { WGT_NONE = 0, WGT_F32 = 1, WGT_F64 = 2, WGT_F32_PRODUCT = 3 };

struct VisData {  // wgridder.rs:934-967
  int kind = VIS_UNIT;
  const void* p = nullptr;
  template <class T>
  std::complex<T> get(size_t i) const {
    if (kind == VIS_C64) {
      const float* f = (const float*)p;
      return {(T)(double)f[2 * i], (T)(double)f[2 * i + 1]};
    }
    if (kind == VIS_C128) {
      const double* f = (const double*)p;
      return {(T)f[2 * i], (T)f[2 * i + 1]};
    }
    return {(T)1, (T)0};
  }
};

struct Weights {  // wgridder.rs:975-1019
  int kind = WGT_NONE;
  const void* a = nullptr;
  const void* b = nullptr;
  bool has() const { return kind != WGT_NONE; }
  template <class T>
  T get(size_t i) const {
    switch (kind) {
      case WGT_F32:
        return (T)(double)((const float*)a)[i];
      case WGT_F64:
        return (T)((const double*)a)[i];
      case WGT_F32_PRODUCT: {
        float x = ((const float*)a)[i] * ((const float*)b)[i];
        return (T)(double)x;
      }
      default:
        return (T)1;
    }
  }
};

struct Activity {  // wgridder.rs:1025-1042
  bool has_vis = false;
  VisData vis;
  Weights wgt;
  const uint8_t* mask = nullptr;
  template <class T>
  bool active(size_t idx) const {
    double tnorm = 1.0;
    if (has_vis) {
      std::complex<T> v = vis.get<T>(idx);
      T n = v.real() * v.real() + v.imag() * v.imag();
      tnorm = (double)n;
    }
    double twgt = wgt.has() ? (double)wgt.get<T>(idx) : 1.0;
    double tmask = mask ? (double)mask[idx] : 1.0;
    return tnorm * twgt * tmask != 0.0;
  }
};

// ---------------------------------------------------------------- geometry

struct Baselines {  // wgridder.rs:547-580
  std::vector<double> coord;  // 3 per row
  std::vector<double> f_over_c;
  Baselines(const double* uvw, size_t nrow, const double* freq, size_t nchan, const bool flips[3],
            double r_l, double r_m) {
    if (nchan == 0 || freq[0] <= 0.0) throw Error("channel frequencies must be positive");
    for (size_t i = 1; i < nchan; i++)
      if (freq[i] < freq[i - 1]) throw Error("channel frequencies must be sorted in ascending order");
    double fu = flips[0] ? -1.0 : 1.0, fv = flips[1] ? -1.0 : 1.0, fw = flips[2] ? -1.0 : 1.0;
    coord.resize(3 * nrow);
    for (size_t r = 0; r < nrow; r++) {
      double tu = fu * uvw[3 * r], tv = fv * uvw[3 * r + 1], tw = fw * uvw[3 * r + 2];
      coord[3 * r] = tu + r_l * tw;
      coord[3 * r + 1] = tv + r_m * tw;
      coord[3 * r + 2] = tw;
    }
    f_over_c.resize(nchan);
    for (size_t i = 0; i < nchan; i++) f_over_c[i] = freq[i] / C_LIGHT;
  }
  size_t nchan() const { return f_over_c.size(); }
  size_t nrow() const { return coord.size() / 3; }
};

// wgridder.rs:583-586 FixW
inline double fix_w(const double* c, double out[3]) {
  double res = 1.0 - 2.0 * (double)(c[2] < 0.0 ? 1 : 0);
  out[0] = c[0] * res;
  out[1] = c[1] * res;
  out[2] = c[2] * res;
  return res;
}

// wgridder.rs:589-599
double nm1_of(double x, double y, double r_l, double r_m) {
  double xsq = x * x, ysq = y * y;
  double tmp = 1.0 - xsq - ysq;
  double nm1 = tmp >= 0.0 ? (-xsq - ysq) / (std::sqrt(tmp) + 1.0) : -std::sqrt(-tmp) - 1.0;
  return nm1 + r_l * x + r_m * y;
}

struct Setup;
template <class T>
std::pair<size_t, std::pair<size_t, size_t>> choose_kernel(const WgridderOptions& o, size_t nvis,
                                                           double wmin_d, double wmax_d,
                                                           double nm1min, double nm1max,
                                                           double nshift);

struct Setup {  // wgridder.rs:516-544, 601-872
  size_t nx, ny;
  double pixsize_x, pixsize_y, lshift, mshift;
  bool lmshift, shifting;
  double r_l, r_m, nshift;
  bool do_wgridding, divide_by_n;
  size_t nu, nv, supp;
  double ushift, vshift;
  int64_t maxiu0, maxiv0;
  EsKernel kernel{0};
  size_t nplanes;
  double wmin, dw, xdw, wshift;
  Plan plan;

  template <class T>
  static Setup make(const WgridderOptions& o, size_t nvis, double wmin_d, double wmax_d,
                    double r_l, double r_m) {
    Setup s;
    s.nx = o.nx;
    s.ny = o.ny;
    double px = o.pixsize_x, py = o.pixsize_y;
    s.pixsize_x = px;
    s.pixsize_y = py;
    s.lshift = o.flip_u ? -o.center_x : o.center_x;
    s.mshift = o.flip_v ? -o.center_y : o.center_y;
    s.lmshift = s.lshift != 0.0 || s.mshift != 0.0;
    double xmin = s.lshift - 0.5 * (double)s.nx * px;
    double xmax = xmin + ((double)s.nx - 1.0) * px;
    double ymin = s.mshift - 0.5 * (double)s.ny * py;
    double ymax = ymin + ((double)s.ny - 1.0) * py;
    std::vector<double> xext{xmin, xmax}, yext{ymin, ymax};
    if (r_l != 0.0 || r_m != 0.0) {
      xext.push_back(s.lshift);
      yext.push_back(s.mshift);
    } else {
      if (xmin * xmax < 0.0) xext.push_back(0.0);
      if (ymin * ymax < 0.0) yext.push_back(0.0);
    }
    double nm1min = 1e300, nm1max = -1e300;
    for (double xc : xext)
      for (double yc : yext) {
        double tmp = xc * xc + yc * yc;
        double nval = tmp <= 1.0 ? std::sqrt(1.0 - tmp) - 1.0 : -std::sqrt(tmp - 1.0) - 1.0;
        nval += r_l * xc + r_m * yc;
        nm1min = std::min(nm1min, nval);
        nm1max = std::max(nm1max, nval);
      }
    bool wgrid = o.do_wgridding != 0;
    s.nshift = (!o.allow_nshift || !wgrid) ? 0.0 : -0.5 * (nm1max + nm1min);
    s.shifting = s.lmshift || s.nshift != 0.0;
    size_t kidx, nu, nv;
    if (o.kernel_index >= 0) {
      if ((size_t)o.kernel_index >= N_KERNEL_ROWS) throw Error("kernel index out of range");
      if ((size_t)KERNEL_ROWS[o.kernel_index].w > Traits<T>::WMAX)
        throw Error("kernel support too large for this precision");
      kidx = (size_t)o.kernel_index;
      nu = o.nu;
      nv = o.nv;
    } else {
      auto c = choose_kernel<T>(o, nvis, wmin_d, wmax_d, nm1min, nm1max, s.nshift);
      kidx = c.first;
      nu = c.second.first;
      nv = c.second.second;
    }
    if ((nu >> 4) >= (1u << 16) || (nv >> 4) >= (1u << 16)) throw Error("grid too large");
    s.kernel = EsKernel(kidx);
    size_t supp = s.kernel.support;
    size_t nsafe = (supp + 1) / 2;
    if (nu < 2 * nsafe || nv < 2 * nsafe) throw Error("grid too small");
    if (s.nx % 2 != 0 || s.ny % 2 != 0 || nu % 2 != 0 || nv % 2 != 0)
      throw Error("image and grid sizes must be even");
    double ofactor = std::min((double)nu / (double)s.nx, (double)nv / (double)s.ny);
    s.ushift = (double)supp * (-0.5) + 1.0 + (double)nu;
    s.vshift = (double)supp * (-0.5) + 1.0 + (double)nv;
    s.maxiu0 = (int64_t)(nu + nsafe) - (int64_t)supp;
    s.maxiv0 = (int64_t)(nv + nsafe) - (int64_t)supp;
    if (wgrid) {
      double dw = 0.5 / ofactor / std::max(std::fabs(nm1max + s.nshift), std::fabs(nm1min + s.nshift));
      double xdw = 1.0 / dw;
      double npl = (wmax_d - wmin_d) / dw + (double)supp;
      size_t nplanes = npl >= 0 ? (size_t)npl : 0;
      if (nplanes >= (1u << 16)) throw Error("too many w planes");
      double wmin = (wmin_d + wmax_d) * 0.5 - 0.5 * ((double)nplanes - 1.0) * dw;
      double wshift = dw - (0.5 * (double)supp * dw) - wmin;
      s.nplanes = nplanes;
      s.wmin = wmin;
      s.dw = dw;
      s.xdw = xdw;
      s.wshift = wshift;
    } else {
      s.nplanes = 0;
      s.wmin = s.dw = s.xdw = s.wshift = 0.0;
    }
    s.r_l = r_l;
    s.r_m = r_m;
    s.do_wgridding = wgrid;
    s.divide_by_n = o.divide_by_n != 0;
    s.nu = nu;
    s.nv = nv;
    s.supp = supp;
    Plan& p = s.plan;
    p.kernel_index = kidx;
    p.supp = supp;
    p.nu = nu;
    p.nv = nv;
    p.nplanes = s.nplanes;
    p.nvis = nvis;
    p.wmin_d = wmin_d;
    p.wmax_d = wmax_d;
    p.nm1min = nm1min;
    p.nm1max = nm1max;
    p.nshift = s.nshift;
    p.dw = s.dw;
    p.wmin = s.wmin;
    p.ofactor = ofactor;
    return s;
  }

  // wgridder.rs:757-767
  void getpix(double uin, double vin, double& uf, double& vf, int64_t& iu0, int64_t& iv0) const {
    double u = uin * pixsize_x;
    u = (u - std::floor(u)) * (double)nu;
    iu0 = std::min((int64_t)(u + ushift) - (int64_t)nu, maxiu0);
    u -= (double)iu0;
    double v = vin * pixsize_y;
    v = (v - std::floor(v)) * (double)nv;
    iv0 = std::min((int64_t)(v + vshift) - (int64_t)nv, maxiv0);
    v -= (double)iv0;
    uf = u;
    vf = v;
  }
  // wgridder.rs:770-776
  size_t minplane(double w) const {
    if (!do_wgridding) return 0;
    // f64::max ignores NaN; `as usize` saturates.
    double t = std::fmax((w + wshift) * xdw, 0.0);
    return t >= 18446744073709551615.0 ? SIZE_MAX : (size_t)t;
  }
  double x0() const { return lshift - 0.5 * (double)nx * pixsize_x; }
  double y0() const { return mshift - 0.5 * (double)ny * pixsize_y; }
  // wgridder.rs:788-803
  void table_dims(size_t& tnx, size_t& tny) const {
    if (lmshift) {
      tnx = nx;
      tny = ny;
    } else {
      tnx = nx / 2 + 1;
      tny = ny / 2 + 1;
    }
  }
  size_t table_index(size_t i, size_t j, size_t tny) const {
    if (lmshift) return i * tny + j;
    return std::min(i, nx - i) * tny + std::min(j, ny - j);
  }
  // wgridder.rs:806-818
  std::vector<double> screen_table() const {
    size_t tnx, tny;
    table_dims(tnx, tny);
    double xx0 = x0(), yy0 = y0();
    std::vector<double> out(tnx * tny);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < tnx; i++) {
      double x = xx0 + (double)i * pixsize_x;
      for (size_t j = 0; j < tny; j++) {
        double y = yy0 + (double)j * pixsize_y;
        out[i * tny + j] = nm1_of(x, y, r_l, r_m) + nshift;
      }
    }
    return out;
  }
  // wgridder.rs:822-861
  std::vector<double> global_corrections() const {
    size_t tnx, tny;
    table_dims(tnx, tny);
    std::vector<double> cfu = kernel.corfunc_table(nx / 2 + 1, 1.0 / (double)nu);
    std::vector<double> cfv = kernel.corfunc_table(ny / 2 + 1, 1.0 / (double)nv);
    double xx0 = x0(), yy0 = y0();
    std::vector<double> out(tnx * tny);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < tnx; i++) {
      double x = xx0 + (double)i * pixsize_x;
      double xsq = x * x;
      size_t iu = nx / 2 - std::min(i, nx - i);
      for (size_t j = 0; j < tny; j++) {
        double y = yy0 + (double)j * pixsize_y;
        double ysq = y * y;
        double tmp = 1.0 - xsq - ysq;
        double fct;
        if (tmp >= 0.0) {
          double nm1 = (-xsq - ysq) / (std::sqrt(tmp) + 1.0);
          double f = kernel.corfunc((nm1 + r_l * x + r_m * y + nshift) * dw);
          if (divide_by_n) f /= nm1 + 1.0;
          fct = f;
        } else if (divide_by_n) {
          fct = 0.0;
        } else {
          fct = kernel.corfunc((-std::sqrt(-tmp) - 1.0 + nshift) * dw);
        }
        size_t iv = ny / 2 - std::min(j, ny - j);
        fct *= cfu[iu] * cfv[iv];
        out[i * tny + j] = fct;
      }
    }
    return out;
  }
};

// wgridder.rs:876-926 getNuNv with one thread
template <class T>
std::pair<size_t, std::pair<size_t, size_t>> choose_kernel(const WgridderOptions& o, size_t nvis,
                                                           double wmin_d, double wmax_d,
                                                           double nm1min, double nm1max,
                                                           double nshift) {
  size_t ndim = o.do_wgridding ? 3 : 2;
  std::vector<size_t> idx =
      available_kernels(o.epsilon, ndim, Traits<T>::SINGLE, o.sigma_min, o.sigma_max);
  const double NREF_FFT = 2048.0, COSTREF_FFT = 0.0693;
  size_t vlen = COST_VLEN;
  double mincost = 1e300;
  size_t bi = SIZE_MAX, bu = 0, bv = 0;
  for (size_t i : idx) {
    const KernelRowData& krn = KERNEL_ROWS[i];
    size_t supp = (size_t)krn.w;
    size_t nvec = (supp + vlen - 1) / vlen;
    double ofactor = krn.ofactor;
    size_t nu = std::max<size_t>(2 * good_size_complex((size_t)((double)o.nx * ofactor * 0.5) + 1), 16);
    size_t nv = std::max<size_t>(2 * good_size_complex((size_t)((double)o.ny * ofactor * 0.5) + 1), 16);
    double logterm = std::log((double)(nu * nv)) / std::log(NREF_FFT * NREF_FFT);
    double fftcost = (double)nu / NREF_FFT * (double)nv / NREF_FFT * logterm * COSTREF_FFT;
    double gridcost = 2.2e-10 * (double)nvis *
                      ((double)(supp * nvec * vlen) + (double)((2 * nvec + 1) * (supp + 3) * vlen));
    if (o.do_wgridding) {
      double dw = 0.5 / ofactor / std::max(std::fabs(nm1max + nshift), std::fabs(nm1min + nshift));
      double npl = (wmax_d - wmin_d) / dw + (double)supp;
      size_t nplanes = npl >= 0 ? (size_t)npl : 0;
      fftcost *= (double)nplanes;
      gridcost *= (double)supp;
    }
    double cost = fftcost + gridcost;
    if (cost < mincost) {
      mincost = cost;
      bi = i;
      bu = nu;
      bv = nv;
    }
  }
  return {bi, {bu, bv}};
}

// wgridder.rs:1080-1100
void recentring(const WgridderOptions& o, double& r_l, double& r_m) {
  double lshift = o.flip_u ? -o.center_x : o.center_x;
  double mshift = o.flip_v ? -o.center_y : o.center_y;
  r_l = r_m = 0.0;
  if (o.do_wgridding && (lshift != 0.0 || mshift != 0.0)) {
    double xext = std::fabs(lshift) + 0.5 * (double)o.nx * o.pixsize_x;
    double yext = std::fabs(mshift) + 0.5 * (double)o.ny * o.pixsize_y;
    if (xext * xext + yext * yext < 1.0) {
      double n0 = std::sqrt(1.0 - lshift * lshift - mshift * mshift);
      r_l = lshift / n0;
      r_m = mshift / n0;
    }
  }
}

// wgridder.rs:1102-1123
void check_common(const WgridderOptions& o, size_t nrow, size_t nchan) {
  if (o.nx == 0 || o.ny == 0) throw Error("image dimensions must be positive");
  if (std::isnan(o.epsilon) || o.epsilon <= 0.0) throw Error("epsilon must be positive");
  if (std::isnan(o.pixsize_x) || std::isnan(o.pixsize_y) || o.pixsize_x <= 0.0 || o.pixsize_y <= 0.0)
    throw Error("pixel sizes must be positive");
  if (nchan == 0) throw Error("uvw must have three values per row");
  if (nrow >= (1ull << 32) || nchan >= (1ull << 32)) throw Error("too many rows or channels");
}

// wgridder.rs:1051-1077
template <class T>
void scan(const Baselines& bl, const Activity& act, size_t& n, double& lo, double& hi) {
  size_t nchan = bl.nchan(), nrow = bl.nrow();
  size_t cnt = 0;
  double l = 1e300, h = -1e300;
#pragma omp parallel for reduction(+ : cnt) reduction(min : l) reduction(max : h) schedule(static)
  for (size_t row = 0; row < nrow; row++) {
    for (size_t ch = 0; ch < nchan; ch++) {
      if (act.active<T>(row * nchan + ch)) {
        cnt++;
        double w = std::fabs(bl.coord[3 * row + 2] * bl.f_over_c[ch]);
        l = std::min(l, w);
        h = std::max(h, w);
      }
    }
  }
  n = cnt;
  lo = l;
  hi = h;
}

// ---------------------------------------------------------------- layout

struct Tiling {  // wgridder.rs:1152-1173
  unsigned log2;
  size_t ntu, ntv, su, sv;
};
template <class T>
Tiling make_tiling(const Setup& s) {
  Tiling t;
  t.log2 = Traits<T>::LOG2TILE;
  size_t tile = (size_t)1 << t.log2;
  t.ntu = (s.nu + tile - 1) / tile;
  t.ntv = (s.nv + tile - 1) / tile;
  t.su = tile + s.supp - 1;
  t.sv = tile + s.supp - 1;
  return t;
}

inline size_t shifted(int64_t i0, size_t n) {  // wgridder.rs:1177-1179
  int64_t m = (int64_t)n;
  int64_t r = (i0 + m / 2) % m;
  if (r < 0) r += m;
  return (size_t)r;
}
inline size_t offset_in(int64_t i0, size_t n, size_t base) {  // wgridder.rs:1183-1192
  int64_t nn = (int64_t)n;
  int64_t d = i0 + nn / 2 - (int64_t)base;
  if (d < 0)
    d += nn;
  else if (d >= nn)
    d -= nn;
  return (size_t)d;
}

struct VisRef {
  uint32_t row, ch;
};
struct Block {
  size_t minplane, start, end;
};
struct Tile {
  size_t tu, tv, b0, b1, plo, phi;
  bool edge;
};
struct Layout {
  Tiling tiling;
  std::vector<VisRef> refs;
  std::vector<Block> blocks;
  std::vector<Tile> tiles;
};

inline void uvw_of(const Baselines& bl, VisRef r, double uvw[3], double& imflip) {  // :1137-1141
  double c[3];
  imflip = fix_w(&bl.coord[3 * (size_t)r.row], c);
  double f = bl.f_over_c[r.ch];
  uvw[0] = c[0] * f;
  uvw[1] = c[1] * f;
  uvw[2] = c[2] * f;
}

// wgridder.rs:1244-1255
inline void locate(const Setup& s, const Tiling& t, const Baselines& bl, size_t row, size_t ch,
                   size_t& tile, size_t& mp, int64_t* piu0 = nullptr, int64_t* piv0 = nullptr) {
  VisRef r{(uint32_t)row, (uint32_t)ch};
  double uvw[3], imflip;
  uvw_of(bl, r, uvw, imflip);
  double uf, vf;
  int64_t iu0, iv0;
  s.getpix(uvw[0], uvw[1], uf, vf, iu0, iv0);
  size_t tu = shifted(iu0, s.nu) >> t.log2;
  size_t tv = shifted(iv0, s.nv) >> t.log2;
  size_t nbuckets = std::max<size_t>(s.nplanes, 1);
  tile = tu * t.ntv + tv;
  mp = std::min(s.minplane(uvw[2]), nbuckets - 1);
  if (piu0) *piu0 = iu0;
  if (piv0) *piv0 = iv0;
}

// wgridder.rs:1261-1376: sorted by (tile, first plane, row, channel).
template <class T>
Layout layout(const Setup& s, const Baselines& bl, const Activity& act) {
  Layout lay;
  lay.tiling = make_tiling<T>(s);
  const Tiling& t = lay.tiling;
  size_t nrow = bl.nrow(), nchan = bl.nchan();
  size_t ntiles = t.ntu * t.ntv;
  size_t nb = std::max<size_t>(s.nplanes, 1);
  std::vector<size_t> counts(ntiles * nb + 1, 0);
  // Key of every visibility (or SIZE_MAX when inactive); counted serially.
  std::vector<uint64_t> key(nrow * nchan);
#pragma omp parallel for schedule(static)
  for (size_t row = 0; row < nrow; row++)
    for (size_t ch = 0; ch < nchan; ch++) {
      size_t idx = row * nchan + ch;
      if (act.active<T>(idx)) {
        size_t tile, mp;
        locate(s, t, bl, row, ch, tile, mp);
        key[idx] = (uint64_t)tile * nb + mp;
      } else {
        key[idx] = UINT64_MAX;
      }
    }
  for (size_t i = 0; i < key.size(); i++)
    if (key[i] != UINT64_MAX) counts[key[i] + 1]++;
  for (size_t i = 1; i <= ntiles * nb; i++) counts[i] += counts[i - 1];
  size_t total = counts[ntiles * nb];
  lay.refs.resize(total);
  std::vector<size_t> pos(counts.begin(), counts.end() - 1);
  for (size_t i = 0; i < key.size(); i++)
    if (key[i] != UINT64_MAX) {
      size_t p = pos[key[i]]++;
      lay.refs[p] = VisRef{(uint32_t)(i / nchan), (uint32_t)(i % nchan)};
    }
  for (size_t tile = 0; tile < ntiles; tile++) {
    size_t b0 = lay.blocks.size();
    for (size_t mp = 0; mp < nb; mp++) {
      size_t a = counts[tile * nb + mp], b = counts[tile * nb + mp + 1];
      if (b > a) lay.blocks.push_back(Block{mp, a, b});
    }
    if (lay.blocks.size() == b0) continue;
    Tile tl;
    tl.tu = tile / t.ntv;
    tl.tv = tile % t.ntv;
    tl.b0 = b0;
    tl.b1 = lay.blocks.size();
    tl.plo = lay.blocks[b0].minplane;
    tl.phi = lay.blocks.back().minplane;
    tl.edge = ((tl.tu << t.log2) + t.su > s.nu) || ((tl.tv << t.log2) + t.sv > s.nv);
    lay.tiles.push_back(tl);
  }
  return lay;
}

// ---------------------------------------------------------------- values

// wgridder.rs:1395-1408
template <class T>
std::complex<T> shift_phase(const Setup& s, const Baselines& bl, VisRef r, double sign) {
  double b[3];
  double imflip = fix_w(&bl.coord[3 * (size_t)r.row], b);
  double fct = sign * imflip * (b[0] * s.lshift + b[1] * s.mshift + b[2] * s.nshift);
  double tmp = fct * bl.f_over_c[r.ch];
  T ang;
  if (Traits<T>::SINGLE)
    ang = (T)(2.0 * PI * (tmp - std::floor(tmp)));
  else
    ang = (T)(2.0 * PI * tmp);
  return {std::cos(ang), std::sin(ang)};
}

template <class T>
inline std::complex<T> cmul(std::complex<T> a, std::complex<T> b) {
  return {a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real()};
}

// wgridder.rs:1414-1424
template <class T>
std::complex<T> unit_value(const Setup& s, const Baselines& bl, VisRef r, bool has_w, T w) {
  std::complex<T> v((T)1, (T)0);
  if (s.shifting) v = cmul(v, shift_phase<T>(s, bl, r, 1.0));
  if (has_w) v = {v.real() * w, v.imag() * w};
  double c[3];
  double imflip = fix_w(&bl.coord[3 * (size_t)r.row], c);
  return {v.real(), v.imag() * (T)imflip};
}

// wgridder.rs:1432-1435
template <class T>
std::complex<T> data_value(std::complex<T> v, std::complex<T> p, T imflip) {
  std::complex<T> d = cmul(v, std::complex<T>(p.real(), p.imag() * imflip));
  return {d.real(), d.imag() * imflip};
}

// wgridder.rs:1439-1475
template <class T>
void values(const Setup& s, const Baselines& bl, const std::vector<VisRef>& refs, bool has_data,
            VisData data, Weights wgt, std::vector<std::complex<T>>& out) {
  size_t nchan = bl.nchan();
  out.resize(refs.size());
#pragma omp parallel for schedule(static)
  for (size_t k = 0; k < refs.size(); k++) {
    VisRef r = refs[k];
    size_t idx = (size_t)r.row * nchan + r.ch;
    std::complex<T> p = unit_value<T>(s, bl, r, wgt.has(), wgt.get<T>(idx));
    if (has_data) {
      double c[3];
      double imflip = fix_w(&bl.coord[3 * (size_t)r.row], c);
      out[k] = data_value<T>(data.get<T>(idx), p, (T)imflip);
    } else {
      out[k] = p;
    }
  }
}

// ---------------------------------------------------------------- kernels

// wgridder.rs:1485-1507
template <class T>
std::vector<T> coeff_even_odd(const EsKernel& k) {
  size_t w = k.support, d = k.degree, d1 = d + 1, dodd = d | 1, ne = (dodd + 1) / 2;
  auto a = [&](size_t i, size_t m) { return m > d ? 0.0 : k.coeff[i * d1 + (d - m)]; };
  std::vector<T> out(2 * ne * w, (T)0);
  for (size_t i = 0; i < w; i++)
    for (size_t kk = 0; kk < ne; kk++) {
      out[kk * w + i] = (T)a(i, dodd - 1 - 2 * kk);
      out[(ne + kk) * w + i] = (T)a(i, dodd - 2 * kk);
    }
  return out;
}

// wgridder.rs:1514-1543
template <class T>
void eval_taps2(const T* c, size_t S, size_t ne, T x, T y, T* ru, T* rv) {
  size_t h = (S + 1) / 2;
  T x2 = x * x, y2 = y * y;
  T ex[16], ey[16], ox[16], oy[16];
  for (size_t i = 0; i < S; i++) {
    ex[i] = ey[i] = c[i];
    ox[i] = oy[i] = c[ne * S + i];
  }
  for (size_t k = 1; k < ne; k++) {
    const T* ce = c + k * S;
    const T* co = c + (ne + k) * S;
    for (size_t i = 0; i < h; i++) {
      ex[i] = std::fma(ex[i], x2, ce[i]);
      ey[i] = std::fma(ey[i], y2, ce[i]);
      ox[i] = std::fma(ox[i], x2, co[i]);
      oy[i] = std::fma(oy[i], y2, co[i]);
    }
  }
  for (size_t i = 0; i < h; i++) {
    ru[i] = std::fma(ox[i], x, ex[i]);
    rv[i] = std::fma(oy[i], y, ey[i]);
  }
  for (size_t i = 0; i < S - h; i++) {
    ru[S - 1 - i] = std::fma(ox[i], -x, ex[i]);
    rv[S - 1 - i] = std::fma(oy[i], -y, ey[i]);
  }
}

// wgridder.rs:1548-1560
template <class T>
T eval_tap(const T* c, size_t S, size_t ne, size_t i, T x) {
  size_t h = (S + 1) / 2;
  if (i >= h) {
    i = S - 1 - i;
    x = -x;
  }
  T x2 = x * x;
  T e = c[i], o = c[ne * S + i];
  for (size_t k = 1; k < ne; k++) {
    e = std::fma(e, x2, c[k * S + i]);
    o = std::fma(o, x2, c[(ne + k) * S + i]);
  }
  return std::fma(o, x, e);
}

// wgridder.rs:1580-1591
template <class T>
T w_factor(const Setup& s, const T* coeff, size_t ne, size_t nth, size_t p, double w) {
  size_t S = s.supp;
  double w0 = s.wmin + (double)p * s.dw;
  T z = (T)(s.xdw * (w0 - w));
  T locz = (z - (T)(double)nth) * (T)2.0 + (T)((double)S - 1.0);
  return eval_tap<T>(coeff, S, ne, nth, locz);
}

// ---------------------------------------------------------------- FFT

// Mixed-radix Stockham FFT (radices 2, 3, 4, 5, 7, 11 and any other prime by
// a direct DFT), unnormalised, sign -1 forward and +1 inverse as rustfft.
template <class T>
struct Fft {
  size_t n = 0;
  std::vector<size_t> radix;
  std::vector<std::vector<std::complex<T>>> tw_f, tw_i;  // per stage, k * R + r
  std::vector<std::vector<std::complex<T>>> root_f, root_i;

  explicit Fft(size_t n_) : n(n_) {
    size_t m = n;
    for (size_t r : {4, 2, 3, 5, 7, 11})
      while (m % r == 0 && !(r == 4 && m % 4 != 0)) {
        radix.push_back(r);
        m /= r;
      }
    for (size_t p = 13; m > 1; p++)
      while (m % p == 0) {
        radix.push_back(p);
        m /= p;
      }
    size_t ns = 1;
    for (size_t R : radix) {
      std::vector<std::complex<T>> tf(ns * R), ti(ns * R);
      for (size_t k = 0; k < ns; k++)
        for (size_t r = 0; r < R; r++) {
          double a = 2.0 * PI * (double)(r * k) / (double)(ns * R);
          tf[k * R + r] = {(T)std::cos(a), (T)-std::sin(a)};
          ti[k * R + r] = {(T)std::cos(a), (T)std::sin(a)};
        }
      tw_f.push_back(tf);
      tw_i.push_back(ti);
      std::vector<std::complex<T>> rf(R * R), ri(R * R);
      for (size_t a = 0; a < R; a++)
        for (size_t b = 0; b < R; b++) {
          double ang = 2.0 * PI * (double)((a * b) % R) / (double)R;
          rf[a * R + b] = {(T)std::cos(ang), (T)-std::sin(ang)};
          ri[a * R + b] = {(T)std::cos(ang), (T)std::sin(ang)};
        }
      root_f.push_back(rf);
      root_i.push_back(ri);
      ns *= R;
    }
  }

  // In place on `data`, `work` holds n values.
  void exec(std::complex<T>* data, std::complex<T>* work, bool inverse) const {
    if (n <= 1) return;
    std::complex<T>* a = data;
    std::complex<T>* b = work;
    size_t ns = 1;
    for (size_t st = 0; st < radix.size(); st++) {
      size_t R = radix[st];
      const auto& tw = inverse ? tw_i[st] : tw_f[st];
      const auto& rt = inverse ? root_i[st] : root_f[st];
      size_t nr = n / R;
      std::vector<std::complex<T>> v(R), y(R);
      for (size_t j = 0; j < nr; j++) {
        size_t k = j % ns;
        for (size_t r = 0; r < R; r++) v[r] = cmul(a[j + r * nr], tw[k * R + r]);
        if (R == 2) {
          y[0] = v[0] + v[1];
          y[1] = v[0] - v[1];
        } else if (R == 4) {
          std::complex<T> s02 = v[0] + v[2], d02 = v[0] - v[2];
          std::complex<T> s13 = v[1] + v[3], d13 = v[1] - v[3];
          // d13 times -i (forward) or +i (inverse)
          std::complex<T> rot = inverse ? std::complex<T>(-d13.imag(), d13.real())
                                        : std::complex<T>(d13.imag(), -d13.real());
          y[0] = s02 + s13;
          y[1] = d02 + rot;
          y[2] = s02 - s13;
          y[3] = d02 - rot;
        } else {
          for (size_t m = 0; m < R; m++) {
            std::complex<T> acc = v[0];
            for (size_t q = 1; q < R; q++) acc += cmul(v[q], rt[m * R + q]);
            y[m] = acc;
          }
        }
        size_t base = (j / ns) * ns * R + k;
        for (size_t m = 0; m < R; m++) b[base + m * ns] = y[m];
      }
      std::swap(a, b);
      ns *= R;
    }
    if (a != data) std::memcpy(data, a, n * sizeof(std::complex<T>));
  }
};

// ---------------------------------------------------------------- gridding

struct Tables {  // wgridder.rs:2500-2541 (the FFT plans live with the callers)
  std::vector<double> table, corr, cfu, cfv;
  std::vector<size_t> rows, cols, inv_rows;
};

Tables make_tables(const Setup& s) {
  Tables t;
  t.rows.resize(s.nx);
  for (size_t i = 0; i < s.nx; i++) t.rows[i] = (s.nu - s.nx / 2 + i) % s.nu;  // :1751-1755
  t.cols.resize(s.ny);
  for (size_t j = 0; j < s.ny; j++) t.cols[j] = (s.nv - s.ny / 2 + j) % s.nv;  // :1745-1749
  t.inv_rows.assign(s.nu, SIZE_MAX);
  for (size_t i = 0; i < s.nx; i++) t.inv_rows[t.rows[i]] = i;
  if (s.do_wgridding) {
    t.table = s.screen_table();
    t.corr = s.global_corrections();
  } else {
    t.cfu = s.kernel.corfunc_table(s.nx / 2 + 1, 1.0 / (double)s.nu);
    t.cfv = s.kernel.corfunc_table(s.ny / 2 + 1, 1.0 / (double)s.nv);
  }
  return t;
}

// wgridder.rs:1831-1847: the tiles active on plane p.
bool tile_active(const Setup& s, const Tile& t, size_t p) {
  return !s.do_wgridding || (t.plo <= p && p < t.phi + s.supp);
}

// wgridder.rs:1818-1827
std::vector<char> tile_rows(const Setup& s, const Layout& lay, size_t p) {
  std::vector<char> rows(s.nu, 0);
  for (const Tile& t : lay.tiles) {
    if (!tile_active(s, t, p)) continue;
    size_t base = t.tu << lay.tiling.log2;
    for (size_t i = 0; i < lay.tiling.su; i++) rows[(base + i + s.nu / 2) % s.nu] = 1;
  }
  return rows;
}

// wgridder.rs:2296-2314
template <class T>
void screen_par(const std::vector<double>& table, double w, bool adjoint,
                std::vector<std::complex<T>>& out) {
  out.resize(table.size());
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < table.size(); i++) {
    double phs = w * table[i];
    if (adjoint) phs *= -1.0;
    T ang;
    if (Traits<T>::SINGLE)
      ang = (T)(2.0 * PI * (phs - std::floor(phs)));
    else
      ang = (T)(2.0 * PI * phs);
    out[i] = {std::cos(ang), std::sin(ang)};
  }
}

template <class T>
struct Gridder {
  const Setup& s;
  const Baselines& bl;
  const Layout& lay;
  const Tables& tab;
  std::vector<T> coeff;
  size_t ne;
  Fft<T> fu, fv;

  Gridder(const Setup& s_, const Baselines& bl_, const Layout& lay_, const Tables& tab_)
      : s(s_), bl(bl_), lay(lay_), tab(tab_), fu(s_.nu), fv(s_.nv) {
    coeff = coeff_even_odd<T>(s.kernel);
    ne = coeff.size() / (2 * s.supp);
  }

  // wgridder.rs:1565-1576
  void taps_uv(double u, double v, T* ku, T* kv, int64_t& iu0, int64_t& iv0) const {
    double uf, vf;
    s.getpix(u, v, uf, vf, iu0, iv0);
    size_t S = s.supp;
    T x0 = (T)(-uf * 2.0 + ((double)S - 1.0));
    T y0 = (T)(-vf * 2.0 + ((double)S - 1.0));
    eval_taps2<T>(coeff.data(), S, ne, x0, y0, ku, kv);
  }

  // The tasks of tile `ti` on plane p (wgridder.rs:1974-2008, one plane).
  void tile_tasks(size_t ti, size_t p, std::vector<std::vector<std::array<size_t, 3>>>& tasks) const {
    const Tile& t = lay.tiles[ti];
    std::vector<std::array<size_t, 3>> cur;
    size_t n = 0;
    for (size_t bi = t.b0; bi < t.b1; bi++) {
      const Block& b = lay.blocks[bi];
      if (s.do_wgridding && !(b.minplane <= p && p < b.minplane + s.supp)) continue;
      size_t st = b.start;
      while (st < b.end) {
        size_t e = std::min(b.end, st + CHUNK - n);
        cur.push_back({b.minplane, st, e});
        n += e - st;
        st = e;
        if (n == CHUNK) {
          tasks.push_back(cur);
          cur.clear();
          n = 0;
        }
      }
    }
    if (n > 0) tasks.push_back(cur);
  }

  // Grid the tasks of tile `ti` on plane p into `grid` (wgridder.rs:2102-2156, 1904-1937).
  void grid_tile(size_t ti, size_t p, const std::vector<std::complex<T>>& stored, bool both,
                 VisData data, std::complex<T>* grid, std::complex<T>* grid2, std::vector<T>& br,
                 std::vector<T>& bi, std::vector<T>& br2, std::vector<T>& bi2) const {
    const Tile& t = lay.tiles[ti];
    const Tiling& tl = lay.tiling;
    size_t S = s.supp, su = tl.su, sv = tl.sv, nchan = bl.nchan();
    size_t bu = t.tu << tl.log2, bv = t.tv << tl.log2;
    std::vector<std::vector<std::array<size_t, 3>>> tasks;
    tile_tasks(ti, p, tasks);
    for (const auto& task : tasks) {
      std::fill(br.begin(), br.end(), (T)0);
      std::fill(bi.begin(), bi.end(), (T)0);
      if (both) {
        std::fill(br2.begin(), br2.end(), (T)0);
        std::fill(bi2.begin(), bi2.end(), (T)0);
      }
      for (const auto& run : task) {
        size_t mp = run[0];
        for (size_t k = run[1]; k < run[2]; k++) {
          VisRef r = lay.refs[k];
          double uvw[3], imflip;
          uvw_of(bl, r, uvw, imflip);
          T ku[16], kv[16];
          int64_t iu0, iv0;
          taps_uv(uvw[0], uvw[1], ku, kv, iu0, iv0);
          size_t ou = offset_in(iu0, s.nu, bu), ov = offset_in(iv0, s.nv, bv);
          std::complex<T> st = stored[k];
          std::complex<T> d;
          if (both) d = data_value<T>(data.get<T>((size_t)r.row * nchan + r.ch), st, (T)imflip);
          if (s.do_wgridding) {
            T kw = w_factor<T>(s, coeff.data(), ne, p - mp, p, uvw[2]);
            for (size_t i = 0; i < S; i++) ku[i] = ku[i] * kw;
          }
          auto acc = [&](std::vector<T>& rr, std::vector<T>& ii, std::complex<T> val) {
            for (size_t cu = 0; cu < S; cu++) {
              T tr = val.real() * ku[cu], tim = val.imag() * ku[cu];
              size_t base = (ou + cu) * sv + ov;
              for (size_t cv = 0; cv < S; cv++) rr[base + cv] = std::fma(tr, kv[cv], rr[base + cv]);
              for (size_t cv = 0; cv < S; cv++) ii[base + cv] = std::fma(tim, kv[cv], ii[base + cv]);
            }
          };
          if (both) {
            acc(br, bi, d);
            acc(br2, bi2, st);
          } else {
            acc(br, bi, st);
          }
        }
      }
      auto dump = [&](std::complex<T>* g, const std::vector<T>& rr, const std::vector<T>& ii) {
        for (size_t i = 0; i < su; i++)
          for (size_t j = 0; j < sv; j++) {
            size_t row = (bu + i + s.nu / 2) % s.nu, col = (bv + j + s.nv / 2) % s.nv;
            std::complex<T>& c = g[row * s.nv + col];
            c = {c.real() + rr[i * sv + j], c.imag() + ii[i * sv + j]};
          }
      };
      dump(grid, br, bi);
      if (both) dump(grid2, br2, bi2);
    }
  }

  // wgridder.rs:2163-2221 for one plane.
  void grid_plane(size_t p, const std::vector<std::complex<T>>& stored, bool both, VisData data,
                  std::complex<T>* grid, std::complex<T>* grid2) const {
    const Tiling& tl = lay.tiling;
    std::vector<size_t> classes[5];
    for (size_t i = 0; i < lay.tiles.size(); i++) {
      const Tile& t = lay.tiles[i];
      if (!tile_active(s, t, p)) continue;
      size_t c = t.edge ? 4 : (t.tu & 1) * 2 + (t.tv & 1);
      classes[c].push_back(i);
    }
    size_t nbuf = tl.su * tl.sv;
    for (int c = 0; c < 5; c++) {
      const auto& cls = classes[c];
      if (c == 4) {
        std::vector<T> br(nbuf), bi(nbuf), br2(nbuf), bi2(nbuf);
        for (size_t ti : cls) grid_tile(ti, p, stored, both, data, grid, grid2, br, bi, br2, bi2);
        continue;
      }
#pragma omp parallel
      {
        std::vector<T> br(nbuf), bi(nbuf), br2(nbuf), bi2(nbuf);
#pragma omp for schedule(dynamic, 1)
        for (size_t q = 0; q < cls.size(); q++)
          grid_tile(cls[q], p, stored, both, data, grid, grid2, br, bi, br2, bi2);
      }
    }
  }

  // wgridder.rs:2320-2399
  void grid_to_image(std::complex<T>* grid, const std::vector<char>& touched,
                     const std::vector<std::complex<T>>& screen, T* image) const {
    size_t nu = s.nu, nv = s.nv, ny = s.ny, nx = s.nx;
    size_t tnx, tny;
    s.table_dims(tnx, tny);
#pragma omp parallel
    {
      std::vector<std::complex<T>> work(std::max(nu, nv));
#pragma omp for schedule(static)
      for (size_t r = 0; r < nu; r++)
        if (touched[r]) fv.exec(grid + r * nv, work.data(), true);
    }
#pragma omp parallel
    {
      std::vector<std::complex<T>> col(nu), work(nu);
#pragma omp for schedule(static)
      for (size_t j = 0; j < ny; j++) {
        size_t jx = tab.cols[j];
        for (size_t r = 0; r < nu; r++) col[r] = touched[r] ? grid[r * nv + jx] : std::complex<T>(0, 0);
        fu.exec(col.data(), work.data(), true);
        for (size_t i = 0; i < nx; i++) {
          std::complex<T> g = col[tab.rows[i]];
          T term;
          if (s.do_wgridding) {
            std::complex<T> ph = screen[s.table_index(i, j, tny)];
            term = g.real() * ph.real() - g.imag() * ph.imag();
          } else {
            term = g.real();
          }
          image[i * ny + j] = image[i * ny + j] + term;
        }
      }
    }
  }

  // wgridder.rs:2403-2428
  void correct_image(T* image) const {
    size_t nx = s.nx, ny = s.ny, tnx, tny;
    s.table_dims(tnx, tny);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < nx; i++) {
      if (s.do_wgridding) {
        for (size_t j = 0; j < ny; j++) image[i * ny + j] = image[i * ny + j] * (T)tab.corr[s.table_index(i, j, tny)];
      } else {
        size_t iu = nx / 2 - std::min(i, nx - i);
        for (size_t j = 0; j < ny; j++) {
          size_t iv = ny / 2 - std::min(j, ny - j);
          image[i * ny + j] = (T)((double)image[i * ny + j] * tab.cfu[iu] * tab.cfv[iv]);
        }
      }
    }
  }

  // wgridder.rs:2584-2683 (plane group 1)
  void grid_images(const std::vector<std::complex<T>>& stored, bool both, VisData data, T* img1,
                   T* img2) const {
    size_t nu = s.nu, nv = s.nv;
    std::vector<std::complex<T>> g1((size_t)nu * nv), g2(both ? (size_t)nu * nv : 0);
    std::vector<std::complex<T>> screen;
    size_t nplanes = std::max<size_t>(s.nplanes, 1);
    for (size_t p = 0; p < nplanes; p++) {
      bool any = false;
      for (const Tile& t : lay.tiles)
        if (tile_active(s, t, p)) {
          any = true;
          break;
        }
      if (!any) continue;
      grid_plane(p, stored, both, data, g1.data(), both ? g2.data() : nullptr);
      std::vector<char> rows = tile_rows(s, lay, p);
      double w0 = s.wmin + (double)p * s.dw;
      if (s.do_wgridding) screen_par<T>(tab.table, w0, true, screen);
      grid_to_image(g1.data(), rows, screen, img1);
      if (both) grid_to_image(g2.data(), rows, screen, img2);
      std::fill(g1.begin(), g1.end(), std::complex<T>(0, 0));
      if (both) std::fill(g2.begin(), g2.end(), std::complex<T>(0, 0));
    }
    correct_image(img1);
    if (both) correct_image(img2);
  }

  // ------------------------------------------------------------ degridding

  // wgridder.rs:2908-2992
  void image_to_grid(const std::vector<T>& image, const std::vector<std::complex<T>>& screen,
                     const std::vector<char>& needed, std::complex<T>* grid) const {
    size_t nu = s.nu, nv = s.nv, ny = s.ny;
    size_t tnx, tny;
    s.table_dims(tnx, tny);
    std::fill(grid, grid + nu * nv, std::complex<T>(0, 0));
#pragma omp parallel
    {
      std::vector<std::complex<T>> col(nu), work(nu);
#pragma omp for schedule(static)
      for (size_t j = 0; j < ny; j++) {
        for (size_t r = 0; r < nu; r++) {
          size_t i = tab.inv_rows[r];
          if (i == SIZE_MAX) {
            col[r] = {0, 0};
            continue;
          }
          T d = image[i * ny + j];
          if (s.do_wgridding) {
            std::complex<T> ph = screen[s.table_index(i, j, tny)];
            col[r] = {d * ph.real(), d * ph.imag()};
          } else {
            col[r] = {d, (T)0};
          }
        }
        fu.exec(col.data(), work.data(), false);
        size_t jx = tab.cols[j];
        for (size_t r = 0; r < nu; r++)
          if (needed[r]) grid[r * nv + jx] = col[r];
      }
    }
#pragma omp parallel
    {
      std::vector<std::complex<T>> work(nv);
#pragma omp for schedule(static)
      for (size_t r = 0; r < nu; r++)
        if (needed[r]) fv.exec(grid + r * nv, work.data(), false);
    }
  }

  // wgridder.rs:2793-2901 for one plane; out in visibility order.
  void degrid_plane(size_t p, const std::complex<T>* grid, std::complex<T>* out) const {
    const Tiling& tl = lay.tiling;
    size_t S = s.supp, su = tl.su, sv = tl.sv, nchan = bl.nchan();
    std::vector<size_t> act;
    for (size_t i = 0; i < lay.tiles.size(); i++)
      if (tile_active(s, lay.tiles[i], p)) act.push_back(i);
#pragma omp parallel
    {
      std::vector<T> br(su * sv), bi(su * sv);
#pragma omp for schedule(dynamic, 1)
      for (size_t q = 0; q < act.size(); q++) {
        size_t ti = act[q];
        const Tile& t = lay.tiles[ti];
        size_t bu = t.tu << tl.log2, bv = t.tv << tl.log2;
        for (size_t i = 0; i < su; i++)
          for (size_t j = 0; j < sv; j++) {
            size_t row = (bu + i + s.nu / 2) % s.nu, col = (bv + j + s.nv / 2) % s.nv;
            std::complex<T> g = grid[row * s.nv + col];
            br[i * sv + j] = g.real();
            bi[i * sv + j] = g.imag();
          }
        for (size_t bix = t.b0; bix < t.b1; bix++) {
          const Block& b = lay.blocks[bix];
          size_t mp = b.minplane;
          if (s.do_wgridding && !(mp <= p && p < mp + S)) continue;
          for (size_t k = b.start; k < b.end; k++) {
            VisRef r = lay.refs[k];
            double uvw[3], imflip;
            uvw_of(bl, r, uvw, imflip);
            T ku[16], kv[16];
            int64_t iu0, iv0;
            taps_uv(uvw[0], uvw[1], ku, kv, iu0, iv0);
            size_t ou = offset_in(iu0, s.nu, bu), ov = offset_in(iv0, s.nv, bv);
            size_t idx = (size_t)r.row * nchan + r.ch;
            if (s.do_wgridding) {
              T kw = w_factor<T>(s, coeff.data(), ne, p - mp, p, uvw[2]);
              for (size_t i = 0; i < S; i++) ku[i] = ku[i] * kw;
            }
            T rr = 0, ri = 0;
            for (size_t cu = 0; cu < S; cu++) {
              size_t base = (ou + cu) * sv + ov;
              T tr = 0, tim = 0;
              for (size_t cv = 0; cv < S; cv++) {
                tr = std::fma(kv[cv], br[base + cv], tr);
                tim = std::fma(kv[cv], bi[base + cv], tim);
              }
              rr = std::fma(ku[cu], tr, rr);
              ri = std::fma(ku[cu], tim, ri);
            }
            std::complex<T> c(rr, ri * (T)imflip);
            out[idx] = c + out[idx];
          }
        }
      }
    }
  }

  // wgridder.rs:3048-3163 (plane group 1, unsorted output)
  void degrid_images(const T* dirty, Weights wgt, std::complex<T>* vis) const {
    size_t nx = s.nx, ny = s.ny, tnx, tny;
    s.table_dims(tnx, tny);
    std::vector<T> image(dirty, dirty + nx * ny);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < nx; i++) {
      if (s.do_wgridding) {
        for (size_t j = 0; j < ny; j++) image[i * ny + j] = image[i * ny + j] * (T)tab.corr[s.table_index(i, j, tny)];
      } else {
        size_t iu = nx / 2 - std::min(i, nx - i);
        for (size_t j = 0; j < ny; j++) {
          size_t iv = ny / 2 - std::min(j, ny - j);
          image[i * ny + j] = image[i * ny + j] * (T)(tab.cfu[iu] * tab.cfv[iv]);
        }
      }
    }
    std::vector<std::complex<T>> grid((size_t)s.nu * s.nv), screen;
    size_t nplanes = std::max<size_t>(s.nplanes, 1);
    for (size_t p = 0; p < nplanes; p++) {
      bool any = false;
      for (const Tile& t : lay.tiles)
        if (tile_active(s, t, p)) {
          any = true;
          break;
        }
      if (!any) continue;
      std::vector<char> needed = tile_rows(s, lay, p);
      double w0 = s.wmin + (double)p * s.dw;
      if (s.do_wgridding) screen_par<T>(tab.table, w0, false, screen);
      image_to_grid(image, screen, needed, grid.data());
      degrid_plane(p, grid.data(), vis);
    }
    size_t nchan = bl.nchan();
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < lay.refs.size(); k++) {
      VisRef r = lay.refs[k];
      size_t idx = (size_t)r.row * nchan + r.ch;
      T twgt = wgt.has() ? wgt.get<T>(idx) : (T)1;
      if (s.shifting) {
        std::complex<T> ph = shift_phase<T>(s, bl, r, -1.0);
        vis[idx] = cmul(vis[idx], std::complex<T>(ph.real() * twgt, ph.imag() * twgt));
      } else {
        vis[idx] = {vis[idx].real() * twgt, vis[idx].imag() * twgt};
      }
    }
  }
};

// ---------------------------------------------------------------- drivers

struct Common {
  WgridderOptions o;
  double r_l = 0, r_m = 0;
};

template <class T>
Plan vis2dirty_multi(const WgridderOptions& o, size_t nrow, size_t nchan, const double* uvw,
                     const double* freq, VisData data, Weights wgt, const uint8_t* mask, T* dirty,
                     T* psf) {
  check_common(o, nrow, nchan);
  size_t npix = o.nx * o.ny;
  if (!dirty && !psf) throw Error("array lengths disagree");
  double r_l, r_m;
  recentring(o, r_l, r_m);
  bool flips[3] = {o.flip_u != 0, o.flip_v != 0, !(o.flip_w != 0)};
  Baselines bl(uvw, nrow, freq, nchan, flips, r_l, r_m);
  Activity act;
  act.has_vis = psf == nullptr;
  act.vis = data;
  act.wgt = wgt;
  act.mask = mask;
  size_t nvis;
  double wmin_d, wmax_d;
  scan<T>(bl, act, nvis, wmin_d, wmax_d);
  if (dirty) std::fill(dirty, dirty + npix, (T)0);
  if (psf) std::fill(psf, psf + npix, (T)0);
  if (nvis == 0) return Plan{};
  Setup s = Setup::make<T>(o, nvis, wmin_d, wmax_d, r_l, r_m);
  Layout lay = layout<T>(s, bl, act);
  Tables tab = make_tables(s);
  Gridder<T> g(s, bl, lay, tab);
  bool both = dirty && psf;
  std::vector<std::complex<T>> stored;
  values<T>(s, bl, lay.refs, psf == nullptr, data, wgt, stored);
  if (both)
    g.grid_images(stored, true, data, dirty, psf);
  else
    g.grid_images(stored, false, data, dirty ? dirty : psf, nullptr);
  return s.plan;
}

template <class T>
Plan dirty2vis_multi(const WgridderOptions& o, size_t nrow, size_t nchan, const double* uvw,
                     const double* freq, const T* dirty, Weights wgt, const uint8_t* mask,
                     std::complex<T>* vis) {
  check_common(o, nrow, nchan);
  double r_l, r_m;
  recentring(o, r_l, r_m);
  bool flips[3] = {o.flip_u != 0, o.flip_v != 0, !(o.flip_w != 0)};
  Baselines bl(uvw, nrow, freq, nchan, flips, r_l, r_m);
  Activity act;
  act.has_vis = false;
  act.wgt = wgt;
  act.mask = mask;
  size_t nvis;
  double wmin_d, wmax_d;
  scan<T>(bl, act, nvis, wmin_d, wmax_d);
  std::fill(vis, vis + nrow * nchan, std::complex<T>(0, 0));
  if (nvis == 0) return Plan{};
  Setup s = Setup::make<T>(o, nvis, wmin_d, wmax_d, r_l, r_m);
  Layout lay = layout<T>(s, bl, act);
  Tables tab = make_tables(s);
  Gridder<T> g(s, bl, lay, tab);
  g.degrid_images(dirty, wgt, vis);
  return s.plan;
}

template <class F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const Error& e) {
    g_last_error = e.what();
    return 1;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return 2;
  }
}

Weights make_weights(const void* wgt, const void* wgt2, int kind) {
  Weights w;
  w.kind = kind;
  w.a = wgt;
  w.b = wgt2;
  if (kind != WGT_NONE && !wgt) throw Error("invalid weight array or kind");
  if (kind == WGT_F32_PRODUCT && !wgt2) throw Error("invalid weight array or kind");
  if (kind < 0 || kind > 3) throw Error("invalid weight array or kind");
  return w;
}

}  // namespace

// ---------------------------------------------------------------- C API

extern "C" {

int oracle_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
}

size_t oracle_last_error(char* buf, size_t len) {
  if (buf) std::memcpy(buf, g_last_error.data(), std::min(len, g_last_error.size()));
  return g_last_error.size();
}

// As rang_core_wgridder_vis2dirty_ex2_{f64,f32} (ffi_wgridder.rs:542-600).
int oracle_vis2dirty(const WgridderOptions* o, size_t nrow, size_t nchan, const double* uvw,
                     const double* freq, const void* vis, int vis_kind, const void* wgt,
                     const void* wgt2, int wgt_kind, const uint8_t* mask, void* dirty, void* psf,
                     double* info, int single) {
  return guarded([&] {
    if (!o || !uvw || !freq || !info || (!dirty && !psf)) throw Error("null array");
    VisData d;
    if (vis_kind < 0 || vis_kind > 2 || (vis_kind != VIS_UNIT && !vis))
      throw Error("invalid visibility array or kind");
    d.kind = vis_kind;
    d.p = vis;
    Weights w = make_weights(wgt, wgt2, wgt_kind);
    Plan p = single ? vis2dirty_multi<float>(*o, nrow, nchan, uvw, freq, d, w, mask, (float*)dirty,
                                             (float*)psf)
                    : vis2dirty_multi<double>(*o, nrow, nchan, uvw, freq, d, w, mask,
                                              (double*)dirty, (double*)psf);
    p.to_array(info);
  });
}

// As rang_core_wgridder_dirty2vis_ex_{f64,f32} (ffi_wgridder.rs:603-716).
int oracle_dirty2vis(const WgridderOptions* o, size_t nrow, size_t nchan, const double* uvw,
                     const double* freq, const void* dirty, const void* wgt, int wgt_kind,
                     const uint8_t* mask, void* vis, double* info, int single) {
  return guarded([&] {
    if (!o || !uvw || !freq || !info || !dirty || !vis) throw Error("null array");
    Weights w = make_weights(wgt, nullptr, wgt_kind);
    Plan p = single ? dirty2vis_multi<float>(*o, nrow, nchan, uvw, freq, (const float*)dirty, w,
                                             mask, (std::complex<float>*)vis)
                    : dirty2vis_multi<double>(*o, nrow, nchan, uvw, freq, (const double*)dirty, w,
                                              mask, (std::complex<double>*)vis);
    p.to_array(info);
  });
}

// The binning of a gridding (with_vis = 1: `|vis|^2 wgt mask != 0`) or
// degridding call: per visibility (row-major) its iu0, iv0, tile and first
// plane (-1 where inactive), and the sorted order as linear indices.
int oracle_binning(const WgridderOptions* o, size_t nrow, size_t nchan, const double* uvw,
                   const double* freq, const void* vis, int vis_kind, const void* wgt,
                   const void* wgt2, int wgt_kind, const uint8_t* mask, int with_vis, int single,
                   int64_t* iu0, int64_t* iv0, int64_t* tile, int64_t* minplane, uint64_t* sorted,
                   size_t* nsorted, double* info) {
  return guarded([&] {
    auto run = [&](auto tag) {
      using T = decltype(tag);
      check_common(*o, nrow, nchan);
      double r_l, r_m;
      recentring(*o, r_l, r_m);
      bool flips[3] = {o->flip_u != 0, o->flip_v != 0, !(o->flip_w != 0)};
      Baselines bl(uvw, nrow, freq, nchan, flips, r_l, r_m);
      Activity act;
      act.has_vis = with_vis != 0;
      act.vis.kind = vis_kind;
      act.vis.p = vis;
      act.wgt = make_weights(wgt, wgt2, wgt_kind);
      act.mask = mask;
      size_t nvis;
      double lo, hi;
      scan<T>(bl, act, nvis, lo, hi);
      size_t n = nrow * nchan;
      for (size_t i = 0; i < n; i++) iu0[i] = iv0[i] = tile[i] = minplane[i] = -1;
      *nsorted = 0;
      if (nvis == 0) {
        Plan{}.to_array(info);
        return;
      }
      Setup s = Setup::make<T>(*o, nvis, lo, hi, r_l, r_m);
      Layout lay = layout<T>(s, bl, act);
      for (size_t row = 0; row < nrow; row++)
        for (size_t ch = 0; ch < nchan; ch++) {
          size_t idx = row * nchan + ch;
          if (!act.active<T>(idx)) continue;
          size_t t, mp;
          locate(s, lay.tiling, bl, row, ch, t, mp, &iu0[idx], &iv0[idx]);
          tile[idx] = (int64_t)t;
          minplane[idx] = (int64_t)mp;
        }
      for (size_t k = 0; k < lay.refs.size(); k++)
        sorted[k] = (uint64_t)lay.refs[k].row * nchan + lay.refs[k].ch;
      *nsorted = lay.refs.size();
      s.plan.to_array(info);
    };
    if (single)
      run(float{});
    else
      run(double{});
  });
}

int oracle_kernel_row(size_t index, double* out) {
  if (index >= N_KERNEL_ROWS || !out) return 1;
  const KernelRowData& r = KERNEL_ROWS[index];
  double a[7] = {(double)r.w, r.ofactor, r.epsilon, r.beta, r.e0, (double)r.ndim, (double)r.single};
  std::memcpy(out, a, sizeof(a));
  return 0;
}

size_t oracle_good_size(size_t n) { return good_size_complex(n); }

// Gauss-Legendre nodes as the reference's gauss_legendre_symmetric.
size_t oracle_gauss_legendre(size_t n, double* x, double* w) {
  std::vector<double> xx, ww;
  gauss_legendre_symmetric(n, xx, ww);
  if (x) std::memcpy(x, xx.data(), xx.size() * sizeof(double));
  if (w) std::memcpy(w, ww.data(), ww.size() * sizeof(double));
  return xx.size();
}

// The kernel's ES function, polynomial approximation and correction function at
// `n` points `v` (what == 0, 1, 2).
int oracle_kernel_eval(size_t index, int what, size_t n, const double* v, double* out) {
  return guarded([&] {
    EsKernel k(index);
    for (size_t i = 0; i < n; i++)
      out[i] = what == 0 ? k.phi(v[i]) : what == 1 ? k.eval(v[i]) : k.corfunc(v[i]);
  });
}

// The even/odd coefficient table in working precision (wgridder.rs:1485-1507).
size_t oracle_coeff_even_odd(size_t index, int single, double* out) {
  EsKernel k(index);
  if (single) {
    auto c = coeff_even_odd<float>(k);
    if (out)
      for (size_t i = 0; i < c.size(); i++) out[i] = c[i];
    return c.size();
  }
  auto c = coeff_even_odd<double>(k);
  if (out) std::memcpy(out, c.data(), c.size() * sizeof(double));
  return c.size();
}

// One FFT of length n in place (interleaved complex doubles), for the tests.
void oracle_fft(size_t n, double* data, int inverse) {
  Fft<double> f(n);
  std::vector<std::complex<double>> work(n);
  f.exec((std::complex<double>*)data, work.data(), inverse != 0);
}

}  // extern "C"
