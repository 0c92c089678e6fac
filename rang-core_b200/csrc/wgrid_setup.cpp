// Host-side planning of a gridder call. Every formula here restates a line of
// the reference's `core/src/wgridder.rs` (cited per function) in the same
// floating-point order, because the kernel index, grid size, plane count and
// binning constants it produces must equal the reference's exactly.
#include "wgrid_setup.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <unordered_map>

namespace wg {

namespace {
const KernelRow KERNEL_ROWS[] = {
#include "kernel_db.inc"
};
constexpr size_t N_ROWS = sizeof(KERNEL_ROWS) / sizeof(KERNEL_ROWS[0]);

double es(double v, double beta, double e0) {  // wgridder.rs:225-232
  double tmp = (1.0 - v) * (1.0 + v);
  return tmp >= 0.0 ? std::exp(beta * (std::pow(tmp, e0) - 1.0)) : 0.0;
}

// Gauss-Legendre: non-negative nodes ascending, positive weights doubled
// (wgridder.rs:237-272).
void gauss_legendre(size_t n, std::vector<double>& x, std::vector<double>& w) {
  size_t m = (n + 1) / 2;
  x.assign(m, 0.0);
  w.assign(m, 0.0);
  for (size_t i = 0; i < m; i++) {
    double z = std::cos(PI * ((double)i + 0.75) / ((double)n + 0.5));
    double pp = 0.0;
    for (int it = 0; it < 100; it++) {
      double p1 = 1.0, p2 = 0.0;
      for (size_t j = 1; j <= n; j++) {
        double p3 = p2;
        p2 = p1;
        p1 = ((double)(2 * j - 1) * z * p2 - (double)(j - 1) * p3) / (double)j;
      }
      pp = (double)n * (z * p1 - p2) / (z * z - 1.0);
      double dz = p1 / pp;
      z -= dz;
      if (std::fabs(dz) <= 1e-16 * std::max(std::fabs(z), 1.0) && it > 0) break;
    }
    x[m - 1 - i] = z;
    w[m - 1 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
  if (n % 2 == 1) {
    x[0] = 0.0;
    w[0] *= 0.5;
  }
  for (double& v : w) v *= 2.0;
}

// Chebyshev interpolation of the kernel on W pieces of degree d, converted to
// monomials, highest power first (wgridder.rs:359-412).
std::vector<double> piecewise_poly(size_t W, size_t d, double beta, double e0) {
  std::vector<double> out(W * (d + 1));
  std::vector<double> root(d + 1), cheb((d + 1) * (d + 1), 0.0);
  for (size_t i = 0; i <= d; i++) root[i] = std::cos((double)(2 * i + 1) * PI / (double)(2 * d + 2));
  cheb[0] = 1.0;
  if (d >= 1) cheb[(d + 1) + 1] = 1.0;
  for (size_t j = 2; j <= d; j++) {
    cheb[j * (d + 1)] = -cheb[(j - 2) * (d + 1)];
    for (size_t k = 1; k <= j; k++)
      cheb[j * (d + 1) + k] = 2.0 * cheb[(j - 1) * (d + 1) + k - 1] - cheb[(j - 2) * (d + 1) + k];
  }
  std::vector<double> y(d + 1), c(d + 1), m(d + 1);
  for (size_t piece = 0; piece < W; piece++) {
    double l = -1.0 + 2.0 * (double)piece / (double)W;
    double r = -1.0 + 2.0 * (double)(piece + 1) / (double)W;
    for (size_t k = 0; k <= d; k++) {
      double at = ((root[k] * (r - l) * 0.5 + (r + l) * 0.5) + 1.0) * 0.5 * (1.0 - -1.0) + -1.0;
      y[k] = es(at, beta, e0);
    }
    double mean = 0.0;
    for (double v : y) mean += v;
    mean /= (double)(d + 1);
    for (double& v : y) v -= mean;
    std::fill(c.begin(), c.end(), 0.0);
    for (size_t j = 0; j <= d; j++)
      for (size_t k = 0; k <= d; k++)
        c[j] += 2.0 / (double)(d + 1) * y[k] * std::cos((double)(j * (2 * k + 1)) * PI / (double)(2 * d + 2));
    c[0] *= 0.5;
    std::fill(m.begin(), m.end(), 0.0);
    for (size_t j = 0; j <= d; j++)
      for (size_t k = 0; k <= d; k++) m[k] += cheb[j * (d + 1) + k] * c[j];
    m[0] += mean;
    for (size_t j = 0; j <= d; j++) out[piece * (d + 1) + j] = m[d - j];
  }
  return out;
}

// getAvailableKernels (wgridder.rs:154-181).
std::vector<size_t> candidate_kernels(double eps, size_t ndim, bool single, double smin, double smax) {
  size_t wlim = single ? 8 : 16;
  double best_of[20];
  size_t pick[20];
  std::fill(best_of, best_of + 20, smax);
  std::fill(pick, pick + 20, SIZE_MAX);
  for (size_t i = 0; i < N_ROWS; i++) {
    const KernelRow& r = KERNEL_ROWS[i];
    if ((size_t)r.ndim == ndim && (r.single != 0) == single && (size_t)r.w <= wlim && r.epsilon <= eps &&
        r.ofactor <= best_of[r.w] && r.ofactor >= smin) {
      best_of[r.w] = r.ofactor;
      pick[r.w] = i;
    }
  }
  std::vector<size_t> out;
  for (size_t i = 0; i < 20; i++)
    if (pick[i] != SIZE_MAX) out.push_back(pick[i]);
  if (out.empty()) throw InvalidArgument("no appropriate kernel for this epsilon, sigma range and precision");
  return out;
}

size_t plane_count(double wmin_d, double wmax_d, double dw, size_t supp) {
  double n = (wmax_d - wmin_d) / dw + (double)supp;
  return n >= 0.0 ? (size_t)n : 0;  // Rust `as usize`: NaN and negatives -> 0
}

}  // namespace

size_t kernel_count() { return N_ROWS; }
const KernelRow* kernel_row(size_t i) { return i < N_ROWS ? &KERNEL_ROWS[i] : nullptr; }

size_t good_size_complex(size_t n) {  // wgridder.rs:185-222
  if (n <= 12) return n;
  size_t best = 2 * n;
  for (size_t a = 1; a < best; a *= 11)
    for (size_t b = a; b < best; b *= 7)
      for (size_t c = b; c < best; c *= 5) {
        size_t x = c;
        while (x < n) x *= 2;
        for (;;) {
          if (x < n) {
            x *= 3;
          } else if (x > n) {
            best = std::min(best, x);
            if (x & 1) break;
            x >>= 1;
          } else {
            return n;
          }
        }
      }
  return best;
}

EsKernel::EsKernel(size_t idx) {
  const KernelRow* row = kernel_row(idx);
  if (!row) throw InvalidArgument("kernel index out of range");
  index = idx;
  support = (size_t)row->w;
  beta = row->beta * (double)support;
  e0 = row->e0;
  degree = support + 3;
  coeff = piecewise_poly(support, degree, beta, e0);
  size_t p = (size_t)(1.5 * (double)support) + 2;  // GLFullCorrection
  gauss_legendre(2 * p, corr_x, corr_w);
  for (size_t i = 0; i < corr_x.size(); i++) {
    corr_w[i] *= es(corr_x[i], beta, e0) * (double)support * 0.5;
    corr_x[i] *= PI * (double)support;
  }
}

double EsKernel::corfunc(double v) const {  // wgridder.rs:344-350
  double s = 0.0;
  for (size_t i = 0; i < corr_x.size(); i++) s += corr_w[i] * std::cos(corr_x[i] * v);
  return 1.0 / s;
}

void check_common(const WgridderOptions& o, size_t nrow, size_t nchan) {  // wgridder.rs:1102-1123
  if (o.nx == 0 || o.ny == 0) throw InvalidArgument("image dimensions must be positive");
  if (std::isnan(o.epsilon) || o.epsilon <= 0.0) throw InvalidArgument("epsilon must be positive");
  if (std::isnan(o.pixsize_x) || std::isnan(o.pixsize_y) || o.pixsize_x <= 0.0 || o.pixsize_y <= 0.0)
    throw InvalidArgument("pixel sizes must be positive");
  if (nchan == 0) throw InvalidArgument("uvw must have three values per row");
  if (nrow >= (1ull << 32) || nchan >= (1ull << 32)) throw InvalidArgument("too many rows or channels");
}

void recentring(const WgridderOptions& o, double& r_l, double& r_m) {  // wgridder.rs:1080-1100
  double ls = o.flip_u ? -o.center_x : o.center_x;
  double ms = o.flip_v ? -o.center_y : o.center_y;
  r_l = r_m = 0.0;
  if (o.do_wgridding && (ls != 0.0 || ms != 0.0)) {
    double xe = std::fabs(ls) + 0.5 * (double)o.nx * o.pixsize_x;
    double ye = std::fabs(ms) + 0.5 * (double)o.ny * o.pixsize_y;
    if (xe * xe + ye * ye < 1.0) {
      double n0 = std::sqrt(1.0 - ls * ls - ms * ms);
      r_l = ls / n0;
      r_m = ms / n0;
    }
  }
}

std::vector<double> f_over_c(const double* freq, size_t nchan) {  // wgridder.rs:560-577
  if (nchan == 0 || !(freq[0] > 0.0)) throw InvalidArgument("channel frequencies must be positive");
  for (size_t i = 1; i < nchan; i++)
    if (freq[i] < freq[i - 1]) throw InvalidArgument("channel frequencies must be sorted in ascending order");
  std::vector<double> f(nchan);
  for (size_t i = 0; i < nchan; i++) f[i] = freq[i] / C_LIGHT;
  return f;
}

namespace {
// Kernels are cached: building one evaluates a few hundred exponentials.
std::mutex g_kernel_mu;
std::unordered_map<size_t, EsKernel*> g_kernels;

EsKernel* cached_kernel(size_t idx) {
  std::lock_guard<std::mutex> lock(g_kernel_mu);
  auto it = g_kernels.find(idx);
  if (it != g_kernels.end()) return it->second;
  EsKernel* k = new EsKernel(idx);  // kept for the life of the process
  g_kernels[idx] = k;
  return k;
}
}  // namespace

template <class T>
void make_geom(const WgridderOptions& o, size_t nrow, size_t nchan, size_t nvis, double wmin_d,
               double wmax_d, double r_l, double r_m, Geom<T>& g, PlanInfo& info, EsKernel*& kernel) {
  const bool single = sizeof(T) == 4;
  const size_t wmax_supp = single ? 8 : 16;
  std::memset(&g, 0, sizeof(g));
  double px = o.pixsize_x, py = o.pixsize_y;
  double ls = o.flip_u ? -o.center_x : o.center_x;
  double ms = o.flip_v ? -o.center_y : o.center_y;
  bool lmshift = ls != 0.0 || ms != 0.0;
  // n - 1 at the corners (and the centre) of the field (getNuNv).
  double xmin = ls - 0.5 * (double)o.nx * px;
  double xmax = xmin + ((double)o.nx - 1.0) * px;
  double ymin = ms - 0.5 * (double)o.ny * py;
  double ymax = ymin + ((double)o.ny - 1.0) * py;
  double xs[3] = {xmin, xmax, 0.0}, ys[3] = {ymin, ymax, 0.0};
  int nxs = 2, nys = 2;
  if (r_l != 0.0 || r_m != 0.0) {
    xs[nxs++] = ls;
    ys[nys++] = ms;
  } else {
    if (xmin * xmax < 0.0) xs[nxs++] = 0.0;
    if (ymin * ymax < 0.0) ys[nys++] = 0.0;
  }
  double nm1min = 1e300, nm1max = -1e300;
  for (int a = 0; a < nxs; a++)
    for (int b = 0; b < nys; b++) {
      double t = xs[a] * xs[a] + ys[b] * ys[b];
      double nval = t <= 1.0 ? std::sqrt(1.0 - t) - 1.0 : -std::sqrt(t - 1.0) - 1.0;
      nval += r_l * xs[a] + r_m * ys[b];
      nm1min = std::min(nm1min, nval);
      nm1max = std::max(nm1max, nval);
    }
  bool wgrid = o.do_wgridding != 0;
  double nshift = (!o.allow_nshift || !wgrid) ? 0.0 : -0.5 * (nm1max + nm1min);
  size_t kidx, nu, nv;
  if (o.kernel_index >= 0) {
    const KernelRow* row = kernel_row((size_t)o.kernel_index);
    if (!row) throw InvalidArgument("kernel index out of range");
    if ((size_t)row->w > wmax_supp) throw InvalidArgument("kernel support too large for this precision");
    kidx = (size_t)o.kernel_index;
    nu = o.nu;
    nv = o.nv;
  } else {
    // The cost model with one thread and a SIMD width of eight.
    std::vector<size_t> cand = candidate_kernels(o.epsilon, wgrid ? 3 : 2, single, o.sigma_min, o.sigma_max);
    const double NREF = 2048.0, COSTREF = 0.0693;
    const size_t vlen = 8;
    double mincost = 1e300;
    kidx = SIZE_MAX;
    nu = nv = 0;
    for (size_t i : cand) {
      const KernelRow& k = *kernel_row(i);
      size_t supp = (size_t)k.w, nvec = (supp + vlen - 1) / vlen;
      size_t cu = std::max<size_t>(2 * good_size_complex((size_t)((double)o.nx * k.ofactor * 0.5) + 1), 16);
      size_t cv = std::max<size_t>(2 * good_size_complex((size_t)((double)o.ny * k.ofactor * 0.5) + 1), 16);
      double logterm = std::log((double)(cu * cv)) / std::log(NREF * NREF);
      double fft = (double)cu / NREF * (double)cv / NREF * logterm * COSTREF;
      double grid = 2.2e-10 * (double)nvis *
                    ((double)(supp * nvec * vlen) + (double)((2 * nvec + 1) * (supp + 3) * vlen));
      if (wgrid) {
        double dw = 0.5 / k.ofactor / std::max(std::fabs(nm1max + nshift), std::fabs(nm1min + nshift));
        fft *= (double)plane_count(wmin_d, wmax_d, dw, supp);
        grid *= (double)supp;
      }
      double cost = fft + grid;
      if (cost < mincost) {
        mincost = cost;
        kidx = i;
        nu = cu;
        nv = cv;
      }
    }
  }
  if ((nu >> 4) >= (1u << 16) || (nv >> 4) >= (1u << 16)) throw InvalidArgument("grid too large");
  kernel = cached_kernel(kidx);
  size_t supp = kernel->support;
  size_t nsafe = (supp + 1) / 2;
  if (nu < 2 * nsafe || nv < 2 * nsafe) throw InvalidArgument("grid too small");
  if (o.nx % 2 || o.ny % 2 || nu % 2 || nv % 2) throw InvalidArgument("image and grid sizes must be even");
  double ofactor = std::min((double)nu / (double)o.nx, (double)nv / (double)o.ny);
  size_t nplanes = 0;
  double wmin = 0, dw = 0, xdw = 0, wshift = 0;
  if (wgrid) {  // countRanges
    dw = 0.5 / ofactor / std::max(std::fabs(nm1max + nshift), std::fabs(nm1min + nshift));
    xdw = 1.0 / dw;
    nplanes = plane_count(wmin_d, wmax_d, dw, supp);
    if (nplanes >= (1u << 16)) throw InvalidArgument("too many w planes");
    wmin = (wmin_d + wmax_d) * 0.5 - 0.5 * ((double)nplanes - 1.0) * dw;
    wshift = dw - (0.5 * (double)supp * dw) - wmin;
  }
  // The image must fit the grid: its rows and columns are distinct grid rows
  // and columns (the column transforms address two disjoint column ranges).
  if (nu < o.nx || nv < o.ny) throw InvalidArgument("grid smaller than the image");
  // Grids beyond the CUDA kernels' 32-bit cell arithmetic are refused.
  if ((double)nu * (double)nv >= 2147483648.0) throw InvalidArgument("grid too large");
  g.nrow = nrow;
  g.nchan = nchan;
  g.nx = (int32_t)o.nx;
  g.ny = (int32_t)o.ny;
  g.nu = (int32_t)nu;
  g.nv = (int32_t)nv;
  g.supp = (int32_t)supp;
  g.nplanes = (int32_t)nplanes;
  g.nbuckets = (int32_t)std::max<size_t>(nplanes, 1);
  g.log2tile = single ? 5 : 4;  // ducc0's tile sizes: 32 cells in f32, 16 in f64
  int tile = 1 << g.log2tile;
  g.ntu = (int32_t)((nu + tile - 1) / tile);
  g.ntv = (int32_t)((nv + tile - 1) / tile);
  g.L = tile + (int32_t)supp - 1;
  // Sub-tiles group the visibilities whose footprints share one 8 x 8 window
  // of the tensor-core gridder and degridder: sube = 9 - supp cells square
  // (sube + supp - 1 = 8), ceil(tile / sube) of them along each side of a
  // tile (the last one partial where sube does not divide the tile). Double
  // precision, which has no tensor-core path, keeps 8 x 8 sub-tiles.
  g.sube = (single || supp <= 8) ? 9 - (int32_t)std::min<size_t>(supp, 8) : 8;
  g.nsub_side = (tile + g.sube - 1) / g.sube;
  g.nsub = g.nsub_side * g.nsub_side;
  g.do_wgridding = wgrid;
  g.lmshift = lmshift;
  g.shifting = lmshift || nshift != 0.0;
  g.divide_by_n = o.divide_by_n != 0;
  g.fu = o.flip_u ? -1.0 : 1.0;
  g.fv = o.flip_v ? -1.0 : 1.0;
  g.fw = o.flip_w ? 1.0 : -1.0;  // rang's convention is ducc0's flip_w = true
  g.r_l = r_l;
  g.r_m = r_m;
  g.pixsize_x = px;
  g.pixsize_y = py;
  g.ushift = (double)supp * (-0.5) + 1.0 + (double)nu;
  g.vshift = (double)supp * (-0.5) + 1.0 + (double)nv;
  g.maxiu0 = (int64_t)(nu + nsafe) - (int64_t)supp;
  g.maxiv0 = (int64_t)(nv + nsafe) - (int64_t)supp;
  g.wmin = wmin;
  g.dw = dw;
  g.xdw = xdw;
  g.wshift = wshift;
  g.lshift = ls;
  g.mshift = ms;
  g.nshift = nshift;
  g.x0 = ls - 0.5 * (double)o.nx * px;
  g.y0 = ms - 0.5 * (double)o.ny * py;
  // Even/odd coefficients (TemplateKernel, wgridder.rs:1485-1507).
  size_t d = kernel->degree, d1 = d + 1, dodd = d | 1, ne = (dodd + 1) / 2;
  g.ne = (int32_t)ne;
  auto a = [&](size_t i, size_t m) { return m > d ? 0.0 : kernel->coeff[i * d1 + (d - m)]; };
  for (size_t i = 0; i < supp; i++)
    for (size_t k = 0; k < ne; k++) {
      g.coeff[k * supp + i] = (T)a(i, dodd - 1 - 2 * k);
      g.coeff[(ne + k) * supp + i] = (T)a(i, dodd - 2 * k);
    }
  double v[N_INFO] = {(double)kidx,  (double)supp, (double)nu, (double)nv, (double)nplanes,
                      (double)nvis,  wmin_d,       wmax_d,     nm1min,     nm1max,
                      nshift,        dw,           wmin,       ofactor};
  std::memcpy(info.v, v, sizeof(v));
}

template void make_geom<float>(const WgridderOptions&, size_t, size_t, size_t, double, double, double,
                               double, Geom<float>&, PlanInfo&, EsKernel*&);
template void make_geom<double>(const WgridderOptions&, size_t, size_t, size_t, double, double, double,
                                double, Geom<double>&, PlanInfo&, EsKernel*&);

}  // namespace wg
