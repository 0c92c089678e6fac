// Host-side planning of a gridder call: the kernel table, the kernel and grid
// choice, the ES kernel's piecewise-polynomial coefficients and correction
// function, and the call geometry handed to the CUDA kernels.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "wgrid_common.h"

namespace wg {

// Status-1 failures (invalid arguments), as the reference's `Err(String)`.
struct InvalidArgument : std::runtime_error {
  using std::runtime_error::runtime_error;
};

struct KernelRow {
  int w;
  double ofactor, epsilon, beta, e0;
  int ndim;
  int single;
};

size_t kernel_count();
const KernelRow* kernel_row(size_t index);
size_t good_size_complex(size_t n);

// The ES kernel of one table row (wgridder.rs:277-356): the monomial
// coefficients of its W polynomial pieces and the Gauss-Legendre data of its
// correction function.
struct EsKernel {
  size_t index = 0, support = 0, degree = 0;
  double beta = 0, e0 = 0;
  std::vector<double> coeff, corr_x, corr_w;
  explicit EsKernel(size_t index);
  double corfunc(double v) const;
};

void check_common(const WgridderOptions& o, size_t nrow, size_t nchan);
void recentring(const WgridderOptions& o, double& r_l, double& r_m);
std::vector<double> f_over_c(const double* freq, size_t nchan);

// The reference's Setup::new (wgridder.rs:604-754) with the kernel choice of
// choose_kernel (wgridder.rs:876-926) and the tiling of Tiling::new.
template <class T>
void make_geom(const WgridderOptions& o, size_t nrow, size_t nchan, size_t nvis, double wmin_d,
               double wmax_d, double r_l, double r_m, Geom<T>& g, PlanInfo& info,
               EsKernel*& kernel);

}  // namespace wg
