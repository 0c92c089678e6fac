// FISTA's vector steps and the learned solver's Gaussian low-pass on device
// images (include/rang_solver.h): the reference's prox_solver::solve
// (core/src/prox_solver.rs:302-445) without its Gram operator, which the
// caller applies with the gridder's plan. The scalars of the iteration
// (t, beta, the misfit, the restart test) stay on the device, so a FISTA
// iteration issues kernels only and never waits for the device.
//
// Every reduction runs on a fixed grid of blocks: each thread sums a fixed
// stride of the pixels in order, each block adds its threads in a fixed
// tree, and one block adds the block partials in a fixed order, so the
// iterates are the same on every run.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <functional>
#include <map>
#include <mutex>
#include <tuple>

#include "rang_solver.h"
#include "wgrid_plan.h"
#include "wgrid_setup.h"

namespace wg {
int32_t status_guarded(const std::function<void()>& f);
cudaStream_t stream_of(void* stream);
}  // namespace wg

using namespace wg;

namespace {

constexpr int THREADS = 256;
constexpr int BLOCKS = 148 * 4;  // fixed: the partial sums do not depend on the device or the launch
constexpr int NPART = 3;         // partial sums per block of a step

enum StateIndex : int { S_T = 0, S_BETA, S_Q0, S_STEP, S_LAM, S_RESTARTS, S_TARGET, S_FIRST, S_MISFIT };

__device__ __forceinline__ double block_reduce(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = THREADS / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

__global__ void k_fista_init(double* st, const double* q0_dev, double q0, double step, double lam, int has_target,
                             double target) {
  for (int i = 0; i < RANG_FISTA_STATE; i++) st[i] = 0.0;
  st[S_T] = 1.0;
  st[S_BETA] = 0.0;
  st[S_Q0] = q0_dev ? *q0_dev : q0;
  st[S_STEP] = step;
  st[S_LAM] = lam;
  st[S_TARGET] = has_target ? target : -INFINITY;
  st[S_FIRST] = -1.0;
  st[S_MISFIT] = NAN;
}

// L1Prior::prox (prox_solver.rs:80-105): the soft threshold by tau, with
// positivity unless signed.
template <class T>
__device__ __forceinline__ T prox(T z, T tau, int is_signed) {
  if (is_signed) {
    const T a = fabs(z) - tau;
    return a > (T)0 ? copysign(a, z) : (T)0;
  }
  const T a = z - tau;
  return a > (T)0 ? a : (T)0;
}

// The pixel pass of one iteration: G x, the prox step from y and the three
// inner products, per block.
template <class T>
__global__ void __launch_bounds__(THREADS)
    k_fista_pixels(uint64_t n, const T* __restrict__ d, const T* __restrict__ x, const T* __restrict__ y,
                   const T* __restrict__ g_y, const T* __restrict__ g_x_prev, T* __restrict__ g_x,
                   T* __restrict__ x_next, const double* __restrict__ st, int is_signed, double* __restrict__ partials) {
  __shared__ double sh[THREADS];
  const double beta = st[S_BETA];
  const T b = (T)beta, step = (T)st[S_STEP], tau = (T)(st[S_STEP] * st[S_LAM]);
  double dx = 0.0, xgx = 0.0, inner = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)THREADS + threadIdx.x; i < n; i += (uint64_t)BLOCKS * THREADS) {
    const T gy = g_y[i];
    const T gx = beta == 0.0 ? gy : (gy + b * g_x_prev[i]) / ((T)1 + b);
    const T xi = x[i], yi = y[i], di = d[i];
    const T xn = prox<T>(yi + step * (di - gy), tau, is_signed);
    g_x[i] = gx;
    x_next[i] = xn;
    dx += (double)di * (double)xi;
    xgx += (double)xi * (double)gx;
    inner += ((double)yi - (double)xn) * ((double)xn - (double)xi);
  }
  dx = block_reduce(dx, sh);
  xgx = block_reduce(xgx, sh);
  inner = block_reduce(inner, sh);
  if (threadIdx.x == 0) {
    partials[NPART * blockIdx.x] = dx;
    partials[NPART * blockIdx.x + 1] = xgx;
    partials[NPART * blockIdx.x + 2] = inner;
  }
}

// The scalars of one iteration (one block): the misfit, the target test and
// the momentum with gradient restart (prox_solver.rs:417-431).
__global__ void __launch_bounds__(THREADS)
    k_fista_scalars(const double* __restrict__ partials, double* st, double* history, int k, int momentum,
                    int restart) {
  __shared__ double sh[THREADS];
  double s[NPART];
  for (int j = 0; j < NPART; j++) {
    double v = 0.0;
    for (int b = threadIdx.x; b < BLOCKS; b += THREADS) v += partials[NPART * b + j];
    s[j] = block_reduce(v, sh);
  }
  if (threadIdx.x != 0) return;
  const double misfit = st[S_Q0] - s[0] + 0.5 * s[1];
  if (history) history[k] = misfit;
  st[S_MISFIT] = misfit;
  if (st[S_FIRST] < 0.0 && misfit <= st[S_TARGET]) st[S_FIRST] = (double)k;
  double next_beta = 0.0;
  if (momentum) {
    const double t = st[S_T];
    if (restart && s[2] > 0.0) {
      st[S_T] = 1.0;
      st[S_RESTARTS] += 1.0;
    } else {
      const double t_next = 0.5 * (1.0 + sqrt(1.0 + 4.0 * t * t));
      next_beta = (t - 1.0) / t_next;
      st[S_T] = t_next;
    }
  }
  st[S_BETA] = next_beta;
}

// y_next = x_next + beta' (x_next - x).
template <class T>
__global__ void __launch_bounds__(THREADS)
    k_fista_momentum(uint64_t n, const T* __restrict__ x_next, const T* __restrict__ x, T* __restrict__ y_next,
                     const double* __restrict__ st) {
  const T b = (T)st[S_BETA];
  for (uint64_t i = blockIdx.x * (uint64_t)THREADS + threadIdx.x; i < n; i += (uint64_t)BLOCKS * THREADS) {
    const T xn = x_next[i];
    y_next[i] = xn + b * (xn - x[i]);
  }
}

template <class T>
__global__ void __launch_bounds__(THREADS)
    k_dot(uint64_t n, const T* __restrict__ a, const T* __restrict__ b, double* __restrict__ partials) {
  __shared__ double sh[THREADS];
  double v = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)THREADS + threadIdx.x; i < n; i += (uint64_t)BLOCKS * THREADS)
    v += (double)a[i] * (double)b[i];
  v = block_reduce(v, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = v;
}

__global__ void __launch_bounds__(THREADS) k_dot_sum(const double* __restrict__ partials, double* out) {
  __shared__ double sh[THREADS];
  double v = 0.0;
  for (int b = threadIdx.x; b < BLOCKS; b += THREADS) v += partials[b];
  v = block_reduce(v, sh);
  if (threadIdx.x == 0) *out = v;
}

// The Gaussian's transfer function on the half spectrum (nx rows, ny / 2 + 1
// columns), with the 1 / (nx ny) of the inverse transform.
__global__ void k_gauss_spectrum(cufftComplex* __restrict__ f, int nx, int ny, double sigma) {
  const int nh = ny / 2 + 1;
  const uint64_t total = (uint64_t)nx * nh;
  const double c = -2.0 * M_PI * M_PI * sigma * sigma, inv = 1.0 / ((double)nx * (double)ny);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / nh), col = (int)(i - (uint64_t)r * nh);
    const double fx = (double)(r <= nx / 2 ? r : r - nx) / nx, fy = (double)col / ny;  // fftfreq, rfftfreq
    const float g = (float)(exp(c * (fx * fx + fy * fy)) * inv);
    f[i].x *= g;
    f[i].y *= g;
  }
}

struct LowpassPlans {
  cufftHandle fwd = 0, inv = 0;
  std::mutex mu;
};

LowpassPlans& lowpass_plans(int dev, int nx, int ny) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int>, LowpassPlans*> plans;
  std::lock_guard<std::mutex> lock(mu);
  LowpassPlans*& p = plans[{dev, nx, ny}];
  if (!p) {
    auto* q = new LowpassPlans();
    if (cufftPlan2d(&q->fwd, nx, ny, CUFFT_R2C) != CUFFT_SUCCESS || cufftPlan2d(&q->inv, nx, ny, CUFFT_C2R) != CUFFT_SUCCESS) {
      delete q;
      throw DeviceError("cuFFT plan for the low-pass failed");
    }
    p = q;
  }
  return *p;
}

}  // namespace

extern "C" {

int32_t rang_b200_fista_init(double* state, const double* q0_dev, double q0_host, double step, double lambda,
                             int32_t has_target, double target, void* stream) {
  return status_guarded([&] {
    if (!state) throw InvalidArgument("null state");
    k_fista_init<<<1, 1, 0, stream_of(stream)>>>(state, q0_dev, q0_host, step, lambda, has_target, target);
    check_cuda(cudaGetLastError(), "fista init");
  });
}

size_t rang_b200_fista_partials(void) { return (size_t)NPART * BLOCKS; }

int32_t rang_b200_fista_step(int32_t single, size_t n, const void* d, const void* x, const void* y, const void* g_y,
                             const void* g_x_prev, void* g_x, void* x_next, void* y_next, double* state,
                             double* history, int32_t k, int32_t is_signed, int32_t momentum, int32_t restart,
                             double* partials, void* stream) {
  return status_guarded([&] {
    if (!d || !x || !y || !g_y || !g_x_prev || !g_x || !x_next || !y_next || !state || !partials)
      throw InvalidArgument("null array");
    if (k < 0) throw InvalidArgument("negative iteration");
    cudaStream_t s = stream_of(stream);
    if (single) {
      k_fista_pixels<float><<<BLOCKS, THREADS, 0, s>>>(n, (const float*)d, (const float*)x, (const float*)y,
                                                       (const float*)g_y, (const float*)g_x_prev, (float*)g_x,
                                                       (float*)x_next, state, is_signed, partials);
    } else {
      k_fista_pixels<double><<<BLOCKS, THREADS, 0, s>>>(n, (const double*)d, (const double*)x, (const double*)y,
                                                        (const double*)g_y, (const double*)g_x_prev, (double*)g_x,
                                                        (double*)x_next, state, is_signed, partials);
    }
    check_cuda(cudaGetLastError(), "fista pixels");
    k_fista_scalars<<<1, THREADS, 0, s>>>(partials, state, history, k, momentum, restart);
    check_cuda(cudaGetLastError(), "fista scalars");
    if (single)
      k_fista_momentum<float><<<BLOCKS, THREADS, 0, s>>>(n, (const float*)x_next, (const float*)x, (float*)y_next, state);
    else
      k_fista_momentum<double><<<BLOCKS, THREADS, 0, s>>>(n, (const double*)x_next, (const double*)x, (double*)y_next,
                                                          state);
    check_cuda(cudaGetLastError(), "fista momentum");
  });
}

int32_t rang_b200_dot(int32_t single, size_t n, const void* a, const void* b, double* out, double* partials,
                      void* stream) {
  return status_guarded([&] {
    if (!a || !b || !out || !partials) throw InvalidArgument("null array");
    cudaStream_t s = stream_of(stream);
    if (single)
      k_dot<float><<<BLOCKS, THREADS, 0, s>>>(n, (const float*)a, (const float*)b, partials);
    else
      k_dot<double><<<BLOCKS, THREADS, 0, s>>>(n, (const double*)a, (const double*)b, partials);
    check_cuda(cudaGetLastError(), "dot");
    k_dot_sum<<<1, THREADS, 0, s>>>(partials, out);
    check_cuda(cudaGetLastError(), "dot sum");
  });
}

int32_t rang_b200_gaussian_lowpass(size_t nx, size_t ny, const float* in, float* out, double sigma, void* stream) {
  return status_guarded([&] {
    if (!in || !out) throw InvalidArgument("null array");
    if (nx < 1 || ny < 1 || nx > (1u << 20) || ny > (1u << 20)) throw InvalidArgument("image size");
    if (!(sigma >= 0.0) || !std::isfinite(sigma)) throw InvalidArgument("sigma must be finite and non-negative");
    cudaStream_t s = stream_of(stream);
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "device");
    LowpassPlans& p = lowpass_plans(dev, (int)nx, (int)ny);
    DevBuf spec(nx * (ny / 2 + 1) * sizeof(cufftComplex), s);
    std::lock_guard<std::mutex> lock(p.mu);
    if (cufftSetStream(p.fwd, s) != CUFFT_SUCCESS || cufftSetStream(p.inv, s) != CUFFT_SUCCESS)
      throw DeviceError("cuFFT stream");
    if (cufftExecR2C(p.fwd, const_cast<float*>(in), spec.as<cufftComplex>()) != CUFFT_SUCCESS)
      throw DeviceError("cuFFT forward transform");
    const uint64_t total = (uint64_t)nx * (ny / 2 + 1);
    k_gauss_spectrum<<<(unsigned)std::min<uint64_t>((total + 255) / 256, 148u * 16u), 256, 0, s>>>(
        spec.as<cufftComplex>(), (int)nx, (int)ny, sigma);
    check_cuda(cudaGetLastError(), "low-pass");
    if (cufftExecC2R(p.inv, spec.as<cufftComplex>(), out) != CUFFT_SUCCESS) throw DeviceError("cuFFT inverse transform");
  });
}

}  // extern "C"
