/* FISTA's vector steps and the Gaussian low-pass of the learned solver on
 * device images: the parts of the reference's `prox_solver::solve`
 * (core/src/prox_solver.rs:302-445) that are not the Gram operator, as
 * library kernels whose scalars stay on the device, so that an iteration
 * makes no host synchronisation.
 *
 * Images are n pixels of float (single = 1) or double; all pointers are
 * device pointers and every call is asynchronous on `stream` (a
 * cudaStream_t; null: the legacy stream). Status 0 on success, 1 for an
 * invalid argument, 2 for a CUDA failure (message: rang_core_wgridder_last_error).
 *
 * The solver state is RANG_FISTA_STATE doubles on the device:
 *   [0] t, [1] beta (the momentum of the current extrapolated point),
 *   [2] q0 = |W^(1/2) v|^2 / 2, [3] step, [4] lambda,
 *   [5] restarts so far, [6] target misfit (stop level; -inf for none),
 *   [7] first iteration whose misfit reached the target (-1: none yet),
 *   [8] the last misfit.
 * Sums are FP64, formed per block and added in a fixed order, so the
 * iterates do not depend on the launch. */
#ifndef RANG_SOLVER_H
#define RANG_SOLVER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RANG_FISTA_STATE 16

/* Fills `state` for a solve: t = 1, beta = 0, q0 from *q0_dev (device;
 * null: q0_host), step, lambda, target (-inf with has_target 0). */
int32_t rang_b200_fista_init(double* state, const double* q0_dev, double q0_host, double step, double lambda,
                             int32_t has_target, double target, void* stream);

/* Iteration k of the reference's loop, after the caller applied the Gram
 * operator to the extrapolated point y (g_y = G y):
 *   g_x = (g_y + beta g_x_prev) / (1 + beta)    (G x from linearity; g_y when beta = 0)
 *   misfit_k = q0 - <d, x> + <x, g_x> / 2        -> history[k], state[8]
 *   x_next = prox(y + step (d - g_y))            (soft threshold by step * lambda;
 *                                                 positivity unless is_signed)
 *   restart when restart != 0 and <y - x_next, x_next - x> > 0 (t = 1, beta' = 0),
 *   else t' = (1 + sqrt(1 + 4 t^2)) / 2, beta' = (t - 1) / t'  (momentum != 0)
 *   y_next = x_next + beta' (x_next - x)
 * `partials` is scratch of rang_b200_fista_partials() doubles. g_x, x_next
 * and y_next are outputs (distinct from the inputs). */
int32_t rang_b200_fista_step(int32_t single, size_t n, const void* d, const void* x, const void* y, const void* g_y,
                             const void* g_x_prev, void* g_x, void* x_next, void* y_next, double* state,
                             double* history, int32_t k, int32_t is_signed, int32_t momentum, int32_t restart,
                             double* partials, void* stream);
/* Doubles of scratch a step needs. */
size_t rang_b200_fista_partials(void);

/* <a, b> in FP64 into *out (device), summed in a fixed order. */
int32_t rang_b200_dot(int32_t single, size_t n, const void* a, const void* b, double* out, double* partials,
                      void* stream);

/* The periodic Gaussian blur of standard deviation `sigma` pixels of an
 * nx * ny float image (row-major, ny fastest): its real FFT times
 * exp(-2 pi^2 sigma^2 (fx^2 + fy^2)), transformed back and divided by
 * nx * ny (cuFFT R2C / C2R). `out` may equal `in`. */
int32_t rang_b200_gaussian_lowpass(size_t nx, size_t ny, const float* in, float* out, double sigma, void* stream);

#ifdef __cplusplus
}
#endif

#endif
