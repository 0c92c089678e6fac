/*
 * rang_gram.h — the visibility-free w-aware normal operator on the B200.
 *
 * The reference's GramOperator (rang-core `core/src/gridder_gram.rs`): a sum
 * of Toeplitz operators, one per w-node, each applied by FFTs on the 2n
 * grid, set up by gridding node-weighted visibilities without w. The
 * reference has it as a Rust type only (its solver and benchmark binaries
 * build it, core/src/prox_solver.rs:1423, core/src/bin/gram_solver_bench.rs:
 * 598-601); these entry points are the C ABI a Rust host would bind in its
 * place. Arrays named `_dev` are device pointers; `freq_host` is on the
 * host; `stream` is the caller's cudaStream_t (null: the legacy default stream).
 * Status codes as rang_wgridder.h: 0 success, 1 invalid arguments, 2 an
 * internal failure; the message is kept per thread for
 * rang_core_wgridder_last_error.
 */
#ifndef RANG_GRAM_H
#define RANG_GRAM_H

#include <stddef.h>
#include <stdint.h>

#include "rang_wgridder.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The setup statistics (gridder_gram.rs:184-206 `Stats`), in this order:
 * planes, stencil, theta, wmin, wmax, x_range, sup_error, lebesgue,
 * active_pairs, cube_bytes, setup_grid_seconds, setup_fft_seconds,
 * spectral_sparsity, hermitian_check. */
#define RANG_GRAM_NSTATS 14

typedef struct RangGram RangGram;

/* WExpansion::new (gridder_gram.rs:88-141): the (8192 + 1) x stencil
 * coefficient table (or null), the measured sup error and the Lebesgue
 * constant of the fit. Host only; needs no GPU. */
int32_t rang_b200_gram_expansion(size_t stencil, double theta, double ridge, double* table, double* sup_error,
                                 double* lebesgue);

/* GramOperator::new (gridder_gram.rs:224-412), or GramOperator::no_w
 * (:415-486) when `no_w` is non-zero (then stencil, theta and ridge are
 * unused). `opts` holds the imaging options with nx = ny = n (even);
 * `uvw_dev` (nrow x 3 metres), `wgt_dev` (nrow x nchan float64 weights);
 * `single` keeps float32 spectra and grids. `stats`: RANG_GRAM_NSTATS doubles. */
int32_t rang_b200_gram_create(const WgridderOptions* opts, size_t nrow, size_t nchan, const double* uvw_dev,
                              const double* freq_host, const double* wgt_dev, size_t stencil, double theta,
                              double ridge, double epsilon, int32_t single, int32_t no_w, void* stream,
                              RangGram** out, double* stats);

/* GramOperator::apply (gridder_gram.rs:518-631): out_dev = G~ m_dev, n x n float64. */
int32_t rang_b200_gram_apply(RangGram* op, const double* m_dev, double* out_dev, void* stream);

/* GramOperator::inverse_filter (gridder_gram.rs:488-511): the circulant
 * preconditioner 1 / (max(K^, 0) + rho) of a one-node operator. */
int32_t rang_b200_gram_inverse_filter(const RangGram* op, double rho, void* stream, RangGram** out);

/* The no-w PSF on the 2n grid, sum over nodes of Re K_k centred on (n, n)
 * (the `psf_no_w` field), into (2n)^2 float64 device memory. */
int32_t rang_b200_gram_psf_no_w(const RangGram* op, double* out_dev, void* stream);

/* GramOperator::planes (gridder_gram.rs:634-637). */
int32_t rang_b200_gram_planes(const RangGram* op);

void rang_b200_gram_destroy(RangGram* op);

#ifdef __cplusplus
}
#endif

#endif /* RANG_GRAM_H */
