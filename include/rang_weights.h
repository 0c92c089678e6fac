/*
 * rang_weights.h — C ABI of the B200 imaging weights and Stokes I formation.
 *
 * The reference's C ABI for its port of WSClean's weighting, symbol for
 * symbol and struct for struct: rang-core `core/src/ffi_weights.rs`. Arrays
 * are HOST arrays borrowed for the call; the library copies them to the GPU,
 * grids, finishes and looks up the weights there and copies the outputs
 * back. Status codes are the reference's: 0 success, 1 invalid arguments,
 * 2 an internal failure (a CUDA error, no device memory); the message is kept
 * per thread for rang_core_wgridder_last_error (rang_wgridder.h).
 */
#ifndef RANG_WEIGHTS_H
#define RANG_WEIGHTS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ffi_weights.rs:8-19: `ncell` cells of four correlations (XX, XY, YX, YY). */
typedef struct StokesIInputs {
  size_t ncell;
  const float* data;     /* ncell * 4 interleaved complex floats */
  const float* weights;  /* ncell * 4 floats */
  const uint8_t* flags;  /* ncell * 4 bytes, non-zero when flagged */
} StokesIInputs;

/* ffi_weights.rs:21-26: ncell interleaved complex floats and ncell weights. */
typedef struct StokesIOutputs {
  float* vis;
  float* weight;
} StokesIOutputs;

/* ffi_weights.rs:28-51: one imaging-weight pass. */
typedef struct ImagingWeightInputs {
  size_t nrow;
  size_t nchan;
  const double* uvw;           /* nrow * 3 metres */
  const double* wavelength;    /* nchan metres */
  const float* weights;        /* nrow * nchan Stokes I visibility weights (zero where flagged) */
  const uint8_t* row_selected; /* nrow bytes, non-zero for rows WSClean selects */
  uint32_t class_;             /* 0 natural, 1 uniform, 2 Briggs (`class` in the reference) */
  double robust;
  size_t width;                /* padded image size */
  size_t height;
  double pixel_scale_x;
  double pixel_scale_y;
  double super_weight;
  double rank_filter_level;
  size_t rank_filter_size;
} ImagingWeightInputs;

/* ffi_weights.rs:53-64: caller-owned outputs; a null grid or sums is skipped. */
typedef struct ImagingWeightOutputs {
  float* weights; /* nrow * nchan floats */
  double* grid;   /* grid_width * grid_height / 2 doubles (rang_core_weight_grid_shape), or null */
  double* sums;   /* visibility weight sum, total weight, max gridded weight, count; or null */
} ImagingWeightOutputs;

/* ffi_weights.rs:84-105: the weight grid's (width, height) after the super weight. */
int32_t rang_core_weight_grid_shape(size_t width, size_t height, double super_weight, size_t* shape);

/* ffi_weights.rs:107-112: WSClean's padded image size; 0 never a valid size. */
size_t rang_core_padded_size(size_t trimmed, double padding);

/* ffi_weights.rs:114-158: Stokes I visibilities and weights (WSClean's -pol I rules). */
int32_t rang_core_stokes_i(const StokesIInputs* inputs, StokesIOutputs* outputs);

/* ffi_weights.rs:160-233: imaging weights of every row and channel. */
int32_t rang_core_imaging_weights(const ImagingWeightInputs* inputs, ImagingWeightOutputs* outputs);

#ifdef __cplusplus
}
#endif

#endif /* RANG_WEIGHTS_H */
