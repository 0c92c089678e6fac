// Shared host/device definitions of the B200 w-gridder.
//
// `WgridderOptions` (include/rang_wgridder.h) keeps the reference's C layout
// byte for byte (core/src/ffi_wgridder.rs:24-42), so a binding written for
// the reference's C ABI works unchanged. `Geom<T>` is everything a kernel needs about one
// call's plan; it is passed to every kernel by value (it lives in the
// kernel-parameter constant bank), so concurrent calls on different streams
// share no device state.
#pragma once

#include <cstddef>
#include <cstdint>

#include "rang_wgridder.h"  // WgridderOptions, the kind codes

namespace wg {

// Data kinds of the `_ex` entry points (ffi_wgridder.rs:297-310).
// VIS_SORTED is internal: complex float values indexed by sorted position
// (a plan's stored values); no entry point accepts it from a caller.
enum VisKind : int { VIS_UNIT = 0, VIS_C64 = 1, VIS_C128 = 2, VIS_SORTED = 3 };
enum WgtKind : int { WGT_NONE = 0, WGT_F32 = 1, WGT_F64 = 2, WGT_F32_PRODUCT = 3 };

constexpr double C_LIGHT = 299792458.0;  // wgridder.rs:58
constexpr double PI = 3.14159265358979323846;
constexpr int N_INFO = 14;
constexpr int MAX_SUPP = 16;
// Even/odd coefficient rows: degree W + 3 padded to odd -> at most 10 rows of
// each parity for W = 16.
constexpr int MAX_COEFF = 2 * 10 * MAX_SUPP;

// The plan report (`Plan`, wgridder.rs:471-511).
struct PlanInfo {
  double v[N_INFO];
};

// Geometry of one call in working precision T, derived on the host from the
// options and the scan (the reference's `Setup`, wgridder.rs:516-544) and the
// layout parameters (`Tiling`, wgridder.rs:1152-1173).
template <class T>
struct Geom {
  uint64_t nrow, nchan;
  int32_t nx, ny, nu, nv;
  int32_t supp, nplanes, nbuckets;  // nbuckets = max(nplanes, 1)
  int32_t log2tile, ntu, ntv, L;    // L = tile + supp - 1
  // Sub-tiles of a tile, sube cells square: nsub_side along each side, nsub
  // in all (sub-tile (a, b) of a tile is a * nsub_side + b).
  int32_t sube, nsub_side, nsub;
  int32_t ne;                       // rows of even (and of odd) coefficients
  int32_t do_wgridding, shifting, lmshift, divide_by_n;
  double fu, fv, fw;  // +-1: flips (w already negated as the reference does)
  double r_l, r_m;    // recentring
  double pixsize_x, pixsize_y;
  double ushift, vshift;
  int64_t maxiu0, maxiv0;
  double wmin, dw, xdw, wshift;
  double lshift, mshift, nshift;
  double x0, y0;  // l, m of pixel (0, 0)
  // Even/odd kernel coefficients (wgridder.rs:1485-1507) in T.
  T coeff[MAX_COEFF];
};

}  // namespace wg
