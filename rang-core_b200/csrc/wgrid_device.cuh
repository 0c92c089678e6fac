// Device functions of the B200 w-gridder: per-visibility coordinates, grid
// position, first w-plane, kernel taps and stored values. Each restates the
// reference function named beside it (`core/src/wgridder.rs`) in the same
// floating-point order; the translation unit is compiled with
// `--fmad=false`, so only the explicit fma()/fmaf() calls (the reference's
// `mul_add`) fuse. The integer results (iu0, iv0, tile, first plane) are
// therefore bit-identical to the reference's.
#pragma once

#include <cuda_runtime.h>

#include "wgrid_common.h"

namespace wg {

template <class T>
struct cplx {
  T re, im;
};

// Borrowed visibility data, weights and mask of one call (device pointers).
struct Inputs {
  const void* vis = nullptr;
  int vis_kind = VIS_UNIT;
  const void* wgt = nullptr;
  const void* wgt2 = nullptr;
  int wgt_kind = WGT_NONE;
  const uint8_t* mask = nullptr;
};

__device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ void sincos_t(float a, float* s, float* c) { sincosf(a, s, c); }
__device__ __forceinline__ void sincos_t(double a, double* s, double* c) { sincos(a, s, c); }

// VisData::get (wgridder.rs:950-957): the value in working precision.
template <class T>
__device__ __forceinline__ cplx<T> vis_get(const Inputs& in, uint64_t i) {
  if (in.vis_kind == VIS_C64) {
    float2 v = reinterpret_cast<const float2*>(in.vis)[i];
    return {(T)(double)v.x, (T)(double)v.y};
  }
  if (in.vis_kind == VIS_C128) {
    double2 v = reinterpret_cast<const double2*>(in.vis)[i];
    return {(T)v.x, (T)v.y};
  }
  return {(T)1, (T)0};
}

// Weights::get (wgridder.rs:997-1005); 1 without weights.
template <class T>
__device__ __forceinline__ T wgt_get(const Inputs& in, uint64_t i) {
  switch (in.wgt_kind) {
    case WGT_F32:
      return (T)(double)reinterpret_cast<const float*>(in.wgt)[i];
    case WGT_F64:
      return (T)reinterpret_cast<const double*>(in.wgt)[i];
    case WGT_F32_PRODUCT: {
      float p = reinterpret_cast<const float*>(in.wgt)[i] * reinterpret_cast<const float*>(in.wgt2)[i];
      return (T)(double)p;
    }
    default:
      return (T)1;
  }
}

// Activity::active (wgridder.rs:1031-1042).
template <class T>
__device__ __forceinline__ bool is_active(const Inputs& in, bool with_vis, uint64_t i) {
  double tnorm = 1.0;
  if (with_vis) {
    cplx<T> v = vis_get<T>(in, i);
    T n = v.re * v.re + v.im * v.im;
    tnorm = (double)n;
  }
  double twgt = in.wgt_kind != WGT_NONE ? (double)wgt_get<T>(in, i) : 1.0;
  double tmask = in.mask ? (double)in.mask[i] : 1.0;
  return tnorm * twgt * tmask != 0.0;
}

// |vis|^2 |w|^2 in double precision: the square of a value's bound. The
// scan and the value-bound pass form it alike and take one square root of
// their maximum, so a plan's bound of its own data equals a pass over it.
template <class T>
__device__ __forceinline__ double value_bound_sq(cplx<T> v, double aw) {
  return ((double)v.re * (double)v.re + (double)v.im * (double)v.im) * (aw * aw);
}

// Baselines::new then FixW (wgridder.rs:568-586): the row's coordinates in
// metres with flips and recentring, flipped to w >= 0; returns the sign.
__device__ __forceinline__ double row_coord_of(double u, double v, double w, double fu, double fv, double fw,
                                               double r_l, double r_m, double b[3]) {
  double tu = fu * u, tv = fv * v, tw = fw * w;
  double c0 = tu + r_l * tw, c1 = tv + r_m * tw, c2 = tw;
  double res = 1.0 - 2.0 * (double)(c2 < 0.0 ? 1 : 0);
  b[0] = c0 * res;
  b[1] = c1 * res;
  b[2] = c2 * res;
  return res;
}
__device__ __forceinline__ double row_coord(const double* uvw, uint64_t row, double fu, double fv,
                                            double fw, double r_l, double r_m, double b[3]) {
  return row_coord_of(uvw[3 * row], uvw[3 * row + 1], uvw[3 * row + 2], fu, fv, fw, r_l, r_m, b);
}

// Setup::getpix (wgridder.rs:757-767), in 32-bit integers: u - floor(u)
// lies in [0, 1] (or is NaN), so u + ushift lies in (0, 2 nu + 1] and every
// intermediate fits an int; NaN converts to 0 in either width. The indices
// equal the reference's 64-bit ones, and I may be int or int64_t.
template <class T, class I>
__device__ __forceinline__ void getpix(const Geom<T>& g, double uin, double vin, double& uf, double& vf, I& iu0,
                                       I& iv0) {
  double u = uin * g.pixsize_x;
  u = (u - floor(u)) * (double)g.nu;
  const int a = min((int)(u + g.ushift) - g.nu, (int)g.maxiu0);
  u -= (double)a;
  double v = vin * g.pixsize_y;
  v = (v - floor(v)) * (double)g.nv;
  const int b = min((int)(v + g.vshift) - g.nv, (int)g.maxiv0);
  v -= (double)b;
  uf = u;
  vf = v;
  iu0 = a;
  iv0 = b;
}

// Setup::minplane and the clamp of Setup::locate (wgridder.rs:770-776, 1253-1254).
template <class T>
__device__ __forceinline__ int minplane(const Geom<T>& g, double w) {
  if (!g.do_wgridding) return 0;
  double t = fmax((w + g.wshift) * g.xdw, 0.0);
  int mp = t >= 2147483647.0 ? 2147483647 : (int)t;
  return min(mp, g.nbuckets - 1);
}

// `shifted` (wgridder.rs:1177-1179). getpix leaves i0 in [-supp/2, n), so
// i0 + n/2 is almost always in [0, 2n) and one compare replaces the 64-bit
// remainder; other values take the remainder, with the same result.
__device__ __forceinline__ int shifted(int64_t i0, int n) {
  int64_t r = i0 + n / 2;
  if (r >= 0 && r < 2 * (int64_t)n) return (int)(r >= n ? r - n : r);
  r %= n;
  return (int)(r < 0 ? r + n : r);
}
__device__ __forceinline__ int shifted(int i0, int n) {  // getpix's 32-bit indices (|i0| < 2^30)
  int r = i0 + n / 2;
  if (r >= 0 && r < 2 * n) return r >= n ? r - n : r;
  r %= n;
  return r < 0 ? r + n : r;
}

// `offset` (wgridder.rs:1183-1192).
__device__ __forceinline__ int offset_in(int64_t i0, int n, int base) {
  int64_t d = i0 + n / 2 - base;
  if (d < 0)
    d += n;
  else if (d >= n)
    d -= n;
  return (int)d;
}

// Rows of even (and of odd) coefficients of the support-S kernel: its
// polynomials have degree S + 3, padded to odd.
__host__ __device__ constexpr int coeff_rows(int S) { return (((S + 3) | 1) + 1) / 2; }

// The u and v taps by Horner's rule in x^2 on the even/odd split, first
// ceil(S/2) taps evaluated and the rest mirrored (wgridder.rs:1514-1543).
// `ne` is coeff_rows(S), which the host checks; the loops run to the
// compile-time count so that they unroll onto constant-bank operands.
template <class T, int S>
__device__ __forceinline__ void eval_taps2(const T* __restrict__ c, int /*ne*/, T x, T y, T* ru, T* rv) {
  constexpr int ne = coeff_rows(S);
  constexpr int H = (S + 1) / 2;
  T x2 = x * x, y2 = y * y;
  T ex[H], ey[H], ox[H], oy[H];
#pragma unroll
  for (int i = 0; i < H; i++) {
    ex[i] = ey[i] = c[i];
    ox[i] = oy[i] = c[ne * S + i];
  }
#pragma unroll
  for (int k = 1; k < ne; k++) {
#pragma unroll
    for (int i = 0; i < H; i++) {
      T ce = c[k * S + i], co = c[(ne + k) * S + i];
      ex[i] = fma_t(ex[i], x2, ce);
      ey[i] = fma_t(ey[i], y2, ce);
      ox[i] = fma_t(ox[i], x2, co);
      oy[i] = fma_t(oy[i], y2, co);
    }
  }
#pragma unroll
  for (int i = 0; i < H; i++) {
    ru[i] = fma_t(ox[i], x, ex[i]);
    rv[i] = fma_t(oy[i], y, ey[i]);
  }
#pragma unroll
  for (int i = 0; i < S - H; i++) {
    ru[S - 1 - i] = fma_t(ox[i], -x, ex[i]);
    rv[S - 1 - i] = fma_t(oy[i], -y, ey[i]);
  }
}

// One tap (wgridder.rs:1548-1560).
template <class T, int S>
__device__ __forceinline__ T eval_tap(const T* __restrict__ c, int /*ne*/, int i, T x) {
  constexpr int ne = coeff_rows(S);
  constexpr int H = (S + 1) / 2;
  if (i >= H) {
    i = S - 1 - i;
    x = -x;
  }
  T x2 = x * x;
  T e = c[i], o = c[ne * S + i];
#pragma unroll
  for (int k = 1; k < ne; k++) {
    e = fma_t(e, x2, c[k * S + i]);
    o = fma_t(o, x2, c[(ne + k) * S + i]);
  }
  return fma_t(o, x, e);
}

// w_factor (wgridder.rs:1580-1591): the w tap `nth` of plane p.
template <class T, int S>
__device__ __forceinline__ T w_factor(const Geom<T>& g, int nth, int p, double w) {
  double w0 = g.wmin + (double)p * g.dw;
  T z = (T)(g.xdw * (w0 - w));
  T locz = (z - (T)(double)nth) * (T)2.0 + (T)((double)S - 1.0);
  return eval_tap<T, S>(g.coeff, g.ne, nth, locz);
}

template <class T>
__device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

// shift_phase (wgridder.rs:1395-1408) from the row's fixed coordinates.
template <class T>
__device__ __forceinline__ cplx<T> shift_phase(const Geom<T>& g, const double b[3], double imflip,
                                               double f_over_c, double sign) {
  double fct = sign * imflip * (b[0] * g.lshift + b[1] * g.mshift + b[2] * g.nshift);
  double tmp = fct * f_over_c;
  T ang;
  if (sizeof(T) == 4)
    ang = (T)(2.0 * PI * (tmp - floor(tmp)));
  else
    ang = (T)(2.0 * PI * tmp);
  T s, c;
  sincos_t(ang, &s, &c);
  return {c, s};
}

// unit_value (wgridder.rs:1414-1424).
template <class T>
__device__ __forceinline__ cplx<T> unit_value(const Geom<T>& g, const double b[3], double imflip,
                                              double f_over_c, bool has_w, T w) {
  cplx<T> v{(T)1, (T)0};
  if (g.shifting) v = cmul(v, shift_phase<T>(g, b, imflip, f_over_c, 1.0));
  if (has_w) v = {v.re * w, v.im * w};
  return {v.re, v.im * (T)imflip};
}

// data_value (wgridder.rs:1432-1435).
template <class T>
__device__ __forceinline__ cplx<T> data_value(cplx<T> v, cplx<T> p, T imflip) {
  cplx<T> d = cmul(v, cplx<T>{p.re, p.im * imflip});
  return {d.re, d.im * imflip};
}

}  // namespace wg
