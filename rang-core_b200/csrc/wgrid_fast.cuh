// The single-precision gridder and degridder on the tensor cores, and the
// fixed-point grid that makes gridding exact and order-independent.
//
// Included by wgrid_plan.cu inside its anonymous namespace (it uses the scan,
// binning and device helpers defined there).
//
// Records. The binning's count pass writes one 32-byte record per active
// visibility at its own index: the tap arguments of u, v and w, the
// visibility's index, its shift phase, its offset inside its sub-tile's
// window, its first plane and its bin. The per-visibility FP64 arithmetic
// (coordinates, getpix, minplane, the phase's argument reduction) is thus
// done once per plan, and the gridder and degridder read records through
// the sorted indices.
//
// Exact gridding. Every grid cell is an int64 fixed-point sum (a pair per
// complex cell) of the footprint terms kw * ku * (value * kv). The gridder
// forms both factors as 23-bit integers, A = rint(kw ku 2^22) and
// B = rint(value kv 2^sb), splits each into three balanced 8-bit limbs
// (x = x2 2^16 + x1 2^8 + x0, x0 and x1 in [-128, 127]) and contracts the
// limbs on the integer tensor cores (mma.sync m16n8k32, s8 x s8 -> s32),
// keeping the limb products of weight 2^32, 2^24 and 2^16: the kept sums are
// exact integers and the dropped terms (weight 2^8 and 1, zero-mean) are
// below 2^-21 of the largest term. Integer sums do not depend on the order
// of their terms, so the result is bit for bit the same whatever the order
// of the visibilities in the sorted layout, however they are split among
// warps and blocks, and whatever the order of the atomic adds into the
// grid: a call is reproducible and a one-pass PSF equals a separate call.
// The grid is converted to floating point once, before the FFTs.

namespace fast {

// A grid cell in fixed point: value = (re + i im) * 2^-q.
struct FixCell {
  long long re, im;
};

// The fixed-point scales of one gridding pass (written on the device).
struct FixScale {
  int sb;         // B = rint(value * kv * 2^sb) in the integer gridder
  int q;          // cell value = int64 * 2^-q
  int nonfinite;  // an active value or tap was not finite: the planes are NaN
  int pad;
};

// Largest |value| of a pass (device scalars, the scan's or k_value_max's).
struct ValueBound {
  unsigned long long vmax_bits;  // max |vis| |wgt| (as the bits of a non-negative double)
  unsigned long long wmax_bits;  // max |wgt|
};

__device__ __forceinline__ void atomic_max_double(unsigned long long* a, double v) {
  if (v > 0.0) atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

// max |vis| |wgt| and max |wgt| over visibilities [i0, i1) that the plan
// keeps (key != INACTIVE), for gridding data other than the plan's own.
template <class T>
__global__ void k_value_max(uint64_t i0, uint64_t i1, Inputs in, const uint32_t* __restrict__ key, ValueBound* vb) {
  double vm = 0.0, wm = 0.0;
  for (uint64_t i = i0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < i1;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (key[i] == INACTIVE) continue;
    const double w = fabs((double)wgt_get<T>(in, i));
    const double a = value_bound_sq(vis_get<T>(in, i), w);
    // NaN compares false and is dropped here; the gridder flags it.
    vm = a > vm ? a : vm;
    wm = w > wm ? w : wm;
  }
  for (int o = 16; o > 0; o >>= 1) {
    vm = fmax(vm, __shfl_down_sync(0xffffffffu, vm, o));
    wm = fmax(wm, __shfl_down_sync(0xffffffffu, wm, o));
  }
  if ((threadIdx.x & 31) == 0) {
    vm = sqrt(vm);
    atomic_max_double(&vb->vmax_bits, vm);
    atomic_max_double(&vb->wmax_bits, wm);
  }
}

__global__ void k_bound_init(ValueBound* vb, unsigned long long vmax_bits, unsigned long long wmax_bits) {
  vb->vmax_bits = vmax_bits;
  vb->wmax_bits = wmax_bits;
}

// The scales of one pass from the value maxima of `values`. `unit`: unit
// values (the PSF), bounded by max |wgt|; otherwise max |vis| |wgt|. The
// integer gridder's terms are at most 2^28 grid units (q = sb + 6), so int64
// holds 2^34 of them. For the floating-point gridders a cell sums at most
// nvis terms, each at most max |value| (taps are at most 1 + eps), and q
// leaves 2 bits of headroom over that bound in the cell's width (64 bits in
// single precision; 94 bits of hi * 2^32 + lo in double, where the unit is
// 2^-(92 - log2 nvis) of the largest value, 2^-60 or finer: a 64-bit cell's
// unit would sit about 2^-48 below the largest term, which the wide-field
// correction factors amplify past double precision's accuracy). The scales
// depend on nothing but the values and the active count, so a plan split
// into row chunks grids to the same bits as one without.
// The exponent the scales take from `values`: vmax < 2^(ev + 1) (clamped,
// so that the scales stay finite floats).
__device__ __forceinline__ int bound_exponent(const ValueBound* values, int unit) {
  double vmax = __longlong_as_double((long long)(unit ? values->wmax_bits : values->vmax_bits));
  if (!(vmax > 0.0) || !isfinite(vmax)) vmax = 1.0;
  return min(max(ilogb(vmax), -90), 90);
}

__device__ __forceinline__ FixScale scale_of(int ev, unsigned long long nvis, int integer, int wide) {
  FixScale r;
  r.nonfinite = 0;
  r.pad = 0;
  if (integer) {
    r.sb = 21 - ev;  // |B| < 2^22
    r.q = r.sb + 6;
  } else {
    r.sb = 0;
    // nvis * vmax * 2^q < 2^62 (int64 cells), < 2^94 (hi * 2^32 + lo cells)
    r.q = (wide ? 92 : 60) - ev - ilogb((double)max(nvis, 1ull));
  }
  return r;
}

__global__ void k_fix_scale(const ValueBound* values, int unit, unsigned long long nvis, int integer, int wide,
                            FixScale* fs) {
  *fs = scale_of(bound_exponent(values, unit), nvis, integer, wide);
}

// Gridding row chunks as they arrive, before the bound of all the values
// is known: the scale depends on the bound only through its exponent, so
// the chunks are gridded with the exponent of the values seen so far, and
// when a chunk changes it, the planes are cleared and the chunks before it
// gridded again (`redo`, which their launches test). After the last chunk
// the exponent, and every term, is the one-pass gridding's.
struct SpecState {
  int ev;
  int redo;
};
__global__ void k_spec_scale(const ValueBound* values, int first, int unit, unsigned long long nvis, int integer,
                             int wide, SpecState* st, FixScale* fs) {
  const int ev = bound_exponent(values, unit);
  if (first || ev != st->ev) {
    st->redo = first ? 0 : 1;
    st->ev = ev;
    *fs = scale_of(ev, nvis, integer, wide);
  } else {
    st->redo = 0;
  }
}

// Zeroes n planes' rows as zero_touched does, when *flag is set.
template <class Cell>
__global__ void k_zero_touched_if(const int* __restrict__ flag, Cell* __restrict__ grids, int n, int nu, int nv,
                                  int rows) {
  if (*flag == 0) return;
  const uint64_t prow = rows == 0 ? (uint64_t)nu : 2ull * rows;  // rows cleared per plane
  const uint64_t total = (uint64_t)n * prow * nv;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = i / (prow * nv), r = (i / nv) % prow, c = i % nv;
    const uint64_t row = (rows == 0 || r < (uint64_t)rows) ? r : (uint64_t)nu - 2ull * rows + r;
    grids[(p * nu + row) * nv + c] = Cell{};
  }
}

__device__ __forceinline__ void fix_add(FixCell* cell, long long re, long long im) {
  if (re) atomicAdd(reinterpret_cast<unsigned long long*>(&cell->re), (unsigned long long)re);
  if (im) atomicAdd(reinterpret_cast<unsigned long long*>(&cell->im), (unsigned long long)im);
}

// A double-precision grid value in fixed point: hi * 2^32 + lo, two int64
// words, and a complex cell of two of them. A term, x * 2^q rounded once to
// an integer t, is split as t_hi = floor(t / 2^32) and t_lo = t - t_hi 2^32 in
// [0, 2^32]; the words sum their parts independently, so adding a term is two
// integer adds that need no carry and no returned value (red.global.add),
// exact in any order. lo stays below 2^63 for fewer than 2^31 terms per cell
// (runs, not visibilities, are the terms), hi below 2^62 by the scale's
// headroom (k_fix_scale).
struct FixWide {
  long long lo, hi;
};
struct FixCell2 {
  FixWide re, im;
};

__device__ __forceinline__ void fix_add_wide(FixWide* cell, FixWide v) {
  if (v.lo) atomicAdd(reinterpret_cast<unsigned long long*>(&cell->lo), (unsigned long long)v.lo);
  if (v.hi) atomicAdd(reinterpret_cast<unsigned long long*>(&cell->hi), (unsigned long long)v.hi);
}

// The fixed-point cell and accumulator of each working precision.
template <class T>
struct FixTraits;
template <>
struct FixTraits<float> {
  using Cell = FixCell;
  using Acc = long long;
  static constexpr int wide = 0;
  // x * 2^q rounded to an integer (sc = 2^q)
  static __device__ __forceinline__ float scale(int q) { return ldexpf(1.0f, q); }
  static __device__ __forceinline__ Acc term(float x, float sc) { return __float2ll_rn(x * sc); }
  static __device__ __forceinline__ Acc zero() { return 0; }
  static __device__ __forceinline__ Acc add(Acc a, Acc b) { return a + b; }
  static __device__ __forceinline__ bool nonzero(Acc a) { return a != 0; }
  static __device__ __forceinline__ void flush(Cell* c, Acc re, Acc im) { fix_add(c, re, im); }
  static __device__ __forceinline__ double value(long long v, int q) { return ldexp((double)v, -q); }
};
template <>
struct FixTraits<double> {
  using Cell = FixCell2;
  using Acc = FixWide;
  static constexpr int wide = 1;
  // sc = 2^(q - 32): y = x * sc (exact), hi = floor(y) (exact; every double
  // from 2^52 up is an integer), lo = rint((y - hi) 2^32) (the fraction is
  // exact, the one rounding is to the grid's unit).
  static __device__ __forceinline__ double scale(int q) { return ldexp(1.0, q - 32); }
  static __device__ __forceinline__ Acc term(double x, double sc) {
    const double y = x * sc, h = floor(y);
    return FixWide{__double2ll_rn((y - h) * 4294967296.0), __double2ll_rn(h)};
  }
  static __device__ __forceinline__ Acc zero() { return FixWide{0ll, 0ll}; }
  static __device__ __forceinline__ Acc add(Acc a, Acc b) { return FixWide{a.lo + b.lo, a.hi + b.hi}; }
  static __device__ __forceinline__ bool nonzero(Acc a) { return (a.lo | a.hi) != 0; }
  static __device__ __forceinline__ void flush(Cell* c, Acc re, Acc im) {
    fix_add_wide(&c->re, re);
    fix_add_wide(&c->im, im);
  }
  static __device__ __forceinline__ double value(FixWide v, int q) {
    return ldexp((double)v.hi, 32 - q) + ldexp((double)v.lo, -q);
  }
};

// One plane of the fixed-point grid to floating point: rows [0, rows) and
// [nu - rows, nu) (every row when rows is 0), each cell rounded once.
template <class T>
__global__ void k_fix_to_plane(const typename FixTraits<T>::Cell* __restrict__ fix, int nu, int nv, int rows,
                               const FixScale* fs, cplx<T>* __restrict__ out) {
  const int q = fs->q;
  const bool nan = fs->nonfinite != 0;
  const int nr = rows == 0 ? nu : 2 * rows;
  const uint64_t n = (uint64_t)nr * nv;
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < n; c += (uint64_t)gridDim.x * blockDim.x) {
    const int r = (int)(c / nv);
    const uint64_t cell = (uint64_t)(rows == 0 || r < rows ? r : nu - 2 * rows + r) * nv + (c - (uint64_t)r * nv);
    const auto f = fix[cell];
    cplx<T> v;
    if (nan) {
      v = {(T)__longlong_as_double(0x7ff8000000000000ll), (T)__longlong_as_double(0x7ff8000000000000ll)};
    } else {
      v = {(T)FixTraits<T>::value(f.re, q), (T)FixTraits<T>::value(f.im, q)};
    }
    out[cell] = v;
  }
}

// ------------------------------------------------------------------ records

struct VisRecord {
  float x0, y0, xw;  // tap arguments (taps_uv, w_factor's locz of the first plane)
  uint32_t idx;      // visibility index, row * nchan + channel
  float ph_re, ph_im;  // shift phase (shift_phase with sign +1), (1, 0) without shifts
  uint32_t meta;     // du | dv << 4 | (w was flipped) << 8 | first plane << 16
  uint32_t bin;      // the sorted key (chunk * nbins + bin)
};
static_assert(sizeof(VisRecord) == 32, "records are one 32-byte sector");

// The loads of one visibility of the count pass: its word of the scan's
// active bits, its row's coordinates and its channel's f / c, issued an
// iteration ahead of their use (the pass otherwise waited on them).
struct CountIn {
  uint32_t word = 0;
  double4 b = {0.0, 0.0, 0.0, 1.0};  // the row's coordinates and sign (k_row_coords)
  double f = 0.0;
};
__device__ __forceinline__ CountIn count_in(const uint32_t* __restrict__ bits, const double4* __restrict__ rowc,
                                            const double* __restrict__ foc, uint64_t i, uint32_t row, uint32_t ch) {
  CountIn c;
  c.word = bits[i >> 5];
  c.b = rowc[row];
  c.f = foc[ch];
  return c;
}

// Each row's coordinates as the binning uses them (row_coord: flips,
// recentring, w made non-negative) and the sign of that flip, once per row:
// the count pass then reads them instead of forming them for every channel
// (the same doubles, so the same keys and records).
__global__ void k_row_coords(uint64_t nrow, const double* __restrict__ uvw, double fu, double fv, double fw,
                             double r_l, double r_m, double4* __restrict__ out) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < nrow;
       r += (uint64_t)gridDim.x * blockDim.x) {
    double b[3];
    const double sgn = row_coord(uvw, r, fu, fv, fw, r_l, r_m, b);
    out[r] = make_double4(b[0], b[1], b[2], sgn);
  }
}

// The count pass of the counting sort (k_bin_count) for single precision,
// writing as well the record of each active visibility at its own index
// (coalesced): its coordinates and taps' arguments are formed here once. The
// scatter then moves only the 4-byte indices, and the gridder and degridder
// read each record through the sorted index. The active set comes from the
// scan's bits (bit i: visibility i), one word per 32 visibilities. The
// plan's uniform choices (w-planes, phase shift, row chunks) are template
// arguments: tested in the loop they cost branches and reloads of the plan's
// constants on every visibility. Three blocks per SM (at most 85 registers)
// measured 9.20 ms per call at 1.06 G visibilities, four 9.32, five 9.61.
constexpr int COUNT_BLOCKS = 3;
template <bool WPL, bool SHIFT, bool CHUNKED>
__global__ void __launch_bounds__(256, COUNT_BLOCKS)
    k_bin_count_rec(const __grid_constant__ Geom<float> g, const double4* __restrict__ rowc,
                    const double* __restrict__ foc, const uint32_t* __restrict__ bits, uint32_t* __restrict__ key,
                    uint32_t* __restrict__ counts, VisRecord* __restrict__ rec, uint32_t rows_per_chunk,
                    uint32_t nbins, uint64_t i0, uint64_t n, uint32_t koff) {
  // Visibilities [i0, n); bin k is counted in counts[k - koff].
  const uint64_t nround = i0 + ((n - i0 + 31) & ~31ull);
  const uint32_t tmask = (1u << g.log2tile) - 1u;
  const uint32_t se = (uint32_t)g.sube, sdiv = (65536u + se - 1u) / se;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t i = i0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  RowCh rc(i, (uint32_t)g.nchan, stride);
  CountIn cur = i < n ? count_in(bits, rowc, foc, i, rc.row, rc.ch) : CountIn{};
  for (; i < nround; i += stride) {
    RowCh nrc = rc;
    nrc.next((uint32_t)g.nchan);
    const CountIn nxt = i + stride < n ? count_in(bits, rowc, foc, i + stride, nrc.row, nrc.ch) : CountIn{};
    bool act = false;
    uint32_t k = INACTIVE;
    if (i < n) {
      act = ((cur.word >> (i & 31)) & 1u) != 0;
      if (act) {
        const double b[3] = {cur.b.x, cur.b.y, cur.b.z};
        const double imflip = cur.b.w;
        const double f = cur.f;
        const double u = b[0] * f, v = b[1] * f, w = b[2] * f;
        double uf, vf;
        int iu0, iv0;
        getpix(g, u, v, uf, vf, iu0, iv0);
        const uint32_t su = (uint32_t)shifted(iu0, g.nu), sv = (uint32_t)shifted(iv0, g.nv);
        // (x / sube) for x < 32 as a multiply and shift (exact: the error of
        // ceil(2^16 / sube) stays below 2^-11 over 32 steps)
        const uint32_t sa = ((su & tmask) * sdiv) >> 16, sb = ((sv & tmask) * sdiv) >> 16;
        const int mp = WPL ? minplane(g, w) : 0;
        // The key of bin_of_rc (Setup::locate refined by the sub-tile).
        k = (((su >> g.log2tile) * (uint32_t)g.ntv + (sv >> g.log2tile)) * (uint32_t)g.nbuckets + (uint32_t)mp) *
                (uint32_t)g.nsub + sa * (uint32_t)g.nsub_side + sb;
        if (CHUNKED) k += (rc.row / rows_per_chunk) * nbins;
        // The record's two 16-byte halves, formed in registers (VisRecord's
        // field order).
        const double s1 = (double)g.supp - 1.0;
        const float x0 = (float)(-uf * 2.0 + s1);
        const float y0 = (float)(-vf * 2.0 + s1);
        float xw = 0.0f;
        if (WPL) {  // w_factor's argument for the first plane (nth 0)
          const float z = (float)(g.xdw * ((g.wmin + (double)mp * g.dw) - w));
          xw = z * 2.0f + (float)s1;
        }
        float ph_re = 1.0f, ph_im = 0.0f;
        if (SHIFT) {
          const cplx<float> ph = shift_phase<float>(g, b, imflip, f, 1.0);
          ph_re = ph.re;
          ph_im = ph.im;
        }
        const uint32_t meta = ((su & tmask) - sa * se) | (((sv & tmask) - sb * se) << 4) |
                              (imflip < 0.0 ? 256u : 0u) | ((uint32_t)mp << 16);
        reinterpret_cast<uint4*>(rec + i)[0] =
            make_uint4(__float_as_uint(x0), __float_as_uint(y0), __float_as_uint(xw), (uint32_t)i);
        reinterpret_cast<uint4*>(rec + i)[1] = make_uint4(__float_as_uint(ph_re), __float_as_uint(ph_im), meta, k);
      }
      key[i] = k;
    }
    warp_aggregated_count(counts, k - koff, act);
    cur = nxt;
    rc = nrc;
  }
}

// The taps of one axis at x (the reference's eval_taps, one of the two axes
// of eval_taps2).
template <int S>
__device__ __forceinline__ void eval_taps1(const float* __restrict__ c, float x, float* r) {
  constexpr int ne = coeff_rows(S);
  constexpr int H = (S + 1) / 2;
  const float x2 = x * x;
  float e[H], o[H];
#pragma unroll
  for (int i = 0; i < H; i++) {
    e[i] = c[i];
    o[i] = c[ne * S + i];
  }
#pragma unroll
  for (int k = 1; k < ne; k++)
#pragma unroll
    for (int i = 0; i < H; i++) {
      e[i] = fmaf(e[i], x2, c[k * S + i]);
      o[i] = fmaf(o[i], x2, c[(ne + k) * S + i]);
    }
#pragma unroll
  for (int i = 0; i < H; i++) r[i] = fmaf(o[i], x, e[i]);
#pragma unroll
  for (int i = 0; i < S - H; i++) r[S - 1 - i] = fmaf(o[i], -x, e[i]);
}

// The stored value of a record's visibility (unit_value, data_value,
// wgridder.rs:1414-1435): value = vis * phase * wgt with the imaginary part
// negated where w was flipped; the phase alone times wgt for unit values.
__device__ __forceinline__ cplx<float> record_value(const VisRecord& r, const Inputs& in, int mode) {
  const float flip = (r.meta & 256u) ? -1.0f : 1.0f;
  float pr = r.ph_re, pi = r.ph_im;
  if (in.wgt_kind != WGT_NONE) {
    const float w = wgt_get<float>(in, r.idx);
    pr *= w;
    pi *= w;
  }
  if (mode == VALUE_DATA) {
    const cplx<float> v = vis_get<float>(in, r.idx);
    const float dr = v.re * pr - v.im * pi, di = v.re * pi + v.im * pr;
    return {dr, di * flip};
  }
  return {pr, pi * flip};
}

// The window of a bin key: the grid row and column of its cell (0, 0) (the
// sub-tile's first cell; windows are 8 x 8) and its first plane.
template <class T>
__device__ __forceinline__ void window_of(const Geom<T>& g, uint32_t key, uint32_t nbins, int& su0, int& sv0,
                                          int& mp) {
  const uint32_t bin = key % nbins;
  const uint32_t sub = bin % (uint32_t)g.nsub, t = bin / (uint32_t)g.nsub;
  mp = (int)(t % (uint32_t)g.nbuckets);
  const uint32_t tile = t / (uint32_t)g.nbuckets;
  const uint32_t tu = tile / (uint32_t)g.ntv, tv = tile - tu * (uint32_t)g.ntv;
  // Tiles are laid out on the shifted indices (i0 + n/2) mod n; the grid is
  // stored unshifted.
  su0 = (int)(((tu << g.log2tile) + (sub / (uint32_t)g.nsub_side) * (uint32_t)g.sube + (uint32_t)(g.nu - g.nu / 2)) %
              (uint32_t)g.nu);
  sv0 = (int)(((tv << g.log2tile) + (sub % (uint32_t)g.nsub_side) * (uint32_t)g.sube + (uint32_t)(g.nv - g.nv / 2)) %
              (uint32_t)g.nv);
}

// The taps t[0..S) placed at rows [off, off + S) of an 8-row window, zero
// elsewhere, in registers (off < 9 - S is a runtime value, the candidates
// compile-time: selects instead of indexed stores).
template <int S, class V>
__device__ __forceinline__ void place8(const V (&t)[S], int off, V zero, V (&row)[8]) {
#pragma unroll
  for (int j = 0; j < 8; j++) {
    V x = zero;
#pragma unroll
    for (int d = 0; d < 9 - S; d++)
      if (j - d >= 0 && j - d < S && off == d) x = t[(j - d >= 0 && j - d < S) ? j - d : 0];
    row[j] = x;
  }
}

// ------------------------------------------------------------------ integer gridder

// ------------------------------------------------------------------ prefetch

// The inputs of one staged record, copied asynchronously (cp.async) into
// shared memory a round ahead of their use, so that the gathers of records,
// visibilities and weights are in flight while the previous round is
// contracted and take no registers.
struct Prefetched {
  uint4 rec[2];  // the record
  uint4 vis;     // the visibility: complex64 in .x, .y or complex128
  uint2 wgt;     // the weight: float32 in .x, float64, or the two float32 factors
};

__device__ __forceinline__ void cp_async(void* dst, const void* src, int bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if (bytes == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
  else if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Starts the copies of record `idx` (at sorted position k) and (with_vis,
// with_wgt) its value's inputs.
__device__ __forceinline__ void prefetch(Prefetched* dst, const VisRecord* __restrict__ rec, const Inputs& in,
                                         bool with_vis, bool with_wgt, uint32_t idx, uint64_t k) {
  const uint4* r = reinterpret_cast<const uint4*>(rec + idx);
  cp_async(&dst->rec[0], r, 16);
  cp_async(&dst->rec[1], r + 1, 16);
  if (with_vis) {
    if (in.vis_kind == VIS_SORTED)
      cp_async(&dst->vis, reinterpret_cast<const float2*>(in.vis) + k, 8);
    else if (in.vis_kind == VIS_C64)
      cp_async(&dst->vis, reinterpret_cast<const float2*>(in.vis) + idx, 8);
    else if (in.vis_kind == VIS_C128)
      cp_async(&dst->vis, reinterpret_cast<const double2*>(in.vis) + idx, 16);
  }
  if (with_wgt) {
    if (in.wgt_kind == WGT_F64) {
      cp_async(&dst->wgt, reinterpret_cast<const double*>(in.wgt) + idx, 8);
    } else if (in.wgt_kind == WGT_F32 || in.wgt_kind == WGT_F32_PRODUCT) {
      cp_async(&dst->wgt.x, reinterpret_cast<const float*>(in.wgt) + idx, 4);
      if (in.wgt_kind == WGT_F32_PRODUCT) cp_async(&dst->wgt.y, reinterpret_cast<const float*>(in.wgt2) + idx, 4);
    }
  }
}

__device__ __forceinline__ VisRecord prefetched_record(const Prefetched& p) {
  const uint4 a = p.rec[0], b = p.rec[1];
  return VisRecord{__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z), a.w,
                   __uint_as_float(b.x), __uint_as_float(b.y), b.z, b.w};
}
// Weights::get and VisData::get (wgridder.rs:950-1005) of the copied values.
__device__ __forceinline__ float prefetched_wgt(const Prefetched& p, const Inputs& in) {
  switch (in.wgt_kind) {
    case WGT_F32:
      return __uint_as_float(p.wgt.x);
    case WGT_F64:
      return (float)__longlong_as_double((long long)(((unsigned long long)p.wgt.y << 32) | p.wgt.x));
    case WGT_F32_PRODUCT:
      return __uint_as_float(p.wgt.x) * __uint_as_float(p.wgt.y);
    default:
      return 1.0f;
  }
}
__device__ __forceinline__ cplx<float> prefetched_vis(const Prefetched& p, const Inputs& in) {
  if (in.vis_kind == VIS_C64 || in.vis_kind == VIS_SORTED) return {__uint_as_float(p.vis.x), __uint_as_float(p.vis.y)};
  if (in.vis_kind == VIS_C128)
    return {(float)__longlong_as_double((long long)(((unsigned long long)p.vis.y << 32) | p.vis.x)),
            (float)__longlong_as_double((long long)(((unsigned long long)p.vis.w << 32) | p.vis.z))};
  return {1.0f, 0.0f};
}

// ------------------------------------------------------------------ integer gridder

constexpr int I8_BATCH = 32;         // records staged per round, one per lane
constexpr uint32_t I8_CHUNK = 8192;  // sorted records per warp
constexpr float I8_ASCALE = 4194304.0f;  // 2^22
// A's integers (w tap x u tap x 2^22, in [-2^16, 2^22 (1 + eps)]) are formed
// without a conversion instruction: y = x + 2^23 + 2^16 + 0x8080 lies in
// (2^23, 2^24), where FP32 spacing is 1, so the FFMA that forms x rounds it
// to the nearest integer, and the bits of y are 0x4B010000 + rint(x) +
// 0x8080: one IADD gives rint(x) with the offset the balanced limbs need.
constexpr float I8_AOFF = 8487040.0f;      // 2^23 + 2^16 + 0x8080
constexpr uint32_t I8_ABIAS = 0x4B010000u;  // bits of 2^23 + 2^16
__device__ __forceinline__ uint32_t i8_aint(float y) { return __float_as_uint(y) - I8_ABIAS; }
// Row strides (words) of the staging rows: with them the reads of the eight
// records of a lane quad (slots 4 tq + j) fall in distinct banks.
constexpr int I8_KU = 10;   // u taps placed on the window's 8 rows
constexpr int I8_B = 9;     // uint2: rint(value * placed v taps * 2^sb) + 0x8080 on the 8 columns
constexpr int I8_KW = 10;   // w taps * 2^22 (8), as float2 pairs of planes

// Staging of one round: per slot (record) the u taps and value * v taps
// placed on the window's rows and columns (zero, or the offset, elsewhere),
// the w taps times 2^22 and the key. Slot I8_BATCH stays zero.
struct I8Slots {
  float* ku;      // [I8_BATCH + 1][I8_KU]
  uint2* bv;      // [I8_BATCH + 1][I8_B]
  float* kw;      // [I8_BATCH + 1][I8_KW]
  uint32_t* key;  // [I8_BATCH + 1]
  __host__ __device__ static constexpr size_t bytes() {
    return ((size_t)(I8_BATCH + 1) * (I8_B * 8 + I8_KU * 4 + I8_KW * 4 + 4) + 15) / 16 * 16;
  }
  // bv and kw are read as float2: both start on 8-byte boundaries.
  __device__ void carve(unsigned char* base) {
    bv = reinterpret_cast<uint2*>(base);
    kw = reinterpret_cast<float*>(bv + (I8_BATCH + 1) * I8_B);
    ku = kw + (I8_BATCH + 1) * I8_KW;
    key = reinterpret_cast<uint32_t*>(ku + (I8_BATCH + 1) * I8_KU);
  }
};

// Three balanced 8-bit limbs of four integers y - 0x8080 (y = x + 0x8080,
// |x| < 2^22 + 2^15), packed per limb (byte j of limb register L holds limb
// L of x[j]): bytes 0 and 1 of y are the low limbs plus 128, y >> 16 (byte 2
// of y, as a signed byte) is the top limb.
__device__ __forceinline__ void limbs4(uint32_t y0, uint32_t y1, uint32_t y2, uint32_t y3, uint32_t& l0, uint32_t& l1,
                                       uint32_t& l2) {
  const uint32_t a01 = __byte_perm(y0, y1, 0x5140), a23 = __byte_perm(y2, y3, 0x5140);  // b0 b0' b1 b1'
  l0 = __byte_perm(a01, a23, 0x5410) ^ 0x80808080u;
  l1 = __byte_perm(a01, a23, 0x7632) ^ 0x80808080u;
  l2 = __byte_perm(__byte_perm(y0, y1, 0x0062), __byte_perm(y2, y3, 0x0062), 0x5410);
}

__device__ __forceinline__ void imma(int (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                     uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k32.row.col.s32.s8.s8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Adds a bin's exact window sums to the fixed-point grid. acc[h][c][g][r]:
// plane pair h, component c (re, im), limb group g (weights 2^32, 2^24,
// 2^16: the grid unit is 2^16 of the products), fragment element r (rows
// gq / gq + 8 are planes 2h / 2h + 1 at window row gq; columns 2tq, 2tq + 1).
template <int NP>
__device__ __forceinline__ void i8_flush(const Geom<float>& g, FixCell* __restrict__ grids, int pg0, int npg,
                                         int su0, int sv0, int mp, const int (&acc)[NP][2][3][4]) {
  const int lane = threadIdx.x & 31, gq = lane >> 2, tq = lane & 3;
  const size_t plane = (size_t)g.nu * g.nv;
  int row = su0 + gq;
  if (row >= g.nu) row -= g.nu;
#pragma unroll
  for (int h = 0; h < NP; h++)
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int p = mp + 2 * h + (r >> 1);
      const long long re = ((long long)acc[h][0][0][r] << 16) + ((long long)acc[h][0][1][r] << 8) + acc[h][0][2][r];
      const long long im = ((long long)acc[h][1][0][r] << 16) + ((long long)acc[h][1][1][r] << 8) + acc[h][1][2][r];
      if ((re | im) == 0 || p < pg0 || p >= pg0 + npg) continue;
      int col = sv0 + 2 * tq + (r & 1);
      if (col >= g.nv) col -= g.nv;
      fix_add(grids + (size_t)(p - pg0) * plane + (size_t)row * g.nv + col, re, im);
    }
}

// Gridding of records [kbase, kend) (single precision): each warp takes
// I8_CHUNK consecutive sorted records, stages I8_BATCH at a time, and per run
// of one bin forms the integer limbs of A (rows: w tap x placed u tap of
// planes 2h and 2h + 1, columns: the run's records) and B (rows: records,
// columns: value x placed v tap) and adds their limb products into int32
// fragments on the tensor cores; at the end of a bin the fragments are
// combined into int64 and added to the grid. Records outside the run read
// the zero slot. The next round's records and values are loaded while the
// current round is contracted.
template <int S>
__global__ void __launch_bounds__(I8_BATCH, S <= 4 ? 16 : S <= 6 ? 12 : 8)
    k_grid_i8(const __grid_constant__ Geom<float> g, Inputs in, int mode, const VisRecord* __restrict__ rec,
              const uint32_t* __restrict__ sorted, uint64_t kbase, uint64_t kend, uint32_t nbins,
              FixCell* __restrict__ grids, int pg0, int npg, FixScale* __restrict__ fs,
              const int* __restrict__ run) {
  static_assert(S >= 1 && S <= 8, "8 x 8 windows");
  if (run && *run == 0) return;  // a speculative pass's regridding, not needed
  constexpr int NP = (S + 1) / 2;  // plane pairs
  extern __shared__ __align__(16) unsigned char smem[];
  I8Slots st;
  st.carve(smem);
  const int lane = threadIdx.x, gq = lane >> 2, tq = lane & 3;
  {  // the zero slot: u and w taps 0, B rows at the offset (value 0)
    float* zk = st.ku + I8_BATCH * I8_KU;
    uint2* zb = st.bv + I8_BATCH * I8_B;
    float* zw = st.kw + I8_BATCH * I8_KW;
    if (lane < I8_KU) zk[lane] = 0.0f;
    if (lane < I8_B) zb[lane] = make_uint2(0x8080u, 0x8080u);
    if (lane < I8_KW) zw[lane] = 0.0f;
    if (lane == 0) st.key[I8_BATCH] = INACTIVE;
  }
  const uint64_t k0 = kbase + (uint64_t)blockIdx.x * I8_CHUNK;
  const uint64_t k1 = min(kend, k0 + I8_CHUNK);
  const float bscale = ldexpf(1.0f, fs->sb);
  bool bad = false;

  int acc[NP][2][3][4];
#pragma unroll
  for (int h = 0; h < NP; h++)
#pragma unroll
    for (int c = 0; c < 2; c++)
#pragma unroll
      for (int q = 0; q < 3; q++)
#pragma unroll
        for (int r = 0; r < 4; r++) acc[h][c][q][r] = 0;
  uint32_t gcur = INACTIVE;
  int su0 = 0, sv0 = 0, mpc = 0;

  // Rounds ahead: this round's inputs are in pre (copied asynchronously),
  // nidx is the next round's index.
  Prefetched* pre = reinterpret_cast<Prefetched*>(smem + I8Slots::bytes()) + lane;
  const bool with_vis = mode == VALUE_DATA && in.vis_kind != VIS_UNIT, with_wgt = in.wgt_kind != WGT_NONE;
  if (k0 + lane < k1) prefetch(pre, rec, in, with_vis, with_wgt, sorted[k0 + lane], k0 + lane);
  cp_async_commit();
  uint32_t nidx = (k0 + I8_BATCH + lane < k1) ? sorted[k0 + I8_BATCH + lane] : 0u;

  for (uint64_t kb = k0; kb < k1; kb += I8_BATCH) {
    const int nb = (int)min((uint64_t)I8_BATCH, k1 - kb);
    cp_async_wait_all();
    __syncwarp();
    if (lane < nb) {  // staging, one record per lane
      const VisRecord r = prefetched_record(*pre);
      const float wt = prefetched_wgt(*pre, in);
      const cplx<float> vv = with_vis ? prefetched_vis(*pre, in) : cplx<float>{1.0f, 0.0f};
      float ku[S], kv[S], kw[S];
      eval_taps2<float, S>(g.coeff, g.ne, r.x0, r.y0, ku, kv);
      if (g.do_wgridding) eval_taps1<S>(g.coeff, r.xw, kw);
      // record_value: value = vis * phase * wgt, imaginary part negated where w was flipped.
      const float flip = (r.meta & 256u) ? -1.0f : 1.0f;
      const float pr = r.ph_re * wt, pi = r.ph_im * wt;
      const float vr = vv.re * pr - vv.im * pi, vi = (vv.re * pi + vv.im * pr) * flip;
      bad |= !isfinite(vr) || !isfinite(vi) || !isfinite(r.x0) || !isfinite(r.y0) || !isfinite(r.xw);
      const int mp = (int)(r.meta >> 16), du = (int)(r.meta & 15u), dv = (int)((r.meta >> 4) & 15u);
      const float br = vr * bscale, bi = vi * bscale;
      uint2 bt[S];
#pragma unroll
      for (int i = 0; i < S; i++)
        bt[i] = make_uint2((uint32_t)(__float2int_rn(br * kv[i]) + 0x8080), (uint32_t)(__float2int_rn(bi * kv[i]) + 0x8080));
      float urow[8];
      uint2 brow[8];
      place8<S>(ku, du, 0.0f, urow);
      place8<S>(bt, dv, make_uint2(0x8080u, 0x8080u), brow);
      float wrow[8];
#pragma unroll
      for (int j = 0; j < 8; j++) {
        float w = 0.0f;
        if (g.do_wgridding) {
          if (j < S && mp + j >= pg0 && mp + j < pg0 + npg) w = kw[j < S ? j : 0] * I8_ASCALE;
        } else if (j == 0) {
          w = I8_ASCALE;
        }
        wrow[j] = w;
      }
      float2* cu = reinterpret_cast<float2*>(st.ku + lane * I8_KU);
      uint2* cb = st.bv + lane * I8_B;
      float2* cw = reinterpret_cast<float2*>(st.kw + lane * I8_KW);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        cu[j] = make_float2(urow[2 * j], urow[2 * j + 1]);
        cw[j] = make_float2(wrow[2 * j], wrow[2 * j + 1]);
      }
#pragma unroll
      for (int j = 0; j < 8; j++) cb[j] = brow[j];
      st.key[lane] = r.bin;
    }
    // The next round's record and value, in flight while this one is contracted.
    __syncwarp();
    if (kb + I8_BATCH + lane < k1) prefetch(pre, rec, in, with_vis, with_wgt, nidx, kb + I8_BATCH + lane);
    cp_async_commit();
    if (kb + 2 * I8_BATCH + lane < k1) nidx = sorted[kb + 2 * I8_BATCH + lane];
    int q = 0;
    while (q < nb) {
      const uint32_t gk = st.key[q];
      if (gk != gcur) {
        if (gcur != INACTIVE) i8_flush<NP>(g, grids, pg0, npg, su0, sv0, mpc, acc);
#pragma unroll
        for (int h = 0; h < NP; h++)
#pragma unroll
          for (int c = 0; c < 2; c++)
#pragma unroll
            for (int qq = 0; qq < 3; qq++)
#pragma unroll
              for (int r = 0; r < 4; r++) acc[h][c][qq][r] = 0;
        gcur = gk;
        window_of(g, gk, nbins, su0, sv0, mpc);
      }
      // The run: slots [q, q + len) of bin gk.
      const unsigned m = __ballot_sync(0xffffffffu, lane >= q && lane < nb && st.key[lane] == gk);
      const int len = __popc(m);
      // This lane's eight records: k = 4tq + j and 16 + 4tq + j, j < 4.
      int slot[8];
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int k = (j < 4 ? 4 * tq : 16 + 4 * tq) + (j & 3);
        slot[j] = (k >= q && k < q + len) ? k : I8_BATCH;
      }
      float kuv[8];
      uint32_t b[2][3][2];  // B limbs per component: registers for k 4tq.. and 16 + 4tq..
#pragma unroll
      for (int hf = 0; hf < 2; hf++) {
        uint2 bvv[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
          kuv[4 * hf + j] = st.ku[slot[4 * hf + j] * I8_KU + gq];
          bvv[j] = st.bv[slot[4 * hf + j] * I8_B + gq];
        }
        limbs4(bvv[0].x, bvv[1].x, bvv[2].x, bvv[3].x, b[0][0][hf], b[0][1][hf], b[0][2][hf]);
        limbs4(bvv[0].y, bvv[1].y, bvv[2].y, bvv[3].y, b[1][0][hf], b[1][1][hf], b[1][2][hf]);
      }
#pragma unroll
      for (int h = 0; h < NP; h++) {
        uint32_t a[3][4];  // per limb: rows gq (plane 2h), gq + 8 (plane 2h + 1) x k halves
#pragma unroll
        for (int hf = 0; hf < 2; hf++) {
          float2 w[4];
#pragma unroll
          for (int j = 0; j < 4; j++)
            w[j] = 2 * h < S ? *reinterpret_cast<const float2*>(st.kw + slot[4 * hf + j] * I8_KW + 2 * h)
                             : make_float2(0.0f, 0.0f);
          limbs4(i8_aint(fmaf(w[0].x, kuv[4 * hf], I8_AOFF)), i8_aint(fmaf(w[1].x, kuv[4 * hf + 1], I8_AOFF)),
                 i8_aint(fmaf(w[2].x, kuv[4 * hf + 2], I8_AOFF)), i8_aint(fmaf(w[3].x, kuv[4 * hf + 3], I8_AOFF)),
                 a[0][2 * hf], a[1][2 * hf], a[2][2 * hf]);
          limbs4(i8_aint(fmaf(w[0].y, kuv[4 * hf], I8_AOFF)), i8_aint(fmaf(w[1].y, kuv[4 * hf + 1], I8_AOFF)),
                 i8_aint(fmaf(w[2].y, kuv[4 * hf + 2], I8_AOFF)), i8_aint(fmaf(w[3].y, kuv[4 * hf + 3], I8_AOFF)),
                 a[0][2 * hf + 1], a[1][2 * hf + 1], a[2][2 * hf + 1]);
        }
#pragma unroll
        for (int c = 0; c < 2; c++) {
          // weight 2^32: a2 b2; 2^24: a2 b1 + a1 b2; 2^16: a2 b0 + a1 b1 + a0 b2
          imma(acc[h][c][0], a[2][0], a[2][1], a[2][2], a[2][3], b[c][2][0], b[c][2][1]);
          imma(acc[h][c][1], a[2][0], a[2][1], a[2][2], a[2][3], b[c][1][0], b[c][1][1]);
          imma(acc[h][c][1], a[1][0], a[1][1], a[1][2], a[1][3], b[c][2][0], b[c][2][1]);
          imma(acc[h][c][2], a[2][0], a[2][1], a[2][2], a[2][3], b[c][0][0], b[c][0][1]);
          imma(acc[h][c][2], a[1][0], a[1][1], a[1][2], a[1][3], b[c][1][0], b[c][1][1]);
          imma(acc[h][c][2], a[0][0], a[0][1], a[0][2], a[0][3], b[c][2][0], b[c][2][1]);
        }
      }
      q += len;
    }
  }
  if (gcur != INACTIVE) i8_flush<NP>(g, grids, pg0, npg, su0, sv0, mpc, acc);
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&fs->nonfinite, 1);
}

// ------------------------------------------------------------------ tensor-core degridder

constexpr int H16_BATCH = 32;
constexpr uint32_t H16_CHUNK = 8192;
constexpr float H16_BSCALE = 16384.0f;  // 2^14: v taps stay clear of FP16 subnormals
constexpr int H16_KU = 10;  // u taps placed on the window's 8 rows (read as float2)
constexpr int H16_KV = 10;  // v taps * 2^14 placed on the 8 columns (read as float2)
constexpr int H16_KW = 12;  // w taps (8, read as float4)

struct H16Slots {
  float4* out;    // [H16_BATCH + 1]: conj(phase) * wgt (re, im), imflip, index bits
  float* kw;      // [H16_BATCH + 1][H16_KW]: w taps (zero outside the pass's planes)
  float* kv;      // [H16_BATCH + 1][H16_KV]
  float* ku;      // [H16_BATCH + 1][H16_KU]
  uint32_t* key;  // [H16_BATCH + 1]
  __host__ __device__ static constexpr size_t bytes() {
    return ((size_t)(H16_BATCH + 1) * (16 + H16_KW * 4 + H16_KV * 4 + H16_KU * 4 + 4) + 15) / 16 * 16;
  }
  // out and kw are read as float4, kv and ku as float2: their offsets are aligned.
  __device__ void carve(unsigned char* base) {
    out = reinterpret_cast<float4*>(base);
    kw = reinterpret_cast<float*>(out + (H16_BATCH + 1));
    kv = kw + (H16_BATCH + 1) * H16_KW;
    ku = kv + (H16_BATCH + 1) * H16_KV;
    key = reinterpret_cast<uint32_t*>(ku + (H16_BATCH + 1) * H16_KU);
  }
};

// (x0, x1) as FP16 hi + lo (x - hi is exact in FP32; lo rounds it to FP16).
__device__ __forceinline__ void split_h2(float x0, float x1, uint32_t& hi, uint32_t& lo) {
  const __half2 h = __floats2half2_rn(x0, x1);
  const float2 hf = __half22float2(h);
  const __half2 l = __floats2half2_rn(x0 - hf.x, x1 - hf.y);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

__device__ __forceinline__ void hmma_zero(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%7,%7,%7,%7};\n"
      : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
      : "r"(a0), "r"(a1), "r"(b0), "f"(0.0f));
}
__device__ __forceinline__ void hmma(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(b0));
}

// Where the degridder's results go. DEGRID_TO_VIS: vis[visibility index],
// times the weights of the call. The two other modes write the plan's stored
// values, indexed by sorted position, for the gridder to read back
// (Prepared::residual, wgridder.rs:3297-3395): DEGRID_GRAM stores w A x
// (the prediction times the weight of `data`), DEGRID_RESIDUAL stores
// w (d - A x) with d the visibility of `data`; both add w |stored / w|^2 into
// an FP64 partial per block (partials[block0 + block], summed by the warp in
// a fixed order) and the largest |stored| into `bound`.
enum DegridMode : int { DEGRID_TO_VIS = 0, DEGRID_GRAM = 1, DEGRID_RESIDUAL = 2 };
struct DegridOut {
  int mode = DEGRID_TO_VIS;
  cplx<float>* vis = nullptr;     // DEGRID_TO_VIS
  cplx<float>* stored = nullptr;  // the other modes
  Inputs data;                    // weights (and visibilities) of the stored modes
  int sorted_data = 0;            // data and weights by sorted position, not by visibility index
  double* partials = nullptr;
  uint32_t block0 = 0;
  ValueBound* bound = nullptr;
};

// Degridding of records [kbase, kend) (single precision, degrid_task_body,
// wgridder.rs:2793-2901): per bin the warp holds the bin's 8 x 8 window of
// each plane as FP16 hi + lo fragments (scaled by a power of two to the
// window's largest value); per block of sixteen records the v contraction
// T[k][u] = sum_v kv_k[v - dv_k] G_p[u][v] of each plane runs on the tensor
// cores as hi*hi + hi*lo + lo*hi (mma.sync m16n8k8, records along M, window
// rows along N, FP32 accumulation, each block from zero); the u and w
// contractions and the final phase and weight (wgridder.rs:3146-3159) run on
// the CUDA cores, reduced over the four lanes that hold a record's window
// rows. Each output depends only on its own record and the window, so the
// result does not depend on the grouping. With plane groups (first / last)
// the partial sums accumulate in `vis` and the final factor is applied with
// the last group. The next round's records are copied while the current
// round is contracted. `out` says where the results go (DegridOut). Up to
// support 6, 24 warps per SM (80 registers) measured 4 % faster than 16 (122
// registers) and 20 (96), and as fast as 28. The w contraction before the u
// taps and one output lane per record (two lanes of each quad) measured 10 %
// faster than u first and one lane writing both records.
template <int S>
__global__ void __launch_bounds__(H16_BATCH, S <= 6 ? 24 : 12)
    k_degrid_h(const __grid_constant__ Geom<float> g, Inputs wts, const VisRecord* __restrict__ rec,
               const uint32_t* __restrict__ sorted, uint64_t kbase, uint64_t kend, uint32_t nbins,
               const cplx<float>* __restrict__ grids, int pg0, int npg, const __grid_constant__ DegridOut out,
               int first, int last, const uint32_t* __restrict__ kb_ptr, const uint32_t* __restrict__ ke_ptr) {
  static_assert(S >= 1 && S <= 8, "8 x 8 windows");
  if (kb_ptr) {  // a range the device computed: the grid covers its largest size
    kbase = *kb_ptr;
    kend = *ke_ptr;
    if (kbase + (uint64_t)blockIdx.x * H16_CHUNK >= kend) return;
  }
  extern __shared__ __align__(16) unsigned char smem[];
  H16Slots st;
  st.carve(smem);
  const int lane = threadIdx.x, gq = lane >> 2, tq = lane & 3;
  {  // the zero slot
    if (lane < H16_KW) st.kw[H16_BATCH * H16_KW + lane] = 0.0f;
    if (lane < H16_KV) st.kv[H16_BATCH * H16_KV + lane] = 0.0f;
    if (lane < H16_KU) st.ku[H16_BATCH * H16_KU + lane] = 0.0f;
    if (lane == 0) {
      st.key[H16_BATCH] = INACTIVE;
      st.out[H16_BATCH] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
  }
  const uint64_t k0 = kbase + (uint64_t)blockIdx.x * H16_CHUNK;
  const uint64_t k1 = min(kend, k0 + H16_CHUNK);
  const size_t plane = (size_t)g.nu * g.nv;

  uint32_t bhi[S][2], blo[S][2];  // [plane][re/im]: window rows gq, columns 2tq, 2tq + 1
  float inv = 0.0f;               // 1 / (window scale * 2^14)
  uint32_t gcur = INACTIVE;
  double part = 0.0, vmax = 0.0;  // the stored modes' misfit partial and largest |stored|

  Prefetched* pre = reinterpret_cast<Prefetched*>(smem + H16Slots::bytes()) + lane;
  const bool with_wgt = wts.wgt_kind != WGT_NONE;
  if (k0 + lane < k1) prefetch(pre, rec, wts, false, with_wgt, sorted[k0 + lane], k0 + lane);
  cp_async_commit();
  uint32_t nidx = (k0 + H16_BATCH + lane < k1) ? sorted[k0 + H16_BATCH + lane] : 0u;

  for (uint64_t kb = k0; kb < k1; kb += H16_BATCH) {
    const int nb = (int)min((uint64_t)H16_BATCH, k1 - kb);
    cp_async_wait_all();
    __syncwarp();
    if (lane < nb) {
      const VisRecord r = prefetched_record(*pre);
      const float tw = prefetched_wgt(*pre, wts);
      float ku[S], kv[S], kw[S];
      eval_taps2<float, S>(g.coeff, g.ne, r.x0, r.y0, ku, kv);
      if (g.do_wgridding) eval_taps1<S>(g.coeff, r.xw, kw);
      const int mp = (int)(r.meta >> 16), du = (int)(r.meta & 15u), dv = (int)((r.meta >> 4) & 15u);
#pragma unroll
      for (int i = 0; i < S; i++) kv[i] *= H16_BSCALE;
      float urow[8], vrow[8], wrow[8];
      place8<S>(ku, du, 0.0f, urow);
      place8<S>(kv, dv, 0.0f, vrow);
#pragma unroll
      for (int j = 0; j < 8; j++) {
        float w = 0.0f;
        if (g.do_wgridding) {
          if (j < S && mp + j >= pg0 && mp + j < pg0 + npg) w = kw[j < S ? j : 0];
        } else if (j == 0 && pg0 == 0) {
          w = 1.0f;
        }
        wrow[j] = w;
      }
      float2* cu = reinterpret_cast<float2*>(st.ku + lane * H16_KU);
      float2* cv = reinterpret_cast<float2*>(st.kv + lane * H16_KV);
      float4* cw = reinterpret_cast<float4*>(st.kw + lane * H16_KW);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        cu[j] = make_float2(urow[2 * j], urow[2 * j + 1]);
        cv[j] = make_float2(vrow[2 * j], vrow[2 * j + 1]);
      }
      cw[0] = make_float4(wrow[0], wrow[1], wrow[2], wrow[3]);
      cw[1] = make_float4(wrow[4], wrow[5], wrow[6], wrow[7]);
      // The final factor conj(phase) * wgt (shift_phase with sign -1).
      st.out[lane] = make_float4(r.ph_re * tw, -r.ph_im * tw, (r.meta & 256u) ? -1.0f : 1.0f,
                                 __uint_as_float(r.idx));
      st.key[lane] = r.bin;
    }
    __syncwarp();
    if (kb + H16_BATCH + lane < k1) prefetch(pre, rec, wts, false, with_wgt, nidx, kb + H16_BATCH + lane);
    cp_async_commit();
    if (kb + 2 * H16_BATCH + lane < k1) nidx = sorted[kb + 2 * H16_BATCH + lane];
    int q = 0;
    while (q < nb) {
      const uint32_t gk = st.key[q];
      if (gk != gcur) {  // load the window of bin gk as FP16 fragments
        gcur = gk;
        int su0, sv0, mp;
        window_of(g, gk, nbins, su0, sv0, mp);
        int row = su0 + gq;
        if (row >= g.nu) row -= g.nu;
        int c0 = sv0 + 2 * tq, c1 = c0 + 1;
        if (c0 >= g.nv) c0 -= g.nv;
        if (c1 >= g.nv) c1 -= g.nv;
        cplx<float> v[S][2];  // [plane][column]
        float m = 0.0f;
#pragma unroll
        for (int p = 0; p < S; p++) {
          const int pp = mp + p;
          const bool ok = pp >= pg0 && pp < pg0 + npg && (g.do_wgridding || pp == 0);
          const cplx<float>* src = grids + (size_t)(ok ? pp - pg0 : 0) * plane + (size_t)row * g.nv;
          v[p][0] = ok ? src[c0] : cplx<float>{0.0f, 0.0f};
          v[p][1] = ok ? src[c1] : cplx<float>{0.0f, 0.0f};
          m = fmaxf(m, fmaxf(fmaxf(fabsf(v[p][0].re), fabsf(v[p][0].im)), fmaxf(fabsf(v[p][1].re), fabsf(v[p][1].im))));
        }
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        // Largest window value to about 2^14 (FP16 tops out at 65504).
        const int e = (m > 0.0f && isfinite(m)) ? ilogbf(m) : 0;
        const float sc = ldexpf(1.0f, 14 - e);
        inv = ldexpf(1.0f, e - 14) / H16_BSCALE;
#pragma unroll
        for (int p = 0; p < S; p++) {
          split_h2(v[p][0].re * sc, v[p][1].re * sc, bhi[p][0], blo[p][0]);
          split_h2(v[p][0].im * sc, v[p][1].im * sc, bhi[p][1], blo[p][1]);
        }
      }
      const unsigned mk = __ballot_sync(0xffffffffu, lane >= q && lane < nb && st.key[lane] == gk);
      const int len = __popc(mk);
      // Blocks of sixteen records of the run: rows gq and gq + 8 of the MMA.
      for (int k16 = q; k16 < q + len; k16 += 16) {
        int sr[2];
        uint32_t ahi[2], alo[2];
        float2 kup[2];
        float kwv[2][8];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int k = k16 + gq + 8 * h;
          sr[h] = (k < q + len) ? k : H16_BATCH;
          const float2 kvp = *reinterpret_cast<const float2*>(st.kv + sr[h] * H16_KV + 2 * tq);
          split_h2(kvp.x, kvp.y, ahi[h], alo[h]);
          kup[h] = *reinterpret_cast<const float2*>(st.ku + sr[h] * H16_KU + 2 * tq);
          const float4 w0 = *reinterpret_cast<const float4*>(st.kw + sr[h] * H16_KW);
          const float4 w1 = *reinterpret_cast<const float4*>(st.kw + sr[h] * H16_KW + 4);
          kwv[h][0] = w0.x;
          kwv[h][1] = w0.y;
          kwv[h][2] = w0.z;
          kwv[h][3] = w0.w;
          kwv[h][4] = w1.x;
          kwv[h][5] = w1.y;
          kwv[h][6] = w1.z;
          kwv[h][7] = w1.w;
        }
        // The w contraction first (per window row, over the planes), then the
        // u taps: two FMAs per plane and output instead of three.
        float wr[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}}, wi[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}};
#pragma unroll
        for (int p = 0; p < S; p++) {
          float dre[4], dim[4];
          hmma_zero(dre, ahi[0], ahi[1], bhi[p][0]);
          hmma(dre, ahi[0], ahi[1], blo[p][0]);
          hmma(dre, alo[0], alo[1], bhi[p][0]);
          hmma_zero(dim, ahi[0], ahi[1], bhi[p][1]);
          hmma(dim, ahi[0], ahi[1], blo[p][1]);
          hmma(dim, alo[0], alo[1], bhi[p][1]);
          // d[0], d[1]: record gq, window rows 2tq, 2tq + 1; d[2], d[3]: record gq + 8
#pragma unroll
          for (int h = 0; h < 2; h++)
#pragma unroll
            for (int c = 0; c < 2; c++) {
              wr[h][c] = fmaf(kwv[h][p], dre[2 * h + c], wr[h][c]);
              wi[h][c] = fmaf(kwv[h][p], dim[2 * h + c], wi[h][c]);
            }
        }
        float tr[2], ti[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          tr[h] = fmaf(kup[h].x, wr[h][0], kup[h].y * wr[h][1]);
          ti[h] = fmaf(kup[h].x, wi[h][0], kup[h].y * wi[h][1]);
        }
#pragma unroll
        for (int h = 0; h < 2; h++)
#pragma unroll
          for (int o = 1; o < 4; o <<= 1) {
            tr[h] += __shfl_xor_sync(0xffffffffu, tr[h], o);
            ti[h] += __shfl_xor_sync(0xffffffffu, ti[h], o);
          }
        // Every lane of a quad holds both records' sums: lane tq = h writes record h.
        const int slot = tq ? sr[1] : sr[0];
        if (tq < 2 && slot != H16_BATCH) {
          {
            const float4 fo = st.out[slot];
            const uint32_t idx = __float_as_uint(fo.w);
            const uint64_t k = kb + (uint64_t)slot;
            cplx<float>* dst = out.mode == DEGRID_TO_VIS ? out.vis + idx : out.stored + k;
            cplx<float> accv{(tq ? tr[1] : tr[0]) * inv, (tq ? ti[1] : ti[0]) * inv * fo.z};
            if (!first) {
              const cplx<float> prev = *dst;
              accv = {accv.re + prev.re, accv.im + prev.im};
            }
            if (last) {
              accv = {accv.re * fo.x - accv.im * fo.y, accv.re * fo.y + accv.im * fo.x};
              if (out.mode != DEGRID_TO_VIS) {
                const uint64_t di = out.sorted_data ? k : (uint64_t)idx;
                const float w = wgt_get<float>(out.data, di);
                if (out.mode == DEGRID_RESIDUAL) {
                  const cplx<float> d = vis_get<float>(out.data, di);
                  accv = {d.re - accv.re, d.im - accv.im};
                }
                part += (double)w * ((double)accv.re * (double)accv.re + (double)accv.im * (double)accv.im);
                accv = {accv.re * w, accv.im * w};
                vmax = fmax(vmax, sqrt((double)accv.re * (double)accv.re + (double)accv.im * (double)accv.im));
              }
            }
            *dst = accv;
          }
        }
      }
      q += len;
    }
  }
  if (out.mode != DEGRID_TO_VIS && last) {
    for (int o = 16; o > 0; o >>= 1) {
      part += __shfl_down_sync(0xffffffffu, part, o);
      vmax = fmax(vmax, __shfl_down_sync(0xffffffffu, vmax, o));
    }
    if (lane == 0) {
      out.partials[out.block0 + blockIdx.x] = part;
      atomic_max_double(&out.bound->vmax_bits, vmax);
    }
  }
}

// ------------------------------------------------------------------ residual without a model, and sums

constexpr uint32_t STORE_CHUNK = 8192;  // sorted positions per block of k_store_values
constexpr int STORE_THREADS = 256;

// Fixed-order sum of one value per thread of a block into thread 0.
__device__ __forceinline__ double block_sum(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  return sh[0];
}

// The residual of the data alone (no model): stored[k] = w d for the
// visibility at sorted position k, w |d|^2 summed into partials[block]
// (each block takes STORE_CHUNK positions, each thread a fixed stride of
// them, then a fixed tree), and the largest |stored| into `bound`.
__global__ void __launch_bounds__(STORE_THREADS)
    k_store_values(uint64_t n, const uint32_t* __restrict__ sorted, Inputs data, int sorted_data,
                   cplx<float>* __restrict__ stored, double* __restrict__ partials, ValueBound* bound) {
  __shared__ double sh[STORE_THREADS];
  const uint64_t k0 = (uint64_t)blockIdx.x * STORE_CHUNK, k1 = min(n, k0 + STORE_CHUNK);
  double part = 0.0, vmax = 0.0;
  for (uint64_t k = k0 + threadIdx.x; k < k1; k += STORE_THREADS) {
    const uint64_t di = sorted_data ? k : (uint64_t)sorted[k];
    const float w = wgt_get<float>(data, di);
    const cplx<float> d = vis_get<float>(data, di);
    part += (double)w * ((double)d.re * (double)d.re + (double)d.im * (double)d.im);
    const cplx<float> v{d.re * w, d.im * w};
    vmax = fmax(vmax, sqrt((double)v.re * (double)v.re + (double)v.im * (double)v.im));
    stored[k] = v;
  }
  const double sum = block_sum(part, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = sum;
  for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_down_sync(0xffffffffu, vmax, o));
  if ((threadIdx.x & 31) == 0) atomic_max_double(&bound->vmax_bits, vmax);
}

// out = sum of partials[0, n) in a fixed order (one block).
__global__ void __launch_bounds__(STORE_THREADS) k_sum_partials(const double* __restrict__ partials, uint32_t n,
                                                                 double* out) {
  __shared__ double sh[STORE_THREADS];
  double v = 0.0;
  for (uint32_t i = threadIdx.x; i < n; i += STORE_THREADS) v += partials[i];
  const double s = block_sum(v, sh);
  if (threadIdx.x == 0) *out = s;
}

}  // namespace fast
