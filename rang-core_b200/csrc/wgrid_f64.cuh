// The double-precision gridder on the FP64 tensor cores.
//
// Included by wgrid_plan.cu inside its anonymous namespace, after
// wgrid_fast.cuh (it uses the fixed-point grid, the windows and the device
// helpers defined there).
//
// A double-precision plan's sorted order is stable (a radix sort by bin key,
// so the visibilities of a bin keep their index order) and every warp takes
// a fixed range of it, so each warp meets the same records in the same
// order on every call. Per run of one bin the warp accumulates the bin's
// 8 x 8 window of each of its S planes on the FP64 tensor cores
// (mma.sync m8n8k4: rows the window's u cells, columns its v cells, k four
// records: A = w tap x placed u taps, B = value x placed v taps), so the run's
// sums are formed in one fixed order, in FP64 as the reference forms them.
// At the end of a run the window is added to the 128-bit fixed-point grid
// (each sum rounded once into the grid's unit; integer adds, exact in any
// order), so the result does not depend on how the runs' atomic adds
// interleave: a call is reproducible bit for bit.

namespace fast {

constexpr int F64_BATCH = 32;        // records staged per round, one per lane
constexpr uint32_t F64_CHUNK = 2048;  // sorted records per warp
constexpr int F64_ROW = 8;           // doubles per staged row (8 window cells)

// Per slot (record): the u taps placed on the window's 8 rows, Re and Im of
// value x v taps placed on its 8 columns, the w taps of the S planes (zero
// outside the pass's planes) and the bin key. Slot F64_BATCH stays zero.
struct F64Slots {
  double* ku;
  double* bre;
  double* bim;
  double* kw;
  uint32_t* key;
  __host__ __device__ static constexpr size_t bytes() {
    return ((size_t)(F64_BATCH + 1) * (4 * F64_ROW * 8 + 4) + 15) / 16 * 16;
  }
  __device__ void carve(unsigned char* base) {
    ku = reinterpret_cast<double*>(base);
    bre = ku + (F64_BATCH + 1) * F64_ROW;
    bim = bre + (F64_BATCH + 1) * F64_ROW;
    kw = bim + (F64_BATCH + 1) * F64_ROW;
    key = reinterpret_cast<uint32_t*>(kw + (F64_BATCH + 1) * F64_ROW);
  }
};

// The inputs of one staged visibility, copied asynchronously (cp.async) a
// round ahead of their use: its row's uvw, its channel's f / c, its value,
// its weight and its bin key.
struct Prefetched64 {
  double uvw[3];
  double foc;
  uint4 vis;  // complex128, or complex64 in .x, .y
  uint2 wgt;  // float64, float32 in .x, or the two float32 factors
  uint32_t key;
  uint32_t idx;
};
static_assert(sizeof(Prefetched64) == 64, "one 64-byte slot per lane");

__device__ __forceinline__ void prefetch64(Prefetched64* dst, const double* __restrict__ uvw,
                                           const double* __restrict__ foc, const Inputs& in, bool with_vis,
                                           bool with_wgt, const uint32_t* __restrict__ key, uint32_t idx,
                                           uint32_t nchan) {
  const uint32_t row = idx / nchan, ch = idx - row * nchan;
  const double* u = uvw + 3 * (size_t)row;
  cp_async(&dst->uvw[0], u, 8);
  cp_async(&dst->uvw[1], u + 1, 8);
  cp_async(&dst->uvw[2], u + 2, 8);
  cp_async(&dst->foc, foc + ch, 8);
  if (with_vis) {
    if (in.vis_kind == VIS_C128)
      cp_async(&dst->vis, reinterpret_cast<const double2*>(in.vis) + idx, 16);
    else if (in.vis_kind == VIS_C64)
      cp_async(&dst->vis, reinterpret_cast<const float2*>(in.vis) + idx, 8);
  }
  if (with_wgt) {
    if (in.wgt_kind == WGT_F64) {
      cp_async(&dst->wgt, reinterpret_cast<const double*>(in.wgt) + idx, 8);
    } else {
      cp_async(&dst->wgt.x, reinterpret_cast<const float*>(in.wgt) + idx, 4);
      if (in.wgt_kind == WGT_F32_PRODUCT) cp_async(&dst->wgt.y, reinterpret_cast<const float*>(in.wgt2) + idx, 4);
    }
  }
  cp_async(&dst->key, key + idx, 4);
  dst->idx = idx;
}

// Weights::get and VisData::get (wgridder.rs:950-1005) in double precision.
__device__ __forceinline__ double prefetched_wgt64(const Prefetched64& p, const Inputs& in) {
  switch (in.wgt_kind) {
    case WGT_F64:
      return __longlong_as_double((long long)(((unsigned long long)p.wgt.y << 32) | p.wgt.x));
    case WGT_F32:
      return (double)__uint_as_float(p.wgt.x);
    case WGT_F32_PRODUCT:
      return (double)(__uint_as_float(p.wgt.x) * __uint_as_float(p.wgt.y));
    default:
      return 1.0;
  }
}
__device__ __forceinline__ cplx<double> prefetched_vis64(const Prefetched64& p, const Inputs& in) {
  if (in.vis_kind == VIS_C128)
    return {__longlong_as_double((long long)(((unsigned long long)p.vis.y << 32) | p.vis.x)),
            __longlong_as_double((long long)(((unsigned long long)p.vis.w << 32) | p.vis.z))};
  if (in.vis_kind == VIS_C64) return {(double)__uint_as_float(p.vis.x), (double)__uint_as_float(p.vis.y)};
  return {1.0, 0.0};
}

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// Adds a run's window sums to the 128-bit grid: acc[p][c][i] is plane
// mp + p, component c, window row gq and column 2 tq + i.
template <int S>
__device__ __forceinline__ void f64_flush(const Geom<double>& g, FixCell2* __restrict__ grids, int pg0, int npg,
                                          int su0, int sv0, int mp, double sc, const double (&acc)[S][2][2]) {
  const int lane = threadIdx.x & 31, gq = lane >> 2, tq = lane & 3;
  const size_t plane = (size_t)g.nu * g.nv;
  int row = su0 + gq;
  if (row >= g.nu) row -= g.nu;
#pragma unroll
  for (int p = 0; p < S; p++) {
    const int pp = mp + p;
    if (pp < pg0 || pp >= pg0 + npg) continue;
#pragma unroll
    for (int i = 0; i < 2; i++) {
      const double re = acc[p][0][i], im = acc[p][1][i];
      if (re == 0.0 && im == 0.0) continue;
      int col = sv0 + 2 * tq + i;
      if (col >= g.nv) col -= g.nv;
      FixTraits<double>::flush(grids + (size_t)(pp - pg0) * plane + (size_t)row * g.nv + col,
                               FixTraits<double>::term(re, sc), FixTraits<double>::term(im, sc));
    }
  }
}

// Gridding of sorted records [kbase, kend) in double precision (the
// reference's grid_task_body, wgridder.rs:2102-2156, on windows): each warp
// takes F64_CHUNK consecutive sorted visibilities, stages F64_BATCH at a time
// (coordinates, taps and value from uvw and the data, as k_grid does) and
// contracts each run of one bin four records at a time.
template <int S>
__global__ void __launch_bounds__(F64_BATCH, 12)
    k_grid_f64(const __grid_constant__ Geom<double> g, Inputs in, int mode, const double* __restrict__ uvw,
               const double* __restrict__ foc, const uint32_t* __restrict__ key, const uint32_t* __restrict__ sorted,
               uint64_t kbase, uint64_t kend, uint32_t nbins, FixCell2* __restrict__ grids, int pg0, int npg,
               FixScale* __restrict__ fs) {
  static_assert(S >= 1 && S <= 8, "8 x 8 windows");
  extern __shared__ __align__(16) unsigned char smem[];
  F64Slots st;
  st.carve(smem);
  const int lane = threadIdx.x, gq = lane >> 2, tq = lane & 3;
  if (lane < F64_ROW) {
    st.ku[F64_BATCH * F64_ROW + lane] = 0.0;
    st.bre[F64_BATCH * F64_ROW + lane] = 0.0;
    st.bim[F64_BATCH * F64_ROW + lane] = 0.0;
    st.kw[F64_BATCH * F64_ROW + lane] = 0.0;
  }
  if (lane == 0) st.key[F64_BATCH] = INACTIVE;
  const uint64_t k0 = kbase + (uint64_t)blockIdx.x * F64_CHUNK;
  const uint64_t k1 = min(kend, k0 + F64_CHUNK);
  const double sc = FixTraits<double>::scale(fs->q);
  const uint32_t nchan = (uint32_t)g.nchan;
  const uint32_t tmask = (1u << g.log2tile) - 1u;
  const bool with_wgt = in.wgt_kind != WGT_NONE;
  bool bad = false;

  double acc[S][2][2];
#pragma unroll
  for (int p = 0; p < S; p++)
#pragma unroll
    for (int c = 0; c < 2; c++) acc[p][c][0] = acc[p][c][1] = 0.0;
  uint32_t gcur = INACTIVE;
  int su0 = 0, sv0 = 0, mpc = 0;

  // This round's inputs are in pre (copied asynchronously); nidx is the next
  // round's index.
  Prefetched64* pre = reinterpret_cast<Prefetched64*>(smem + F64Slots::bytes()) + lane;
  const bool with_vis = mode == VALUE_DATA && in.vis_kind != VIS_UNIT;
  if (k0 + lane < k1) prefetch64(pre, uvw, foc, in, with_vis, with_wgt, key, sorted[k0 + lane], nchan);
  cp_async_commit();
  uint32_t nidx = (k0 + F64_BATCH + lane < k1) ? sorted[k0 + F64_BATCH + lane] : 0u;

  for (uint64_t kb = k0; kb < k1; kb += F64_BATCH) {
    const int nb = (int)min((uint64_t)F64_BATCH, k1 - kb);
    cp_async_wait_all();
    __syncwarp();
    if (lane < nb) {  // staging, one record per lane
      const Prefetched64& pr = *pre;
      double b[3];
      const double imflip = row_coord_of(pr.uvw[0], pr.uvw[1], pr.uvw[2], g.fu, g.fv, g.fw, g.r_l, g.r_m, b);
      const double f = pr.foc;
      const double u = b[0] * f, v = b[1] * f, w = b[2] * f;
      double uf, vf;
      int iu0, iv0;
      getpix(g, u, v, uf, vf, iu0, iv0);
      const int mp = minplane(g, w);
      const uint32_t su = (uint32_t)shifted(iu0, g.nu) & tmask, sv = (uint32_t)shifted(iv0, g.nv) & tmask;
      const int du = (int)(su % (uint32_t)g.sube), dv = (int)(sv % (uint32_t)g.sube);
      double ku[S], kv[S];
      eval_taps2<double, S>(g.coeff, g.ne, -uf * 2.0 + ((double)S - 1.0), -vf * 2.0 + ((double)S - 1.0), ku, kv);
      cplx<double> val = unit_value<double>(g, b, imflip, f, with_wgt, prefetched_wgt64(pr, in));
      if (mode == VALUE_DATA) val = data_value<double>(prefetched_vis64(pr, in), val, imflip);
      bad |= !isfinite(val.re) || !isfinite(val.im) || !isfinite(uf) || !isfinite(vf) || !isfinite(w);
      double* cu = st.ku + lane * F64_ROW;
      double* cr = st.bre + lane * F64_ROW;
      double* ci = st.bim + lane * F64_ROW;
      double* cw = st.kw + lane * F64_ROW;
#pragma unroll
      for (int j = 0; j < F64_ROW; j++) {
        double a = 0.0, br = 0.0, bi = 0.0;
#pragma unroll
        for (int d = 0; d < 9 - S; d++) {
          if (j - d >= 0 && j - d < S) {
            const int t = (j - d >= 0 && j - d < S) ? j - d : 0;
            if (du == d) a = ku[t];
            if (dv == d) {
              br = val.re * kv[t];
              bi = val.im * kv[t];
            }
          }
        }
        cu[j] = a;
        cr[j] = br;
        ci[j] = bi;
        double kwj = 0.0;
        if (j < S) {
          if (g.do_wgridding) {
            const int p = mp + j;
            if (p >= pg0 && p < pg0 + npg) kwj = w_factor<double, S>(g, j, p, w);
          } else if (j == 0 && pg0 == 0) {
            kwj = 1.0;
          }
        }
        cw[j] = kwj;
      }
      st.key[lane] = pr.key;
    }
    // The next round's inputs, in flight while this one is contracted.
    __syncwarp();
    if (kb + F64_BATCH + lane < k1) prefetch64(pre, uvw, foc, in, with_vis, with_wgt, key, nidx, nchan);
    cp_async_commit();
    if (kb + 2 * F64_BATCH + lane < k1) nidx = sorted[kb + 2 * F64_BATCH + lane];
    int q = 0;
    while (q < nb) {
      const uint32_t gk = st.key[q];
      if (gk != gcur) {
        if (gcur != INACTIVE) f64_flush<S>(g, grids, pg0, npg, su0, sv0, mpc, sc, acc);
#pragma unroll
        for (int p = 0; p < S; p++)
#pragma unroll
          for (int c = 0; c < 2; c++) acc[p][c][0] = acc[p][c][1] = 0.0;
        gcur = gk;
        window_of(g, gk, nbins, su0, sv0, mpc);
      }
      const unsigned m = __ballot_sync(0xffffffffu, lane >= q && lane < nb && st.key[lane] == gk);
      const int len = __popc(m);
      for (int k4 = q; k4 < q + len; k4 += 4) {
        const int kk = k4 + tq;
        const int slot = kk < q + len ? kk : F64_BATCH;
        const double kur = st.ku[slot * F64_ROW + gq];   // A: row gq, k tq
        const double bre = st.bre[slot * F64_ROW + gq];  // B: k tq, column gq
        const double bim = st.bim[slot * F64_ROW + gq];
#pragma unroll
        for (int p = 0; p < S; p++) {
          const double a = kur * st.kw[slot * F64_ROW + p];
          dmma(acc[p][0], a, bre);
          dmma(acc[p][1], a, bim);
        }
      }
      q += len;
    }
  }
  if (gcur != INACTIVE) f64_flush<S>(g, grids, pg0, npg, su0, sv0, mpc, sc, acc);
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&fs->nonfinite, 1);
}

}  // namespace fast
