// The B200 w-gridder pipeline.
//
//   scan        active count and |w| range (one pass over the visibilities)
//   plan        kernel, grid and w-planes on the host (wgrid_setup.cpp)
//   binning     counting sort of the active visibilities by (uv tile, first
//               w-plane): per-visibility key, bin counts, exclusive scan,
//               scatter; then a task list of <= TASK_CHUNK visibilities of
//               one tile each
//   gridding    one CTA per task: the visibilities' ES-kernel footprints on
//               all their w-planes accumulate in a shared-memory window of
//               the tile (tile + support - 1 cells square per plane), which
//               is then added to the HBM-resident w-planes
//   FFT         cuFFT: inverse along v on every grid row, along u on the
//               image columns only
//   project     per pixel, the planes' w-screens applied and summed in
//               plane order, then the global correction
// and the adjoint for degridding (corrected image times w-screen placed on
// the grid, forward FFTs, then one CTA per task gathering each visibility's
// footprint from a shared-memory copy of the tile's planes).
//
// All w-planes of a call stay resident in HBM when they fit (a 9450^2
// complex64 plane is 714 MB), so every visibility is read once per
// direction and the footprint on all of its planes is formed in one pass.
#include <cuda_fp16.h>
#include <cufft.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cstdlib>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <type_traits>

#include "wgrid_plan.h"

namespace wg {

namespace {

constexpr uint32_t INACTIVE = 0xffffffffu;
constexpr uint32_t TASK_CHUNK = 16384;
constexpr int GRID_THREADS = 256;
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr size_t SMEM_WINDOW_BYTES = 80 * 1024;

unsigned blocks_for(uint64_t n, int threads, unsigned cap = 148u * 32u) {
  uint64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  return (unsigned)std::min<uint64_t>(b, cap);
}

// ------------------------------------------------------------------ scan

struct ScanOut {
  unsigned long long count;    // active visibilities
  unsigned long long finite;   // of which with a non-NaN |w|
  unsigned long long lo_bits;  // min |w| as the bits of a non-negative double
  unsigned long long hi_bits;  // max |w|
  unsigned long long u_bits;   // max |u| in metres over all rows (k_umax); +inf if any is not finite
  unsigned long long vmax_bits;  // max |vis| |wgt| over the active set (a scan with the visibilities)
  unsigned long long wmax_bits;  // max |wgt| over the active set
};

// The largest |u| (metres) over all rows, +inf when one is not finite: times
// the largest f / c it bounds every visibility's |u| in wavelengths, which
// is what the touched-row pruning needs (rows, not visibilities: cheaper
// than the scan, and flagged rows only widen the bound).
__global__ void k_umax(uint32_t nrow, const double* __restrict__ uvw, ScanOut* out) {
  double m = 0.0;
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < nrow; r += (uint64_t)gridDim.x * blockDim.x) {
    const double a = fabs(uvw[3 * r]);
    m = isfinite(a) ? fmax(m, a) : __longlong_as_double(0x7ff0000000000000ll);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&out->u_bits, (unsigned long long)__double_as_longlong(m));
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Row and channel of a grid-stride loop's linear index, advanced by the
// constant stride without a division per element.
struct RowCh {
  uint32_t row, ch, srow, sch;
  __device__ RowCh(uint64_t i, uint32_t nchan, uint64_t stride) {
    row = (uint32_t)(i / nchan);
    ch = (uint32_t)(i - (uint64_t)row * nchan);
    srow = (uint32_t)(stride / nchan);
    sch = (uint32_t)(stride - (uint64_t)srow * nchan);
  }
  __device__ __forceinline__ void next(uint32_t nchan) {
    row += srow;
    ch += sch;
    if (ch >= nchan) {
      ch -= nchan;
      row++;
    }
  }
};

// The scan's reduction target before the scan: no visibilities, min |w| =
// 1e300, max |w| = 0 (a kernel, so that no host buffer is copied).
__global__ void k_scan_init(ScanOut* so) {
  so->count = 0;
  so->finite = 0;
  so->lo_bits = (unsigned long long)__double_as_longlong(1e300);
  so->hi_bits = 0;
  so->u_bits = 0;
  so->vmax_bits = 0;
  so->wmax_bits = 0;
}

// The activity inputs of four consecutive visibilities e .. e + 3 (e a
// multiple of 4): by 16-byte loads when `vec` (every input 16-byte aligned)
// and all four exist, else one by one; those at or past n get mask 0.
template <class T>
struct Quad {
  cplx<T> v[4];
  T w[4];
  uint32_t m;  // the four mask bytes, visibility e in the low byte
};

// VIS: the values read (0 none, 1 complex64, 2 complex128); WGT: weights read.
template <class T, int VIS, bool WGT>
__device__ __forceinline__ void load_quad(const Inputs& in, bool vec, uint64_t e, uint64_t n, Quad<T>& q) {
#pragma unroll
  for (int k = 0; k < 4; k++) {
    q.v[k] = {(T)1, (T)0};
    q.w[k] = (T)1;
  }
  if (vec && e + 4 <= n) {
    if (VIS == 1) {
      const float4 a = reinterpret_cast<const float4*>(in.vis)[e / 2];
      const float4 b = reinterpret_cast<const float4*>(in.vis)[e / 2 + 1];
      q.v[0] = {(T)a.x, (T)a.y};
      q.v[1] = {(T)a.z, (T)a.w};
      q.v[2] = {(T)b.x, (T)b.y};
      q.v[3] = {(T)b.z, (T)b.w};
    } else if (VIS == 2) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const double2 d = reinterpret_cast<const double2*>(in.vis)[e + k];
        q.v[k] = {(T)d.x, (T)d.y};
      }
    }
    if (!WGT) {
    } else if (in.wgt_kind == WGT_F32 || in.wgt_kind == WGT_F32_PRODUCT) {
      float4 a = reinterpret_cast<const float4*>(in.wgt)[e / 4];
      if (in.wgt_kind == WGT_F32_PRODUCT) {
        const float4 b = reinterpret_cast<const float4*>(in.wgt2)[e / 4];
        a = make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w);
      }
      q.w[0] = (T)a.x;
      q.w[1] = (T)a.y;
      q.w[2] = (T)a.z;
      q.w[3] = (T)a.w;
    } else if (in.wgt_kind == WGT_F64) {
      const double2 a = reinterpret_cast<const double2*>(in.wgt)[e / 2];
      const double2 b = reinterpret_cast<const double2*>(in.wgt)[e / 2 + 1];
      q.w[0] = (T)a.x;
      q.w[1] = (T)a.y;
      q.w[2] = (T)b.x;
      q.w[3] = (T)b.y;
    }
    q.m = in.mask ? reinterpret_cast<const uint32_t*>(in.mask)[e / 4] : 0x01010101u;
    return;
  }
  q.m = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    if (e + k < n) {
      if (VIS) q.v[k] = vis_get<T>(in, e + k);
      if (WGT) q.w[k] = wgt_get<T>(in, e + k);
      q.m |= (in.mask ? (uint32_t)in.mask[e + k] : 1u) << (8 * k);
    }
  }
}

// is_active's test, (double) |vis|^2 * (double) wgt * (double) mask != 0,
// for single-precision factors: a double product of floats neither
// overflows nor underflows, so it is zero exactly when a factor is zero and
// none is infinite or NaN. Double-precision factors take the product.
__device__ __forceinline__ bool active_of(float vn, float w, uint32_t m) {
  return !isfinite(vn) || !isfinite(w) || (vn != 0.0f && w != 0.0f && m != 0u);
}
__device__ __forceinline__ bool active_of(double vn, double w, uint32_t m) { return vn * w * (double)m != 0.0; }

// Whether every channel factor f / c is finite (they are positive): the
// scan's |w| range then takes two products per group of four.
bool all_finite(const std::vector<double>& foc) {
  for (double f : foc)
    if (!std::isfinite(f)) return false;
  return true;
}

// Whether the scan's 16-byte loads may be used: every input present is
// 16-byte aligned (the mask 4-byte).
bool scan_vectors(const Inputs& in, bool with_vis) {
  auto al = [](const void* p, uintptr_t a) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) % a) == 0; };
  return (!with_vis || in.vis_kind == VIS_UNIT || al(in.vis, 16)) &&
         (in.wgt_kind == WGT_NONE || (al(in.wgt, 16) && al(in.wgt2, 16))) && al(in.mask, 4);
}

// Groups of four visibilities each lane has in flight (half as many in
// double precision, whose values take twice the registers): at four blocks
// per SM that is 72 bytes per lane, 73 KB per SM, of complex64 values and
// mask in flight; more groups spill.
constexpr int SCAN_GROUPS = 2;

// scan (wgridder.rs:1051-1077): the count is exact and min/max are order
// independent, so the result is the reference's bit for bit. A warp takes
// blocks of 128 G consecutive visibilities, a grid stride apart; in group q
// of a block lane l takes the four visibilities from 128 q + 4 l, its inputs
// in 16-byte loads (one byte per lane per load left the pass waiting on
// memory at a third of the HBM rate). With `bits`, bit i of the u32 array is
// set when visibility i is active (is_active): the count pass then reads one
// word per 32 visibilities instead of their inputs.
//
// The |w| range of a group inside one row needs two products, not four:
// |w| = |(fw w_row) f_c| with the channels' f_c ascending and, when `clean`
// (every f_c finite; they are positive), rounding is monotone, so the
// smallest and largest |w| of the group's active visibilities are those of
// its first and last active channel, and each is NaN exactly when
// fw w_row is. Four blocks per SM (at most 64 registers) measured 1.81 ms
// per scan at 1.06 G visibilities, three (up to 80 registers) 2.05.
template <class T, int VIS, bool WGT>
__global__ void __launch_bounds__(256, 4) k_scan(uint32_t nrow, uint32_t nchan, const double* __restrict__ uvw,
                       const double* __restrict__ foc, double fw, Inputs in, int vec, int clean,
                       ScanOut* out, uint32_t* __restrict__ bits) {
  const uint64_t n = (uint64_t)nrow * nchan;
  constexpr int G = sizeof(T) == 4 ? SCAN_GROUPS : SCAN_GROUPS / 2;
  constexpr uint64_t BLOCK = 128ull * G;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t wid = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t wstride = (((uint64_t)gridDim.x * blockDim.x) >> 5) * BLOCK;
  uint32_t cnt32 = 0, fin32 = 0;  // per thread: far below 2^32
  double lo = 1e300, hi = 0.0, vm = 0.0;
  T wm = (T)0;  // max |wgt|: the conversion to double is exact and monotone
  uint64_t b0 = wid * BLOCK;
  RowCh rc(b0 + 4 * lane, nchan, wstride);
  const uint32_t srow = 128u / nchan, sch = 128u % nchan;  // one group: 128 visibilities
  for (; b0 < n; b0 += wstride, rc.next(nchan)) {
    Quad<T> q[G];
#pragma unroll
    for (int g = 0; g < G; g++) load_quad<T, VIS, WGT>(in, vec != 0, b0 + 128 * g + 4 * lane, n, q[g]);
    uint32_t row = rc.row, ch = rc.ch;
#pragma unroll
    for (int g = 0; g < G; g++) {
      uint32_t nib = 0;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        // is_active, keeping the magnitudes for the value bound
        const T vn = VIS ? q[g].v[k].re * q[g].v[k].re + q[g].v[k].im * q[g].v[k].im : (T)1;
        if (active_of(vn, q[g].w[k], (q[g].m >> (8 * k)) & 0xffu)) {
          nib |= 1u << k;
          const T awt = fabs(q[g].w[k]);
          wm = awt > wm ? awt : wm;
          // |vis|^2 |wgt|^2, the value bound's square (value_bound_sq)
          const double aw = (double)awt;
          const double av = VIS ? value_bound_sq(q[g].v[k], aw) : aw * aw;
          vm = av > vm ? av : vm;
        }
      }
      if (nib) {
        cnt32 += __popc(nib);
        if (clean && ch + 3 < nchan) {  // one row
          const double a = fw * uvw[3 * (uint64_t)row + 2];
          if (!isnan(a)) {
            fin32 += __popc(nib);
            lo = fmin(lo, fabs(a * foc[ch + __ffs(nib) - 1]));
            hi = fmax(hi, fabs(a * foc[ch + 31 - __clz(nib)]));
          }
        } else {
          uint32_t r = row, c = ch;
#pragma unroll
          for (int k = 0; k < 4; k++) {
            if (nib & (1u << k)) {
              const double w = fabs(fw * uvw[3 * (uint64_t)r + 2] * foc[c]);
              if (!isnan(w)) {
                fin32++;
                lo = fmin(lo, w);
                hi = fmax(hi, w);
              }
            }
            if (++c == nchan) {
              c = 0;
              r++;
            }
          }
        }
      }
      if (bits) {  // eight lanes' nibbles make the word of 32 visibilities
        uint32_t x = nib << (4 * (lane & 7));
        x |= __shfl_xor_sync(0xffffffffu, x, 1);
        x |= __shfl_xor_sync(0xffffffffu, x, 2);
        x |= __shfl_xor_sync(0xffffffffu, x, 4);
        const uint64_t e = b0 + 128 * g + 4 * lane;
        if ((lane & 7) == 0 && e < n) bits[e >> 5] = x;
      }
      row += srow;
      ch += sch;
      if (ch >= nchan) {
        ch -= nchan;
        row++;
      }
    }
  }
  unsigned long long cnt = cnt32, fin = fin32;
  cnt = warp_sum(cnt);
  fin = warp_sum(fin);
  lo = warp_min(lo);
  hi = warp_max(hi);
  vm = warp_max(vm);
  double wmd = warp_max((double)wm);
  if ((threadIdx.x & 31) == 0 && cnt) {
    vm = sqrt(vm);  // one square root per warp: the largest |vis| |wgt|
    if (vm > 0.0) atomicMax(&out->vmax_bits, (unsigned long long)__double_as_longlong(vm));
    if (wmd > 0.0) atomicMax(&out->wmax_bits, (unsigned long long)__double_as_longlong(wmd));
    atomicAdd(&out->count, cnt);
    if (fin) {
      atomicAdd(&out->finite, fin);
      atomicMin(&out->lo_bits, (unsigned long long)__double_as_longlong(lo));
      atomicMax(&out->hi_bits, (unsigned long long)__double_as_longlong(hi));
    }
  }
}

// k_scan for the activity inputs present: the values (with_vis, of kind
// complex64 or complex128) and the weights, each a template argument so that
// a scan of the mask alone tests a byte per visibility and no more.
template <class T>
void launch_scan(uint32_t nrow, uint32_t nchan, const double* uvw, const double* foc, double fw, const Inputs& in,
                 bool with_vis, bool clean, ScanOut* out, uint32_t* bits, cudaStream_t s) {
  const uint64_t n = (uint64_t)nrow * nchan;
  const int vec = scan_vectors(in, with_vis) ? 1 : 0;
  const int vis = !with_vis ? 0 : in.vis_kind == VIS_C64 ? 1 : in.vis_kind == VIS_C128 ? 2 : 0;
  const bool wgt = in.wgt_kind != WGT_NONE;
  auto go = [&](auto kv, auto kw) {
    k_scan<T, decltype(kv)::value, decltype(kw)::value><<<blocks_for(n, 256), 256, 0, s>>>(
        nrow, nchan, uvw, foc, fw, in, vec, clean ? 1 : 0, out, bits);
  };
  using W1 = std::true_type;
  using W0 = std::false_type;
  if (vis == 1) {
    if (wgt) go(std::integral_constant<int, 1>{}, W1{}); else go(std::integral_constant<int, 1>{}, W0{});
  } else if (vis == 2) {
    if (wgt) go(std::integral_constant<int, 2>{}, W1{}); else go(std::integral_constant<int, 2>{}, W0{});
  } else {
    if (wgt) go(std::integral_constant<int, 0>{}, W1{}); else go(std::integral_constant<int, 0>{}, W0{});
  }
}

// ------------------------------------------------------------------ binning

// Setup::locate (wgridder.rs:1244-1255) as one key: the tile and first plane
// of the reference's layout, refined by the sub-tile of the first tap:
// ((tile * nbuckets + plane) * nsub + sub-tile). Sorting by it keeps the
// reference's (tile, plane) order and groups each plane's visibilities by
// sub-tile, whose footprints the tensor-core kernels take as one window.
template <class T>
__device__ __forceinline__ uint32_t bin_of_rc(const Geom<T>& g, const double* __restrict__ uvw,
                                              const double* __restrict__ foc, uint32_t row, uint32_t ch,
                                              int64_t* piu0 = nullptr, int64_t* piv0 = nullptr) {
  double b[3];
  row_coord(uvw, row, g.fu, g.fv, g.fw, g.r_l, g.r_m, b);
  double f = foc[ch];
  double u = b[0] * f, v = b[1] * f, w = b[2] * f;
  double uf, vf;
  int iu0, iv0;
  getpix(g, u, v, uf, vf, iu0, iv0);
  const uint32_t su = (uint32_t)shifted(iu0, g.nu), sv = (uint32_t)shifted(iv0, g.nv);
  const uint32_t tu = su >> g.log2tile, tv = sv >> g.log2tile;
  const uint32_t mask = (1u << g.log2tile) - 1u;
  const uint32_t sub = ((su & mask) / (uint32_t)g.sube) * (uint32_t)g.nsub_side + (sv & mask) / (uint32_t)g.sube;
  if (piu0) *piu0 = iu0;
  if (piv0) *piv0 = iv0;
  return ((tu * (uint32_t)g.ntv + tv) * (uint32_t)g.nbuckets + (uint32_t)minplane(g, w)) * (uint32_t)g.nsub + sub;
}
template <class T>
__device__ __forceinline__ uint32_t bin_of(const Geom<T>& g, const double* __restrict__ uvw,
                                           const double* __restrict__ foc, uint32_t idx, int64_t* piu0 = nullptr,
                                           int64_t* piv0 = nullptr) {
  const uint32_t nchan = (uint32_t)g.nchan;
  const uint32_t row = idx / nchan, ch = idx - row * nchan;
  return bin_of_rc(g, uvw, foc, row, ch, piu0, piv0);
}

// One counting atomic per distinct counter in the warp, without waiting for
// its result (the count pass needs no positions).
__device__ __forceinline__ void warp_aggregated_count(uint32_t* counters, uint32_t key, bool active) {
  const unsigned mask = __ballot_sync(0xffffffffu, active);
  if (active) {
    const unsigned peers = __match_any_sync(mask, key);
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&counters[key], (uint32_t)__popc(peers));
  }
}

// One atomic per distinct counter in the warp; each active lane gets the
// counter's old value plus its rank among the lanes with the same counter.
__device__ __forceinline__ uint32_t warp_aggregated_add(uint32_t* counters, uint32_t key, bool active) {
  unsigned mask = __ballot_sync(0xffffffffu, active);
  uint32_t res = 0;
  if (active) {
    unsigned peers = __match_any_sync(mask, key);
    int lane = threadIdx.x & 31;
    int leader = __ffs(peers) - 1;
    unsigned rank = __popc(peers & ((1u << lane) - 1));
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&counters[key], (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    res = base + rank;
  }
  return res;
}

// With rows_per_chunk > 0 the key is chunk * nbins + bin, chunk = row / rows_per_chunk.
// With `bits` the active set is the scan's (bit i: visibility i), else each
// visibility's inputs are read. Capped at 32 registers (eight 256-thread blocks, every warp slot of an SM):
// the kernel is bound by instruction issue, and the extra warps measured 11 %
// faster than 36 registers (6 blocks) despite a 4-byte spill.
template <class T>
__global__ void __launch_bounds__(256, 8) k_bin_count(const __grid_constant__ Geom<T> g, const double* __restrict__ uvw,
                            const double* __restrict__ foc, Inputs in, int with_vis, uint32_t* __restrict__ key,
                            uint32_t* __restrict__ counts, uint32_t rows_per_chunk = 0, uint32_t nbins = 0,
                            const uint32_t* __restrict__ bits = nullptr) {
  uint64_t n = g.nrow * g.nchan;
  uint64_t nround = (n + 31) & ~31ull;
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  RowCh rc(i, (uint32_t)g.nchan, (uint64_t)gridDim.x * blockDim.x);
  for (; i < nround; i += (uint64_t)gridDim.x * blockDim.x, rc.next((uint32_t)g.nchan)) {
    bool act = false;
    uint32_t k = INACTIVE;
    if (i < n) {
      act = bits ? ((bits[i >> 5] >> (i & 31)) & 1u) != 0 : is_active<T>(in, with_vis != 0, i);
      if (act) {
        k = bin_of_rc(g, uvw, foc, rc.row, rc.ch);
        if (rows_per_chunk) k += (rc.row / rows_per_chunk) * nbins;
      }
      key[i] = k;
    }
    warp_aggregated_count(counts, k, act);
  }
}

// out[i] = i: the values of the double-precision plan's radix sort.
__global__ void k_iota(uint64_t n, uint32_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (uint32_t)i;
}

// The active bits of each 32-visibility word.
__global__ void k_word_counts(const uint32_t* __restrict__ bits, uint64_t nwords, uint32_t* __restrict__ out) {
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nwords; w += (uint64_t)gridDim.x * blockDim.x)
    out[w] = (uint32_t)__popc(bits[w]);
}

// The active visibilities' keys and indices, in index order: visibility i
// goes to its word's offset (woff, the exclusive scan of k_word_counts) plus
// the active bits below it in its word.
__global__ void k_compact_active(uint64_t n, const uint32_t* __restrict__ bits, const uint32_t* __restrict__ woff,
                                 const uint32_t* __restrict__ key, uint32_t* __restrict__ kc,
                                 uint32_t* __restrict__ ic) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t w = bits[i >> 5], b = 1u << (i & 31);
    if (w & b) {
      const uint32_t pos = woff[i >> 5] + (uint32_t)__popc(w & (b - 1u));
      kc[pos] = key[i];
      ic[pos] = (uint32_t)i;
    }
  }
}

// Each thread takes four indices a grid-stride apart per round, so that four
// independent atomics (each returning its run's base) are in flight at once:
// the kernel is bound by their latency. The order within a bin is free.
// Visibilities [i0, n); bin k's cursor is cursor[k - koff].
__global__ void k_bin_scatter(uint64_t n, const uint32_t* __restrict__ key, uint32_t* __restrict__ cursor,
                              uint32_t* __restrict__ sorted, uint64_t i0 = 0, uint32_t koff = 0) {
  constexpr int U = 4;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;  // a multiple of 32: warps stay aligned
  const uint64_t nround = i0 + ((n - i0 + 31) & ~31ull);
  for (uint64_t i = i0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nround; i += U * stride) {
    uint32_t k[U], pos[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const uint64_t j = i + u * stride;
      k[u] = j < n ? key[j] : INACTIVE;
    }
#pragma unroll
    for (int u = 0; u < U; u++) pos[u] = warp_aggregated_add(cursor, k[u] - koff, k[u] != INACTIVE);
#pragma unroll
    for (int u = 0; u < U; u++)
      if (k[u] != INACTIVE) sorted[pos[u]] = (uint32_t)(i + u * stride);
  }
}

#include "wgrid_fast.cuh"
#include "wgrid_f64.cuh"

// ------------------------------------------------------------------ exclusive scan (u32)

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
  __shared__ uint32_t warp_tot[SCAN_THREADS / 32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    uint32_t t = lane < nw ? warp_tot[lane] : 0;
    uint32_t s = t;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) warp_tot[lane] = s - t;
    if (lane == nw - 1) *total = s;
  }
  __syncthreads();
  uint32_t r = x - v + warp_tot[wid];
  __syncthreads();
  return r;
}

__global__ void k_scan_tiles(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint64_t n,
                             uint32_t* __restrict__ tile_sums) {
  uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
  uint32_t v[SCAN_ITEMS];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    v[k] = base + k < n ? in[base + k] : 0;
    s += v[k];
  }
  __shared__ uint32_t total;
  uint32_t run = block_exclusive_scan(s, &total);
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_add(uint32_t* __restrict__ out, uint64_t n, const uint32_t* __restrict__ offs) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += offs[i / SCAN_TILE];
}

// out[i] = sum of in[0..i) for i < n (in and out may alias).
void exclusive_scan(const uint32_t* in, uint32_t* out, uint64_t n, cudaStream_t s) {
  uint64_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  DevBuf sums(ntiles * 4, s);
  {
    StageTimer timer_(ST_PREFIX, s);
    k_scan_tiles<<<(unsigned)ntiles, SCAN_THREADS, 0, s>>>(in, out, n, sums.as<uint32_t>());
  }
  check_cuda(cudaGetLastError(), "scan");
  if (ntiles > 1) {
    exclusive_scan(sums.as<uint32_t>(), sums.as<uint32_t>(), ntiles, s);
    {
      StageTimer timer_(ST_PREFIX, s);
      k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, n, sums.as<uint32_t>());
    }
    check_cuda(cudaGetLastError(), "scan");
  }
}

// a[i] += base[c] for i < n, and base[c + 1] = the new a[n - 1]: one row
// chunk's bin offsets after the earlier chunks' visibilities.
__global__ void k_add_base(uint32_t* __restrict__ a, uint64_t n, uint32_t* __restrict__ base, int c) {
  const uint32_t b = base[c];
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = a[i] + b;
    a[i] = v;
    if (i == n - 1) base[c + 1] = v;
  }
}

// ------------------------------------------------------------------ tasks

// Tasks per tile; `stride` bins per tile (nbuckets * nsub).
__global__ void k_task_count(const uint32_t* __restrict__ starts, uint32_t stride, uint32_t ntiles,
                             uint32_t* __restrict__ ntask) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < ntiles) {
    uint32_t c = starts[(uint64_t)(t + 1) * stride] - starts[(uint64_t)t * stride];
    ntask[t] = (c + TASK_CHUNK - 1) / TASK_CHUNK;
  } else if (t == ntiles) {
    ntask[t] = 0;
  }
}

// The first plane of sorted visibility k of the tile whose bins start at b0:
// the bin m with starts[b0 + m] <= k < starts[b0 + m + 1] (binary search).
__device__ __forceinline__ uint32_t plane_at(const uint32_t* starts, uint64_t b0, uint32_t stride, uint32_t nsub,
                                             uint32_t k) {
  uint32_t lo = 0, hi = stride - 1;
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) >> 1;
    if (starts[b0 + mid] <= k)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo / nsub;
}

// `ntiles` counts the (row chunk, tile) pairs; the task keeps the tile.
__global__ void k_task_emit(const uint32_t* __restrict__ starts, uint32_t stride, uint32_t nsub, uint32_t ntiles,
                            uint32_t tiles_per_chunk, const uint32_t* __restrict__ off, Task* __restrict__ tasks,
                            uint32_t* __restrict__ ntotal) {
  // One thread per task: task q belongs to the last tile t with off[t] <= q
  // (that tile has at least one task, as off[t + 1] > q), and is its
  // (q - off[t])-th run of at most TASK_CHUNK visibilities. A dense tile's
  // many tasks are thus emitted in parallel.
  const uint32_t total = off[ntiles];
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q == 0) *ntotal = total;
  if (q >= total) return;
  uint32_t lo = 0, hi = ntiles - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (off[mid] <= q)
      lo = mid;
    else
      hi = mid - 1;
  }
  const uint32_t t = lo;
  const uint64_t b0 = (uint64_t)t * stride;
  const uint32_t e = starts[b0 + stride];
  const uint32_t k0 = starts[b0] + (q - off[t]) * TASK_CHUNK;
  const uint32_t k1 = min(k0 + TASK_CHUNK, e);
  Task tk;
  tk.tile = t % tiles_per_chunk;
  tk.k0 = k0;
  tk.k1 = k1;
  tk.plo = (uint16_t)plane_at(starts, b0, stride, nsub, k0);
  tk.phi = (uint16_t)plane_at(starts, b0, stride, nsub, k1 - 1);
  tasks[q] = tk;
}

// ------------------------------------------------------------------ gridding


// Thread layout of the gridding kernel. Thread (x, y, z) owns the window
// cells whose u index is x mod S, v index y mod S and plane (z + k Z) mod S:
// every footprint (S x S cells on each of S planes) holds exactly one cell of
// each owner and plane residue, so the threads accumulate in shared memory
// without atomics. Each term is added in the grid's fixed-point unit, so the
// sums do not depend on the order of the visibilities.
template <int S>
struct GridLayout {
  static constexpr int S2 = S * S;
  // At most 512 threads (128 registers each) for the large f64 supports.
  static constexpr int Z = S2 * S <= 512 ? S : (512 / S2 > 0 ? 512 / S2 : 1);  // plane-residue groups
  static constexpr int NOWN = S2 * Z;                        // owning threads
  static constexpr int THREADS = (NOWN + 31) / 32 * 32;
  static constexpr int JPER = (S + Z - 1) / Z;  // plane residues per thread
};

// Staging of one batch of visibilities, in two phases. Phase 1 (one thread
// per visibility): the offsets of its first taps in the tile window, its
// first plane, its u and v taps and its value times the w tap of each plane
// (the reference's taps_uv, w_factor, unit_value and data_value,
// wgridder.rs:1565-1591, 1414-1435). Phase 2 (all threads): per visibility
// and owner (x, y) the window offset of the owner's cell and the tap product
// ku * kv there, and per plane residue r the plane's window index and value.
template <class T, int S>
struct GridStaging {
  struct Cell {
    int off;
    T kk;
  };
  struct PlaneVal {
    T re, im;
    int pl;  // plane index in the window, -1 outside it
    int pad;
  };
  int* meta;     // [B] ou | ov << 8, or -1: not gridded in this window
  int* mp;       // [B] first plane
  T* ku;         // [B][S]
  T* kv;         // [B][S]
  cplx<T>* cw;   // [B][S] value * kw(plane mp + j), zero outside the window
  Cell* rc;      // [B][S*S]
  PlaneVal* pw;  // [B][S]
  static constexpr size_t bytes_per_vis() {
    return 2 * sizeof(int) + 2 * S * sizeof(T) + S * sizeof(cplx<T>) + S * S * sizeof(Cell) + S * sizeof(PlaneVal);
  }
  __device__ void carve(unsigned char* base, int B) {
    // Largest alignment first.
    pw = reinterpret_cast<PlaneVal*>(base);
    rc = reinterpret_cast<Cell*>(pw + (size_t)B * S);
    cw = reinterpret_cast<cplx<T>*>(rc + (size_t)B * S * S);
    ku = reinterpret_cast<T*>(cw + (size_t)B * S);
    kv = ku + (size_t)B * S;
    meta = reinterpret_cast<int*>(kv + (size_t)B * S);
    mp = meta + B;
  }
};

template <class T, int S>
int staging_batch() {
  int b = (int)(28672 / GridStaging<T, S>::bytes_per_vis());
  return std::max(1, std::min(b, GridLayout<S>::THREADS));
}

template <class T, int S>
__global__ void __launch_bounds__(GridLayout<S>::THREADS)
    k_grid(const __grid_constant__ Geom<T> g, Inputs in, int mode, const double* __restrict__ uvw,
           const double* __restrict__ foc, const uint32_t* __restrict__ sorted, const Task* __restrict__ tasks,
           const uint32_t* __restrict__ ntasks, typename fast::FixTraits<T>::Cell* __restrict__ grids, int pg0,
           int npg, int gmax, int batch, int* __restrict__ err, fast::FixScale* __restrict__ fs) {
  using Lay = GridLayout<S>;
  using St = GridStaging<T, S>;
  // Each term is rounded once in working precision, then scaled exactly and
  // rounded to an integer in the grid's unit, so the sums are exact.
  using Fx = fast::FixTraits<T>;
  using Acc = typename Fx::Acc;
  struct FixCell {
    Acc re, im;
  };
  constexpr int S2 = S * S;
  if (blockIdx.x >= *ntasks) return;
  extern __shared__ __align__(16) unsigned char smem[];
  const int L = g.L, LL = L * L;
  FixCell* buf = reinterpret_cast<FixCell*>(smem);
  St st;
  st.carve(smem + (size_t)gmax * LL * sizeof(FixCell), batch);
  const T sc = Fx::scale(fs->q);
  bool bad = false;
  const Task t = tasks[blockIdx.x];
  const int tu = (int)(t.tile / (uint32_t)g.ntv), tv = (int)(t.tile - (uint32_t)tu * (uint32_t)g.ntv);
  const int bu = tu << g.log2tile, bv = tv << g.log2tile;
  const unsigned tilesz = 1u << g.log2tile;
  int lo = 0, hi = 0;
  if (g.do_wgridding) {
    lo = max((int)t.plo, pg0);
    hi = min((int)t.phi + S - 1, pg0 + npg - 1);
  }
  const uint32_t nchan = (uint32_t)g.nchan;
  const int tid = threadIdx.x;
  const bool owner = tid < Lay::NOWN;
  const int oz = tid % Lay::Z, oxy = tid / Lay::Z;
  for (int w0 = lo; w0 <= hi; w0 += gmax) {
    const int gw = min(gmax, hi - w0 + 1);
    for (int c = tid; c < gw * LL; c += blockDim.x) buf[c] = FixCell{Fx::zero(), Fx::zero()};
    // The owner's running sums: consecutive contributions to one cell are
    // added in registers and the sum added to the window when the cell changes.
    FixCell acc[Lay::JPER];
    int cur[Lay::JPER];
#pragma unroll
    for (int jj = 0; jj < Lay::JPER; jj++) {
      acc[jj] = FixCell{Fx::zero(), Fx::zero()};
      cur[jj] = -1;
    }
    for (uint32_t kb = t.k0; kb < t.k1; kb += (uint32_t)batch) {
      const int nb = (int)min((uint32_t)batch, t.k1 - kb);
      __syncthreads();
      if (tid < nb) {  // phase 1
        int meta = -1, mpq = 0;
        const uint32_t idx = sorted[kb + tid];
        const uint32_t row = idx / nchan, ch = idx - row * nchan;
        double b[3];
        const double imflip = row_coord(uvw, row, g.fu, g.fv, g.fw, g.r_l, g.r_m, b);
        const double f = foc[ch];
        const double u = b[0] * f, v = b[1] * f, w = b[2] * f;
        const int mp = minplane(g, w);
        if (!g.do_wgridding || (mp <= w0 + gw - 1 && mp + S - 1 >= w0)) {
          double uf, vf;
          int64_t iu0, iv0;
          getpix(g, u, v, uf, vf, iu0, iv0);
          const int ou = offset_in(iu0, g.nu, bu), ov = offset_in(iv0, g.nv, bv);
          if ((unsigned)ou >= tilesz || (unsigned)ov >= tilesz) {
            atomicOr(err, 1);
          } else {
            T ku[S], kv[S];
            const T x0 = (T)(-uf * 2.0 + ((double)S - 1.0));
            const T y0 = (T)(-vf * 2.0 + ((double)S - 1.0));
            eval_taps2<T, S>(g.coeff, g.ne, x0, y0, ku, kv);
            cplx<T> val = unit_value<T>(g, b, imflip, f, in.wgt_kind != WGT_NONE, wgt_get<T>(in, idx));
            if (mode == VALUE_DATA) val = data_value<T>(vis_get<T>(in, idx), val, (T)imflip);
#pragma unroll
            for (int j = 0; j < S; j++) {
              st.ku[tid * S + j] = ku[j];
              st.kv[tid * S + j] = kv[j];
              T kw = (T)0;
              if (g.do_wgridding) {
                const int p = mp + j;
                if (p >= w0 && p < w0 + gw) kw = w_factor<T, S>(g, j, p, w);
              } else if (j == 0) {
                kw = (T)1;
              }
              st.cw[tid * S + j] = cplx<T>{val.re * kw, val.im * kw};
            }
            meta = ou | (ov << 8);
            mpq = mp;
          }
        }
        st.meta[tid] = meta;
        st.mp[tid] = mpq;
      }
      __syncthreads();
      for (int e = tid; e < nb * (S2 + S); e += blockDim.x) {  // phase 2
        if (e < nb * S2) {
          const int q = e / S2, xy = e - q * S2, x = xy / S, y = xy - x * S;
          const int m = st.meta[q];
          typename St::Cell c{0, (T)0};
          if (m >= 0) {
            const int ou = m & 255, ov = m >> 8;
            const int cu = (x - ou % S + S) % S, cv = (y - ov % S + S) % S;
            c.off = (ou + cu) * L + ov + cv;
            c.kk = st.ku[q * S + cu] * st.kv[q * S + cv];
          }
          st.rc[e] = c;
        } else {
          const int e2 = e - nb * S2, q = e2 / S, r = e2 - q * S;
          const int mp = st.mp[q];
          const int j = (r - mp % S + S) % S;
          const int p = mp + j;
          typename St::PlaneVal pv;
          pv.pad = 0;
          const bool in_win = g.do_wgridding ? (p >= w0 && p < w0 + gw) : (j == 0);
          pv.pl = st.meta[q] >= 0 && in_win ? p - w0 : -1;
          pv.re = st.cw[q * S + j].re;
          pv.im = st.cw[q * S + j].im;
          st.pw[e2] = pv;
        }
      }
      __syncthreads();
      if (owner) {  // accumulation, in sorted order
        for (int q = 0; q < nb; q++) {
          if (st.meta[q] < 0) continue;
          const typename St::Cell c = st.rc[q * S2 + oxy];
#pragma unroll
          for (int jj = 0; jj < Lay::JPER; jj++) {
            const int r = oz + jj * Lay::Z;
            if (r >= S) break;
            const typename St::PlaneVal pv = st.pw[q * S + r];
            if (pv.pl < 0) continue;
            const int at = pv.pl * LL + c.off;
            if (at != cur[jj]) {
              if (cur[jj] >= 0) {
                FixCell o = buf[cur[jj]];
                buf[cur[jj]] = FixCell{Fx::add(o.re, acc[jj].re), Fx::add(o.im, acc[jj].im)};
              }
              cur[jj] = at;
              acc[jj] = FixCell{Fx::zero(), Fx::zero()};
            }
            const T tr = pv.re * c.kk, ti = pv.im * c.kk;
            bad |= !isfinite(tr) || !isfinite(ti);
            acc[jj].re = Fx::add(acc[jj].re, Fx::term(tr, sc));
            acc[jj].im = Fx::add(acc[jj].im, Fx::term(ti, sc));
          }
        }
      }
    }
    if (owner) {
#pragma unroll
      for (int jj = 0; jj < Lay::JPER; jj++)
        if (cur[jj] >= 0) {
          FixCell o = buf[cur[jj]];
          buf[cur[jj]] = FixCell{Fx::add(o.re, acc[jj].re), Fx::add(o.im, acc[jj].im)};
        }
    }
    __syncthreads();
    for (int c = tid; c < gw * LL; c += blockDim.x) {
      const FixCell v = buf[c];
      if (!Fx::nonzero(v.re) && !Fx::nonzero(v.im)) continue;
      const int pl = c / LL, rem = c - pl * LL, i = rem / L, j = rem - i * L;
      const int row = (bu + i + g.nu / 2) % g.nu, col = (bv + j + g.nv / 2) % g.nv;
      Fx::flush(grids + ((size_t)(w0 + pl - pg0) * g.nu + row) * g.nv + col, v.re, v.im);
    }
    __syncthreads();
  }
  if (bad) atomicOr(&fs->nonfinite, 1);
}

// ------------------------------------------------------------------ tensor-core gridding (3 x TF32)

// The footprints of K visibilities that share a sub-tile and first w-plane
// (one bin of the sorted order) form, on each of their planes j, a rank-K
// update of one 16 x 8 window of the grid:
//   W_j[i][n] += sum_k A_j[i][k] B[k][n],
//   A_j[i][k] = kw_k(j) ku_k[i - du_k],   B[k][n] = value_k kv_k[n - dv_k],
// with du_k, dv_k the visibility's first tap inside the window. One warp
// takes the bins of a contiguous range of the sorted visibilities, 8 at a
// time, and issues mma.sync m16n8k8 (TF32 inputs, FP32 accumulation) for the
// real and imaginary parts of every plane, keeping all planes' windows in
// registers until the bin ends; the window is then added to the HBM-resident
// planes with float2 atomics. Operands are split as x = hi + lo in TF32 and
// each product formed as hi*hi + hi*lo + lo*hi (3 x TF32), keeping about 21
// bits of each factor. The tensor cores' FP32 accumulation does not round to
// nearest, so each block's three products start from zero and are added to
// the window with rounded FP32 adds: no sum is carried inside the tensor core
// from one block to the next.
//
// Staging (one visibility per lane) stores, per slot, the u taps at [8, 8+S)
// of a zero-padded 24-entry column, the B entries (value * v tap, complex) at
// [4, 4+S) of a 12-entry column, and the S w-taps; the zero padding makes
// every operand fetch a plain load (at row - du + 8, column - dv + 4). Slot
// TC_BATCH is all zero and stands in for the missing visibilities of a short
// block. B is split into TF32 hi and lo where a block loads it, which keeps a
// slot at 256 bytes and lets more warps share an SM.
constexpr int TC_BATCH = 32;
constexpr uint32_t TC_CHUNK = 8192;  // sorted visibilities per warp
// u-tap columns: 24 entries, taps at [8, 8 + S), read at row - du + 8; the
// slot stride (25) is odd so that the lanes' stores fall in distinct banks.
constexpr int TC_USTRIDE = 25;
// B columns: 12 float2 entries, taps at [4, 4 + S), read at column - dv + 4
// (dv < sube <= 5); a slot stride of 96 bytes puts the four slots a half-warp reads
// (eight bytes per lane, four consecutive columns each) 32 bytes apart mod
// 128, in distinct banks.
constexpr int TC_VSTRIDE = 12;
constexpr int TC_WSTRIDE = 9;  // w taps, odd stride as the u taps

struct TcSlots {
  float2* kb;     // [TC_BATCH + 1][TC_VSTRIDE]: value * kv (re, im)
  float* ku;      // [TC_BATCH + 1][TC_USTRIDE]
  float* kw;      // [TC_BATCH + 1][TC_WSTRIDE]
  uint32_t* key;  // [TC_BATCH + 1]
  uint32_t* duv;  // [TC_BATCH + 1]: du | dv << 8
  // Rounded up to whole float4s, all of which the kernel zeroes.
  __host__ __device__ static constexpr size_t bytes() {
    return ((size_t)(TC_BATCH + 1) * (TC_VSTRIDE * sizeof(float2) + (TC_USTRIDE + TC_WSTRIDE) * sizeof(float) + 8) +
            15) / 16 * 16;
  }
  __device__ void carve(unsigned char* base) {
    kb = reinterpret_cast<float2*>(base);
    ku = reinterpret_cast<float*>(kb + (TC_BATCH + 1) * TC_VSTRIDE);
    kw = ku + (TC_BATCH + 1) * TC_USTRIDE;
    key = reinterpret_cast<uint32_t*>(kw + (TC_BATCH + 1) * TC_WSTRIDE);
    duv = key + (TC_BATCH + 1);
  }
};

// x = hi + lo with hi rounded to TF32 (to nearest, ties away; a carry out of
// the mantissa moves into the exponent as rounding requires); lo is exact in
// FP32 and the tensor core reads its leading TF32 bits.
__device__ __forceinline__ void split_fast(float x, uint32_t& hi, uint32_t& lo) {
  hi = (__float_as_uint(x) + 0x1000u) & 0xffffe000u;
  lo = __float_as_uint(x - __uint_as_float(hi));
}
// d = a * b from zero: the first product of a block.
__device__ __forceinline__ void mma_tf32_zero(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%10,%10,%10,%10};\n"
      : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1), "f"(0.0f));
}
__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// The window origin (grid row and column of cell (0, 0)) and first plane of a bin key.
__device__ __forceinline__ void tc_decode(const Geom<float>& g, uint32_t key, int& su0, int& sv0, int& mp) {
  const uint32_t sub = key % (uint32_t)g.nsub, t = key / (uint32_t)g.nsub;
  mp = (int)(t % (uint32_t)g.nbuckets);
  const uint32_t tile = t / (uint32_t)g.nbuckets;
  const uint32_t tu = tile / (uint32_t)g.ntv, tv = tile - tu * (uint32_t)g.ntv;
  // Tiles are laid out on the shifted indices (i0 + n/2) mod n; the grid
  // itself is stored unshifted.
  su0 = (int)(((tu << g.log2tile) + (sub / (uint32_t)g.nsub_side) * (uint32_t)g.sube + (uint32_t)(g.nu - g.nu / 2)) %
              (uint32_t)g.nu);
  sv0 = (int)(((tv << g.log2tile) + (sub % (uint32_t)g.nsub_side) * (uint32_t)g.sube + (uint32_t)(g.nv - g.nv / 2)) %
              (uint32_t)g.nv);
}

// Adds a bin's windows to its planes of the fixed-point grid (each sum
// rounded once to the grid's unit, `sc` = 2^q).
template <int S>
__device__ __forceinline__ void tc_flush(const Geom<float>& g, fast::FixCell* __restrict__ grids, int pg0, int su0,
                                         int sv0, int mp, unsigned pact, const float (&acc)[S][2][4], float sc) {
  const int lane = threadIdx.x & 31, gq = lane >> 2, tq = lane & 3;
  const size_t plane = (size_t)g.nu * g.nv;
#pragma unroll
  for (int j = 0; j < S; j++) {
    if (!((pact >> j) & 1u)) continue;
    fast::FixCell* pl = grids + (size_t)(mp + j - pg0) * plane;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const float re = acc[j][0][r], im = acc[j][1][r];
      if (re == 0.0f && im == 0.0f) continue;
      int row = su0 + gq + (r >= 2 ? 8 : 0), col = sv0 + 2 * tq + (r & 1);
      while (row >= g.nu) row -= g.nu;
      while (col >= g.nv) col -= g.nv;
      fast::fix_add(pl + (size_t)row * g.nv + col, __float2ll_rn(re * sc), __float2ll_rn(im * sc));
    }
  }
}

// Supports up to 6 fit 96 registers (20 warps per SM); wider ones are not capped.
template <int S>
__global__ void __launch_bounds__(TC_BATCH, S <= 6 ? 20 : 12)
    k_grid_tc(const __grid_constant__ Geom<float> g, Inputs in, int mode, const double* __restrict__ uvw,
              const double* __restrict__ foc, const uint32_t* __restrict__ sorted, uint64_t kbase, uint64_t kend,
              fast::FixCell* __restrict__ grids, int pg0, int npg, const fast::FixScale* __restrict__ fs) {
  static_assert(S <= 8, "windows hold 8 + S - 1 <= 16 rows");
  const float fsc = ldexpf(1.0f, fs->q);
  extern __shared__ __align__(16) unsigned char smem[];
  TcSlots st;
  st.carve(smem);
  const int lane = threadIdx.x, gq = lane >> 2, tq = lane & 3;
  for (int c = lane; c < (int)(TcSlots::bytes() / 16); c += TC_BATCH)
    reinterpret_cast<float4*>(smem)[c] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  __syncwarp();
  const uint64_t k0 = kbase + (uint64_t)blockIdx.x * TC_CHUNK;
  const uint64_t k1 = min(kend, k0 + TC_CHUNK);
  const uint32_t nchan = (uint32_t)g.nchan;
  const int np = g.do_wgridding ? S : 1;
  const uint32_t tmask = (1u << g.log2tile) - 1u;
  const uint32_t se = (uint32_t)g.sube;

  float acc[S][2][4];
#pragma unroll
  for (int j = 0; j < S; j++)
#pragma unroll
    for (int c = 0; c < 2; c++)
#pragma unroll
      for (int r = 0; r < 4; r++) acc[j][c][r] = 0.0f;
  uint32_t gcur = INACTIVE;
  int su0 = 0, sv0 = 0, mpc = 0;
  unsigned pact = 0;

  for (uint64_t kb = k0; kb < k1; kb += TC_BATCH) {
    const int nb = (int)min((uint64_t)TC_BATCH, k1 - kb);
    __syncwarp();
    if (lane < nb) {  // staging: one visibility per lane
      uint32_t key = INACTIVE, duv = 0;
      const uint32_t idx = sorted[kb + lane];
      const uint32_t row = idx / nchan, ch = idx - row * nchan;
      double b[3];
      const double imflip = row_coord(uvw, row, g.fu, g.fv, g.fw, g.r_l, g.r_m, b);
      const double f = foc[ch];
      const double u = b[0] * f, v = b[1] * f, w = b[2] * f;
      const int mp = minplane(g, w);
      if (!g.do_wgridding || (mp <= pg0 + npg - 1 && mp + S - 1 >= pg0)) {
        double uf, vf;
        int64_t iu0, iv0;
        getpix(g, u, v, uf, vf, iu0, iv0);
        const uint32_t su = (uint32_t)shifted(iu0, g.nu), sv = (uint32_t)shifted(iv0, g.nv);
        const uint32_t sa = (su & tmask) / se, sb = (sv & tmask) / se;
        key = (((su >> g.log2tile) * (uint32_t)g.ntv + (sv >> g.log2tile)) * (uint32_t)g.nbuckets + (uint32_t)mp) *
                  (uint32_t)g.nsub + sa * (uint32_t)g.nsub_side + sb;
        duv = ((su & tmask) - sa * se) | (((sv & tmask) - sb * se) << 8);
        float ku[S], kv[S];
        const float x0 = (float)(-uf * 2.0 + ((double)S - 1.0));
        const float y0 = (float)(-vf * 2.0 + ((double)S - 1.0));
        eval_taps2<float, S>(g.coeff, g.ne, x0, y0, ku, kv);
        cplx<float> val = unit_value<float>(g, b, imflip, f, in.wgt_kind != WGT_NONE, wgt_get<float>(in, idx));
        if (mode == VALUE_DATA) val = data_value<float>(vis_get<float>(in, idx), val, (float)imflip);
        float* cu = st.ku + lane * TC_USTRIDE + 8;
        float2* cb = st.kb + lane * TC_VSTRIDE + 4;
        float* cw = st.kw + lane * TC_WSTRIDE;
#pragma unroll
        for (int i = 0; i < S; i++) {
          cu[i] = ku[i];
          cb[i] = make_float2(val.re * kv[i], val.im * kv[i]);
        }
        if (g.do_wgridding) {
#pragma unroll
          for (int j = 0; j < S; j++) {
            const int p = mp + j;
            cw[j] = (p >= pg0 && p < pg0 + npg) ? w_factor<float, S>(g, j, p, w) : 0.0f;
          }
        } else {
          cw[0] = 1.0f;
        }
      }
      st.key[lane] = key;
      st.duv[lane] = duv;
    }
    __syncwarp();
    int q = 0;
    while (q < nb) {
      const uint32_t gk = st.key[q];
      if (gk != gcur) {
        if (gcur != INACTIVE) tc_flush<S>(g, grids, pg0, su0, sv0, mpc, pact, acc, fsc);
#pragma unroll
        for (int j = 0; j < S; j++)
#pragma unroll
          for (int c = 0; c < 2; c++)
#pragma unroll
            for (int r = 0; r < 4; r++) acc[j][c][r] = 0.0f;
        gcur = gk;
        pact = 0;
        if (gk != INACTIVE) {
          tc_decode(g, gk, su0, sv0, mpc);
          for (int j = 0; j < np; j++)
            if (mpc + j >= pg0 && mpc + j < pg0 + npg) pact |= 1u << j;
        }
      }
      // The block: the leading visibilities (at most 8) of the current bin.
      const bool same = lane < 8 && q + lane < nb && st.key[q + lane] == gk;
      const unsigned m = __ballot_sync(0xffffffffu, same);
      const int kbk = __ffs(~m) - 1;
      if (gk != INACTIVE) {
        const int e0 = tq < kbk ? q + tq : TC_BATCH, e1 = tq + 4 < kbk ? q + tq + 4 : TC_BATCH;
        const uint32_t d0 = st.duv[e0], d1 = st.duv[e1];
        const int du0 = (int)(d0 & 255u), dv0 = (int)(d0 >> 8), du1 = (int)(d1 & 255u), dv1 = (int)(d1 >> 8);
        const float* u0 = st.ku + e0 * TC_USTRIDE + gq - du0 + 8;
        const float* u1 = st.ku + e1 * TC_USTRIDE + gq - du1 + 8;
        const float ku00 = u0[0], ku01 = u0[8], ku10 = u1[0], ku11 = u1[8];
        const float2 b0 = st.kb[e0 * TC_VSTRIDE + gq - dv0 + 4];
        const float2 b1 = st.kb[e1 * TC_VSTRIDE + gq - dv1 + 4];
        uint32_t brh0, brl0, bih0, bil0, brh1, brl1, bih1, bil1;
        split_fast(b0.x, brh0, brl0);
        split_fast(b0.y, bih0, bil0);
        split_fast(b1.x, brh1, brl1);
        split_fast(b1.y, bih1, bil1);
        const float* w0p = st.kw + e0 * TC_WSTRIDE;
        const float* w1p = st.kw + e1 * TC_WSTRIDE;
        // Planes in pairs: four independent accumulator chains in flight.
#pragma unroll
        for (int j = 0; j < S; j += 2) {
          const bool two = j + 1 < S;
          if (!((pact >> j) & (two ? 3u : 1u))) continue;
          uint32_t ah[2][4], al[2][4];
          float d[2][2][4];  // each block's products start from zero
#pragma unroll
          for (int h = 0; h < 2; h++) {
            if (h == 1 && !two) break;
            const float w0 = w0p[j + h], w1 = w1p[j + h];
            split_fast(w0 * ku00, ah[h][0], al[h][0]);  // A[gq][tq]
            split_fast(w0 * ku01, ah[h][1], al[h][1]);  // A[gq + 8][tq]
            split_fast(w1 * ku10, ah[h][2], al[h][2]);  // A[gq][tq + 4]
            split_fast(w1 * ku11, ah[h][3], al[h][3]);  // A[gq + 8][tq + 4]
          }
#pragma unroll
          for (int h = 0; h < 2; h++)
            if (h == 0 || two) {
              mma_tf32_zero(d[h][0], ah[h], brh0, brh1);
              mma_tf32_zero(d[h][1], ah[h], bih0, bih1);
            }
#pragma unroll
          for (int h = 0; h < 2; h++)
            if (h == 0 || two) {
              mma_tf32(d[h][0], ah[h], brl0, brl1);
              mma_tf32(d[h][1], ah[h], bil0, bil1);
            }
#pragma unroll
          for (int h = 0; h < 2; h++)
            if (h == 0 || two) {
              mma_tf32(d[h][0], al[h], brh0, brh1);
              mma_tf32(d[h][1], al[h], bih0, bih1);
            }
#pragma unroll
          for (int h = 0; h < 2; h++)
            if (h == 0 || two) {
#pragma unroll
              for (int r = 0; r < 4; r++) {
                acc[j + h][0][r] += d[h][0][r];
                acc[j + h][1][r] += d[h][1][r];
              }
            }
        }
      }
      q += kbk;
    }
  }
  if (gcur != INACTIVE) tc_flush<S>(g, grids, pg0, su0, sv0, mpc, pact, acc, fsc);
}

// ------------------------------------------------------------------ tensor-core gridding (3 x BF16)

// The same rank-K window updates as k_grid_tc, with mma.sync m16n8k16 on BF16
// operands: a block holds up to 16 visibilities of one bin, and each operand
// is split as x = hi + lo with both halves rounded to BF16 (8 significant
// bits each, about 16 bits of x), the product formed as hi*hi + hi*lo + lo*hi.
// Each dropped term is below 2^-16 of the product, so a visibility's footprint
// carries a relative error of a few 1e-6; k_grid_tc's 3 x TF32 keeps about 21
// bits. Staging, bins and the flush are k_grid_tc's.

// x0 in the low half, x1 in the high half (the lower column or k index).
__device__ __forceinline__ uint32_t pack_bf16(float x0, float x1) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(x1), "f"(x0));
  return r;
}
// (x0, x1) = hi + lo, both packed as BF16 pairs; x - hi is exact in FP32.
__device__ __forceinline__ void split_bf16(float x0, float x1, uint32_t& hi, uint32_t& lo) {
  hi = pack_bf16(x0, x1);
  lo = pack_bf16(x0 - __uint_as_float(hi << 16), x1 - __uint_as_float(hi & 0xffff0000u));
}
__device__ __forceinline__ void mma_bf16_zero(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%10,%10,%10,%10};\n"
      : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1), "f"(0.0f));
}
__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Supports up to 5 fit 96 registers (20 warps per SM), 6 fits 128 (16 warps)
// without spilling; wider ones are not capped.
template <int S>
__global__ void __launch_bounds__(TC_BATCH, S <= 5 ? 20 : S == 6 ? 16 : 12)
    k_grid_bf16(const __grid_constant__ Geom<float> g, Inputs in, int mode, const double* __restrict__ uvw,
                const double* __restrict__ foc, const uint32_t* __restrict__ sorted, uint64_t kbase, uint64_t kend,
                fast::FixCell* __restrict__ grids, int pg0, int npg, const fast::FixScale* __restrict__ fs) {
  static_assert(S <= 8, "windows hold 8 + S - 1 <= 16 rows");
  const float fsc = ldexpf(1.0f, fs->q);
  extern __shared__ __align__(16) unsigned char smem[];
  TcSlots st;
  st.carve(smem);
  const int lane = threadIdx.x, gq = lane >> 2, tq = lane & 3;
  for (int c = lane; c < (int)(TcSlots::bytes() / 16); c += TC_BATCH)
    reinterpret_cast<float4*>(smem)[c] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  __syncwarp();
  const uint64_t k0 = kbase + (uint64_t)blockIdx.x * TC_CHUNK;
  const uint64_t k1 = min(kend, k0 + TC_CHUNK);
  const uint32_t nchan = (uint32_t)g.nchan;
  const int np = g.do_wgridding ? S : 1;
  const uint32_t tmask = (1u << g.log2tile) - 1u;
  const uint32_t se = (uint32_t)g.sube;

  float acc[S][2][4];
#pragma unroll
  for (int j = 0; j < S; j++)
#pragma unroll
    for (int c = 0; c < 2; c++)
#pragma unroll
      for (int r = 0; r < 4; r++) acc[j][c][r] = 0.0f;
  uint32_t gcur = INACTIVE;
  int su0 = 0, sv0 = 0, mpc = 0;
  unsigned pact = 0;

  for (uint64_t kb = k0; kb < k1; kb += TC_BATCH) {
    const int nb = (int)min((uint64_t)TC_BATCH, k1 - kb);
    __syncwarp();
    if (lane < nb) {  // staging: one visibility per lane, as in k_grid_tc
      uint32_t key = INACTIVE, duv = 0;
      const uint32_t idx = sorted[kb + lane];
      const uint32_t row = idx / nchan, ch = idx - row * nchan;
      double b[3];
      const double imflip = row_coord(uvw, row, g.fu, g.fv, g.fw, g.r_l, g.r_m, b);
      const double f = foc[ch];
      const double u = b[0] * f, v = b[1] * f, w = b[2] * f;
      const int mp = minplane(g, w);
      if (!g.do_wgridding || (mp <= pg0 + npg - 1 && mp + S - 1 >= pg0)) {
        double uf, vf;
        int64_t iu0, iv0;
        getpix(g, u, v, uf, vf, iu0, iv0);
        const uint32_t su = (uint32_t)shifted(iu0, g.nu), sv = (uint32_t)shifted(iv0, g.nv);
        const uint32_t sa = (su & tmask) / se, sb = (sv & tmask) / se;
        key = (((su >> g.log2tile) * (uint32_t)g.ntv + (sv >> g.log2tile)) * (uint32_t)g.nbuckets + (uint32_t)mp) *
                  (uint32_t)g.nsub + sa * (uint32_t)g.nsub_side + sb;
        duv = ((su & tmask) - sa * se) | (((sv & tmask) - sb * se) << 8);
        float ku[S], kv[S];
        const float x0 = (float)(-uf * 2.0 + ((double)S - 1.0));
        const float y0 = (float)(-vf * 2.0 + ((double)S - 1.0));
        eval_taps2<float, S>(g.coeff, g.ne, x0, y0, ku, kv);
        cplx<float> val = unit_value<float>(g, b, imflip, f, in.wgt_kind != WGT_NONE, wgt_get<float>(in, idx));
        if (mode == VALUE_DATA) val = data_value<float>(vis_get<float>(in, idx), val, (float)imflip);
        float* cu = st.ku + lane * TC_USTRIDE + 8;
        float2* cb = st.kb + lane * TC_VSTRIDE + 4;
        float* cw = st.kw + lane * TC_WSTRIDE;
#pragma unroll
        for (int i = 0; i < S; i++) {
          cu[i] = ku[i];
          cb[i] = make_float2(val.re * kv[i], val.im * kv[i]);
        }
        if (g.do_wgridding) {
#pragma unroll
          for (int j = 0; j < S; j++) {
            const int p = mp + j;
            cw[j] = (p >= pg0 && p < pg0 + npg) ? w_factor<float, S>(g, j, p, w) : 0.0f;
          }
        } else {
          cw[0] = 1.0f;
        }
      }
      st.key[lane] = key;
      st.duv[lane] = duv;
    }
    __syncwarp();
    int q = 0;
    while (q < nb) {
      const uint32_t gk = st.key[q];
      if (gk != gcur) {
        if (gcur != INACTIVE) tc_flush<S>(g, grids, pg0, su0, sv0, mpc, pact, acc, fsc);
#pragma unroll
        for (int j = 0; j < S; j++)
#pragma unroll
          for (int c = 0; c < 2; c++)
#pragma unroll
            for (int r = 0; r < 4; r++) acc[j][c][r] = 0.0f;
        gcur = gk;
        pact = 0;
        if (gk != INACTIVE) {
          tc_decode(g, gk, su0, sv0, mpc);
          for (int j = 0; j < np; j++)
            if (mpc + j >= pg0 && mpc + j < pg0 + npg) pact |= 1u << j;
        }
      }
      // The block: the leading visibilities (at most 16) of the current bin.
      const bool same = lane < 16 && q + lane < nb && st.key[q + lane] == gk;
      const unsigned m = __ballot_sync(0xffffffffu, same);
      const int kbk = __ffs(~m) - 1;
      if (gk != INACTIVE) {
        // This lane's k indices: 2 tq, 2 tq + 1, 2 tq + 8, 2 tq + 9.
        int e[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const int k = 2 * tq + (i & 1) + (i >> 1) * 8;
          e[i] = k < kbk ? q + k : TC_BATCH;
        }
        float ku0[4], ku1[4];  // u taps at rows gq and gq + 8
        float2 bv[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const uint32_t d = st.duv[e[i]];
          const int du = (int)(d & 255u), dv = (int)(d >> 8);
          const float* u = st.ku + e[i] * TC_USTRIDE + gq - du + 8;
          ku0[i] = u[0];
          ku1[i] = u[8];
          bv[i] = st.kb[e[i] * TC_VSTRIDE + gq - dv + 4];
        }
        uint32_t brh0, brl0, bih0, bil0, brh1, brl1, bih1, bil1;
        split_bf16(bv[0].x, bv[1].x, brh0, brl0);
        split_bf16(bv[0].y, bv[1].y, bih0, bil0);
        split_bf16(bv[2].x, bv[3].x, brh1, brl1);
        split_bf16(bv[2].y, bv[3].y, bih1, bil1);
        // Planes in pairs: four independent accumulator chains in flight.
#pragma unroll
        for (int j = 0; j < S; j += 2) {
          const bool two = j + 1 < S;
          if (!((pact >> j) & (two ? 3u : 1u))) continue;
          uint32_t ah[2][4], al[2][4];
          float d[2][2][4];  // each block's products start from zero
#pragma unroll
          for (int h = 0; h < 2; h++) {
            if (h == 1 && !two) break;
            float w[4];
#pragma unroll
            for (int i = 0; i < 4; i++) w[i] = st.kw[e[i] * TC_WSTRIDE + j + h];
            split_bf16(w[0] * ku0[0], w[1] * ku0[1], ah[h][0], al[h][0]);  // A[gq][2tq, 2tq+1]
            split_bf16(w[0] * ku1[0], w[1] * ku1[1], ah[h][1], al[h][1]);  // A[gq+8][2tq, 2tq+1]
            split_bf16(w[2] * ku0[2], w[3] * ku0[3], ah[h][2], al[h][2]);  // A[gq][2tq+8, 2tq+9]
            split_bf16(w[2] * ku1[2], w[3] * ku1[3], ah[h][3], al[h][3]);  // A[gq+8][2tq+8, 2tq+9]
          }
#pragma unroll
          for (int h = 0; h < 2; h++)
            if (h == 0 || two) {
              mma_bf16_zero(d[h][0], ah[h], brh0, brh1);
              mma_bf16_zero(d[h][1], ah[h], bih0, bih1);
            }
#pragma unroll
          for (int h = 0; h < 2; h++)
            if (h == 0 || two) {
              mma_bf16(d[h][0], ah[h], brl0, brl1);
              mma_bf16(d[h][1], ah[h], bil0, bil1);
            }
#pragma unroll
          for (int h = 0; h < 2; h++)
            if (h == 0 || two) {
              mma_bf16(d[h][0], al[h], brh0, brh1);
              mma_bf16(d[h][1], al[h], bih0, bih1);
            }
#pragma unroll
          for (int h = 0; h < 2; h++)
            if (h == 0 || two) {
#pragma unroll
              for (int r = 0; r < 4; r++) {
                acc[j + h][0][r] += d[h][0][r];
                acc[j + h][1][r] += d[h][1][r];
              }
            }
        }
      }
      q += kbk;
    }
  }
  if (gcur != INACTIVE) tc_flush<S>(g, grids, pg0, su0, sv0, mpc, pact, acc, fsc);
}

// ------------------------------------------------------------------ degridding

// Row stride of the degridder's shared-memory window: the smallest stride of
// at least L cells that is 2 mod 4. The lanes of a warp mostly read one
// 8 x 2 sub-tile's footprints, at offsets du * stride + dv (du < 8, dv < 2)
// from a common cell; with such a stride those 16 offsets of 8-byte cells
// fall in 16 distinct bank pairs.
__host__ __device__ __forceinline__ int window_stride(int L) { return L + (6 - L % 4) % 4; }

template <class T, int S>
__global__ void __launch_bounds__(GRID_THREADS)
    k_degrid(const __grid_constant__ Geom<T> g, Inputs wts, const double* __restrict__ uvw,
             const double* __restrict__ foc, const uint32_t* __restrict__ sorted, const Task* __restrict__ tasks,
             const uint32_t* __restrict__ ntasks, const cplx<T>* __restrict__ grids, int pg0, int npg, int gmax,
             cplx<T>* __restrict__ vis, int first_group, int last_group, int* __restrict__ err) {
  if (blockIdx.x >= *ntasks) return;
  extern __shared__ __align__(16) unsigned char smem[];
  const int L = g.L, Lp = window_stride(L), LLp = L * Lp;
  cplx<T>* buf = reinterpret_cast<cplx<T>*>(smem);
  const Task t = tasks[blockIdx.x];
  const int tu = (int)(t.tile / (uint32_t)g.ntv), tv = (int)(t.tile - (uint32_t)tu * (uint32_t)g.ntv);
  const int bu = tu << g.log2tile, bv = tv << g.log2tile;
  const unsigned tilesz = 1u << g.log2tile;
  int lo = 0, hi = 0;
  if (g.do_wgridding) {
    lo = max((int)t.plo, pg0);
    hi = min((int)t.phi + S - 1, pg0 + npg - 1);
  }
  const int nwin = lo <= hi ? (hi - lo + gmax) / gmax : 0;
  const int nloop = max(nwin, last_group ? 1 : 0);
  const uint32_t nchan = (uint32_t)g.nchan;
  for (int wi = 0; wi < nloop; wi++) {
    const int w0 = lo + wi * gmax;
    const int gw = wi < nwin ? min(gmax, hi - w0 + 1) : 0;
    // One warp per window row, lanes along the row.
    for (int rr = threadIdx.x >> 5; rr < gw * L; rr += blockDim.x >> 5) {
      const int pl = rr / L, i = rr - pl * L;
      int row = bu + i + g.nu / 2;
      while (row >= g.nu) row -= g.nu;
      const cplx<T>* srow = grids + ((size_t)(w0 + pl - pg0) * g.nu + row) * g.nv;
      cplx<T>* drow = buf + ((size_t)pl * L + i) * Lp;
      for (int j = threadIdx.x & 31; j < L; j += 32) {
        int col = bv + j + g.nv / 2;
        while (col >= g.nv) col -= g.nv;
        drow[j] = srow[col];
      }
    }
    __syncthreads();
    const bool finalize = last_group && wi == nloop - 1;
    const bool fresh = first_group && wi == 0;
    for (uint32_t k = t.k0 + threadIdx.x; k < t.k1; k += blockDim.x) {
      const uint32_t idx = sorted[k];
      const uint32_t row = idx / nchan, ch = idx - row * nchan;
      double b[3];
      const double imflip = row_coord(uvw, row, g.fu, g.fv, g.fw, g.r_l, g.r_m, b);
      const double f = foc[ch];
      const double u = b[0] * f, v = b[1] * f, w = b[2] * f;
      const int mp = minplane(g, w);
      const int plo = g.do_wgridding ? max(mp, w0) : 0;
      const int phi = g.do_wgridding ? min(mp + S - 1, w0 + gw - 1) : (gw > 0 ? 0 : -1);
      cplx<T> acc = fresh ? cplx<T>{(T)0, (T)0} : vis[idx];
      if (plo <= phi) {
        double uf, vf;
        int64_t iu0, iv0;
        getpix(g, u, v, uf, vf, iu0, iv0);
        const int ou = offset_in(iu0, g.nu, bu), ov = offset_in(iv0, g.nv, bv);
        if ((unsigned)ou >= tilesz || (unsigned)ov >= tilesz) {
          atomicOr(err, 1);
          continue;
        }
        T ku[S], kv[S];
        const T x0 = (T)(-uf * 2.0 + ((double)S - 1.0));
        const T y0 = (T)(-vf * 2.0 + ((double)S - 1.0));
        eval_taps2<T, S>(g.coeff, g.ne, x0, y0, ku, kv);
        for (int p = plo; p <= phi; p++) {
          T kk[S];
          if (g.do_wgridding) {
            const T kw = w_factor<T, S>(g, p - mp, p, w);
#pragma unroll
            for (int cu = 0; cu < S; cu++) kk[cu] = ku[cu] * kw;
          } else {
#pragma unroll
            for (int cu = 0; cu < S; cu++) kk[cu] = ku[cu];
          }
          const cplx<T>* src = buf + (size_t)(p - w0) * LLp + ou * Lp + ov;
          T rr = 0, ri = 0;
#pragma unroll
          for (int cu = 0; cu < S; cu++) {
            T tr = 0, tim = 0;
#pragma unroll
            for (int cv = 0; cv < S; cv++) {
              const cplx<T> c = src[cu * Lp + cv];
              tr = fma_t(kv[cv], c.re, tr);
              tim = fma_t(kv[cv], c.im, tim);
            }
            rr = fma_t(kk[cu], tr, rr);
            ri = fma_t(kk[cu], tim, ri);
          }
          acc = {rr + acc.re, ri * (T)imflip + acc.im};
        }
      }
      if (finalize) {  // wgridder.rs:3146-3159
        const T tw = wgt_get<T>(wts, idx);
        if (g.shifting) {
          const cplx<T> ph = shift_phase<T>(g, b, imflip, f, -1.0);
          acc = cmul(acc, cplx<T>{ph.re * tw, ph.im * tw});
        } else {
          acc = {acc.re * tw, acc.im * tw};
        }
      }
      vis[idx] = acc;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ per-pixel stages

struct CorrNodes {
  int n;
  double x[32], w[32];
};

__device__ __forceinline__ double corfunc_dev(const CorrNodes& c, double v) {
  double s = 0.0;
  for (int i = 0; i < c.n; i++) s += c.w[i] * cos(c.x[i] * v);
  return 1.0 / s;
}

// nm1 + r_l x + r_m y + nshift of the pixel's table entry (wgridder.rs:589-599, 806-818).
template <class T>
__device__ __forceinline__ double screen_arg(const Geom<T>& g, int i, int j) {
  int ti = g.lmshift ? i : min(i, g.nx - i), tj = g.lmshift ? j : min(j, g.ny - j);
  double x = g.x0 + (double)ti * g.pixsize_x, y = g.y0 + (double)tj * g.pixsize_y;
  double xsq = x * x, ysq = y * y;
  double tmp = 1.0 - xsq - ysq;
  double nm1 = tmp >= 0.0 ? (-xsq - ysq) / (sqrt(tmp) + 1.0) : -sqrt(-tmp) - 1.0;
  return nm1 + g.r_l * x + g.r_m * y + g.nshift;
}

// The w-screen of plane p at one pixel (screen_par, wgridder.rs:2296-2314).
template <class T>
__device__ __forceinline__ cplx<T> screen(const Geom<T>& g, double s, int p, bool adjoint) {
  double w0 = g.wmin + (double)p * g.dw;
  double phs = w0 * s;
  if (adjoint) phs *= -1.0;
  T ang;
  if (sizeof(T) == 4)
    ang = (T)(2.0 * PI * (phs - floor(phs)));
  else
    ang = (T)(2.0 * PI * phs);
  T sn, cs;
  sincos_t(ang, &sn, &cs);
  return {cs, sn};
}

// global_corrections (wgridder.rs:822-861) per pixel, full image.
template <class T>
__global__ void k_corr(const __grid_constant__ Geom<T> g, const __grid_constant__ CorrNodes cn,
                       const double* __restrict__ cfu, const double* __restrict__ cfv, double* __restrict__ corr) {
  uint64_t npix = (uint64_t)g.nx * g.ny;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < npix; q += (uint64_t)gridDim.x * blockDim.x) {
    int i = (int)(q / g.ny), j = (int)(q - (uint64_t)i * g.ny);
    int ti = g.lmshift ? i : min(i, g.nx - i), tj = g.lmshift ? j : min(j, g.ny - j);
    double x = g.x0 + (double)ti * g.pixsize_x, y = g.y0 + (double)tj * g.pixsize_y;
    double xsq = x * x, ysq = y * y;
    double tmp = 1.0 - xsq - ysq;
    double fct;
    if (tmp >= 0.0) {
      double nm1 = (-xsq - ysq) / (sqrt(tmp) + 1.0);
      double fv = corfunc_dev(cn, (nm1 + g.r_l * x + g.r_m * y + g.nshift) * g.dw);
      if (g.divide_by_n) fv /= nm1 + 1.0;
      fct = fv;
    } else if (g.divide_by_n) {
      fct = 0.0;
    } else {
      fct = corfunc_dev(cn, (-sqrt(-tmp) - 1.0 + g.nshift) * g.dw);
    }
    int iu = g.nx / 2 - min(ti, g.nx - ti), iv = g.ny / 2 - min(tj, g.ny - tj);
    fct *= cfu[iu] * cfv[iv];
    corr[q] = fct;
  }
}

// After the FFTs of a plane group: each pixel's planes, w-screened, summed in
// plane order into `acc`; on the last group the correction gives the image
// (grid_to_image's projection and correct_image, wgridder.rs:2371-2428).
template <class T>
__global__ void k_project(const __grid_constant__ Geom<T> g, const cplx<T>* __restrict__ grids, int pg0, int npg,
                          T* __restrict__ acc, int first, int last, const double* __restrict__ corr,
                          const double* __restrict__ cfu, const double* __restrict__ cfv, T* __restrict__ out) {
  uint64_t npix = (uint64_t)g.nx * g.ny;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < npix; q += (uint64_t)gridDim.x * blockDim.x) {
    int i = (int)(q / g.ny), j = (int)(q - (uint64_t)i * g.ny);
    int ix = (g.nu - g.nx / 2 + i) % g.nu, jx = (g.nv - g.ny / 2 + j) % g.nv;
    T a = first ? (T)0 : acc[q];
    double s = g.do_wgridding ? screen_arg(g, i, j) : 0.0;
    for (int p = pg0; p < pg0 + npg; p++) {
      cplx<T> gv = grids[((size_t)(p - pg0) * g.nu + ix) * g.nv + jx];
      T term;
      if (g.do_wgridding) {
        cplx<T> ph = screen<T>(g, s, p, true);
        term = gv.re * ph.re - gv.im * ph.im;
      } else {
        term = gv.re;
      }
      a = a + term;
    }
    if (!last) {
      acc[q] = a;
    } else if (g.do_wgridding) {
      out[q] = a * (T)corr[q];
    } else {
      int iu = g.nx / 2 - min(i, g.nx - i), iv = g.ny / 2 - min(j, g.ny - j);
      out[q] = (T)((double)a * cfu[iu] * cfv[iv]);
    }
  }
}

// k_project on the transposed columns: plane p's column of image column j is
// t[(p - pg0) * ny + j][.]. Consecutive threads take consecutive image rows i,
// so the reads of t are contiguous.
template <class T>
__global__ void k_project_t(const __grid_constant__ Geom<T> g, const cplx<T>* __restrict__ t, int pg0, int npg,
                            T* __restrict__ acc, int first, int last, const double* __restrict__ corr,
                            const double* __restrict__ cfu, const double* __restrict__ cfv, T* __restrict__ out) {
  uint64_t npix = (uint64_t)g.nx * g.ny;
  for (uint64_t qq = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; qq < npix; qq += (uint64_t)gridDim.x * blockDim.x) {
    int j = (int)(qq / g.nx), i = (int)(qq - (uint64_t)j * g.nx);
    uint64_t q = (uint64_t)i * g.ny + j;
    int ix = (g.nu - g.nx / 2 + i) % g.nu;
    T a = first ? (T)0 : acc[q];
    double s = g.do_wgridding ? screen_arg(g, i, j) : 0.0;
    for (int p = pg0; p < pg0 + npg; p++) {
      cplx<T> gv = t[((size_t)(p - pg0) * g.ny + j) * g.nu + ix];
      T term;
      if (g.do_wgridding) {
        cplx<T> ph = screen<T>(g, s, p, true);
        term = gv.re * ph.re - gv.im * ph.im;
      } else {
        term = gv.re;
      }
      a = a + term;
    }
    if (!last) {
      acc[q] = a;
    } else if (g.do_wgridding) {
      out[q] = a * (T)corr[q];
    } else {
      int iu = g.nx / 2 - min(i, g.nx - i), iv = g.ny / 2 - min(j, g.ny - j);
      out[q] = (T)((double)a * cfu[iu] * cfv[iv]);
    }
  }
}

// The corrected image of a degridding call (wgridder.rs:3064-3091).
template <class T>
__global__ void k_correct_input(const __grid_constant__ Geom<T> g, const T* __restrict__ dirty,
                                const double* __restrict__ corr, const double* __restrict__ cfu,
                                const double* __restrict__ cfv, T* __restrict__ out) {
  uint64_t npix = (uint64_t)g.nx * g.ny;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < npix; q += (uint64_t)gridDim.x * blockDim.x) {
    if (g.do_wgridding) {
      out[q] = dirty[q] * (T)corr[q];
    } else {
      int i = (int)(q / g.ny), j = (int)(q - (uint64_t)i * g.ny);
      int iu = g.nx / 2 - min(i, g.nx - i), iv = g.ny / 2 - min(j, g.ny - j);
      out[q] = dirty[q] * (T)(cfu[iu] * cfv[iv]);
    }
  }
}

// The corrected image times plane p's w-screen, placed on the (zeroed) grid
// at the image rows and columns (image_to_grid, wgridder.rs:2937-2963).
template <class T>
__global__ void k_place(const __grid_constant__ Geom<T> g, const T* __restrict__ img, int p,
                        cplx<T>* __restrict__ grid) {
  uint64_t npix = (uint64_t)g.nx * g.ny;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < npix; q += (uint64_t)gridDim.x * blockDim.x) {
    int i = (int)(q / g.ny), j = (int)(q - (uint64_t)i * g.ny);
    int ix = (g.nu - g.nx / 2 + i) % g.nu, jx = (g.nv - g.ny / 2 + j) % g.nv;
    T d = img[q];
    cplx<T> v;
    if (g.do_wgridding) {
      cplx<T> ph = screen<T>(g, screen_arg(g, i, j), p, false);
      v = {d * ph.re, d * ph.im};
    } else {
      v = {d, (T)0};
    }
    grid[(size_t)ix * g.nv + jx] = v;
  }
}

// The u transforms run on the image columns transposed: t[j][u] holds column
// jx(j) = (nv - ny/2 + j) mod nv of a plane, so that each is one contiguous
// length-nu transform (a single cuFFT pass, where the strided columns took
// four). `rows` is the touched-row count of fft_touched_rows (0: all rows):
// the other rows are zero after gridding and are written as zeros unread.
template <class T>
__global__ void k_cols_to_t(const __grid_constant__ Geom<T> g, const cplx<T>* __restrict__ plane, int rows,
                            cplx<T>* __restrict__ t) {
  __shared__ cplx<T> tile[32][33];
  const int u0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {  // plane rows: consecutive j
    const int u = u0 + k, j = j0 + threadIdx.x;
    cplx<T> v = {(T)0, (T)0};
    if (u < g.nu && j < g.ny && (rows == 0 || u < rows || u >= g.nu - rows))
      v = plane[(size_t)u * g.nv + (g.nv - g.ny / 2 + j) % g.nv];
    tile[k][threadIdx.x] = v;
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {  // t rows: consecutive u
    const int j = j0 + k, u = u0 + threadIdx.x;
    if (u < g.nu && j < g.ny) t[(size_t)j * g.nu + u] = tile[threadIdx.x][k];
  }
}

// The inverse of k_cols_to_t for the rows the degridder reads (`rows` as
// there): plane[u][jx(j)] = t[j][u].
template <class T>
__global__ void k_t_to_cols(const __grid_constant__ Geom<T> g, const cplx<T>* __restrict__ t, int rows,
                            cplx<T>* __restrict__ plane) {
  __shared__ cplx<T> tile[32][33];
  const int u0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {  // t rows: consecutive u
    const int j = j0 + k, u = u0 + threadIdx.x;
    tile[k][threadIdx.x] = (u < g.nu && j < g.ny) ? t[(size_t)j * g.nu + u] : cplx<T>{(T)0, (T)0};
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {  // plane rows: consecutive j
    const int u = u0 + k, j = j0 + threadIdx.x;
    if (u < g.nu && j < g.ny && (rows == 0 || u < rows || u >= g.nu - rows))
      plane[(size_t)u * g.nv + (g.nv - g.ny / 2 + j) % g.nv] = tile[threadIdx.x][k];
  }
}

// k_place into the transposed columns: t[j][ix] (t zeroed first). Consecutive
// threads take consecutive image rows i, so that the writes are contiguous.
template <class T>
__global__ void k_place_t(const __grid_constant__ Geom<T> g, const T* __restrict__ img, int p,
                          cplx<T>* __restrict__ t) {
  uint64_t npix = (uint64_t)g.nx * g.ny;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < npix; q += (uint64_t)gridDim.x * blockDim.x) {
    int j = (int)(q / g.nx), i = (int)(q - (uint64_t)j * g.nx);
    int ix = (g.nu - g.nx / 2 + i) % g.nu;
    T d = img[(size_t)i * g.ny + j];
    cplx<T> v;
    if (g.do_wgridding) {
      cplx<T> ph = screen<T>(g, screen_arg(g, i, j), p, false);
      v = {d * ph.re, d * ph.im};
    } else {
      v = {d, (T)0};
    }
    t[(size_t)j * g.nu + ix] = v;
  }
}

template <class T>
__global__ void k_pixels(const __grid_constant__ Geom<T> g, const double* __restrict__ uvw,
                         const double* __restrict__ foc, Inputs in, int with_vis, int64_t* __restrict__ iu0,
                         int64_t* __restrict__ iv0) {
  uint64_t n = g.nrow * g.nchan;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    if (is_active<T>(in, with_vis != 0, i)) {
      bin_of(g, uvw, foc, (uint32_t)i, &iu0[i], &iv0[i]);
    } else {
      iu0[i] = -1;
      iv0[i] = -1;
    }
  }
}

// ------------------------------------------------------------------ cuFFT plans

template <class T>
struct FftTraits;
template <>
struct FftTraits<float> {
  static constexpr cufftType type = CUFFT_C2C;
  static cufftResult exec(cufftHandle h, cplx<float>* p, int dir) {
    return cufftExecC2C(h, reinterpret_cast<cufftComplex*>(p), reinterpret_cast<cufftComplex*>(p), dir);
  }
};
template <>
struct FftTraits<double> {
  static constexpr cufftType type = CUFFT_Z2Z;
  static cufftResult exec(cufftHandle h, cplx<double>* p, int dir) {
    return cufftExecZ2Z(h, reinterpret_cast<cufftDoubleComplex*>(p), reinterpret_cast<cufftDoubleComplex*>(p), dir);
  }
};

struct FftPair {
  cufftHandle rows = 0, cols = 0;
  std::mutex mu;
};

void check_fft(cufftResult r, const char* what) {
  if (r != CUFFT_SUCCESS) throw DeviceError(std::string("cuFFT ") + what + " failed (" + std::to_string((int)r) + ")");
}

// Row transforms (length nv, nu rows) and image-column transforms (length nu,
// ny/2 columns of stride nv) of one grid size, per device, kept for the life
// of the process.
template <class T>
FftPair& fft_plans(int nu, int nv, int ny) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int, int>, std::unique_ptr<FftPair>> cache;
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "device");
  std::lock_guard<std::mutex> lock(mu);
  auto key = std::make_tuple(dev, nu, nv, ny);
  auto& slot = cache[key];
  if (!slot) {
    auto p = std::make_unique<FftPair>();
    int n_row[1] = {nv};
    check_fft(cufftPlanMany(&p->rows, 1, n_row, nullptr, 1, nv, nullptr, 1, nv, FftTraits<T>::type, nu), "row plan");
    int n_col[1] = {nu};
    int emb[1] = {nu};
    check_fft(cufftPlanMany(&p->cols, 1, n_col, emb, nv, 1, emb, nv, 1, FftTraits<T>::type, ny / 2), "column plan");
    slot = std::move(p);
  }
  return *slot;
}

// The image-column transforms of one plane: columns [nv - ny/2, nv) and [0, ny/2).
template <class T>
void fft_cols(FftPair& f, cplx<T>* plane, int nv, int ny, int dir, cudaStream_t s) {
  std::lock_guard<std::mutex> lock(f.mu);
  check_fft(cufftSetStream(f.cols, s), "stream");
  check_fft(FftTraits<T>::exec(f.cols, plane + (nv - ny / 2), dir), "columns");
  check_fft(FftTraits<T>::exec(f.cols, plane, dir), "columns");
}

template <class T>
void fft_rows(FftPair& f, cplx<T>* plane, int dir, cudaStream_t s) {
  std::lock_guard<std::mutex> lock(f.mu);
  check_fft(cufftSetStream(f.rows, s), "stream");
  check_fft(FftTraits<T>::exec(f.rows, plane, dir), "rows");
}

// Row transforms (length nv) of `batch` consecutive rows, per device, kept
// for the life of the process; batches are rounded up to 64 rows so that few
// plans exist.
template <class T>
FftPair& fft_row_plan(int nv, int batch) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int>, std::unique_ptr<FftPair>> cache;
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "device");
  std::lock_guard<std::mutex> lock(mu);
  auto& slot = cache[std::make_tuple(dev, nv, batch)];
  if (!slot) {
    auto p = std::make_unique<FftPair>();
    int n_row[1] = {nv};
    check_fft(cufftPlanMany(&p->rows, 1, n_row, nullptr, 1, nv, nullptr, 1, nv, FftTraits<T>::type, batch),
              "row plan");
    slot = std::move(p);
  }
  return *slot;
}

// The touched rows as transformed: urows rounded up to 64, or 0 (every row)
// when that would cover the plane.
int touched_row_count(int urows, int nu) {
  const int b = urows > 0 ? (urows + 63) / 64 * 64 : 0;
  return (b == 0 || 2 * b >= nu) ? 0 : b;
}

// The v transforms of the rows footprints can touch: storage rows [0, b)
// and [nu - b, nu), b = touched_row_count (every row when b is 0).
template <class T>
void fft_touched_rows(FftPair& all, cplx<T>* plane, int nu, int nv, int b, int dir, cudaStream_t s) {
  if (b == 0) {
    fft_rows<T>(all, plane, dir, s);
    return;
  }
  FftPair& f = fft_row_plan<T>(nv, b);
  std::lock_guard<std::mutex> lock(f.mu);
  check_fft(cufftSetStream(f.rows, s), "stream");
  check_fft(FftTraits<T>::exec(f.rows, plane, dir), "rows");
  check_fft(FftTraits<T>::exec(f.rows, plane + (size_t)(nu - b) * nv, dir), "rows");
}

template <class T, int S>
void launch_grid(int smem, unsigned nblocks, cudaStream_t s, const Geom<T>& g, const Inputs& in, int mode,
                 const double* uvw, const double* foc, const uint32_t* sorted, const Task* tasks,
                 const uint32_t* ntasks, typename fast::FixTraits<T>::Cell* grids, int pg0, int npg, int gmax,
                 int* err, fast::FixScale* fs) {
  if (nblocks == 0) return;
  const int batch = staging_batch<T, S>();
  const int total = smem + batch * (int)GridStaging<T, S>::bytes_per_vis();
  check_cuda(cudaFuncSetAttribute(k_grid<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, total), "smem");
  {
    StageTimer timer_(ST_GRID, s);
    k_grid<T, S><<<nblocks, GridLayout<S>::THREADS, total, s>>>(g, in, mode, uvw, foc, sorted, tasks, ntasks, grids,
                                                                pg0, npg, gmax, batch, err, fs);
  }
  check_cuda(cudaGetLastError(), "grid kernel");
}

template <int S>
void launch_grid_tc(cudaStream_t s, const Geom<float>& g, const Inputs& in, int mode, const double* uvw,
                    const double* foc, const uint32_t* sorted, uint64_t kbase, uint64_t kend, fast::FixCell* grids,
                    int pg0, int npg, const fast::FixScale* fs) {
  if (kend <= kbase) return;
  const int smem = (int)TcSlots::bytes();
  const unsigned nblocks = (unsigned)((kend - kbase + TC_CHUNK - 1) / TC_CHUNK);
  check_cuda(cudaFuncSetAttribute(k_grid_tc<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem");
  {
    StageTimer timer_(ST_GRID, s);
    k_grid_tc<S><<<nblocks, TC_BATCH, smem, s>>>(g, in, mode, uvw, foc, sorted, kbase, kend, grids, pg0, npg, fs);
  }
  check_cuda(cudaGetLastError(), "grid kernel (tensor cores)");
}

template <int S>
void launch_grid_bf16(cudaStream_t s, const Geom<float>& g, const Inputs& in, int mode, const double* uvw,
                      const double* foc, const uint32_t* sorted, uint64_t kbase, uint64_t kend, fast::FixCell* grids,
                      int pg0, int npg, const fast::FixScale* fs) {
  if (kend <= kbase) return;
  const int smem = (int)TcSlots::bytes();
  const unsigned nblocks = (unsigned)((kend - kbase + TC_CHUNK - 1) / TC_CHUNK);
  check_cuda(cudaFuncSetAttribute(k_grid_bf16<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem");
  {
    StageTimer timer_(ST_GRID, s);
    k_grid_bf16<S><<<nblocks, TC_BATCH, smem, s>>>(g, in, mode, uvw, foc, sorted, kbase, kend, grids, pg0, npg, fs);
  }
  check_cuda(cudaGetLastError(), "grid kernel (tensor cores, 3 x BF16)");
}

// The record count pass for the plan's w-planes, shift and row chunks.
void launch_count_rec(const Geom<float>& g, const double4* rowc, const double* foc, const uint32_t* bits, uint32_t* key,
                      uint32_t* counts, fast::VisRecord* rec, uint32_t rows_per_chunk, uint32_t nbins, uint64_t n,
                      cudaStream_t s, uint64_t i0 = 0, uint32_t koff = 0) {
  auto go = [&](auto wpl, auto shift, auto chunked) {
    fast::k_bin_count_rec<decltype(wpl)::value, decltype(shift)::value, decltype(chunked)::value>
        <<<blocks_for(n - i0, 256), 256, 0, s>>>(g, rowc, foc, bits, key, counts, rec, rows_per_chunk, nbins, i0, n,
                                                 koff);
  };
  using T_ = std::true_type;
  using F_ = std::false_type;
  const bool w = g.do_wgridding != 0, sh = g.shifting != 0, ch = rows_per_chunk != 0;
  if (w) {
    if (sh) {
      if (ch) go(T_{}, T_{}, T_{}); else go(T_{}, T_{}, F_{});
    } else {
      if (ch) go(T_{}, F_{}, T_{}); else go(T_{}, F_{}, F_{});
    }
  } else {
    if (sh) {
      if (ch) go(F_{}, T_{}, T_{}); else go(F_{}, T_{}, F_{});
    } else {
      if (ch) go(F_{}, F_{}, T_{}); else go(F_{}, F_{}, F_{});
    }
  }
}

template <int S>
void launch_grid_i8(cudaStream_t s, const Geom<float>& g, const Inputs& in, int mode, const fast::VisRecord* rec,
                    const uint32_t* sorted, uint64_t kbase, uint64_t kend, uint32_t nbins, fast::FixCell* grids,
                    int pg0, int npg, fast::FixScale* fs, const int* run = nullptr) {
  if (kend <= kbase) return;
  const int smem = (int)(fast::I8Slots::bytes() + fast::I8_BATCH * sizeof(fast::Prefetched));
  const unsigned nblocks = (unsigned)((kend - kbase + fast::I8_CHUNK - 1) / fast::I8_CHUNK);
  check_cuda(cudaFuncSetAttribute(fast::k_grid_i8<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem");
  {
    StageTimer timer_(ST_GRID, s);
    fast::k_grid_i8<S><<<nblocks, fast::I8_BATCH, smem, s>>>(g, in, mode, rec, sorted, kbase, kend, nbins, grids,
                                                             pg0, npg, fs, run);
  }
  check_cuda(cudaGetLastError(), "grid kernel (integer tensor cores)");
}

template <int S>
void launch_grid_f64(cudaStream_t s, const Geom<double>& g, const Inputs& in, int mode, const double* uvw,
                     const double* foc, const uint32_t* key, const uint32_t* sorted, uint64_t kbase, uint64_t kend,
                     uint32_t nbins, fast::FixCell2* grids, int pg0, int npg, fast::FixScale* fs) {
  if (kend <= kbase) return;
  const int smem = (int)(fast::F64Slots::bytes() + fast::F64_BATCH * sizeof(fast::Prefetched64));
  const unsigned nblocks = (unsigned)((kend - kbase + fast::F64_CHUNK - 1) / fast::F64_CHUNK);
  {
    StageTimer timer_(ST_GRID, s);
    fast::k_grid_f64<S><<<nblocks, fast::F64_BATCH, smem, s>>>(g, in, mode, uvw, foc, key, sorted, kbase, kend, nbins,
                                                               grids, pg0, npg, fs);
  }
  check_cuda(cudaGetLastError(), "grid kernel (FP64 tensor cores)");
}

template <int S>
void launch_degrid_h(cudaStream_t s, const Geom<float>& g, const Inputs& wts, const fast::VisRecord* rec,
                     const uint32_t* sorted, uint64_t kbase, uint64_t kend, uint32_t nbins,
                     const cplx<float>* grids, int pg0, int npg, const fast::DegridOut& out, int first, int last,
                     const uint32_t* kb_ptr = nullptr, const uint32_t* ke_ptr = nullptr) {
  // With kb_ptr / ke_ptr the range is read on the device; [kbase, kend)
  // then only bounds its size (the grid covers kend - kbase records).
  if (kend <= kbase) return;
  const int smem = (int)(fast::H16Slots::bytes() + fast::H16_BATCH * sizeof(fast::Prefetched));
  const unsigned nblocks = (unsigned)((kend - kbase + fast::H16_CHUNK - 1) / fast::H16_CHUNK);
  check_cuda(cudaFuncSetAttribute(fast::k_degrid_h<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem");
  {
    StageTimer timer_(ST_DEGRID, s);
    fast::k_degrid_h<S><<<nblocks, fast::H16_BATCH, smem, s>>>(g, wts, rec, sorted, kbase, kend, nbins, grids, pg0,
                                                               npg, out, first, last, kb_ptr, ke_ptr);
  }
  check_cuda(cudaGetLastError(), "degrid kernel (tensor cores)");
}

template <class T, int S>
void launch_degrid(int smem, unsigned nblocks, cudaStream_t s, const Geom<T>& g, const Inputs& wts,
                   const double* uvw, const double* foc, const uint32_t* sorted, const Task* tasks,
                   const uint32_t* ntasks, const cplx<T>* grids, int pg0, int npg, int gmax, cplx<T>* vis,
                   int first, int last, int* err) {
  if (nblocks == 0) return;
  check_cuda(cudaFuncSetAttribute(k_degrid<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem");
  {
    StageTimer timer_(ST_DEGRID, s);
    k_degrid<T, S><<<nblocks, GRID_THREADS, smem, s>>>(g, wts, uvw, foc, sorted, tasks, ntasks, grids, pg0, npg, gmax,
                                                       vis, first, last, err);
  }
  check_cuda(cudaGetLastError(), "degrid kernel");
}

// Dispatch on the support (the reference's with_supp!, wgridder.rs:2225-2244).
template <class F>
void with_supp_float(int supp, F&& f) {
  switch (supp) {
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 5: f(std::integral_constant<int, 5>{}); break;
    case 6: f(std::integral_constant<int, 6>{}); break;
    case 7: f(std::integral_constant<int, 7>{}); break;
    case 8: f(std::integral_constant<int, 8>{}); break;
    default: throw InvalidArgument("kernel support outside 4..=8 in single precision");
  }
}
template <class F>
void with_supp_double(int supp, F&& f) {
  switch (supp) {
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 5: f(std::integral_constant<int, 5>{}); break;
    case 6: f(std::integral_constant<int, 6>{}); break;
    case 7: f(std::integral_constant<int, 7>{}); break;
    case 8: f(std::integral_constant<int, 8>{}); break;
    case 9: f(std::integral_constant<int, 9>{}); break;
    case 10: f(std::integral_constant<int, 10>{}); break;
    case 11: f(std::integral_constant<int, 11>{}); break;
    case 12: f(std::integral_constant<int, 12>{}); break;
    case 13: f(std::integral_constant<int, 13>{}); break;
    case 14: f(std::integral_constant<int, 14>{}); break;
    case 15: f(std::integral_constant<int, 15>{}); break;
    case 16: f(std::integral_constant<int, 16>{}); break;
    default: throw InvalidArgument("kernel support outside 4..=16");
  }
}
}  // namespace

void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw DeviceError(std::string(what) + ": " + cudaGetErrorString(e));
}

const char* const STAGE_NAMES[N_STAGES] = {"scan", "bin_count", "prefix", "bin_scatter", "tasks", "corr", "grid",
                                           "fft", "project", "correct_input", "place", "degrid", "fixed_point", "other"};

namespace {
struct Profiler {
  std::atomic<bool> on{false};
  std::atomic<long long> launches{0};
  std::mutex mu;
  struct Rec {
    int stage;
    int n;
    cudaEvent_t a, b;
  };
  std::vector<Rec> recs;
  long long counts[N_STAGES] = {};
};
Profiler& profiler() {
  static Profiler p;
  return p;
}
}  // namespace

StageTimer::StageTimer(Stage st, cudaStream_t s, int launches) : st_(st), s_(s) {
  Profiler& p = profiler();
  if (st != ST_FFT) p.launches += launches;
  if (p.on.load()) {
    check_cuda(cudaEventCreate(&a_), "event");
    check_cuda(cudaEventCreate(&b_), "event");
    check_cuda(cudaEventRecord(a_, s_), "event");
    std::lock_guard<std::mutex> lock(p.mu);
    p.counts[st] += launches;
  }
}

StageTimer::~StageTimer() {
  if (!a_) return;
  Profiler& p = profiler();
  cudaEventRecord(b_, s_);
  std::lock_guard<std::mutex> lock(p.mu);
  p.recs.push_back({(int)st_, 0, a_, b_});
}

void profile_enable(bool on) { profiler().on = on; }

long long launch_count() { return profiler().launches.load(); }

void profile_read(long long* launches, double* ms) {
  Profiler& p = profiler();
  std::lock_guard<std::mutex> lock(p.mu);
  for (int i = 0; i < N_STAGES; i++) {
    launches[i] = p.counts[i];
    ms[i] = 0.0;
    p.counts[i] = 0;
  }
  for (auto& r : p.recs) {
    float t = 0.0f;
    if (cudaEventSynchronize(r.b) == cudaSuccess && cudaEventElapsedTime(&t, r.a, r.b) == cudaSuccess) ms[r.stage] += t;
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  p.recs.clear();
}

DevBuf& DevBuf::operator=(DevBuf&& o) noexcept {
  if (this != &o) {
    release();
    p_ = o.p_;
    n_ = o.n_;
    s_ = o.s_;
    o.p_ = nullptr;
    o.n_ = 0;
  }
  return *this;
}

namespace {
// A released buffer kept for reuse: free once `ready` (recorded on the
// releasing stream) has passed.
struct CachedBuf {
  void* p;
  size_t bytes;
  int dev;
  cudaEvent_t ready;
};
std::mutex g_cache_mu;
std::vector<CachedBuf> g_cache;  // oldest first

constexpr size_t CACHED_MAX = 128;

// The device's memory in bytes (looked up once per device).
size_t device_bytes(int dev) {
  static std::mutex mu;
  static std::map<int, size_t> total;
  std::lock_guard<std::mutex> lock(mu);
  auto it = total.find(dev);
  if (it != total.end()) return it->second;
  size_t f = 0, t = 0;
  if (cudaMemGetInfo(&f, &t) != cudaSuccess) t = 0;
  total[dev] = t;
  return t;
}

// Returns one cached buffer to the pool, ordered after its release.
void free_cached(const CachedBuf& b, cudaStream_t s) {
  cudaStreamWaitEvent(s, b.ready, 0);
  cudaEventDestroy(b.ready);
  cudaFreeAsync(b.p, s);
}
}  // namespace

size_t cached_free_bytes(int dev) {
  std::lock_guard<std::mutex> lock(g_cache_mu);
  size_t t = 0;
  for (const CachedBuf& b : g_cache)
    if (b.dev == dev) t += b.bytes;
  return t;
}

void flush_cache(int dev) {
  std::vector<CachedBuf> out;
  {
    std::lock_guard<std::mutex> lock(g_cache_mu);
    auto keep = std::stable_partition(g_cache.begin(), g_cache.end(), [&](const CachedBuf& b) { return b.dev != dev; });
    out.assign(keep, g_cache.end());
    g_cache.erase(keep, g_cache.end());
  }
  for (const CachedBuf& b : out) free_cached(b, nullptr);
  if (!out.empty()) cudaStreamSynchronize(nullptr);  // the pool has them back before a retry
}

void DevBuf::alloc(size_t bytes, cudaStream_t s) {
  release();
  if (bytes == 0) return;
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "no CUDA device");
  if (bytes >= CACHED_MIN) {
    bool hit = false;
    CachedBuf b{};
    {
      std::lock_guard<std::mutex> lock(g_cache_mu);
      for (size_t i = g_cache.size(); i-- > 0;)  // the most recent of this size
        if (g_cache[i].dev == dev && g_cache[i].bytes == bytes) {
          b = g_cache[i];
          g_cache.erase(g_cache.begin() + (std::ptrdiff_t)i);
          hit = true;
          break;
        }
    }
    if (hit) {
      const cudaError_t e = cudaStreamWaitEvent(s, b.ready, 0);
      cudaEventDestroy(b.ready);
      if (e != cudaSuccess) {
        cudaFreeAsync(b.p, nullptr);
        check_cuda(e, "device memory");
      }
      p_ = b.p;
      n_ = bytes;
      s_ = s;
      return;
    }
  }
  cudaError_t e = cudaMallocAsync(&p_, bytes, s);
  if (e == cudaErrorMemoryAllocation && cached_free_bytes(dev) > 0) {
    cudaGetLastError();
    flush_cache(dev);
    e = cudaMallocAsync(&p_, bytes, s);
  }
  if (e != cudaSuccess) p_ = nullptr;
  check_cuda(e, "device memory");
  n_ = bytes;
  s_ = s;
}

void DevBuf::release() {
  if (!p_) return;
  cudaEvent_t ev = nullptr;
  int dev = 0;
  if (n_ >= CACHED_MIN && cudaGetDevice(&dev) == cudaSuccess &&
      cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess) {
    if (cudaEventRecord(ev, s_) == cudaSuccess) {
      std::vector<CachedBuf> old;
      {
        // At most CACHED_MAX buffers and three quarters of the device's
        // memory per device (a step of two plans holds about 100 GB at 1 G
        // visibilities); the oldest go back to the pool.
        std::lock_guard<std::mutex> lock(g_cache_mu);
        g_cache.push_back(CachedBuf{p_, n_, dev, ev});
        size_t count = 0, bytes = 0;
        for (const CachedBuf& b : g_cache)
          if (b.dev == dev) {
            count++;
            bytes += b.bytes;
          }
        const size_t cap = device_bytes(dev) / 4 * 3;
        for (size_t i = 0; i < g_cache.size() && (count > CACHED_MAX || bytes > cap);) {
          if (g_cache[i].dev != dev) {
            i++;
            continue;
          }
          count--;
          bytes -= g_cache[i].bytes;
          old.push_back(g_cache[i]);
          g_cache.erase(g_cache.begin() + (std::ptrdiff_t)i);
        }
      }
      for (const CachedBuf& b : old) free_cached(b, s_);
      p_ = nullptr;
      n_ = 0;
      return;
    }
    cudaEventDestroy(ev);
  }
  cudaFreeAsync(p_, s_);
  p_ = nullptr;
  n_ = 0;
}

namespace {
std::atomic<int> g_method{-1};
}

int grid_method() {
  int m = g_method.load();
  if (m < 0) {
    const char* e = std::getenv("RANG_WGRIDDER_GPU_METHOD");
    const std::string v = e ? e : "";
    m = v == "fp32" ? GRID_FP32 : v == "bf16x3" ? GRID_BF16X3 : v == "tf32x3" ? GRID_TF32X3 : GRID_INT8;
    g_method = m;
  }
  return m;
}

void set_grid_method(int m) { g_method = m; }

int max_window_planes(int L, size_t cell_bytes) {
  size_t per = (size_t)L * L * cell_bytes;
  return (int)std::max<size_t>(1, SMEM_WINDOW_BYTES / per);
}

template <class T>
Plan<T>::Plan(const WgridderOptions& o, size_t nrow, size_t nchan, const double* uvw_dev, const double* freq_host,
              const Inputs& act, bool with_vis, cudaStream_t s, int row_chunks, int layout)
    : o_(o), nrow_(nrow), nchan_(nchan), n_(nrow * nchan) {
  rows_per_chunk_ = chunk_rows(nrow, row_chunks);
  nchunk_ = (int)((std::max<size_t>(nrow, 1) + rows_per_chunk_ - 1) / rows_per_chunk_);
  check_common(o, nrow, nchan);
  if (n_ >= 0xffffffffull) throw InvalidArgument("too many visibilities for one call (at most 2^32 - 2)");
  recentring(o, r_l_, r_m_);
  std::vector<double> foc = f_over_c(freq_host, nchan);
  foc_finite_ = all_finite(foc);
  uvw_.alloc(nrow * 3 * sizeof(double), s);
  foc_.alloc(nchan * sizeof(double), s);
  if (nrow) check_cuda(cudaMemcpyAsync(uvw_.get(), uvw_dev, nrow * 3 * sizeof(double), cudaMemcpyDeviceToDevice, s), "copy uvw");
  check_cuda(cudaMemcpyAsync(foc_.get(), foc.data(), nchan * sizeof(double), cudaMemcpyHostToDevice, s), "copy freq");
  err_.alloc(sizeof(int), s);
  check_cuda(cudaMemsetAsync(err_.get(), 0, sizeof(int), s), "memset");
  // Scan.
  DevBuf so(sizeof(ScanOut), s);
  k_scan_init<<<1, 1, 0, s>>>(so.as<ScanOut>());
  double fw = o.flip_w ? 1.0 : -1.0;
  // The active set as bits, for the count pass (one bit per visibility).
  DevBuf bits;
  if (layout && n_) bits.alloc((n_ + 31) / 32 * 4, s);
  if (n_) {
    {
      StageTimer timer_(ST_SCAN, s);
      launch_scan<T>((uint32_t)nrow, (uint32_t)nchan, uvw_.as<double>(), foc_.as<double>(), fw, act, with_vis,
                     foc_finite_, so.as<ScanOut>(), bits.as<uint32_t>(), s);
      k_umax<<<blocks_for(nrow, 256, 148u * 8u), 256, 0, s>>>((uint32_t)nrow, uvw_.as<double>(), so.as<ScanOut>());
    }
    check_cuda(cudaGetLastError(), "scan kernel");
  }
  ScanOut r;
  check_cuda(cudaMemcpyAsync(&r, so.get(), sizeof(r), cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "scan");
  nvis_ = r.count;
  scan_[0] = r.count;
  scan_[1] = r.finite;
  scan_[2] = r.lo_bits;
  scan_[3] = r.hi_bits;
  double wmin_d = 1e300, wmax_d = -1e300;
  if (r.finite) {
    std::memcpy(&wmin_d, &r.lo_bits, sizeof(double));
    std::memcpy(&wmax_d, &r.hi_bits, sizeof(double));
  }
  if (nvis_ == 0) {
    std::memset(&info_, 0, sizeof(info_));
    return;
  }
  bound_.alloc(sizeof(fast::ValueBound), s);
  check_cuda(cudaMemsetAsync(bound_.get(), 0, sizeof(fast::ValueBound), s), "memset");
  fast::k_bound_init<<<1, 1, 0, s>>>(bound_.as<fast::ValueBound>(), r.vmax_bits, r.wmax_bits);
  scale_.alloc(sizeof(fast::FixScale), s);
  scan_in_ = act;
  scan_vis_ = with_vis;
  make_geom<T>(o, nrow, nchan, nvis_, wmin_d, wmax_d, r_l_, r_m_, g_, info_, kernel_);
  double umax_d = 0.0;  // metres; times the largest f / c
  std::memcpy(&umax_d, &r.u_bits, sizeof(double));
  urows_ = touched_rows(umax_d * *std::max_element(foc.begin(), foc.end()), wmax_d);
  if (layout == LAYOUT_FULL) build_layout(act, with_vis, bits.as<uint32_t>(), s);
  if (layout == LAYOUT_STREAMED) {
    bits_ = std::move(bits);
    streamed_ = true;
  }
}

// The grid rows footprints can reach, from the scan's largest |u| and |w|
// (wavelengths): the recentred coordinate is u + r_l w, at most
// |u|max + |r_l| |w|max; its cell offset from the centre is that times
// pixsize_x * nu, and a footprint spans the support around it. Rows beyond
// a margin of a tile plus the support are left untransformed along v (they
// are zero when gridding, and nothing reads them when degridding): the
// reference's touched-row pruning (grid_to_image, wgridder.rs:2320-2399).
template <class T>
int Plan<T>::touched_rows(double umax, double wmax) const {
  if (!(umax >= 0.0) || !std::isfinite(umax) || !(wmax >= 0.0) || !std::isfinite(wmax)) return 0;
  const double ext = (umax + std::fabs(r_l_) * wmax) * g_.pixsize_x;  // in cycles of the grid
  if (!(ext < 0.4)) return 0;  // near the aliasing limit: transform every row
  const double rows = std::ceil(ext * g_.nu) + 2.0 * g_.supp + 64.0;
  if (2.0 * rows >= 0.9 * g_.nu) return 0;
  return (int)rows;
}

template <class T>
void Plan<T>::row_coords(DevBuf& out, cudaStream_t s) const {
  if (nrow_ == 0) return;
  fast::k_row_coords<<<blocks_for(nrow_, 256, 148u * 8u), 256, 0, s>>>(nrow_, uvw_.as<double>(), g_.fu, g_.fv, g_.fw,
                                                                       g_.r_l, g_.r_m, out.as<double4>());
  check_cuda(cudaGetLastError(), "row coordinates");
}

template <class T>
void Plan<T>::build_layout(const Inputs& act, bool with_vis, const uint32_t* bits, cudaStream_t s) {
  ntiles_ = (size_t)g_.ntu * g_.ntv;
  nbins_ = ntiles_ * (size_t)g_.nbuckets * (size_t)g_.nsub;
  if (nbins_ >= 0xffffffffull) throw InvalidArgument("too many uv tiles and w-planes for one call");
  if ((size_t)nchunk_ * nbins_ >= 0xffffffffull) {
    // Row chunks are an optimisation: as many as the 32-bit key space holds
    // (chunks x bins keys, below the inactive key), down to one.
    const size_t kmax = std::max<size_t>(1, (0xffffffffull - 1) / nbins_);
    rows_per_chunk_ = chunk_rows(nrow_, (int)std::min<size_t>(kmax, (size_t)nchunk_));
    nchunk_ = (int)((std::max<size_t>(nrow_, 1) + rows_per_chunk_ - 1) / rows_per_chunk_);
  }
  const size_t K = (size_t)nchunk_, nkeys = K * nbins_, nvt = K * ntiles_;
  key_.alloc(n_ * 4, s);
  starts_.alloc((nkeys + 1) * 4, s);
  check_cuda(cudaMemsetAsync(starts_.get(), 0, (nkeys + 1) * 4, s), "memset");
  if constexpr (sizeof(T) == 4) {  // with the records of the tensor-core kernels
    rec_.alloc(n_ * sizeof(fast::VisRecord), s);
    DevBuf rowc(nrow_ * sizeof(double4), s);
    StageTimer timer_(ST_BIN_COUNT, s);
    row_coords(rowc, s);
    launch_count_rec(g_, rowc.as<double4>(), foc_.as<double>(), bits, key_.as<uint32_t>(), starts_.as<uint32_t>(),
                     rec_.as<fast::VisRecord>(), K > 1 ? (uint32_t)rows_per_chunk_ : 0u, (uint32_t)nbins_, n_, s);
  } else {
    StageTimer timer_(ST_BIN_COUNT, s);
    k_bin_count<T><<<blocks_for(n_, 256), 256, 0, s>>>(g_, uvw_.as<double>(), foc_.as<double>(), act,
                                                        with_vis ? 1 : 0, key_.as<uint32_t>(), starts_.as<uint32_t>(),
                                                        K > 1 ? (uint32_t)rows_per_chunk_ : 0u, (uint32_t)nbins_,
                                                        bits);
  }
  check_cuda(cudaGetLastError(), "bin count");
  exclusive_scan(starts_.as<uint32_t>(), starts_.as<uint32_t>(), nkeys + 1, s);
  if constexpr (sizeof(T) == 8) {
    // A stable radix sort of the visibility indices by bin key: inside a bin
    // the visibilities keep their index order (the reference's layout
    // order), so the double-precision gridder's sums, which follow this
    // order, come out the same on every call. Inactive keys (all ones in
    // the sorted bits: 2^nbits - 1 exceeds every bin key) would sort last.
    int nbits = 1;
    while (nbits < 32 && ((1ull << nbits) - 1ull) < (unsigned long long)nkeys) nbits++;
    if (bits) {
      // Only the active visibilities' (key, index) pairs, compacted in index
      // order through the scan's bits (a bit count per word, its exclusive
      // scan, a place per active bit), are sorted: the radix sort is stable.
      const size_t nwords = (n_ + 31) / 32;
      DevBuf woff(nwords * 4, s), kc(nvis_ * 4, s), ic(nvis_ * 4, s), keys_out(nvis_ * 4, s);
      sorted_.alloc(nvis_ * 4, s);
      StageTimer timer_(ST_BIN_SCATTER, s);
      k_word_counts<<<blocks_for(nwords, 256), 256, 0, s>>>(bits, nwords, woff.as<uint32_t>());
      exclusive_scan(woff.as<uint32_t>(), woff.as<uint32_t>(), nwords, s);
      k_compact_active<<<blocks_for(n_, 256), 256, 0, s>>>(n_, bits, woff.as<uint32_t>(), key_.as<uint32_t>(),
                                                            kc.as<uint32_t>(), ic.as<uint32_t>());
      check_cuda(cudaGetLastError(), "compaction");
      size_t temp = 0;
      check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, temp, kc.as<uint32_t>(), keys_out.as<uint32_t>(),
                                                 ic.as<uint32_t>(), sorted_.as<uint32_t>(), (long long)nvis_, 0,
                                                 nbits, s),
                 "radix sort");
      DevBuf work(temp, s);
      check_cuda(cub::DeviceRadixSort::SortPairs(work.get(), temp, kc.as<uint32_t>(), keys_out.as<uint32_t>(),
                                                 ic.as<uint32_t>(), sorted_.as<uint32_t>(), (long long)nvis_, 0,
                                                 nbits, s),
                 "radix sort");
    } else {  // every visibility's key, inactive ones sorting last
      DevBuf iota(n_ * 4, s), keys_out(n_ * 4, s), vals_out(n_ * 4, s);
      {
        StageTimer timer_(ST_BIN_SCATTER, s);
        k_iota<<<blocks_for(n_, 256), 256, 0, s>>>(n_, iota.as<uint32_t>());
        size_t temp = 0;
        check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, temp, key_.as<uint32_t>(), keys_out.as<uint32_t>(),
                                                   iota.as<uint32_t>(), vals_out.as<uint32_t>(), (long long)n_, 0,
                                                   nbits, s),
                   "radix sort");
        DevBuf work(temp, s);
        check_cuda(cub::DeviceRadixSort::SortPairs(work.get(), temp, key_.as<uint32_t>(), keys_out.as<uint32_t>(),
                                                   iota.as<uint32_t>(), vals_out.as<uint32_t>(), (long long)n_, 0,
                                                   nbits, s),
                   "radix sort");
      }
      sorted_.alloc(nvis_ * 4, s);
      check_cuda(cudaMemcpyAsync(sorted_.get(), vals_out.get(), nvis_ * 4, cudaMemcpyDeviceToDevice, s), "copy");
    }
  } else {
    DevBuf cursor((nkeys + 1) * 4, s);
    check_cuda(cudaMemcpyAsync(cursor.get(), starts_.get(), (nkeys + 1) * 4, cudaMemcpyDeviceToDevice, s), "copy");
    sorted_.alloc(nvis_ * 4, s);
    {
      StageTimer timer_(ST_BIN_SCATTER, s);
      k_bin_scatter<<<blocks_for(n_, 256), 256, 0, s>>>(n_, key_.as<uint32_t>(), cursor.as<uint32_t>(),
                                                         sorted_.as<uint32_t>());
    }
    check_cuda(cudaGetLastError(), "bin scatter");
  }
  // Tasks, over (row chunk, tile) pairs.
  max_tasks_ = nvis_ / TASK_CHUNK + nvt + 1;
  DevBuf ntask((nvt + 1) * 4, s);
  {
    StageTimer timer_(ST_TASKS, s);
    k_task_count<<<(unsigned)((nvt + 1 + 255) / 256), 256, 0, s>>>(starts_.as<uint32_t>(),
                                                                   (uint32_t)(g_.nbuckets * g_.nsub), (uint32_t)nvt,
                                                                   ntask.as<uint32_t>());
  }
  check_cuda(cudaGetLastError(), "tasks");
  exclusive_scan(ntask.as<uint32_t>(), ntask.as<uint32_t>(), nvt + 1, s);
  tasks_.alloc(max_tasks_ * sizeof(Task), s);
  ntasks_.alloc(4, s);
  {
    StageTimer timer_(ST_TASKS, s);
    k_task_emit<<<(unsigned)((max_tasks_ + 255) / 256), 256, 0, s>>>(starts_.as<uint32_t>(),
                                                              (uint32_t)(g_.nbuckets * g_.nsub), (uint32_t)g_.nsub,
                                                              (uint32_t)nvt, (uint32_t)ntiles_, ntask.as<uint32_t>(),
                                                              tasks_.as<Task>(), ntasks_.as<uint32_t>());
  }
  check_cuda(cudaGetLastError(), "tasks");
  // Where each row chunk starts in the sorted order and in the task list.
  // One chunk needs no read-back (and no wait for the device): it spans
  // the whole sorted order, and its launches take the task bound, the
  // kernels stopping at the device-side task count.
  if (K == 1) {
    chunk_sorted_.assign({0u, (uint32_t)nvis_});
    chunk_tasks_.assign({0u, (uint32_t)max_tasks_});
  } else {
    std::vector<uint32_t> so(K + 1), to(K + 1);
    for (size_t c = 0; c <= K; c++) {
      check_cuda(cudaMemcpyAsync(&so[c], starts_.as<uint32_t>() + c * nbins_, 4, cudaMemcpyDeviceToHost, s), "copy");
      check_cuda(cudaMemcpyAsync(&to[c], ntask.as<uint32_t>() + c * ntiles_, 4, cudaMemcpyDeviceToHost, s), "copy");
    }
    check_cuda(cudaStreamSynchronize(s), "layout");
    chunk_sorted_.assign(so.begin(), so.end());
    chunk_tasks_.assign(to.begin(), to.end());
  }
  corrections(s);
}

template <class T>
bool Plan<T>::same_scan(const Inputs& act, bool with_vis, cudaStream_t s) const {
  DevBuf so(sizeof(ScanOut), s);
  k_scan_init<<<1, 1, 0, s>>>(so.as<ScanOut>());
  if (n_) {
    {
      StageTimer timer_(ST_SCAN, s);
      launch_scan<T>((uint32_t)nrow_, (uint32_t)nchan_, uvw_.as<double>(), foc_.as<double>(),
                     o_.flip_w ? 1.0 : -1.0, act, with_vis, foc_finite_, so.as<ScanOut>(), nullptr, s);
    }
    check_cuda(cudaGetLastError(), "scan kernel");
  }
  ScanOut r;
  check_cuda(cudaMemcpyAsync(&r, so.get(), sizeof(r), cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "scan");
  if (r.count != scan_[0] || r.finite != scan_[1]) return false;
  if (!(r.finite == 0 || (r.lo_bits == scan_[2] && r.hi_bits == scan_[3]))) return false;
  if (nvis_ && bound_.get()) {  // the same active set: this scan's value maxima hold for it
    fast::k_bound_init<<<1, 1, 0, s>>>(bound_.as<fast::ValueBound>(), r.vmax_bits, r.wmax_bits);
    scan_in_ = act;
    scan_vis_ = with_vis;
  }
  return true;
}

template <class T>
bool Plan<T>::bound_of(const Inputs& d, ValueMode mode) const {
  if (d.wgt != scan_in_.wgt || d.wgt2 != scan_in_.wgt2 || d.wgt_kind != scan_in_.wgt_kind) return false;
  if (mode == VALUE_UNIT) return true;
  return scan_vis_ && d.vis == scan_in_.vis && d.vis_kind == scan_in_.vis_kind;
}

// The kernel's correction function at the image's pixel frequencies, cfu =
// corfunc(i / nu) for i <= nx / 2 then cfv = corfunc(j / nv) for j <= ny / 2,
// on the current device: computed on the host once per (kernel, grid,
// image) and kept for the life of the process, so that a plan copies it on
// its stream without waiting for the device.
const double* correction_table(const EsKernel* k, size_t nu, size_t nv, size_t nx, size_t ny) {
  static std::mutex mu;
  static std::map<std::tuple<int, const EsKernel*, size_t, size_t, size_t, size_t>, double*> cache;
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "device");
  std::lock_guard<std::mutex> lock(mu);
  double*& slot = cache[std::make_tuple(dev, k, nu, nv, nx, ny)];
  if (!slot) {
    const size_t nu2 = nx / 2 + 1, nv2 = ny / 2 + 1;
    std::vector<double> tab(nu2 + nv2);
    for (size_t i = 0; i < nu2; i++) tab[i] = k->corfunc((double)i * (1.0 / (double)nu));
    for (size_t j = 0; j < nv2; j++) tab[nu2 + j] = k->corfunc((double)j * (1.0 / (double)nv));
    double* d = nullptr;
    check_cuda(cudaMalloc(&d, tab.size() * sizeof(double)), "device memory");
    check_cuda(cudaMemcpy(d, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice), "copy");
    slot = d;
  }
  return slot;
}

template <class T>
void Plan<T>::corrections(cudaStream_t s) {
  // cfu, cfv tables on the host (corfunc_table, wgridder.rs:353-355).
  size_t nu2 = (size_t)g_.nx / 2 + 1, nv2 = (size_t)g_.ny / 2 + 1;
  const double* tab = correction_table(kernel_, g_.nu, g_.nv, g_.nx, g_.ny);
  size_t npix = (size_t)g_.nx * g_.ny;
  corr_.alloc((nu2 + nv2 + (g_.do_wgridding ? npix : 0)) * sizeof(double), s);
  check_cuda(cudaMemcpyAsync(corr_.get(), tab, (nu2 + nv2) * sizeof(double), cudaMemcpyDeviceToDevice, s), "copy");
  if (g_.do_wgridding) {
    CorrNodes cn{};
    cn.n = (int)kernel_->corr_x.size();
    if (cn.n > 32) throw DeviceError("correction quadrature too long");
    for (int i = 0; i < cn.n; i++) {
      cn.x[i] = kernel_->corr_x[i];
      cn.w[i] = kernel_->corr_w[i];
    }
    double* base = corr_.as<double>();
    {
      StageTimer timer_(ST_CORR, s);
      k_corr<T><<<blocks_for(npix, 256), 256, 0, s>>>(g_, cn, base, base + nu2, base + nu2 + nv2);
    }
    check_cuda(cudaGetLastError(), "corrections");
  }
}

// Planes that fit at once: each takes `plane_bytes` (its grid and its image
// columns, transposed); `fixed` bytes more are needed whatever the group.
template <class T>
size_t Plan<T>::plane_group(size_t plane_bytes, size_t fixed) const {
  size_t nplanes = (size_t)std::max(g_.nplanes, 1);
  size_t freeb = 0, total = 0;
  check_cuda(cudaMemGetInfo(&freeb, &total), "memory info");
  auto group_of = [&](size_t avail) {
    size_t budget = std::min<size_t>(avail / 2, (size_t)64 << 30);
    budget = budget > fixed ? budget - fixed : 0;
    return std::min(std::max<size_t>(1, budget / plane_bytes), nplanes);
  };
  int cur = 0;
  if (cudaGetDevice(&cur) == cudaSuccess) freeb += cached_free_bytes(cur);  // this library's to reuse
  size_t group = group_of(freeb);
  if (group < nplanes) {
    // Memory the stream-ordered pool holds without using it is this
    // library's to reuse, though the device does not count it as free. (The
    // query waits for the device, so it is made only when it can matter.)
    int dev = 0;
    cudaMemPool_t pool;
    uint64_t reserved = 0, used = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
      group = group_of(freeb + (size_t)(reserved - used));
  }
  return group;
}

// Zeroes the rows of n planes that the gridder writes and the transforms
// read: every row when `rows` is 0, else storage rows [0, rows) and
// [nu - rows, nu) of each plane (the others are never read).
void zero_touched(void* grids, size_t cell_bytes, int n, int nu, int nv, int rows, cudaStream_t s) {
  const size_t plane = (size_t)nu * nv * cell_bytes, row = (size_t)nv * cell_bytes;
  unsigned char* base = static_cast<unsigned char*>(grids);
  if (rows == 0) {
    check_cuda(cudaMemsetAsync(base, 0, (size_t)n * plane, s), "memset");
    return;
  }
  for (int p = 0; p < n; p++) {
    unsigned char* pl = base + (size_t)p * plane;
    check_cuda(cudaMemsetAsync(pl, 0, (size_t)rows * row, s), "memset");
    check_cuda(cudaMemsetAsync(pl + (size_t)(nu - rows) * row, 0, (size_t)rows * row, s), "memset");
  }
}

// A gridding pass's work space: per plane of a group its fixed-point grid and
// its image columns (transposed), and whatever the group the floating-point
// plane being transformed and the image accumulator.
template <class T>
void Plan<T>::grid_sizes(size_t& plane_bytes, size_t& fixed, size_t& group) const {
  using FixCell = typename fast::FixTraits<T>::Cell;
  const size_t npix = (size_t)o_.nx * o_.ny;
  const size_t plane = (size_t)g_.nu * g_.nv;
  const size_t tplane = (size_t)g_.ny * g_.nu;
  plane_bytes = plane * sizeof(FixCell) + tplane * sizeof(cplx<T>);
  fixed = plane * sizeof(cplx<T>) + npix * sizeof(T);
  group = plane_group(plane_bytes, fixed);
}

template <class T>
size_t Plan<T>::footprint(int nout) const {
  if (nvis_ == 0) return 0;
  size_t plane_bytes, fixed, group;
  grid_sizes(plane_bytes, fixed, group);
  return (size_t)std::max(nout, 1) * (group * plane_bytes + fixed);
}

template <class T>
void Plan<T>::grid(const Inputs& data, ValueMode mode, T* image, cudaStream_t s, const cudaEvent_t* ready,
                   bool scanned, const void* bound) {
  size_t npix = (size_t)o_.nx * o_.ny;
  if (nvis_ == 0) {
    check_cuda(cudaMemsetAsync(image, 0, npix * sizeof(T), s), "memset");
    return;
  }
  if (!sorted_.get()) throw InvalidArgument("this plan was made without the visibility layout");
  using FixCell = typename fast::FixTraits<T>::Cell;
  const size_t cell = sizeof(cplx<T>);
  const size_t nplanes = (size_t)std::max(g_.nplanes, 1);
  const size_t plane = (size_t)g_.nu * g_.nv;
  const size_t tplane = (size_t)g_.ny * g_.nu;  // a plane's image columns, transposed
  size_t plane_bytes, fixed, group;
  grid_sizes(plane_bytes, fixed, group);
  DevBuf grids(group * plane * sizeof(FixCell), s);
  DevBuf fpl(plane * cell, s);  // the plane being transformed, in floating point
  DevBuf cols(group * tplane * cell, s);
  DevBuf acc(group < nplanes ? npix * sizeof(T) : 0, s);
  FftPair& fft = fft_plans<T>(g_.nu, g_.nv, g_.ny);
  const int gmax =
      std::min<int>(max_window_planes(g_.L, sizeof(FixCell)), (int)std::min<size_t>(nplanes, 64));
  const int smem = gmax * g_.L * g_.L * (int)sizeof(FixCell);
  const double* corr = corr_.as<double>();
  const size_t nu2 = (size_t)g_.nx / 2 + 1, nv2 = (size_t)g_.ny / 2 + 1;
  const bool integer = sizeof(T) == 4 && grid_method() == GRID_INT8;
  if (data.vis_kind == VIS_SORTED && !(integer && bound))
    throw DeviceError("stored values need the integer gridder and their bound");
  const bool own_bound = !bound && !(scanned && bound_of(data, mode));
  // Row chunks arriving (`ready`) are gridded as they come when the integer
  // gridder takes all planes at once (k_spec_scale); otherwise the pass
  // waits for all of them.
  const bool speculate = ready && integer && own_bound && nchunk_ > 1 && group >= nplanes && g_.supp <= 8;
  if (ready && !speculate)
    for (int c = 0; c < nchunk_; c++) check_cuda(cudaStreamWaitEvent(s, ready[c], 0), "wait");
  // The fixed-point scales: from the scan's value maxima when `data` is the
  // scanned input, else from a pass over `data`.
  const fast::ValueBound* values = bound_.as<fast::ValueBound>();
  DevBuf vb, spec;
  if (bound) {
    values = static_cast<const fast::ValueBound*>(bound);
  } else if (own_bound) {
    vb.alloc(sizeof(fast::ValueBound), s);
    check_cuda(cudaMemsetAsync(vb.get(), 0, sizeof(fast::ValueBound), s), "memset");
    if (!speculate) {
      StageTimer timer_(ST_OTHER, s);
      fast::k_value_max<T><<<blocks_for(n_, 256, 148u * 8u), 256, 0, s>>>(0, n_, data, key_.as<uint32_t>(),
                                                                         vb.as<fast::ValueBound>());
    }
    check_cuda(cudaGetLastError(), "value bound");
    values = vb.as<fast::ValueBound>();
  }
  if (speculate) {
    spec.alloc(sizeof(fast::SpecState), s);
  } else {
    StageTimer timer_(ST_OTHER, s);
    fast::k_fix_scale<<<1, 1, 0, s>>>(values, mode == VALUE_UNIT ? 1 : 0, (unsigned long long)nvis_, integer ? 1 : 0,
                                      fast::FixTraits<T>::wide, scale_.as<fast::FixScale>());
  }
  check_cuda(cudaGetLastError(), "scale");
  fast::FixScale* fs = scale_.as<fast::FixScale>();
  const int rows = touched_row_count(urows_, g_.nu);
  for (size_t pg0 = 0; pg0 < nplanes; pg0 += group) {
    int n = (int)std::min(group, nplanes - pg0);
    zero_touched(grids.get(), sizeof(FixCell), n, g_.nu, g_.nv, rows, s);
    FixCell* fg = grids.as<FixCell>();
    auto run = [&](auto S) {
      constexpr int SV = decltype(S)::value;
      for (int c = 0; c < nchunk_; c++) {
        if constexpr (sizeof(T) == 4) {
          const uint64_t k0 = chunk_sorted_[c], k1 = chunk_sorted_[c + 1];
          if (speculate) {
            if constexpr (SV <= 8) {
              check_cuda(cudaStreamWaitEvent(s, ready[c], 0), "wait");
              fast::SpecState* st = spec.as<fast::SpecState>();
              {
                StageTimer timer_(ST_OTHER, s);
                fast::k_value_max<T><<<blocks_for(n_ / nchunk_ + 1, 256, 148u * 8u), 256, 0, s>>>(
                    (uint64_t)row_begin(c) * nchan_, (uint64_t)row_begin(c + 1) * nchan_, data, key_.as<uint32_t>(),
                    vb.as<fast::ValueBound>());
                fast::k_spec_scale<<<1, 1, 0, s>>>(vb.as<fast::ValueBound>(), c == 0 ? 1 : 0,
                                                   mode == VALUE_UNIT ? 1 : 0, (unsigned long long)nvis_, 1,
                                                   fast::FixTraits<T>::wide, st, fs);
              }
              check_cuda(cudaGetLastError(), "scale");
              if (c > 0) {
                fast::k_zero_touched_if<FixCell><<<148u * 8u, 256, 0, s>>>(&st->redo, fg, n, g_.nu, g_.nv, rows);
                check_cuda(cudaGetLastError(), "zero");
                for (int j = 0; j < c; j++)
                  launch_grid_i8<SV>(s, g_, data, (int)mode, rec_.as<fast::VisRecord>(), sorted_.as<uint32_t>(),
                                     chunk_sorted_[j], chunk_sorted_[j + 1], (uint32_t)nbins_, fg, (int)pg0, n, fs,
                                     &st->redo);
              }
              launch_grid_i8<SV>(s, g_, data, (int)mode, rec_.as<fast::VisRecord>(), sorted_.as<uint32_t>(), k0, k1,
                                 (uint32_t)nbins_, fg, (int)pg0, n, fs);
            }
            continue;
          }
          if (integer) {
            if constexpr (SV <= 8)
              launch_grid_i8<SV>(s, g_, data, (int)mode, rec_.as<fast::VisRecord>(), sorted_.as<uint32_t>(), k0, k1,
                                 (uint32_t)nbins_, fg, (int)pg0, n, fs);
            continue;
          }
          if (grid_method() == GRID_TF32X3) {
            launch_grid_tc<SV>(s, g_, data, (int)mode, uvw_.as<double>(), foc_.as<double>(), sorted_.as<uint32_t>(),
                               k0, k1, fg, (int)pg0, n, fs);
            continue;
          }
          if (grid_method() == GRID_BF16X3) {
            launch_grid_bf16<SV>(s, g_, data, (int)mode, uvw_.as<double>(), foc_.as<double>(),
                                 sorted_.as<uint32_t>(), k0, k1, fg, (int)pg0, n, fs);
            continue;
          }
        } else if constexpr (SV <= 8) {
          launch_grid_f64<SV>(s, g_, data, (int)mode, uvw_.as<double>(), foc_.as<double>(), key_.as<uint32_t>(),
                              sorted_.as<uint32_t>(), chunk_sorted_[c], chunk_sorted_[c + 1], (uint32_t)nbins_, fg,
                              (int)pg0, n, fs);
          continue;
        }
        launch_grid<T, SV>(smem, chunk_tasks_[c + 1] - chunk_tasks_[c], s, g_, data, (int)mode, uvw_.as<double>(),
                           foc_.as<double>(), sorted_.as<uint32_t>(), tasks_.as<Task>() + chunk_tasks_[c],
                           ntasks_.as<uint32_t>(), fg, (int)pg0, n, gmax, err_.as<int>(), fs);
      }
    };
    if constexpr (sizeof(T) == 4)
      with_supp_float(g_.supp, run);
    else
      with_supp_double(g_.supp, run);
    const dim3 tgrid((unsigned)((g_.nu + 31) / 32), (unsigned)((g_.ny + 31) / 32)), tblock(32, 8);
    FftPair& tf = fft_row_plan<T>(g_.nu, g_.ny);  // the image columns, transposed: ny transforms of length nu
    for (int p = 0; p < n; p++) {
      const FixCell* fpg = fg + (size_t)p * plane;
      cplx<T>* pl = fpl.as<cplx<T>>();
      cplx<T>* tp = cols.as<cplx<T>>() + (size_t)p * tplane;
      {
        StageTimer timer_(ST_FIXED, s);
        const uint64_t ncell = (uint64_t)(rows == 0 ? g_.nu : 2 * rows) * g_.nv;
        fast::k_fix_to_plane<T><<<blocks_for(ncell, 256), 256, 0, s>>>(fpg, g_.nu, g_.nv, rows, fs, pl);
      }
      check_cuda(cudaGetLastError(), "fixed point");
      StageTimer timer_(ST_FFT, s, 3);
      fft_touched_rows<T>(fft, pl, g_.nu, g_.nv, rows, CUFFT_INVERSE, s);
      k_cols_to_t<T><<<tgrid, tblock, 0, s>>>(g_, pl, rows, tp);
      check_cuda(cudaGetLastError(), "transpose");
      std::lock_guard<std::mutex> lock(tf.mu);
      check_fft(cufftSetStream(tf.rows, s), "stream");
      check_fft(FftTraits<T>::exec(tf.rows, tp, CUFFT_INVERSE), "columns");
    }
    bool first = pg0 == 0, last = pg0 + n >= nplanes;
    {
      StageTimer timer_(ST_PROJECT, s);
      k_project_t<T><<<blocks_for(npix, 256), 256, 0, s>>>(g_, cols.as<cplx<T>>(), (int)pg0, n, acc.as<T>(), first,
                                                           last, g_.do_wgridding ? corr + nu2 + nv2 : nullptr, corr,
                                                           corr + nu2, image);
    }
    check_cuda(cudaGetLastError(), "project");
  }
}

template <class T>
void Plan<T>::degrid(const T* image, const Inputs& wts, T* vis, cudaStream_t s, cudaEvent_t* done) {
  degrid_to(image, wts, vis, nullptr, s, done);
}

template <class T>
void Plan<T>::degrid_streamed(const T* image, const Inputs& wts, T* vis, cudaStream_t s, cudaEvent_t* done) {
  if (!streamed_) throw InvalidArgument("this plan was not made for a streamed degridding");
  degrid_to(image, wts, vis, nullptr, s, done);
  // The streamed binning serves this pass only (its chunk offsets stay on
  // the device): the layout goes, and later passes report its absence.
  key_.release();
  starts_.release();
  sorted_.release();
  rec_.release();
}

template <class T>
void Plan<T>::degrid_to(const T* image, const Inputs& wts, T* vis, const void* fused, cudaStream_t s,
                        cudaEvent_t* done) {
  if (vis) check_cuda(cudaMemsetAsync(vis, 0, n_ * 2 * sizeof(T), s), "memset");
  // A LAYOUT_STREAMED plan: bin each row chunk just before degridding it
  // when the tensor-core degridder takes all planes at once, else bin now.
  bool stream_bins = false;
  if (streamed_ && nvis_ > 0) {
    streamed_ = false;
    const size_t nb = (size_t)g_.ntu * g_.ntv * (size_t)g_.nbuckets * (size_t)g_.nsub;
    const size_t np = (size_t)std::max(g_.nplanes, 1), pl = (size_t)g_.nu * g_.nv;
    const size_t npx = (size_t)o_.nx * o_.ny, tpl = (size_t)g_.ny * g_.nu;
    stream_bins = sizeof(T) == 4 && !fused && g_.supp <= 8 && nchunk_ > 1 &&
                  (size_t)nchunk_ * nb < 0xffffffffull &&
                  plane_group(pl * sizeof(cplx<T>), tpl * sizeof(cplx<T>) + npx * sizeof(T)) >= np;
    if (stream_bins) {
      ntiles_ = (size_t)g_.ntu * g_.ntv;
      nbins_ = nb;
      key_.alloc(n_ * 4, s);
      rec_.alloc(n_ * sizeof(fast::VisRecord), s);
      starts_.alloc(((size_t)nchunk_ * nbins_ + 1) * 4, s);
      sorted_.alloc(nvis_ * 4, s);
      corrections(s);
    } else {
      build_layout(scan_in_, scan_vis_, bits_.as<uint32_t>(), s);
    }
  }
  if (nvis_ > 0 && !sorted_.get()) throw InvalidArgument("this plan was made without the visibility layout");
  DevBuf counts, cursor, base, rowc;  // the streamed binning's scratch
  if (stream_bins) {
    rowc.alloc(nrow_ * sizeof(double4), s);
    row_coords(rowc, s);
    counts.alloc((nbins_ + 1) * 4, s);
    cursor.alloc(nbins_ * 4, s);
    base.alloc(((size_t)nchunk_ + 1) * 4, s);
    check_cuda(cudaMemsetAsync(base.get(), 0, ((size_t)nchunk_ + 1) * 4, s), "memset");
  }
  // Row chunk c's binning: its counts, its offsets after the earlier chunks'
  // (base), its placement; the keys are the full plan's (chunk-major).
  auto bin_chunk = [&](int c) {
    const uint64_t i0 = (uint64_t)row_begin(c) * nchan_, i1 = (uint64_t)row_begin(c + 1) * nchan_;
    const uint32_t koff = (uint32_t)((size_t)c * nbins_);
    uint32_t* st = starts_.as<uint32_t>() + (size_t)c * nbins_;
    check_cuda(cudaMemsetAsync(counts.get(), 0, (nbins_ + 1) * 4, s), "memset");
    {
      StageTimer timer_(ST_BIN_COUNT, s);
      if constexpr (sizeof(T) == 4)
        launch_count_rec(g_, rowc.as<double4>(), foc_.as<double>(), bits_.as<uint32_t>(), key_.as<uint32_t>(),
                         counts.as<uint32_t>(), rec_.as<fast::VisRecord>(), (uint32_t)rows_per_chunk_,
                         (uint32_t)nbins_, i1, s, i0, koff);
    }
    check_cuda(cudaGetLastError(), "bin count");
    exclusive_scan(counts.as<uint32_t>(), st, nbins_ + 1, s);
    {
      StageTimer timer_(ST_PREFIX, s);
      k_add_base<<<blocks_for(nbins_ + 1, 256), 256, 0, s>>>(st, nbins_ + 1, base.as<uint32_t>(), c);
    }
    check_cuda(cudaGetLastError(), "offsets");
    check_cuda(cudaMemcpyAsync(cursor.get(), st, nbins_ * 4, cudaMemcpyDeviceToDevice, s), "copy");
    {
      StageTimer timer_(ST_BIN_SCATTER, s);
      k_bin_scatter<<<blocks_for(i1 - i0, 256), 256, 0, s>>>(i1, key_.as<uint32_t>(), cursor.as<uint32_t>(),
                                                              sorted_.as<uint32_t>(), i0, koff);
    }
    check_cuda(cudaGetLastError(), "bin scatter");
  };
  if (nvis_ == 0) {
    if (done)
      for (int c = 0; c < nchunk_; c++) check_cuda(cudaEventRecord(done[c], s), "record");
    return;
  }
  const size_t npix = (size_t)o_.nx * o_.ny;
  const size_t cell = sizeof(cplx<T>);
  const size_t nplanes = (size_t)std::max(g_.nplanes, 1);
  const size_t plane = (size_t)g_.nu * g_.nv;
  const size_t tplane = (size_t)g_.ny * g_.nu;  // a plane's image columns, transposed
  const size_t group = plane_group(plane * cell, tplane * cell + npix * sizeof(T));
  DevBuf grids(group * plane * cell, s);
  DevBuf img(npix * sizeof(T), s);
  FftPair& fft = fft_plans<T>(g_.nu, g_.nv, g_.ny);
  const double* corr = corr_.as<double>();
  const size_t nu2 = (size_t)g_.nx / 2 + 1, nv2 = (size_t)g_.ny / 2 + 1;
  {
    StageTimer timer_(ST_CORRECT_INPUT, s);
    k_correct_input<T><<<blocks_for(npix, 256), 256, 0, s>>>(g_, image, g_.do_wgridding ? corr + nu2 + nv2 : nullptr,
                                                             corr, corr + nu2, img.as<T>());
  }
  check_cuda(cudaGetLastError(), "correct");
  const int Lp = window_stride(g_.L);
  const int gmax = std::min<int>(
      std::max<int>(1, (int)(SMEM_WINDOW_BYTES / ((size_t)g_.L * Lp * sizeof(cplx<T>)))),
      (int)std::min<size_t>(nplanes, 64));
  const int smem = gmax * g_.L * Lp * (int)sizeof(cplx<T>);
  const int rows = touched_row_count(urows_, g_.nu);
  DevBuf cols(tplane * cell, s);
  const dim3 tgrid((unsigned)((g_.nu + 31) / 32), (unsigned)((g_.ny + 31) / 32)), tblock(32, 8);
  FftPair& tf = fft_row_plan<T>(g_.nu, g_.ny);
  for (size_t pg0 = 0; pg0 < nplanes; pg0 += group) {
    int n = (int)std::min(group, nplanes - pg0);
    zero_touched(grids.get(), cell, n, g_.nu, g_.nv, rows, s);
    for (int p = 0; p < n; p++) {
      cplx<T>* pl = grids.as<cplx<T>>() + (size_t)p * plane;
      check_cuda(cudaMemsetAsync(cols.get(), 0, tplane * cell, s), "memset");
      {
        StageTimer timer_(ST_PLACE, s);
        k_place_t<T><<<blocks_for(npix, 256), 256, 0, s>>>(g_, img.as<T>(), (int)pg0 + p, cols.as<cplx<T>>());
      }
      check_cuda(cudaGetLastError(), "place");
      {
        StageTimer timer_(ST_FFT, s, 3);
        {
          std::lock_guard<std::mutex> lock(tf.mu);
          check_fft(cufftSetStream(tf.rows, s), "stream");
          check_fft(FftTraits<T>::exec(tf.rows, cols.as<cplx<T>>(), CUFFT_FORWARD), "columns");
        }
        k_t_to_cols<T><<<tgrid, tblock, 0, s>>>(g_, cols.as<cplx<T>>(), rows, pl);
        check_cuda(cudaGetLastError(), "transpose");
        fft_touched_rows<T>(fft, pl, g_.nu, g_.nv, rows, CUFFT_FORWARD, s);
      }
    }
    bool first = pg0 == 0, last = pg0 + n >= nplanes;
    auto run = [&](auto S) {
      constexpr int SV = decltype(S)::value;
      uint32_t block0 = 0;  // the stored modes' partial sums: blocks of the earlier chunks
      for (int c = 0; c < nchunk_; c++) {  // row chunk c, final after the last plane group
        bool fast_path = false;
        if constexpr (sizeof(T) == 4 && SV <= 8) {
          fast::DegridOut out;
          if (fused) {
            out = *static_cast<const fast::DegridOut*>(fused);
            out.block0 = block0;
            block0 += (uint32_t)((chunk_sorted_[c + 1] - chunk_sorted_[c] + fast::H16_CHUNK - 1) / fast::H16_CHUNK);
          } else {
            out.vis = reinterpret_cast<cplx<float>*>(vis);
          }
          if (stream_bins) {  // the chunk's sorted range is on the device: at most its rows' visibilities
            if (pg0 == 0) bin_chunk(c);
            const uint32_t* st = starts_.as<uint32_t>() + (size_t)c * nbins_;
            launch_degrid_h<SV>(s, g_, wts, rec_.as<fast::VisRecord>(), sorted_.as<uint32_t>(), 0,
                                (uint64_t)(row_begin(c + 1) - row_begin(c)) * nchan_, (uint32_t)nbins_,
                                reinterpret_cast<const cplx<float>*>(grids.as<cplx<T>>()), (int)pg0, n, out, first,
                                last, st, st + nbins_);
          } else {
            launch_degrid_h<SV>(s, g_, wts, rec_.as<fast::VisRecord>(), sorted_.as<uint32_t>(), chunk_sorted_[c],
                                chunk_sorted_[c + 1], (uint32_t)nbins_,
                                reinterpret_cast<const cplx<float>*>(grids.as<cplx<T>>()), (int)pg0, n, out, first,
                                last);
          }
          fast_path = true;
        }
        if (!fast_path && fused) throw DeviceError("stored values need the tensor-core degridder");
        if (!fast_path)
          launch_degrid<T, SV>(smem, chunk_tasks_[c + 1] - chunk_tasks_[c], s, g_, wts, uvw_.as<double>(),
                               foc_.as<double>(), sorted_.as<uint32_t>(), tasks_.as<Task>() + chunk_tasks_[c],
                               ntasks_.as<uint32_t>(), grids.as<cplx<T>>(), (int)pg0, n, gmax,
                               reinterpret_cast<cplx<T>*>(vis), first, last, err_.as<int>());
        if (done && last) check_cuda(cudaEventRecord(done[c], s), "record");
      }
    };
    if constexpr (sizeof(T) == 4)
      with_supp_float(g_.supp, run);
    else
      with_supp_double(g_.supp, run);
  }
}

namespace {

// The residual or Gram values of the paths without the tensor-core kernels
// (double precision, other single-precision methods), by visibility index:
// work[idx] holds the unweighted prediction (has_model) and becomes
// w (d - prediction), w d or, for the Gram operator, w prediction; the
// weighted squares w |value / w|^2 are summed per block as k_store_values
// sums them (fixed order).
template <class T>
__global__ void __launch_bounds__(fast::STORE_THREADS)
    k_values_dense(uint64_t n, const uint32_t* __restrict__ sorted, Inputs data, int sorted_data, int has_model,
                   int gram, cplx<T>* __restrict__ work, double* __restrict__ partials) {
  __shared__ double sh[fast::STORE_THREADS];
  const uint64_t k0 = (uint64_t)blockIdx.x * fast::STORE_CHUNK, k1 = min(n, k0 + fast::STORE_CHUNK);
  double part = 0.0;
  for (uint64_t k = k0 + threadIdx.x; k < k1; k += fast::STORE_THREADS) {
    const uint64_t idx = sorted[k], di = sorted_data ? k : idx;
    const T w = wgt_get<T>(data, di);
    cplx<T> v = has_model ? work[idx] : cplx<T>{(T)0, (T)0};
    if (!gram) {
      const cplx<T> d = vis_get<T>(data, di);
      v = {d.re - v.re, d.im - v.im};
    }
    part += (double)w * ((double)v.re * (double)v.re + (double)v.im * (double)v.im);
    work[idx] = {v.re * w, v.im * w};
  }
  const double sum = fast::block_sum(part, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = sum;
}

// out[k] = dense[sorted[k]] for elements of B bytes.
template <class E>
__global__ void k_gather_sorted(uint64_t n, const uint32_t* __restrict__ sorted, const E* __restrict__ dense,
                                E* __restrict__ out) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
    out[k] = dense[sorted[k]];
}

}  // namespace

template <class T>
bool Plan<T>::fused_values() const {
  return sizeof(T) == 4 && g_.supp <= 8 && grid_method() == GRID_INT8;
}

template <class T>
void Plan<T>::values_pass(bool gram, const Inputs& data, bool sorted_data, const T* model, T* image, double* sum,
                          cudaStream_t s) {
  const size_t npix = (size_t)o_.nx * o_.ny;
  if (nvis_ == 0) {
    check_cuda(cudaMemsetAsync(image, 0, npix * sizeof(T), s), "memset");
    if (sum) check_cuda(cudaMemsetAsync(sum, 0, sizeof(double), s), "memset");
    return;
  }
  if (!sorted_.get()) throw InvalidArgument("this plan was made without the visibility layout");
  const uint64_t nblk = (nvis_ + fast::STORE_CHUNK - 1) / fast::STORE_CHUNK;
  // Partial sums: one per block of the degridder (its chunks rounded up
  // separately) or of the value kernels.
  const size_t nparts_max = nblk + (size_t)nchunk_ + 1;
  if (partials_.size() < nparts_max * sizeof(double)) partials_.alloc(nparts_max * sizeof(double), s);
  if (!res_bound_.get()) res_bound_.alloc(sizeof(fast::ValueBound), s);
  double* partials = partials_.as<double>();
  uint32_t nparts = (uint32_t)nblk;
  const Inputs none{};
  if (fused_values()) {
    if (!stored_.get()) stored_.alloc(nvis_ * sizeof(cplx<float>), s);
    check_cuda(cudaMemsetAsync(res_bound_.get(), 0, sizeof(fast::ValueBound), s), "memset");
    cplx<float>* stored = stored_.as<cplx<float>>();
    if (model) {
      fast::DegridOut out;
      out.mode = gram ? fast::DEGRID_GRAM : fast::DEGRID_RESIDUAL;
      out.stored = stored;
      out.data = data;
      out.sorted_data = sorted_data ? 1 : 0;
      out.partials = partials;
      out.bound = res_bound_.as<fast::ValueBound>();
      degrid_to(model, none, nullptr, &out, s, nullptr);
      nparts = 0;
      for (int c = 0; c < nchunk_; c++)
        nparts += (uint32_t)((chunk_sorted_[c + 1] - chunk_sorted_[c] + fast::H16_CHUNK - 1) / fast::H16_CHUNK);
    } else {
      {
        StageTimer timer_(ST_OTHER, s);
        fast::k_store_values<<<(unsigned)nblk, fast::STORE_THREADS, 0, s>>>(
            nvis_, sorted_.as<uint32_t>(), data, sorted_data ? 1 : 0, stored, partials,
            res_bound_.as<fast::ValueBound>());
      }
      check_cuda(cudaGetLastError(), "stored values");
    }
    const Inputs vals{stored, VIS_SORTED, nullptr, nullptr, WGT_NONE, nullptr};
    grid(vals, VALUE_DATA, image, s, nullptr, false, res_bound_.get());
  } else {
    if (!work_.get()) work_.alloc(n_ * sizeof(cplx<T>), s);
    cplx<T>* work = work_.as<cplx<T>>();
    if (model) degrid_to(model, none, reinterpret_cast<T*>(work), nullptr, s, nullptr);
    {
      StageTimer timer_(ST_OTHER, s);
      k_values_dense<T><<<(unsigned)nblk, fast::STORE_THREADS, 0, s>>>(
          nvis_, sorted_.as<uint32_t>(), data, sorted_data ? 1 : 0, model ? 1 : 0, gram ? 1 : 0, work, partials);
    }
    check_cuda(cudaGetLastError(), "residual values");
    const Inputs vals{work, sizeof(T) == 4 ? VIS_C64 : VIS_C128, nullptr, nullptr, WGT_NONE, nullptr};
    grid(vals, VALUE_DATA, image, s, nullptr, false);
  }
  if (sum) {
    {
      StageTimer timer_(ST_OTHER, s);
      fast::k_sum_partials<<<1, fast::STORE_THREADS, 0, s>>>(partials, nparts, sum);
    }
    check_cuda(cudaGetLastError(), "misfit sum");
  }
}

template <class T>
void Plan<T>::residual(const Inputs& data, bool sorted_data, const T* model, T* image, double* misfit,
                       cudaStream_t s) {
  values_pass(false, data, sorted_data, model, image, misfit, s);
}

template <class T>
void Plan<T>::gram(const T* x, const Inputs& wts, bool sorted_wts, T* image, double* xgx, cudaStream_t s) {
  Inputs w = wts;
  w.vis = nullptr;
  w.vis_kind = VIS_UNIT;
  values_pass(true, w, sorted_wts, x, image, xgx, s);
}

template <class T>
void Plan<T>::gather_sorted(const void* dense, int elem_bytes, void* out, cudaStream_t s) const {
  if (nvis_ == 0) return;
  if (!sorted_.get()) throw InvalidArgument("this plan was made without the visibility layout");
  const uint32_t* srt = sorted_.as<uint32_t>();
  const unsigned nb = blocks_for(nvis_, 256);
  switch (elem_bytes) {
    case 1:
      k_gather_sorted<uint8_t><<<nb, 256, 0, s>>>(nvis_, srt, (const uint8_t*)dense, (uint8_t*)out);
      break;
    case 4:
      k_gather_sorted<uint32_t><<<nb, 256, 0, s>>>(nvis_, srt, (const uint32_t*)dense, (uint32_t*)out);
      break;
    case 8:
      k_gather_sorted<uint2><<<nb, 256, 0, s>>>(nvis_, srt, (const uint2*)dense, (uint2*)out);
      break;
    case 16:
      k_gather_sorted<uint4><<<nb, 256, 0, s>>>(nvis_, srt, (const uint4*)dense, (uint4*)out);
      break;
    default:
      throw InvalidArgument("element size must be 1, 4, 8 or 16 bytes");
  }
  check_cuda(cudaGetLastError(), "gather");
}

template <class T>
std::vector<const char*> Plan<T>::memory_names() {
  return {"gridder: coordinates (uvw per row, f/c per channel)",
          "gridder: bin keys and offsets",
          "gridder: sorted visibility index",
          "gridder: visibility records",
          "gridder: tasks",
          "gridder: corrections",
          "gridder: stored sorted values",
          "gridder: scalars and partial sums"};
}

template <class T>
std::vector<std::pair<const char*, size_t>> Plan<T>::memory() const {
  const std::vector<const char*> n = memory_names();
  const size_t b[] = {uvw_.size() + foc_.size(),
                      key_.size() + starts_.size(),
                      sorted_.size(),
                      rec_.size(),
                      tasks_.size() + ntasks_.size(),
                      corr_.size(),
                      stored_.size() + work_.size(),
                      bound_.size() + scale_.size() + err_.size() + partials_.size() + res_bound_.size()};
  std::vector<std::pair<const char*, size_t>> out;
  for (size_t i = 0; i < n.size(); i++) out.emplace_back(n[i], b[i]);
  return out;
}

template <class T>
void Plan<T>::release_work() {
  stored_.release();
  work_.release();
}

template <class T>
int Plan<T>::kernel_errors(cudaStream_t s) const {
  int e = 0;
  if (!err_.get()) return 0;
  check_cuda(cudaMemcpyAsync(&e, err_.get(), sizeof(int), cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "stream");
  return e;
}

template <class T>
void Plan<T>::export_binning(uint32_t* key_host, uint32_t* sorted_host, cudaStream_t s) const {
  if (nvis_ == 0) return;
  if (nchunk_ != 1) throw DeviceError("binning export of a plan with row chunks");
  check_cuda(cudaMemcpyAsync(key_host, key_.get(), n_ * 4, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "copy");
  // The reference's key, tile * nbuckets + plane, without the sub-tile.
  for (size_t i = 0; i < n_; i++)
    if (key_host[i] != INACTIVE) key_host[i] /= (uint32_t)g_.nsub;
  // The reference's layout order (tile, first plane, row, channel): the
  // device's keys ordered by a stable counting sort. The device's own sorted
  // order leaves the order inside a bin free; gridding sums exact terms, so
  // the results do not depend on it.
  const size_t nref = (size_t)g_.ntu * g_.ntv * (size_t)g_.nbuckets;
  std::vector<uint32_t> start(nref + 1, 0);
  for (size_t i = 0; i < n_; i++)
    if (key_host[i] != INACTIVE) start[key_host[i] + 1]++;
  for (size_t b = 0; b < nref; b++) start[b + 1] += start[b];
  for (size_t i = 0; i < n_; i++)
    if (key_host[i] != INACTIVE) sorted_host[start[key_host[i]]++] = (uint32_t)i;
}

template <class T>
void Plan<T>::export_pixels(const Inputs& act, bool with_vis, int64_t* iu0_host, int64_t* iv0_host,
                            cudaStream_t s) const {
  if (nvis_ == 0) return;
  DevBuf a(n_ * 8, s), b(n_ * 8, s);
  {
    StageTimer timer_(ST_OTHER, s);
    k_pixels<T><<<blocks_for(n_, 256), 256, 0, s>>>(g_, uvw_.as<double>(), foc_.as<double>(), act, with_vis ? 1 : 0,
                                                    a.as<int64_t>(), b.as<int64_t>());
  }
  check_cuda(cudaGetLastError(), "pixels");
  check_cuda(cudaMemcpyAsync(iu0_host, a.get(), n_ * 8, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaMemcpyAsync(iv0_host, b.get(), n_ * 8, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "copy");
}

template class Plan<float>;
template class Plan<double>;

}  // namespace wg

// ------------------------------------------------------------------ binning without allocation

// The visibility binning of a call with every temporary in one file-scope
// device array instead of allocated memory, for callers that must not
// allocate device memory. The array is NOALLOC_SCRATCH_BYTES on every device
// that loads the library, for the life of the process. Its address is taken
// once per device with cudaGetSymbolAddress (a symbol's host-side name is not
// a device address). All calls share it: the counters are cleared on every
// call, and calls whose work overlaps on the GPU race on it.
namespace wg {

constexpr size_t NOALLOC_SCRATCH_BYTES = 16u << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {

// The scratch address on the current device, looked up on first use.
unsigned char* noalloc_scratch() {
  static std::mutex mu;
  static std::map<int, unsigned char*> addr;
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "no CUDA device");
  std::lock_guard<std::mutex> lock(mu);
  auto it = addr.find(dev);
  if (it != addr.end()) return it->second;
  void* p = nullptr;
  check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "no-allocation scratch address");
  addr[dev] = static_cast<unsigned char*>(p);
  return addr[dev];
}

// exclusive_scan with the tile sums of every level in `tmp` (no allocation).
void exclusive_scan_in(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* tmp, cudaStream_t s) {
  uint64_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  k_scan_tiles<<<(unsigned)ntiles, SCAN_THREADS, 0, s>>>(in, out, n, tmp);
  check_cuda(cudaGetLastError(), "scan");
  if (ntiles > 1) {
    exclusive_scan_in(tmp, tmp, ntiles, tmp + ntiles, s);
    k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, n, tmp);
    check_cuda(cudaGetLastError(), "scan");
  }
}

uint64_t scan_tmp_words(uint64_t n) {
  uint64_t words = 0;
  for (uint64_t m = (n + SCAN_TILE - 1) / SCAN_TILE; m > 1; m = (m + SCAN_TILE - 1) / SCAN_TILE) words += m;
  return words + 2;
}

__global__ void k_reference_key(uint64_t n, uint32_t nsub, uint32_t* __restrict__ key) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    if (key[i] != INACTIVE) key[i] /= nsub;
}

template <class T>
void bin_noalloc(const WgridderOptions& o, size_t nrow, size_t nchan, const double* uvw, const double* freq,
                 const Inputs& act, cudaStream_t s, uint32_t* key, uint32_t* sorted, size_t* nsorted, double* info) {
  check_common(o, nrow, nchan);
  const uint64_t n = (uint64_t)nrow * nchan;
  if (n >= 0xffffffffull) throw InvalidArgument("too many visibilities for one call (at most 2^32 - 2)");
  double r_l, r_m;
  recentring(o, r_l, r_m);
  std::vector<double> foc = f_over_c(freq, nchan);
  // Scratch layout: the scan result, the channel factors, then u32 words.
  unsigned char* base = noalloc_scratch();
  const size_t foc_off = 256, words_off = (foc_off + nchan * sizeof(double) + 255) / 256 * 256;
  if (words_off > NOALLOC_SCRATCH_BYTES)
    throw InvalidArgument("too many channels for the no-allocation scratch (" +
                          std::to_string(NOALLOC_SCRATCH_BYTES) + " bytes)");
  ScanOut* so = reinterpret_cast<ScanOut*>(base);
  double* dfoc = reinterpret_cast<double*>(base + foc_off);
  k_scan_init<<<1, 1, 0, s>>>(so);
  check_cuda(cudaMemcpyAsync(dfoc, foc.data(), nchan * sizeof(double), cudaMemcpyHostToDevice, s), "copy");
  const double fw = o.flip_w ? 1.0 : -1.0;
  if (n) {
    launch_scan<T>((uint32_t)nrow, (uint32_t)nchan, uvw, dfoc, fw, act, false, all_finite(foc), so, nullptr, s);
    check_cuda(cudaGetLastError(), "scan kernel");
  }
  ScanOut r;
  check_cuda(cudaMemcpyAsync(&r, so, sizeof(r), cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "scan");
  *nsorted = r.count;
  if (r.count == 0) {
    std::memset(info, 0, N_INFO * sizeof(double));
    if (n) check_cuda(cudaMemsetAsync(key, 0xff, n * sizeof(uint32_t), s), "memset");
    check_cuda(cudaStreamSynchronize(s), "binning");
    return;
  }
  double wmin_d = 1e300, wmax_d = -1e300;
  if (r.finite) {
    std::memcpy(&wmin_d, &r.lo_bits, sizeof(double));
    std::memcpy(&wmax_d, &r.hi_bits, sizeof(double));
  }
  Geom<T> g;
  PlanInfo pi;
  EsKernel* kernel = nullptr;
  make_geom<T>(o, nrow, nchan, r.count, wmin_d, wmax_d, r_l, r_m, g, pi, kernel);
  // The export orders by (tile, first plane) only: one sub-tile per tile, so
  // the counters are one per (tile, plane), the reference's bins.
  g.sube = 1 << g.log2tile;
  g.nsub_side = 1;
  g.nsub = 1;
  const uint64_t nbins = (uint64_t)g.ntu * g.ntv * g.nbuckets * g.nsub;
  const uint64_t need_words = 2 * (nbins + 1) + scan_tmp_words(nbins + 1);
  const uint64_t have_words = (NOALLOC_SCRATCH_BYTES - words_off) / sizeof(uint32_t);
  if (need_words > have_words)
    throw InvalidArgument("the binning needs " + std::to_string(words_off + need_words * 4) +
                          " bytes of scratch; the no-allocation scratch holds " +
                          std::to_string(NOALLOC_SCRATCH_BYTES) + " bytes");
  uint32_t* counts = reinterpret_cast<uint32_t*>(base + words_off);
  uint32_t* cursor = counts + (nbins + 1);
  uint32_t* tmp = cursor + (nbins + 1);
  check_cuda(cudaMemsetAsync(counts, 0, (nbins + 1) * sizeof(uint32_t), s), "memset");
  k_bin_count<T><<<blocks_for(n, 256), 256, 0, s>>>(g, uvw, dfoc, act, 0, key, counts);
  check_cuda(cudaGetLastError(), "bin count");
  exclusive_scan_in(counts, counts, nbins + 1, tmp, s);
  check_cuda(cudaMemcpyAsync(cursor, counts, (nbins + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s), "copy");
  k_bin_scatter<<<blocks_for(n, 256), 256, 0, s>>>(n, key, cursor, sorted);
  check_cuda(cudaGetLastError(), "bin scatter");
  k_reference_key<<<blocks_for(n, 256), 256, 0, s>>>(n, (uint32_t)g.nsub, key);
  check_cuda(cudaGetLastError(), "keys");
  check_cuda(cudaStreamSynchronize(s), "binning");
  std::memcpy(info, pi.v, sizeof(pi.v));
}

}  // namespace
}  // namespace wg

extern "C" int32_t rang_b200_wgridder_bin_noalloc(const WgridderOptions* opts, size_t nrow, size_t nchan,
                                                  const double* uvw_dev, const double* freq, const void* wgt_dev,
                                                  int32_t wgt_kind, const uint8_t* mask_dev, int32_t single,
                                                  void* stream, uint32_t* key_dev, uint32_t* sorted_dev,
                                                  size_t* nsorted, double* info) {
  using namespace wg;
  std::string* err = last_error_slot();
  try {
    if (!opts) throw InvalidArgument("null options");
    if ((!uvw_dev && nrow) || !freq || !info || !nsorted || ((!key_dev || !sorted_dev) && nrow))
      throw InvalidArgument("null array");
    if (!((wgt_kind == WGT_NONE) || (wgt_dev && (wgt_kind == WGT_F32 || wgt_kind == WGT_F64))))
      throw InvalidArgument("invalid weight array or kind");
    Inputs act{nullptr, VIS_UNIT, wgt_dev, nullptr, wgt_kind, mask_dev};
    if (single)
      bin_noalloc<float>(*opts, nrow, nchan, uvw_dev, freq, act, (cudaStream_t)stream, key_dev, sorted_dev, nsorted,
                         info);
    else
      bin_noalloc<double>(*opts, nrow, nchan, uvw_dev, freq, act, (cudaStream_t)stream, key_dev, sorted_dev, nsorted,
                          info);
    return 0;
  } catch (const InvalidArgument& e) {
    *err = e.what();
    return 1;
  } catch (const std::exception& e) {
    *err = e.what();
    return 2;
  }
}
