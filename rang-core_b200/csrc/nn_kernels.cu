// Kernels of the learned FISTA proposal network: a 4-level U-Net on a
// residual patch and a PSF patch, trained and run on the GPU by these
// kernels alone (C ABI in include/rang_nn.h).
//
// Tensors are NHWC in bfloat16 with a pixel stride `ld` (elements between
// consecutive pixels, a multiple of 8 so that every 8-channel group is a
// 16-byte vector; a channel slice of a wider tensor is a pointer offset plus
// the wider stride, which is how the skip connections concatenate without a
// copy). Every sum is accumulated in float32; master weights, gradients of
// the weights and the optimiser state are float32.
//
// The 3x3 convolution runs on the fifth-generation tensor cores (tcgen05.mma
// with TMA operands and a TMEM accumulator, nn_conv_tc.cu) wherever the image
// tiles into 16 x 8 patches; otherwise, and on request
// (rang_b200_nn_set_conv_path), it is an implicit GEMM on the legacy tensor
// core path (mma.sync m16n8k16 bf16 -> f32): M = pixels (128 per block), N = output
// channels (32 or 64 per block), K = 9 taps x input channels in chunks of 32,
// with the A (pixel x channel, zero-filled outside the image) and B (weight)
// tiles staged in shared memory by cp.async in a 3-stage pipeline and read
// with ldmatrix. The gradient with respect to the input is the same
// convolution with the weights flipped and transposed; the gradient with
// respect to the weights is a second GEMM whose K dimension is the pixels,
// on tcgen05 (nn_conv_tc.cu) where the channel counts are multiples of 64 and
// otherwise the mma.sync kernel below.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "nn_conv_tc.h"
#include "rang_nn.h"

namespace {

using bf16 = __nv_bfloat16;
using bf162 = __nv_bfloat162;

constexpr int kSMs = 148;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// 16-byte global -> shared copy; `valid` false writes zeros and reads nothing.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(n));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void ldsm4(uint32_t (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm4t(uint32_t (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}

// c += a (16x16, row) * b (16x8, col), bf16 operands, f32 accumulators.
__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

unsigned grid_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > (int64_t)kSMs * 32) b = (int64_t)kSMs * 32;
  return (unsigned)b;
}

// ------------------------------------------------------------------ 3x3 convolution

struct ConvArgs {
  const bf16* in;
  const bf16* w;  // [Cout][9][Cin]
  const float* bias;
  bf16* out;
  const bf16* mask;
  int64_t P;  // batch * H * W
  int H, W, ld_in, ld_out, ld_mask, Cin, Cout, relu, accumulate;
};

constexpr int CONV_BM = 128;    // pixels per block
constexpr int CONV_KC = 32;     // input channels per K step
constexpr int CONV_ROW = 40;    // shared row stride (bf16): 80 bytes, conflict-free for ldmatrix
constexpr int CONV_STAGES = 3;

// out[p, co] = epilogue(bias[co] + sum_{tap, ci} w[co, tap, ci] in[p + off(tap), ci]),
// off(tap) = (tap / 3 - 1) rows + (tap % 3 - 1) columns, zero outside the image.
// The epilogue adds the old value (accumulate), applies ReLU (relu), and
// zeroes the result where mask <= 0 (mask).
template <int BN>
__global__ void __launch_bounds__(128) k_conv3(const ConvArgs a) {
  __shared__ __align__(128) bf16 sA[CONV_STAGES][CONV_BM * CONV_ROW];
  __shared__ __align__(128) bf16 sB[CONV_STAGES][BN * CONV_ROW];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int64_t m0 = (int64_t)blockIdx.x * CONV_BM;
  const int n0 = blockIdx.y * BN;
  const int64_t p = m0 + t;  // the pixel whose A row this thread stages
  const bool pin = p < a.P;
  const int x = pin ? (int)(p % a.W) : 0;
  const int y = pin ? (int)((p / a.W) % a.H) : 0;
  const int nc = a.Cin / CONV_KC;
  const int nk = 9 * nc;

  auto load = [&](int kk, int s) {
    const int tap = kk / nc, cc = kk - tap * nc;
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;
    const bool ok = pin && (unsigned)(y + dy) < (unsigned)a.H && (unsigned)(x + dx) < (unsigned)a.W;
    const bf16* src = ok ? a.in + (p + (int64_t)dy * a.W + dx) * a.ld_in + cc * CONV_KC : a.in;
    bf16* dst = &sA[s][t * CONV_ROW];
#pragma unroll
    for (int j = 0; j < 4; j++) cp_async16(dst + 8 * j, ok ? src + 8 * j : a.in, ok);
#pragma unroll
    for (int q = t; q < BN * 4; q += 128) {
      const int row = q >> 2, j = q & 3;
      const bf16* ws = a.w + ((int64_t)(n0 + row) * 9 + tap) * a.Cin + cc * CONV_KC + 8 * j;
      cp_async16(&sB[s][row * CONV_ROW + 8 * j], ws, true);
    }
  };

  float acc[2][BN / 8][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < BN / 8; j++)
#pragma unroll
      for (int e = 0; e < 4; e++) acc[i][j][e] = 0.0f;

#pragma unroll
  for (int s = 0; s < CONV_STAGES - 1; s++) {
    if (s < nk) load(s, s);
    cp_commit();
  }
  for (int kk = 0; kk < nk; kk++) {
    cp_wait<CONV_STAGES - 2>();
    __syncthreads();
    const int kn = kk + CONV_STAGES - 1;
    if (kn < nk) load(kn, kn % CONV_STAGES);
    cp_commit();
    const bf16* As = sA[kk % CONV_STAGES];
    const bf16* Bs = sB[kk % CONV_STAGES];
#pragma unroll
    for (int ks = 0; ks < 2; ks++) {
      uint32_t af[2][4];
#pragma unroll
      for (int mt = 0; mt < 2; mt++) {
        const int row = warp * 32 + mt * 16 + (lane & 7) + ((lane >> 3) & 1) * 8;
        const int col = ks * 16 + (lane >> 4) * 8;
        ldsm4(af[mt], As + row * CONV_ROW + col);
      }
#pragma unroll
      for (int np = 0; np < BN / 16; np++) {
        uint32_t b[4];
        const int row = np * 16 + (lane & 7) + (lane >> 4) * 8;
        const int col = ks * 16 + ((lane >> 3) & 1) * 8;
        ldsm4(b, Bs + row * CONV_ROW + col);
#pragma unroll
        for (int mt = 0; mt < 2; mt++) {
          mma_bf16(acc[mt][2 * np], af[mt], b[0], b[1]);
          mma_bf16(acc[mt][2 * np + 1], af[mt], b[2], b[3]);
        }
      }
    }
  }
  cp_wait<0>();

  const int g = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 2; mt++)
#pragma unroll
    for (int half = 0; half < 2; half++) {
      const int64_t pp = m0 + warp * 32 + mt * 16 + g + half * 8;
      if (pp >= a.P) continue;
#pragma unroll
      for (int nt = 0; nt < BN / 8; nt++) {
        const int co = n0 + nt * 8 + 2 * tq;
        float v0 = acc[mt][nt][2 * half], v1 = acc[mt][nt][2 * half + 1];
        if (a.bias) {
          v0 += a.bias[co];
          v1 += a.bias[co + 1];
        }
        bf162* o = reinterpret_cast<bf162*>(a.out + pp * a.ld_out + co);
        if (a.accumulate) {
          const float2 old = __bfloat1622float2(*o);
          v0 += old.x;
          v1 += old.y;
        }
        if (a.relu) {
          v0 = fmaxf(v0, 0.0f);
          v1 = fmaxf(v1, 0.0f);
        }
        if (a.mask) {
          const float2 m = __bfloat1622float2(*reinterpret_cast<const bf162*>(a.mask + pp * a.ld_mask + co));
          if (!(m.x > 0.0f)) v0 = 0.0f;
          if (!(m.y > 0.0f)) v1 = 0.0f;
        }
        *o = __floats2bfloat162_rn(v0, v1);
      }
    }
}

// ------------------------------------------------------------------ weight gradient

struct DwArgs {
  const bf16* in;  // forward input of the layer
  const bf16* dz;  // gradient at the layer's pre-activation output
  float* dw;       // [Cout][9][Cin], accumulated
  int64_t P, chunks_per_warp;
  int H, W, ld_in, ld_dz, Cin, Cout;
};

constexpr int DW_ROWS = 32;  // pixels per K chunk

template <int TM>
constexpr int dw_smem_bytes() {
  return 4 * 2 * DW_ROWS * ((TM + 8) + 40) * 2;
}

// dw[co, tap, ci] += sum_p dz[p, co] in[p + off(tap), ci] for one tap
// (blockIdx.z), a TM x 32 (co, ci) tile (blockIdx.y) and a pixel range
// (blockIdx.x): M = co, N = ci, K = pixels. Each warp runs its own
// double-buffered pixel chunks; the four warps' tiles are summed in shared
// memory and added to dw atomically.
template <int TM>
__global__ void __launch_bounds__(128) k_conv3_dw(const DwArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  constexpr int ZROW = TM + 8, IROW = 40;
  constexpr int WARP_ELEMS = 2 * DW_ROWS * (ZROW + IROW);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bf16* wz = reinterpret_cast<bf16*>(smem) + warp * WARP_ELEMS;
  bf16* wi = wz + 2 * DW_ROWS * ZROW;
  const int tap = blockIdx.z, dy = tap / 3 - 1, dx = tap % 3 - 1;
  const int ncb = a.Cin / 32;
  const int co0 = (blockIdx.y / ncb) * TM, ci0 = (blockIdx.y % ncb) * 32;
  const int64_t nchunks = (a.P + DW_ROWS - 1) / DW_ROWS;
  const int64_t c0 = ((int64_t)blockIdx.x * 4 + warp) * a.chunks_per_warp;
  int64_t c1 = c0 + a.chunks_per_warp;
  if (c1 > nchunks) c1 = nchunks;

  auto load = [&](int64_t c, int s) {
#pragma unroll
    for (int q = lane; q < DW_ROWS * (TM / 8); q += 32) {
      const int r = q / (TM / 8), j = q % (TM / 8);
      const int64_t p = c * DW_ROWS + r;
      const bool ok = p < a.P;
      cp_async16(wz + (s * DW_ROWS + r) * ZROW + 8 * j, ok ? a.dz + p * a.ld_dz + co0 + 8 * j : a.dz, ok);
    }
#pragma unroll
    for (int q = lane; q < DW_ROWS * 4; q += 32) {
      const int r = q >> 2, j = q & 3;
      const int64_t p = c * DW_ROWS + r;
      bool ok = false;
      const bf16* src = a.in;
      if (p < a.P) {
        const int x = (int)(p % a.W), y = (int)((p / a.W) % a.H);
        if ((unsigned)(y + dy) < (unsigned)a.H && (unsigned)(x + dx) < (unsigned)a.W) {
          ok = true;
          src = a.in + (p + (int64_t)dy * a.W + dx) * a.ld_in + ci0 + 8 * j;
        }
      }
      cp_async16(wi + (s * DW_ROWS + r) * IROW + 8 * j, src, ok);
    }
  };

  float acc[TM / 16][4][4];
#pragma unroll
  for (int i = 0; i < TM / 16; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int e = 0; e < 4; e++) acc[i][j][e] = 0.0f;

  const int i8 = lane >> 3, r8 = lane & 7;
  if (c0 < c1) load(c0, 0);
  cp_commit();
  for (int64_t c = c0; c < c1; c++) {
    const int s = (int)((c - c0) & 1);
    if (c + 1 < c1) load(c + 1, s ^ 1);
    cp_commit();
    cp_wait<1>();
    __syncwarp();
    const bf16* Z = wz + s * DW_ROWS * ZROW;
    const bf16* I = wi + s * DW_ROWS * IROW;
#pragma unroll
    for (int ks = 0; ks < 2; ks++) {
      uint32_t bfr[2][4];
#pragma unroll
      for (int np = 0; np < 2; np++) {
        const int krow = ks * 16 + r8 + (i8 & 1) * 8;
        const int ncol = np * 16 + (i8 >> 1) * 8;
        ldsm4t(bfr[np], I + krow * IROW + ncol);
      }
#pragma unroll
      for (int mt = 0; mt < TM / 16; mt++) {
        uint32_t af[4];
        const int krow = ks * 16 + r8 + (i8 >> 1) * 8;
        const int mcol = mt * 16 + (i8 & 1) * 8;
        ldsm4t(af, Z + krow * ZROW + mcol);
#pragma unroll
        for (int np = 0; np < 2; np++) {
          mma_bf16(acc[mt][2 * np], af, bfr[np][0], bfr[np][1]);
          mma_bf16(acc[mt][2 * np + 1], af, bfr[np][2], bfr[np][3]);
        }
      }
    }
    __syncwarp();
  }
  cp_wait<0>();
  __syncthreads();

  float* red = reinterpret_cast<float*>(smem);  // [4][TM][32]
  const int g = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int mt = 0; mt < TM / 16; mt++)
#pragma unroll
    for (int nt = 0; nt < 4; nt++)
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int m = mt * 16 + g + (e >> 1) * 8, n = nt * 8 + 2 * tq + (e & 1);
        red[(warp * TM + m) * 32 + n] = acc[mt][nt][e];
      }
  __syncthreads();
  for (int i = threadIdx.x; i < TM * 32; i += 128) {
    const float s = red[i] + red[TM * 32 + i] + red[2 * TM * 32 + i] + red[3 * TM * 32 + i];
    const int m = i >> 5, n = i & 31;
    atomicAdd(&a.dw[((int64_t)(co0 + m) * 9 + tap) * a.Cin + ci0 + n], s);
  }
}

// dbias[c] += sum_p dz[p, c]: threads take channel pairs, blocks take pixel ranges.
__global__ void k_bias_grad(const bf16* __restrict__ dz, int ld, int64_t P, int C, float* __restrict__ db,
                            int64_t rows_per_block) {
  __shared__ float red[256][2];
  const int pairs = C / 2, lanes = 256 / pairs;
  const int t = threadIdx.x, c2 = t % pairs, r = t / pairs;
  float s0 = 0.0f, s1 = 0.0f;
  if (r < lanes) {
    const int64_t p0 = (int64_t)blockIdx.x * rows_per_block;
    int64_t p1 = p0 + rows_per_block;
    if (p1 > P) p1 = P;
    for (int64_t p = p0 + r; p < p1; p += lanes) {
      const float2 v = __bfloat1622float2(*reinterpret_cast<const bf162*>(dz + p * ld + 2 * c2));
      s0 += v.x;
      s1 += v.y;
    }
  }
  red[t][0] = s0;
  red[t][1] = s1;
  __syncthreads();
  if (r == 0) {
    for (int k = 1; k < lanes; k++) {
      s0 += red[k * pairs + c2][0];
      s1 += red[k * pairs + c2][1];
    }
    atomicAdd(&db[2 * c2], s0);
    atomicAdd(&db[2 * c2 + 1], s1);
  }
}

// wt[ci][tap][co] = w[co][8 - tap][ci]: the weights of the input-gradient convolution.
__global__ void k_flip(const bf16* __restrict__ w, bf16* __restrict__ wt, int Cin, int Cout) {
  const int64_t n = (int64_t)Cin * 9 * Cout;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int co = (int)(i % Cout);
    const int tap = (int)((i / Cout) % 9);
    const int ci = (int)(i / ((int64_t)Cout * 9));
    wt[i] = w[((int64_t)co * 9 + (8 - tap)) * Cin + ci];
  }
}

// ------------------------------------------------------------------ pooling, upsampling

union V8 {
  uint4 u;
  bf162 h[4];
};

// out[b, y, x, c] = mean of in[b, 2y + i, 2x + j, c] (H, W the input size).
__global__ void k_pool(const bf16* __restrict__ in, int ld_in, bf16* __restrict__ out, int ld_out, int64_t B, int H,
                       int W, int C) {
  const int h = H / 2, w = W / 2, c8 = C / 8;
  const int64_t n = B * h * w * c8;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % c8) * 8;
    const int64_t q = i / c8;
    const int x = (int)(q % w), y = (int)((q / w) % h);
    const int64_t b = q / ((int64_t)w * h);
    const int64_t p = (b * H + 2 * y) * W + 2 * x;
    V8 v[4], o;
    v[0].u = *reinterpret_cast<const uint4*>(in + p * ld_in + c);
    v[1].u = *reinterpret_cast<const uint4*>(in + (p + 1) * ld_in + c);
    v[2].u = *reinterpret_cast<const uint4*>(in + (p + W) * ld_in + c);
    v[3].u = *reinterpret_cast<const uint4*>(in + (p + W + 1) * ld_in + c);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const float2 s0 = __bfloat1622float2(v[0].h[k]), s1 = __bfloat1622float2(v[1].h[k]);
      const float2 s2 = __bfloat1622float2(v[2].h[k]), s3 = __bfloat1622float2(v[3].h[k]);
      o.h[k] = __floats2bfloat162_rn(0.25f * (((s0.x + s1.x) + s2.x) + s3.x), 0.25f * (((s0.y + s1.y) + s2.y) + s3.y));
    }
    *reinterpret_cast<uint4*>(out + q * ld_out + c) = o.u;
  }
}

// g[p, c] = (g[p, c] + dpool[p / 2, c] / 4) * (act[p, c] > 0), in place: the
// gradient of an encoder output that feeds both the skip connection (g holds
// that part) and the pooling.
__global__ void k_pool_backward(bf16* __restrict__ g, int ld_g, const bf16* __restrict__ dpool, int ld_dp,
                                const bf16* __restrict__ act, int ld_act, int64_t B, int H, int W, int C) {
  const int c8 = C / 8, h = H / 2, w = W / 2;
  const int64_t n = B * H * W * c8;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % c8) * 8;
    const int64_t p = i / c8;
    const int x = (int)(p % W), y = (int)((p / W) % H);
    const int64_t b = p / ((int64_t)W * H);
    const int64_t q = (b * h + y / 2) * w + x / 2;
    V8 gv, dv, av;
    gv.u = *reinterpret_cast<const uint4*>(g + p * ld_g + c);
    dv.u = *reinterpret_cast<const uint4*>(dpool + q * ld_dp + c);
    av.u = *reinterpret_cast<const uint4*>(act + p * ld_act + c);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const float2 s = __bfloat1622float2(gv.h[k]), d = __bfloat1622float2(dv.h[k]), m = __bfloat1622float2(av.h[k]);
      const float v0 = m.x > 0.0f ? s.x + 0.25f * d.x : 0.0f;
      const float v1 = m.y > 0.0f ? s.y + 0.25f * d.y : 0.0f;
      gv.h[k] = __floats2bfloat162_rn(v0, v1);
    }
    *reinterpret_cast<uint4*>(g + p * ld_g + c) = gv.u;
  }
}

// out[b, y, x, c] = in[b, y / 2, x / 2, c] (H, W the output size).
__global__ void k_upsample(const bf16* __restrict__ in, int ld_in, bf16* __restrict__ out, int ld_out, int64_t B,
                           int H, int W, int C) {
  const int c8 = C / 8, h = H / 2, w = W / 2;
  const int64_t n = B * H * W * c8;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % c8) * 8;
    const int64_t p = i / c8;
    const int x = (int)(p % W), y = (int)((p / W) % H);
    const int64_t b = p / ((int64_t)W * H);
    const int64_t q = (b * h + y / 2) * w + x / 2;
    *reinterpret_cast<uint4*>(out + p * ld_out + c) = *reinterpret_cast<const uint4*>(in + q * ld_in + c);
  }
}

// out[b, y, x, c] = sum of g[b, 2y + i, 2x + j, c] (H, W the output size).
__global__ void k_upsample_backward(const bf16* __restrict__ g, int ld_g, bf16* __restrict__ out, int ld_out,
                                    int64_t B, int H, int W, int C) {
  const int c8 = C / 8, W2 = 2 * W;
  const int64_t n = B * H * W * c8;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % c8) * 8;
    const int64_t q = i / c8;
    const int x = (int)(q % W), y = (int)((q / W) % H);
    const int64_t b = q / ((int64_t)W * H);
    const int64_t p = (b * 2 * H + 2 * y) * W2 + 2 * x;
    V8 v[4], o;
    v[0].u = *reinterpret_cast<const uint4*>(g + p * ld_g + c);
    v[1].u = *reinterpret_cast<const uint4*>(g + (p + 1) * ld_g + c);
    v[2].u = *reinterpret_cast<const uint4*>(g + (p + W2) * ld_g + c);
    v[3].u = *reinterpret_cast<const uint4*>(g + (p + W2 + 1) * ld_g + c);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const float2 s0 = __bfloat1622float2(v[0].h[k]), s1 = __bfloat1622float2(v[1].h[k]);
      const float2 s2 = __bfloat1622float2(v[2].h[k]), s3 = __bfloat1622float2(v[3].h[k]);
      o.h[k] = __floats2bfloat162_rn(((s0.x + s1.x) + s2.x) + s3.x, ((s0.y + s1.y) + s2.y) + s3.y);
    }
    *reinterpret_cast<uint4*>(out + q * ld_out + c) = o.u;
  }
}

// ------------------------------------------------------------------ input, head, loss

// x[b, y, x, :] = (resid[offs[b] + y * ld_r + x] * s_r, psf[y * ld_p + x] * s_p, 0, ..., 0)
// as 32 channels (the network input, padded to the convolution's channel step).
__global__ void k_pack(const float* __restrict__ resid, const int64_t* __restrict__ offs, int64_t ld_r,
                       const float* __restrict__ psf, int64_t ld_p, float s_r, float s_p, bf16* __restrict__ x,
                       int64_t B, int H, int W) {
  const int64_t n = B * H * W;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int xx = (int)(i % W), yy = (int)((i / W) % H);
    const int64_t b = i / ((int64_t)W * H);
    V8 v;
    v.u = make_uint4(0, 0, 0, 0);
    v.h[0] = __floats2bfloat162_rn(resid[offs[b] + yy * ld_r + xx] * s_r, psf[yy * ld_p + xx] * s_p);
    uint4* dst = reinterpret_cast<uint4*>(x + i * 32);
    dst[0] = v.u;
    const uint4 z = make_uint4(0, 0, 0, 0);
    dst[1] = z;
    dst[2] = z;
    dst[3] = z;
  }
}

// out[b, y, x] (float) = bias + sum_{c < 32} w[c] act[p, c].
__global__ void k_head(const bf16* __restrict__ act, int ld, const float* __restrict__ w, const float* __restrict__ bias,
                       float* __restrict__ out, int64_t P) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P; p += (int64_t)gridDim.x * blockDim.x) {
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      V8 v;
      v.u = *reinterpret_cast<const uint4*>(act + p * ld + 8 * k);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const float2 f = __bfloat1622float2(v.h[j]);
        s += w[8 * k + 2 * j] * f.x;
        s += w[8 * k + 2 * j + 1] * f.y;
      }
    }
    out[p] = bias[0] + s;
  }
}

// The head's backward: dact[p, c] = dout[p] w[c] (act > 0), dw[c] += sum_p
// dout[p] act[p, c], dbias += sum_p dout[p].
__global__ void __launch_bounds__(256) k_head_backward(const bf16* __restrict__ act, int ld, const float* __restrict__ w,
                                                       const float* __restrict__ dout, bf16* __restrict__ dact,
                                                       int ld_d, float* __restrict__ dw, float* __restrict__ dbias,
                                                       int64_t P) {
  __shared__ float red[8][33];
  float part[33];
#pragma unroll
  for (int c = 0; c < 33; c++) part[c] = 0.0f;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P; p += (int64_t)gridDim.x * blockDim.x) {
    const float d = dout[p];
    part[32] += d;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      V8 v, o;
      v.u = *reinterpret_cast<const uint4*>(act + p * ld + 8 * k);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const float2 f = __bfloat1622float2(v.h[j]);
        const int c = 8 * k + 2 * j;
        part[c] += d * f.x;
        part[c + 1] += d * f.y;
        o.h[j] = __floats2bfloat162_rn(f.x > 0.0f ? d * w[c] : 0.0f, f.y > 0.0f ? d * w[c + 1] : 0.0f);
      }
      *reinterpret_cast<uint4*>(dact + p * ld_d + 8 * k) = o.u;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 33; c++) {
    float s = part[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp][c] = s;
  }
  __syncthreads();
  if (threadIdx.x < 33) {
    float s = 0.0f;
    for (int k = 0; k < 8; k++) s += red[k][threadIdx.x];
    atomicAdd(threadIdx.x < 32 ? &dw[threadIdx.x] : dbias, s);
  }
}

// loss += sum (pred - target)^2 / n; grad = 2 (pred - target) / n, with the
// target of sample b at target[offs[b] + y * ld + x].
__global__ void k_mse(const float* __restrict__ pred, const float* __restrict__ target, const int64_t* __restrict__ offs,
                      int64_t ld, float* __restrict__ grad, float* __restrict__ loss, int64_t B, int H, int W) {
  const int64_t n = B * H * W;
  const float inv = 1.0f / (float)n;
  float part = 0.0f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int xx = (int)(i % W), yy = (int)((i / W) % H);
    const int64_t b = i / ((int64_t)W * H);
    const float d = pred[i] - target[offs[b] + yy * ld + xx];
    grad[i] = 2.0f * d * inv;
    part += d * d * inv;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, part);
}

// dst[offs[b] + y * ld + x] = out[b, y, x] * scale for rows [win[4b], win[4b+1])
// and columns [win[4b+2], win[4b+3]) of each patch.
__global__ void k_unpack(const float* __restrict__ out, const int64_t* __restrict__ offs, const int32_t* __restrict__ win,
                         int64_t ld, float scale, float* __restrict__ dst, int64_t B, int H, int W) {
  const int64_t n = B * H * W;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int xx = (int)(i % W), yy = (int)((i / W) % H);
    const int64_t b = i / ((int64_t)W * H);
    if (yy >= win[4 * b] && yy < win[4 * b + 1] && xx >= win[4 * b + 2] && xx < win[4 * b + 3])
      dst[offs[b] + yy * ld + xx] = out[i] * scale;
  }
}

// One Adam step on float master weights p (bias-corrected moments), writing
// their bfloat16 copy where `pb` is given, then clearing the gradient.
__global__ void k_adam(float* __restrict__ p, bf16* __restrict__ pb, float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * (gi * gi);
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (pb) pb[i] = __float2bfloat16_rn(pi);
    g[i] = 0.0f;
  }
}

__global__ void k_to_bf16(const float* __restrict__ src, bf16* __restrict__ dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = __float2bfloat16_rn(src[i]);
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }
bool aligned4(const void* p) { return ((uintptr_t)p & 3u) == 0; }

int32_t launched() { return cudaGetLastError() == cudaSuccess ? 0 : 2; }

// Which kernel rang_b200_nn_conv3 runs: 0 the tcgen05 / TMA kernel where the
// shapes allow it, else the mma.sync kernel; 1 always the mma.sync kernel.
std::atomic<int> g_conv_path{0};

}  // namespace

extern "C" {

int32_t rang_b200_nn_conv3(const void* in, int64_t ld_in, const void* w, const float* bias, void* out, int64_t ld_out,
                           const void* mask, int64_t ld_mask, int64_t batch, int32_t height, int32_t width,
                           int32_t cin, int32_t cout, int32_t relu, int32_t accumulate, void* stream) {
  if (!in || !w || !out || batch <= 0 || height <= 0 || width <= 0 || cin <= 0 || cout <= 0) return 1;
  if (cin % 32 || cout % 32 || ld_in < cin || ld_out < cout || ld_in % 8 || ld_out % 8) return 1;
  if (!aligned16(in) || !aligned16(w) || !aligned4(out) || (mask && (ld_mask % 8 || !aligned4(mask)))) return 1;
  if (ld_in > INT32_MAX || ld_out > INT32_MAX || ld_mask > INT32_MAX) return 1;
  if (g_conv_path.load() == 0) {
    const TcConvArgs t{(const bf16*)in, (const bf16*)w, bias, (bf16*)out, (const bf16*)mask, batch, height, width,
                       (int)ld_in, (int)ld_out, (int)ld_mask, cin, cout, relu, accumulate};
    if (conv3_tc_supported(t)) return conv3_tc(t, (cudaStream_t)stream);
  }
  ConvArgs a{(const bf16*)in, (const bf16*)w, bias, (bf16*)out, (const bf16*)mask,
             batch * height * width, height, width, (int)ld_in, (int)ld_out, (int)ld_mask, cin, cout, relu, accumulate};
  const unsigned gx = (unsigned)((a.P + CONV_BM - 1) / CONV_BM);
  if (cout % 64 == 0)
    k_conv3<64><<<dim3(gx, cout / 64), 128, 0, (cudaStream_t)stream>>>(a);
  else
    k_conv3<32><<<dim3(gx, cout / 32), 128, 0, (cudaStream_t)stream>>>(a);
  return launched();
}

int32_t rang_b200_nn_conv3_weight_grad(const void* in, int64_t ld_in, const void* dz, int64_t ld_dz, float* dw,
                                       float* dbias, int64_t batch, int32_t height, int32_t width, int32_t cin,
                                       int32_t cout, void* stream) {
  if (!in || !dz || !dw || batch <= 0 || height <= 0 || width <= 0 || cin <= 0 || cout <= 0) return 1;
  if (cin % 32 || cout % 32 || ld_in < cin || ld_dz < cout || ld_in % 8 || ld_dz % 8 || cout > 512) return 1;
  if (!aligned16(in) || !aligned16(dz) || ld_in > INT32_MAX || ld_dz > INT32_MAX) return 1;
  if (g_conv_path.load() == 0) {
    const TcDwArgs t{(const bf16*)in, (const bf16*)dz, dw, batch, 0, 0, height, width, (int)ld_in, (int)ld_dz,
                     cin, cout};
    if (conv3_dw_tc_supported(t)) {
      const int st = conv3_dw_tc(t, (cudaStream_t)stream);
      if (st != 0) return st;
      if (dbias) {
        const int64_t rows = 4096, P = batch * height * width;
        k_bias_grad<<<(unsigned)((P + rows - 1) / rows), 256, 0, (cudaStream_t)stream>>>((const bf16*)dz,
                                                                                        (int)ld_dz, P, cout, dbias,
                                                                                        rows);
      }
      return launched();
    }
  }
  // per call: the attribute belongs to the current device's context
  cudaFuncSetAttribute(k_conv3_dw<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, dw_smem_bytes<64>());
  cudaFuncSetAttribute(k_conv3_dw<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, dw_smem_bytes<32>());
  DwArgs a{(const bf16*)in, (const bf16*)dz, dw, batch * height * width, 0, height, width, (int)ld_in, (int)ld_dz,
           cin, cout};
  const int tm = cout % 64 == 0 ? 64 : 32;
  const int tiles = (cout / tm) * (cin / 32);
  const int64_t nchunks = (a.P + DW_ROWS - 1) / DW_ROWS;
  int64_t splits = (4 * kSMs + tiles * 9 - 1) / (tiles * 9);
  const int64_t max_splits = (nchunks + 4 * 8 - 1) / (4 * 8);  // at least 8 chunks per warp
  if (splits > max_splits) splits = max_splits;
  if (splits < 1) splits = 1;
  a.chunks_per_warp = (nchunks + 4 * splits - 1) / (4 * splits);
  const dim3 grid((unsigned)splits, tiles, 9);
  if (tm == 64)
    k_conv3_dw<64><<<grid, 128, dw_smem_bytes<64>(), (cudaStream_t)stream>>>(a);
  else
    k_conv3_dw<32><<<grid, 128, dw_smem_bytes<32>(), (cudaStream_t)stream>>>(a);
  if (dbias) {
    const int64_t rows = 4096;
    k_bias_grad<<<(unsigned)((a.P + rows - 1) / rows), 256, 0, (cudaStream_t)stream>>>((const bf16*)dz, (int)ld_dz,
                                                                                       a.P, cout, dbias, rows);
  }
  return launched();
}

int32_t rang_b200_nn_set_conv_path(int32_t path) { return g_conv_path.exchange(path == 1 ? 1 : 0); }

int32_t rang_b200_nn_wait_probe(int64_t limit_ns, void* stream) {
  if (limit_ns < 0 || limit_ns > 10000000000ll) return 1;
  return conv3_tc_wait_probe((unsigned long long)limit_ns, (cudaStream_t)stream);
}

int32_t rang_b200_nn_device_status(void* stream) { return conv3_tc_status((cudaStream_t)stream); }

int32_t rang_b200_nn_conv3_flip(const void* w, void* wt, int32_t cin, int32_t cout, void* stream) {
  if (!w || !wt || cin <= 0 || cout <= 0) return 1;
  k_flip<<<grid_for((int64_t)cin * 9 * cout), 256, 0, (cudaStream_t)stream>>>((const bf16*)w, (bf16*)wt, cin, cout);
  return launched();
}

int32_t rang_b200_nn_pool(const void* in, int64_t ld_in, void* out, int64_t ld_out, int64_t batch, int32_t height,
                          int32_t width, int32_t channels, void* stream) {
  if (!in || !out || batch <= 0 || height <= 0 || width <= 0 || height % 2 || width % 2 || channels % 8) return 1;
  if (ld_in % 8 || ld_out % 8 || !aligned16(in) || !aligned16(out)) return 1;
  k_pool<<<grid_for(batch * (height / 2) * (width / 2) * (channels / 8)), 256, 0, (cudaStream_t)stream>>>(
      (const bf16*)in, (int)ld_in, (bf16*)out, (int)ld_out, batch, height, width, channels);
  return launched();
}

int32_t rang_b200_nn_pool_backward(void* grad, int64_t ld_grad, const void* dpool, int64_t ld_dpool, const void* act,
                                   int64_t ld_act, int64_t batch, int32_t height, int32_t width, int32_t channels,
                                   void* stream) {
  if (!grad || !dpool || !act || batch <= 0 || height <= 0 || width <= 0 || height % 2 || width % 2 || channels % 8)
    return 1;
  if (ld_grad % 8 || ld_dpool % 8 || ld_act % 8 || !aligned16(grad) || !aligned16(dpool) || !aligned16(act)) return 1;
  k_pool_backward<<<grid_for(batch * height * width * (channels / 8)), 256, 0, (cudaStream_t)stream>>>(
      (bf16*)grad, (int)ld_grad, (const bf16*)dpool, (int)ld_dpool, (const bf16*)act, (int)ld_act, batch, height, width,
      channels);
  return launched();
}

int32_t rang_b200_nn_upsample(const void* in, int64_t ld_in, void* out, int64_t ld_out, int64_t batch, int32_t height,
                              int32_t width, int32_t channels, void* stream) {
  if (!in || !out || batch <= 0 || height <= 0 || width <= 0 || height % 2 || width % 2 || channels % 8) return 1;
  if (ld_in % 8 || ld_out % 8 || !aligned16(in) || !aligned16(out)) return 1;
  k_upsample<<<grid_for(batch * height * width * (channels / 8)), 256, 0, (cudaStream_t)stream>>>(
      (const bf16*)in, (int)ld_in, (bf16*)out, (int)ld_out, batch, height, width, channels);
  return launched();
}

int32_t rang_b200_nn_upsample_backward(const void* grad, int64_t ld_grad, void* out, int64_t ld_out, int64_t batch,
                                       int32_t height, int32_t width, int32_t channels, void* stream) {
  if (!grad || !out || batch <= 0 || height <= 0 || width <= 0 || channels % 8) return 1;
  if (ld_grad % 8 || ld_out % 8 || !aligned16(grad) || !aligned16(out)) return 1;
  k_upsample_backward<<<grid_for(batch * height * width * (channels / 8)), 256, 0, (cudaStream_t)stream>>>(
      (const bf16*)grad, (int)ld_grad, (bf16*)out, (int)ld_out, batch, height, width, channels);
  return launched();
}

int32_t rang_b200_nn_pack(const float* resid, const int64_t* offsets, int64_t ld_resid, const float* psf,
                          int64_t ld_psf, float scale_resid, float scale_psf, void* x, int64_t batch, int32_t height,
                          int32_t width, void* stream) {
  if (!resid || !offsets || !psf || !x || batch <= 0 || height <= 0 || width <= 0 || !aligned16(x)) return 1;
  k_pack<<<grid_for(batch * height * width), 256, 0, (cudaStream_t)stream>>>(
      resid, offsets, ld_resid, psf, ld_psf, scale_resid, scale_psf, (bf16*)x, batch, height, width);
  return launched();
}

int32_t rang_b200_nn_head(const void* act, int64_t ld, const float* w, const float* bias, float* out, int64_t pixels,
                          void* stream) {
  if (!act || !w || !bias || !out || pixels <= 0 || ld % 8 || !aligned16(act)) return 1;
  k_head<<<grid_for(pixels), 256, 0, (cudaStream_t)stream>>>((const bf16*)act, (int)ld, w, bias, out, pixels);
  return launched();
}

int32_t rang_b200_nn_head_backward(const void* act, int64_t ld, const float* w, const float* dout, void* dact,
                                   int64_t ld_dact, float* dw, float* dbias, int64_t pixels, void* stream) {
  if (!act || !w || !dout || !dact || !dw || !dbias || pixels <= 0 || ld % 8 || ld_dact % 8) return 1;
  if (!aligned16(act) || !aligned16(dact)) return 1;
  k_head_backward<<<grid_for(pixels), 256, 0, (cudaStream_t)stream>>>((const bf16*)act, (int)ld, w, dout, (bf16*)dact,
                                                                      (int)ld_dact, dw, dbias, pixels);
  return launched();
}

int32_t rang_b200_nn_mse(const float* pred, const float* target, const int64_t* offsets, int64_t ld_target,
                         float* grad, float* loss, int64_t batch, int32_t height, int32_t width, void* stream) {
  if (!pred || !target || !offsets || !grad || !loss || batch <= 0 || height <= 0 || width <= 0) return 1;
  k_mse<<<grid_for(batch * height * width), 256, 0, (cudaStream_t)stream>>>(pred, target, offsets, ld_target, grad,
                                                                            loss, batch, height, width);
  return launched();
}

int32_t rang_b200_nn_unpack(const float* out, const int64_t* offsets, const int32_t* windows, int64_t ld, float scale,
                            float* dst, int64_t batch, int32_t height, int32_t width, void* stream) {
  if (!out || !offsets || !windows || !dst || batch <= 0 || height <= 0 || width <= 0) return 1;
  k_unpack<<<grid_for(batch * height * width), 256, 0, (cudaStream_t)stream>>>(out, offsets, windows, ld, scale, dst,
                                                                               batch, height, width);
  return launched();
}

int32_t rang_b200_nn_adam(float* p, void* pb, float* g, float* m, float* v, int64_t n, float lr, float beta1,
                          float beta2, float eps, int32_t step, void* stream) {
  if (!p || !g || !m || !v || n <= 0 || step < 1) return 1;
  const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  k_adam<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(p, (bf16*)pb, g, m, v, n, lr, beta1, beta2, eps, c1, c2);
  return launched();
}

int32_t rang_b200_nn_to_bf16(const float* src, void* dst, int64_t n, void* stream) {
  if (!src || !dst || n <= 0) return 1;
  k_to_bf16<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(src, (bf16*)dst, n);
  return launched();
}

}  // extern "C"
