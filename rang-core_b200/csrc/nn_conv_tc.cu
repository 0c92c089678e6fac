// The 3x3 convolution of the proposal network on the fifth-generation tensor
// cores: an implicit GEMM with M = 128 pixels (an 8 x 16 patch of one image),
// N = 32, 64 or 128 output channels and K = 9 taps x input channels, the
// accumulator in tensor memory (TMEM), operands in shared memory, fetched by
// the tensor memory accelerator (TMA).
//
// Per K block (one tap, KC = 64 or 32 input channels) the A tile is one 4-D
// TMA box of the NHWC input, (KC channels, 16 columns, 8 rows, 1 image) at the
// patch origin shifted by the tap: the box's rows (pixels) land in shared
// memory as consecutive KC x 2-byte rows in the 128- or 64-byte swizzled
// K-major layout that tcgen05.mma reads, and the pixels outside the image
// come back as zeros (the convolution's zero padding, with no bounds code).
// The B tile is one 2-D box of the weights w[co][tap][ci] (K-major rows of
// 9 x Cin), (KC, N) at (tap * Cin + ci0, co0).
//
// One thread issues the TMA loads into a 4-stage ring, one thread issues
// tcgen05.mma (kind::f16, bf16 inputs, f32 accumulation; KC / 16 MMAs per K
// block) and commits each stage back to the loader; after the last block the
// four warps read the 128 x N accumulator out of TMEM (warp w owns lanes
// 32w .. 32w + 31, one pixel per thread) and apply the epilogue of the
// mma.sync kernel: bias, accumulate, ReLU, mask, bf16.
//
// The weight gradient (k_conv3_dw_tc, further down) is the same machinery with
// K = pixels and both operands read channel-contiguous (MN-major).
//
// Every wait on an mbarrier gives up after about two seconds of device time;
// the block then records the failure in a device flag
// (rang_b200_nn_device_status) and returns after its own copies have landed
// (again with a limit) and its TMEM is freed.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "nn_conv_tc.h"

namespace {

using bf16 = __nv_bfloat16;

constexpr int TC_TW = 16, TC_TH = 8, TC_M = TC_TW * TC_TH;  // pixels per tile
constexpr int TC_STAGES = 4;
constexpr unsigned long long WAIT_NS = 2000000000ull;  // a wait gives up after this long

__device__ int g_conv_tc_error = 0;

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}
// True once the phase of this parity has completed; false after limit_ns.
__device__ __forceinline__ bool mbar_wait_for(uint64_t* bar, uint32_t parity, unsigned long long limit_ns) {
  const uint32_t a = saddr(bar);
  unsigned long long t0 = 0;
  for (uint32_t i = 0;; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((i & 255u) == 0) {
      const unsigned long long t = now_ns();
      if (i == 0)
        t0 = t;
      else if (t - t0 > limit_ns)
        return false;
    }
  }
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) { return mbar_wait_for(bar, parity, WAIT_NS); }

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
      "[%2];" ::"r"(saddr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(saddr(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
      : "memory");
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          saddr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(saddr(bar)), "r"(c0), "r"(c1)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major operand whose rows are
// `row_bytes` (64 or 128) long and swizzled over that span: 8-row groups are
// 8 x row_bytes apart (stride byte offset); the leading byte offset is unused
// by swizzled K-major layouts; descriptor version 1; layout type 2 (128-byte
// swizzle) or 4 (64-byte swizzle). Addresses are in 16-byte units.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t row_bytes) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(((8u * row_bytes) >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)(row_bytes == 128 ? 2 : 4) << 61;
  return d;
}
// Instruction descriptor: f32 accumulator, bf16 A and B, both K-major, M = 128, N.
__host__ __device__ constexpr uint32_t instr_desc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive f32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

template <int KC, int BN>
struct TcConvLayout {
  static constexpr int A_BYTES = TC_M * KC * 2;
  static constexpr int B_BYTES = BN * KC * 2;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  // stages, then full[STAGES], empty[STAGES], done, the TMEM address and the
  // failure flag; 1024 bytes of slack align the stages for the 128-byte swizzle
  static constexpr int BYTES = TC_STAGES * STAGE + (2 * TC_STAGES + 1) * 8 + 8 + 1024;
};

template <int KC, int BN>
__global__ void __launch_bounds__(128, 1)
    k_conv3_tc(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tw, const TcConvArgs a) {
  using L = TcConvLayout<KC, BN>;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + TC_STAGES * L::STAGE);
  uint64_t* empty = full + TC_STAGES;
  uint64_t* done = empty + TC_STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* bad = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tiles_x = a.W / TC_TW, tiles_y = a.H / TC_TH;
  int t = blockIdx.x;
  const int tx = t % tiles_x;
  t /= tiles_x;
  const int ty = t % tiles_y;
  const int img = t / tiles_y;
  const int x0 = tx * TC_TW, y0 = ty * TC_TH, n0 = blockIdx.y * BN;
  const int nc = a.Cin / KC, nk = 9 * nc;

  if (threadIdx.x == 0) {
    for (int s = 0; s < TC_STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *bad = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {  // BN columns of TMEM: the 128 x BN f32 accumulator
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tmem_slot)),
                 "r"((uint32_t)BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {  // loader
    int issued = 0;
    for (int kb = 0; kb < nk; kb++) {
      const int s = kb % TC_STAGES;
      if (kb >= TC_STAGES && !mbar_wait(&empty[s], ((kb / TC_STAGES) - 1) & 1)) {
        *bad = 1;
        break;
      }
      const int tap = kb / nc, cb = kb - tap * nc;
      unsigned char* st = smem + s * L::STAGE;
      mbar_expect_tx(&full[s], (uint32_t)L::STAGE);
      tma_load_4d(st, &tin, &full[s], cb * KC, x0 + tap % 3 - 1, y0 + tap / 3 - 1, img);
      tma_load_2d(st + L::A_BYTES, &tw, &full[s], tap * a.Cin + cb * KC, n0);
      issued = kb + 1;
    }
    // the last loads of every stage have landed before the block can leave
    for (int kb = issued > TC_STAGES ? issued - TC_STAGES : 0; kb < issued; kb++)
      if (!mbar_wait(&full[kb % TC_STAGES], (kb / TC_STAGES) & 1)) *bad = 1;
  } else if (warp == 1 && lane == 0) {  // MMA issuer
    const uint32_t idesc = instr_desc(BN);
    for (int kb = 0; kb < nk; kb++) {
      const int s = kb % TC_STAGES;
      if (!mbar_wait(&full[s], (kb / TC_STAGES) & 1)) {
        *bad = 1;
        break;
      }
      tc_fence_after();
      const uint32_t sa = saddr(smem + s * L::STAGE), sb = sa + L::A_BYTES;
#pragma unroll
      for (int k = 0; k < KC / 16; k++)
        umma(tmem, smem_desc(sa + 32u * k, KC * 2), smem_desc(sb + 32u * k, KC * 2), idesc, (kb | k) != 0);
      umma_commit(&empty[s]);
    }
    umma_commit(done);  // arrives once every MMA issued above has completed
  }
  __syncwarp();
  const bool ok = mbar_wait(done, 0);
  tc_fence_after();

  // Epilogue: thread (warp, lane) owns TMEM lane r = 32 warp + lane, pixel r of the patch.
  const int r = warp * 32 + lane;
  const int64_t p = ((int64_t)img * a.H + y0 + r / TC_TW) * a.W + x0 + r % TC_TW;
  bf16* orow = a.out + p * a.ld_out + n0;
  const bf16* mrow = a.mask ? a.mask + p * a.ld_mask + n0 : nullptr;
#pragma unroll 1
  for (int c = 0; c < BN; c += 16) {
    float v[16];
    tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
    if (!ok) continue;
    if (a.bias) {
#pragma unroll
      for (int i = 0; i < 16; i++) v[i] += a.bias[n0 + c + i];
    }
    uint4* o = reinterpret_cast<uint4*>(orow + c);
    if (a.accumulate) {
      const uint4 old[2] = {o[0], o[1]};
      const bf16* ob = reinterpret_cast<const bf16*>(old);
#pragma unroll
      for (int i = 0; i < 16; i++) v[i] += __bfloat162float(ob[i]);
    }
    if (a.relu) {
#pragma unroll
      for (int i = 0; i < 16; i++) v[i] = fmaxf(v[i], 0.0f);
    }
    if (mrow) {
      const uint4 mv[2] = {reinterpret_cast<const uint4*>(mrow + c)[0], reinterpret_cast<const uint4*>(mrow + c)[1]};
      const bf16* mb = reinterpret_cast<const bf16*>(mv);
#pragma unroll
      for (int i = 0; i < 16; i++)
        if (!(__bfloat162float(mb[i]) > 0.0f)) v[i] = 0.0f;
    }
    uint4 res[2];
    __nv_bfloat162* rb = reinterpret_cast<__nv_bfloat162*>(res);
#pragma unroll
    for (int i = 0; i < 8; i++) rb[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    o[0] = res[0];
    o[1] = res[1];
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN));
  }
  if (threadIdx.x == 0 && (*bad || !ok)) atomicExch(&g_conv_tc_error, 1);
}

// ------------------------------------------------------------------ weight gradient

// dw[co][tap][ci] += sum_p dz[p][co] in[p + off(tap)][ci] on the tcgen05 path,
// one GEMM per tap: M = 128 output channels, N = BN input channels, K = the
// pixels of a range of 8 x 16 patches (one patch, 128 pixels, per K block).
// Both operands are channel-contiguous (MN-major): the A tile is 128 / CA TMA
// boxes of dz, CA channels x 16 x 8 pixels each at the patch (channels past
// cout come back as zeros, so narrow layers fill M = 128 with zeros), the B
// tile BN / CB boxes of the input at the patch shifted by the tap (zeros
// outside the image). A box of C channels is 128 rows (pixels, the K index)
// of 2C bytes in the 2C-byte swizzle: 8-row groups are 16C bytes apart and
// the channel groups one box apart. The block's 128 x BN sum, accumulated in
// TMEM over its patches, is added to dw with vector atomics.
constexpr int DW_STAGES = 3;

template <int CA, int CB, int BN>
struct TcDwLayout {
  static constexpr int A_BOX = TC_M * CA * 2, B_BOX = TC_M * CB * 2;
  static constexpr int A_BYTES = (128 / CA) * A_BOX;
  static constexpr int B_BYTES = (BN / CB) * B_BOX;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int BYTES = DW_STAGES * STAGE + (2 * DW_STAGES + 1) * 8 + 8 + 1024;
};

// MN-major operand whose channel groups of C (64 or 32) elements are
// swizzled rows of 2C bytes: 8-row K groups 16C bytes apart (stride byte
// offset), channel groups `group_bytes` apart (leading byte offset).
__device__ __forceinline__ uint64_t smem_desc_mn(uint32_t addr, uint32_t row_bytes, uint32_t group_bytes) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((group_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)(((8u * row_bytes) >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)(row_bytes == 128 ? 2 : 4) << 61;
  return d;
}
// f32 accumulator, bf16 A and B, both MN-major, M = 128, N.
__host__ __device__ constexpr uint32_t instr_desc_mn(int n) {
  return instr_desc(n) | (1u << 15) | (1u << 16);
}

template <int CA, int CB, int BN>
__global__ void __launch_bounds__(128, 1)
    k_conv3_dw_tc(const __grid_constant__ CUtensorMap tdz, const __grid_constant__ CUtensorMap tin,
                  const TcDwArgs a) {
  using L = TcDwLayout<CA, CB, BN>;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + DW_STAGES * L::STAGE);
  uint64_t* empty = full + DW_STAGES;
  uint64_t* done = empty + DW_STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* bad = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tap = blockIdx.z, dx = tap % 3 - 1, dy = tap / 3 - 1;
  const int ci_tiles = a.Cin / BN;
  const int co0 = (blockIdx.y / ci_tiles) * 128, ci0 = (blockIdx.y % ci_tiles) * BN;
  const int tiles_x = a.W / TC_TW, tiles_y = a.H / TC_TH;
  const int64_t q0 = (int64_t)blockIdx.x * a.patches_per_block;
  const int64_t q1 = q0 + a.patches_per_block < a.patches ? q0 + a.patches_per_block : a.patches;
  const int nk = (int)(q1 - q0);

  // A boxes wholly past Cout are never loaded: they are zeroed here, once, in
  // every stage, and the MMA reads the zeros.
  const int a_boxes = (a.Cout - co0 + CA - 1) / CA < 128 / CA ? (a.Cout - co0 + CA - 1) / CA : 128 / CA;
  if (a_boxes < 128 / CA) {
    for (int s = 0; s < DW_STAGES; s++) {
      uint4* z = reinterpret_cast<uint4*>(smem + s * L::STAGE + a_boxes * L::A_BOX);
      const int n = (128 / CA - a_boxes) * L::A_BOX / 16;
      for (int i = threadIdx.x; i < n; i += blockDim.x) z[i] = make_uint4(0, 0, 0, 0);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic stores -> the MMA's reads
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < DW_STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *bad = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tmem_slot)),
                 "r"((uint32_t)BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {  // loader
    int issued = 0;
    const uint32_t bytes = (uint32_t)(a_boxes * L::A_BOX + L::B_BYTES);
    for (int kb = 0; kb < nk; kb++) {
      const int s = kb % DW_STAGES;
      if (kb >= DW_STAGES && !mbar_wait(&empty[s], ((kb / DW_STAGES) - 1) & 1)) {
        *bad = 1;
        break;
      }
      int64_t q = q0 + kb;
      const int tx = (int)(q % tiles_x);
      q /= tiles_x;
      const int ty = (int)(q % tiles_y);
      const int img = (int)(q / tiles_y);
      const int x0 = tx * TC_TW, y0 = ty * TC_TH;
      unsigned char* st = smem + s * L::STAGE;
      mbar_expect_tx(&full[s], bytes);
      for (int h = 0; h < a_boxes; h++) tma_load_4d(st + h * L::A_BOX, &tdz, &full[s], co0 + CA * h, x0, y0, img);
#pragma unroll
      for (int h = 0; h < BN / CB; h++)
        tma_load_4d(st + L::A_BYTES + h * L::B_BOX, &tin, &full[s], ci0 + CB * h, x0 + dx, y0 + dy, img);
      issued = kb + 1;
    }
    for (int kb = issued > DW_STAGES ? issued - DW_STAGES : 0; kb < issued; kb++)
      if (!mbar_wait(&full[kb % DW_STAGES], (kb / DW_STAGES) & 1)) *bad = 1;
  } else if (warp == 1 && lane == 0) {  // MMA issuer
    const uint32_t idesc = instr_desc_mn(BN);
    for (int kb = 0; kb < nk; kb++) {
      const int s = kb % DW_STAGES;
      if (!mbar_wait(&full[s], (kb / DW_STAGES) & 1)) {
        *bad = 1;
        break;
      }
      tc_fence_after();
      const uint32_t sa = saddr(smem + s * L::STAGE), sb = sa + L::A_BYTES;
#pragma unroll
      for (int k = 0; k < TC_M / 16; k++)  // 16 pixels (two 8-row groups) per MMA
        umma(tmem, smem_desc_mn(sa + 32u * CA * k, 2 * CA, L::A_BOX),
             smem_desc_mn(sb + 32u * CB * k, 2 * CB, L::B_BOX), idesc, (kb | k) != 0);
      umma_commit(&empty[s]);
    }
    umma_commit(done);
  }
  __syncwarp();
  const bool ok = mbar_wait(done, 0);
  tc_fence_after();

  // Epilogue: thread (warp, lane) owns TMEM lane 32 warp + lane, output channel co.
  const int co = co0 + warp * 32 + lane;
#pragma unroll 1
  for (int c = 0; c < BN; c += 16) {
    float v[16];
    tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
    if (!ok || nk == 0 || co >= a.Cout) continue;
    float* row = a.dw + ((int64_t)co * 9 + tap) * a.Cin + ci0 + c;
#pragma unroll
    for (int j = 0; j < 4; j++)
      atomicAdd(reinterpret_cast<float4*>(row + 4 * j), make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]));
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN));
  }
  if (threadIdx.x == 0 && (*bad || !ok)) atomicExch(&g_conv_tc_error, 1);
}

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

template <int KC, int BN>
int launch(const TcConvArgs& a, cudaStream_t s) {
  using L = TcConvLayout<KC, BN>;
  auto enc = encoder();
  if (!enc) return 2;
  const CUtensorMapSwizzle sw = KC == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B;
  CUtensorMap tin, tw;
  const cuuint64_t px = (cuuint64_t)a.ld_in * 2;
  cuuint64_t dims[4] = {(cuuint64_t)a.Cin, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.batch};
  cuuint64_t strides[3] = {px, px * (cuuint64_t)a.W, px * (cuuint64_t)a.W * (cuuint64_t)a.H};
  cuuint32_t box[4] = {(cuuint32_t)KC, (cuuint32_t)TC_TW, (cuuint32_t)TC_TH, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  if (enc(&tin, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(a.in), dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return 1;
  cuuint64_t wdims[2] = {(cuuint64_t)9 * a.Cin, (cuuint64_t)a.Cout};
  cuuint64_t wstrides[1] = {(cuuint64_t)9 * a.Cin * 2};
  cuuint32_t wbox[2] = {(cuuint32_t)KC, (cuuint32_t)BN};
  cuuint32_t westr[2] = {1, 1};
  if (enc(&tw, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(a.w), wdims, wstrides, wbox, westr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return 1;
  // per launch: the attribute belongs to the current device's context
  if (cudaFuncSetAttribute(k_conv3_tc<KC, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::BYTES) != cudaSuccess)
    return 2;
  const unsigned tiles = (unsigned)((a.W / TC_TW) * (a.H / TC_TH) * a.batch);
  k_conv3_tc<KC, BN><<<dim3(tiles, a.Cout / BN), 128, L::BYTES, s>>>(tin, tw, a);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

template <int KC>
int launch_kc(const TcConvArgs& a, cudaStream_t s) {
  if (a.Cout % 128 == 0) return launch<KC, 128>(a, s);
  if (a.Cout % 64 == 0) return launch<KC, 64>(a, s);
  return launch<KC, 32>(a, s);
}

// A 4-D map of an NHWC bf16 tensor, box (C channels, 16, 8, 1), 2C-byte swizzle.
bool nhwc_map(CUtensorMap* m, const bf16* base, int channels, int ld, int W, int H, int64_t batch, int C) {
  const cuuint64_t px = (cuuint64_t)ld * 2;
  cuuint64_t dims[4] = {(cuuint64_t)channels, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)batch};
  cuuint64_t strides[3] = {px, px * (cuuint64_t)W, px * (cuuint64_t)W * (cuuint64_t)H};
  cuuint32_t box[4] = {(cuuint32_t)C, (cuuint32_t)TC_TW, (cuuint32_t)TC_TH, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  return encoder()(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, C == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int CA, int CB, int BN>
int launch_dw(TcDwArgs a, cudaStream_t s, int sms) {
  using L = TcDwLayout<CA, CB, BN>;
  if (!encoder()) return 2;
  CUtensorMap tdz, tin;
  if (!nhwc_map(&tdz, a.dz, a.Cout, a.ld_dz, a.W, a.H, a.batch, CA) ||
      !nhwc_map(&tin, a.in, a.Cin, a.ld_in, a.W, a.H, a.batch, CB))
    return 1;
  if (cudaFuncSetAttribute(k_conv3_dw_tc<CA, CB, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::BYTES) !=
      cudaSuccess)
    return 2;
  a.patches = a.batch * (a.W / TC_TW) * (a.H / TC_TH);
  const int tiles = ((a.Cout + 127) / 128) * (a.Cin / BN);
  // about two blocks per SM over all taps and tiles, at least 8 patches each
  int64_t splits = (2 * sms + 9 * tiles - 1) / (9 * tiles);
  const int64_t max_splits = (a.patches + 7) / 8;
  if (splits > max_splits) splits = max_splits;
  if (splits < 1) splits = 1;
  a.patches_per_block = (a.patches + splits - 1) / splits;
  splits = (a.patches + a.patches_per_block - 1) / a.patches_per_block;
  k_conv3_dw_tc<CA, CB, BN><<<dim3((unsigned)splits, tiles, 9), 128, L::BYTES, s>>>(tdz, tin, a);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

template <int CA>
int launch_dw_ca(const TcDwArgs& a, cudaStream_t s, int sms) {
  if (a.Cin % 128 == 0) return launch_dw<CA, 64, 128>(a, s, sms);
  if (a.Cin % 64 == 0) return launch_dw<CA, 64, 64>(a, s, sms);
  return launch_dw<CA, 32, 32>(a, s, sms);
}

}  // namespace

// Cout a multiple of 64: with 32 output channels the 128-row tile is three
// quarters zeros and the kernel measured slower than the mma.sync one (51
// against 59-65 TFLOP/s at 256^2, batch 16).
bool conv3_dw_tc_supported(const TcDwArgs& a) {
  const auto a16 = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
  return a.W % TC_TW == 0 && a.H % TC_TH == 0 && a.Cin % 32 == 0 && a.Cout % 64 == 0 && a.ld_in % 8 == 0 &&
         a.ld_dz % 8 == 0 && a16(a.in) && a16(a.dz) && a16(a.dw) && encoder() != nullptr;
}

int conv3_dw_tc(const TcDwArgs& a, cudaStream_t s) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return launch_dw_ca<64>(a, s, sms);
}

bool conv3_tc_supported(const TcConvArgs& a) {
  const auto a16 = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
  return a.W % TC_TW == 0 && a.H % TC_TH == 0 && a.Cin % 32 == 0 && a.Cout % 32 == 0 && a.ld_in % 8 == 0 &&
         a.ld_out % 8 == 0 && (!a.mask || (a.ld_mask % 8 == 0 && a16(a.mask))) && a16(a.in) && a16(a.w) &&
         a16(a.out) && a.batch * (int64_t)(a.W / TC_TW) * (a.H / TC_TH) < (1ll << 31) && encoder() != nullptr;
}

int conv3_tc(const TcConvArgs& a, cudaStream_t s) {
  return a.Cin % 64 == 0 ? launch_kc<64>(a, s) : launch_kc<32>(a, s);
}

// The timeout path of the convolutions' waits, exercised: a block holds TMEM
// as a convolution does, waits on an mbarrier on which nothing arrives until
// the wait gives up after limit_ns, sets the flag, frees its TMEM and
// returns. Nothing else runs in the block, so nothing is left in flight.
__global__ void __launch_bounds__(128) k_wait_probe(unsigned long long limit_ns) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int gave_up;
  const int warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    gave_up = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&tmem_slot)),
                 "r"(32u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  if (threadIdx.x == 0 && !mbar_wait_for(&bar, 0, limit_ns)) gave_up = 1;
  tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32u));
  }
  if (threadIdx.x == 0 && gave_up) atomicExch(&g_conv_tc_error, 1);
}

int conv3_tc_wait_probe(unsigned long long limit_ns, cudaStream_t s) {
  k_wait_probe<<<1, 128, 0, s>>>(limit_ns);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int conv3_tc_status(cudaStream_t s) {
  int v = 0;
  if (cudaStreamSynchronize(s) != cudaSuccess) return 2;
  if (cudaMemcpyFromSymbol(&v, g_conv_tc_error, sizeof(int)) != cudaSuccess) return 2;
  const int zero = 0;
  if (v && cudaMemcpyToSymbol(g_conv_tc_error, &zero, sizeof(int)) != cudaSuccess) return 2;
  return v ? 3 : 0;
}
