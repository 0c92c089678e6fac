// The tcgen05 / TMA 3x3 convolution (nn_conv_tc.cu) behind rang_b200_nn_conv3.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

struct TcConvArgs {
  const __nv_bfloat16* in;  // NHWC, pixel stride ld_in
  const __nv_bfloat16* w;   // [Cout][9][Cin]
  const float* bias;
  __nv_bfloat16* out;
  const __nv_bfloat16* mask;
  int64_t batch;
  int H, W, ld_in, ld_out, ld_mask, Cin, Cout, relu, accumulate;
};

// Whether the shapes and alignments fit the kernel: W a multiple of 16, H of
// 8, channels of 32, pixel strides of 8, 16-byte aligned tensors.
bool conv3_tc_supported(const TcConvArgs& a);
// Launches on s; 0, 1 (the tensor maps were refused) or 2 (launch error).
int conv3_tc(const TcConvArgs& a, cudaStream_t s);
// Waits for s and reads (and clears) the device flag that a block sets when
// one of its waits gave up: 0, 3 (a wait gave up) or 2 (CUDA error).
int conv3_tc_status(cudaStream_t s);
// One block that holds TMEM and waits on an mbarrier nothing completes, with
// the given limit: the convolutions' timeout path, for the tests.
int conv3_tc_wait_probe(unsigned long long limit_ns, cudaStream_t s);

struct TcDwArgs {
  const __nv_bfloat16* in;  // NHWC forward input of the layer, pixel stride ld_in
  const __nv_bfloat16* dz;  // gradient at the layer's output, pixel stride ld_dz
  float* dw;                // [Cout][9][Cin], accumulated
  int64_t batch, patches, patches_per_block;
  int H, W, ld_in, ld_dz, Cin, Cout;
};

// Whether the weight gradient's shapes fit the tcgen05 kernel: W a multiple
// of 16, H of 8, input channels of 32, output channels of 64, pixel strides
// of 8, 16-byte aligned tensors.
bool conv3_dw_tc_supported(const TcDwArgs& a);
// dw += the weight gradient on s; 0, 1 (the tensor maps were refused) or 2.
int conv3_dw_tc(const TcDwArgs& a, cudaStream_t s);
