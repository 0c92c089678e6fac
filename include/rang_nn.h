/*
 * rang_nn.h — the layers of the learned FISTA proposal network on the B200.
 *
 * The reference has no network on its imaging path. Its nearest relatives are
 * the learned-stage interpreter (core/src/learned_interp.rs:1-22: NCHW f32
 * Conv/Relu inference of a dilated CNN read from ONNX) and the learned
 * deconvolution trial (examples/dl4b_train.py:51-72, a dilated CNN trained
 * with PyTorch). The proposal network here is new: a 4-level U-Net
 * (32/64/128/256 channels, 3x3 convolutions with ReLU, 2x2 average pooling,
 * nearest 2x upsampling, skip connections by concatenation, a 1x1 head) that
 * maps a residual patch and a PSF patch to a model update, trained and run by
 * these entry points alone. The layer sequence is driven from the host
 * (python: rang.learned); every entry point launches on `stream` (the
 * caller's cudaStream_t; null: the legacy default stream) and returns 0, or
 * 1 for invalid arguments, or 2 when the launch failed.
 *
 * Tensors are NHWC bfloat16 device arrays addressed by a pointer and a pixel
 * stride `ld_*` in elements (a multiple of 8; pointers 16-byte aligned): a
 * channel slice of a wider tensor is a pointer offset by its first channel
 * plus the wider tensor's stride. Convolution weights are bfloat16
 * [cout][9][cin] (tap = 3 * ky + kx); biases, weight gradients and the
 * optimiser state are float32. All sums accumulate in float32.
 */
#ifndef RANG_NN_H
#define RANG_NN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* out[p, co] = bias[co] + sum_{tap, ci} w[co, tap, ci] in[p + (ky - 1, kx - 1), ci]
 * with zeros outside each height x width image, then (in this order) plus
 * the old out (accumulate), max(., 0) (relu), and zero where mask <= 0
 * (mask non-null). cin and cout are multiples of 32. Tensor cores: tcgen05
 * where the shapes allow it (rang_b200_nn_set_conv_path). */
int32_t rang_b200_nn_conv3(const void* in, int64_t ld_in, const void* w, const float* bias, void* out, int64_t ld_out,
                           const void* mask, int64_t ld_mask, int64_t batch, int32_t height, int32_t width,
                           int32_t cin, int32_t cout, int32_t relu, int32_t accumulate, void* stream);

/* dw[co, tap, ci] += sum_p dz[p, co] in[p + (ky - 1, kx - 1), ci] and, when
 * dbias is non-null, dbias[co] += sum_p dz[p, co]. Tensor cores: tcgen05
 * where width is a multiple of 16, height of 8 and cout of 64
 * (rang_b200_nn_set_conv_path). */
int32_t rang_b200_nn_conv3_weight_grad(const void* in, int64_t ld_in, const void* dz, int64_t ld_dz, float* dw,
                                       float* dbias, int64_t batch, int32_t height, int32_t width, int32_t cin,
                                       int32_t cout, void* stream);

/* Which kernels conv3 and conv3_weight_grad run: 0 (the default) the tcgen05
 * kernels (TMA operands, TMEM accumulator) wherever the shapes and alignments
 * allow them, else the mma.sync kernels; 1 always the mma.sync kernels.
 * Process-wide; returns the previous value. */
int32_t rang_b200_nn_set_conv_path(int32_t path);

/* Waits for the stream and reports whether a tcgen05 convolution gave up on
 * a wait (a stalled pipeline, which then leaves its output unspecified):
 * 0 none, 3 one did (the flag is cleared), 2 a CUDA error. */
int32_t rang_b200_nn_device_status(void* stream);

/* The timeout path of the tcgen05 convolutions, for tests: one block holds
 * TMEM and waits on an mbarrier that nothing completes until the wait gives
 * up after limit_ns (at most 10 s), then frees its TMEM and sets the flag
 * that rang_b200_nn_device_status reports as 3. 0, 1 (bad limit) or 2. */
int32_t rang_b200_nn_wait_probe(int64_t limit_ns, void* stream);

/* wt[ci, tap, co] = w[co, 8 - tap, ci]: the weights with which conv3 computes
 * the gradient with respect to its input. */
int32_t rang_b200_nn_conv3_flip(const void* w, void* wt, int32_t cin, int32_t cout, void* stream);

/* 2x2 average pooling of height x width images (both even). */
int32_t rang_b200_nn_pool(const void* in, int64_t ld_in, void* out, int64_t ld_out, int64_t batch, int32_t height,
                          int32_t width, int32_t channels, void* stream);

/* grad = (grad + dpool / 4 at the pooled pixel) * (act > 0), in place, on
 * height x width images: the gradient of an encoder output that feeds both a
 * skip connection (grad holds that part) and the pooling. */
int32_t rang_b200_nn_pool_backward(void* grad, int64_t ld_grad, const void* dpool, int64_t ld_dpool, const void* act,
                                   int64_t ld_act, int64_t batch, int32_t height, int32_t width, int32_t channels,
                                   void* stream);

/* Nearest 2x upsampling to height x width (both even). */
int32_t rang_b200_nn_upsample(const void* in, int64_t ld_in, void* out, int64_t ld_out, int64_t batch, int32_t height,
                              int32_t width, int32_t channels, void* stream);

/* out (height x width) = the sum over each 2x2 block of grad (2 height x 2 width). */
int32_t rang_b200_nn_upsample_backward(const void* grad, int64_t ld_grad, void* out, int64_t ld_out, int64_t batch,
                                       int32_t height, int32_t width, int32_t channels, void* stream);

/* The network input, 32 channels: (resid[offsets[b] + y ld_resid + x] *
 * scale_resid, psf[y ld_psf + x] * scale_psf, 0, ...) for patch b. Float32
 * sources on the device; offsets is a device array of batch int64. */
int32_t rang_b200_nn_pack(const float* resid, const int64_t* offsets, int64_t ld_resid, const float* psf,
                          int64_t ld_psf, float scale_resid, float scale_psf, void* x, int64_t batch, int32_t height,
                          int32_t width, void* stream);

/* The 1x1 head, 32 channels to one float32 output: out[p] = bias[0] + sum_c w[c] act[p, c]. */
int32_t rang_b200_nn_head(const void* act, int64_t ld, const float* w, const float* bias, float* out, int64_t pixels,
                          void* stream);

/* The head's backward: dact = dout w (act > 0) (bfloat16), dw += sum dout act,
 * dbias += sum dout. */
int32_t rang_b200_nn_head_backward(const void* act, int64_t ld, const float* w, const float* dout, void* dact,
                                   int64_t ld_dact, float* dw, float* dbias, int64_t pixels, void* stream);

/* Mean squared error of pred (batch x height x width float32) against the
 * targets target[offsets[b] + y ld_target + x]: *loss += the mean, grad = its
 * gradient. */
int32_t rang_b200_nn_mse(const float* pred, const float* target, const int64_t* offsets, int64_t ld_target,
                         float* grad, float* loss, int64_t batch, int32_t height, int32_t width, void* stream);

/* dst[offsets[b] + y ld + x] = out[b, y, x] * scale inside the window
 * [windows[4b], windows[4b+1]) x [windows[4b+2], windows[4b+3]) of each patch
 * (int32 device array): a tiled image from the network's patches. */
int32_t rang_b200_nn_unpack(const float* out, const int64_t* offsets, const int32_t* windows, int64_t ld, float scale,
                            float* dst, int64_t batch, int32_t height, int32_t width, void* stream);

/* One Adam step with bias-corrected moments (step >= 1) on float32 master
 * weights p, refreshing their bfloat16 copy pb (non-null) and clearing g. */
int32_t rang_b200_nn_adam(float* p, void* pb, float* g, float* m, float* v, int64_t n, float lr, float beta1,
                          float beta2, float eps, int32_t step, void* stream);

/* dst = bfloat16(src), round to nearest even. */
int32_t rang_b200_nn_to_bf16(const float* src, void* dst, int64_t n, void* stream);

#ifdef __cplusplus
}
#endif

#endif
