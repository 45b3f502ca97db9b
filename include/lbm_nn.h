/*
 * lbm_nn.h -- kernels of the warm-start surrogate: a small 2D U-Net that
 * predicts the steady rho, u, T of a porous geometry so that the lattice can be
 * started near its steady state.
 *
 * No counterpart in the reference: its only learned-model code is a torch
 * import test (tests/test_pytorch.py); the surrogate exists to shorten the time
 * the plain solver (src/LBM/LBM2D/_evolution.py:12-25) needs to reach steady
 * state, and it never changes the converged answer.
 *
 * Conventions (same as lbm_b200.h): int32 status, lbm_last_error() for the
 * message, caller-owned device memory, work on the caller's stream.
 * Activations are NHWC bf16 with channel counts, channel strides and channel
 * offsets that are multiples of 8 (a layer can read or write a slice of a wider
 * buffer); weights are bf16 [Cout][ksize*ksize][Cin]; gradients of weights and
 * biases are FP32 and accumulate (zero them first).
 */
#ifndef LBM_NN_H
#define LBM_NN_H

#include <stddef.h>
#include <stdint.h>

#include "lbm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_NN_ERR_ARG LBM_ERR_ARG
#define LBM_NN_ERR_CUDA LBM_ERR_CUDA

/* The 3D forms of the four calls above (NDHWC, B x D x H x W pixels, x fastest;
 * 3 x 3 x 3 or 1 x 1 x 1 taps in z, y, x order with x fastest, weights
 * [Cout][taps][Cin]; 2 x 2 x 2 pooling and nearest upsampling; D, H, W are the
 * input's sizes).  For the 3D variant of the warm-start network (16 base
 * channels); lbm_nn_flip_weights, bias_grad, mse, adam, relu_bwd and to_bf16
 * serve both. */
LBM_API int32_t lbm_nn_conv3d(const void* in, int32_t in_cstride, int32_t in_coff, const void* w, const float* bias,
                              const void* gate, void* out_bf16, float* out_f32, int32_t out_cstride, int32_t out_coff,
                              int32_t B, int32_t D, int32_t H, int32_t W, int32_t Cin, int32_t Cout, int32_t ksize,
                              int32_t relu, int32_t accumulate, void* stream);
LBM_API int32_t lbm_nn_conv3d_wgrad(const void* in, int32_t in_cstride, int32_t in_coff, const void* dout,
                                    int32_t dout_cstride, int32_t dout_coff, float* dw, int32_t B, int32_t D, int32_t H,
                                    int32_t W, int32_t Cin, int32_t Cout, int32_t ksize, void* stream);
LBM_API int32_t lbm_nn_avgpool2_3d(const void* in, int32_t in_cstride, int32_t in_coff, void* out, int32_t B,
                                   int32_t D, int32_t H, int32_t W, int32_t C, void* stream);
LBM_API int32_t lbm_nn_avgpool2_3d_bwd(const void* dout, void* din, int32_t din_cstride, int32_t din_coff, int32_t B,
                                       int32_t D, int32_t H, int32_t W, int32_t C, int32_t accumulate, void* stream);
LBM_API int32_t lbm_nn_upsample2_3d(const void* in, void* out, int32_t out_cstride, int32_t out_coff, int32_t B,
                                    int32_t D, int32_t H, int32_t W, int32_t C, void* stream);
LBM_API int32_t lbm_nn_upsample2_3d_bwd(const void* dout, int32_t dout_cstride, int32_t dout_coff, void* din,
                                        int32_t B, int32_t D, int32_t H, int32_t W, int32_t C, void* stream);

/* out = act(conv(in, w) + bias), same padding, stride 1, ksize 1 or 3, on the
 * tensor cores (bf16 inputs, FP32 accumulation).  act: ReLU if relu; then, if
 * gate is not NULL, out = 0 where gate <= 0 (gate laid out like out: the ReLU
 * gradient mask of a backward pass).  Exactly one of out_bf16 / out_f32;
 * accumulate adds to it.  The input gradient of a layer is this call on the
 * output gradient with lbm_nn_flip_weights() weights (Cin and Cout swapped). */
LBM_API int32_t lbm_nn_conv(const void* in, int32_t in_cstride, int32_t in_coff, const void* w, const float* bias,
                            const void* gate, void* out_bf16, float* out_f32, int32_t out_cstride, int32_t out_coff,
                            int32_t B, int32_t H, int32_t W, int32_t Cin, int32_t Cout, int32_t ksize, int32_t relu,
                            int32_t accumulate, void* stream);
/* dw[n][t][c] += sum over pixels of dout[p][n] * in[p + off(t)][c] (tensor cores). */
LBM_API int32_t lbm_nn_conv_wgrad(const void* in, int32_t in_cstride, int32_t in_coff, const void* dout,
                                  int32_t dout_cstride, int32_t dout_coff, float* dw, int32_t B, int32_t H, int32_t W,
                                  int32_t Cin, int32_t Cout, int32_t ksize, void* stream);
/* dbias[n] += sum over P pixels of dout[p][n]. */
LBM_API int32_t lbm_nn_bias_grad(const void* dout, int32_t cstride, int32_t coff, int32_t P, int32_t Cout, float* dbias,
                                 void* stream);
/* wt[c][taps-1-t][n] = w[n][t][c]. */
LBM_API int32_t lbm_nn_flip_weights(const void* w, void* wt, int32_t Cout, int32_t taps, int32_t Cin, void* stream);
/* 2x2 average pooling of a channel slice into a dense [B][H/2][W/2][C] tensor, and its gradient. */
LBM_API int32_t lbm_nn_avgpool2(const void* in, int32_t in_cstride, int32_t in_coff, void* out, int32_t B, int32_t H,
                                int32_t W, int32_t C, void* stream);
LBM_API int32_t lbm_nn_avgpool2_bwd(const void* dout, void* din, int32_t din_cstride, int32_t din_coff, int32_t B,
                                    int32_t H, int32_t W, int32_t C, int32_t accumulate, void* stream);
/* Nearest 2x upsampling of a dense [B][H][W][C] tensor into a channel slice, and its gradient. */
LBM_API int32_t lbm_nn_upsample2(const void* in, void* out, int32_t out_cstride, int32_t out_coff, int32_t B, int32_t H,
                                 int32_t W, int32_t C, void* stream);
LBM_API int32_t lbm_nn_upsample2_bwd(const void* dout, int32_t dout_cstride, int32_t dout_coff, void* din, int32_t B,
                                     int32_t H, int32_t W, int32_t C, void* stream);
/* Weighted squared error: partial[b] = block sums of weight*(pred-target)^2,
 * grad = 2*scale*weight*(pred-target) as bf16 (weight may be NULL). */
LBM_API int32_t lbm_nn_mse(const float* pred, const float* target, const float* weight, size_t n, float scale,
                           void* grad, float* partial, int32_t nblocks, void* stream);
/* Adam (bias-corrected; weight_decay adds an L2 term to the gradient) on FP32
 * master weights; refreshes the bf16 copy w_bf16 when not NULL. */
LBM_API int32_t lbm_nn_adam(float* w, const float* g, float* m, float* v, void* w_bf16, size_t n, float lr, float beta1,
                            float beta2, float eps, int32_t step, float weight_decay, void* stream);
/* ReLU gradient on a channel slice: dy = 0 where the activation y <= 0. */
LBM_API int32_t lbm_nn_relu_bwd(void* dy, int32_t dy_cstride, int32_t dy_coff, const void* y, int32_t y_cstride,
                                int32_t y_coff, int32_t P, int32_t C, void* stream);
LBM_API int32_t lbm_nn_to_bf16(const float* x, void* y, size_t n, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LBM_NN_H */
