/* coffee_surrogate.h -- C ABI of the learned warm start's kernels.
 *
 * A small 3D convolutional network that predicts a magnetosphere's fields
 * from its star's dipole (no counterpart in the reference: COFFEE always
 * starts from the vacuum dipole).  Training and inference run on these
 * kernels: 3x3x3 "same" convolutions as BF16 tensor-core implicit GEMMs
 * (mma.sync m16n8k16, FP32 accumulation) for the forward pass and both
 * gradients, plus the elementwise, pooling, loss and Adam kernels around them.
 *
 * Layout: activations channels-last, (N, D, H, W, C) with C a multiple of
 * 16; weights (K, 27, C), tap t = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1), zero
 * padding of one point.  Every pointer is device memory; every call is
 * asynchronous on `stream` (a cudaStream_t, NULL for the legacy default)
 * and returns COFFEE_OK or a negative status (coffee_b200.h).
 */
#ifndef COFFEE_SURROGATE_H
#define COFFEE_SURROGATE_H

#include <stddef.h>

#include "coffee_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* y = conv(x, w) + bias.  z (FP32, or NULL) receives y; a (BF16, or NULL)
 * receives leaky(y) = max(y, slope y) when act != 0, else y.  C % 16 == 0,
 * K % 8 == 0, K <= 64; bias may be NULL. */
COFFEE_API int coffee_conv3d_forward(const void* x, int n, int d, int h, int w, int c,
                                     const void* weight, int k, const float* bias, float* z,
                                     void* a, int act, float slope, void* stream);
/* The same convolution on the tcgen05 tensor cores (sm_100a): A fetched by
 * TMA (one shifted box per tap, zero fill at the edges), weights staged once
 * per CTA, the accumulator in tensor memory (two, so the epilogue overlaps), one
 * persistent CTA per resident slot.  K = 16, 32, 48 or 64; C % 16 == 0 with
 * 54 K C bytes of weights fitting shared memory (K C <= 3500); x and weight
 * 16-byte aligned.  Results equal coffee_conv3d_forward's up to the order of
 * the FP32 additions.  Also the input gradient: call it on dy with the
 * flipped weights (coffee_conv3d_flip_weights), bias NULL, act 0. */
COFFEE_API int coffee_conv3d_forward_tc(const void* x, int n, int d, int h, int w, int c,
                                        const void* weight, int k, const float* bias, float* z,
                                        void* a, int act, float slope, void* stream);
/* Every pipeline wait of the tcgen05 kernel is bounded (about 2 s).  A wait
 * that runs out makes the kernel drain what it has in flight, free its
 * tensor memory and return with its results invalid; it sets a fault that
 * every later coffee_conv3d_forward_tc call reports as COFFEE_E_TIMEOUT
 * (without synchronising) until it is cleared.  coffee_conv3d_tc_fault:
 * *fault = 1 if such a wait ran out since the last clear; clear != 0 resets
 * it.  Synchronous. */
COFFEE_API int coffee_conv3d_tc_fault(int* fault, int clear);
/* Test hook of the timeout path (no counterpart in the reference): the
 * following coffee_conv3d_forward_tc launches bound their waits by `cycles`
 * GPU clock cycles (0 restores the default) and, with stall_producer != 0,
 * issue no TMA loads at all, so that the MMA thread's first
 * wait runs out while nothing is in flight. */
COFFEE_API int coffee_conv3d_tc_set_test_wait(long long cycles, int stall_producer);
/* wt (C, 27, K) = w (K, 27, C) with the taps reversed: the weights of the
 * transposed convolution. */
COFFEE_API int coffee_conv3d_flip_weights(const void* weight, int k, int c, void* wt,
                                          void* stream);
/* dx (FP32, N D H W C) = dL/dx for dy (BF16, N D H W K): a forward pass with
 * the flipped weights wt.  K % 16 == 0, C % 8 == 0, C <= 64. */
COFFEE_API int coffee_conv3d_backward_data(const void* dy, int n, int d, int h, int w, int k,
                                           const void* wt, int c, float* dx, void* stream);
/* dw (FP32, K 27 C) = dL/dw for dy (BF16) and the layer input x (BF16).
 * K % 16 == 0, C % 8 == 0, C <= 64.  workspace: at least
 * coffee_conv3d_backward_weight_workspace(k, c) bytes of device memory
 * (per-chunk partial sums, added in a fixed order: deterministic). */
COFFEE_API size_t coffee_conv3d_backward_weight_workspace(int k, int c);
COFFEE_API int coffee_conv3d_backward_weight(const void* dy, const void* x, int n, int d, int h,
                                             int w, int k, int c, float* dw, void* workspace,
                                             void* stream);
/* The same weight gradient on the fifth-generation tensor cores (sm_100a):
 * a GEMM over points with both operands MN-major in shared memory (the layer
 * input shifted by each tap and dy, loaded by TMA, zeros outside the grid),
 * FP32 accumulation in tensor memory, per-chunk partial sums added in a
 * fixed order (deterministic; the summation order differs from
 * coffee_conv3d_backward_weight's, so the two agree to FP32 rounding).
 * C in {16, 32, 48, 64}, K in {16, 32, 64}; dy, x and workspace 16-byte
 * aligned; workspace as above.  Bounded waits as coffee_conv3d_forward_tc
 * (the same fault word and COFFEE_E_TIMEOUT). */
COFFEE_API int coffee_conv3d_backward_weight_tc(const void* dy, const void* x, int n, int d,
                                                int h, int w, int k, int c, float* dw,
                                                void* workspace, void* stream);
/* db[k] = sum over points of dz[., k] (FP32), k <= 64: per-range partial
 * sums in a library-owned device buffer, added in a fixed order
 * (deterministic); calls that could overlap on the GPU (other streams, other
 * host threads) must not share a device. */
COFFEE_API int coffee_bias_grad(const float* dz, long long npts, int k, float* db, void* stream);
/* dz = da * leaky'(z) (FP32 and a BF16 copy). */
COFFEE_API int coffee_leaky_backward(const float* da, const float* z, long long count, float slope,
                                     float* dz, void* dz_bf16, void* stream);
/* 2 x 2 x 2 average pooling of BF16 activations (N, D, H, W, C) ->
 * (N, D/2, H/2, W/2, C); its gradient added to dx (FP32, full size). */
COFFEE_API int coffee_pool2_forward(const void* x, int n, int d, int h, int w, int c, void* y,
                                    void* stream);
COFFEE_API int coffee_pool2_backward_add(const float* dy, int n, int d, int h, int w, int c,
                                         float* dx, void* stream);
/* Nearest 2x upsampling of BF16 (N, D, H, W, C) into channels [off, off + C)
 * of y (N, 2D, 2H, 2W, cy); its gradient: dx (FP32, N D H W C) = the sum of
 * the eight children's channels [off, off + C) of dy (FP32, cy channels). */
COFFEE_API int coffee_up2_forward(const void* x, int n, int d, int h, int w, int c, void* y,
                                  int cy, int off, void* stream);
COFFEE_API int coffee_up2_backward(const float* dy, int n, int d, int h, int w, int c, int cy,
                                   int off, float* dx, void* stream);
/* Channel slices: BF16 copy dst[p, doff + i] = src[p, i] (i < c), and the
 * FP32 gradient add dx[p, i] += dsrc[p, soff + i]. */
COFFEE_API int coffee_channels_copy(const void* src, long long npts, int c, void* dst, int cdst,
                                    int doff, void* stream);
COFFEE_API int coffee_channels_add(const float* dsrc, long long npts, int csrc, int soff, int c,
                                   float* dx, void* stream);
/* Masked mean-square error: loss[0] (FP64, device) = sum(mask (out - target)^2) / count,
 * dout = 2 mask (out - target) / count; mask (FP32, one per point) may be NULL.
 * loss points to 257 doubles (loss[1..256] hold the per-block partial sums,
 * added in a fixed order). */
COFFEE_API int coffee_mse(const float* out, const float* target, const float* mask,
                          long long npts, int c, double count, float* dout, double* loss,
                          void* stream);
/* Adam step on FP32 master weights w with moments m, v (bias-corrected with
 * step t >= 1); w_bf16 receives the BF16 copy the convolutions read. */
COFFEE_API int coffee_adam(float* w, const float* g, float* m, float* v, long long count,
                           float lr, float beta1, float beta2, float eps, int t, void* w_bf16,
                           void* stream);
/* FP32 -> BF16, round to nearest even. */
COFFEE_API int coffee_to_bf16(const float* src, long long count, void* dst, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* COFFEE_SURROGATE_H */
