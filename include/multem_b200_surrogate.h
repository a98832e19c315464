/* Kernels of the learned phonon-convergence surrogate (multem_b200/surrogate.py).
 *
 * None of these has a counterpart in the reference: MULTEM always averages all frozen-phonon
 * configurations explicitly. The surrogate predicts the many-configuration HAADF image from one
 * averaged over a few, with a per-pixel error estimate used to fall back to the plain simulation.
 *
 * Tensors are device pointers in NCHW layout; "bf16" arguments point to __nv_bfloat16 data, the
 * others to float. Convolutions are 3x3 with zero padding 1, computed as BF16 GEMMs on the tensor
 * cores (tcgen05) with FP32 accumulation; all reductions run in a fixed order. Every call is
 * asynchronous on `stream` (a cudaStream_t, NULL = default) and returns MT_OK or an error status
 * without a message. The convolutions of one device share a workspace from the library's memory
 * pool (grown on demand): issue them on one stream, or order them. */
#ifndef MULTEM_B200_SURROGATE_H
#define MULTEM_B200_SURROGATE_H

#include "multem_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* out[b,o] = bias[o] + sum_i w[o,i] (*) in[b,i], optionally ReLU; written as bf16 (out_bf16) and/or
 * float (out_f32). in: bf16 [B,Cin,H,W]; w: bf16 [Cout,Cin,3,3]; bias: float [Cout] or NULL. */
mt_status mt_sg_conv3x3_forward(const void* in, const void* w, const float* bias, void* out_bf16, float* out_f32,
                                int B, int Cin, int Cout, int H, int W, int relu, void* stream);
/* din (bf16 [B,Cin,H,W]) = data gradient for the output gradient dout (bf16 [B,Cout,H,W]), masked
 * by out_mask > 0 when out_mask (the layer's ReLU output) is not NULL. */
mt_status mt_sg_conv3x3_backward_data(const void* dout, const void* out_mask, const void* w, void* din, int B, int Cin,
                                      int Cout, int H, int W, void* stream);
/* dw (float [Cout,Cin,3,3]) and db (float [Cout]) for input `in` and output gradient dout (masked as
 * above). */
mt_status mt_sg_conv3x3_backward_weight(const void* in, const void* dout, const void* out_mask, float* dw, float* db,
                                        int B, int Cin, int Cout, int H, int W, void* stream);
/* Loss of the two-channel head (float [B,2,H,W]) in units of a per-item scale s_b (float [B], or
 * NULL for 1): channel 0 corrects the input image x (bf16 [B,1,H,W]) towards target (float
 * [B,1,H,W]) as x + s_b * head0, channel 1 estimates |x + s_b * head0 - target| / s_b. Per pixel
 * dn^2 + lambda * (head1 - |dn|)^2 with dn = (x + s_b * head0 - target) / s_b. Writes dloss/dhead
 * (bf16 [B,2,H,W], mean over pixels) and the per-pixel loss terms (float [B,H,W]). */
mt_status mt_sg_loss(const float* head, const void* x, const float* target, const float* scale, void* dhead,
                     float* terms, int B, int H, int W, float lambda, void* stream);
/* Adam step (1-based `step`) on float master weights w with moments m, v; also writes the bf16 copy
 * w_bf16 when not NULL. */
mt_status mt_sg_adam(float* w, void* w_bf16, const float* g, float* m, float* v, int n, float lr, float b1, float b2,
                     float eps, int step, void* stream);
/* out (bf16 [B,C,H/2,W/2]) = scale * sum of each 2x2 block of in (bf16 [B,C,H,W]); H and W even.
 * scale 1/4 is average pooling, scale 1 the gradient of mt_sg_upsample2. */
mt_status mt_sg_pool2(const void* in, void* out, int B, int C, int H, int W, float scale, void* stream);
/* out (bf16 [B,C,2H,2W]) = scale * in[b,c,y/2,x/2] (in: bf16 [B,C,H,W]). scale 1 is nearest-neighbour
 * upsampling, scale 1/4 the gradient of average pooling. */
mt_status mt_sg_upsample2(const void* in, void* out, int B, int C, int H, int W, float scale, void* stream);
/* out = a + b, n bf16 values (skip connections and the sum of two gradients). */
mt_status mt_sg_add(const void* a, const void* b, void* out, long long n, void* stream);
/* b (bf16) = a (float), n values. */
mt_status mt_sg_to_bf16(const float* a, void* b, int n, void* stream);
/* Synchronises `stream`; MT_ERR_TIMEOUT (and the flag cleared) when a convolution's GEMM issued
 * before gave up waiting for its operands (every wait is bounded at 1 s), MT_OK otherwise. */
mt_status mt_sg_check(void* stream);

#ifdef __cplusplus
}
#endif

#endif
