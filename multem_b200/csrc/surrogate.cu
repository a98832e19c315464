// Kernels of the learned phonon-convergence surrogate: a small convolutional network that maps a
// HAADF image averaged over a few frozen-phonon configurations to the image averaged over many.
//
// Tensors are NCHW. Activations and weights are stored in BF16, every product is accumulated in
// FP32, biases and gradients are FP32, and the optimiser keeps FP32 master weights. Convolutions
// are 3x3 with zero padding 1 ("same" size):
//   forward      out[b,o,y,x]   = bias[o] + sum_{i,ky,kx} w[o,i,ky,kx] * in[b,i,y+ky-1,x+kx-1]
//   data grad    din[b,i,y,x]   = sum_{o,ky,kx} w[o,i,ky,kx] * dout'[b,o,y-ky+1,x-kx+1]
//   weight grad  dw[o,i,ky,kx]  = sum_{b,y,x} dout'[b,o,y,x] * in[b,i,y+ky-1,x+kx-1]
// where dout' is the output gradient masked by the ReLU of the output when the layer has one.
// Reductions run in a fixed order (deterministic results).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "common.hpp"
#include "multem_b200_surrogate.h"

namespace {

constexpr int TILE = 16;  // output tile edge per CTA (16 x 16 threads)
constexpr int OB = 8;     // output channels per CTA

__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }

// Forward (and, with TRANSPOSE, the data gradient: channels swapped and the kernel flipped).
// grid: (ceil(W/16) * ceil(H/16), ceil(Cout/OB), B); block 16 x 16.
template <bool TRANSPOSE>
__global__ void __launch_bounds__(256) conv3x3_kernel(const __nv_bfloat16* __restrict__ in, const __nv_bfloat16* __restrict__ w,
                                                      const float* __restrict__ bias, const __nv_bfloat16* __restrict__ mask,
                                                      __nv_bfloat16* __restrict__ out_bf, float* __restrict__ out_f,
                                                      int B, int Cin, int Cout, int H, int W, int relu) {
    __shared__ float tile[TILE + 2][TILE + 2];
    __shared__ float wt[OB][9];
    const int tiles_x = (W + TILE - 1) / TILE;
    const int tx0 = (blockIdx.x % tiles_x) * TILE, ty0 = (blockIdx.x / tiles_x) * TILE;
    const int o0 = blockIdx.y * OB, b = blockIdx.z;
    const int lx = threadIdx.x, ly = threadIdx.y, tid = ly * TILE + lx;
    const int x = tx0 + lx, y = ty0 + ly;
    float acc[OB];
#pragma unroll
    for (int k = 0; k < OB; k++) acc[k] = 0.0f;
    for (int i = 0; i < Cin; i++) {
        // input tile with a one-pixel halo; in the data-gradient form the "input" is the masked
        // output gradient of channel i
        for (int e = tid; e < (TILE + 2) * (TILE + 2); e += TILE * TILE) {
            const int yy = ty0 - 1 + e / (TILE + 2), xx = tx0 - 1 + e % (TILE + 2);
            float v = 0.0f;
            if (yy >= 0 && yy < H && xx >= 0 && xx < W) {
                const size_t idx = (((size_t)b * Cin + i) * H + yy) * W + xx;
                v = bf(in[idx]);
                if (mask && !(bf(mask[idx]) > 0.0f)) v = 0.0f;
            }
            tile[e / (TILE + 2)][e % (TILE + 2)] = v;
        }
        for (int e = tid; e < OB * 9; e += TILE * TILE) {
            const int k = e / 9, q = e % 9, o = o0 + k;
            float v = 0.0f;
            if (o < Cout) {
                // forward: w[o][i][q]; data gradient: w[i][o][8 - q] (flipped, channels swapped)
                v = TRANSPOSE ? bf(w[((size_t)i * Cout + o) * 9 + (8 - q)]) : bf(w[((size_t)o * Cin + i) * 9 + q]);
            }
            wt[k][q] = v;
        }
        __syncthreads();
#pragma unroll
        for (int ky = 0; ky < 3; ky++)
#pragma unroll
            for (int kx = 0; kx < 3; kx++) {
                const float v = tile[ly + ky][lx + kx];
#pragma unroll
                for (int k = 0; k < OB; k++) acc[k] = __fmaf_rn(wt[k][ky * 3 + kx], v, acc[k]);
            }
        __syncthreads();
    }
    if (x >= W || y >= H) return;
#pragma unroll
    for (int k = 0; k < OB; k++) {
        const int o = o0 + k;
        if (o >= Cout) break;
        float v = acc[k] + (bias ? bias[o] : 0.0f);
        if (relu) v = fmaxf(v, 0.0f);
        const size_t idx = (((size_t)b * Cout + o) * H + y) * W + x;
        if (out_bf) out_bf[idx] = __float2bfloat16_rn(v);
        if (out_f) out_f[idx] = v;
    }
}

// Weight and bias gradients: one CTA per (o, i) pair (i == Cin computes the bias gradient of o).
// 256 threads stride over the B*H*W output pixels; per-thread partial sums are reduced in a fixed
// tree order.
__global__ void __launch_bounds__(256) conv3x3_wgrad_kernel(const __nv_bfloat16* __restrict__ in, const __nv_bfloat16* __restrict__ dout,
                                                            const __nv_bfloat16* __restrict__ mask, float* __restrict__ dw,
                                                            float* __restrict__ db, int B, int Cin, int Cout, int H, int W) {
    const int o = blockIdx.x / (Cin + 1), i = blockIdx.x % (Cin + 1);
    const bool bias_only = (i == Cin);
    float acc[9];
#pragma unroll
    for (int q = 0; q < 9; q++) acc[q] = 0.0f;
    const int npix = B * H * W;
    for (int p = threadIdx.x; p < npix; p += blockDim.x) {
        const int b = p / (H * W), yx = p % (H * W), y = yx / W, x = yx % W;
        const size_t oi = (((size_t)b * Cout + o) * H + y) * W + x;
        float g = bf(dout[oi]);
        if (mask && !(bf(mask[oi]) > 0.0f)) g = 0.0f;
        if (g == 0.0f) continue;
        if (bias_only) {
            acc[0] += g;
            continue;
        }
#pragma unroll
        for (int ky = 0; ky < 3; ky++)
#pragma unroll
            for (int kx = 0; kx < 3; kx++) {
                const int yy = y + ky - 1, xx = x + kx - 1;
                if (yy >= 0 && yy < H && xx >= 0 && xx < W)
                    acc[ky * 3 + kx] = __fmaf_rn(g, bf(in[(((size_t)b * Cin + i) * H + yy) * W + xx]), acc[ky * 3 + kx]);
            }
    }
    __shared__ float red[9][256];
#pragma unroll
    for (int q = 0; q < 9; q++) red[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
#pragma unroll
            for (int q = 0; q < 9; q++) red[q][threadIdx.x] += red[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (bias_only) {
            db[o] = red[0][0];
        } else {
#pragma unroll
            for (int q = 0; q < 9; q++) dw[((size_t)o * Cin + i) * 9 + q] = red[q][0];
        }
    }
}

// Loss of the two-channel head in units of a per-item scale s_b (the item's noise level; 1 when
// no scales are given). Channel 0 is a correction r to the input image x (prediction
// yh = x + s_b * r), channel 1 an estimate e of |yh - t| / s_b per pixel. Per pixel, with
// dn = (yh - t) / s_b:
//   loss = dn^2 + lambda * (e - |dn|)^2   (the error target is not differentiated)
// gradients (scaled by 1/n) go to dhead as BF16; per-pixel losses to `terms` for a fixed-order sum.
__global__ void surrogate_loss_kernel(const float* __restrict__ head, const __nv_bfloat16* __restrict__ x,
                                      const float* __restrict__ t, const float* __restrict__ scale,
                                      __nv_bfloat16* __restrict__ dhead, float* __restrict__ terms, int B, int HW,
                                      float lambda) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= B * HW) return;
    const int b = p / HW, q = p % HW;
    const float sc = scale ? scale[b] : 1.0f;
    const float r = head[(size_t)b * 2 * HW + q], e = head[(size_t)b * 2 * HW + HW + q];
    const float yh = __fmaf_rn(sc, r, bf(x[p]));
    const float dn = __fdiv_rn(yh - t[p], sc);
    const float ad = fabsf(dn);
    const float n = (float)(B * HW);
    dhead[(size_t)b * 2 * HW + q] = __float2bfloat16_rn(2.0f * dn / n);
    dhead[(size_t)b * 2 * HW + HW + q] = __float2bfloat16_rn(2.0f * lambda * (e - ad) / n);
    terms[p] = dn * dn + lambda * (e - ad) * (e - ad);
}

// Adam step on FP32 master weights; writes the BF16 copy the kernels read.
__global__ void adam_kernel(float* __restrict__ wm, __nv_bfloat16* __restrict__ wb, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, int n, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float w = wm[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    wm[i] = w;
    if (wb) wb[i] = __float2bfloat16_rn(w);
}

// 2 x 2 block sum times `scale` ([B*C, H, W] -> [B*C, H/2, W/2]): average pooling with scale 1/4,
// the gradient of nearest-neighbour upsampling with scale 1.
__global__ void pool2_kernel(const __nv_bfloat16* __restrict__ in, __nv_bfloat16* __restrict__ out, int planes, int H,
                             int W, float scale) {
    const int Ho = H / 2, Wo = W / 2;
    const size_t n = (size_t)planes * Ho * Wo;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const size_t pl = k / ((size_t)Ho * Wo);
        const int r = (int)(k % ((size_t)Ho * Wo)), y = r / Wo, x = r % Wo;
        const __nv_bfloat16* s = in + (pl * H + 2 * y) * W + 2 * x;
        const float v = (bf(s[0]) + bf(s[1])) + (bf(s[W]) + bf(s[W + 1]));
        out[k] = __float2bfloat16_rn(v * scale);
    }
}

// Nearest-neighbour 2x upsampling times `scale` ([B*C, H, W] -> [B*C, 2H, 2W]): upsampling with
// scale 1, the gradient of average pooling with scale 1/4.
__global__ void upsample2_kernel(const __nv_bfloat16* __restrict__ in, __nv_bfloat16* __restrict__ out, int planes,
                                 int H, int W, float scale) {
    const int Ho = 2 * H, Wo = 2 * W;
    const size_t n = (size_t)planes * Ho * Wo;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const size_t pl = k / ((size_t)Ho * Wo);
        const int r = (int)(k % ((size_t)Ho * Wo)), y = r / Wo, x = r % Wo;
        out[k] = __float2bfloat16_rn(bf(in[(pl * H + y / 2) * W + x / 2]) * scale);
    }
}

__global__ void add_kernel(const __nv_bfloat16* __restrict__ a, const __nv_bfloat16* __restrict__ b,
                           __nv_bfloat16* __restrict__ out, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        out[k] = __float2bfloat16_rn(bf(a[k]) + bf(b[k]));
}

unsigned elem_grid(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); }

__global__ void to_bf16_kernel(const float* __restrict__ a, __nv_bfloat16* __restrict__ b, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16_rn(a[i]);
}

template <class F>
mt_status run(F f) {
    try {
        f();
        return MT_OK;
    } catch (const mtb::Error& e) {
        return e.status;
    } catch (...) {
        return MT_ERR_INTERNAL;
    }
}

void check_shape(int B, int Cin, int Cout, int H, int W) {
    if (B <= 0 || Cin <= 0 || Cout <= 0 || H <= 0 || W <= 0 || (size_t)B * H * W > (1u << 30))
        mtb::fail(MT_ERR_INVALID_ARG, "bad convolution shape");
}

dim3 conv_grid(int B, int Cout, int H, int W) {
    return dim3((unsigned)(((W + TILE - 1) / TILE) * ((H + TILE - 1) / TILE)), (unsigned)((Cout + OB - 1) / OB),
                (unsigned)B);
}

}  // namespace

extern "C" {

mt_status mt_sg_conv3x3_forward(const void* in, const void* w, const float* bias, void* out_bf16, float* out_f32,
                                int B, int Cin, int Cout, int H, int W, int relu, void* stream) {
    return run([&] {
        check_shape(B, Cin, Cout, H, W);
        if (!in || !w || (!out_bf16 && !out_f32)) mtb::fail(MT_ERR_INVALID_ARG, "NULL tensor");
        conv3x3_kernel<false><<<conv_grid(B, Cout, H, W), dim3(TILE, TILE), 0, (cudaStream_t)stream>>>(
            (const __nv_bfloat16*)in, (const __nv_bfloat16*)w, bias, nullptr, (__nv_bfloat16*)out_bf16, out_f32, B, Cin,
            Cout, H, W, relu);
        MTB_CUDA(cudaGetLastError());
    });
}

mt_status mt_sg_conv3x3_backward_data(const void* dout, const void* out_mask, const void* w, void* din, int B, int Cin,
                                      int Cout, int H, int W, void* stream) {
    return run([&] {
        check_shape(B, Cin, Cout, H, W);
        if (!dout || !w || !din) mtb::fail(MT_ERR_INVALID_ARG, "NULL tensor");
        // the data gradient is a convolution from Cout "input" channels to Cin outputs
        conv3x3_kernel<true><<<conv_grid(B, Cin, H, W), dim3(TILE, TILE), 0, (cudaStream_t)stream>>>(
            (const __nv_bfloat16*)dout, (const __nv_bfloat16*)w, nullptr, (const __nv_bfloat16*)out_mask,
            (__nv_bfloat16*)din, nullptr, B, Cout, Cin, H, W, 0);
        MTB_CUDA(cudaGetLastError());
    });
}

mt_status mt_sg_conv3x3_backward_weight(const void* in, const void* dout, const void* out_mask, float* dw, float* db,
                                        int B, int Cin, int Cout, int H, int W, void* stream) {
    return run([&] {
        check_shape(B, Cin, Cout, H, W);
        if (!in || !dout || !dw || !db) mtb::fail(MT_ERR_INVALID_ARG, "NULL tensor");
        conv3x3_wgrad_kernel<<<(unsigned)(Cout * (Cin + 1)), 256, 0, (cudaStream_t)stream>>>(
            (const __nv_bfloat16*)in, (const __nv_bfloat16*)dout, (const __nv_bfloat16*)out_mask, dw, db, B, Cin, Cout,
            H, W);
        MTB_CUDA(cudaGetLastError());
    });
}

mt_status mt_sg_loss(const float* head, const void* x, const float* target, const float* scale, void* dhead,
                     float* terms, int B, int H, int W, float lambda, void* stream) {
    return run([&] {
        check_shape(B, 1, 2, H, W);
        if (!head || !x || !target || !dhead || !terms) mtb::fail(MT_ERR_INVALID_ARG, "NULL tensor");
        const int n = B * H * W;
        surrogate_loss_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
            head, (const __nv_bfloat16*)x, target, scale, (__nv_bfloat16*)dhead, terms, B, H * W, lambda);
        MTB_CUDA(cudaGetLastError());
    });
}

mt_status mt_sg_adam(float* w, void* w_bf16, const float* g, float* m, float* v, int n, float lr, float b1, float b2,
                     float eps, int step, void* stream) {
    return run([&] {
        if (n <= 0 || step <= 0) mtb::fail(MT_ERR_INVALID_ARG, "bad Adam arguments");
        const float c1 = 1.0f - std::pow(b1, (float)step), c2 = 1.0f - std::pow(b2, (float)step);
        adam_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(w, (__nv_bfloat16*)w_bf16, g, m, v, n, lr, b1, b2,
                                                                        eps, c1, c2);
        MTB_CUDA(cudaGetLastError());
    });
}

mt_status mt_sg_pool2(const void* in, void* out, int B, int C, int H, int W, float scale, void* stream) {
    return run([&] {
        check_shape(B, C, 1, H, W);
        if (H % 2 || W % 2) mtb::fail(MT_ERR_INVALID_ARG, "pooling needs even H and W");
        if (!in || !out) mtb::fail(MT_ERR_INVALID_ARG, "NULL tensor");
        const size_t n = (size_t)B * C * (H / 2) * (W / 2);
        pool2_kernel<<<elem_grid(n), 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)in, (__nv_bfloat16*)out, B * C,
                                                                     H, W, scale);
        MTB_CUDA(cudaGetLastError());
    });
}

mt_status mt_sg_upsample2(const void* in, void* out, int B, int C, int H, int W, float scale, void* stream) {
    return run([&] {
        check_shape(B, C, 1, 2 * H, 2 * W);
        if (!in || !out) mtb::fail(MT_ERR_INVALID_ARG, "NULL tensor");
        const size_t n = (size_t)B * C * (2 * H) * (2 * W);
        upsample2_kernel<<<elem_grid(n), 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)in, (__nv_bfloat16*)out,
                                                                         B * C, H, W, scale);
        MTB_CUDA(cudaGetLastError());
    });
}

mt_status mt_sg_add(const void* a, const void* b, void* out, long long n, void* stream) {
    return run([&] {
        if (n < 0 || (n > 0 && (!a || !b || !out))) mtb::fail(MT_ERR_INVALID_ARG, "bad add arguments");
        if (n == 0) return;
        add_kernel<<<elem_grid((size_t)n), 256, 0, (cudaStream_t)stream>>>(
            (const __nv_bfloat16*)a, (const __nv_bfloat16*)b, (__nv_bfloat16*)out, (size_t)n);
        MTB_CUDA(cudaGetLastError());
    });
}

mt_status mt_sg_to_bf16(const float* a, void* b, int n, void* stream) {
    return run([&] {
        if (n <= 0) return;
        to_bf16_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(a, (__nv_bfloat16*)b, n);
        MTB_CUDA(cudaGetLastError());
    });
}

}  // extern "C"
