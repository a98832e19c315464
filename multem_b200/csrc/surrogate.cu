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
//
// The three convolutions run on the tensor cores as GEMMs (umma_gemm.cuh), with k = c*9 + ky*3 + kx
// and pixels p = (b, y, x):
//   forward      C[p][o]   = A[p][k] . Wf[o][k],      A = im2col(in),     Wf[o][k] = w[o][k]
//   data grad    C[p][i]   = A'[p][k'] . Wd[i][k'],   A' = im2col(dout'), Wd[i][o*9+q] = w[o][i][8-q]
//   weight grad  C[k][o]   = X[k][p] . Y[o][p],       X = im2col(in) transposed plus a row of ones
//                                                     (its C row is the bias gradient), Y = dout'
// The operand layouts are written by small gather kernels into a per-device workspace; the GEMM
// writes FP32 partial sums per K split, and a finalize kernel adds them in split order (fixed-order
// reductions: deterministic results), applies bias and ReLU and writes the NCHW (or [o][k]) result.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>

#include "common.hpp"
#include "devmem.hpp"
#include "multem_b200_surrogate.h"
#include "umma_gemm.cuh"

namespace {

__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }

// ---------------------------------------------------------------------------------------------
// GEMM operand layouts

// A[m][k] = in[b][c][y+ky-1][x+kx-1] for k = c*9 + ky*3 + kx < 9*C (zero outside the image and for
// the padding k in [9C, ldk)); with `mask`, zero where mask (same layout as in) is not positive.
// Thread (m, chunk) gathers the 8 values k = 8*chunk .. 8*chunk+7 of pixel m with independent loads
// (the 32 lanes of a warp take 32 consecutive pixels: each load is contiguous across the warp) and
// stores them as one 16-byte vector. grid: (ceil(M/32), ceil(ldk/64)), block 32 x 8.
__global__ void __launch_bounds__(256) im2col_kernel(const __nv_bfloat16* __restrict__ in,
                                                     const __nv_bfloat16* __restrict__ mask,
                                                     __nv_bfloat16* __restrict__ A, int B, int C, int H, int W,
                                                     int ldk) {
    const int HW = H * W, M = B * HW, K = 9 * C;
    const int m = blockIdx.x * 32 + threadIdx.x;
    const int k0 = blockIdx.y * 64 + threadIdx.y * 8;
    if (m >= M || k0 >= ldk) return;  // ldk and k0 are multiples of 8: the 8 values stay in the row
    const int b = m / HW, yx = m - b * HW, y = yx / W, x = yx - y * W;
    __align__(16) __nv_bfloat16 v8[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int k = k0 + j;
        __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
        if (k < K) {
            const int c = k / 9, q = k - 9 * c;
            const int yy = y + q / 3 - 1, xx = x + q % 3 - 1;
            if (yy >= 0 && yy < H && xx >= 0 && xx < W) {
                const size_t idx = (((size_t)b * C + c) * H + yy) * W + xx;
                v = in[idx];
                if (mask && !(bf(mask[idx]) > 0.0f)) v = __float2bfloat16_rn(0.0f);
            }
        }
        v8[j] = v;
    }
    *reinterpret_cast<uint4*>(A + (size_t)m * ldk + k0) = *reinterpret_cast<const uint4*>(v8);
}

// X[k][p] = in[b][c][y+ky-1][x+kx-1] (the transposed im2col, p = (b, y, x)) for k = c*9 + q < 9C,
// X[9C][p] = 1, zero for the padding p in [B*H*W, ldp). grid: (ceil(ldp/256), C + 1); the CTA row
// c writes the nine rows of channel c (the last CTA row the row of ones), consecutive threads
// consecutive pixels.
__global__ void __launch_bounds__(256) im2col_t_kernel(const __nv_bfloat16* __restrict__ in,
                                                       __nv_bfloat16* __restrict__ X, int B, int C, int H, int W,
                                                       int ldp) {
    const int HW = H * W, P = B * HW;
    const int c = blockIdx.y;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < ldp; p += gridDim.x * blockDim.x) {
        if (c == C) {
            X[(size_t)9 * C * ldp + p] = __float2bfloat16_rn(p < P ? 1.0f : 0.0f);
            continue;
        }
        int b = 0, y = 0, x = 0;
        if (p < P) {
            b = p / HW;
            const int yx = p - b * HW;
            y = yx / W;
            x = yx - y * W;
        }
        const __nv_bfloat16* plane = in + ((size_t)b * C + c) * HW;
#pragma unroll
        for (int q = 0; q < 9; q++) {
            const int yy = y + q / 3 - 1, xx = x + q % 3 - 1;
            const float v = (p < P && yy >= 0 && yy < H && xx >= 0 && xx < W) ? bf(plane[yy * W + xx]) : 0.0f;
            X[(size_t)(9 * c + q) * ldp + p] = __float2bfloat16_rn(v);
        }
    }
}

// Y[c][p] = d[b][c][y][x] (channel-major, p = (b, y, x)), zero where mask is not positive and for
// the padding p in [B*HW, ldp). grid: (ceil(ldp/256), C).
__global__ void __launch_bounds__(256) channel_major_kernel(const __nv_bfloat16* __restrict__ d,
                                                            const __nv_bfloat16* __restrict__ mask,
                                                            __nv_bfloat16* __restrict__ Y, int B, int C, int HW,
                                                            int ldp) {
    const int P = B * HW, c = blockIdx.y;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < ldp; p += gridDim.x * blockDim.x) {
        __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
        if (p < P) {
            const int b = p / HW;
            const size_t idx = ((size_t)b * C + c) * HW + (p - b * HW);
            v = d[idx];
            if (mask && !(bf(mask[idx]) > 0.0f)) v = __float2bfloat16_rn(0.0f);
        }
        Y[(size_t)c * ldp + p] = v;
    }
}

// Weights as the GEMM's B operand [rows][ldk]: forward Wf[o][k] = w[o][k] (k < 9*Cin); data
// gradient Wd[i][o*9 + q] = w[o][i][8 - q] (k < 9*Cout, the kernel flipped); zero padding.
__global__ void pack_weights_kernel(const __nv_bfloat16* __restrict__ w, __nv_bfloat16* __restrict__ Bm, int Cout,
                                    int Cin, int ldk, int data_grad) {
    const int rows = data_grad ? Cin : Cout, K = data_grad ? 9 * Cout : 9 * Cin;
    const size_t n = (size_t)rows * ldk;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(e % ldk), r = (int)(e / ldk);
        __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
        if (k < K) v = data_grad ? w[((size_t)(k / 9) * Cin + r) * 9 + (8 - k % 9)] : w[(size_t)r * K + k];
        Bm[e] = v;
    }
}

// out[(m / mdiv) * s_mq + (m % mdiv) * s_mr + n * s_n] = act(bias[n] + sum over splits s, in order,
// of part[s][row0 + m][n]) for m < M, n < N; n runs fastest over the threads, so the reads of the
// partial sums (splits times the output) are contiguous.
__global__ void gemm_finalize_kernel(const float* __restrict__ part, int splits, int Mtot, int N, int row0, int M,
                                     const float* __restrict__ bias, int relu, __nv_bfloat16* __restrict__ out_bf,
                                     float* __restrict__ out_f, long long mdiv, long long s_mq, long long s_mr,
                                     long long s_n) {
    const size_t n_all = (size_t)M * N;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n_all; e += (size_t)gridDim.x * blockDim.x) {
        const int n = (int)(e % N), m = (int)(e / N);
        float acc = 0.0f;
        for (int s = 0; s < splits; s++) acc += part[((size_t)s * Mtot + row0 + m) * N + n];
        float v = acc + (bias ? bias[n] : 0.0f);
        if (relu) v = fmaxf(v, 0.0f);
        const long long idx = (m / mdiv) * s_mq + (m % mdiv) * s_mr + n * s_n;
        if (out_bf) out_bf[idx] = __float2bfloat16_rn(v);
        if (out_f) out_f[idx] = v;
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

constexpr long long kWaitNs = 1000000000ll;  // bound of every wait of the GEMM (1 s)

size_t align256(size_t v) { return (v + 255) / 256 * 256; }
int round8(int v) { return (v + 7) / 8 * 8; }

// Per-device workspace of the convolutions (GEMM operands and partial sums), grown on demand from
// the library's pool, and the error flag of the GEMM's bounded waits. Calls on one device share
// them, so they must be issued on one stream (or otherwise ordered), as the surrogate's host code
// does.
struct Workspace {
    unsigned char* p = nullptr;
    size_t bytes = 0;
    int* err = nullptr;
    int dev = 0;
};
std::mutex g_ws_mu;
std::map<int, Workspace> g_ws;

Workspace& workspace(size_t bytes) {
    int dev = 0;
    MTB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_ws_mu);
    Workspace& w = g_ws[dev];
    if (!w.err) {
        w.err = static_cast<int*>(mtb::dev_alloc(256, &w.dev));
        MTB_CUDA(cudaMemset(w.err, 0, sizeof(int)));
    }
    if (w.bytes < bytes) {
        const size_t nb = std::max(bytes, 2 * w.bytes);  // grow geometrically
        if (w.p) mtb::dev_free(w.p, w.dev);  // waits for the device: earlier calls may still use it
        w.p = nullptr;
        w.bytes = 0;
        w.p = static_cast<unsigned char*>(mtb::dev_alloc(nb, &w.dev));
        w.bytes = nb;
    }
    return w;
}

// Tensor map of a bf16 [rows][ld] K-major operand: boxes of 64 k x box_rows rows with the 128-byte
// swizzle (the canonical layout of the MMA's shared-memory descriptors); out-of-bounds reads are 0.
void encode_kmajor(CUtensorMap* map, const void* base, int rows, int ld, int box_rows) {
    static const PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        MTB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn) mtb::fail(MT_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    const cuuint64_t dims[2] = {(cuuint64_t)ld, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)mtb::umma::BK, (cuuint32_t)box_rows};
    const cuuint32_t estride[2] = {1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box,
                              estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) mtb::fail(MT_ERR_CUDA, "cuTensorMapEncodeTiled failed for a GEMM operand");
}

int gemm_bn(int N) { return N <= 16 ? 16 : N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256; }

// K split of an M x N x K product: enough CTAs to cover the SMs twice when the tiles alone do not,
// at least two K blocks per split.
void gemm_split(int M, int N, int K, int* splits, int* kb_per_split) {
    const int nkb = (K + mtb::umma::BK - 1) / mtb::umma::BK;
    const int bn = gemm_bn(N);
    const int tiles = ((M + mtb::umma::BM - 1) / mtb::umma::BM) * ((N + bn - 1) / bn);
    int want = tiles >= 296 ? 1 : (296 + tiles - 1) / tiles;
    int kps = std::max(2, (nkb + want - 1) / want);
    if (kps > nkb) kps = nkb;
    *kb_per_split = kps;
    *splits = (nkb + kps - 1) / kps;
}

template <int BN>
void gemm_launch(const CUtensorMap& ma, const CUtensorMap& mb, const mtb::umma::GemmOut& out, int M, int N, int nkb,
                 int splits, int kps, int* err, cudaStream_t st) {
    using T = mtb::umma::Tile<BN>;
    auto kern = mtb::umma::gemm_kernel<BN>;
    MTB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM));
    // resident CTAs per SM are bounded by shared memory; their tensor-memory columns must fit the
    // SM's 512, or an allocation would wait for another CTA to exit
    int occ = 0;
    MTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 128, T::SMEM));
    if (occ < 1 || occ * T::TCOLS > 512) mtb::fail(MT_ERR_INTERNAL, "GEMM tile does not fit an SM's tensor memory");
    const dim3 grid((unsigned)((M + mtb::umma::BM - 1) / mtb::umma::BM), (unsigned)splits, (unsigned)((N + BN - 1) / BN));
    kern<<<grid, 128, T::SMEM, st>>>(ma, mb, out, M, N, nkb, kps, err, kWaitNs);
    MTB_CUDA(cudaGetLastError());
}

// A[M][lda] . B[N][ldb]^T over the first K columns (bf16): the partial sums of each split, or the
// finished result with one split (mtb::umma::GemmOut).
void gemm(const __nv_bfloat16* A, int M, int lda, const __nv_bfloat16* Bm, int N, int ldb, int K,
          const mtb::umma::GemmOut& out, int splits, int kps, int* err, cudaStream_t st) {
    if (!out.part && splits != 1) mtb::fail(MT_ERR_INTERNAL, "a split-K product needs a partial-sum buffer");
    const int bn = gemm_bn(N);
    CUtensorMap ma, mb;
    encode_kmajor(&ma, A, M, lda, mtb::umma::BM);
    encode_kmajor(&mb, Bm, N, ldb, bn);
    const int nkb = (K + mtb::umma::BK - 1) / mtb::umma::BK;
    switch (bn) {
        case 16: gemm_launch<16>(ma, mb, out, M, N, nkb, splits, kps, err, st); break;
        case 32: gemm_launch<32>(ma, mb, out, M, N, nkb, splits, kps, err, st); break;
        case 64: gemm_launch<64>(ma, mb, out, M, N, nkb, splits, kps, err, st); break;
        case 128: gemm_launch<128>(ma, mb, out, M, N, nkb, splits, kps, err, st); break;
        default: gemm_launch<256>(ma, mb, out, M, N, nkb, splits, kps, err, st); break;
    }
}

void finalize(const float* part, int splits, int Mtot, int N, int row0, int M, const float* bias, int relu,
              __nv_bfloat16* out_bf, float* out_f, long long mdiv, long long s_mq, long long s_mr, long long s_n,
              cudaStream_t st) {
    gemm_finalize_kernel<<<elem_grid((size_t)M * N), 256, 0, st>>>(part, splits, Mtot, N, row0, M, bias, relu, out_bf,
                                                                  out_f, mdiv, s_mq, s_mr, s_n);
    MTB_CUDA(cudaGetLastError());
}

// out (NCHW, Cout channels) = conv of `in` (Cin channels, masked where given) with the forward
// or data-gradient weight layout.
void conv_as_gemm(const __nv_bfloat16* in, const __nv_bfloat16* mask, int Cin_eff, const __nv_bfloat16* w, int Cout,
                  int Cin, bool data_grad, const float* bias, int relu, __nv_bfloat16* out_bf, float* out_f, int B,
                  int H, int W, cudaStream_t st) {
    const int P = B * H * W, K = 9 * Cin_eff, ldk = round8(K);
    const int N = data_grad ? Cin : Cout;
    int splits = 1, kps = 1;
    gemm_split(P, N, K, &splits, &kps);
    const size_t offB = align256((size_t)P * ldk * 2), offP = offB + align256((size_t)N * ldk * 2);
    Workspace& ws = workspace(offP + (splits > 1 ? (size_t)splits * P * N * 4 : 0));
    auto* A = reinterpret_cast<__nv_bfloat16*>(ws.p);
    auto* Bm = reinterpret_cast<__nv_bfloat16*>(ws.p + offB);
    const dim3 ig((unsigned)((P + 31) / 32), (unsigned)((ldk + 63) / 64));
    im2col_kernel<<<ig, dim3(32, 8), 0, st>>>(in, mask, A, B, Cin_eff, H, W, ldk);
    MTB_CUDA(cudaGetLastError());
    pack_weights_kernel<<<elem_grid((size_t)N * ldk), 256, 0, st>>>(w, Bm, Cout, Cin, ldk, data_grad ? 1 : 0);
    MTB_CUDA(cudaGetLastError());
    const long long HW = (long long)H * W;
    mtb::umma::GemmOut o{};
    if (splits == 1) {  // the GEMM's epilogue writes the NCHW result itself
        o = {nullptr, bias, relu, out_bf, out_f, HW, (long long)N * HW, 1, HW};
        gemm(A, P, ldk, Bm, N, ldk, K, o, 1, kps, ws.err, st);
        return;
    }
    o.part = reinterpret_cast<float*>(ws.p + offP);
    gemm(A, P, ldk, Bm, N, ldk, K, o, splits, kps, ws.err, st);
    finalize(o.part, splits, P, N, 0, P, bias, relu, out_bf, out_f, HW, (long long)N * HW, 1, HW, st);
}

}  // namespace

extern "C" {

mt_status mt_sg_conv3x3_forward(const void* in, const void* w, const float* bias, void* out_bf16, float* out_f32,
                                int B, int Cin, int Cout, int H, int W, int relu, void* stream) {
    return run([&] {
        check_shape(B, Cin, Cout, H, W);
        if (!in || !w || (!out_bf16 && !out_f32)) mtb::fail(MT_ERR_INVALID_ARG, "NULL tensor");
        conv_as_gemm((const __nv_bfloat16*)in, nullptr, Cin, (const __nv_bfloat16*)w, Cout, Cin, false, bias, relu,
                     (__nv_bfloat16*)out_bf16, out_f32, B, H, W, (cudaStream_t)stream);
    });
}

mt_status mt_sg_conv3x3_backward_data(const void* dout, const void* out_mask, const void* w, void* din, int B, int Cin,
                                      int Cout, int H, int W, void* stream) {
    return run([&] {
        check_shape(B, Cin, Cout, H, W);
        if (!dout || !w || !din) mtb::fail(MT_ERR_INVALID_ARG, "NULL tensor");
        // the data gradient is a convolution of the masked output gradient (Cout channels) with the
        // flipped, transposed kernel
        conv_as_gemm((const __nv_bfloat16*)dout, (const __nv_bfloat16*)out_mask, Cout, (const __nv_bfloat16*)w, Cout,
                     Cin, true, nullptr, 0, (__nv_bfloat16*)din, nullptr, B, H, W, (cudaStream_t)stream);
    });
}

mt_status mt_sg_conv3x3_backward_weight(const void* in, const void* dout, const void* out_mask, float* dw, float* db,
                                        int B, int Cin, int Cout, int H, int W, void* stream) {
    return run([&] {
        check_shape(B, Cin, Cout, H, W);
        if (!in || !dout || !dw || !db) mtb::fail(MT_ERR_INVALID_ARG, "NULL tensor");
        const cudaStream_t st = (cudaStream_t)stream;
        const int HW = H * W, P = B * HW, ldp = round8(P), M = 9 * Cin + 1;
        int splits = 1, kps = 1;
        gemm_split(M, Cout, P, &splits, &kps);
        const size_t offY = align256((size_t)M * ldp * 2), offP = offY + align256((size_t)Cout * ldp * 2);
        Workspace& ws = workspace(offP + (size_t)splits * M * Cout * 4);
        auto* X = reinterpret_cast<__nv_bfloat16*>(ws.p);
        auto* Y = reinterpret_cast<__nv_bfloat16*>(ws.p + offY);
        auto* part = reinterpret_cast<float*>(ws.p + offP);
        const unsigned gx = (unsigned)std::min((ldp + 255) / 256, 1024);
        im2col_t_kernel<<<dim3(gx, (unsigned)(Cin + 1)), 256, 0, st>>>((const __nv_bfloat16*)in, X, B, Cin, H, W, ldp);
        MTB_CUDA(cudaGetLastError());
        channel_major_kernel<<<dim3(gx, (unsigned)Cout), 256, 0, st>>>(
            (const __nv_bfloat16*)dout, (const __nv_bfloat16*)out_mask, Y, B, Cout, HW, ldp);
        MTB_CUDA(cudaGetLastError());
        mtb::umma::GemmOut o{};
        o.part = part;
        gemm(X, M, ldp, Y, Cout, ldp, P, o, splits, kps, ws.err, st);
        // rows k < 9*Cin: dw[o][k]; row 9*Cin: db[o]
        finalize(part, splits, M, Cout, 0, M - 1, nullptr, 0, nullptr, dw, M - 1, 0, 1, M - 1, st);
        finalize(part, splits, M, Cout, M - 1, 1, nullptr, 0, nullptr, db, 1, 0, 0, 1, st);
    });
}

mt_status mt_sg_check(void* stream) {
    return run([&] {
        MTB_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
        int dev = 0;
        MTB_CUDA(cudaGetDevice(&dev));
        int* err = nullptr;
        {
            std::lock_guard<std::mutex> lk(g_ws_mu);
            auto it = g_ws.find(dev);
            if (it != g_ws.end()) err = it->second.err;
        }
        if (!err) return;
        int e = 0;
        MTB_CUDA(cudaMemcpy(&e, err, sizeof(int), cudaMemcpyDeviceToHost));
        if (e) {
            MTB_CUDA(cudaMemset(err, 0, sizeof(int)));
            mtb::fail(MT_ERR_TIMEOUT, "a tensor-core GEMM gave up waiting for its operands");
        }
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
