// Device kernels of the multislice engine (sm_100a).
//
// Data layout in HBM follows the reference (column-major, element (iy, ix) at ix*ny + iy, real
// space fft-shifted the way Grid_2d::ind_col_pbc_shift stores the potential, src/types.cuh:2229).
// A probe wave between passes is kept "hybrid": Fourier transformed along y (contiguous lines)
// and real along x. One multislice step psi <- IFFT2[P * FFT2[T * psi]] is then two passes, each
// reading and writing the wave once:
//   rows  (contiguous y-lines): S <- F_y( T * F_y^-1 S )
//   cols  (strided x-lines)   : S <- F_x^-1( P * F_x S )
// because F = F_x F_y and the two 1-D transforms commute. The annular-detector sums of the
// reference's get_psi + sum_square_over_Det (src/wave_function.cuh:96-155) are taken inside the
// column pass right after the P multiply, where the registers hold FFT2(psi)/N.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>

#include "common.hpp"
#include "fft_core.cuh"
#include "kernels.cuh"

namespace mtb {

// Kernel launches issued by the calling thread (an engine runs on one host thread). A CUDA graph
// replay adds the launches it holds through add_launches.
static thread_local long long g_launches = 0;
long long launches_issued() { return g_launches; }
void note_launch() { g_launches++; }
void add_launches(long long n) { g_launches += n; }

void encode_tile_map(CUtensorMap* map, const float2* base, int nx, int ldy, int nprobe, int w, int boxr) {
    static const PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        MTB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn) fail(MT_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    // float32 [nprobe][nx][2*ldy]; box: 2w floats (w complex columns) x boxr rows x 1 probe
    const cuuint64_t dims[3] = {(cuuint64_t)2 * ldy, (cuuint64_t)nx, (cuuint64_t)nprobe};
    const cuuint64_t strides[2] = {(cuuint64_t)2 * ldy * sizeof(float), (cuuint64_t)2 * ldy * nx * sizeof(float)};
    const cuuint32_t box[3] = {(cuuint32_t)(2 * w), (cuuint32_t)boxr, 1};
    const cuuint32_t estride[3] = {1, 1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float2*>(base), dims, strides, box,
                              estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(MT_ERR_CUDA, "cuTensorMapEncodeTiled failed for the column-pass tile map");
}

// =============================================================================================
// Projected potential splat fused with the transmission function.
//
// Projected_Potential::operator() (src/projected_potential.cuh:127-156) evaluates, for every atom
// of a slice and every pixel of its footprint box (get_bn, src/cpu_fcns.hpp:1670-1684),
//   R2 = (ix*dRx + Rx_0 - x)^2 + (iy*dRy + Ry_0 - y)^2;  if R2 < R2_max:
//   V[ind_col_pbc_shift(ix, iy)] += occ * cubic(R2)   (eval_cubic_poly, src/cgpu_fcns.cuh:1498-1567)
// with an FP32 atomicAdd per contribution. Here one CTA owns a 64 x 32 tile of the stored
// (shifted) grid of one slice (8 pixels per thread, 8 rows apart), culls the slice's atoms against
// its tile, and sums the contributions of the surviving atoms in atom order in registers
// (deterministic, no atomics; the tile size changes no sum).
// The epilogue writes T = exp(i*w*V) (functor::transmission_function, src/cgpu_fcns.cuh:3072-3086)
// directly; V never goes to HBM unless asked for. Float products and sums use the _rn intrinsics
// so they are not fused into FMAs and round like the reference's host float path.
// =============================================================================================
constexpr int SPLAT_TX = 64;   // tile extent along x (slow index)
constexpr int SPLAT_PX = SPLAT_TX / 8;  // pixels per thread along x
constexpr int SPLAT_TY = 32;   // tile extent along y (contiguous index)
constexpr int SPLAT_THREADS = 256;
constexpr int SPLAT_MAXT_SMEM = 8;

__device__ __forceinline__ int pmod(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

struct AtomFoot {
    float x, y, occ;
    int type;
    int ix0, nxa, iy0, nya;
    int sx, sy;  // first footprint pixel in stored (shifted) coordinates
};

__global__ void __launch_bounds__(SPLAT_THREADS) splat_kernel(SplatArgs a, int islice_0) {
    extern __shared__ float sm_tab[];
    __shared__ AtomFoot s_list[SPLAT_THREADS];
    __shared__ int s_warp_cnt[SPLAT_THREADS / 32];
    __shared__ int s_n;

    const int nR = a.nR;
    const int ntab = (a.n_types <= SPLAT_MAXT_SMEM) ? a.n_types : 0;
    for (int i = threadIdx.x; i < ntab * 5 * nR; i += blockDim.x) sm_tab[i] = a.tab[i];
    const float* tab = (ntab > 0) ? sm_tab : a.tab;

    const GridDev g = a.g;
    const int islice = islice_0 + blockIdx.z;
    const int tx0 = blockIdx.y * SPLAT_TX;
    const int ty0 = blockIdx.x * SPLAT_TY;
    const int ly = threadIdx.x % SPLAT_TY;
    const int lx = threadIdx.x / SPLAT_TY;  // 0..7: this thread's pixels are tx0 + lx + 8p
    const int jy = ty0 + ly;
    float V[SPLAT_PX];
#pragma unroll
    for (int p = 0; p < SPLAT_PX; p++) V[p] = 0.0f;

    const int2 rng = a.slice_range[islice];
    __syncthreads();
    for (int c0 = rng.x; c0 <= rng.y; c0 += SPLAT_THREADS) {
        const int ia = c0 + threadIdx.x;
        AtomFoot f;
        bool hit = false;
        if (ia <= rng.y) {
            float4 at = a.atoms[ia];
            f.x = at.x;
            f.y = at.y;
            f.occ = at.z;
            f.type = __float_as_int(at.w);
            const float Rm = a.R_max[f.type];
            // get_bn (src/cpu_fcns.hpp:1670-1684), periodic
            int i0 = (int)floorf(__fdiv_rn(__fsub_rn(f.x, Rm), g.dRx));
            int ie = (int)ceilf(__fdiv_rn(__fadd_rn(f.x, Rm), g.dRx));
            f.ix0 = i0;
            f.nxa = (i0 == ie) ? 0 : ie - i0 + 1;
            i0 = (int)floorf(__fdiv_rn(__fsub_rn(f.y, Rm), g.dRy));
            ie = (int)ceilf(__fdiv_rn(__fadd_rn(f.y, Rm), g.dRy));
            f.iy0 = i0;
            f.nya = (i0 == ie) ? 0 : ie - i0 + 1;
            f.sx = (pmod(f.ix0, g.nx) + g.nxh) % g.nx;
            f.sy = (pmod(f.iy0, g.ny) + g.nyh) % g.ny;
            // circular overlap of [sx, sx+nxa) with [tx0, tx0+TX) (and y)
            bool ox = (f.nxa >= g.nx) || (pmod(tx0 - f.sx, g.nx) < f.nxa) || (pmod(f.sx - tx0, g.nx) < SPLAT_TX);
            bool oy = (f.nya >= g.ny) || (pmod(ty0 - f.sy, g.ny) < f.nya) || (pmod(f.sy - ty0, g.ny) < SPLAT_TY);
            hit = ox && oy && f.nxa > 0 && f.nya > 0;
        }
        // deterministic compaction in atom order
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane == 0) s_warp_cnt[warp] = __popc(m);
        __syncthreads();
        if (threadIdx.x == 0) {
            int acc = 0;
            for (int w = 0; w < SPLAT_THREADS / 32; w++) {
                int cnt = s_warp_cnt[w];
                s_warp_cnt[w] = acc;
                acc += cnt;
            }
            s_n = acc;
        }
        __syncthreads();
        if (hit) s_list[s_warp_cnt[warp] + __popc(m & ((1u << lane) - 1u))] = f;
        __syncthreads();
        const int n = s_n;
        for (int k = 0; k < n; k++) {
            const AtomFoot af = s_list[k];
            const float* T = tab + (size_t)af.type * 5 * nR;
            const float Rm = a.R_max[af.type];
            const float R2_max = __fmul_rn(Rm, Rm);
            // knot index guess: the knots are log-spaced in R, so log2(R^2) is linear in the index
            const float lg0 = __log2f(T[0]);
            const float lgs = (float)(nR - 1) / (__log2f(T[nR - 1]) - lg0);
            // y offset, shared by every pixel of this thread (jy and sy are both in [0, ny))
            int offy = jy - af.sy;
            if (offy < 0) offy += g.ny;
#pragma unroll
            for (int p = 0; p < SPLAT_PX; p++) {
                const int jx = tx0 + lx + 8 * p;
                int offx = jx - af.sx;
                if (offx < 0) offx += g.nx;
                for (int ox = offx; ox < af.nxa; ox += g.nx) {
                    const int ix = af.ix0 + ox;
                    const float Rx = __fsub_rn(__fadd_rn(__fmul_rn((float)ix, g.dRx), g.Rx_0), af.x);
                    for (int oy = offy; oy < af.nya; oy += g.ny) {
                        const int iy = af.iy0 + oy;
                        const float Ry = __fsub_rn(__fadd_rn(__fmul_rn((float)iy, g.dRy), g.Ry_0), af.y);
                        const float R2 = __fadd_rn(__fmul_rn(Rx, Rx), __fmul_rn(Ry, Ry));
                        if (R2 < R2_max) {
                            // the interval of unrolledBinarySearch_c_nR (src/cgpu_fcns.cuh:1498-1518):
                            // the largest i0 in [0, nR-2] with T[i0] <= R2 (0 below the first knot),
                            // from the logarithmic guess and exact comparisons with the knots
                            int i0 = (int)fminf(fmaxf(__fmul_rn(__log2f(R2) - lg0, lgs), 0.0f), (float)(nR - 2));
                            while (i0 > 0 && R2 < T[i0]) i0--;
                            while (i0 < nR - 2 && !(R2 < T[i0 + 1])) i0++;
                            const float dx = __fsub_rn(R2, T[i0]);
                            const float c3 = T[4 * nR + i0], c2 = T[3 * nR + i0], c1 = T[2 * nR + i0], c0v = T[nR + i0];
                            float v = __fadd_rn(__fmul_rn(c3, dx), c2);
                            v = __fadd_rn(__fmul_rn(v, dx), c1);
                            v = __fadd_rn(__fmul_rn(v, dx), c0v);
                            v = __fmul_rn(af.occ, v);
                            V[p] += v;
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
    const size_t base = (size_t)islice * g.nx * g.ny;
#pragma unroll
    for (int p = 0; p < SPLAT_PX; p++) {
        const int jx = tx0 + lx + 8 * p;
        const size_t idx = base + (size_t)jx * g.ny + jy;
        if (a.V) a.V[idx] = V[p];
        if (a.trans) {
            const float th = __fmul_rn(a.w, V[p]);
            float sn, cs;
            if (a.wpo) {
                cs = 1.0f;
                sn = th;
            } else {
                sincosf(th, &sn, &cs);
            }
            a.trans[idx] = make_float2(cs, sn);
        }
    }
}

void launch_splat(const SplatArgs& a, int islice_0, int n_slice, cudaStream_t s) {
    if (a.g.nx % SPLAT_TX || a.g.ny % SPLAT_TY) fail(MT_ERR_UNSUPPORTED, "grid must be a multiple of 64 x 32");
    dim3 grid(a.g.ny / SPLAT_TY, a.g.nx / SPLAT_TX, n_slice);
    size_t sm = (a.n_types <= SPLAT_MAXT_SMEM) ? (size_t)a.n_types * 5 * a.nR * sizeof(float) : 0;
    splat_kernel<<<grid, SPLAT_THREADS, sm, s>>>(a, islice_0);
    g_launches++;
    MTB_CUDA(cudaGetLastError());
}

// =============================================================================================
// Line passes
// =============================================================================================
template <int NY>
void rows_dispatch_mode(RowMode mode, const RowArgs& a, int grid_ctas, cudaStream_t s);
template <int NX>
void cols_dispatch_flags(int flags, const ColArgs& a, int grid_ctas, cudaStream_t s);

template <int N>
constexpr int lines_per_cta() {
    return LinePlan<N>::T / (N / LinePlan<N>::E);
}

static int lines_per_cta(int n) {
    switch (n) {
        case 64: return lines_per_cta<64>();
        case 128: return lines_per_cta<128>();
        case 256: return lines_per_cta<256>();
        case 384: return lines_per_cta<384>();
        case 512: return lines_per_cta<512>();
        case 1024: return lines_per_cta<1024>();
        case 2048: return lines_per_cta<2048>();
        default: fail(MT_ERR_UNSUPPORTED, "grid sizes must be one of 64, 128, 256, 384, 512, 1024, 2048");
    }
    return 0;
}

template <int NX>
int cols_det_width();

int col_det_width(int nx) {
    switch (nx) {
        case 64: return cols_det_width<64>();
        case 128: return cols_det_width<128>();
        case 256: return cols_det_width<256>();
        case 384: return cols_det_width<384>();
        case 512: return cols_det_width<512>();
        case 1024: return cols_det_width<1024>();
        case 2048: return cols_det_width<2048>();
        default: fail(MT_ERR_UNSUPPORTED, "nx must be one of 64, 128, 256, 384, 512, 1024, 2048");
    }
    return 0;
}

int col_tiles(int nx, int ny) {
    const int w = col_det_width(nx);
    if (ny % w != 0) fail(MT_ERR_UNSUPPORTED, "ny must be a multiple of the column-pass tile width");
    return ny / w;
}

void launch_rows(int ny, RowMode mode, const RowArgs& a, int grid_ctas, cudaStream_t s) {
    if (a.nx % lines_per_cta(ny) != 0) fail(MT_ERR_UNSUPPORTED, "nx must be a multiple of the row-pass line group");
    switch (ny) {
        case 64: rows_dispatch_mode<64>(mode, a, grid_ctas, s); break;
        case 128: rows_dispatch_mode<128>(mode, a, grid_ctas, s); break;
        case 256: rows_dispatch_mode<256>(mode, a, grid_ctas, s); break;
        case 384: rows_dispatch_mode<384>(mode, a, grid_ctas, s); break;
        case 512: rows_dispatch_mode<512>(mode, a, grid_ctas, s); break;
        case 1024: rows_dispatch_mode<1024>(mode, a, grid_ctas, s); break;
        case 2048: rows_dispatch_mode<2048>(mode, a, grid_ctas, s); break;
        default: fail(MT_ERR_UNSUPPORTED, "ny must be one of 64, 128, 256, 384, 512, 1024, 2048");
    }
}

void launch_cols(int nx, int flags, const ColArgs& a, int grid_ctas, cudaStream_t s) {
    if (a.ny % lines_per_cta(nx) != 0) fail(MT_ERR_UNSUPPORTED, "ny must be a multiple of the column-pass tile width");
    switch (nx) {
        case 64: cols_dispatch_flags<64>(flags, a, grid_ctas, s); break;
        case 128: cols_dispatch_flags<128>(flags, a, grid_ctas, s); break;
        case 256: cols_dispatch_flags<256>(flags, a, grid_ctas, s); break;
        case 384: cols_dispatch_flags<384>(flags, a, grid_ctas, s); break;
        case 512: cols_dispatch_flags<512>(flags, a, grid_ctas, s); break;
        case 1024: cols_dispatch_flags<1024>(flags, a, grid_ctas, s); break;
        case 2048: cols_dispatch_flags<2048>(flags, a, grid_ctas, s); break;
        default: fail(MT_ERR_UNSUPPORTED, "nx must be one of 64, 128, 256, 384, 512, 1024, 2048");
    }
}

// =============================================================================================
// Detector reduction: one thread per (probe, detector); tiles summed in order (deterministic).
__global__ void det_reduce_kernel(const double* __restrict__ partial, int nprobe, int n_tiles, int n_det,
                                  const int* __restrict__ scan_index, double w, double* __restrict__ image,
                                  int n_scan) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nprobe * n_det) return;
    const int b = i / n_det, d = i % n_det;
    double s = 0.0;
    for (int k = 0; k < n_tiles; k++) s += partial[((size_t)b * n_tiles + k) * n_det + d];
    image[(size_t)d * n_scan + scan_index[b]] += w * s;
}

void launch_det_reduce(const double* partial, int nprobe, int n_tiles, int n_det, const int* scan_index, double w,
                       double* image, int n_scan, cudaStream_t s) {
    const int n = nprobe * n_det;
    det_reduce_kernel<<<(n + 127) / 128, 128, 0, s>>>(partial, nprobe, n_tiles, n_det, scan_index, w, image, n_scan);
    g_launches++;
    MTB_CUDA(cudaGetLastError());
}

// =============================================================================================
__global__ void tilt_ramp_kernel(GridDev g, float gx, float gy, float rxc, float ryc, float2* __restrict__ out) {
    const int iy = blockIdx.x * blockDim.x + threadIdx.x, ix = blockIdx.y;
    if (iy >= g.ny) return;
    const float rx = __fsub_rn(__fadd_rn(__fmul_rn((float)((ix < g.nxh) ? ix + g.nxh : ix - g.nxh), g.dRx), g.Rx_0), rxc);
    const float ry = __fsub_rn(__fadd_rn(__fmul_rn((float)((iy < g.nyh) ? iy + g.nyh : iy - g.nyh), g.dRy), g.Ry_0), ryc);
    const double th = (double)__fadd_rn(__fmul_rn(gx, rx), __fmul_rn(gy, ry));
    double sn, cs;
    sincos(th, &sn, &cs);
    const double s = 1.0 / (double)g.ny;
    out[(size_t)ix * g.ny + iy] = make_float2((float)(cs * s), (float)(sn * s));
}

void launch_tilt_ramp(const GridDev& g, float gx, float gy, float rxc, float ryc, float2* out, cudaStream_t s) {
    tilt_ramp_kernel<<<dim3((unsigned)((g.ny + 127) / 128), (unsigned)g.nx), 128, 0, s>>>(g, gx, gy, rxc, ryc, out);
    g_launches++;
    MTB_CUDA(cudaGetLastError());
}

__global__ void mul_tables_kernel(float2* __restrict__ a, const float2* __restrict__ b, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        a[i] = cmul(a[i], b[i]);
}

void launch_mul_tables(float2* a, const float2* b, size_t n, cudaStream_t s) {
    mul_tables_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 8), 256, 0, s>>>(a, b, n);
    g_launches++;
    MTB_CUDA(cudaGetLastError());
}

__global__ void sum_waves_kernel(const float2* __restrict__ src, int n, size_t nxy, float2* __restrict__ dst) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nxy; i += (size_t)gridDim.x * blockDim.x) {
        float2 acc = src[i];
        for (int j = 1; j < n; j++) {
            const float2 v = src[(size_t)j * nxy + i];
            acc = make_float2(__fadd_rn(acc.x, v.x), __fadd_rn(acc.y, v.y));
        }
        dst[i] = acc;
    }
}

// dst += w * src over nxy complex values (add_scale, src/output_multislice.hpp:770-780)
__global__ void axpy_wave_kernel(const float2* __restrict__ src, float w, size_t nxy, float2* __restrict__ dst) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nxy; i += (size_t)gridDim.x * blockDim.x) {
        const float2 v = src[i], d = dst[i];
        dst[i] = make_float2(__fadd_rn(d.x, __fmul_rn(w, v.x)), __fadd_rn(d.y, __fmul_rn(w, v.y)));
    }
}

void launch_axpy_wave(const float2* src, float w, size_t nxy, float2* dst, cudaStream_t s) {
    axpy_wave_kernel<<<(unsigned)std::min<size_t>((nxy + 255) / 256, 148 * 8), 256, 0, s>>>(src, w, nxy, dst);
    g_launches++;
    MTB_CUDA(cudaGetLastError());
}

void launch_sum_waves(const float2* src, int n, size_t nxy, float2* dst, cudaStream_t s) {
    sum_waves_kernel<<<(unsigned)std::min<size_t>((nxy + 255) / 256, 148 * 8), 256, 0, s>>>(src, n, nxy, dst);
    g_launches++;
    MTB_CUDA(cudaGetLastError());
}

// One CTA per (thickness, scan position): detector sums of |psi_coh|^2 over the grid, per-thread
// partials in FP64 reduced in a fixed order.
__global__ void coh_detect_kernel(const float2* __restrict__ coh, int n_scan, ColArgs a, double* __restrict__ image) {
    const int ithk = blockIdx.x / n_scan, iscan = blockIdx.x % n_scan;
    const size_t nxy = (size_t)a.g.nx * a.g.ny;
    const float2* c = coh + ((size_t)ithk * n_scan + iscan) * nxy;
    double acc[kMaxDet];
#pragma unroll
    for (int d = 0; d < kMaxDet; d++) acc[d] = 0.0;
    for (size_t p = threadIdx.x; p < nxy; p += blockDim.x) {
        const int ix = (int)(p / a.g.ny), iy = (int)(p % a.g.ny);
        const float2 v = c[p];
        const float v2 = __fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y));
        if (a.det_mat) {
#pragma unroll
            for (int d = 0; d < kMaxDet; d++)
                if (d < a.n_det) acc[d] += (double)__fmul_rn(a.det_mat[d * nxy + p], v2);
        } else {
            const float gx = __fmul_rn((float)((ix < a.g.nxh) ? ix : ix - a.g.nx), a.g.dgx);
            const float gy = __fmul_rn((float)((iy < a.g.nyh) ? iy : iy - a.g.ny), a.g.dgy);
            const float g2 = __fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy));
#pragma unroll
            for (int d = 0; d < kMaxDet; d++)
                if (d < a.n_det && a.det_g2_min[d] <= g2 && g2 < a.det_g2_max[d]) acc[d] += (double)v2;
        }
    }
    __shared__ double red[kMaxDet][256];
#pragma unroll
    for (int d = 0; d < kMaxDet; d++) red[d][threadIdx.x] = acc[d];
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
#pragma unroll
            for (int d = 0; d < kMaxDet; d++) red[d][threadIdx.x] += red[d][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < (unsigned)a.n_det)
        image[((size_t)ithk * a.n_det + threadIdx.x) * n_scan + iscan] = red[threadIdx.x][0];
}

void launch_coh_detect(const float2* coh, int n_thk, int n_scan, const ColArgs& det, double* image_coh,
                       cudaStream_t s) {
    coh_detect_kernel<<<(unsigned)(n_thk * n_scan), 256, 0, s>>>(coh, n_scan, det, image_coh);
    g_launches++;
    MTB_CUDA(cudaGetLastError());
}

// EW output accumulation with fft-shift and crop (add_scale_crop_shift_2d /
// add_scale_square_crop_shift_2d / assign_crop_shift_2d, src/cgpu_fcns.cuh:1681-1780).
__global__ void ew_accumulate_kernel(const float2* __restrict__ psi, int nx, int ny, int ix0, int ix1, int iy0,
                                     int iy1, double w, int assign, double* __restrict__ psi_out,
                                     double* __restrict__ m2_out, int nwave) {
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    const int ix = blockIdx.y;
    if (iy >= ny || ix >= nx) return;
    if (ix < ix0 || ix >= ix1 || iy < iy0 || iy >= iy1) return;
    // output pixel (ix, iy) takes the stored pixel shifted by half the grid
    const int sx = (ix + nx / 2) % nx, sy = (iy + ny / 2) % ny;
    const float2 v = psi[(size_t)sx * ny + sy];
    const size_t o = (size_t)(ix - ix0) * (iy1 - iy0) + (iy - iy0);
    if (psi_out) {
        if (assign) {
            psi_out[2 * o] = v.x;
            psi_out[2 * o + 1] = v.y;
        } else {
            psi_out[2 * o] += w * v.x;
            psi_out[2 * o + 1] += w * v.y;
        }
    }
    if (m2_out) {
        double acc = 0.0;
        for (int j = 0; j < nwave; j++) {
            const float2 u = (j == 0) ? v : psi[(size_t)j * nx * ny + (size_t)sx * ny + sy];
            const float n2 = __fadd_rn(__fmul_rn(u.x, u.x), __fmul_rn(u.y, u.y));
            acc += w * (double)n2;
        }
        m2_out[o] += acc;
    }
}

void launch_ew_accumulate(const float2* psi, int nx, int ny, int ix0, int ix1, int iy0, int iy1, double w,
                          int assign, double* psi_out, double* m2_out, cudaStream_t s, int nwave) {
    dim3 grid((ny + 127) / 128, nx);
    ew_accumulate_kernel<<<grid, 128, 0, s>>>(psi, nx, ny, ix0, ix1, iy0, iy1, w, assign, psi_out, m2_out, nwave);
    g_launches++;
    MTB_CUDA(cudaGetLastError());
}

}  // namespace mtb
