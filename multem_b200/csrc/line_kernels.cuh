// Line-pass kernels (contiguous y-lines and strided x-lines), templated on the line length.
// Each supported length is instantiated in its own translation unit (lines_<N>.cu) so the build
// parallelises; kernels.cu dispatches on the runtime size.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "common.hpp"
#include "fft_core.cuh"
#include "kernels.cuh"
#include "mbarrier.cuh"

namespace mtb {

void note_launch();

template <int N>
constexpr int min_radix() {
    int r = LinePlan<N>::R[0];
    for (int s = 1; s < LinePlan<N>::NS; s++) r = LinePlan<N>::R[s] < r ? LinePlan<N>::R[s] : r;
    return r;
}

template <int N>
struct LineGeom {
    static constexpr int E = LinePlan<N>::E;
    static constexpr int TPL = N / E;
    static constexpr int THREADS = LinePlan<N>::T;  // threads per CTA (per group when pipelined)
    static constexpr int LPC = THREADS / TPL;       // lines per CTA (per group)
    static constexpr int NSG = LinePlan<N>::NS;
    static constexpr int R1 = LinePlan<N>::R[0];
    static constexpr int RL = LinePlan<N>::R[NSG - 1];
    static constexpr int RMIN = min_radix<N>();
    static constexpr int LS = N + N / RMIN + 1;  // padded line buffer (float2); odd
    static constexpr int TW_I = TwTable<N, false, 0>::SIZE + TwTable<N, false, 1>::SIZE + (NSG > 2 ? TwTable<N, false, 2>::SIZE : 0);
    static constexpr int TW_F = TwTable<N, true, 0>::SIZE + TwTable<N, true, 1>::SIZE + (NSG > 2 ? TwTable<N, true, 2>::SIZE : 0);
};

// Line stride of the column passes' full exchange buffers. A warp's lanes hold W adjacent columns
// (lines) and 32/W consecutive line threads, and an 8-byte shared access is served one half-warp
// (16 lanes, one 128-byte wavefront) at a time: its 16 lanes hold W lines x 16/W threads. The
// exchanges address consecutive threads' points 1 mod 16 points apart, so the lines' starts must step
// by 16/W points mod 16 for a half-warp to hit the 16 8-byte bank slots once each. The padded line
// of LineGeom (1 mod 16) does that for W = 16; for 8-column tiles of 1024-point lines it conflicted
// 2-way per half-warp, for 4- and 2-column tiles up to 4-way.
template <int NX, int W>
constexpr int col_ls() {
    constexpr int base = LineGeom<NX>::LS;
    if constexpr (W > 8) {
        return base;
    } else {
        constexpr int r = (16 / W) % 16;
        return base + ((r - base % 16) % 16 + 16) % 16;
    }
}

template <int N>
__device__ __forceinline__ void setup_twiddles(float2* base, const float2** twI, const float2** twF) {
    constexpr int NSG = LinePlan<N>::NS;
    float2* p = base;
    static_for<0, NSG>([&](auto sc) {
        constexpr int s = decltype(sc)::value;
        twI[s] = p;
        fill_twiddles<N, false, s>(p, threadIdx.x, blockDim.x);
        p += TwTable<N, false, s>::SIZE;
    });
    static_for<0, NSG>([&](auto sc) {
        constexpr int s = decltype(sc)::value;
        twF[s] = p;
        fill_twiddles<N, true, s>(p, threadIdx.x, blockDim.x);
        p += TwTable<N, true, s>::SIZE;
    });
}

struct WarpSync {
    int grp = 0;  // unused; lets the pipelined kernels construct either barrier from the group index
    __device__ __forceinline__ void operator()() const { __syncwarp(); }
};
struct BlockSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
// Barrier over the T threads of group `grp` (named barrier 1 + grp; barrier 15 is the row pass's
// CTA-wide barrier).
template <int T>
struct GroupSync {
    int grp;
    __device__ __forceinline__ void operator()() const { asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "r"(T) : "memory"); }
};

// ---------------------------------------------------------------------------------------------
// Contiguous-line pass. LinePlan<NY>::T threads; each line of NY points is owned by TPL = NY/E
// threads.
template <int NY, int MODE>
__global__ void __launch_bounds__(LineGeom<NY>::THREADS, LinePlan<NY>::B) rows_kernel(RowArgs a) {
    using G = LineGeom<NY>;
    constexpr int E = G::E, TPL = G::TPL, LPC = G::LPC;
    extern __shared__ float2 smem2[];
    const float2* twI[3] = {nullptr, nullptr, nullptr};
    const float2* twF[3] = {nullptr, nullptr, nullptr};
    setup_twiddles<NY>(smem2, twI, twF);
    float2* lines = smem2 + G::TW_I + G::TW_F;
    __syncthreads();

    const int li = threadIdx.x / TPL, t = threadIdx.x % TPL;
    float2* buf = lines + li * G::LS;
    const int groups = a.nx / LPC;
    const int items = groups * a.nprobe;
    // a line's exchanges synchronise only its own threads: one warp, or a named barrier per line
    static_assert(TPL <= 32 || LPC <= 15, "one named barrier per line");
    using Sync = typename std::conditional<(TPL <= 32), WarpSync, GroupSync<TPL>>::type;
    const Sync sync{li};

    for (int item = blockIdx.x; item < items; item += gridDim.x) {
        const int b = item / groups;
        const int ix = (item % groups) * LPC + li;
        const size_t off = ((size_t)b * a.nx + ix) * NY;
        float2 x[E];
        if constexpr (MODE == ROW_STEP || MODE == ROW_INVERSE) {
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = a.in[off + reg_pos<NY, G::R1>(i, t)];
            line_fft<NY, false, +1>(x, buf, twI, t, sync);
        } else if constexpr (MODE == ROW_FIRST_REAL) {
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = a.in[off + reg_pos<NY, G::RL>(i, t)];
        } else {
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = make_float2(1.0f, 0.0f);
        }
        if constexpr (MODE == ROW_INVERSE) {
#pragma unroll
            for (int i = 0; i < E; i++) a.out[off + reg_pos<NY, G::RL>(i, t)] = cscale(x[i], a.scale);
        } else {
            const float2* Tr = a.trans + (size_t)b * a.trans_stride + (size_t)ix * NY;
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = cmul(x[i], __ldg(&Tr[reg_pos<NY, G::RL>(i, t)]));
            line_fft<NY, true, -1>(x, buf, twF, t, sync);
#pragma unroll
            for (int i = 0; i < E; i++) a.out[off + reg_pos<NY, G::R1>(i, t)] = x[i];
        }
    }
}

template <int NY>
static size_t rows_smem() {
    using G = LineGeom<NY>;
    return sizeof(float2) * (size_t)(G::TW_I + G::TW_F + G::LPC * G::LS);
}

// ---------------------------------------------------------------------------------------------
// Strided-line pass. LinePlan<NX>::T threads; W = T/TPL adjacent columns per CTA (coalesced rows
// of W complex values); column c is owned by threads c, c+W, c+2W, ...
__device__ __forceinline__ int ig_shift(int i, int nh, int n) { return (i < nh) ? i : (i - n); }

// exp_i_chi (src/cgpu_fcns.cuh:1951-1980) for one Fourier-space pixel, times the normalisation.
__device__ __forceinline__ float2 probe_value(const ProbeDev& pr, const GridDev& g, int ix, int iy, float2 beam) {
    const float gx = __fadd_rn(__fmul_rn((float)ig_shift(ix, g.nxh, g.nx), g.dgx), pr.gxu);
    const float gy = __fadd_rn(__fmul_rn((float)ig_shift(iy, g.nyh, g.ny), g.dgy), pr.gyu);
    const float g2 = __fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy));
    if (!((pr.g2_min <= g2) && (g2 < pr.g2_max))) return make_float2(0.0f, 0.0f);
    const float g4 = __fmul_rn(g2, g2);
    const float g6 = __fmul_rn(g4, g2);
    float chi = __fadd_rn(__fmul_rn(beam.x, gx), __fmul_rn(beam.y, gy));
    chi = __fadd_rn(chi, pr.nz_c10 ? __fmul_rn(pr.c_c_10, g2) : 0.0f);
    chi = __fadd_rn(chi, pr.nz_c30 ? __fmul_rn(pr.c_c_30, g4) : 0.0f);
    chi = __fadd_rn(chi, pr.nz_c50 ? __fmul_rn(pr.c_c_50, g6) : 0.0f);
    if (pr.phi_required) {
        const float gg = sqrtf(g2);
        const float g3 = __fmul_rn(g2, gg), g5 = __fmul_rn(g4, gg);
        const float ph = atan2f(gy, gx);
        auto term = [](float cc, float gp, float k, float ph, float ph0) {
            return (cc != 0.0f) ? __fmul_rn(__fmul_rn(cc, gp), sinf(__fmul_rn(k, __fsub_rn(ph, ph0)))) : 0.0f;
        };
        float t1 = __fadd_rn((ph != 0.0f) ? __fmul_rn((float)pr.m, ph) : 0.0f, term(pr.c_c_12, g2, 2.0f, ph, pr.phi_12));
        chi = __fadd_rn(chi, t1);
        float t2 = __fadd_rn(__fadd_rn(term(pr.c_c_21, g3, 1.0f, ph, pr.phi_21), term(pr.c_c_23, g3, 3.0f, ph, pr.phi_23)),
                             __fadd_rn(term(pr.c_c_32, g4, 2.0f, ph, pr.phi_32), term(pr.c_c_34, g4, 4.0f, ph, pr.phi_34)));
        chi = __fadd_rn(chi, t2);
        float t3 = __fadd_rn(__fadd_rn(__fadd_rn(term(pr.c_c_41, g5, 1.0f, ph, pr.phi_41), term(pr.c_c_43, g5, 3.0f, ph, pr.phi_43)),
                                       term(pr.c_c_45, g5, 5.0f, ph, pr.phi_45)),
                             __fadd_rn(__fadd_rn(term(pr.c_c_52, g6, 2.0f, ph, pr.phi_52), term(pr.c_c_54, g6, 4.0f, ph, pr.phi_54)),
                                       term(pr.c_c_56, g6, 6.0f, ph, pr.phi_56)));
        chi = __fadd_rn(chi, t3);
    }
    float sn, cs;
    sincosf(chi, &sn, &cs);
    return make_float2(__fmul_rn(cs, pr.norm), __fmul_rn(sn, pr.norm));
}

// Detector partials are kept per det_w columns (ColArgs::det_w, the narrowest tile width of the
// column kernels for this size): a tile of W >= det_w columns starting at column iy0 writes its
// sum to the first of its W/det_w partials and zero to the others.
template <class Sum>
__device__ __forceinline__ void write_det_partials(const ColArgs& a, int b, int iy0, int W, int tid, int nthreads,
                                                   Sum sum) {
    const int nsub = W / a.det_w;
    const int det_tiles = a.ny / a.det_w;
    const size_t base = ((size_t)b * det_tiles + iy0 / a.det_w) * a.n_det;
    for (int i = tid; i < nsub * a.n_det; i += nthreads) {
        const int sub = i / a.n_det, d = i % a.n_det;
        a.det_partial[base + (size_t)sub * a.n_det + d] = (sub == 0) ? sum(d) : 0.0;
    }
}

// A thread's contribution to detector d's sum from its E pixels of column iy, in the layout the
// last stage leaves (sum_square_over_Det, src/cgpu_fcns.cuh:1796-1814): |psi_hat|^2 where
// g2_min <= |g|^2 < g2_max (rings), or weighted by the detector's sensitivity map (matrix
// detectors). One detector at a time keeps one FP64 accumulator live; the pixels are added in the
// same order for every detector.
template <int NX>
__device__ __forceinline__ double det_pixels(const ColArgs& a, const float2 (&x)[LineGeom<NX>::E], int t, int iy,
                                             int d) {
    using G = LineGeom<NX>;
    double acc = 0.0;
    if (a.det_mat) {
        const size_t nxy = (size_t)a.g.nx * a.g.ny;
        const float* m = a.det_mat + (size_t)d * nxy + iy;
#pragma unroll
        for (int i = 0; i < G::E; i++) {
            const int ix = reg_pos<NX, G::RL>(i, t);
            const float v2 = __fadd_rn(__fmul_rn(x[i].x, x[i].x), __fmul_rn(x[i].y, x[i].y));
            acc += (double)__fmul_rn(__ldg(m + (size_t)ix * a.g.ny), v2);
        }
        return acc;
    }
    const float g2_min = a.det_g2_min[d], g2_max = a.det_g2_max[d];
    const float gy = __fsub_rn(__fmul_rn((float)ig_shift(iy, a.g.nyh, a.g.ny), a.g.dgy), 0.0f);
    const float gy2 = __fmul_rn(gy, gy);
#pragma unroll
    for (int i = 0; i < G::E; i++) {
        const int ix = reg_pos<NX, G::RL>(i, t);
        const float gx = __fmul_rn((float)ig_shift(ix, a.g.nxh, a.g.nx), a.g.dgx);
        const float g2 = __fadd_rn(__fmul_rn(gx, gx), gy2);
        const float v2 = __fadd_rn(__fmul_rn(x[i].x, x[i].x), __fmul_rn(x[i].y, x[i].y));
        if (g2_min <= g2 && g2 < g2_max) acc += (double)v2;
    }
    return acc;
}

// Coherent part of STEM (Output_Multislice::add_scale_psi_coh, src/output_multislice.hpp:770-780):
// psi_coh += coh_w * psi_hat at this probe's pixels, in FP32 like the reference.
template <int NX>
__device__ __forceinline__ void coh_add(const ColArgs& a, int b, const float2 (&x)[LineGeom<NX>::E], int t, int iy) {
    using G = LineGeom<NX>;
    float2* c = a.coh + (size_t)b * a.g.nx * a.g.ny + iy;
#pragma unroll
    for (int i = 0; i < G::E; i++) {
        float2* q = c + (size_t)reg_pos<NX, G::RL>(i, t) * a.g.ny;
        const float2 v = *q;
        *q = make_float2(__fadd_rn(__fmul_rn(a.coh_w, x[i].x), v.x), __fadd_rn(__fmul_rn(a.coh_w, x[i].y), v.y));
    }
}

// LDY is the line stride (= ny) when known at compile time (square grids), 0 for a runtime stride.
template <int NX, int FLAGS, int LDY>
__global__ void __launch_bounds__(LineGeom<NX>::THREADS, LinePlan<NX>::B) cols_kernel(ColArgs a) {
    using G = LineGeom<NX>;
    constexpr int E = G::E, W = G::LPC, NWARP = G::THREADS / 32;
    constexpr bool LOAD = FLAGS & COL_LOAD, PROP = FLAGS & COL_PROP, DET = FLAGS & COL_DETECT;
    constexpr bool INV = FLAGS & COL_INVERSE, STORE = FLAGS & COL_STORE;
    extern __shared__ float2 smem2[];
    const float2* twF[3] = {nullptr, nullptr, nullptr};  // forward (plan order)
    const float2* twI[3] = {nullptr, nullptr, nullptr};  // inverse (reversed order)
    // forward transform uses plan order (REV=false), inverse uses reversed order (REV=true)
    {
        float2* p = smem2;
        static_for<0, G::NSG>([&](auto sc) {
            constexpr int s = decltype(sc)::value;
            twF[s] = p;
            fill_twiddles<NX, false, s>(p, threadIdx.x, blockDim.x);
            p += TwTable<NX, false, s>::SIZE;
        });
        static_for<0, G::NSG>([&](auto sc) {
            constexpr int s = decltype(sc)::value;
            twI[s] = p;
            fill_twiddles<NX, true, s>(p, threadIdx.x, blockDim.x);
            p += TwTable<NX, true, s>::SIZE;
        });
    }
    float2* s_px = smem2 + G::TW_I + G::TW_F;
    float2* lines = s_px + (PROP ? NX : 0);
    __shared__ double s_red[NWARP][kMaxDet];
    if constexpr (PROP) {
        for (int i = threadIdx.x; i < NX; i += blockDim.x) s_px[i] = a.Px[i];
    }
    __syncthreads();

    const int c = threadIdx.x % W, t = threadIdx.x / W;
    float2* buf = lines + c * col_ls<NX, W>();
    const int ldy = LDY ? LDY : a.ny;
    const int tiles = ldy / W;
    const int items = tiles * a.nprobe;
    const size_t pstride = (size_t)NX * ldy;

    for (int item = blockIdx.x; item < items; item += gridDim.x) {
        const int b = item / tiles;
        const int ct = item % tiles;
        const int iy = ct * W + c;
        const size_t off = (size_t)b * pstride + iy + (size_t)t * ldy;
        const float2* src = a.in + off;
        float2* dst = a.out + off;
        float2 x[E];
        if constexpr (LOAD) {
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = src[(reg_pos<NX, G::R1>(i, t) - t) * ldy];
            line_fft<NX, false, -1>(x, buf, twF, t, BlockSync{});
        } else {
            const float2 beam = a.beam[b];
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = probe_value(a.probe, a.g, reg_pos<NX, G::RL>(i, t), iy, beam);
        }
        if constexpr (PROP) {
            const float2 py = a.Py[iy];
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = cmul(x[i], cmul(s_px[reg_pos<NX, G::RL>(i, t)], py));
            if constexpr (FLAGS & COL_P2) {
                const float2* p2 = a.P2 + iy;
#pragma unroll
                for (int i = 0; i < E; i++) x[i] = cmul(x[i], __ldg(p2 + (size_t)reg_pos<NX, G::RL>(i, t) * a.g.ny));
            }
        }
        if constexpr (DET) {
            if (a.coh) coh_add<NX>(a, b, x, t, iy);
            // deterministic block reduction: warp shuffles, then warps in order
#pragma unroll 1
            for (int d = 0; d < a.n_det; d++) {
                double v = det_pixels<NX>(a, x, t, iy, d);
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5][d] = v;
            }
            __syncthreads();
            write_det_partials(a, b, ct * W, W, threadIdx.x, G::THREADS, [&](int d) {
                double s = 0.0;
                for (int w = 0; w < NWARP; w++) s += s_red[w][d];
                return s;
            });
            __syncthreads();
        }
        if constexpr (INV) {
            line_fft<NX, true, +1>(x, buf, twI, t, BlockSync{});
#pragma unroll
            for (int i = 0; i < E; i++) dst[(reg_pos<NX, G::R1>(i, t) - t) * ldy] = x[i];
        } else if constexpr (STORE) {
#pragma unroll
            for (int i = 0; i < E; i++) dst[(reg_pos<NX, G::RL>(i, t) - t) * ldy] = x[i];
        }
    }
}

template <int NX, int FLAGS>
static size_t cols_smem() {
    using G = LineGeom<NX>;
    constexpr bool PROP = FLAGS & COL_PROP;
    return sizeof(float2) * (size_t)(G::TW_I + G::TW_F + (PROP ? NX : 0) + G::LPC * col_ls<NX, G::LPC>());
}

// ---------------------------------------------------------------------------------------------
// Bulk-copy-fed line passes.
//
// Bounded waits. Every wait for a copy gives up after the pass's wait_ns (from the first failed
// check), sets the engine's error flag and returns false. Once the flag is set, by this CTA or any
// other, waits return at once, no thread issues a new copy, and a pass launched later returns on
// entry; each group's copy thread then waits (bounded by kDrainLimitNs) for the copies it issued
// that nobody has seen land, so a CTA never exits with a copy in flight into its shared memory.
// The loops keep their structure (the transforms of the remaining items run on stale data), so
// every named barrier is still reached by all of its threads. The host reads the flag after the
// run and reports MT_ERR_TIMEOUT.
//
// One CTA per SM with two groups of T threads; group g transforms the CTA's items k = g, g+2,
// g+4, ... (line groups of the row pass, column tiles of the column pass). Each group owns a
// landing buffer in shared memory that the copy engine fills with the input lines of its next
// item (cp.async.bulk for the contiguous lines of the row pass, a 3-D tensor copy for the
// strided tile of the column pass; completion on mbarrier full[g], the group's j-th item being
// that barrier's phase j). A group waits for its landing buffer, reads it into registers,
// synchronises its own threads on a named barrier and issues the copy of its item k+2 into the
// same buffer before it transforms item k, so each SM keeps two items' reads in flight while
// both groups compute, and no thread waits on a global load of the wave. The exchanges between
// the two radix stages go through a per-group half-line buffer in two rounds
// (stage_exchange_half), which is what makes two landing buffers fit. Results are stored
// straight from registers.

__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// 3-D tile copy (no multicast) of the box at (x, y, z) described by the tensor map.
__device__ __forceinline__ void tensor_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                               unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}


constexpr size_t kPipeSmemMax = 232448 - 2048;  // opt-in shared memory per CTA less static use


// Row pass, bulk-copy fed, with the transmission rows resident in shared memory.
//
// The transmission function is the same for every probe, so a CTA takes a contiguous range of
// (line group, probe) items in line-group-major order, in units of NG items that never straddle
// a line group (nprobe % NG == 0): the CTA's NG groups of GT threads always work on the same
// line group g, and its LPC = GT/TPL transmission rows stay in shared memory (one bulk copy per
// change of g, after every group has finished with the previous rows). Group x transforms the
// items k = x, x+NG, ... from its own landing slot (mbarrier full[x], the group's j-th item being
// its phase j). The pipeline mode PM says where the exchanges go and when the next copy is issued:
//   PM 1: the group issues the copy of its next item as soon as it has read the slot, and exchanges
//         through its own half-line buffer (stage_exchange_half; plans with a half-line exchange);
//   PM 2: early issue as in PM 1, exchanges through its own full line buffer;
//   PM 0: the slot, sized for the full exchange buffer, serves as the exchange buffer and the next
//         copy is issued once the forward transform's exchange has been read back.
template <int NY, int GT, int NG, int PM>
struct RowPipe {
    using G = LineGeom<NY>;
    static constexpr int TPL = G::TPL;
    static constexpr int LPC = GT / TPL;
    static constexpr size_t TW = (size_t)G::TW_I + G::TW_F;
    static constexpr size_t LAND = (size_t)LPC * NY;
    // slots and per-group buffers in whole 16-byte units (bulk-copy targets follow them)
    static constexpr size_t SLOT0 = PM != 0 ? LAND : ((size_t)LPC * G::LS > LAND ? (size_t)LPC * G::LS : LAND);
    static constexpr size_t SLOT = (SLOT0 + 1) / 2 * 2;
    static constexpr size_t LBUF = PM == 1 ? (size_t)HalfLineSmem<NY>::value : (size_t)G::LS;  // per line
    static constexpr size_t HBUF = PM != 0 ? ((size_t)LPC * LBUF + 1) / 2 * 2 : 0;
    static constexpr size_t SMEM = sizeof(float2) * (TW + LAND + NG * SLOT + NG * HBUF);
    static constexpr bool OK = (GT % TPL == 0) && (GT % 32 == 0) && (SLOT % 2 == 0) && (HBUF % 2 == 0) &&
                               (TW % 2 == 0) &&
                               SMEM <= kPipeSmemMax && (GT == 32 || NG <= 14) &&
                               (PM != 1 || (HalfExchange<NY, false>::OK && HalfExchange<NY, true>::OK));
};

template <int NY, int MODE, int GT, int NG, int PM>
__global__ void __launch_bounds__(GT * NG, 1) rows_pipe_kernel(RowArgs a) {
    using G = LineGeom<NY>;
    using P = RowPipe<NY, GT, NG, PM>;
    constexpr bool EARLY = PM != 0, HALF = PM == 1;
    constexpr int E = G::E, TPL = G::TPL, LPC = P::LPC;
    static_assert(MODE == ROW_STEP || MODE == ROW_INVERSE || MODE == ROW_FIRST_REAL, "mode without a load");
    constexpr bool TRANS = MODE != ROW_INVERSE;
    constexpr unsigned LINE_BYTES = NY * sizeof(float2);
    extern __shared__ __align__(1024) unsigned char pipe_smem[];
    __shared__ unsigned long long full[NG], tbar;
    __shared__ int s_skip;
    float2* sm = reinterpret_cast<float2*>(pipe_smem);
    const float2* twI[3] = {nullptr, nullptr, nullptr};
    const float2* twF[3] = {nullptr, nullptr, nullptr};
    setup_twiddles<NY>(sm, twI, twF);
    float2* s_trans = sm + P::TW;  // [LPC][NY]
    float2* slots = s_trans + P::LAND;
    const int grp = threadIdx.x / GT, gtid = threadIdx.x % GT;
    const int li = gtid / TPL, t = gtid % TPL;
    float2* slot = slots + grp * P::SLOT;
    float2* buf = EARLY ? slots + NG * P::SLOT + grp * P::HBUF + (size_t)li * P::LBUF : slot + (size_t)li * G::LS;
    if (threadIdx.x == 0) {
        s_skip = err_set(a.err);  // an earlier pass timed out: the CTA returns (one decision for all)
        for (int i = 0; i < NG; i++) mbar_init(&full[i], 1);
        mbar_init(&tbar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (s_skip) return;

    // this CTA's items: [i0, i0 + K), item = g * nprobe + b, in units of NG
    const long long units = (long long)a.nx / LPC * a.nprobe / NG;
    const long long u0 = units * blockIdx.x / gridDim.x, u1 = units * (blockIdx.x + 1) / gridDim.x;
    const long long i0 = NG * u0;
    const int K = (int)(NG * (u1 - u0));
    // whether a warp may issue a copy: not once the error flag is set (lane 0 decides for the warp)
    auto may_issue = [&](int lane) {
        const int ok = lane == 0 ? !err_set(a.err) : 0;
        return __shfl_sync(0xffffffffu, ok, 0) != 0;
    };
    // issued by a whole warp: item k's LPC lines into slot k % NG
    int last_k = -1;  // the last item this warp issued (drained at exit)
    auto issue = [&](int k, int lane) {
        if (!may_issue(lane)) return;
        const long long item = i0 + k;
        const int g = (int)(item / a.nprobe), b = (int)(item % a.nprobe);
        const float2* src = a.in + ((size_t)b * a.nx + (size_t)g * LPC) * NY;
        unsigned long long* bar = &full[k % NG];
        float2* dst = slots + (k % NG) * P::SLOT;
        if (lane == 0) {
            fence_proxy_async();
            mbar_expect_tx(bar, LPC * LINE_BYTES);
        }
        __syncwarp();
        for (int l = lane; l < LPC; l += 32) bulk_load(dst + (size_t)l * NY, src + (size_t)l * NY, LINE_BYTES, bar);
        last_k = k;
    };
    // issued by warp 0: the transmission rows of line group g, phase `ph` of tbar
    int last_tph = -1;  // parity of the last transmission copy warp 0 issued (drained at exit)
    auto issue_trans = [&](int g, int lane, unsigned ph) {
        if (!may_issue(lane)) return;
        const float2* src = a.trans + (size_t)g * LPC * NY;
        if (lane == 0) {
            fence_proxy_async();
            mbar_expect_tx(&tbar, LPC * LINE_BYTES);
        }
        __syncwarp();
        for (int l = lane; l < LPC; l += 32) bulk_load(s_trans + (size_t)l * NY, src + (size_t)l * NY, LINE_BYTES, &tbar);
        last_tph = (int)ph;
    };
    if (gtid < 32 && grp < K) issue(grp, gtid);
    int g_cur = K > 0 ? (int)(i0 / a.nprobe) : 0;
    unsigned tphase = 0;
    if constexpr (TRANS) {
        if (threadIdx.x < 32 && K > 0) issue_trans(g_cur, threadIdx.x, tphase);
    }

    using Sync = typename std::conditional<(TPL <= 32), WarpSync, GroupSync<GT>>::type;
    using GSync = typename std::conditional<(GT == 32), WarpSync, GroupSync<GT>>::type;
    const GSync gsync{grp};
    for (int k = grp; k < K; k += NG) {
        const long long item = i0 + k;
        const int g = (int)(item / a.nprobe), b = (int)(item % a.nprobe);
        if constexpr (TRANS) {
            if (g != g_cur) {
                // every group reaches this point at the first unit of the new line group, after
                // finishing its last item of the old one
                asm volatile("bar.sync 15, %0;" ::"r"(NG * GT) : "memory");
                tphase ^= 1u;
                if (threadIdx.x < 32) issue_trans(g, threadIdx.x, tphase);
                g_cur = g;
            }
        }
        const int ix = g * LPC + li;
        const size_t off = ((size_t)b * a.nx + ix) * NY;
        mbar_wait(&full[grp], (unsigned)(k / NG) & 1u, a.err, a.wait_ns);
        const float2* lsrc = slot + (size_t)li * NY;
        float2 x[E];
        if constexpr (MODE == ROW_FIRST_REAL) {
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = lsrc[reg_pos<NY, G::RL>(i, t)];
        } else {
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = lsrc[reg_pos<NY, G::R1>(i, t)];
        }
        gsync();  // the slot's lines are in registers
        if constexpr (EARLY) {
            if (gtid < 32 && k + NG < K) issue(k + NG, gtid);
        }
        if constexpr (MODE == ROW_STEP || MODE == ROW_INVERSE) {
            if constexpr (HALF) line_fft_half<NY, false, +1>(x, buf, twI, t, Sync{grp});
            else line_fft<NY, false, +1>(x, buf, twI, t, Sync{grp});
        }
        if constexpr (MODE == ROW_INVERSE) {
            if constexpr (!EARLY) {
                gsync();
                if (gtid < 32 && k + NG < K) issue(k + NG, gtid);
            }
#pragma unroll
            for (int i = 0; i < E; i++) a.out[off + reg_pos<NY, G::RL>(i, t)] = cscale(x[i], a.scale);
        } else {
            mbar_wait(&tbar, tphase, a.err, a.wait_ns);
            const float2* Tr = s_trans + (size_t)li * NY;
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = cmul(x[i], Tr[reg_pos<NY, G::RL>(i, t)]);
            if constexpr (HALF) {
                line_fft_half<NY, true, -1>(x, buf, twF, t, Sync{grp});
            } else {
                line_fft<NY, true, -1>(x, buf, twF, t, Sync{grp});
                if constexpr (!EARLY) {
                    gsync();  // every exchange read of the slot is done
                    if (gtid < 32 && k + NG < K) issue(k + NG, gtid);
                }
            }
#pragma unroll
            for (int i = 0; i < E; i++) a.out[off + reg_pos<NY, G::R1>(i, t)] = x[i];
        }
    }
    // copies this warp issued and nobody saw land (only after an error): wait them out
    if (gtid == 0 && last_k >= 0) mbar_drain(&full[grp], (unsigned)(last_k / NG) & 1u);
    if (threadIdx.x == 0 && last_tph >= 0) mbar_drain(&tbar, (unsigned)last_tph);
}

// Row-pass pipeline shapes per line length: threads per group, groups, pipeline mode. Shape 0 is
// the default of every row pass (early issue with the half-line exchange where the plan has one,
// else late issue); shape 1, one warp per group (so a group synchronises with __syncwarp only) and
// 16 groups, and shape 2, early issue with full exchange buffers in as many groups (8, 4 or 2) as
// shared memory holds, are the alternatives the autotuner may pick for the slice step.
template <int NY, int V = 0>
struct RowPipeShape {
    static constexpr int GT = V == 0 ? 64 : 32, NG = V == 0 ? 8 : 16;
    static constexpr int PM = (HalfExchange<NY, false>::OK && HalfExchange<NY, true>::OK) ? 1 : 0;
};
template <int NY>
struct RowPipeShape<NY, 2> {
    static constexpr int GT = 64, PM = 2;
    static constexpr int NG = RowPipe<NY, 64, 8, 2>::OK ? 8 : RowPipe<NY, 64, 4, 2>::OK ? 4 : 2;
};

// Column pass, bulk-copy fed: NG groups of GT threads, W = GT/TPL columns per tile. The tensor
// map describes the probe batch as float32 [nprobe][NX][2*ldy] (re, im interleaved) with a box
// of 2W x BOXR x 1: one box is BOXR rows of a W-column tile, landing as [row][W]. Group x
// transforms the items k = x, x+NG, ... of the CTA (item = blockIdx.x + k*gridDim.x) from its
// own landing buffer, issues the copy of its next item as soon as it has read the buffer, and
// exchanges through its own buffers. Pipeline mode PM:
//   PM 1: the next tile is issued as soon as the group has read its slot, the exchanges use a
//         separate half-line buffer (HalfExchange);
//   PM 2: early issue as in PM 1, the exchanges use a separate full line buffer per column;
//   PM 0: (lengths without a half-line exchange, 1024) the slot doubles as the full exchange
//         buffer and the next tile is issued once the group's last exchange read is done; the other
//         groups keep the copy engine busy meanwhile.
template <int NX, int GT, int NG, int PM = (HalfExchange<NX, false>::OK && HalfExchange<NX, true>::OK) ? 1 : 0>
struct ColPipe {
    using G = LineGeom<NX>;
    static constexpr int PM_V = PM;
    static constexpr bool EARLY = PM != 0;
    static constexpr int W = GT / G::TPL;
    static constexpr int LSH = PM == 1 ? HalfLineSmem<NX>::value : col_ls<NX, W>();  // exchange buffer per column
    static constexpr size_t TW = (size_t)G::TW_I + G::TW_F;
    static constexpr size_t LAND0 = (size_t)W * NX;
    static constexpr size_t LAND1 = EARLY ? LAND0 : ((size_t)W * LSH > LAND0 ? (size_t)W * LSH : LAND0);
    static constexpr size_t LAND = (LAND1 + 15) / 16 * 16;  // slots on 128-byte boundaries (bulk-copy targets)
    static constexpr size_t HBUF = EARLY ? (size_t)W * LSH : 0;
    static constexpr size_t SMEM = sizeof(float2) * (TW + NX + NG * LAND + NG * HBUF);
    // rows per bulk-copy box: the boxes must tile the NX rows exactly (a box reaching past NX would
    // write past the slot and count bytes the barrier does not expect)
    static constexpr int BOXR = (NX <= 256) ? NX : (NX % 256 == 0) ? 256 : (NX % 128 == 0) ? 128 : 0;
    static constexpr bool OK = (PM != 1 || (HalfExchange<NX, false>::OK && HalfExchange<NX, true>::OK)) &&
                               (BOXR > 0) && (NX % (BOXR > 0 ? BOXR : 1) == 0) && ((size_t)NX * W <= LAND) &&
                               (((TW + NX) * sizeof(float2)) % 128 == 0) &&
                               (GT % G::TPL == 0) && (GT % 32 == 0) && (W % 2 == 0) && (2 * W <= 256) &&
                               (HBUF % 2 == 0) && SMEM <= kPipeSmemMax && (GT == 32 || NG <= 14);
};

// Column-pass pipeline shapes: 2 groups of 256 threads (default), and the alternatives the
// autotuner may pick for the slice step: 4 groups of 128 threads (narrower tiles), and groups of
// 128 threads in early-issue mode with full exchange buffers, as many (4, 3 or 2) as shared memory
// holds.
template <int NX, int V = 0>
struct ColPipeShape {
    static constexpr int GT = V == 0 ? 256 : 128, NG = V == 0 ? 2 : 4;
    static constexpr int PM = (HalfExchange<NX, false>::OK && HalfExchange<NX, true>::OK) ? 1 : 0;
};
template <int NX>
struct ColPipeShape<NX, 2> {
    static constexpr int GT = 128, PM = 2;
    static constexpr int NG = ColPipe<NX, 128, 4, 2>::OK ? 4 : ColPipe<NX, 128, 3, 2>::OK ? 3 : 2;
};

template <int NX, int FLAGS, int LDY, int GT, int NG, int PM>
__global__ void __launch_bounds__(GT * NG, 1) cols_pipe_kernel(ColArgs a, const __grid_constant__ CUtensorMap map) {
    using G = LineGeom<NX>;
    using P = ColPipe<NX, GT, NG, PM>;
    constexpr bool EARLY = PM != 0, HALF = PM == 1;
    constexpr int E = G::E, W = P::W, NWARP = GT / 32;
    constexpr bool PROP = FLAGS & COL_PROP, DET = FLAGS & COL_DETECT;
    constexpr bool INV = FLAGS & COL_INVERSE, STORE = FLAGS & COL_STORE;
    static_assert(FLAGS & COL_LOAD, "column pass without a load");
    static_assert(P::BOXR > 0 && NX % P::BOXR == 0 && (size_t)NX * W <= P::LAND, "bulk-copy boxes must fit the slot");
    constexpr unsigned TILE_BYTES = NX * W * sizeof(float2);
    extern __shared__ __align__(1024) unsigned char pipe_smem[];
    __shared__ unsigned long long full[NG];
    __shared__ double s_red[NG][NWARP][kMaxDet];
    __shared__ int s_skip;
    float2* sm = reinterpret_cast<float2*>(pipe_smem);
    const float2* twP[3] = {nullptr, nullptr, nullptr};  // plan order: the forward transform here
    const float2* twR[3] = {nullptr, nullptr, nullptr};  // reversed order: the inverse transform
    setup_twiddles<NX>(sm, twP, twR);
    float2* s_px = sm + P::TW;
    float2* land0 = s_px + NX;  // NG landing buffers, [row][W] each
    const int grp = threadIdx.x / GT, gtid = threadIdx.x % GT;
    const int c = gtid % W, t = gtid / W;
    float2* land = land0 + grp * P::LAND;
    float2* buf = EARLY ? land0 + NG * P::LAND + grp * P::HBUF + (size_t)c * P::LSH : land + (size_t)c * P::LSH;
    (void)HALF;
    if constexpr (PROP) {
        for (int i = threadIdx.x; i < NX; i += blockDim.x) s_px[i] = a.Px[i];
    }
    if (threadIdx.x == 0) {
        s_skip = err_set(a.err);  // an earlier pass timed out: the CTA returns (one decision for all)
        for (int i = 0; i < NG; i++) mbar_init(&full[i], 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (s_skip) return;

    const int ldy = LDY ? LDY : a.ny;
    const int tiles = ldy / W;
    const int items = tiles * a.nprobe;
    const size_t pstride = (size_t)NX * ldy;
    const int K = (int)blockIdx.x < items ? (items - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;
    // issued by one thread: item k's tile into landing buffer k % NG (none once the error flag is set)
    int last_k = -1;  // the last item this thread issued (drained at exit)
    auto issue = [&](int k) {
        if (err_set(a.err)) return;
        last_k = k;
        const int item = blockIdx.x + k * gridDim.x;
        unsigned long long* bar = &full[k % NG];
        float2* dst = land0 + (k % NG) * P::LAND;
        fence_proxy_async();
        mbar_expect_tx(bar, TILE_BYTES);
#pragma unroll
        for (int r0 = 0; r0 < NX; r0 += P::BOXR)
            tensor_load_3d(dst + (size_t)r0 * W, &map, (item % tiles) * 2 * W, r0, item / tiles, bar);
    };
    if (gtid == 0 && grp < K) issue(grp);

    using GSync = typename std::conditional<(GT == 32), WarpSync, GroupSync<GT>>::type;
    const GSync gsync{grp};
    for (int k = grp; k < K; k += NG) {
        const int item = blockIdx.x + k * gridDim.x;
        const int b = item / tiles, ct = item % tiles;
        const int iy = ct * W + c;
        const size_t off = (size_t)b * pstride + iy + (size_t)t * ldy;
        float2* dst = a.out + off;
        mbar_wait(&full[grp], (unsigned)(k / NG) & 1u, a.err, a.wait_ns);
        float2 x[E];
#pragma unroll
        for (int i = 0; i < E; i++) x[i] = land[(size_t)reg_pos<NX, G::R1>(i, t) * W + c];
        gsync();  // the whole group has read its landing buffer
        if constexpr (EARLY) {
            if (gtid == 0 && k + NG < K) issue(k + NG);
        }
        if constexpr (HALF) line_fft_half<NX, false, -1>(x, buf, twP, t, gsync);
        else line_fft<NX, false, -1>(x, buf, twP, t, gsync);
        if constexpr (PROP) {
            const float2 py = a.Py[iy];
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = cmul(x[i], cmul(s_px[reg_pos<NX, G::RL>(i, t)], py));
            if constexpr (FLAGS & COL_P2) {
                const float2* p2 = a.P2 + iy;
#pragma unroll
                for (int i = 0; i < E; i++) x[i] = cmul(x[i], __ldg(p2 + (size_t)reg_pos<NX, G::RL>(i, t) * a.g.ny));
            }
        }
        if constexpr (DET) {
            if (a.coh) coh_add<NX>(a, b, x, t, iy);
            // deterministic group reduction: warp shuffles, then the group's warps in order
#pragma unroll 1
            for (int d = 0; d < a.n_det; d++) {
                double v = det_pixels<NX>(a, x, t, iy, d);
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                if ((gtid & 31) == 0) s_red[grp][gtid >> 5][d] = v;
            }
            gsync();
            write_det_partials(a, b, ct * W, W, gtid, GT, [&](int d) {
                double s = 0.0;
                for (int w = 0; w < NWARP; w++) s += s_red[grp][w][d];
                return s;
            });
            gsync();
        }
        if constexpr (INV) {
            if constexpr (HALF) {
                line_fft_half<NX, true, +1>(x, buf, twR, t, gsync);
            } else {
                line_fft<NX, true, +1>(x, buf, twR, t, gsync);
                if constexpr (!EARLY) {
                    gsync();  // every exchange read of the slot is done
                    if (gtid == 0 && k + NG < K) issue(k + NG);
                }
            }
#pragma unroll
            for (int i = 0; i < E; i++) dst[(reg_pos<NX, G::R1>(i, t) - t) * ldy] = x[i];
            continue;
        }
        if constexpr (!EARLY) {
            gsync();  // the forward transform's exchange reads of the slot are done
            if (gtid == 0 && k + NG < K) issue(k + NG);
        }
        if constexpr (STORE) {
#pragma unroll
            for (int i = 0; i < E; i++) dst[(reg_pos<NX, G::RL>(i, t) - t) * ldy] = x[i];
        }
    }
    // a tile this thread issued and nobody saw land (only after an error): wait it out
    if (gtid == 0 && last_k >= 0) mbar_drain(&full[grp], (unsigned)(last_k / NG) & 1u);
}

// Tensor map for cols_pipe_kernel over a probe batch at `base` (cuTensorMapEncodeTiled through
// the runtime's driver entry point, so the library needs no link to the driver library).
void encode_tile_map(CUtensorMap* map, const float2* base, int nx, int ldy, int nprobe, int w, int boxr);

// ---------------------------------------------------------------------------------------------
// launch helpers (the per-kernel occupancy caps are function-local statics, initialised once and
// thread-safe, so engines on several host threads may launch concurrently)
template <class K>
static int max_ctas(K kernel, int threads, size_t smem) {
    static const int nsm = [] {
        int dev = 0, n = 0;
        MTB_CUDA(cudaGetDevice(&dev));
        MTB_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
        return n;
    }();
    MTB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    MTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem));
    if (occ < 1) fail(MT_ERR_UNSUPPORTED, "line-pass kernel does not fit on an SM");
    return nsm * occ;
}

// Launches the bulk-copy-fed row pass in pipeline shape V when that shape fits this line length and
// the probe count; returns false otherwise.
template <int NY, int MODE, int V>
static bool rows_pipe_try(const RowArgs& a, int grid_ctas, cudaStream_t s) {
    using S = RowPipeShape<NY, V>;
    using RP = RowPipe<NY, S::GT, S::NG, S::PM>;
    if constexpr (RP::OK && MODE != ROW_FIRST_ONE) {
        // the resident transmission rows are shared by every wave of the batch
        if (a.nprobe % S::NG != 0 || (a.trans_stride != 0 && MODE != ROW_INVERSE)) return false;
        auto kern = rows_pipe_kernel<NY, MODE, S::GT, S::NG, S::PM>;
        static const int cap = max_ctas(kern, S::GT * S::NG, RP::SMEM);
        const int units = (a.nx / RP::LPC) * a.nprobe / S::NG;
        int grid = grid_ctas > 0 ? grid_ctas : cap;
        if (grid > units) grid = units;
        kern<<<grid, S::GT * S::NG, RP::SMEM, s>>>(a);
        note_launch();
        MTB_CUDA(cudaGetLastError());
        return true;
    } else {
        (void)a, (void)grid_ctas, (void)s;
        return false;
    }
}

// The bulk-copy-fed kernels run where their shared memory fits and the pass loads its input;
// they need the error flag of their bounded waits (a.err), and without it the per-thread-load
// kernels run. The slice step may use an alternative pipeline shape (a.shape 1 or 2).
template <int NY, int MODE>
static void rows_launch(const RowArgs& a, int grid_ctas, cudaStream_t s) {
    using G = LineGeom<NY>;
    if (a.err) {
        if constexpr (MODE == ROW_STEP) {
            if (a.shape == 1 && rows_pipe_try<NY, MODE, 1>(a, grid_ctas, s)) return;
            if (a.shape == 2 && rows_pipe_try<NY, MODE, 2>(a, grid_ctas, s)) return;
        }
        if (rows_pipe_try<NY, MODE, 0>(a, grid_ctas, s)) return;
    }
    const size_t sm = rows_smem<NY>();
    static const int cap = max_ctas(rows_kernel<NY, MODE>, G::THREADS, sm);
    const int items = (a.nx / G::LPC) * a.nprobe;
    int grid = grid_ctas > 0 ? grid_ctas : cap;
    if (grid > items) grid = items;
    rows_kernel<NY, MODE><<<grid, G::THREADS, sm, s>>>(a);
    note_launch();
    MTB_CUDA(cudaGetLastError());
}

template <int NY>
void rows_dispatch_mode(RowMode mode, const RowArgs& a, int grid_ctas, cudaStream_t s) {
    switch (mode) {
        case ROW_STEP: rows_launch<NY, ROW_STEP>(a, grid_ctas, s); break;
        case ROW_FIRST_ONE: rows_launch<NY, ROW_FIRST_ONE>(a, grid_ctas, s); break;
        case ROW_FIRST_REAL: rows_launch<NY, ROW_FIRST_REAL>(a, grid_ctas, s); break;
        case ROW_INVERSE: rows_launch<NY, ROW_INVERSE>(a, grid_ctas, s); break;
    }
}

// Launches the bulk-copy-fed column pass in pipeline shape V when that shape fits this line length;
// returns false otherwise.
template <int NX, int FLAGS, int LDY, int V>
static bool cols_pipe_try(const ColArgs& a, int grid_ctas, cudaStream_t s) {
    using S = ColPipeShape<NX, V>;
    using CP = ColPipe<NX, S::GT, S::NG, S::PM>;
    if constexpr (CP::OK && (FLAGS & COL_LOAD)) {
        auto kern = cols_pipe_kernel<NX, FLAGS, LDY, S::GT, S::NG, S::PM>;
        static const int cap = max_ctas(kern, S::GT * S::NG, CP::SMEM);
        const int items = (a.ny / CP::W) * a.nprobe;
        int grid = grid_ctas > 0 ? grid_ctas : cap;
        if (grid > items) grid = items;
        CUtensorMap map;
        encode_tile_map(&map, a.in, NX, a.ny, a.nprobe, CP::W, CP::BOXR);
        kern<<<grid, S::GT * S::NG, CP::SMEM, s>>>(a, map);
        note_launch();
        MTB_CUDA(cudaGetLastError());
        return true;
    } else {
        (void)a, (void)grid_ctas, (void)s;
        return false;
    }
}

template <int NX, int FLAGS, int LDY>
static void cols_launch_ld(const ColArgs& a, int grid_ctas, cudaStream_t s) {
    using G = LineGeom<NX>;
    if (a.err) {
        if constexpr (FLAGS == (COL_LOAD | COL_PROP | COL_INVERSE | COL_STORE)) {
            if (a.shape == 1 && cols_pipe_try<NX, FLAGS, LDY, 1>(a, grid_ctas, s)) return;
            if (a.shape == 2 && cols_pipe_try<NX, FLAGS, LDY, 2>(a, grid_ctas, s)) return;
        }
        if (cols_pipe_try<NX, FLAGS, LDY, 0>(a, grid_ctas, s)) return;
    }
    const size_t sm = cols_smem<NX, FLAGS>();
    static const int cap = max_ctas(cols_kernel<NX, FLAGS, LDY>, G::THREADS, sm);
    const int items = (a.ny / G::LPC) * a.nprobe;
    int grid = grid_ctas > 0 ? grid_ctas : cap;
    if (grid > items) grid = items;
    cols_kernel<NX, FLAGS, LDY><<<grid, G::THREADS, sm, s>>>(a);
    note_launch();
    MTB_CUDA(cudaGetLastError());
}

template <int NX, int FLAGS>
static void cols_launch(const ColArgs& a, int grid_ctas, cudaStream_t s) {
    if (a.ny == NX) cols_launch_ld<NX, FLAGS, NX>(a, grid_ctas, s);
    else cols_launch_ld<NX, FLAGS, 0>(a, grid_ctas, s);
}

constexpr int COL_F_PROBE = COL_INVERSE | COL_STORE;
constexpr int COL_F_STEP = COL_LOAD | COL_PROP | COL_INVERSE | COL_STORE;
constexpr int COL_F_STEP_DET = COL_LOAD | COL_PROP | COL_DETECT | COL_INVERSE | COL_STORE;
constexpr int COL_F_LAST_DET = COL_LOAD | COL_PROP | COL_DETECT;
constexpr int COL_F_FOURIER = COL_LOAD | COL_PROP | COL_STORE;
constexpr int COL_F_PROBE_FS = COL_STORE;

// Columns per detector partial: the narrowest tile of the column kernels for this length.
template <int NX>
int cols_det_width() {
    constexpr int wc = LineGeom<NX>::LPC;
    using S = ColPipeShape<NX>;
    using CP = ColPipe<NX, S::GT, S::NG, S::PM>;
    constexpr int wp = CP::OK ? CP::W : wc;
    return wp < wc ? wp : wc;
}

template <int NX>
void cols_dispatch_flags(int flags, const ColArgs& a, int grid_ctas, cudaStream_t s) {
    // the [nx][ny] factor is a compile-time variant, so passes without it keep their registers
    if (a.P2 && (flags & COL_PROP)) flags |= COL_P2;
    switch (flags) {
        case COL_F_STEP | COL_P2: cols_launch<NX, COL_F_STEP | COL_P2>(a, grid_ctas, s); break;
        case COL_F_STEP_DET | COL_P2: cols_launch<NX, COL_F_STEP_DET | COL_P2>(a, grid_ctas, s); break;
        case COL_F_LAST_DET | COL_P2: cols_launch<NX, COL_F_LAST_DET | COL_P2>(a, grid_ctas, s); break;
        case COL_F_FOURIER | COL_P2: cols_launch<NX, COL_F_FOURIER | COL_P2>(a, grid_ctas, s); break;
        case COL_F_PROBE: cols_launch<NX, COL_F_PROBE>(a, grid_ctas, s); break;
        case COL_F_STEP: cols_launch<NX, COL_F_STEP>(a, grid_ctas, s); break;
        case COL_F_STEP_DET: cols_launch<NX, COL_F_STEP_DET>(a, grid_ctas, s); break;
        case COL_F_LAST_DET: cols_launch<NX, COL_F_LAST_DET>(a, grid_ctas, s); break;
        case COL_F_FOURIER: cols_launch<NX, COL_F_FOURIER>(a, grid_ctas, s); break;
        case COL_F_PROBE_FS: cols_launch<NX, COL_F_PROBE_FS>(a, grid_ctas, s); break;
        default: fail(MT_ERR_INTERNAL, "unsupported column-pass flag combination");
    }
}

}  // namespace mtb
