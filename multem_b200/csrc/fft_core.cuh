// Register/shared-memory FFT building blocks for the multislice passes (sm_100a).
//
// A line of N complex points is transformed by TPL = N / E threads, each holding E points in
// registers. The transform is a Stockham autosort FFT (Govindaraju et al., "High performance
// discrete Fourier transforms on graphics processors", SC'08) over a compile-time list of radices:
//
//   stage with radix R, Ns = product of the earlier radices, butterflies j in [0, N/R):
//     k = j % Ns;  v_r = in[j + r*N/R] * w^(r*k), w = exp(dir*2*pi*i/(Ns*R));  DFT_R(v);
//     out[(j/Ns)*Ns*R + k + r*Ns] = v_r
//
// Thread t owns butterflies j = t + TPL*m (m in [0, E/R)) and keeps v in x[m*R + r]. Points move
// between stages through a padded shared-memory line buffer. The first stage reads positions
// j + r*N/R and the last stage produces positions j + r*N/R_last, so
//   * the first stage can load straight from global memory (coalesced over t), and
//   * an inverse transform with radices (R1..Rs) followed by a forward transform with radices
//     (Rs..R1) needs no exchange between them: the inverse's outputs already sit in the registers
//     the forward's first stage reads. The pointwise multiply between them (transmission
//     function or Fresnel propagator) is applied there, in natural order.
#pragma once

#include <cuda_runtime.h>
#include <type_traits>
#include <utility>

namespace mtb {

// ---------------------------------------------------------------------------------------------
// compile-time helpers

template <int I>
using ic = std::integral_constant<int, I>;

template <int I, int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
    if constexpr (I < N) {
        f(ic<I>{});
        static_for<I + 1, N>(f);
    }
}

// cos/sin(2*pi*k/n) at compile time: octant reduction + Taylor series on [0, pi/4].
constexpr double cx_pi = 3.141592653589793238462643383279502884;

constexpr double cx_sin_series(double x) {
    double x2 = x * x, term = x, sum = x;
    for (int n = 1; n < 14; ++n) {
        term *= -x2 / ((2.0 * n) * (2.0 * n + 1.0));
        sum += term;
    }
    return sum;
}

constexpr double cx_cos_series(double x) {
    double x2 = x * x, term = 1.0, sum = 1.0;
    for (int n = 1; n < 14; ++n) {
        term *= -x2 / ((2.0 * n - 1.0) * (2.0 * n));
        sum += term;
    }
    return sum;
}

// returns cos (c=true) or sin (c=false) of 2*pi*k/n
constexpr double cx_trig2pi(long long k, long long n, bool c) {
    long long m = ((k % n) + n) % n;
    long long o = (8 * m) / n;                 // octant
    long long rem = 8 * m - o * n;             // angle within octant = (pi/4) * rem / n
    double th = (cx_pi / 4.0) * (double)rem / (double)n;
    double cth = (cx_pi / 4.0) * (double)(n - rem) / (double)n;  // pi/4 - th
    double cs = 0, sn = 0;
    switch (o) {
        case 0: cs = cx_cos_series(th); sn = cx_sin_series(th); break;
        case 1: cs = cx_sin_series(cth); sn = cx_cos_series(cth); break;
        case 2: cs = -cx_sin_series(th); sn = cx_cos_series(th); break;
        case 3: cs = -cx_cos_series(cth); sn = cx_sin_series(cth); break;
        case 4: cs = -cx_cos_series(th); sn = -cx_sin_series(th); break;
        case 5: cs = -cx_sin_series(cth); sn = -cx_cos_series(cth); break;
        case 6: cs = cx_sin_series(th); sn = -cx_cos_series(th); break;
        default: cs = cx_cos_series(cth); sn = -cx_sin_series(cth); break;
    }
    return c ? cs : sn;
}

// ---------------------------------------------------------------------------------------------
// complex helpers (float2 = (re, im))

// Complex sums as one packed FP32 instruction each (add/sub .rn.f32x2 on a register pair): the
// same two IEEE round-to-nearest sums as the scalar form, in half the issue slots.
__device__ __forceinline__ unsigned long long pack2(float2 a) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ float2 unpack2(unsigned long long r) {
    float2 d;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(r));
    return d;
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pack2(a)), "l"(pack2(b)));
    return unpack2(d);
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pack2(a)), "l"(pack2(b)));
    return unpack2(d);
}

// a + (DIR*i)^Q * b. The quarter turns swap the components of b, so they stay two scalar sums
// (the same roundings as adding the rotated value); Q = 0 and 2 are packed sums.
template <int Q, int DIR>
__device__ __forceinline__ float2 cadd_rot(float2 a, float2 b) {
    constexpr int q = ((Q % 4) + 4) % 4;
    if constexpr (q == 0) {
        return cadd(a, b);
    } else if constexpr (q == 2) {
        return csub(a, b);
    } else if constexpr ((q == 1) == (DIR > 0)) {  // +i * b = (-b.y, b.x)
        return make_float2(a.x - b.y, a.y + b.x);
    } else {                                       // -i * b = (b.y, -b.x)
        return make_float2(a.x + b.y, a.y - b.x);
    }
}

// Quarter turns Q (exp(DIR*2*pi*i*K/R) = (DIR*i)^Q) of a compile-time twiddle, or -1.
template <int K, int R>
constexpr int twiddle_quarter() {
    constexpr int k = ((K % R) + R) % R;
    return (4 * k) % R == 0 ? (4 * k) / R : -1;
}
// Complex products with their rounding fixed (one rounded product, one fused multiply-add per
// component), so that every kernel variant computes bit-identical results whatever the compiler
// would otherwise contract.
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(__fmaf_rn(a.x, b.x, -__fmul_rn(a.y, b.y)), __fmaf_rn(a.x, b.y, __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(__fmaf_rn(a.x, b.x, __fmul_rn(a.y, b.y)), __fmaf_rn(a.y, b.x, -__fmul_rn(a.x, b.y)));
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// multiply by exp(DIR * 2*pi*i * K / R), K and R compile-time
template <int K, int R, int DIR>
__device__ __forceinline__ float2 twiddle_const(float2 v) {
    constexpr int k = ((K % R) + R) % R;
    if constexpr (k == 0) {
        return v;
    } else if constexpr (4 * k == R) {          // exp(DIR*i*pi/2) = DIR*i
        return DIR > 0 ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
    } else if constexpr (2 * k == R) {          // -1
        return make_float2(-v.x, -v.y);
    } else if constexpr (4 * k == 3 * R) {      // exp(DIR*i*3pi/2) = -DIR*i
        return DIR > 0 ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
    } else if constexpr (8 * k == R || 8 * k == 3 * R || 8 * k == 5 * R || 8 * k == 7 * R) {
        constexpr float h = 0.70710678118654752440f;
        constexpr float c = (8 * k == R || 8 * k == 7 * R) ? h : -h;
        constexpr float s = (float)(DIR * ((8 * k == R || 8 * k == 3 * R) ? 1 : -1)) * h;
        return cmul(v, make_float2(c, s));
    } else {
        constexpr float c = (float)cx_trig2pi(k, R, true);
        constexpr float s = (float)(DIR * cx_trig2pi(k, R, false));
        return cmul(v, make_float2(c, s));
    }
}

// 3-point DFT: y0 = a + t1, y1,2 = (a - t1/2) +- DIR*i*(sqrt(3)/2)*t2, t1 = b + c, t2 = b - c.
template <int DIR>
__device__ __forceinline__ void dft3(float2& a, float2& b, float2& c) {
    constexpr float h = 0.86602540378443864676f;  // sqrt(3)/2
    const float2 t1 = cadd(b, c), t2 = csub(b, c);
    const float2 m = make_float2(__fmaf_rn(-0.5f, t1.x, a.x), __fmaf_rn(-0.5f, t1.y, a.y));
    const float2 s = DIR > 0 ? make_float2(-__fmul_rn(h, t2.y), __fmul_rn(h, t2.x))
                             : make_float2(__fmul_rn(h, t2.y), -__fmul_rn(h, t2.x));
    a = cadd(a, t1);
    b = cadd(m, s);
    c = csub(m, s);
}

// a +- w * b for the compile-time twiddle w = exp(DIR*2*pi*i*K/R); quarter turns cost no product.
template <int K, int R, int DIR>
__device__ __forceinline__ void tw_butterfly(float2 a, float2 b, float2& p, float2& m) {
    constexpr int q = twiddle_quarter<K, R>();
    if constexpr (q >= 0) {
        p = cadd_rot<q, DIR>(a, b);
        m = cadd_rot<q + 2, DIR>(a, b);
    } else {
        const float2 t = twiddle_const<K, R, DIR>(b);
        p = cadd(a, t);
        m = csub(a, t);
    }
}

// In-register DFT of length R (natural order in and out), dir = -1 forward, +1 inverse,
// unnormalised. Radix-4 / radix-3 / radix-2 decimation in time, fully unrolled; trivial twiddles
// folded.
template <int R, int DIR>
__device__ __forceinline__ void dft(float2* v) {
    if constexpr (R == 1) {
    } else if constexpr (R == 3) {
        dft3<DIR>(v[0], v[1], v[2]);
    } else if constexpr (R == 2) {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
        float2 t2 = cadd(v[1], v[3]), t3 = csub(v[1], v[3]);
        v[0] = cadd(t0, t2);
        v[2] = csub(t0, t2);
        v[1] = cadd_rot<1, DIR>(t1, t3);
        v[3] = cadd_rot<3, DIR>(t1, t3);
    } else if constexpr (R % 4 == 0) {
        // radix-4 DIT: four interleaved sub-DFTs of length R/4
        constexpr int Q = R / 4;
        float2 a[Q], b[Q], c[Q], d[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            a[i] = v[4 * i];
            b[i] = v[4 * i + 1];
            c[i] = v[4 * i + 2];
            d[i] = v[4 * i + 3];
        }
        dft<Q, DIR>(a);
        dft<Q, DIR>(b);
        dft<Q, DIR>(c);
        dft<Q, DIR>(d);
        static_for<0, Q>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            float2 bb = twiddle_const<k, R, DIR>(b[k]);
            float2 s0, s1, s2, d3;
            tw_butterfly<2 * k, R, DIR>(a[k], c[k], s0, s1);
            tw_butterfly<3 * k, R, DIR>(bb, d[k], s2, d3);
            v[k] = cadd(s0, s2);
            v[k + 2 * Q] = csub(s0, s2);
            v[k + Q] = cadd_rot<1, DIR>(s1, d3);
            v[k + 3 * Q] = cadd_rot<3, DIR>(s1, d3);
        });
    } else if constexpr (R % 3 == 0) {
        // radix-3 DIT: X[k + m*Q] = DFT3 over r of w_R^(k*r) * S_r[k], S_r = DFT_Q of v[3i + r]
        constexpr int Q = R / 3;
        float2 a[Q], b[Q], c[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            a[i] = v[3 * i];
            b[i] = v[3 * i + 1];
            c[i] = v[3 * i + 2];
        }
        dft<Q, DIR>(a);
        dft<Q, DIR>(b);
        dft<Q, DIR>(c);
        static_for<0, Q>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            float2 x0 = a[k], x1 = twiddle_const<k, R, DIR>(b[k]), x2 = twiddle_const<2 * k, R, DIR>(c[k]);
            dft3<DIR>(x0, x1, x2);
            v[k] = x0;
            v[k + Q] = x1;
            v[k + 2 * Q] = x2;
        });
    } else {
        static_assert(R % 2 == 0, "radix must factor into 2, 3 and 4");
        constexpr int H = R / 2;
        float2 e[H], o[H];
#pragma unroll
        for (int i = 0; i < H; ++i) {
            e[i] = v[2 * i];
            o[i] = v[2 * i + 1];
        }
        dft<H, DIR>(e);
        dft<H, DIR>(o);
        static_for<0, H>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            tw_butterfly<k, R, DIR>(e[k], o[k], v[k], v[k + H]);
        });
    }
}

// ---------------------------------------------------------------------------------------------
// Line plans: N points, E points per thread, T threads per CTA (per group, in the pipelined
// passes) of the line passes, B resident CTAs per SM the per-thread-load kernels are compiled for
// (caps registers at 65536 / (B*T)), radices of the forward transform in stage order. The inverse
// uses the same radices reversed (see the header comment).

template <int N>
struct LinePlan;

template <> struct LinePlan<64>   { static constexpr int E = 16, T = 256, B = 2, NS = 2; static constexpr int R[3] = {16, 4, 1}; };
template <> struct LinePlan<128>  { static constexpr int E = 16, T = 256, B = 2, NS = 2; static constexpr int R[3] = {16, 8, 1}; };
template <> struct LinePlan<256>  { static constexpr int E = 16, T = 256, B = 2, NS = 2; static constexpr int R[3] = {16, 16, 1}; };
template <> struct LinePlan<384>  { static constexpr int E = 24, T = 256, B = 2, NS = 3; static constexpr int R[3] = {24, 4, 4}; };
template <> struct LinePlan<512>  { static constexpr int E = 32, T = 256, B = 2, NS = 2; static constexpr int R[3] = {32, 16, 1}; };
template <> struct LinePlan<1024> { static constexpr int E = 32, T = 512, B = 1, NS = 2; static constexpr int R[3] = {32, 32, 1}; };
template <> struct LinePlan<2048> { static constexpr int E = 32, T = 256, B = 2, NS = 3; static constexpr int R[3] = {32, 8, 8}; };

// Radix of stage s of a transform whose stage order is `rev` ? reversed : plan order.
template <int N, bool REV, int S>
struct StageRadix {
    static constexpr int NSTAGE = LinePlan<N>::NS;
    static constexpr int value = S < NSTAGE ? LinePlan<N>::R[REV ? (NSTAGE - 1 - S) : S] : 1;  // 1 past the last stage
};

// Product of the radices before stage s.
template <int N, bool REV, int S>
struct StageNs {
    static constexpr int value = (S == 0) ? 1 : StageNs<N, REV, (S > 0 ? S - 1 : 0)>::value * StageRadix<N, REV, (S > 0 ? S - 1 : 0)>::value;
};
template <int N, bool REV>
struct StageNs<N, REV, 0> {
    static constexpr int value = 1;
};

// Padded shared-memory index for an exchange written by a stage of radix RW.
template <int RW>
__device__ __forceinline__ int pad_idx(int p) {
    return p + p / RW;
}

// Shared-memory floats needed per line (max over the paddings used).
template <int N>
struct LineSmem {
    static constexpr int value = N + N / 4 + 1;  // smallest radix 4 -> largest padding
};

// Per-stage twiddle table in shared memory: tw[(m*R + r)*TPL + t] = exp(-2*pi*i*r*k/(Ns*R)),
// k = (t + TPL*m) % Ns (N entries, one per thread and register), or, where the stage has fewer
// distinct twiddles than points (Ns*R < N: the middle stage of a three-stage plan), the compact
// tw[r*Ns + k] (Ns*R entries, 8x fewer for 2048 = 32 x 8 x 8; consecutive threads still read
// consecutive entries). The inverse direction uses the conjugate.
template <int N, bool REV, int S>
struct TwTable {
    static constexpr int E = LinePlan<N>::E;
    static constexpr int TPL = N / E;
    static constexpr int R = StageRadix<N, REV, S>::value;
    static constexpr int NSV = StageNs<N, REV, S>::value;
    static constexpr bool COMPACT = (NSV > 1) && (NSV * R < E * TPL);
    static constexpr int SIZE = (NSV > 1) ? (COMPACT ? NSV * R : E * TPL) : 0;
};

template <int N, bool REV, int S>
__device__ void fill_twiddles(float2* tw, int tid, int nthreads) {
    using TT = TwTable<N, REV, S>;
    if constexpr (TT::SIZE > 0) {
        for (int i = tid; i < TT::SIZE; i += nthreads) {
            int r, k;
            if constexpr (TT::COMPACT) {
                r = i / TT::NSV;
                k = i % TT::NSV;
            } else {
                const int t = i % TT::TPL;
                const int mr = i / TT::TPL;
                const int m = mr / TT::R;
                r = mr % TT::R;
                k = (t + TT::TPL * m) % TT::NSV;
            }
            double s, c;
            sincospi(-2.0 * (double)(r * k) / (double)(TT::NSV * TT::R), &s, &c);
            tw[i] = make_float2((float)c, (float)s);
        }
    }
}

// Compute stage S (twiddle + DFT) in registers. x[m*R + r] holds input j + r*N/R, j = t + TPL*m.
template <int N, bool REV, int S, int DIR>
__device__ __forceinline__ void stage_compute(float2* x, int t, const float2* tw) {
    constexpr int E = LinePlan<N>::E;
    constexpr int TPL = N / E;
    constexpr int R = StageRadix<N, REV, S>::value;
    constexpr int NSV = StageNs<N, REV, S>::value;
    static_for<0, E / R>([&](auto mc) {
        constexpr int m = decltype(mc)::value;
        if constexpr (NSV > 1) {
            const int kc = (t + TPL * m) % NSV;  // the butterfly's k (compact tables)
            (void)kc;
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 w = TwTable<N, REV, S>::COMPACT ? tw[r * NSV + kc] : tw[(m * R + r) * TPL + t];
                x[m * R + r] = (DIR < 0) ? cmul(x[m * R + r], w) : cmulc(x[m * R + r], w);
            }
        }
        dft<R, DIR>(&x[m * R]);
    });
}

// Padded buffer index of the exchange after stage S, for thread t and register i, on the writing
// side (stage S's output position) and the reading side (stage S+1's input position). When both
// are t * stride + f(i) for every t and i (checked at compile time), each access is a per-thread
// base plus a compile-time offset.
template <int N, bool REV, int S>
struct ExchangeMap {
    static constexpr int E = LinePlan<N>::E;
    static constexpr int TPL = N / E;
    static constexpr int R = StageRadix<N, REV, S>::value;
    static constexpr int NSV = StageNs<N, REV, S>::value;
    static constexpr int R2 = StageRadix<N, REV, S + 1>::value;
    static constexpr int wpos(int t, int i) {
        const int j = t + TPL * (i / R);
        const int p = (j / NSV) * NSV * R + (j % NSV) + (i % R) * NSV;
        return p + p / R;
    }
    static constexpr int rpos(int t, int i) {
        const int p = t + TPL * (i / R2) + (i % R2) * (N / R2);
        return p + p / R;
    }
    static constexpr int SW = wpos(1, 0) - wpos(0, 0);
    static constexpr int SR = rpos(1, 0) - rpos(0, 0);
    static constexpr bool linear() {
        for (int t = 0; t < TPL; t++)
            for (int i = 0; i < E; i++)
                if (wpos(t, i) != t * SW + wpos(0, i) || rpos(t, i) != t * SR + rpos(0, i)) return false;
        return true;
    }
    static constexpr bool LINEAR = linear();
};

// Exchange after stage S through the line buffer `buf` (floats as float2), then load the inputs
// of stage S+1. Caller provides the barrier functor (warp- or block-level).
template <int N, bool REV, int S, class Sync>
__device__ __forceinline__ void stage_exchange(float2* x, float2* buf, int t, Sync sync) {
    using M = ExchangeMap<N, REV, S>;
    constexpr int E = M::E, TPL = M::TPL, R = M::R, NSV = M::NSV, R2 = M::R2;
    if constexpr (M::LINEAR) {
        sync();
        float2* bw = buf + t * M::SW;
        static_for<0, E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            bw[M::wpos(0, i)] = x[i];
        });
        sync();
        const float2* br = buf + t * M::SR;
        static_for<0, E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            x[i] = br[M::rpos(0, i)];
        });
    } else {
        sync();
#pragma unroll
        for (int m = 0; m < E / R; ++m) {
            int j = t + TPL * m;
            int base = (j / NSV) * NSV * R + (j % NSV);
#pragma unroll
            for (int r = 0; r < R; ++r) buf[pad_idx<R>(base + r * NSV)] = x[m * R + r];
        }
        sync();
#pragma unroll
        for (int m = 0; m < E / R2; ++m) {
            int j = t + TPL * m;
#pragma unroll
            for (int r = 0; r < R2; ++r) x[m * R2 + r] = buf[pad_idx<R>(j + r * (N / R2))];
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Half-line exchange: the same permutation through a buffer of N/2 positions, in two rounds.
//
// For a two-stage plan the first stage (Ns = 1, radix R) writes position p = (t + TPL*m)*R + r
// and the second (radix R2) reads p = t + TPL*m' + r'*N/R2. A position bit B >= log2(TPL) that
// the writer fixes through (m, r) alone is fixed for the reader through (m', r') alone too, so
// round h moves exactly the positions whose bit B is h, with compile-time register selection
// on both sides. B exists when R > TPL (B = log2 TPL, a bit of r) or E/R >= 2 (B = log2(R*TPL),
// a bit of m); it does not for plans with R = TPL and E = R (256 and 1024 here).

constexpr int ilog2c(int v) { return v <= 1 ? 0 : 1 + ilog2c(v / 2); }

template <int N, bool REV>
struct HalfExchange {
    static constexpr int E = LinePlan<N>::E;
    static constexpr int TPL = N / E;
    static constexpr int R = StageRadix<N, REV, 0>::value;
    static constexpr int R2 = StageRadix<N, REV, 1>::value;
    static constexpr int LT = ilog2c(TPL), LR = ilog2c(R);
    static constexpr int B = (LinePlan<N>::NS != 2) ? -1 : (LR > LT) ? LT : ((E / R >= 2) ? LR + LT : -1);
    // thread stride of the writer's positions after removing bit B; padding by it keeps the
    // writes of consecutive threads on distinct banks
    static constexpr int PADW = (B >= 0 && B < LR) ? R / 2 : R;
    // round 1 writes must not read registers that round 0's reads already replaced
    static constexpr bool disjoint() {
        if (B < 0) return false;
        const int sb = B < 0 ? 0 : B;
        for (int i = 0; i < E; i++) {
            const int mw = i / R, rw = i % R;  // writer register i
            const int mr = i / R2, rr = i % R2;  // reader register i
            const bool w1 = ((TPL * mw * R + rw) >> sb) & 1;
            const bool r0 = !(((TPL * mr + rr * (N / R2)) >> sb) & 1);
            if (w1 && r0) return false;
        }
        return true;
    }
    static constexpr bool OK = (B >= 0) && disjoint();
};

template <int B>
__device__ __forceinline__ int drop_bit(int p) {
    return (p & ((1 << B) - 1)) | ((p >> (B + 1)) << B);
}
constexpr int drop_bit_c(int p, int b) { return (p & ((1 << b) - 1)) | ((p >> (b + 1)) << b); }

// Line buffer length (float2) for the half-line exchange: N/2 positions padded by the smallest
// PADW of the plan (>= RMIN/2), odd.
template <int N>
struct HalfLineSmem {
    static constexpr int RMIN = (LinePlan<N>::R[0] < LinePlan<N>::R[1]) ? LinePlan<N>::R[0] : LinePlan<N>::R[1];
    static constexpr int value = N / 2 + N / RMIN + 1;
};

// Buffer index of the half-line exchange (as ExchangeMap, with bit B of the position dropped).
template <int N, bool REV>
struct HalfExchangeMap {
    using H = HalfExchange<N, REV>;
    static constexpr int E = H::E, TPL = H::TPL, R = H::R, R2 = H::R2, B = H::B < 0 ? 0 : H::B, PW = H::PADW;
    static constexpr int wcpos(int i) { return TPL * (i / R) * R + (i % R); }        // writer position less t*R
    static constexpr int rcpos(int i) { return TPL * (i / R2) + (i % R2) * (N / R2); }  // reader position less t
    static constexpr int idx(int p) { return drop_bit_c(p, B) + drop_bit_c(p, B) / PW; }
    static constexpr int wpos(int t, int i) { return idx(t * R + wcpos(i)); }
    static constexpr int rpos(int t, int i) { return idx(t + rcpos(i)); }
    static constexpr int SW = wpos(1, 0) - wpos(0, 0);
    static constexpr int SR = rpos(1, 0) - rpos(0, 0);
    static constexpr bool linear() {
        for (int t = 0; t < TPL; t++)
            for (int i = 0; i < E; i++)
                if (wpos(t, i) != t * SW + wpos(0, i) || rpos(t, i) != t * SR + rpos(0, i)) return false;
        return true;
    }
    static constexpr bool LINEAR = H::OK && linear();
};

template <int N, bool REV, class Sync>
__device__ __forceinline__ void stage_exchange_half(float2* x, float2* buf, int t, Sync sync) {
    using H = HalfExchange<N, REV>;
    using M = HalfExchangeMap<N, REV>;
    constexpr int E = H::E, R = H::R, B = H::B, PW = H::PADW;
    static_assert(H::OK, "plan has no half-line exchange");
    float2* bw = buf + (M::LINEAR ? t * M::SW : 0);
    const float2* br = buf + (M::LINEAR ? t * M::SR : 0);
    static_for<0, 2>([&](auto hc) {
        constexpr int h = decltype(hc)::value;
        sync();
        static_for<0, E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            constexpr int cpos = M::wcpos(i);
            if constexpr (((cpos >> B) & 1) == h) {
                if constexpr (M::LINEAR) bw[M::wpos(0, i)] = x[i];
                else buf[pad_idx<PW>(drop_bit<B>(t * R + cpos))] = x[i];
            }
        });
        sync();
        static_for<0, E>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            constexpr int cpos = M::rcpos(i);
            if constexpr (((cpos >> B) & 1) == h) {
                if constexpr (M::LINEAR) x[i] = br[M::rpos(0, i)];
                else x[i] = buf[pad_idx<PW>(drop_bit<B>(t + cpos))];
            }
        });
    });
}

// Two-stage transform with the half-line exchange (see line_fft below).
template <int N, bool REV, int DIR, class Sync>
__device__ __forceinline__ void line_fft_half(float2* x, float2* buf, const float2* const* tw, int t, Sync sync) {
    static_assert(LinePlan<N>::NS == 2, "half-line exchange needs a two-stage plan");
    stage_compute<N, REV, 0, DIR>(x, t, tw[0]);
    stage_exchange_half<N, REV>(x, buf, t, sync);
    stage_compute<N, REV, 1, DIR>(x, t, tw[1]);
}

// Full transform: x holds the first stage's inputs (positions j + r*N/R_first); on return it
// holds outputs at positions j + r*N/R_last. tw[s] are the stage twiddle tables.
template <int N, bool REV, int DIR, class Sync>
__device__ __forceinline__ void line_fft(float2* x, float2* buf, const float2* const* tw, int t, Sync sync) {
    constexpr int NSTAGE = LinePlan<N>::NS;
    static_for<0, NSTAGE>([&](auto sc) {
        constexpr int s = decltype(sc)::value;
        stage_compute<N, REV, s, DIR>(x, t, tw[s]);
        if constexpr (s + 1 < NSTAGE) stage_exchange<N, REV, s>(x, buf, t, sync);
    });
}

// Position held by register i after a transform whose last stage has radix RL:
// i = m*RL + r  ->  j + r*N/RL with j = t + TPL*m.
template <int N, int RL>
__device__ __forceinline__ int reg_pos(int i, int t) {
    constexpr int TPL = N / LinePlan<N>::E;
    return (t + TPL * (i / RL)) + (i % RL) * (N / RL);
}

}  // namespace mtb
