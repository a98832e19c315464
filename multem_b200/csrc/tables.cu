// FP64 build of the radial projected-potential spline tables on the GPU.
//
// Follows Atomic_Data::get_atom_coef (src/atomic_data.hpp:1547-1668) for neutral atoms of the five
// parameterisations with a closed-form projected potential (potential_type 1-4 and 6):
//   6 Lobato (0-12), set_Lobato_neutral_coef (src/atomic_data.hpp:1441-1486):
//     VR.cl = 2*Potf*pi^2*cl/cnl^1.5, VR.cnl = 2*pi/sqrt(cnl)        (projected potential)
//     Vr.cl =   Potf*pi^2*cl/cnl^1.5, Vr.cnl = 2*pi/sqrt(cnl)        (3-D potential)
//     VR(R) = sum_5 cl*(2*K0(cnl*R)/cnl + R*K1(cnl*R)), dVR/dR = -sum_5 cl*(cnl*R*K0 + 2*K1)
//     (VR_dVR_Lobato_neutral_0_12, src/cgpu_fcns.cuh:1256-1268)
//   1 Doyle-Turner (0-4, 4 Gaussians), 2 Peng (0-4, 5 Gaussians), 3 Peng (0-12, 5 Gaussians),
//     set_Doyle_Peng_neutral_coef (src/atomic_data.hpp:1303-1348), with b = cnl/4:
//     Vr.cl = Potf*cl*(pi/b)^1.5, VR.cl = Potf*pi*cl/b, Vr.cnl = VR.cnl = pi^2/b
//     Vr(r) = sum cl*exp(-cnl*r^2), VR(R) = sum cl*exp(-cnl*R^2)   (add_Gauss_Fn,
//     src/cgpu_fcns.cuh:491-520; Vr_/VR_Doyle/Peng_neutral_*, src/cgpu_fcns.cuh:1023-1063, 1162-1201)
//   4 Kirkland (0-12, 3 Yukawa + 3 Gaussians), set_Kirkland_neutral_coef (src/atomic_data.hpp:1351-1400):
//     Yukawa terms j < 3: Vr.cl = Potf*pi*cl, VR.cl = Potf*2*pi*cl, Vr.cnl = VR.cnl = 2*pi*sqrt(cnl)
//     Gaussian terms j = 3..5: as above with b = cnl
//     Vr(r) = sum_3 cl*exp(-cnl*r)/r + Gaussians (add_Yukawa_Fn, src/cgpu_fcns.cuh:557-570)
//     VR(R) = sum_3 cl*K0(cnl*R) + Gaussians, dVR = -sum_3 cl*cnl*K1(cnl*R) + Gaussian derivatives
//     (VR_dVR_Kirkland_neutral_0_12, src/cgpu_fcns.cuh:1203-1230)
// Common to all types:
//   R_min = max(dR_min, rn_c), rn_c = 1.2e-5*A^(1/3)
//   R_max = root of Vr(r) = Vrl by bisection on [rn_c, 25] (Atom_Cal::AtomicRadius_Cutoff,
//           src/atomic_fcns_mt.hpp:269-295; Root_Finder, src/cgpu_fcns.cuh:262-286), or 0 when
//           Vr.cl[0] is zero; R_max = max(R_max, 2*R_min), or 1.75*ra when it is zero
//   R_tap = R_min + 0.85*(R_max - R_min), tap_cf = (pi/2)/(R_max^2 - R_tap^2)
//   nR log-spaced knots R_i = R_min*exp(i*ln(R_max/R_min)/(nR-1)), spline variable R^2
//   c0 = VR, c1 = dVR/d(R^2) = 0.5*dVR/R, both cosine-tapered beyond R_tap^2 (apply_tapering,
//   src/cgpu_fcns.cuh:1530-1540); c2, c3 from the Hermite conditions between knots
//   (src/atomic_data.hpp:1652-1663).
//   Ions (atoms whose charge q has an entry in Peng's ionic table, whatever potential_type):
//     set_Peng_ions_coef (src/atomic_data.hpp:1489-1543): five Gaussian terms as for type 2 from
//     the ionic table, plus a screened Coulomb term for the net charge, cl = q/(2 pi^2 a0),
//     cnl = (2 pi r0)^-2 with r0 = 2 A, turned into a Yukawa term as Kirkland's; VR adds
//     cl*K0(cnl*R) (VR_dVR_Peng_ion_0_4, src/cgpu_fcns.cuh:1271-1284); R_max is the neutral
//     atom's (src/atomic_data.hpp:1612). A charge without an entry uses the neutral coefficients
//     (Atom_Type::charge_to_idx, src/types.cuh:4125-4137).
// Weickenmeier-Kohl (type 5) has no closed-form projected potential (the reference integrates Vr
// numerically along z) and is refused by the input validation.
// The modified Bessel functions K0, K1 use the polynomial approximations of Abramowitz & Stegun,
// Handbook of Mathematical Functions, 9.8.1-9.8.8 (I0, I1 for x <= 3.75; K0, K1 for x <= 2 and
// x > 2), the same published approximations the reference uses (src/math.cuh:465-630).
// R_min/R_max/R_tap come from element_head() on the host (a sequential root find in FP64); one
// CUDA block then builds the knots and coefficients of one element, one thread per knot, in FP64.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "common.hpp"
#include "devmem.hpp"
#include "tables.hpp"

namespace mtb {

namespace {

#include "atomic_params.inc"

constexpr double kPotf = 47.877645145863056;
constexpr double kPi = 3.141592653589793238463;
constexpr double kPi2 = 9.869604401089358618834;
constexpr double k2Pi = 6.283185307179586476925;
constexpr double kHalfPi = 1.570796326794896619231;

struct ElemCoef {
    double VRcl[6], VRcnl[6], Vrcl[6], Vrcnl[6];  // unused terms: cl = 0, cnl = 1
    double rn_c, ra;
    int type;  // potential_type, or kIonType for a Peng ion
};

constexpr int kIonType = 7;
constexpr double k2Pi2a0 = 10.445539456905012;  // 2 pi^2 a0 (Bohr radius in A)

// Gaussian terms of each parameterisation: [g0, g1); Kirkland's Yukawa terms are [0, 3)
__host__ __device__ inline int gauss_first(int type) { return type == 4 ? 3 : 0; }
__host__ __device__ inline int gauss_end(int type) { return type == 1 ? 4 : (type == 4 ? 6 : 5); }

// Index of charge q in the reference's per-element coefficient list (2q for q > 0, -2q - 1 below)
int charge_index(int q) { return q >= 0 ? 2 * q : -2 * q - 1; }

const PengIon* find_ion(int Z, int q) {
    if (q == 0) return nullptr;
    const int idx = charge_index(q);
    for (const PengIon& e : kPengIon)
        if (e.Z == Z && e.idx == idx) return &e;
    return nullptr;
}

__device__ double as_i0(double x) {  // A&S 9.8.1 / 9.8.2
    double ax = fabs(x), y;
    if (ax < 3.75) {
        y = x / 3.75;
        y = y * y;
        return 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 + y * (0.2659732 + y * (0.360768e-1 + y * 0.45813e-2)))));
    }
    y = 3.75 / ax;
    return (exp(ax) / sqrt(ax)) *
           (0.39894228 + y * (0.1328592e-1 + y * (0.225319e-2 + y * (-0.157565e-2 + y * (0.916281e-2 + y * (-0.2057706e-1 + y * (0.2635537e-1 + y * (-0.1647633e-1 + y * 0.392377e-2))))))));
}

__device__ double as_i1(double x) {  // A&S 9.8.3 / 9.8.4
    double ax = fabs(x), y, ans;
    if (ax < 3.75) {
        y = x / 3.75;
        y = y * y;
        ans = ax * (0.5 + y * (0.87890594 + y * (0.51498869 + y * (0.15084934 + y * (0.2658733e-1 + y * (0.301532e-2 + y * 0.32411e-3))))));
    } else {
        y = 3.75 / ax;
        ans = 0.2282967e-1 + y * (-0.2895312e-1 + y * (0.1787654e-1 - y * 0.420059e-2));
        ans = 0.39894228 + y * (-0.3988024e-1 + y * (-0.362018e-2 + y * (0.163801e-2 + y * (-0.1031555e-1 + y * ans))));
        ans *= (exp(ax) / sqrt(ax));
    }
    return (x < 0.0) ? -ans : ans;
}

__device__ double as_k0(double x) {  // A&S 9.8.5 / 9.8.6
    double y;
    if (x <= 2.0) {
        y = x * x / 4.0;
        return (-log(x / 2.0) * as_i0(x)) +
               (-0.57721566 + y * (0.42278420 + y * (0.23069756 + y * (0.3488590e-1 + y * (0.262698e-2 + y * (0.10750e-3 + y * 0.74e-5))))));
    }
    y = 2.0 / x;
    return (exp(-x) / sqrt(x)) *
           (1.25331414 + y * (-0.7832358e-1 + y * (0.2189568e-1 + y * (-0.1062446e-1 + y * (0.587872e-2 + y * (-0.251540e-2 + y * 0.53208e-3))))));
}

__device__ double as_k1(double x) {  // A&S 9.8.7 / 9.8.8
    double y;
    if (x <= 2.0) {
        y = x * x / 4.0;
        return (log(x / 2.0) * as_i1(x)) +
               (1.0 / x) * (1.0 + y * (0.15443144 + y * (-0.67278579 + y * (-0.18156897 + y * (-0.1919402e-1 + y * (-0.110404e-2 + y * (-0.4686e-4)))))));
    }
    y = 2.0 / x;
    return (exp(-x) / sqrt(x)) *
           (1.25331414 + y * (0.23498619 + y * (-0.3655620e-1 + y * (0.1504268e-1 + y * (-0.780353e-2 + y * (0.325614e-2 + y * (-0.68245e-3)))))));
}

__global__ void build_tables_kernel(const ElemCoef* __restrict__ coef, const TableHead* __restrict__ head,
                                    int n_elem, int nR, float* __restrict__ tab) {
    const int ie = blockIdx.x;
    if (ie >= n_elem) return;
    const ElemCoef c = coef[ie];
    const TableHead h = head[ie];
    extern __shared__ double sdyn[];
    double* c0 = sdyn;
    double* c1 = sdyn + nR;
    double* R2 = sdyn + 2 * nR;
    const double R_min = h.R_min, R_max = h.R_max, R_tap = h.R_tap, tap_cf = h.tap_cf;
    const double dlnr = log(R_max / R_min) / (double)(nR - 1);
    const double x_tap = pow(R_tap, 2);
    for (int iR = threadIdx.x; iR < nR; iR += blockDim.x) {
        double R = R_min * exp(iR * dlnr);
        double r2 = pow(R, 2);
        double y = 0, dy = 0;
        if (c.type == 6) {
            for (int i = 0; i < 5; i++) {
                double k0 = as_k0(c.VRcnl[i] * R);
                double k1 = as_k1(c.VRcnl[i] * R);
                y += c.VRcl[i] * (2 * k0 / c.VRcnl[i] + R * k1);
                dy += -c.VRcl[i] * (c.VRcnl[i] * R * k0 + 2 * k1);
            }
        } else {
            if (c.type == kIonType) {
                y += c.VRcl[5] * as_k0(c.VRcnl[5] * R);
                dy += -c.VRcl[5] * c.VRcnl[5] * as_k1(c.VRcnl[5] * R);
            }
            if (c.type == 4)
                for (int i = 0; i < 3; i++) {
                    y += c.VRcl[i] * as_k0(c.VRcnl[i] * R);
                    dy += -c.VRcl[i] * c.VRcnl[i] * as_k1(c.VRcnl[i] * R);
                }
            for (int i = gauss_first(c.type); i < gauss_end(c.type); i++) {
                double yt = c.VRcl[i] * exp(-c.VRcnl[i] * (R * R));
                y += yt;
                dy += -2 * c.VRcnl[i] * R * yt;
            }
        }
        dy = 0.5 * dy / R;
        if (x_tap < r2) {
            double s, co;
            sincos(tap_cf * (r2 - x_tap), &s, &co);
            dy = dy * co - tap_cf * y * s;
            y *= co;
        }
        c0[iR] = y;
        c1[iR] = dy;
        R2[iR] = r2;
    }
    __syncthreads();
    float* t = tab + (size_t)ie * 5 * nR;
    for (int iR = threadIdx.x; iR < nR; iR += blockDim.x) {
        double c2 = 0, c3 = 0;
        if (iR < nR - 1) {
            double idR = 1.0 / (R2[iR + 1] - R2[iR]);
            double V = c0[iR], Vn = c0[iR + 1], dV = c1[iR], dVn = c1[iR + 1];
            double mm = (Vn - V) * idR, n = dV + dVn;
            c2 = (3.0 * mm - n - dV) * idR;
            c3 = (n - 2.0 * mm) * idR * idR;
        }
        t[iR] = (float)R2[iR];
        t[nR + iR] = (float)c0[iR];
        t[2 * nR + iR] = (float)c1[iR];
        t[3 * nR + iR] = (float)c2;
        t[4 * nR + iR] = (float)c3;
    }
}

// Coefficients of element Z for potential_type `type` (set_*_neutral_coef,
// src/atomic_data.hpp:1303-1486) and the rn_c of To_atom_type_CPU (src/atomic_data.hpp:148-176)
ElemCoef element_coef(int Z, int type, int charge = 0) {
    ElemCoef e{};
    const int iZ = Z - 1;
    for (int j = 0; j < 6; j++) {
        e.Vrcl[j] = e.VRcl[j] = 0.0;
        e.Vrcnl[j] = e.VRcnl[j] = 1.0;
    }
    auto zero = [](double v) { return std::fabs(v) <= 1e-13; };
    const PengIon* ion = find_ion(Z, charge);
    if (ion && !zero(ion->cl[0]) && !zero(ion->cnl[0])) {
        for (int j = 0; j < 5; j++) {
            double cl = ion->cl[j];
            double cnl = zero(cl) ? 0.0 : ion->cnl[j] / 4.0;
            if (zero(cl) || zero(cnl)) continue;
            e.Vrcl[j] = kPotf * cl * std::pow(kPi / cnl, 1.5);
            e.VRcl[j] = kPotf * kPi * cl / cnl;
            e.Vrcnl[j] = e.VRcnl[j] = kPi2 / cnl;
        }
        const double cl = charge / k2Pi2a0, cnl = std::pow(k2Pi * 2.0, -2.0);
        e.Vrcl[5] = kPotf * kPi * cl;
        e.VRcl[5] = kPotf * k2Pi * cl;
        e.Vrcnl[5] = e.VRcnl[5] = k2Pi * std::sqrt(cnl);
        type = kIonType;
    } else if (type == 6) {
        for (int j = 0; j < 5; j++) {
            double cl = kLobatoCl[iZ][j];
            double cnl = zero(cl) ? 0.0 : kLobatoCnl[iZ][j];
            if (!zero(cl) && !zero(cnl)) {
                e.Vrcl[j] = kPotf * kPi2 * cl / std::pow(cnl, 1.5);
                e.Vrcnl[j] = k2Pi / std::sqrt(cnl);
                e.VRcl[j] = 2.0 * kPotf * kPi2 * cl / std::pow(cnl, 1.5);
                e.VRcnl[j] = k2Pi / std::sqrt(cnl);
            }
        }
    } else {
        const double* fcl = kFegCl[type - 1][iZ];
        const double* fcnl = kFegCnl[type - 1][iZ];
        for (int j = 0; j < gauss_end(type); j++) {
            double cl = fcl[j];
            double cnl = zero(cl) ? 0.0 : (type == 4 ? fcnl[j] : fcnl[j] / 4.0);
            if (zero(cl) || zero(cnl)) continue;
            if (j < gauss_first(type)) {  // Kirkland's Yukawa terms
                e.Vrcl[j] = kPotf * kPi * cl;
                e.VRcl[j] = kPotf * k2Pi * cl;
                e.Vrcnl[j] = e.VRcnl[j] = k2Pi * std::sqrt(cnl);
            } else {
                e.Vrcl[j] = kPotf * cl * std::pow(kPi / cnl, 1.5);
                e.VRcl[j] = kPotf * kPi * cl / cnl;
                e.Vrcnl[j] = e.VRcnl[j] = kPi2 / cnl;
            }
        }
    }
    e.rn_c = 1.2e-05 * std::pow((double)kMassNumber[iZ], 1.0 / 3.0);
    e.ra = kAtomicRadius[iZ];
    e.type = type;
    return e;
}

}  // namespace

// 3-D potential Vr(r) of the element (Vr_Lobato_neutral_0_12, src/cgpu_fcns.cuh:1111-1120; the
// Gaussian and Yukawa sums of Vr_Doyle/Peng/Kirkland_neutral_*, src/cgpu_fcns.cuh:1023-1070)
static double vr_host(double x, const ElemCoef& c) {
    double ix = 1.0 / x, y = 0;
    if (c.type == 6) {
        for (int i = 0; i < 5; i++) y += c.Vrcl[i] * std::exp(-c.Vrcnl[i] * x) * ix * (2.0 / c.Vrcnl[i] + x);
        return y;
    }
    if (c.type == 4)
        for (int i = 0; i < 3; i++) y += c.Vrcl[i] * std::exp(-c.Vrcnl[i] * x) * ix;
    for (int i = gauss_first(c.type); i < gauss_end(c.type); i++) y += c.Vrcl[i] * std::exp(-c.Vrcnl[i] * (x * x));
    return y;
}

bool potential_type_supported(int type) { return (type >= 1 && type <= 4) || type == 6; }

int effective_charge(int Z, int charge) {
    const PengIon* ion = find_ion(Z, charge);
    return (ion && !(std::fabs(ion->cl[0]) <= 1e-13) && !(std::fabs(ion->cnl[0]) <= 1e-13)) ? charge : 0;
}

TableHead element_head(int Z, int type, float dR_min, float Vrl_f) {
    if (!potential_type_supported(type)) fail(MT_ERR_UNSUPPORTED, "potential_type " + std::to_string(type) + " has no table build");
    const ElemCoef c = element_coef(Z, type);
    const double Vrl = (double)Vrl_f;
    const double R_min = std::fmax(c.rn_c, (double)dR_min);
    double R_max = 0;
    const bool nonzero = !(std::fabs(Vrl) <= 1e-13) && !(std::fabs(c.Vrcl[0]) <= 1e-13);
    if (nonzero) {
        // Root_Finder (src/cgpu_fcns.cuh:262-286): bisection on [rn_c, 25], |f| <= 1e-8 or 200 steps
        double x0 = c.rn_c, xe = 25.0, x = 0, fx;
        double fxe = vr_host(xe, c) - Vrl;
        int it = 0;
        do {
            x = 0.5 * (x0 + xe);
            fx = vr_host(x, c) - Vrl;
            if (fx * fxe < 0) {
                x0 = x;
            } else {
                xe = x;
                fxe = fx;
            }
            it++;
        } while ((std::fabs(fx) > 1e-8) && (it < 200));
        R_max = x;
    }
    R_max = std::fmax(R_max, 2.0 * R_min);
    if (std::fabs(R_max) <= 1e-13) R_max = 1.75 * c.ra;
    const double R_tap = R_min + 0.85 * (R_max - R_min);
    const double tap_cf = kHalfPi / (std::pow(R_max, 2) - std::pow(R_tap, 2));
    return TableHead{R_min, R_max, R_tap, tap_cf};
}

void build_tables(const std::vector<int>& Zs, int type, const std::vector<TableHead>& heads, int nR, float* d_tab,
                  cudaStream_t stream, const std::vector<int>& charges) {
    const int n = (int)Zs.size();
    std::vector<ElemCoef> h(n);
    for (int i = 0; i < n; i++) h[i] = element_coef(Zs[i], type, charges.empty() ? 0 : charges[i]);
    int dev = 0;
    auto* d_coef = static_cast<ElemCoef*>(dev_alloc(sizeof(ElemCoef) * n, &dev));
    auto* d_head = static_cast<TableHead*>(dev_alloc(sizeof(TableHead) * n, &dev));
    MTB_CUDA(cudaMemcpyAsync(d_coef, h.data(), sizeof(ElemCoef) * n, cudaMemcpyHostToDevice, stream));
    MTB_CUDA(cudaMemcpyAsync(d_head, heads.data(), sizeof(TableHead) * n, cudaMemcpyHostToDevice, stream));
    build_tables_kernel<<<n, 128, 3 * nR * sizeof(double), stream>>>(d_coef, d_head, n, nR, d_tab);
    MTB_CUDA(cudaGetLastError());
    MTB_CUDA(cudaStreamSynchronize(stream));
    dev_free_idle(d_coef, dev);  // only `stream` used them
    dev_free_idle(d_head, dev);
}

// ---------------------------------------------------------------------------------------------
// Allocation-free variant of build_tables.
//
// The per-call scratch of build_tables (the element coefficients and table heads the kernel reads)
// lives here in one file-scope device array instead of memory allocated from the device pool. The
// array is kNoAllocMaxElements * (sizeof(ElemCoef) + sizeof(TableHead)) bytes (about 32 KB) and is
// held by every GPU that loads this library until the process exits. All calls share it: each
// call overwrites the entries it uses before its kernel reads them (nothing has to start at zero),
// and two calls whose fills and kernels overlap on the GPU (different streams, or different host
// threads on one device) race on it.
//
// The host-side values reach the scratch array as kernel parameters (noalloc_fill_kernel, a few
// elements per launch), not through a host-to-device copy: the call then neither blocks on a
// pageable-memory copy nor leaves a copy reading host memory that goes away when the call returns.
constexpr int kNoAllocMaxElements = 128;
static __device__ __align__(256) unsigned char
    g_noalloc_table_scratch[kNoAllocMaxElements * (sizeof(ElemCoef) + sizeof(TableHead))];

// Elements per fill launch: their coefficients and heads travel in the launch's parameter block,
// kept well inside the classic 4 KB parameter limit.
constexpr int kNoAllocFillChunk = 12;
struct NoAllocChunk {
    ElemCoef coef[kNoAllocFillChunk];
    TableHead head[kNoAllocFillChunk];
    int first, count;
};
static_assert(sizeof(NoAllocChunk) < 4000, "fill chunk must fit a kernel parameter block");

__global__ void noalloc_fill_kernel(const __grid_constant__ NoAllocChunk ch, ElemCoef* coef, TableHead* head) {
    for (int i = threadIdx.x; i < ch.count; i += blockDim.x) {
        coef[ch.first + i] = ch.coef[i];
        head[ch.first + i] = ch.head[i];
    }
}

// Device address of the scratch array on the current device. Host code may not use the symbol
// itself (it names a host-side stand-in, not device memory). The address is looked up with
// cudaGetSymbolAddress once per device, with that device current, and cached together with the
// CUDA context it was taken in; a call made in another context (the device's primary context
// destroyed and created anew) looks it up again.
using CtxGetCurrentFn = int (*)(void**);
static void* current_context() {
    static CtxGetCurrentFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        MTB_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !f) fail(MT_ERR_CUDA, "cuCtxGetCurrent is not available");
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    void* ctx = nullptr;
    if (fn(&ctx) != 0) fail(MT_ERR_CUDA, "cuCtxGetCurrent failed");
    return ctx;
}

static unsigned char* noalloc_scratch_address(int dev) {
    constexpr int kMaxDevices = 64;
    static unsigned char* addr[kMaxDevices] = {};
    static void* ctx_of[kMaxDevices] = {};
    static std::mutex mu;
    if (dev < 0 || dev >= kMaxDevices) fail(MT_ERR_INVALID_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(mu);
    // before the runtime's first call on this device no context is current (NULL): the lookup
    // below then creates the primary context and the cache records it
    void* ctx = current_context();
    if (!addr[dev] || !ctx || ctx_of[dev] != ctx) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_table_scratch);
        if (e != cudaSuccess) throw Error(MT_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        addr[dev] = static_cast<unsigned char*>(p);
        ctx_of[dev] = current_context();
    }
    return addr[dev];
}

void build_tables_noalloc(const std::vector<int>& Zs, int type, const std::vector<TableHead>& heads, int nR,
                          float* d_tab, cudaStream_t stream, const std::vector<int>& charges) {
    const int n = (int)Zs.size();
    if (n < 1 || n > kNoAllocMaxElements)
        fail(MT_ERR_INVALID_ARG, "allocation-free table build takes 1.." + std::to_string(kNoAllocMaxElements) +
                                     " elements, got " + std::to_string(n));
    if (nR < 2 || nR > 1024) fail(MT_ERR_INVALID_ARG, "nR must be in 2..1024");
    int dev = 0;
    MTB_CUDA(cudaGetDevice(&dev));
    unsigned char* base = noalloc_scratch_address(dev);
    ElemCoef* d_coef = reinterpret_cast<ElemCoef*>(base);
    TableHead* d_head = reinterpret_cast<TableHead*>(base + kNoAllocMaxElements * sizeof(ElemCoef));
    for (int i0 = 0; i0 < n; i0 += kNoAllocFillChunk) {
        NoAllocChunk ch{};
        ch.first = i0;
        ch.count = n - i0 < kNoAllocFillChunk ? n - i0 : kNoAllocFillChunk;
        for (int i = 0; i < ch.count; i++) {
            ch.coef[i] = element_coef(Zs[i0 + i], type, charges.empty() ? 0 : charges[i0 + i]);
            ch.head[i] = heads[i0 + i];
        }
        noalloc_fill_kernel<<<1, 32, 0, stream>>>(ch, d_coef, d_head);
        MTB_CUDA(cudaGetLastError());
    }
    build_tables_kernel<<<n, 128, 3 * nR * sizeof(double), stream>>>(d_coef, d_head, n, nR, d_tab);
    MTB_CUDA(cudaGetLastError());
}

}  // namespace mtb
