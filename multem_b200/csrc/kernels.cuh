// Device kernels of the multislice engine and their launch wrappers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace mtb {

constexpr int kMaxDet = 8;
constexpr int kMaxTypes = 16;

// Grid_2d<float> fields the kernels use (src/types.cuh:2107-2655).
struct GridDev {
    int nx, ny, nxh, nyh;
    float lx, ly, dRx, dRy, Rx_0, Ry_0, dgx, dgy;
};

// ---- projected potential + transmission (splat) ----
struct SplatArgs {
    GridDev g;
    const float4* atoms;       // (x, y, occ, type index as int bits), z-sorted
    const int2* slice_range;   // per slice (iatom_0, iatom_e), empty when iatom_0 > iatom_e
    const float* tab;          // per type 5*nR floats: R2, c0, c1, c2, c3
    const float* R_max;        // per type (float)
    int n_types;
    int nR;
    float w;                   // Vr_factor: T = exp(i*w*V)
    int wpo;                   // weak phase object: T = 1 + i*w*V
    float2* trans;             // [n_slice][nx*ny] or null
    float* V;                  // [n_slice][nx*ny] or null
};
void launch_splat(const SplatArgs& a, int islice_0, int n_slice, cudaStream_t s);

// ---- line passes ----
// Contiguous-line (y) pass modes.
enum RowMode : int {
    ROW_STEP = 0,       // load hybrid, inverse FFT_y, * T, forward FFT_y, store
    ROW_FIRST_ONE = 1,  // psi = 1 (plane wave), * T, forward FFT_y, store
    ROW_FIRST_REAL = 2, // load real-space psi, * T, forward FFT_y, store
    ROW_INVERSE = 3     // load hybrid, inverse FFT_y, * scale, store (real-space output)
};
struct RowArgs {
    const float2* in;
    float2* out;
    const float2* trans;   // [nx*ny] of the slice
    size_t trans_stride;   // elements between the transmission functions of consecutive waves of the
                           // batch (0: one function shared by every wave, as for STEM probes)
    int nx;                // lines per probe
    int nprobe;
    float scale;
    int* err;              // device flag, set when a bounded wait inside the pass gives up
    long long wait_ns;     // bound of each wait for a bulk copy (0: a copy not landed at the first check times out)
    int shape;             // pipeline shape of the bulk-copy-fed step pass (0 default, 1 or 2 alternatives)
};
void launch_rows(int ny, RowMode mode, const RowArgs& a, int grid_ctas, cudaStream_t s);

// Strided-line (x) pass modes (bit flags).
enum ColFlags : int {
    COL_LOAD = 1,      // load hybrid and forward FFT_x (else generate the probe)
    COL_PROP = 2,      // multiply by Px[ix]*Py[iy]
    COL_DETECT = 4,    // ring sums of |psi_hat|^2 into partials
    COL_INVERSE = 8,   // inverse FFT_x before the store
    COL_STORE = 16,    // store the result
    COL_P2 = 32        // with COL_PROP: also multiply by P2[ix][iy] (set from ColArgs::P2 by the launcher)
};
struct ProbeDev {
    float c_c_10, c_c_30, c_c_50;
    float g2_min, g2_max;
    float gxu, gyu;
    float norm;
    int phi_required;
    // phi-dependent aberrations (c_c_xx, phi_xx) and vortex momentum
    float c_c_12, phi_12, c_c_21, phi_21, c_c_23, phi_23, c_c_32, phi_32, c_c_34, phi_34;
    float c_c_41, phi_41, c_c_43, phi_43, c_c_45, phi_45, c_c_52, phi_52, c_c_54, phi_54, c_c_56, phi_56;
    int m;
    int nz_c10, nz_c30, nz_c50;
};
struct ColArgs {
    const float2* in;
    float2* out;
    int ny;                    // line stride (elements) and number of columns
    int nprobe;
    GridDev g;
    const float2* Px;          // [nx] propagator factor along x (includes 1/N)
    const float2* Py;          // [ny]
    const float2* P2;          // optional [nx][ny] factor applied after Px * Py (HRTEM transfer function)
    // probe generation
    const float2* beam;        // per probe (x, y) = exp_factor_R(beam position)
    ProbeDev probe;
    // detectors
    int n_det;
    float det_g2_min[kMaxDet], det_g2_max[kMaxDet];
    const float* det_mat;      // matrix detectors: [n_det][nx][ny] sensitivity in FFT order, else NULL
    float2* coh;               // coherent part: [nprobe][nx][ny] sums of coh_w * psi_hat, else NULL
    float coh_w;
    float gx_0, gy_0;
    double* det_partial;       // [nprobe][ny / det_w][n_det]
    int det_w;                 // columns per detector partial (col_det_width)
    int* err;                  // device flag, set when a bounded wait inside the pass gives up
    long long wait_ns;         // bound of each wait for a bulk copy (0: a copy not landed at the first check times out)
    int shape;                 // pipeline shape of the bulk-copy-fed step pass (0 default, 1 or 2 alternatives)
};
void launch_cols(int nx, int flags, const ColArgs& a, int grid_ctas, cudaStream_t s);
int col_det_width(int nx);      // columns per detector partial
int col_tiles(int nx, int ny);  // detector partials per probe per detector (ny / col_det_width)

// Sum detector partials over tiles and add w * sum into image[(idet*n_scan) + scan_index].
void launch_det_reduce(const double* partial, int nprobe, int n_tiles, int n_det, const int* scan_index,
                       double w, double* image, int n_scan, cudaStream_t s);

// HRTEM transfer functions over the Fourier grid ([ix][iy], FFT order): exp_i_chi of `lens` (apply_CTF,
// src/cgpu_fcns.cuh:1995-2006), or the partially coherent one with temporal and spatial envelopes
// (apply_PCTF, :2010-2040).
struct PctfArgs {
    float g2_min, g2_max, c_c_10, c_c_30, c_10, c_30, lambda, lambda2, si_theta_c, ti_iehwgd;
};
void launch_ctf_table(const ProbeDev& lens, const GridDev& g, float2* out, cudaStream_t s);
void launch_pctf_table(const PctfArgs& p, const GridDev& g, float2* out, cudaStream_t s);

// Output phase ramp of a tilted beam, / ny, [ix][iy]: exp(i (gx Rx + gy Ry)) with Rx = Rx_shift(ix) -
// rxc (two rounded products and a rounded sum in float, the phase's sine and cosine in double).
void launch_tilt_ramp(const GridDev& g, float gx, float gy, float rxc, float ryc, float2* out, cudaStream_t s);

// a[i] *= b[i] (complex), n values.
void launch_mul_tables(float2* a, const float2* b, size_t n, cudaStream_t s);

// dst = sum over j < n of src[j * nxy + i] (the beams of a convergent incident wave, in order).
void launch_sum_waves(const float2* src, int n, size_t nxy, float2* dst, cudaStream_t s);
// dst[i] += w * src[i], i < nxy
void launch_axpy_wave(const float2* src, float w, size_t nxy, float2* dst, cudaStream_t s);

// STEM coherent images (Wave_Function::set_m2psi_coh, src/wave_function.cuh:189-209): for each
// thickness and scan position, the detector sums of |psi_coh|^2 (weight 1) into
// image_coh[(ithk*n_det + idet)*n_scan + iscan]; coh is [n_thk][n_scan][nx][ny] in FFT order.
void launch_coh_detect(const float2* coh, int n_thk, int n_scan, const ColArgs& det, double* image_coh,
                       cudaStream_t s);

// EW output: out[(ix-ix0)*oy + (iy-iy0)] accumulates psi (complex) and |psi|^2 over the output
// area after an fft-shift by (nx/2, ny/2) (add_scale_crop_shift_2d, src/cgpu_fcns.cuh:1701-1739).
// With nwave > 1 (ISTEM) the |psi|^2 of nwave consecutive waves are summed in order (m2 only).
void launch_ew_accumulate(const float2* psi, int nx, int ny, int ix0, int ix1, int iy0, int iy1, double w,
                          int assign, double* psi_out, double* m2_out, cudaStream_t s, int nwave = 1);

// Device-side counters of this library's launches (for reporting).
long long launches_issued();
void add_launches(long long n);

// ---- frozen-phonon displacements on the device (phonon.cu) ----
// out[i] = base[i] with x, y moved by sigma[i] times two standard normals drawn from
// Philox4x32-10(key (seed, 0), counter (i, iconf, 0, 0)) through Box-Muller; z is never displaced.
void launch_phonon_displace(const float4* base, const float* sigma, int n, uint32_t seed, int iconf, bool pn_x,
                            bool pn_y, float4* out, cudaStream_t s);
// Philox4x32-10 of n (counter, key) pairs, for checking the generator against published vectors.
void launch_philox(const uint4* ctr, const uint2* key, int n, uint4* out, cudaStream_t s);

}  // namespace mtb
