/*
 * multem_b200 — C ABI of a B200-native multislice engine.
 *
 * This is the drop-in boundary for MULTEM's plain multislice loop. It replaces the reference's
 * entry points:
 *   - mexFunction / run_multislice           mex_files_multem/ilc_multem.cu:484-546
 *   - read_input_multislice (field parsing)  mex_files_multem/ilc_multem.cu:38-379
 *   - set_struct_multislice (output packing) mex_files_multem/ilc_multem.cu:382-481
 *   - mt_run_multislice / mt_stop_multislice / mt_niter / mt_iter   gui_multem/multem.cu:28-138
 *   - Multislice<T,dev>::set_input_data + operator()                src/tem_simulation.cuh:51-97
 *   - the operator-level MEX entries ilc_projected_potential, ilc_transmission_function,
 *     ilc_propagate, ilc_incident_wave (mex_files_multem/ilc_*.cu)
 *
 * Conventions kept identical to the reference so a thin MATLAB/Python shim maps 1:1:
 *   - field names follow the MATLAB input class matlab_functions/+multem_input/parameters.m;
 *   - enum codes are the reference's (src/types.cuh:137-310), e.g. simulation_type 11 = STEM,
 *     52 = EWRS; potential_type 1-4, 6 (1 Doyle-Turner, 2/3 Peng, 4 Kirkland, 6 Lobato); potential_slicing 1 = planes, 2 = dz_Proj;
 *     pn_model 3 = frozen phonon; pn_dim 110 = x,y;
 *   - units are the MATLAB input's: lengths in Angstrom, E_0 in keV, theta/phi and lens azimuths in
 *     degrees, apertures and detector angles in mrad, c_30/c_50 in mm;
 *   - 2-D arrays are column-major (MATLAB order, element (iy, ix) at ix*ny + iy);
 *   - spec_atoms is the reference's n x 8 column-major matrix [Z x y z sigma occ region charge]
 *     (src/atomic_data_mt.hpp:769-787); fewer columns use the reference's defaults.
 *
 * Every call returns an mt_status; mt_last_error() gives a message for the calling thread.
 * Inputs are never modified. Handles are independent and may be used from different threads.
 */
#ifndef MULTEM_B200_H
#define MULTEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MT_ABI_VERSION 1

typedef enum mt_status {
    MT_OK = 0,
    MT_ERR_INVALID_ARG = 1,  /* bad or inconsistent input */
    MT_ERR_OOM = 2,          /* device or host allocation failed */
    MT_ERR_CUDA = 3,         /* CUDA runtime error */
    MT_ERR_CANCELLED = 4,    /* mt_multislice_cancel() was called */
    MT_ERR_TIMEOUT = 5,      /* a bounded device wait ran out */
    MT_ERR_UNSUPPORTED = 6,  /* valid reference input outside what this engine implements */
    MT_ERR_INTERNAL = 7
} mt_status;

/* Simulation types (src/types.cuh eTEM_Sim_Type). */
enum { MT_SIM_STEM = 11, MT_SIM_ISTEM = 12, MT_SIM_CBED = 21, MT_SIM_CBEI = 22, MT_SIM_ED = 31,
       MT_SIM_HRTEM = 32, MT_SIM_PED = 41, MT_SIM_HCTEM = 42, MT_SIM_EWFS = 51, MT_SIM_EWRS = 52,
       MT_SIM_EELS = 61, MT_SIM_EFTEM = 62, MT_SIM_IWFS = 71, MT_SIM_IWRS = 72, MT_SIM_PPFS = 81,
       MT_SIM_PPRS = 82, MT_SIM_TFFS = 91, MT_SIM_TFRS = 92, MT_SIM_PROPFS = 101, MT_SIM_PROPRS = 102 };

/* System configuration: mirrors System_Configuration (src/types.cuh:4447-4520) and the MATLAB
 * system_conf struct read by read_system_conf (src/matlab_mex.cuh:263-288).
 * precision 1 = float, 2 = double; device 1 = host, 2 = device (GPU). This engine computes the
 * multislice loop in FP32 on the GPU; precision 2 or device 1 are rejected (MT_ERR_UNSUPPORTED). */
typedef struct mt_system_conf {
    int precision;
    int device;
    int cpu_nthread;
    int gpu_device;
} mt_system_conf;

/* Lens parameters: cond_lens_* / obj_lens_* fields of the MATLAB input
 * (read at mex_files_multem/ilc_multem.cu:155-268; Lens<T> in src/types.cuh:2824-3296). */
typedef struct mt_lens {
    int m;
    double c_10, c_12, phi_12;
    double c_21, phi_21, c_23, phi_23;
    double c_30, c_32, phi_32, c_34, phi_34;
    double c_41, phi_41, c_43, phi_43, c_45, phi_45;
    double c_50, c_52, phi_52, c_54, phi_54, c_56, phi_56;
    double inner_aper_ang, outer_aper_ang;
    double ti_a, ti_sigma, ti_beta;
    int ti_npts;
    double si_a, si_sigma, si_beta;
    int si_rad_npts, si_azm_npts;
    int zero_defocus_type;       /* 1 first, 2 middle, 3 last, 4 user defined */
    double zero_defocus_plane;
} mt_lens;

/* Input: the fields of Input_Multislice that the plain multislice path reads
 * (src/input_multislice.cuh:456-535, filled by mex_files_multem/ilc_multem.cu:38-379). */
typedef struct mt_input_multislice {
    int simulation_type;
    int interaction_model;       /* 1 multislice, 2 phase object, 3 weak phase object */
    int potential_type;          /* 1 Doyle-Turner (0-4), 2 Peng (0-4), 3 Peng (0-12), 4 Kirkland (0-12),
                                    6 Lobato (0-12); 5 Weickenmeier-Kohl is refused */
    int operation_mode;
    int reverse_multislice;

    int pn_model;                /* 1 still atom, 2 absorptive, 3 frozen phonon */
    int pn_coh_contrib;
    int pn_single_conf;
    int pn_nconf;
    int pn_dim;                  /* 110, 111, ... */
    int pn_seed;
    /* phonon generator (no counterpart in the reference): 0 = the reference's own draws on the host
     * (mt19937_64 + std::normal_distribution, the configurations MULTEM simulates; default),
     * 1 = counter-based draws on the GPU (Philox4x32-10 + Box-Muller from pn_seed, configuration and
     * atom index: the same displacement statistics, different configurations, no host work per
     * configuration) */
    int pn_rng;

    const double* spec_atoms;    /* column-major spec_atoms_rows x spec_atoms_cols */
    int spec_atoms_rows;
    int spec_atoms_cols;
    double spec_lx, spec_ly, spec_lz, spec_dz;
    int spec_cryst_na, spec_cryst_nb, spec_cryst_nc;
    double spec_cryst_a, spec_cryst_b, spec_cryst_c, spec_cryst_x0, spec_cryst_y0;
    int spec_amorp_n;            /* amorphous layers (z_0, z_e, dz), spec_amorp_n entries each */
    const double* spec_amorp_z_0;
    const double* spec_amorp_z_e;
    const double* spec_amorp_dz;
    double spec_rot_theta;       /* degrees */
    double spec_rot_u0[3];
    int spec_rot_center_type;
    double spec_rot_center_p[3];

    int thick_type;              /* 1 whole specimen, 2 through thickness, 3 through slices */
    const double* thick;
    int n_thick;

    int potential_slicing;       /* 1 planes, 2 dz_Proj */

    int nx, ny;
    int bwl;

    int iw_type;                 /* 1 plane, 2 convergent, 3 user defined, 4 auto */
    const double* iw_psi;        /* user-defined wave: interleaved (re, im), column-major ny x nx */
    const double* iw_x;
    const double* iw_y;
    int n_iw_xy;

    double E_0;                  /* keV */
    double theta, phi;           /* degrees */
    /* precession (PED, simulation_type 41) and hollow-cone illumination (HCTEM, 42): beam tilt in
     * degrees and number of azimuthal rotations (ilc_multem.cu:338-347) */
    double ped_theta, hci_theta;
    int ped_nrot, hci_nrot;

    int illumination_model;
    int temporal_spatial_incoh;

    mt_lens cond_lens;
    mt_lens obj_lens;

    int scanning_type;           /* 1 line, 2 area */
    int scanning_periodic;
    int scanning_square_pxs;
    int scanning_ns;
    double scanning_x0, scanning_y0, scanning_xe, scanning_ye;

    int detector_type;           /* 1 circular, 3 matrix */
    int n_detector;
    const double* detector_inner_ang;   /* type 1: mrad */
    const double* detector_outer_ang;   /* type 1: mrad */
    /* type 3: n_detector sensitivity maps over the Fourier grid, centred (zero frequency at
     * (nx/2, ny/2)) as the reference's detector.matrix(d).fR; value (ix, iy) of map d at
     * [(d * nx + ix) * ny + iy] (ilc_multem.cu:316-335) */
    const double* detector_fR;

    int output_area_ix_0, output_area_iy_0, output_area_ix_e, output_area_iy_e;  /* 1-based */
} mt_input_multislice;

/* Output sizes, from mt_output_query(). */
typedef struct mt_output_dims {
    int n_thick;                 /* thicknesses reported */
    int n_detector;              /* STEM detectors (0 otherwise) */
    int nx, ny;                  /* output image size (scan raster for STEM, output area otherwise) */
    int has_image_tot;           /* STEM: image_tot[ithk][idet][ny*nx] */
    int has_image_coh;           /* STEM with pn_coh_contrib */
    int has_m2psi_tot;           /* EW/HRTEM-like: m2psi_tot[ithk][ny*nx] */
    int has_psi_coh;             /* EW: psi_coh[ithk][ny*nx] complex */
    int n_x, n_y;                /* lengths of the x and y coordinate arrays: the output grid's
                                    axes, or every scan position for a STEM area scan (as the
                                    reference's output x/y, src/output_multislice.hpp:1207-1245) */
    int has_m2psi_coh;           /* ED/CBED/PED/HRTEM/CBEI with pn_coh_contrib: m2psi_coh[ithk][ny*nx],
                                    the intensity of the configuration-averaged wave, or its image
                                    through the objective (set_m2psi_coh, src/wave_function.cuh:189-227) */
} mt_output_dims;

/* Output buffers, caller-owned, sized from mt_output_dims (set_struct_multislice,
 * mex_files_multem/ilc_multem.cu:382-481). Unused pointers may be NULL. Images are double, like
 * the MATLAB output; psi_coh is interleaved (re, im). */
typedef struct mt_output_multislice {
    double dx, dy;
    double* x;                   /* n_x */
    double* y;                   /* n_y */
    double* thick;               /* n_thick */
    double* image_tot;           /* n_thick * n_detector * ny * nx */
    double* image_coh;           /* n_thick * n_detector * ny * nx */
    double* m2psi_tot;           /* n_thick * ny * nx */
    double* psi_coh;             /* n_thick * ny * nx * 2 */
    double* m2psi_coh;           /* n_thick * ny * nx */
} mt_output_multislice;

typedef struct mt_engine mt_engine;

/* ---- version / errors ---- */
int mt_abi_version(void);
const char* mt_last_error(void);
/* Number of device allocations the library has made in this process (engine buffers and the
 * scratch of the operator-level calls all come from its per-device memory pools); no
 * counterpart in the reference. For callers that watch the library's allocations. */
mt_status mt_device_alloc_count(long long* count);

/* ---- whole simulation (ilc_multem / mt_run_multislice) ---- */

/* Sizes of the output a run of `in` produces (Output_Multislice::set_input_data,
 * src/output_multislice.hpp:415-520). Validates the input like validate_parameters
 * (src/input_multislice.cuh:622-796). */
mt_status mt_output_query(const mt_input_multislice* in, mt_output_dims* dims);

/* The values validate_parameters (src/input_multislice.cuh:622-796) changes without telling the
 * caller, for `in`: pn_seed below 1, pn_nconf, the z phonon displacement without subslicing,
 * requested thicknesses matched to slice planes, atoms beyond the last thickness, a caller-given
 * output area that had to be reordered or clipped. Writes one line per change into buf (NUL
 * terminated, truncated to n bytes) and their number into *n_changes. Host only. No counterpart in
 * the reference, which applies them silently; with MTB_STRICT=1 in the environment the run entry
 * points fail with MT_ERR_INVALID_ARG instead of applying any of them. */
mt_status mt_input_report(const mt_input_multislice* in, char* buf, size_t n, int* n_changes);

/* One-shot run: create an engine on conf->gpu_device, run, copy results to `out`, destroy.
 * Equivalent of mt_run_multislice (gui_multem/multem.cu:28-50) / run_multislice
 * (mex_files_multem/ilc_multem.cu:484-518). */
mt_status mt_multislice_run(const mt_system_conf* conf, const mt_input_multislice* in,
                            mt_output_multislice* out);

/* Run n independent simulations (different specimens, grids, simulation types), each like
 * mt_multislice_run on in[i] -> out[i]. The reference runs one input per call
 * (mex_files_multem/ilc_multem.cu:484-546); this batched form has no counterpart there. Inputs are
 * taken largest first by several host workers, each with its own engine and CUDA stream on
 * conf->gpu_device, so small simulations overlap on the GPU (MTB_BATCH_WORKERS, default 4).
 * status[i] (optional) receives each run's status; the return value is MT_OK or the first failure
 * in input order, with mt_last_error() naming that input. */
mt_status mt_multislice_run_batch(const mt_system_conf* conf, int n, const mt_input_multislice* in,
                                  mt_output_multislice* out, mt_status* status);

/* ---- MATLAB files (level-5 MAT-files, MATLAB -v6 / -v7) ----
 * The file-level form of the MATLAB entry `output_multislice = ilc_multem(prms.system_conf, prms)`
 * (mex_files_multem/ilc_multem.cu:520-546, matlab_functions/+multem_input/parameters.m:247-250):
 * the input is the struct that multem_input.parameters.toStruct returns, saved with `save`
 * (read as read_input_multislice reads it, mex_files_multem/ilc_multem.cu:38-379; absent fields
 * take the class defaults); the output is the struct set_struct_multislice builds
 * (mex_files_multem/ilc_multem.cu:382-481). Big-endian, -v7.3 (HDF5), sparse and object values are
 * rejected with MT_ERR_INVALID_ARG. */
typedef struct mt_mat_input mt_mat_input;
/* Reads struct variable `var` (NULL or "": the first struct in the file) of the MAT-file at `path`
 * into *in (pointers into storage owned by *handle, valid until mt_mat_input_close) and, when conf
 * is not NULL, its system_conf field into *conf (defaults when the struct has none). Host only. */
mt_status mt_mat_input_open(const char* path, const char* var, mt_mat_input** handle, mt_system_conf* conf,
                            mt_input_multislice* in);
mt_status mt_mat_input_close(mt_mat_input* handle);
/* Writes the output of a run of `in` (sizes from mt_output_query) as the struct variable
 * "output_multislice" (or `var`) of a new MAT-file at `path`; compress != 0 writes -v7 (zlib)
 * elements. Host only. */
mt_status mt_mat_output_write(const char* path, const char* var, const mt_input_multislice* in,
                              const mt_output_multislice* out, int compress);
/* mt_mat_input_open + mt_multislice_run on the file's system_conf + mt_mat_output_write. */
mt_status mt_multislice_run_mat(const char* in_path, const char* var, const char* out_path, int compress);

/* Handle-based form: set-up once (tables, specimen, buffers), run many times.
 * mt_engine_create = Multislice::set_input_data (src/tem_simulation.cuh:51-69). */
mt_status mt_engine_create(const mt_system_conf* conf, const mt_input_multislice* in, mt_engine** eng);
/* Run all phonon configurations [fp_iconf_0, pn_nconf] (Multislice::operator(),
 * src/tem_simulation.cuh:71-97) and write the output. */
mt_status mt_engine_run(mt_engine* eng, mt_output_multislice* out);
/* Run a subset of phonon configurations [iconf_0, iconf_e] (1-based, inclusive) and accumulate
 * their weighted detector sums into the engine's FP64 accumulators without writing output. Used to
 * shard configurations over GPUs; mt_engine_read_stem() then returns the partial sums. */
mt_status mt_engine_run_confs(mt_engine* eng, int iconf_0, int iconf_e);
/* Zero the engine's accumulators. */
mt_status mt_engine_reset(mt_engine* eng);
/* STEM: copy the FP64 accumulators image_tot[ithk][idet][ny*nx] to host memory. */
mt_status mt_engine_read_stem(mt_engine* eng, double* image_tot, size_t n);
/* Cancel a run in progress from another thread (mt_stop_multislice, gui_multem/multem.cu:56-75).
 * The run returns MT_ERR_CANCELLED between launches. */
mt_status mt_engine_cancel(mt_engine* eng);
/* Bound (seconds, 0..60; default 2) of every wait of a line pass for the copies that feed it. A
 * wait that runs out sets the engine's error flag: the pass stops issuing copies, waits (bounded)
 * for those in flight and returns, later passes of the run return at once, and the run returns
 * MT_ERR_TIMEOUT; the engine stays usable. 0: a copy not yet landed at the first check times out
 * (a way to exercise the timeout path). No counterpart in the reference, whose GPU loop only
 * stops between probes (ext_stop_sim, src/tem_simulation.cuh:47,512). */
mt_status mt_engine_set_wait_limit(mt_engine* eng, double seconds);
/* Progress counters (mt_niter / mt_iter, gui_multem/multem.cu:98-138): iterations are
 * (configuration, probe batch) pairs. */
mt_status mt_engine_progress(mt_engine* eng, int* iter, int* niter);
/* Device-resident hot path for timing and sharding: run configurations [iconf_0, iconf_e] with all
 * specimen data already on the device (displaced atoms and slicing generated by
 * mt_engine_prepare_confs). No host<->device copies inside. */
mt_status mt_engine_prepare_confs(mt_engine* eng, int iconf_0, int iconf_e);
mt_status mt_engine_run_prepared(mt_engine* eng, int iconf_0, int iconf_e);
/* Number of kernel launches the last run issued (own kernels only). */
mt_status mt_engine_launch_count(mt_engine* eng, long long* n);
/* Line-pass variants in effect (no counterpart in the reference): bit 0 set = bulk-copy-fed row
 * pass, bit 1 = bulk-copy-fed column pass; chosen per grid and batch shape by the engine's
 * autotuner at the first run, or pinned by MTB_PIPE. All variants give bit-identical results. */
mt_status mt_engine_pass_variants(mt_engine* eng, int* variants);
/* The autotuner's full choice for the engine's grid (no counterpart in the reference, whose FFT
 * shapes come from cuFFT plans, src/fft.cuh:364-478): the variant of the row and of the column
 * pass of the slice step (0 per-thread loads, 1 bulk-copy fed, 2 and 3 bulk-copy fed in the two
 * alternative pipeline shapes: narrower groups, and early issue with full exchange buffers) and the
 * probes per launch; valid after a run. */
mt_status mt_engine_tuning(mt_engine* eng, int* rows_variant, int* cols_variant, int* probes_per_launch);
/* Device timing (no counterpart in the reference): with timing on, each run records CUDA events on
 * the engine's stream around the whole run and around every line-pass launch. mt_engine_timing
 * returns the last run's device time and the summed durations and counts of the contiguous-line
 * (rows) and strided-line (cols) passes. */
mt_status mt_engine_set_timing(mt_engine* eng, int on);
mt_status mt_engine_timing(mt_engine* eng, double* total_ms, double* rows_ms, long long* n_rows, double* cols_ms,
                           long long* n_cols);
mt_status mt_engine_destroy(mt_engine* eng);

/* ---- operator-level entries (ilc_projected_potential, ilc_transmission_function,
 *      ilc_propagate, ilc_incident_wave) ---- */

/* Projected potential of slice `islice` (0-based) of phonon configuration `iconf` (1-based):
 * V[ny*nx] column-major in the reference's stored layout, which is fft-shifted: pixel (iy, ix)
 * holds the potential at ((ix - nx/2) dx, (iy - ny/2) dy) modulo the box, exactly what
 * ilc_projected_potential returns (mex_files_multem/ilc_projected_potential.cu:134-160;
 * Projected_Potential::operator(), src/projected_potential.cuh:127-167). */
mt_status mt_projected_potential(const mt_system_conf* conf, const mt_input_multislice* in,
                                 int iconf, int islice, double* V);
/* Transmission function exp(i*sigma*V) of slice `islice`, same layout as V
 * (ilc_transmission_function.cu:152; Transmission_Function::trans,
 * src/transmission_function.cuh:54-85). trans: interleaved complex. */
mt_status mt_transmission_function(const mt_system_conf* conf, const mt_input_multislice* in,
                                   int iconf, int islice, double* trans);
/* Propagate the user wave in->iw_psi (iw_type 3) by distance z (ilc_propagate.cu:125-147, which
 * passes obj_lens_c_10 as z; Propagator::operator(), src/propagator.cuh:51-103). Reads only nx, ny,
 * spec_lx/ly, iw_psi, E_0, theta, phi. space 1 = real, 2 = reciprocal. psi_out: interleaved
 * complex, column-major like iw_psi. */
mt_status mt_propagate(const mt_system_conf* conf, const mt_input_multislice* in, int space,
                       double z, double* psi_out);
/* Incident wave at in->iw_x/iw_y (ilc_incident_wave.cu:154; Incident_Wave::operator(),
 * src/incident_wave.cuh:44-116). space 1 = real, 2 = reciprocal. psi_out: interleaved complex. */
mt_status mt_incident_wave(const mt_system_conf* conf, const mt_input_multislice* in, int space,
                           double* psi_out);

/* Radial projected-potential spline tables of the elements Z[0..n) built on the GPU in FP64
 * (Atomic_Data::get_atom_coef, src/atomic_data.hpp:1547-1668, Lobato 0-12, neutral atoms) for a
 * grid of minimum sampling dR_min and cut-off potential Vrl. heads[4*i..] = R_min, R_max, R_tap,
 * tap_cf; tab[5*nR*i..] = R2[nR], c0[nR], c1[nR], c2[nR], c3[nR] as float (the tables the
 * projected-potential splat evaluates). Host buffers. */
mt_status mt_spline_tables(const mt_system_conf* conf, const int* Z, int n, double dR_min, double Vrl, int nR,
                           double* heads, float* tab);
/* mt_spline_tables for the parameterisation `potential_type` (MULTEM's ePotential_Type): 1 Doyle-Turner
 * (0-4), 2 Peng (0-4), 3 Peng (0-12), 4 Kirkland (0-12) or 6 Lobato (0-12); the tables of
 * Atomic_Data::get_atom_coef built with that type (src/atomic_data.hpp:1303-1400, 1547-1668).
 * 5 (Weickenmeier-Kohl, no closed-form projected potential) returns MT_ERR_UNSUPPORTED.
 * charge (optional, NULL = neutral): the ionic charge of each entry; a charge with an entry in
 * Peng's ionic table (0-4) gets its ionic table (set_Peng_ions_coef, src/atomic_data.hpp:1489-1543,
 * whatever potential_type), any other charge the neutral one, as the reference.
 * mt_spline_tables is this call with potential_type 6 and no charges. */
mt_status mt_spline_tables_ex(const mt_system_conf* conf, int potential_type, const int* Z, const int* charge, int n,
                              double dR_min, double Vrl, int nR, double* heads, float* tab);

/* Allocation-free form of mt_spline_tables; it has no counterpart in the reference. It is for
 * callers that cannot call cudaMalloc: code whose GPU memory is owned by a framework's pool
 * allocator (an allocation outside the pool escapes its budget, or fails once the pool holds the
 * device's memory), and loops that must not allocate while they run. The caller passes the output:
 * d_tab is a device buffer of n*5*nR floats on the current device, laid out as mt_spline_tables'
 * tab; heads (optional) is a host buffer of 4*n doubles, written before the call returns. The only
 * scratch is a fixed 32 KB device array inside the library (held on every GPU that loads the
 * library until the process exits): n is limited to 128 elements and nR to 1024, larger requests
 * return MT_ERR_INVALID_ARG. The call allocates nothing (no cudaMalloc, cudaFree or pool
 * allocation). The element coefficients reach the scratch array as kernel parameters, so the work
 * is a few kernel launches on `stream` (a cudaStream_t, NULL for the legacy default stream),
 * complete when that stream is, and the call does not wait for the GPU. The first call on a device
 * looks up the scratch array's device address (cudaGetSymbolAddress) with that device current and
 * keeps it for that device's context. Calls share the scratch array: two calls that overlap on the
 * GPU (different streams or threads on one device) race on it. */
mt_status mt_spline_tables_noalloc(const int* Z, int n, double dR_min, double Vrl, int nR, double* heads,
                                   float* d_tab, void* stream);
/* mt_spline_tables_noalloc for `potential_type` (as mt_spline_tables_ex); mt_spline_tables_noalloc
 * is this call with potential_type 6. */
mt_status mt_spline_tables_noalloc_ex(int potential_type, const int* Z, const int* charge, int n, double dR_min,
                                      double Vrl, int nR, double* heads, float* d_tab, void* stream);

/* ---- specimen host logic, exposed for parity checks ---- */

/* Number of atoms kept after validation and the slice count for configuration `iconf`. */
mt_status mt_specimen_info(const mt_input_multislice* in, int iconf, int* n_atoms, int* n_slice,
                           int* n_thick);
/* Displaced, z-sorted atoms of configuration `iconf` (Spec::move_atoms, src/spec.hpp:85-127):
 * Z[n], xyz[3n] as (x, y, z) triples, in the working precision of the engine (float) widened to
 * double. */
mt_status mt_specimen_atoms(const mt_input_multislice* in, int iconf, int* Z, double* xyz, int n);
/* The atoms of configuration `iconf` as the engine simulates them, in mt_specimen_atoms' layout:
 * with pn_rng 0 the same as mt_specimen_atoms (no GPU); with pn_rng 1 the undisplaced atoms moved
 * in x and y by the device generator (a GPU call on conf->gpu_device). No counterpart in the
 * reference. */
mt_status mt_phonon_atoms(const mt_system_conf* conf, const mt_input_multislice* in, int iconf, int* Z,
                          double* xyz, int n);
/* Philox4x32-10 on the device, the generator of pn_rng 1: out[4i..4i+3] from counter ctr[4i..4i+3]
 * and key key[2i..2i+1], for checks against the published known-answer vectors. */
mt_status mt_philox4x32_10(const unsigned* ctr, const unsigned* key, int n, unsigned* out);
/* Slices of configuration `iconf` (Slicing::calculate, src/slicing.hpp:93-100):
 * z_0, z_e, iatom_0, iatom_e, ithk per slice. With pn_rng 1, the slicing of the undisplaced atoms,
 * which every device-generated configuration uses. */
mt_status mt_specimen_slices(const mt_input_multislice* in, int iconf, double* z_0, double* z_e,
                             int* iatom_0, int* iatom_e, int* ithk, int n);

#ifdef __cplusplus
}
#endif

#endif /* MULTEM_B200_H */
