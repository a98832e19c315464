// Host-side model of a multislice run: validated input, specimen, frozen-phonon displacements and
// slicing. This is the part of the reference's Input_Multislice / Spec / Slicing / Atom_Data logic
// that decides *what* is simulated (src/input_multislice.cuh, src/spec.hpp, src/slicing.hpp,
// src/atomic_data_mt.hpp, src/cgpu_rand.cuh). It is computed in the reference's float working
// precision, expression by expression, so atom positions, slice boundaries and the atom ranges of
// every slice come out identical to the reference's float path.
#pragma once

#include <cstdint>
#include <random>
#include <string>
#include <vector>

#include "multem_b200.h"

namespace mtb {

// Grid_2d<float> (src/types.cuh:2107-2655): sampling of the simulation box.
struct GridF {
    int nx = 0, ny = 0, nxh = 0, nyh = 0;
    float lx = 0, ly = 0, dz = 0;
    bool bwl = false, pbc_xy = true;
    float Rx_0 = 0, Ry_0 = 0;
    float dRx = 0, dRy = 0, dgx = 0, dgy = 0;
    float gl2_max = 0, alpha = 0;

    void set(int nx_, int ny_, float lx_, float ly_, float dz_, bool bwl_, bool pbc_);
    float dR_min() const { return dRx < dRy ? dRx : dRy; }
    float dg_min() const { return dgx < dgy ? dgx : dgy; }
    float g_max() const;
    float gl_max() const;
    float g2_max() const { float g = g_max(); return g * g; }
    float lxh() const { return 0.5 * lx; }
    float lyh() const { return 0.5 * ly; }
    float exp_factor_Rx(float x) const;
    float exp_factor_Ry(float y) const;
    float Rx(int ix) const { return (float)ix * dRx + Rx_0; }
    float Ry(int iy) const { return (float)iy * dRy + Ry_0; }
    float gx(int ix) const { return (float)(ix - nxh) * dgx; }
    float gy(int iy) const { return (float)(iy - nyh) * dgy; }
};

// Lens<float> (src/types.cuh:2824-3296): the coefficient subset the incident wave needs.
struct LensF {
    int m = 0;
    float c_10 = 0, c_12 = 0, phi_12 = 0, c_21 = 0, phi_21 = 0, c_23 = 0, phi_23 = 0;
    float c_30 = 0, c_32 = 0, phi_32 = 0, c_34 = 0, phi_34 = 0;
    float c_41 = 0, phi_41 = 0, c_43 = 0, phi_43 = 0, c_45 = 0, phi_45 = 0;
    float c_50 = 0, c_52 = 0, phi_52 = 0, c_54 = 0, phi_54 = 0, c_56 = 0, phi_56 = 0;
    float inner_aper_ang = 0, outer_aper_ang = 0;
    float si_sigma = 0;
    float si_a = 1, si_beta = 0;     // source spread (spatial incoherence): Gaussian share, exponential
    int si_rad_npts = 1, si_azm_npts = 1;
    float ti_a = 1, ti_sigma = 0, ti_beta = 0;  // defocus spread (temporal incoherence)
    int ti_npts = 1;
    int zero_defocus_type = 1;
    float zero_defocus_plane = 0;
    float lambda = 0;
    float c_c_10 = 0, c_c_12 = 0, c_c_21 = 0, c_c_23 = 0, c_c_30 = 0, c_c_32 = 0, c_c_34 = 0;
    float c_c_41 = 0, c_c_43 = 0, c_c_45 = 0, c_c_50 = 0, c_c_52 = 0, c_c_54 = 0, c_c_56 = 0;
    float g2_min = 0, g2_max = 0;

    void from_input(const mt_lens& l);
    void set_input_data(float E_0, const GridF& grid);
    void set_defocus(float f);
    float get_zero_defocus_plane(float z_min, float z_max) const;
    bool is_phi_required() const;
};

// Atom_Data<float> (src/atomic_data_mt.hpp:103-791): atoms plus the statistics slicing uses.
struct AtomsF {
    std::vector<int> Z;
    std::vector<float> x, y, z;
    std::vector<float> sigma, occ;
    std::vector<int> region, charge;
    float l_x = 0, l_y = 0, l_z = 0, dz = 0.25f;
    float z_min = 0, z_max = 0;
    float sigma_max = 0;
    float R_int_min = 0, R_int_max = 0;
    float z_int_min = 0, z_int_max = 0, s_z_int = 0;
    struct Amorp { float z_0, z_e, dz; int region; int type; };
    std::vector<Amorp> amorp;

    size_t size() const { return Z.size(); }
    void resize(size_t n);
    // get_statistic with per-element R_max (R_max_of_Z[Z-1]) or the 2.5 A default when null
    void statistic(const float* R_max_of_Z);
    void sort_by_z();
};

// Slice / Thick records (src/types.cuh Slice<T>, Thick<T>)
struct SliceF {
    float z_0, z_e, z_int_0, z_int_e;
    int iatom_0, iatom_e, ithk;
    float z_m() const { return 0.5f * (z_0 + z_e); }
};
struct ThickF {
    float z, z_zero_def_plane, z_back_prop;
    int islice, iatom_e;
};

// Everything a run needs, validated. Mirrors Input_Multislice::validate_parameters
// (src/input_multislice.cuh:622-796) for the paths this engine implements.
struct Model {
    // simulation switches
    int simulation_type = 52;
    int interaction_model = 1;
    int potential_type = 6;
    int pn_model = 1;
    int illumination_model = 1, temporal_spatial_incoh = 1;
    // defocus offsets (A) and weights of the condenser's temporal-incoherence quadrature; one
    // point (0, 1) unless STEM integrates the illumination in full
    std::vector<double> ti_x{0.0}, ti_w{1.0};
    // source-spread quadrature of CBED/CBEI under full integration: beam offsets (A) and weights
    std::vector<double> si_x{0.0}, si_y{0.0}, si_w{1.0};
    // HRTEM image formation (Microscope_Effects): 1 coherent CTF, 2 partially coherent CTF
    // (envelopes), 4 numerical integration over the objective's defocus spread; obj_c10 and obj_w
    // are the defocus and weight of each point (one point unless 4)
    int ctf_mode = 1;
    std::vector<float> obj_c10;
    std::vector<double> obj_w;
    bool pn_coh_contrib = false, pn_single_conf = false;
    int pn_nconf = 1, fp_iconf_0 = 1, pn_seed = 300183;
    int pn_rng = 0;  // 0 host draws of the reference, 1 counter-based draws on the device
    bool pn_x = true, pn_y = true, pn_z = false;
    int thick_type = 1;
    int potential_slicing = 1;
    int iw_type = 1;
    int mul_sign = 1;
    float E_0 = 300, lambda = 0, theta = 0, phi = 0;
    float Vrl = 0.015f;
    int nR = 128;

    GridF grid;
    LensF cond_lens, obj_lens;
    std::vector<float> thick;

    // incident wave
    std::vector<float> iw_x, iw_y;
    std::vector<float> iw_psi;  // interleaved complex, user-defined wave
    std::vector<std::string> clamps;  // values validate_parameters changed silently, as text

    // scanning (Scanning<float>::set_grid, src/types.cuh:4294-4390)
    int scan_type = 2;
    bool scan_pbc = false, scan_spxs = true;
    int scan_ns = 0, scan_nx = 0, scan_ny = 0;
    float scan_x0 = 0, scan_y0 = 0, scan_xe = 0, scan_ye = 0, scan_dRx = 0, scan_dRy = 0;
    std::vector<float> scan_x, scan_y;  // every scan position, index ix*ny + iy

    // circular detectors (g in 1/A, float)
    std::vector<float> det_g_inner, det_g_outer;  // one entry per detector (zeros for matrices)
    int det_type = 1;                              // 1 circular, 3 matrix
    std::vector<float> det_fR;                     // type 3: [d][ix][iy] in FFT order

    // output area (0-based, [ix_0, ix_e) x [iy_0, iy_e))
    int out_ix_0 = 0, out_ix_e = 0, out_iy_0 = 0, out_iy_e = 0;

    // specimen as given (after the z-range filter of validate_parameters)
    AtomsF atoms_in;

    bool is_multislice() const { return interaction_model == 1; }
    bool is_STEM() const { return simulation_type == 11; }
    bool is_ISTEM() const { return simulation_type == 12; }
    bool is_scanning() const { return is_STEM() || is_ISTEM(); }
    bool is_EWFS() const { return simulation_type == 51; }
    bool is_EWRS() const { return simulation_type == 52; }
    bool is_EW() const { return is_EWFS() || is_EWRS(); }
    bool is_CBED() const { return simulation_type == 21; }
    bool is_PED() const { return simulation_type == 41; }
    bool is_HCTEM() const { return simulation_type == 42; }
    bool is_CBEI() const { return simulation_type == 22; }
    bool is_ED() const { return simulation_type == 31; }
    bool is_HRTEM() const { return simulation_type == 32; }
    // one incident wave (plane, convergent beams summed, or user-defined) per configuration, and
    // per beam rotation for PED / HCTEM, through the slice loop
    bool is_wave_sim() const {
        return is_EW() || is_ED() || is_HRTEM() || is_CBED() || is_CBEI() || is_PED() || is_HCTEM();
    }
    // image formation through the objective lens (Microscope_Effects): HRTEM, CBEI, HCTEM, ISTEM
    bool is_imaging() const { return is_HRTEM() || is_CBEI() || is_HCTEM() || is_ISTEM(); }
    // outputs on the Fourier grid (is_grid_FS, src/input_multislice.cuh:367-372)
    bool is_grid_FS() const { return is_EWFS() || is_ED() || is_CBED() || is_PED(); }
    bool is_frozen_phonon() const { return pn_model == 3; }
    bool is_EW_SC() const { return is_EW() && is_frozen_phonon() && pn_single_conf; }
    bool is_plane_wave() const { return iw_type == 1; }
    bool is_convergent_wave() const { return iw_type == 2; }
    bool is_user_wave() const { return iw_type == 3; }
    int number_conf() const { return pn_nconf - fp_iconf_0 + 1; }
    int n_scan() const { return scan_nx * scan_ny; }
    float gx_0() const;
    float gy_0() const;
    bool tilted() const;
    // beam rotations of PED / HCTEM (nrot > 1): azimuth of rotation irot (Input_Multislice::set_phi,
    // src/input_multislice.cuh:903-906), and the tilt offsets there
    int nrot = 1;
    bool dp_shift = false;  // PED: the diffraction pattern is not shifted back (no output phase ramp)
    float rot_phi(int irot) const;
    float gx_0(int irot) const;
    float gy_0(int irot) const;
    bool ramp_needed(int irot) const;
    float Vr_factor() const;
    float propagator_factor(float z) const;
    float phonon_weight() const;
};

// Validate `in` like read_input_multislice + validate_parameters; throws mtb::Error.
Model build_model(const mt_input_multislice* in);
// Line lengths with a compiled FFT plan: 64, 128, 256, 384, 512, 1024, 2048.
bool line_size_supported(int n);
// The fields ilc_propagate reads (grid, user wave, E_0, tilt); throws mtb::Error.
Model build_prop_model(const mt_input_multislice* in);
void snap_incident_angle(Model& m);
void gauss_hermite(int n, std::vector<double>& x, std::vector<double>& w);
void temporal_quadrature(const LensF& L, std::vector<double>& x, std::vector<double>& w);
// Generalized Gauss-Laguerre rule of weight t exp(-t) on (0, inf) (alpha = 1): nodes and weights.
void gauss_laguerre1(int n, std::vector<double>& x, std::vector<double>& w);
void spatial_quadrature(const LensF& L, std::vector<double>& x, std::vector<double>& y, std::vector<double>& w);
void hrtem_ctf_points(Model& m);

// Per-element spline-table header needed on the host (R_max drives statistics and footprints).
struct AtomTypeHead {
    double R_min, R_max, R_tap, tap_cf;
};

// Specimen with frozen-phonon configurations: Spec<float> (src/spec.hpp:36-147).
class Specimen {
  public:
    // R_max_of_Z[103] comes from the spline tables (float R_max per element).
    Specimen(const Model& m, const std::vector<float>& R_max_of_Z);

    // Spec::move_atoms(fp_iconf): displace, (re)sort, statistics, slicing.
    void move_atoms(int iconf);
    // The undisplaced atoms with their statistics and slicing: the device phonon generator
    // displaces x and y only, so this slicing holds for every configuration.
    void still_atoms();
    const AtomsF& atoms_undisplaced() const { return atoms_u_; }

    const AtomsF& atoms() const { return atoms_; }
    const std::vector<SliceF>& slices() const { return slice_; }
    const std::vector<ThickF>& thicks() const { return thick_; }
    float dz(int islice) const;  // slice thickness / cos(theta)
    bool phase_object() const { return phase_object_; }

  private:
    const Model& m_;
    std::vector<float> R_max_of_Z_;
    AtomsF atoms_u_;   // undisplaced, z-sorted
    AtomsF atoms_;     // displaced
    std::vector<float> z_plane_;
    std::vector<float> z_slice_;
    std::vector<SliceF> slice_;
    std::vector<ThickF> thick_;
    bool phase_object_ = false;
    int thick_type_ = 1;  // the model's, changed to 2 when a through-slice run becomes a phase object
    float grid_dz_ = 0;

    void calculate();
};

}  // namespace mtb
