// Oracle driver around the reference's own CPU path (test and baseline infrastructure only).
//
// Built by oracle/Makefile from the reference sources where they lie, into oracle/_ref/. It fills
// the reference's Input_Multislice from the same POD struct the product's C ABI takes
// (include/multem_b200.h), following read_input_multislice (mex_files_multem/ilc_multem.cu:38-379)
// field by field, then runs the reference's Multislice<T, e_host> exactly as run_multislice
// (mex_files_multem/ilc_multem.cu:484-518) and the GUI entry mt_run_multislice
// (gui_multem/multem.cu:28-50) do. Extra entry points expose the reference's intermediate results
// (displaced atoms, slicing, projected potential, transmission, spline tables, incident wave,
// propagation) with the granularity of its operator-level MEX files (mex_files_multem/ilc_*.cu).
#include <mex.h>
#include "math.cuh"
#include "types.cuh"
#include "fft.cuh"
#include "stream.cuh"
#include "input_multislice.cuh"
#include "output_multislice.hpp"
#include "tem_simulation.cuh"
#include "propagator.cuh"

#include <cstring>
#include <stdexcept>
#include <exception>
#include <string>

#include "multem_b200.h"

namespace {

thread_local std::string g_err;

template <class T>
void fill_lens(const mt_lens& l, mt::Lens<T>& lens, T E_0, mt::Grid_2d<T>& grid) {
    lens.m = l.m;
    lens.c_10 = l.c_10;
    lens.c_12 = l.c_12;
    lens.phi_12 = l.phi_12 * mt::c_deg_2_rad;
    lens.c_21 = l.c_21;
    lens.phi_21 = l.phi_21 * mt::c_deg_2_rad;
    lens.c_23 = l.c_23;
    lens.phi_23 = l.phi_23 * mt::c_deg_2_rad;
    lens.c_30 = l.c_30 * mt::c_mm_2_Angs;
    lens.c_32 = l.c_32;
    lens.phi_32 = l.phi_32 * mt::c_deg_2_rad;
    lens.c_34 = l.c_34;
    lens.phi_34 = l.phi_34 * mt::c_deg_2_rad;
    lens.c_41 = l.c_41;
    lens.phi_41 = l.phi_41 * mt::c_deg_2_rad;
    lens.c_43 = l.c_43;
    lens.phi_43 = l.phi_43 * mt::c_deg_2_rad;
    lens.c_45 = l.c_45;
    lens.phi_45 = l.phi_45 * mt::c_deg_2_rad;
    lens.c_50 = l.c_50 * mt::c_mm_2_Angs;
    lens.c_52 = l.c_52;
    lens.phi_52 = l.phi_52 * mt::c_deg_2_rad;
    lens.c_54 = l.c_54;
    lens.phi_54 = l.phi_54 * mt::c_deg_2_rad;
    lens.c_56 = l.c_56;
    lens.phi_56 = l.phi_56 * mt::c_deg_2_rad;
    lens.inner_aper_ang = l.inner_aper_ang * mt::c_mrad_2_rad;
    lens.outer_aper_ang = l.outer_aper_ang * mt::c_mrad_2_rad;
    lens.ti_a = l.ti_a;
    lens.ti_sigma = l.ti_sigma;
    lens.ti_beta = l.ti_beta;
    lens.ti_npts = l.ti_npts;
    lens.si_a = l.si_a;
    lens.si_sigma = l.si_sigma;
    lens.si_beta = l.si_beta;
    lens.si_rad_npts = l.si_rad_npts;
    lens.si_azm_npts = l.si_azm_npts;
    lens.zero_defocus_type = static_cast<mt::eZero_Defocus_Type>(l.zero_defocus_type);
    lens.zero_defocus_plane = l.zero_defocus_plane;
    lens.set_input_data(E_0, grid);
}

// Mirrors read_input_multislice (mex_files_multem/ilc_multem.cu:38-379), reading from the POD
// struct instead of a MATLAB struct. The objective lens takes its source-spread fields from the
// cond_lens_* values, as the reference does at ilc_multem.cu:250-254.
template <class T>
void fill_input(const mt_input_multislice* in, mt::Input_Multislice<T>& im, int nthreads,
                mt::eDevice dev = mt::e_host) {
    im.system_conf.precision = std::is_same<T, float>::value ? mt::eP_float : mt::eP_double;
    im.system_conf.device = dev;
    im.system_conf.cpu_nthread = nthreads;
    if (dev == mt::e_device) {
        // read_system_conf (src/matlab_mex.cuh:263-288): one stream, the requested GPU
        im.system_conf.gpu_device = 0;
        im.system_conf.gpu_nstream = 0;
    }
    im.system_conf.validate_parameters();
    if (dev == mt::e_device) {
        if (!im.system_conf.is_device()) throw std::runtime_error("no GPU for the reference's device path");
        im.system_conf.set_device();
    }

    im.simulation_type = static_cast<mt::eTEM_Sim_Type>(in->simulation_type);
    im.interaction_model = static_cast<mt::eElec_Spec_Int_Model>(in->interaction_model);
    im.potential_type = static_cast<mt::ePotential_Type>(in->potential_type);
    im.operation_mode = static_cast<mt::eOperation_Mode>(in->operation_mode);
    im.reverse_multislice = in->reverse_multislice != 0;

    im.pn_model = static_cast<mt::ePhonon_Model>(in->pn_model);
    im.pn_coh_contrib = in->pn_coh_contrib != 0;
    im.pn_single_conf = in->pn_single_conf != 0;
    im.pn_nconf = in->pn_nconf;
    im.pn_dim.set(in->pn_dim);
    im.pn_seed = in->pn_seed;

    T lx = in->spec_lx, ly = in->spec_ly, lz = in->spec_lz, dz = in->spec_dz;
    bool pbc_xy = true;

    if (im.is_specimen_required()) {
        mt::Vector<mt::Amorp_Lay_Info<T>, mt::e_host> amorp(in->spec_amorp_n);
        for (int i = 0; i < in->spec_amorp_n; i++) {
            amorp[i].z_0 = in->spec_amorp_z_0[i];
            amorp[i].z_e = in->spec_amorp_z_e[i];
            amorp[i].dz = in->spec_amorp_dz[i];
        }
        im.atoms.set_crystal_parameters(in->spec_cryst_na, in->spec_cryst_nb, in->spec_cryst_nc, in->spec_cryst_a,
                                        in->spec_cryst_b, in->spec_cryst_c, in->spec_cryst_x0, in->spec_cryst_y0);
        im.atoms.set_amorphous_parameters(amorp);
        im.atoms.set_atoms(in->spec_atoms_rows, in->spec_atoms_cols, const_cast<double*>(in->spec_atoms), lx, ly,
                           lz, dz);

        im.spec_rot_theta = in->spec_rot_theta * mt::c_deg_2_rad;
        im.spec_rot_u0 = mt::r3d<T>(in->spec_rot_u0[0], in->spec_rot_u0[1], in->spec_rot_u0[2]);
        im.spec_rot_u0.normalized();
        im.spec_rot_center_type = static_cast<mt::eRot_Point_Type>(in->spec_rot_center_type);
        im.spec_rot_center_p =
            mt::r3d<T>(in->spec_rot_center_p[0], in->spec_rot_center_p[1], in->spec_rot_center_p[2]);

        im.thick_type = static_cast<mt::eThick_Type>(in->thick_type);
        if (!im.is_whole_spec()) {
            im.thick.assign(in->thick, in->thick + in->n_thick);
        }
        im.potential_slicing = static_cast<mt::ePotential_Slicing>(in->potential_slicing);
    }

    im.grid_2d.set_input_data(in->nx, in->ny, lx, ly, dz, in->bwl != 0, pbc_xy);

    im.set_incident_wave_type(static_cast<mt::eIncident_Wave_Type>(in->iw_type));
    if (im.is_user_define_wave()) {
        size_t n = (size_t)in->nx * in->ny;
        im.iw_psi.resize(n);
        using TC = typename std::decay<decltype(im.iw_psi[0])>::type;
        for (size_t i = 0; i < n; i++) im.iw_psi[i] = TC(in->iw_psi[2 * i], in->iw_psi[2 * i + 1]);
    }
    im.iw_x.assign(in->iw_x, in->iw_x + in->n_iw_xy);
    im.iw_y.assign(in->iw_y, in->iw_y + in->n_iw_xy);

    im.E_0 = in->E_0;
    im.theta = in->theta * mt::c_deg_2_rad;
    im.phi = in->phi * mt::c_deg_2_rad;
    if (im.is_PED()) {  // ilc_multem.cu:338-347
        im.theta = in->ped_theta * mt::c_deg_2_rad;
        im.nrot = in->ped_nrot;
    } else if (im.is_HCTEM()) {
        im.theta = in->hci_theta * mt::c_deg_2_rad;
        im.nrot = in->hci_nrot;
    }

    im.illumination_model = static_cast<mt::eIllumination_Model>(in->illumination_model);
    im.temporal_spatial_incoh = static_cast<mt::eTemporal_Spatial_Incoh>(in->temporal_spatial_incoh);

    fill_lens(in->cond_lens, im.cond_lens, im.E_0, im.grid_2d);
    mt_lens obj = in->obj_lens;
    obj.si_a = in->cond_lens.si_a;
    obj.si_sigma = in->cond_lens.si_sigma;
    obj.si_beta = in->cond_lens.si_beta;
    obj.si_rad_npts = in->cond_lens.si_rad_npts;
    obj.si_azm_npts = in->cond_lens.si_azm_npts;
    fill_lens(obj, im.obj_lens, im.E_0, im.grid_2d);

    if (im.is_scanning()) {
        im.scanning.type = static_cast<mt::eScanning_Type>(in->scanning_type);
        im.scanning.pbc = in->scanning_periodic != 0;
        im.scanning.spxs = in->scanning_square_pxs != 0;
        im.scanning.ns = in->scanning_ns;
        im.scanning.x0 = in->scanning_x0;
        im.scanning.y0 = in->scanning_y0;
        im.scanning.xe = in->scanning_xe;
        im.scanning.ye = in->scanning_ye;
        im.scanning.set_grid();
    }

    if (im.is_STEM()) {
        T lambda = mt::get_lambda(im.E_0);
        im.detector.type = static_cast<mt::eDetector_Type>(in->detector_type);
        if (im.detector.type == mt::eDT_Circular && in->n_detector > 0) {
            im.detector.resize(in->n_detector);
            for (int i = 0; i < in->n_detector; i++) {
                auto inner_ang = in->detector_inner_ang[i] * mt::c_mrad_2_rad;
                im.detector.g_inner[i] = sin(inner_ang) / lambda;
                auto outer_ang = in->detector_outer_ang[i] * mt::c_mrad_2_rad;
                im.detector.g_outer[i] = sin(outer_ang) / lambda;
            }
        } else if (im.detector.type == mt::eDT_Matrix && in->n_detector > 0) {
            // as ilc_multem.cu:316-335: each map is assigned linearly (column-major ny x nx)
            im.detector.resize(in->n_detector);
            const size_t nxy = (size_t)in->nx * in->ny;
            for (int i = 0; i < in->n_detector; i++) {
                im.detector.fR[i].resize(nxy);
                for (size_t k = 0; k < nxy; k++) im.detector.fR[i][k] = (T)in->detector_fR[i * nxy + k];
            }
        }
    }

    im.output_area.ix_0 = in->output_area_ix_0 - 1;
    im.output_area.iy_0 = in->output_area_iy_0 - 1;
    im.output_area.ix_e = in->output_area_ix_e - 1;
    im.output_area.iy_e = in->output_area_iy_e - 1;

    im.validate_parameters();
}

template <class V>
void copy_real(const V& v, double* dst, size_t n = (size_t)-1) {
    for (size_t i = 0; i < v.size() && i < n; i++) dst[i] = (double)v[i];
}

template <class V>
void copy_cplx(const V& v, double* dst, size_t n = (size_t)-1) {
    for (size_t i = 0; i < v.size() && i < n; i++) {
        dst[2 * i] = (double)v[i].real();
        dst[2 * i + 1] = (double)v[i].imag();
    }
}

template <class T, mt::eDevice dev = mt::e_host>
int run(const mt_input_multislice* in, int nthreads, mt_output_multislice* out, mt_output_dims* dims) {
    mt::Input_Multislice<T> im;
    fill_input(in, im, nthreads, dev);
    mt::Output_Multislice<T> om;
    mt::Stream<dev> stream(im.system_conf.nstream);
    mt::FFT<T, dev> fft_2d;
    fft_2d.create_plan_2d(im.grid_2d.ny, im.grid_2d.nx, im.system_conf.nstream);
    mt::Multislice<T, dev>::ext_stop_sim = false;
    mt::Multislice<T, dev> sim;
    sim.set_input_data(&im, &stream, &fft_2d);
    om.set_input_data(&im);
    if (out != nullptr) {
        sim(om);
        stream.synchronize();
        om.gather();
        om.clean_temporal();
    }
    fft_2d.cleanup();

    if (dims) {
        dims->n_thick = (int)om.thick.size();
        dims->n_detector = (int)om.ndetector;
        dims->nx = om.nx;
        dims->ny = om.ny;
        dims->has_image_tot = (int)om.image_tot.size() > 0;
        dims->has_image_coh = (int)om.image_coh.size() > 0;
        dims->has_m2psi_tot = (int)om.m2psi_tot.size() > 0;
        dims->has_psi_coh = (int)om.psi_coh.size() > 0;
        dims->has_m2psi_coh = (int)om.m2psi_coh.size() > 0 && om.pn_coh_contrib && !om.is_EWFS_EWRS();
        dims->n_x = (int)om.x.size();
        dims->n_y = (int)om.y.size();
    }
    if (out == nullptr) return 0;
    out->dx = om.dx;
    out->dy = om.dy;
    if (out->x) copy_real(om.x, out->x);
    if (out->y) copy_real(om.y, out->y);
    if (out->thick) copy_real(om.thick, out->thick);
    size_t nxy = (size_t)om.nx * om.ny;
    for (size_t ithk = 0; ithk < om.thick.size(); ithk++) {
        if (out->image_tot && om.image_tot.size())
            for (int idet = 0; idet < om.ndetector; idet++)
                copy_real(om.image_tot[ithk].image[idet], out->image_tot + (ithk * om.ndetector + idet) * nxy, nxy);
        if (out->image_coh && om.image_coh.size())
            for (int idet = 0; idet < om.ndetector; idet++)
                copy_real(om.image_coh[ithk].image[idet], out->image_coh + (ithk * om.ndetector + idet) * nxy, nxy);
        if (out->m2psi_tot && om.m2psi_tot.size()) copy_real(om.m2psi_tot[ithk], out->m2psi_tot + ithk * nxy, nxy);
        if (out->m2psi_coh && om.m2psi_coh.size() && om.pn_coh_contrib && !om.is_EWFS_EWRS())
            copy_real(om.m2psi_coh[ithk], out->m2psi_coh + ithk * nxy, nxy);
        // psi_coh is held at the full grid size; like set_struct_multislice (ilc_multem.cu:382-481)
        // only the first nx*ny values of the output area are returned
        if (out->psi_coh && om.psi_coh.size()) copy_cplx(om.psi_coh[ithk], out->psi_coh + 2 * ithk * nxy, nxy);
    }
    return 0;
}

// Wave_Function gives access to the specimen (Spec), slicing, potential and transmission of one
// phonon configuration, the state Multislice::operator() drives (src/wave_function.cuh:37-75).
template <class T>
struct WF {
    mt::Input_Multislice<T> im;
    mt::Stream<mt::e_host> stream{1};
    mt::FFT<T, mt::e_host> fft_2d;
    mt::Wave_Function<T, mt::e_host> wf;
    WF(const mt_input_multislice* in, int nthreads) {
        fill_input(in, im, nthreads);
        stream.resize(im.system_conf.nstream);
        fft_2d.create_plan_2d(im.grid_2d.ny, im.grid_2d.nx, im.system_conf.nstream);
        wf.set_input_data(&im, &stream, &fft_2d);
    }
    ~WF() { fft_2d.cleanup(); }
};

template <class F>
int guarded(F fn) {
    try {
        return fn();
    } catch (std::exception& e) {
        g_err = e.what();
        return -1;
    } catch (...) {
        g_err = "unknown exception";
        return -1;
    }
}

}  // namespace

extern "C" {

const char* mtref_last_error(void) { return g_err.c_str(); }

// Full simulation; precision 1 = float, 2 = double.
int mtref_run(const mt_input_multislice* in, int precision, int nthreads, mt_output_multislice* out) {
    return guarded([&] { return precision == 2 ? run<double>(in, nthreads, out, nullptr) : run<float>(in, nthreads, out, nullptr); });
}

// The reference's own GPU path (run_multislice<float, e_device>, mex_files_multem/ilc_multem.cu:
// 484-518 and :538-541): Multislice<float, e_device> with cuFFT, one stream, GPU 0. Used only as a
// timed baseline.
int mtref_run_device(const mt_input_multislice* in, mt_output_multislice* out) {
    return guarded([&] { return run<float, mt::e_device>(in, 1, out, nullptr); });
}

int mtref_output_dims(const mt_input_multislice* in, int precision, mt_output_dims* dims) {
    return guarded([&] { return precision == 2 ? run<double>(in, 1, nullptr, dims) : run<float>(in, 1, nullptr, dims); });
}

// Validated scalar parameters after validate_parameters(): lambda, Vr_factor, z zero-defocus plane
// of the condenser lens, and the slice count / atom count after set_input_data.
int mtref_params(const mt_input_multislice* in, int precision, double* vals, int nvals) {
    return guarded([&] {
        auto body = [&](auto& w) {
            double v[8] = {(double)w.im.lambda, (double)w.im.Vr_factor(), (double)w.im.cond_lens.zero_defocus_plane,
                           (double)w.wf.slicing.slice.size(), (double)w.wf.atoms.size(),
                           (double)w.im.grid_2d.dz, (double)w.im.thick.size(), (double)w.im.interaction_model};
            for (int i = 0; i < nvals && i < 8; i++) vals[i] = v[i];
            return 0;
        };
        if (precision == 2) { WF<double> w(in, 1); return body(w); }
        WF<float> w(in, 1);
        return body(w);
    });
}

// Displaced atoms and slicing of configuration iconf (Spec::move_atoms, src/spec.hpp:85-127;
// Slicing::calculate, src/slicing.hpp:93-100). Arrays sized by the caller: n_atoms_max atoms,
// n_slice_max slices; the actual counts are returned in *n_atoms / *n_slice.
int mtref_specimen(const mt_input_multislice* in, int precision, int iconf, int n_atoms_max, int* n_atoms, int* Z,
                   double* xyz, int n_slice_max, int* n_slice, double* z_0, double* z_e, int* iatom_0, int* iatom_e,
                   int* ithk, double* thick_z_back_prop) {
    return guarded([&] {
        auto body = [&](auto& w) {
            w.wf.move_atoms(iconf);
            auto& at = w.wf.atoms;
            *n_atoms = (int)at.size();
            for (int i = 0; i < (int)at.size() && i < n_atoms_max; i++) {
                Z[i] = at.Z[i];
                xyz[3 * i] = (double)at.x[i];
                xyz[3 * i + 1] = (double)at.y[i];
                xyz[3 * i + 2] = (double)at.z[i];
            }
            auto& sl = w.wf.slicing.slice;
            *n_slice = (int)sl.size();
            for (int i = 0; i < (int)sl.size() && i < n_slice_max; i++) {
                z_0[i] = (double)sl[i].z_0;
                z_e[i] = (double)sl[i].z_e;
                iatom_0[i] = sl[i].iatom_0;
                iatom_e[i] = sl[i].iatom_e;
                ithk[i] = sl[i].ithk;
            }
            auto& th = w.wf.slicing.thick;
            for (int i = 0; i < (int)th.size(); i++) thick_z_back_prop[i] = (double)th[i].z_back_prop;
            return 0;
        };
        if (precision == 2) { WF<double> w(in, 1); return body(w); }
        WF<float> w(in, 1);
        return body(w);
    });
}

// Projected potential of one slice in the reference's stored layout (fft-shifted: pixel
// (iy, ix) holds the potential at ((ix - nx/2) dx, (iy - ny/2) dy) modulo the box), as
// ilc_projected_potential returns it (mex_files_multem/ilc_projected_potential.cu:134-160).
int mtref_projected_potential(const mt_input_multislice* in, int precision, int nthreads, int iconf, int islice,
                              double* V) {
    return guarded([&] {
        auto body = [&](auto& w) {
            w.wf.move_atoms(iconf);
            w.wf(islice, w.wf.V_0);
            copy_real(w.wf.V_0, V);
            return 0;
        };
        if (precision == 2) { WF<double> w(in, nthreads); return body(w); }
        WF<float> w(in, nthreads);
        return body(w);
    });
}

// Transmission function of one slice, same layout (ilc_transmission_function.cu:152-170).
int mtref_transmission_function(const mt_input_multislice* in, int precision, int nthreads, int iconf, int islice,
                                double* trans) {
    return guarded([&] {
        auto body = [&](auto& w) {
            w.wf.move_atoms(iconf);
            w.wf.trans(islice, w.wf.trans_0);
            copy_cplx(w.wf.trans_0, trans);
            return 0;
        };
        if (precision == 2) { WF<double> w(in, nthreads); return body(w); }
        WF<float> w(in, nthreads);
        return body(w);
    });
}

// Spline table of element Z with ionic charge `charge` (Atomic_Data::get_atom_coef,
// src/atomic_data.hpp:1547-1668; the coefficient set Atom_Type::charge_to_idx selects), as stored in
// the working precision: R_min, R_max, R_tap, tap_cf, then R2[nR], c0..c3[nR].
int mtref_atom_type_q(const mt_input_multislice* in, int precision, int Z, int charge, double* head, double* tab,
                      int nR) {
    return guarded([&] {
        auto body = [&](auto& w) {
            using TT = typename std::decay<decltype(w.im)>::type::value_type;
            auto& at = static_cast<mt::Spec<TT>&>(w.wf).atom_type[Z - 1];
            auto& c = at.coef[at.charge_to_idx(charge)];
            head[0] = (double)c.R_min;
            head[1] = (double)c.R_max;
            head[2] = (double)c.R_tap;
            head[3] = (double)c.tap_cf;
            for (int i = 0; i < nR; i++) {
                tab[i] = (double)c.R2[i];
                tab[nR + i] = (double)c.ciVR.c0[i];
                tab[2 * nR + i] = (double)c.ciVR.c1[i];
                tab[3 * nR + i] = (double)c.ciVR.c2[i];
                tab[4 * nR + i] = (double)c.ciVR.c3[i];
            }
            return 0;
        };
        if (precision == 2) { WF<double> w(in, 1); return body(w); }
        WF<float> w(in, 1);
        return body(w);
    });
}

int mtref_atom_type(const mt_input_multislice* in, int precision, int Z, double* head, double* tab, int nR) {
    return mtref_atom_type_q(in, precision, Z, 0, head, tab, nR);
}

// Incident wave (Incident_Wave::operator()(space, output), src/incident_wave.cuh:98-116), with the
// beam positions in->iw_x/iw_y; space 1 = real, 2 = reciprocal.
int mtref_incident_wave(const mt_input_multislice* in, int precision, int space, double* psi) {
    return guarded([&] {
        auto body = [&](auto& w) {
            using TT = typename std::decay<decltype(w.im)>::type::value_type;
            typename std::decay<decltype(w.wf.psi_z)>::type p(w.im.grid_2d.nxy());
            mt::Incident_Wave<TT, mt::e_host> iw;
            iw.set_input_data(&w.im, &w.stream, &w.fft_2d);
            TT gxu = w.im.gx_0(), gyu = w.im.gy_0();
            iw(p, gxu, gyu, w.im.iw_x, w.im.iw_y);
            if (space == 2) {
                w.fft_2d.forward(p);
                mt::scale(w.stream, w.im.grid_2d.inxy(), p);
            }
            copy_cplx(p, psi);
            return 0;
        };
        if (precision == 2) { WF<double> w(in, 1); return body(w); }
        WF<float> w(in, 1);
        return body(w);
    });
}

// Propagation of the user wave in->iw_psi by z, as ilc_propagate does it (read_input_multislice and
// run_propagate, mex_files_multem/ilc_propagate.cu:34-147): simulation type PropRS, still atoms,
// grid from spec_lx/ly and nx/ny with lz = 0, dz = 0.25, no band-width limit, then
// Propagator::operator()(space, gx_0, gy_0, z, output) (src/propagator.cuh:95-103), which fft-shifts
// the wave in, propagates and shifts it back. The MEX file passes obj_lens_c_10 as z.
int mtref_propagate(const mt_input_multislice* in, int precision, int space, double z, double* psi) {
    return guarded([&] {
        auto body = [&](auto tag) {
            using TT = decltype(tag);
            mt::Input_Multislice<TT> im;
            im.system_conf.precision = std::is_same<TT, float>::value ? mt::eP_float : mt::eP_double;
            im.system_conf.device = mt::e_host;
            im.system_conf.cpu_nthread = 1;
            im.system_conf.validate_parameters();
            im.simulation_type = mt::eTEMST_PropRS;
            im.pn_model = mt::ePM_Still_Atom;
            im.grid_2d.set_input_data(in->nx, in->ny, (TT)in->spec_lx, (TT)in->spec_ly, (TT)0.25, false, true);
            im.set_incident_wave_type(static_cast<mt::eIncident_Wave_Type>(in->iw_type));
            const int nxy = in->nx * in->ny;
            im.iw_psi.resize(nxy);
            for (int i = 0; i < nxy; i++) im.iw_psi[i] = std::complex<TT>((TT)in->iw_psi[2 * i], (TT)in->iw_psi[2 * i + 1]);
            for (int i = 0; i < in->n_iw_xy; i++) {
                im.iw_x.push_back((TT)in->iw_x[i]);
                im.iw_y.push_back((TT)in->iw_y[i]);
            }
            im.E_0 = (TT)in->E_0;
            im.theta = (TT)(in->theta * mt::c_deg_2_rad);
            im.phi = (TT)(in->phi * mt::c_deg_2_rad);
            im.obj_lens.c_10 = (TT)z;
            im.obj_lens.set_input_data(im.E_0, im.grid_2d);
            im.output_area.ix_0 = in->output_area_ix_0 - 1;
            im.output_area.iy_0 = in->output_area_iy_0 - 1;
            im.output_area.ix_e = in->output_area_ix_e - 1;
            im.output_area.iy_e = in->output_area_iy_e - 1;
            im.validate_parameters();
            mt::Stream<mt::e_host> stream(1);
            mt::FFT<TT, mt::e_host> fft_2d;
            fft_2d.create_plan_2d(im.grid_2d.ny, im.grid_2d.nx, 1);
            mt::Propagator<TT, mt::e_host> prop;
            prop.set_input_data(&im, &stream, &fft_2d);
            mt::Output_Multislice<TT> out;
            out.set_input_data(&im);
            prop(space == 2 ? mt::eS_Reciprocal : mt::eS_Real, im.gx_0(), im.gy_0(), im.obj_lens.c_10, out);
            stream.synchronize();
            const auto& v = out.psi_coh[0];
            for (size_t i = 0; i < v.size(); i++) {
                psi[2 * i] = (double)v[i].real();
                psi[2 * i + 1] = (double)v[i].imag();
            }
            fft_2d.cleanup();
            return 0;
        };
        if (precision == 2) return body(double());
        return body(float());
    });
}

}  // extern "C"
