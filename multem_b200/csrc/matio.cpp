// MATLAB-facing I/O: the input struct of a multislice run read from a MAT-file into the C ABI's
// mt_input_multislice, and the output struct written as ilc_multem returns it.
//
// Input: the struct that multem_input.parameters.toStruct produces (the value ilc_multem receives,
// matlab_functions/+multem_input/parameters.m:247-250), field by field as read_input_multislice
// reads it (mex_files_multem/ilc_multem.cu:38-379): flat scalar fields, spec_atoms (rows x 8),
// spec_amorp (struct array z_0, z_e, dz), thick, iw_psi (complex ny x nx), iw_x, iw_y, the
// cond_lens_* / obj_lens_* fields, detector (struct: type; cir(i).inner_ang/outer_ang in mrad;
// matrix(i).fR, ny x nx), scanning_*, output_area_* (1-based), and system_conf (struct: precision,
// device, cpu_nthread, gpu_device) as ilc_multem(prms.system_conf, prms) passes it. A field the
// struct lacks takes the default of multem_input.parameters.
//
// Output: struct {dx, dy, x, y, thick, data} with data a 1 x n_thick struct array of
// image_tot(idet).image (and image_coh) for STEM, m2psi_tot and psi_coh for exit waves, m2psi_tot
// (and m2psi_coh) otherwise, every image ny x nx (set_struct_multislice,
// mex_files_multem/ilc_multem.cu:382-481).
#include "matio.hpp"

#include <cstring>

#include "common.hpp"
#include "host_model.hpp"

namespace mtb {
namespace matio {
namespace {

using mat::Value;

double num(const Value& s, const char* name, double def) {
    const Value* f = s.field(name);
    if (!f || !f->is_numeric() || f->re.empty()) return def;
    return f->re[0];
}

int inum(const Value& s, const char* name, int def) { return (int)num(s, name, (double)def); }

// the field's numeric data (column-major), or `def` when absent or empty
std::vector<double> arr(const Value& s, const char* name, std::vector<double> def) {
    const Value* f = s.field(name);
    if (!f || !f->is_numeric() || f->re.empty()) return def;
    return f->re;
}

void lens(const Value& s, const std::string& p, bool cond, mt_lens* L) {
    auto d = [&](const char* k, double def) { return num(s, (p + "_" + k).c_str(), def); };
    auto i = [&](const char* k, int def) { return (int)d(k, (double)def); };
    L->m = i("m", 0);
    L->c_10 = d("c_10", 14.0312);
    L->c_12 = d("c_12", 0); L->phi_12 = d("phi_12", 0);
    L->c_21 = d("c_21", 0); L->phi_21 = d("phi_21", 0); L->c_23 = d("c_23", 0); L->phi_23 = d("phi_23", 0);
    L->c_30 = d("c_30", 1e-3); L->c_32 = d("c_32", 0); L->phi_32 = d("phi_32", 0);
    L->c_34 = d("c_34", 0); L->phi_34 = d("phi_34", 0);
    L->c_41 = d("c_41", 0); L->phi_41 = d("phi_41", 0); L->c_43 = d("c_43", 0); L->phi_43 = d("phi_43", 0);
    L->c_45 = d("c_45", 0); L->phi_45 = d("phi_45", 0);
    L->c_50 = d("c_50", 0); L->c_52 = d("c_52", 0); L->phi_52 = d("phi_52", 0);
    L->c_54 = d("c_54", 0); L->phi_54 = d("phi_54", 0); L->c_56 = d("c_56", 0); L->phi_56 = d("phi_56", 0);
    L->inner_aper_ang = d("inner_aper_ang", 0);
    L->outer_aper_ang = d("outer_aper_ang", cond ? 21.0 : 24.0);
    L->ti_a = d("ti_a", 1.0); L->ti_sigma = d("ti_sigma", 32.0); L->ti_beta = d("ti_beta", 0); L->ti_npts = i("ti_npts", 10);
    L->si_a = d("si_a", 1.0); L->si_sigma = d("si_sigma", 0.0072); L->si_beta = d("si_beta", 0);
    L->si_rad_npts = i("si_rad_npts", 4); L->si_azm_npts = i("si_azm_npts", 4);
    L->zero_defocus_type = i("zero_defocus_type", 1);
    L->zero_defocus_plane = d("zero_defocus_plane", 0);
}

}  // namespace

std::unique_ptr<Input> read_input(const std::string& path, const std::string& var) {
    mat::Variables vars = mat::read_file(path);
    const Value* sp = nullptr;
    for (auto& [name, v] : vars)
        if ((var.empty() && v.is_struct()) || (!var.empty() && name == var)) {
            sp = &v;
            break;
        }
    if (!sp) fail(MT_ERR_INVALID_ARG, var.empty() ? path + " holds no struct variable" : path + " has no variable " + var);
    const Value& s = *sp;
    if (!s.is_struct() || s.numel() != 1) fail(MT_ERR_INVALID_ARG, "the input variable must be a 1x1 struct");

    auto h = std::make_unique<Input>();
    auto keep = [&](std::vector<double> v) -> const double* {
        if (v.empty()) v.push_back(0.0);
        h->store.push_back(std::move(v));
        return h->store.back().data();
    };
    mt_system_conf& c = h->conf;
    c.precision = 1; c.device = 2; c.cpu_nthread = 1; c.gpu_device = 0;
    if (const Value* sc = s.field("system_conf"); sc && sc->is_struct() && sc->numel() >= 1) {
        c.precision = inum(*sc, "precision", 1);
        c.device = inum(*sc, "device", 2);
        c.cpu_nthread = inum(*sc, "cpu_nthread", 1);
        c.gpu_device = inum(*sc, "gpu_device", 0);
    }
    mt_input_multislice& in = h->in;
    std::memset(&in, 0, sizeof(in));
    in.simulation_type = inum(s, "simulation_type", 52);
    in.interaction_model = inum(s, "interaction_model", 1);
    in.potential_type = inum(s, "potential_type", 6);
    in.operation_mode = inum(s, "operation_mode", 1);
    in.reverse_multislice = inum(s, "reverse_multislice", 0);
    in.pn_model = inum(s, "pn_model", 1);
    in.pn_coh_contrib = inum(s, "pn_coh_contrib", 0);
    in.pn_single_conf = inum(s, "pn_single_conf", 0);
    in.pn_nconf = inum(s, "pn_nconf", 1);
    in.pn_dim = inum(s, "pn_dim", 110);
    in.pn_seed = inum(s, "pn_seed", 300183);
    in.pn_rng = inum(s, "pn_rng", 0);

    const Value* at = s.field("spec_atoms");
    if (at && at->is_numeric() && at->numel() > 0) {
        in.spec_atoms_rows = (int)at->dims[0];
        in.spec_atoms_cols = (int)(at->numel() / (size_t)at->dims[0]);
        in.spec_atoms = keep(at->re);
    } else {
        in.spec_atoms_rows = 0;
        in.spec_atoms_cols = 8;
        in.spec_atoms = keep({});
    }
    in.spec_lx = num(s, "spec_lx", 10); in.spec_ly = num(s, "spec_ly", 10);
    in.spec_lz = num(s, "spec_lz", 10); in.spec_dz = num(s, "spec_dz", 0.25);
    in.spec_cryst_na = inum(s, "spec_cryst_na", 1); in.spec_cryst_nb = inum(s, "spec_cryst_nb", 1);
    in.spec_cryst_nc = inum(s, "spec_cryst_nc", 1);
    in.spec_cryst_a = num(s, "spec_cryst_a", 0); in.spec_cryst_b = num(s, "spec_cryst_b", 0);
    in.spec_cryst_c = num(s, "spec_cryst_c", 0);
    in.spec_cryst_x0 = num(s, "spec_cryst_x0", 0); in.spec_cryst_y0 = num(s, "spec_cryst_y0", 0);
    std::vector<double> z0, ze, dz;
    if (const Value* am = s.field("spec_amorp"); am && am->is_struct()) {
        for (size_t i = 0; i < am->numel(); i++) {
            const Value* a = am->field("z_0", i);
            if (!a || a->re.empty()) continue;  // an empty layer entry (the class default)
            z0.push_back(a->re[0]);
            const Value* e = am->field("z_e", i);
            ze.push_back(e && !e->re.empty() ? e->re[0] : 0.0);
            const Value* d = am->field("dz", i);
            dz.push_back(d && !d->re.empty() ? d->re[0] : 2.0);
        }
    }
    in.spec_amorp_n = (int)z0.size();
    in.spec_amorp_z_0 = keep(z0);
    in.spec_amorp_z_e = keep(ze);
    in.spec_amorp_dz = keep(dz);
    in.spec_rot_theta = num(s, "spec_rot_theta", 0);
    const std::vector<double> u0 = arr(s, "spec_rot_u0", {0, 0, 1}), cp = arr(s, "spec_rot_center_p", {0, 0, 0});
    for (int i = 0; i < 3; i++) {
        in.spec_rot_u0[i] = i < (int)u0.size() ? u0[i] : 0.0;
        in.spec_rot_center_p[i] = i < (int)cp.size() ? cp[i] : 0.0;
    }
    in.spec_rot_center_type = inum(s, "spec_rot_center_type", 1);

    in.thick_type = inum(s, "thick_type", 1);
    const std::vector<double> th = arr(s, "thick", {0.0});
    in.n_thick = (int)th.size();
    in.thick = keep(th);
    in.potential_slicing = inum(s, "potential_slicing", 1);
    in.nx = inum(s, "nx", 256);
    in.ny = inum(s, "ny", 256);
    in.bwl = inum(s, "bwl", 0);

    in.iw_type = inum(s, "iw_type", 4);
    if (const Value* ps = s.field("iw_psi"); ps && ps->is_numeric() && !ps->re.empty()) {
        std::vector<double> il(2 * ps->re.size(), 0.0);
        for (size_t i = 0; i < ps->re.size(); i++) {
            il[2 * i] = ps->re[i];
            il[2 * i + 1] = ps->complex ? ps->im[i] : 0.0;
        }
        in.iw_psi = keep(il);
    } else {
        in.iw_psi = nullptr;
    }
    const std::vector<double> ix = arr(s, "iw_x", {0.0}), iy = arr(s, "iw_y", {0.0});
    in.n_iw_xy = (int)std::min(ix.size(), iy.size());
    in.iw_x = keep(std::vector<double>(ix.begin(), ix.begin() + in.n_iw_xy));
    in.iw_y = keep(std::vector<double>(iy.begin(), iy.begin() + in.n_iw_xy));

    in.E_0 = num(s, "E_0", 300);
    in.theta = num(s, "theta", 0);
    in.phi = num(s, "phi", 0);
    in.ped_theta = num(s, "ped_theta", 3); in.ped_nrot = inum(s, "ped_nrot", 360);
    in.hci_theta = num(s, "hci_theta", 3); in.hci_nrot = inum(s, "hci_nrot", 360);
    in.illumination_model = inum(s, "illumination_model", 3);
    in.temporal_spatial_incoh = inum(s, "temporal_spatial_incoh", 1);
    lens(s, "cond_lens", true, &in.cond_lens);
    lens(s, "obj_lens", false, &in.obj_lens);

    in.scanning_type = inum(s, "scanning_type", 2);
    in.scanning_periodic = inum(s, "scanning_periodic", 0);
    in.scanning_square_pxs = inum(s, "scanning_square_pxs", 1);
    in.scanning_ns = inum(s, "scanning_ns", 10);
    in.scanning_x0 = num(s, "scanning_x0", 0); in.scanning_y0 = num(s, "scanning_y0", 0);
    in.scanning_xe = num(s, "scanning_xe", 4.078); in.scanning_ye = num(s, "scanning_ye", 4.078);

    // detector (read for every simulation type; only STEM uses it)
    std::vector<double> inner, outer, fr;
    in.detector_type = 1;
    if (const Value* det = s.field("detector"); det && det->is_struct() && det->numel() >= 1) {
        in.detector_type = inum(*det, "type", 1);
        if (in.detector_type == 1) {
            if (const Value* cir = det->field("cir"); cir && cir->is_struct())
                for (size_t i = 0; i < cir->numel(); i++) {
                    const Value* a = cir->field("inner_ang", i);
                    const Value* b = cir->field("outer_ang", i);
                    if (!a || !b || a->re.empty() || b->re.empty()) continue;
                    inner.push_back(a->re[0]);
                    outer.push_back(b->re[0]);
                }
            in.n_detector = (int)inner.size();
        } else if (in.detector_type == 3) {
            int n = 0;
            if (const Value* m = det->field("matrix"); m && m->is_struct())
                for (size_t i = 0; i < m->numel(); i++) {
                    const Value* f = m->field("fR", i);
                    if (!f || f->re.empty()) continue;
                    if (f->re.size() != (size_t)in.nx * in.ny)
                        fail(MT_ERR_INVALID_ARG, "detector.matrix(" + std::to_string(i + 1) + ").fR is not ny x nx");
                    fr.insert(fr.end(), f->re.begin(), f->re.end());  // column-major ny x nx = [ix][iy]
                    n++;
                }
            in.n_detector = n;
        }
    } else {
        inner = {60.0};
        outer = {180.0};
        in.n_detector = 1;
    }
    in.detector_inner_ang = keep(inner);
    in.detector_outer_ang = keep(outer);
    in.detector_fR = keep(fr);

    in.output_area_ix_0 = inum(s, "output_area_ix_0", 0);
    in.output_area_iy_0 = inum(s, "output_area_iy_0", 0);
    in.output_area_ix_e = inum(s, "output_area_ix_e", 0);
    in.output_area_iy_e = inum(s, "output_area_iy_e", 0);
    return h;
}

void write_output(const std::string& path, const std::string& var, const mt_output_dims& d,
                  const mt_output_multislice& out, bool compress) {
    Value o = Value::struct_array(1, 1, {"dx", "dy", "x", "y", "thick", "data"});
    o.at(0, "dx") = Value::scalar(out.dx);
    o.at(0, "dy") = Value::scalar(out.dy);
    o.at(0, "x") = Value::row(std::vector<double>(out.x, out.x + d.n_x));
    o.at(0, "y") = Value::row(std::vector<double>(out.y, out.y + d.n_y));
    o.at(0, "thick") = Value::row(std::vector<double>(out.thick, out.thick + d.n_thick));
    const size_t nxy = (size_t)d.nx * d.ny;
    Value data;
    if (d.has_image_tot) {
        std::vector<std::string> f{"image_tot"};
        if (d.has_image_coh) f.push_back("image_coh");
        data = Value::struct_array(1, d.n_thick, f);
        for (int t = 0; t < d.n_thick; t++) {
            for (auto& name : f) {
                const double* src = name == "image_tot" ? out.image_tot : out.image_coh;
                Value det = Value::struct_array(1, d.n_detector, {"image"});
                for (int k = 0; k < d.n_detector; k++)
                    det.at(k, "image") = Value::matrix(d.ny, d.nx, src + ((size_t)t * d.n_detector + k) * nxy);
                data.at(t, name) = std::move(det);
            }
        }
    } else if (d.has_psi_coh) {
        std::vector<std::string> f;
        if (d.has_m2psi_tot) f.push_back("m2psi_tot");
        f.push_back("psi_coh");
        data = Value::struct_array(1, d.n_thick, f);
        for (int t = 0; t < d.n_thick; t++) {
            if (d.has_m2psi_tot) data.at(t, "m2psi_tot") = Value::matrix(d.ny, d.nx, out.m2psi_tot + (size_t)t * nxy);
            const double* p = out.psi_coh + 2 * (size_t)t * nxy;
            data.at(t, "psi_coh") = Value::matrix(d.ny, d.nx, p, p + 1, 2);
        }
    } else {
        std::vector<std::string> f{"m2psi_tot"};
        if (d.has_m2psi_coh) f.push_back("m2psi_coh");
        data = Value::struct_array(1, d.n_thick, f);
        for (int t = 0; t < d.n_thick; t++) {
            data.at(t, "m2psi_tot") = Value::matrix(d.ny, d.nx, out.m2psi_tot + (size_t)t * nxy);
            if (d.has_m2psi_coh) data.at(t, "m2psi_coh") = Value::matrix(d.ny, d.nx, out.m2psi_coh + (size_t)t * nxy);
        }
    }
    o.at(0, "data") = std::move(data);
    mat::write_file(path, {{var.empty() ? std::string("output_multislice") : var, std::move(o)}}, compress);
}

}  // namespace matio
}  // namespace mtb
