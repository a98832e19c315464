// Host-side model: validation, specimen, frozen phonons and slicing (see host_model.hpp).
//
// Each function restates the reference's algorithm in the reference's float working precision;
// the comment above it names the reference function it follows. Where the reference evaluates an
// expression in double and stores it as float (constants are double literals), the same
// promotion is written out explicitly.
#include "host_model.hpp"

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <string>

#include "common.hpp"
#include "tables.hpp"

namespace mtb {

namespace {

constexpr double kPi = 3.141592653589793238463;
constexpr double kMrad = 1.0e-03;
constexpr double kDeg = 0.01745329251994329576924;
constexpr double kMm2A = 1.0e+07;

// isEqual<float> (src/types.cuh:564-577)
bool is_equal_f(float a, float b) {
    const float eps_abs = 1e-5f, eps_rel = 1e-4f;
    float diff = std::fabs(a - b);
    if (diff <= eps_abs) return true;
    float fa = std::fabs(a), fb = std::fabs(b);
    return diff <= ((fa < fb ? fb : fa) * eps_rel);
}
bool is_zero_f(float a) { return is_equal_f(a, 0.0f); }

// get_lambda<float> (src/cgpu_fcns.cuh:50-58)
float lambda_f(float E_0) {
    float emass = 510.99906f;
    float hc = 12.3984244f;
    return hc / std::sqrt(E_0 * (2 * emass + E_0));
}

// get_gamma<float> and get_Vr_factor<float> (src/cgpu_fcns.cuh:75-145)
float vr_factor_f(float E_0, float theta) {
    float emass = 510.99906f;
    float gamma = 1 + E_0 / emass;
    float c_Potf = 47.877645145863056f;
    return gamma * lambda_f(E_0) / (c_Potf * std::cos(theta));
}

// Identify_Planes::hist (src/types.cuh:1310-1370)
std::vector<int> plane_hist(const std::vector<float>& v, double dv, double v_min, double v_max) {
    const double v_l = std::fmax(v_max - v_min, dv);
    const int nbins = (int)std::ceil(v_l / dv);
    std::vector<int> h(nbins, 0);
    for (size_t iv = 0; iv < v.size(); iv++) {
        double v_id = (double)v[iv];
        int ih = (int)std::floor((v_id - v_min) / dv);
        double v_imin = v_min + (ih - 1) * dv;
        double v_imax = v_imin + dv;
        if (v_id < v_imin) {
            for (int ik = ih; ik >= 0; ik--) {
                v_imin = v_min + (ik - 1) * dv;
                v_imax = v_imin + dv;
                if ((v_imin <= v_id) && (v_id < v_imax)) {
                    ih = ik - 1;
                    break;
                }
            }
        } else if (v_id > v_imax) {
            for (int ik = ih; ik < nbins; ik++) {
                v_imin = v_min + ik * dv;
                v_imax = v_imin + dv;
                if ((v_imin <= v_id) && (v_id < v_imax)) {
                    ih = ik;
                    break;
                }
            }
        }
        ih = std::max(0, std::min(nbins - 1, ih));
        h[ih]++;
    }
    while (!h.empty() && h.back() == 0) h.pop_back();
    for (int ih = 1; ih < (int)h.size() - 1; ih++) {
        bool bn = (ih < (int)h.size() - 2) ? (0 < h[ih + 2]) : false;
        bn = (0 < h[ih - 1]) && ((0 < h[ih + 1]) || bn);
        if ((h[ih] == 0) && bn) h[ih] = 1;
    }
    return h;
}

// kh_sum (src/cgpu_fcns.cuh:250-258): Kahan summation step
void kahan(float& sum, float v, float& err) {
    v = v - err;
    float t = sum + v;
    err = (t - sum) - v;
    sum = t;
}

// Identify_Planes::operator()(v) (src/types.cuh:1176-1241): planes of sorted z values
std::vector<float> planes_from_values(const std::vector<float>& v) {
    std::vector<float> out;
    if (v.empty()) return out;
    const float dv = 0.1f;
    float v_min = v.front(), v_max = v.back();
    auto h = plane_hist(v, (double)dv, (double)v_min, (double)v_max);
    if (h.size() == 1) {
        float s = 0;
        for (float x : v) s += x;
        out.push_back(s / (float)v.size());
        return out;
    }
    std::vector<float> v_lim;
    for (int iz = 0; iz < (int)h.size() - 1; iz++)
        if ((h[iz] > 0) && (h[iz + 1] == 0)) v_lim.push_back(v.front() + (iz + 1) * dv);
    v_lim.push_back(v.back() + dv);
    float v_m = v.front(), v_m_ee = 0;
    int v_c = 1, izl = 0;
    for (size_t iz = 0; iz < v.size(); iz++) {
        float v_v = v[iz];
        if (v_v < v_lim[izl]) {
            kahan(v_m, v_v, v_m_ee);
            v_c++;
        } else {
            out.push_back(v_m / v_c);
            v_m = v_v;
            v_m_ee = 0;
            v_c = 1;
            izl++;
        }
    }
    out.push_back(v_m / v_c);
    return out;
}

// Identify_Planes::operator()(v_min, v_max, dv, eMB_MinMax) (src/types.cuh:1243-1306)
std::vector<float> planes_regular(float v_min, float v_max, float dv) {
    const float v_eps = 1e-4f;
    std::vector<float> out;
    if (std::fabs(v_max - v_min) < v_eps) {
        out.push_back((float)(0.5 * (v_min + v_max)));
        return out;
    }
    if (v_max < v_min) return out;
    auto quot = [v_eps](float a, float b) { return (int)std::floor(a / b + v_eps); };
    float s_v = v_max - v_min;
    const int nv = std::max(1, quot(s_v, dv)) + 1;
    const double dv_b = dv + 0.5 * (s_v - (nv - 1) * dv);
    out.resize(nv);
    out[0] = v_min;
    for (int iv = 1; iv < nv; iv++) {
        const double dv_t = ((iv == 1) || (iv == nv - 1)) ? dv_b : (double)dv;
        out[iv] = (float)(out[iv - 1] + dv_t);
    }
    return out;
}

// Slicing::get_spacing (src/slicing.hpp:118-127)
float spacing(size_t ix, const std::vector<float>& x, float dz = 0.5f) {
    if (x.size() == 1) return dz;
    ix = (ix == 0) ? 1 : std::min(ix, x.size() - 1);
    return (x.size() > 1) ? x[ix] - x[ix - 1] : 0.0f;
}

// unique_vector (src/cpu_fcns.hpp:3604-3611)
void unique_sorted(std::vector<float>& v) {
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end(), is_equal_f), v.end());
}

// Atom_Data::validate_amorphous_parameters (src/atomic_data_mt.hpp:539-590) on a copy of the layer
// list: layers thinner than 1e-4 A are dropped, the rest get the mean region of the atoms strictly
// inside them (Amorp_Lay_Info::set_region, src/types.cuh:1105-1126), are sorted by z_0, and a zero
// slice thickness becomes 2 A. (The layer type the reference also sets is not used by slicing.)
std::vector<AtomsF::Amorp> valid_amorphous_layers(const AtomsF& atoms) {
    std::vector<AtomsF::Amorp> out;
    for (const auto& l : atoms.amorp) {
        if (std::fabs(l.z_e - l.z_0) < 1e-4f) continue;
        AtomsF::Amorp a = l;
        int f_region = 0, c_region = 0;
        for (size_t i = 0; i < atoms.size(); i++) {
            const float z = atoms.z[i];
            if ((a.z_0 < z) && (z < a.z_e)) {
                f_region += atoms.region[i];
                c_region++;
            }
        }
        c_region = std::max(1, c_region);
        a.region = (int)std::round((float)f_region / (float)c_region);
        out.push_back(a);
    }
    std::sort(out.begin(), out.end(), [](const AtomsF::Amorp& a, const AtomsF::Amorp& b) { return a.z_0 < b.z_0; });
    for (auto& a : out)
        if (is_zero_f(a.dz)) a.dz = 2.0f;
    return out;
}

// Slicing::get_z_plane (src/slicing.hpp:130-193): planes of the crystal (region 0) atoms, then, if
// the specimen extends above / below them, regular planes of the first / last amorphous layer.
std::vector<float> z_planes(int pot_sli, const AtomsF& atoms) {
    if (atoms.size() == 0) return {0.0f};
    const auto amorp = valid_amorphous_layers(atoms);
    std::vector<float> z_ct;
    for (size_t i = 0; i < atoms.size(); i++)
        if (atoms.region[i] == 0) z_ct.push_back(atoms.z[i]);
    if (z_ct.empty()) fail(MT_ERR_UNSUPPORTED, "specimen has no atoms in region 0");
    std::sort(z_ct.begin(), z_ct.end());
    std::vector<float> zp = (pot_sli == 1) ? planes_from_values(z_ct) : planes_regular(z_ct.front(), z_ct.back(), atoms.dz);
    const float z_eps = 1e-3f;
    if (!amorp.empty() && (std::fabs(atoms.z_min - zp.front()) > z_eps)) {
        const float dz_b = spacing(1, zp);
        const auto& a = amorp.front();
        auto top = planes_regular(a.z_0, a.z_e - dz_b, a.dz);
        zp.insert(zp.begin(), top.begin(), top.end());
    }
    if (!amorp.empty() && (std::fabs(zp.back() - atoms.z_max) > z_eps)) {
        const float dz_b = spacing(zp.size() - 1, zp);
        const auto& a = amorp.back();
        auto bottom = planes_regular(a.z_0 + dz_b, a.z_e, a.dz);
        zp.insert(zp.end(), bottom.begin(), bottom.end());
    }
    unique_sorted(zp);
    return zp;
}

// Slicing::get_z_slice (src/slicing.hpp:196-250) for planes / dz_Proj
std::vector<float> z_slices(int pot_sli, const std::vector<float>& zp, const AtomsF& atoms) {
    std::vector<float> zs;
    if (zp.size() == 1) return {atoms.z_int_min, atoms.z_int_max};
    zs.resize(zp.size() + 1);
    zs[0] = (float)(zp[0] - 0.5 * spacing(0, zp, atoms.dz));
    for (size_t iz = 1; iz < zs.size() - 1; iz++) zs[iz] = (float)(0.5 * (zp[iz] + zp[iz - 1]));
    zs[zs.size() - 1] = zs[zs.size() - 2] + spacing(zp.size(), zp, atoms.dz);
    (void)pot_sli;
    return zs;
}

// Slicing::fd_by_z (src/slicing.hpp:406-429): last atom with z below z_e
int last_atom_below(const std::vector<float>& z, float z_e) {
    if (z.empty()) return -1;
    if (z_e < z.front()) return -1;
    int iz_e = (z.back() <= z_e) ? (int)z.size() - 1
                                 : (int)(std::lower_bound(z.begin(), z.end(), z_e) - z.begin()) - 1;
    if (iz_e < 0 || z[iz_e] < z.front()) return -1;
    return iz_e;
}

// Slicing::fd_by_z (src/slicing.hpp:432-452): atoms with z in [z_0, z_e)
void atoms_in_range(const std::vector<float>& z, float z_0, float z_e, int& iz_0, int& iz_e) {
    if (z.empty() || (z_0 > z_e) || (z.back() < z_0) || (z_e < z.front())) {
        iz_0 = 1;
        iz_e = 0;
        return;
    }
    iz_0 = (z_0 <= z.front()) ? 0 : (int)(std::lower_bound(z.begin(), z.end(), z_0) - z.begin());
    iz_e = (z.back() <= z_e) ? (int)z.size() - 1 : (int)(std::lower_bound(z.begin(), z.end(), z_e) - z.begin()) - 1;
    if ((iz_0 > iz_e) || (iz_e < 0) || (z[iz_e] < z_0) || (z_e < z[iz_0])) {
        iz_0 = 1;
        iz_e = 0;
    }
}

// match_vectors (src/cpu_fcns.hpp:3613-3653): snap requested thicknesses to planes
void match_thick(const std::vector<float>& vr_in, std::vector<float>& vs, float dv) {
    dv = std::fmax(dv, 0.1f);
    std::vector<float> vr(vr_in);
    float vr_min = *std::min_element(vr.begin(), vr.end()) - dv;
    float vr_max = *std::max_element(vr.begin(), vr.end()) + dv;
    vs.erase(std::remove_if(vs.begin(), vs.end(), [&](float a) { return (a < vr_min) || (a > vr_max); }), vs.end());
    std::vector<bool> free_(vr.size(), true);
    std::vector<float> out;
    for (float val : vs) {
        const float da = 1e-4f;
        auto it = std::min_element(vr.begin(), vr.end(), [&](float a, float b) {
            return std::fabs(a - val - da) < std::fabs(b - val);
        });
        size_t imin = it - vr.begin();
        if (free_[imin]) {
            free_[imin] = false;
            out.push_back(*it);
        }
    }
    vs = out;
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Grid_2d<float>::set_input_data (src/types.cuh:2155-2180)
void GridF::set(int nx_, int ny_, float lx_, float ly_, float dz_, bool bwl_, bool pbc_) {
    nx = nx_;
    ny = ny_;
    nxh = nx / 2;
    nyh = ny / 2;
    lx = lx_;
    ly = ly_;
    dz = dz_;
    bwl = bwl_;
    pbc_xy = pbc_;
    Rx_0 = Ry_0 = 0;
    dRx = (nx == 0) ? 0.0f : lx / (float)nx;
    dRy = (ny == 0) ? 0.0f : ly / (float)ny;
    dgx = is_zero_f(lx) ? 0.0f : 1.0f / lx;
    dgy = is_zero_f(ly) ? 0.0f : 1.0f / ly;
    float glm = gl_max();
    gl2_max = glm * glm;
    float dg0 = 0.25f, fg0 = 1e-02f;
    float gd = glm + dg0;
    alpha = (float)(std::log(1.0 / fg0 - 1.0) / (double)(gd * gd - gl2_max));
}

float GridF::g_max() const { return std::fmin((float)nxh * dgx, (float)nyh * dgy); }
float GridF::gl_max() const { return (float)(2.0 * g_max() / 3.0); }
float GridF::exp_factor_Rx(float x) const {
    const float c_2Pi = 6.283185307179586476925f;
    return -c_2Pi * (x - lxh());
}
float GridF::exp_factor_Ry(float y) const {
    const float c_2Pi = 6.283185307179586476925f;
    return -c_2Pi * (y - lyh());
}

// ---------------------------------------------------------------------------------------------
// Lens: fields as read by read_input_multislice (mex_files_multem/ilc_multem.cu:155-209)
void LensF::from_input(const mt_lens& l) {
    m = l.m;
    c_10 = (float)l.c_10;
    c_12 = (float)l.c_12;
    phi_12 = (float)((float)l.phi_12 * kDeg);
    c_21 = (float)l.c_21;
    phi_21 = (float)((float)l.phi_21 * kDeg);
    c_23 = (float)l.c_23;
    phi_23 = (float)((float)l.phi_23 * kDeg);
    c_30 = (float)((float)l.c_30 * kMm2A);
    c_32 = (float)l.c_32;
    phi_32 = (float)((float)l.phi_32 * kDeg);
    c_34 = (float)l.c_34;
    phi_34 = (float)((float)l.phi_34 * kDeg);
    c_41 = (float)l.c_41;
    phi_41 = (float)((float)l.phi_41 * kDeg);
    c_43 = (float)l.c_43;
    phi_43 = (float)((float)l.phi_43 * kDeg);
    c_45 = (float)l.c_45;
    phi_45 = (float)((float)l.phi_45 * kDeg);
    c_50 = (float)((float)l.c_50 * kMm2A);
    c_52 = (float)l.c_52;
    phi_52 = (float)((float)l.phi_52 * kDeg);
    c_54 = (float)l.c_54;
    phi_54 = (float)((float)l.phi_54 * kDeg);
    c_56 = (float)l.c_56;
    phi_56 = (float)((float)l.phi_56 * kDeg);
    inner_aper_ang = (float)((float)l.inner_aper_ang * kMrad);
    outer_aper_ang = (float)((float)l.outer_aper_ang * kMrad);
    si_sigma = (float)l.si_sigma;
    si_a = (float)l.si_a;
    si_beta = (float)l.si_beta;
    si_rad_npts = l.si_rad_npts;
    si_azm_npts = l.si_azm_npts;
    ti_a = (float)l.ti_a;
    ti_sigma = (float)l.ti_sigma;
    ti_beta = (float)l.ti_beta;
    ti_npts = l.ti_npts;
    zero_defocus_type = l.zero_defocus_type;
    zero_defocus_plane = (float)l.zero_defocus_plane;
}

// Lens<float>::set_input_data (src/types.cuh:2936-2985)
void LensF::set_input_data(float E_0, const GridF& grid) {
    // Lens::set_input_data (src/types.cuh:2953-2956)
    ti_a = std::max(0.0f, std::min(1.0f, ti_a));
    ti_sigma = std::max(0.0f, ti_sigma);
    ti_beta = std::max(0.0f, ti_beta);
    ti_npts = std::max(1, ti_npts);
    si_a = std::max(0.0f, std::min(1.0f, si_a));
    si_sigma = std::max(0.0f, si_sigma);
    si_beta = std::max(0.0f, si_beta);
    si_rad_npts = std::max(1, si_rad_npts);
    si_azm_npts = std::max(1, si_azm_npts);
    lambda = lambda_f(E_0);
    const double L = (double)lambda;
    auto cc = [&](float c, double f) -> float { return is_zero_f(c) ? 0.0f : (float)(f * (double)c); };
    c_c_10 = cc(c_10, -kPi * L);
    c_c_12 = cc(c_12, -kPi * L);
    c_c_21 = is_zero_f(c_21) ? 0.0f : (float)(-2.0 * kPi * c_21 * std::pow(L, 2) / 3.0);
    c_c_23 = is_zero_f(c_23) ? 0.0f : (float)(-2.0 * kPi * c_23 * std::pow(L, 2) / 3.0);
    c_c_30 = is_zero_f(c_30) ? 0.0f : (float)(-kPi * c_30 * std::pow(L, 3) / 2.0);
    c_c_32 = is_zero_f(c_32) ? 0.0f : (float)(-kPi * c_32 * std::pow(L, 3) / 2.0);
    c_c_34 = is_zero_f(c_34) ? 0.0f : (float)(-kPi * c_34 * std::pow(L, 3) / 2.0);
    c_c_41 = is_zero_f(c_41) ? 0.0f : (float)(-2.0 * kPi * c_41 * std::pow(L, 4) / 5.0);
    c_c_43 = is_zero_f(c_43) ? 0.0f : (float)(-2.0 * kPi * c_43 * std::pow(L, 4) / 5.0);
    c_c_45 = is_zero_f(c_45) ? 0.0f : (float)(-2.0 * kPi * c_45 * std::pow(L, 4) / 5.0);
    c_c_50 = is_zero_f(c_50) ? 0.0f : (float)(-kPi * c_50 * std::pow(L, 5) / 3.0);
    c_c_52 = is_zero_f(c_52) ? 0.0f : (float)(-kPi * c_52 * std::pow(L, 5) / 3.0);
    c_c_54 = is_zero_f(c_54) ? 0.0f : (float)(-kPi * c_54 * std::pow(L, 5) / 3.0);
    c_c_56 = is_zero_f(c_56) ? 0.0f : (float)(-kPi * c_56 * std::pow(L, 5) / 3.0);
    if (is_zero_f(inner_aper_ang) || inner_aper_ang < 0) {
        g2_min = 0;
    } else {
        float q = std::sin(inner_aper_ang) / lambda;
        g2_min = (float)std::pow((double)q, 2);
    }
    if (is_zero_f(outer_aper_ang) || outer_aper_ang < 0) {
        g2_max = grid.g2_max();
    } else {
        float q = std::sin(outer_aper_ang) / lambda;
        g2_max = (float)std::pow((double)q, 2);
    }
}

// Lens<float>::set_defocus (src/types.cuh:2993-2997)
void LensF::set_defocus(float f) {
    c_10 = f;
    c_c_10 = is_zero_f(c_10) ? 0.0f : (float)(-kPi * (double)c_10 * (double)lambda);
}

// Lens<float>::get_zero_defocus_plane (src/types.cuh:2998-3023)
float LensF::get_zero_defocus_plane(float z_min, float z_max) const {
    switch (zero_defocus_type) {
        case 1: return z_min;
        case 2: return (float)(0.5 * (z_min + z_max));
        case 3: return z_max;
        default: return zero_defocus_plane;
    }
}

// Lens<float>::is_phi_required (src/types.cuh:3166-3172)
bool LensF::is_phi_required() const {
    return (m != 0) || !is_zero_f(c_12) || !is_zero_f(c_21) || !is_zero_f(c_23) || !is_zero_f(c_32) ||
           !is_zero_f(c_34) || !is_zero_f(c_41) || !is_zero_f(c_43) || !is_zero_f(c_45) || !is_zero_f(c_52) ||
           !is_zero_f(c_54) || !is_zero_f(c_56);
}

// ---------------------------------------------------------------------------------------------
void AtomsF::resize(size_t n) {
    Z.resize(n);
    x.resize(n);
    y.resize(n);
    z.resize(n);
    sigma.resize(n);
    occ.resize(n);
    region.resize(n);
    charge.resize(n);
}

// Atom_Data::get_statistic (src/atomic_data_mt.hpp:429-512), the fields slicing reads
void AtomsF::statistic(const float* R_max_of_Z) {
    if (Z.empty()) return;
    auto mm = std::minmax_element(z.begin(), z.end());
    z_min = *mm.first;
    z_max = *mm.second;
    sigma_max = *std::max_element(sigma.begin(), sigma.end());
    float s_x = *std::max_element(x.begin(), x.end()) - *std::min_element(x.begin(), x.end());
    float s_y = *std::max_element(y.begin(), y.end()) - *std::min_element(y.begin(), y.end());
    R_int_min = R_int_max = 2.5f;
    if (R_max_of_Z) {
        R_int_min = R_int_max = R_max_of_Z[(Z[0] % 1000) - 1];
        for (size_t i = 0; i < Z.size(); i++) {
            float r = R_max_of_Z[(Z[i] % 1000) - 1];
            R_int_min = std::min(r, R_int_min);
            R_int_max = std::max(r, R_int_max);
        }
    }
    float s_z = z_max - z_min;
    z_int_min = z_min - R_int_max;
    z_int_max = z_max + R_int_max;
    s_z_int = z_int_max - z_int_min;
    if (is_zero_f(l_x)) l_x = s_x;
    if (is_zero_f(l_y)) l_y = s_y;
    l_z = std::fmax(s_z, l_z);
}

// Atom_Data::sort_by_z (src/atomic_data_mt.hpp:515-521). thrust::sort on the host is a stable
// merge sort, so atoms with equal z keep their input order.
void AtomsF::sort_by_z() {
    std::vector<size_t> idx(Z.size());
    for (size_t i = 0; i < idx.size(); i++) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return z[a] < z[b]; });
    AtomsF s = *this;
    for (size_t i = 0; i < idx.size(); i++) {
        Z[i] = s.Z[idx[i]];
        x[i] = s.x[idx[i]];
        y[i] = s.y[idx[i]];
        z[i] = s.z[idx[i]];
        sigma[i] = s.sigma[idx[i]];
        occ[i] = s.occ[idx[i]];
        region[i] = s.region[idx[i]];
        charge[i] = s.charge[idx[i]];
    }
}

// ---------------------------------------------------------------------------------------------
// Input_Multislice::set_incident_angle (src/input_multislice.cuh:891-895, applied at :655): the
// tilt is snapped so that sin(theta)/lambda is a whole number of Fourier pixels dg_min.
void snap_incident_angle(Model& m) {
    if (is_zero_f(m.theta)) {
        m.theta = 0;
    } else {
        const float dg = m.grid.dg_min();
        const float n = std::round(std::sin(m.theta) / (m.lambda * dg));
        m.theta = std::asin(n * m.lambda * dg);
    }
}

// Gauss-Hermite rule for the weight exp(-t^2) on the real line (n points). The nodes are the
// eigenvalues of the Jacobi matrix of the orthonormal Hermite polynomials (zero diagonal,
// off-diagonal sqrt(k/2)), found by bisection on Sturm counts; the weights are the Christoffel
// numbers 1 / sum_{k<n} p_k(x)^2. The weights sum to sqrt(pi).
void gauss_hermite(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    auto below = [&](double s) {  // eigenvalues below s: negative pivots of (J - s I) = L D L^T
        int c = 0;
        double d = 1.0;
        for (int k = 0; k < n; k++) {
            d = -s - (k > 0 ? 0.5 * k / d : 0.0);
            if (d == 0.0) d = -1e-300;
            if (d < 0.0) c++;
        }
        return c;
    };
    const double R = std::sqrt(2.0 * n) + 2.0;  // every eigenvalue lies in (-R, R) (Gershgorin)
    for (int i = 0; i < n; i++) {
        double lo = -R, hi = R;
        for (int it = 0; it < 200 && hi - lo > 1e-15 * std::max(1.0, std::fabs(lo)); it++) {
            const double mid = 0.5 * (lo + hi);
            if (below(mid) > i) hi = mid; else lo = mid;
        }
        const double t = 0.5 * (lo + hi);
        double p0 = std::pow(3.141592653589793238463, -0.25), p1 = std::sqrt(2.0) * t * p0;
        double sum = p0 * p0 + (n > 1 ? p1 * p1 : 0.0);
        for (int k = 1; k + 1 < n; k++) {
            const double p2 = std::sqrt(2.0 / (k + 1)) * t * p1 - std::sqrt((double)k / (k + 1)) * p0;
            sum += p2 * p2;
            p0 = p1;
            p1 = p2;
        }
        x[i] = t;
        w[i] = 1.0 / sum;
    }
}

void gauss_laguerre1(int n, std::vector<double>& x, std::vector<double>& w) {
    // Jacobi matrix of the monic Laguerre polynomials L_k^(1): diagonal 2k + 2, off-diagonal
    // sqrt(k (k + 1)); nodes by Sturm-count bisection, weights by the Christoffel sum of the
    // orthonormal polynomials (mu_0 = Gamma(2) = 1)
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    auto diag = [](int k) { return 2.0 * k + 2.0; };
    auto off2 = [](int k) { return (double)k * (k + 1); };  // squared off-diagonal between k-1 and k
    auto below = [&](double s) {
        int c = 0;
        double d = 1.0;
        for (int k = 0; k < n; k++) {
            d = (diag(k) - s) - (k > 0 ? off2(k) / d : 0.0);
            if (d == 0.0) d = -1e-300;
            if (d < 0.0) c++;
        }
        return c;
    };
    const double R = 4.0 * n + 4.0;  // every eigenvalue lies in (0, R) (Gershgorin)
    for (int i = 0; i < n; i++) {
        double lo = 0.0, hi = R;
        for (int it = 0; it < 200 && hi - lo > 1e-15 * std::max(1.0, std::fabs(lo)); it++) {
            const double mid = 0.5 * (lo + hi);
            if (below(mid) > i) hi = mid; else lo = mid;
        }
        const double t = 0.5 * (lo + hi);
        double p0 = 1.0, p1 = (n > 1) ? (t - diag(0)) / std::sqrt(off2(1)) : 0.0;
        double sum = p0 * p0 + p1 * p1;
        for (int k = 1; k + 1 < n; k++) {
            const double p2 = ((t - diag(k)) * p1 - std::sqrt(off2(k)) * p0) / std::sqrt(off2(k + 1));
            sum += p2 * p2;
            p0 = p1;
            p1 = p2;
        }
        x[i] = t;
        w[i] = 1.0 / sum;
    }
}

// Spatial part of cond_lens_temporal_spatial_quadratures (src/cpu_fcns.hpp:1573-1626): the source
// spread is a 2-D Gaussian (share si_a, sigma si_sigma) plus an exponential (si_beta) component;
// the radius is integrated with the generalized Laguerre rule of weight r exp(-b_q r) (quadrature
// type 25 with alpha = 1: nodes t / b_q, weights / b_q^2), b_q = 1 / sigma_t,
// sigma_t^2 = (2 si_a si_sigma^2 + 6 (1 - si_a) si_beta^2) / 6, each weight times the ratio of the
// spread function to exp(-b_q r); the azimuth with si_azm_npts equal steps of 2 pi / si_azm_npts.
void spatial_quadrature(const LensF& L, std::vector<double>& x, std::vector<double>& y, std::vector<double>& w) {
    x.assign(1, 0.0);
    y.assign(1, 0.0);
    w.assign(1, 1.0);
    if (!((L.si_rad_npts > 1 || L.si_azm_npts > 1) && (!is_zero_f(L.si_sigma) || !is_zero_f(L.si_beta)))) return;
    const double kTwoPi = 6.283185307179586476925;
    const double s2 = (double)L.si_sigma * L.si_sigma, b2 = (double)L.si_beta * L.si_beta;
    const double a = is_zero_f(L.si_sigma) ? 0.0 : L.si_a / (kTwoPi * s2);
    const double b = is_zero_f(L.si_sigma) ? 0.0 : 0.5 / s2;
    const double c = is_zero_f(L.si_beta) ? 0.0 : (1.0 - L.si_a) / (kTwoPi * b2);
    const double d = is_zero_f(L.si_beta) ? 0.0 : 1.0 / L.si_beta;
    const double sigma_t = std::sqrt((2.0 * L.si_a * s2 + 6.0 * (1.0 - L.si_a) * b2) / 6.0);
    const double b_q = 1.0 / sigma_t;
    std::vector<double> r, wr;
    gauss_laguerre1(L.si_rad_npts, r, wr);
    for (int i = 0; i < L.si_rad_npts; i++) {
        r[i] /= b_q;
        wr[i] /= b_q * b_q;
        const double ra = std::fabs(r[i]);
        wr[i] *= a * std::exp(-b * ra * ra + b_q * ra) + c * std::exp(-d * ra + b_q * ra);
    }
    const double h = kTwoPi / L.si_azm_npts;
    x.clear();
    y.clear();
    w.clear();
    for (int i = 0; i < L.si_rad_npts; i++)
        for (int j = 0; j < L.si_azm_npts; j++) {
            const double th = j * h;
            x.push_back(r[i] * std::cos(th));
            y.push_back(r[i] * std::sin(th));
            w.push_back(wr[i] * h);
        }
}

// Temporal part of cond_lens_temporal_spatial_quadratures (src/cpu_fcns.hpp:1540-1571): the
// defocus spread is a Gaussian (height ti_a, sigma ti_sigma) plus an exponential (ti_beta)
// component, integrated with the generalized Hermite rule of weight exp(-b_q x^2), b_q =
// 1/(2 sigma_t^2), sigma_t^2 = ti_a ti_sigma^2 + 2 (1 - ti_a) ti_beta^2 (quadrature type 26 with
// alpha = 0: Gauss-Hermite nodes / sqrt(b_q), weights / sqrt(b_q)), each weight times the ratio
// of the spread function to that weight at the node.
void temporal_quadrature(const LensF& L, std::vector<double>& x, std::vector<double>& w) {
    if (!(L.ti_npts > 1 && !is_zero_f(L.ti_sigma))) {
        x.assign(1, 0.0);
        w.assign(1, 1.0);
        return;
    }
    const double s2 = (double)L.ti_sigma * L.ti_sigma, b2 = (double)L.ti_beta * L.ti_beta;
    const double a = L.ti_a / (std::sqrt(2.0 * 3.141592653589793238463) * L.ti_sigma);
    const double b = 0.5 / s2;
    const double c = is_zero_f(L.ti_beta) ? 0.0 : (1.0 - L.ti_a) / (2.0 * L.ti_beta);
    const double d = is_zero_f(L.ti_beta) ? 0.0 : 1.0 / L.ti_beta;
    const double sigma_t = std::sqrt(L.ti_a * s2 + 2.0 * (1.0 - L.ti_a) * b2);
    const double b_q = 0.5 / (sigma_t * sigma_t);
    gauss_hermite(L.ti_npts, x, w);
    const double sc = 1.0 / std::sqrt(b_q);
    for (int i = 0; i < L.ti_npts; i++) {
        x[i] *= sc;
        w[i] *= sc;
        const double r = std::fabs(x[i]);
        w[i] *= a * std::exp(-b * r * r + b_q * r * r) + c * std::exp(-d * r + b_q * r * r);
    }
}

// Microscope_Effects (src/microscope_effects.cuh:32-200) for HRTEM: the coherent CTF
// (illumination 1), the partially coherent CTF with temporal and spatial envelopes (2), or the
// sum over the objective's defocus spread (4: Gauss-Hermite points of
// obj_lens_temporal_spatial_quadratures, src/cpu_fcns.hpp:1504-1510, weights / sqrt(pi), defocus
// c_10 + sqrt(2) ti_sigma x). The reference's spatial quadrature for 4 ends empty (its qs.resize(0),
// cpu_fcns.hpp:1535, so those images are zero) and 3 computes nothing; both are refused.
void hrtem_ctf_points(Model& m) {
    const LensF& L = m.obj_lens;
    m.obj_c10.assign(1, L.c_10);
    m.obj_w.assign(1, 1.0);
    switch (m.illumination_model) {
        case 1:
        case 2:
            m.ctf_mode = m.illumination_model;
            return;
        case 4:
            if (m.temporal_spatial_incoh != 2)
                fail(MT_ERR_UNSUPPORTED, "HRTEM full integration with spatial incoherence: the reference's spatial "
                                         "quadrature is empty (zero images); use temporal_spatial_incoh 2");
            m.ctf_mode = 4;
            {
                std::vector<double> x, w;
                gauss_hermite(L.ti_npts, x, w);
                const float iehwgd = (float)(1.414213562373095048802 * (double)L.ti_sigma);
                m.obj_c10.clear();
                m.obj_w.clear();
                for (int j = 0; j < L.ti_npts; j++) {
                    m.obj_c10.push_back((float)((double)iehwgd * (float)x[j] + (double)L.c_10));
                    m.obj_w.push_back((double)(float)(w[j] / std::sqrt(3.141592653589793238463)));
                }
            }
            return;
        default:
            fail(MT_ERR_UNSUPPORTED, "HRTEM needs illumination_model 1, 2 or 4 (3 computes nothing in the reference)");
    }
}

// isZero(gx_0, gy_0) of Wave_Function::phase_multiplication (src/wave_function.cuh:79)
bool Model::tilted() const {
    for (int r = 0; r < nrot; r++)
        if (ramp_needed(r)) return true;
    return false;
}

float Model::gx_0() const { return (float)(std::sin(theta) * std::cos(phi) / lambda); }
float Model::gy_0() const { return (float)(std::sin(theta) * std::sin(phi) / lambda); }
float Model::rot_phi(int irot) const {
    if (!(is_PED() || is_HCTEM())) return phi;
    return (irot == 0) ? 0.0f : (float)((2.0 * 3.141592653589793238463 * (double)(float)irot) / (double)(float)nrot);
}
float Model::gx_0(int irot) const { return (float)(std::sin(theta) * std::cos(rot_phi(irot)) / lambda); }
float Model::gy_0(int irot) const { return (float)(std::sin(theta) * std::sin(rot_phi(irot)) / lambda); }
// Wave_Function::phase_multiplication is skipped for PED (dp_Shift) and for no tilt
bool Model::ramp_needed(int irot) const { return !dp_shift && !(is_zero_f(gx_0(irot)) && is_zero_f(gy_0(irot))); }
// Input_Multislice::Vr_factor (src/input_multislice.cuh:914-917)
float Model::Vr_factor() const { return (float)mul_sign * vr_factor_f(E_0, theta); }
// Input_Multislice::get_propagator_factor (src/input_multislice.cuh:909-912)
float Model::propagator_factor(float z) const { return (float)(-mul_sign * kPi * lambda * z); }
// Input_Multislice::get_phonon_rot_weight (src/input_multislice.cuh:897-901)
// Input_Multislice::get_phonon_rot_weight (src/input_multislice.cuh:897-901)
float Model::phonon_weight() const {
    int nconf = (!is_frozen_phonon() || pn_single_conf) ? 1 : pn_nconf;
    return 1.0f / (float)(nconf * nrot);
}

// read_input_multislice + validate_parameters (mex_files_multem/ilc_multem.cu:38-379,
// src/input_multislice.cuh:622-796) for the simulation types, slicing and incident waves this
// engine implements; anything else is rejected with MT_ERR_UNSUPPORTED.
// Line lengths with a compiled FFT plan (LinePlan in fft_core.cuh).
bool line_size_supported(int n) {
    return n == 64 || n == 128 || n == 256 || n == 384 || n == 512 || n == 1024 || n == 2048;
}

// read_input_multislice of ilc_propagate (mex_files_multem/ilc_propagate.cu:34-95): the grid from
// spec_lx/ly and nx/ny (lz = 0, dz = 0.25, no band-width limit, periodic), the user wave, E_0 and
// the beam tilt; nothing of the specimen is read.
Model build_prop_model(const mt_input_multislice* in) {
    if (!in) fail(MT_ERR_INVALID_ARG, "input is NULL");
    if (!line_size_supported(in->nx) || !line_size_supported(in->ny))
        fail(MT_ERR_UNSUPPORTED, "nx and ny must be one of 64, 128, 256, 384, 512, 1024, 2048");
    if (!(in->spec_lx > 0) || !(in->spec_ly > 0)) fail(MT_ERR_INVALID_ARG, "spec_lx and spec_ly must be positive");
    if (in->iw_type != 3 || !in->iw_psi)
        fail(MT_ERR_INVALID_ARG, "propagation needs a user-defined wave (iw_type 3 with iw_psi)");
    Model m;
    m.simulation_type = in->simulation_type;
    m.grid.set(in->nx, in->ny, (float)in->spec_lx, (float)in->spec_ly, 0.25f, false, true);
    m.iw_type = 3;
    const size_t n = (size_t)in->nx * in->ny;
    m.iw_psi.resize(2 * n);
    for (size_t i = 0; i < 2 * n; i++) m.iw_psi[i] = (float)in->iw_psi[i];
    m.E_0 = (float)in->E_0;
    m.theta = (float)((float)in->theta * kDeg);
    m.phi = (float)((float)in->phi * kDeg);
    m.lambda = lambda_f(m.E_0);
    m.mul_sign = 1;
    snap_incident_angle(m);
    return m;
}

Model build_model(const mt_input_multislice* in) {
    if (!in) fail(MT_ERR_INVALID_ARG, "input is NULL");
    Model m;
    m.simulation_type = in->simulation_type;
    if (!(m.is_scanning() || m.is_wave_sim()))
        fail(MT_ERR_UNSUPPORTED, "simulation_type " + std::to_string(in->simulation_type) +
                                     " is outside the plain multislice path (supported: 11 STEM, 12 ISTEM, 21 CBED, 22 CBEI, "
                                     "31 ED, 32 HRTEM, 41 PED, 42 HCTEM, 51 EWFS, 52 EWRS)");
    m.interaction_model = in->interaction_model;
    if (m.interaction_model < 1 || m.interaction_model > 3)
        fail(MT_ERR_UNSUPPORTED, "interaction_model must be 1 (multislice), 2 (phase object) or 3 (weak phase object)");
    m.potential_type = in->potential_type;
    if (m.potential_type == 5)
        fail(MT_ERR_UNSUPPORTED, "potential_type 5 (Weickenmeier-Kohl) has no closed-form projected potential; "
                                 "use 1-4 or 6");
    if (!potential_type_supported(m.potential_type))
        fail(MT_ERR_INVALID_ARG, "potential_type must be 1-6, got " + std::to_string(m.potential_type));
    m.mul_sign = in->reverse_multislice ? -1 : 1;
    m.pn_model = in->pn_model;
    m.pn_coh_contrib = in->pn_coh_contrib != 0;
    m.pn_single_conf = in->pn_single_conf != 0;
    m.pn_nconf = in->pn_nconf;
    switch (in->pn_dim) {  // FP_Dim::set (src/types.cuh:1687-1730)
        case 111: m.pn_x = m.pn_y = m.pn_z = true; break;
        case 110: m.pn_x = m.pn_y = true; m.pn_z = false; break;
        case 101: m.pn_x = true; m.pn_y = false; m.pn_z = true; break;
        case 11: m.pn_x = false; m.pn_y = true; m.pn_z = true; break;
        case 100: m.pn_x = true; m.pn_y = m.pn_z = false; break;
        case 10: m.pn_x = false; m.pn_y = true; m.pn_z = false; break;
        case 1: m.pn_x = m.pn_y = false; m.pn_z = true; break;
        default: break;
    }
    m.pn_seed = in->pn_seed;
    m.pn_rng = in->pn_rng;
    if (m.pn_rng != 0 && m.pn_rng != 1) fail(MT_ERR_INVALID_ARG, "pn_rng must be 0 (host) or 1 (device)");

    const float lx = (float)in->spec_lx, ly = (float)in->spec_ly, lz = (float)in->spec_lz, dz = (float)in->spec_dz;
    if (in->spec_atoms_rows < 0 || (in->spec_atoms_rows > 0 && (!in->spec_atoms || in->spec_atoms_cols < 4)))
        fail(MT_ERR_INVALID_ARG, "spec_atoms must be an n x (4..8) matrix");
    // Atom_Data::set_atoms + read_atom (src/atomic_data_mt.hpp:320-350, 774-787)
    AtomsF& A = m.atoms_in;
    const int nr = in->spec_atoms_rows, nc = in->spec_atoms_cols;
    A.resize(nr);
    A.l_x = lx;
    A.l_y = ly;
    A.l_z = lz;
    A.dz = dz;
    for (int i = 0; i < nr; i++) {
        const double* a = in->spec_atoms;
        A.Z[i] = (int)a[0 * nr + i];
        A.x[i] = (float)a[1 * nr + i];
        A.y[i] = (float)a[2 * nr + i];
        A.z[i] = (float)a[3 * nr + i];
        A.sigma[i] = (float)(float)((nc > 4) ? a[4 * nr + i] : 0.085);
        A.occ[i] = (float)(float)((nc > 5) ? a[5 * nr + i] : 1.0);
        A.region[i] = std::abs((int)((nc > 6) ? a[6 * nr + i] : 0));
        A.charge[i] = (int)((nc > 7) ? a[7 * nr + i] : 0);
        int Zi = A.Z[i] % 1000;
        if (Zi < 1 || Zi > 103) fail(MT_ERR_INVALID_ARG, "atomic number out of range 1..103");
    }
    if (nr == 0) fail(MT_ERR_INVALID_ARG, "specimen has no atoms");
    A.statistic(nullptr);
    // Atom_Data::set_amorphous_parameters (src/atomic_data_mt.hpp:313-317)
    if (in->spec_amorp_n > 0 && (!in->spec_amorp_z_0 || !in->spec_amorp_z_e || !in->spec_amorp_dz))
        fail(MT_ERR_INVALID_ARG, "spec_amorp_z_0, spec_amorp_z_e and spec_amorp_dz must hold spec_amorp_n values");
    for (int i = 0; i < in->spec_amorp_n; i++)
        A.amorp.push_back({(float)in->spec_amorp_z_0[i], (float)in->spec_amorp_z_e[i], (float)in->spec_amorp_dz[i], 0, 0});
    m.thick_type = in->thick_type;
    if (m.thick_type < 1 || m.thick_type > 3) fail(MT_ERR_INVALID_ARG, "thick_type must be 1, 2 or 3");
    if (m.thick_type != 1) {
        if (in->n_thick <= 0 || !in->thick) fail(MT_ERR_INVALID_ARG, "thick is empty");
        for (int i = 0; i < in->n_thick; i++) m.thick.push_back((float)in->thick[i]);
    }
    m.potential_slicing = in->potential_slicing;
    if (m.potential_slicing != 1 && m.potential_slicing != 2)
        fail(MT_ERR_UNSUPPORTED, "only potential_slicing 1 (planes) and 2 (dz_Proj) are implemented");

    if (in->nx <= 0 || in->ny <= 0) fail(MT_ERR_INVALID_ARG, "nx and ny must be positive");
    m.grid.set(in->nx, in->ny, lx, ly, dz, in->bwl != 0, true);

    // validate_incident_wave_type (src/input_multislice.cuh:438-448)
    int iw = in->iw_type;
    if (iw == 4) iw = (m.is_scanning() || m.is_CBED() || m.is_CBEI()) ? 2 : 1;
    m.iw_type = iw;
    if (m.is_scanning() && iw != 2) fail(MT_ERR_UNSUPPORTED, "STEM and ISTEM need a convergent incident wave");
    if (m.is_wave_sim() && iw == 3) {
        if (!in->iw_psi) fail(MT_ERR_INVALID_ARG, "iw_type 3 needs iw_psi");
        size_t n = (size_t)in->nx * in->ny;
        m.iw_psi.resize(2 * n);
        for (size_t i = 0; i < 2 * n; i++) m.iw_psi[i] = (float)in->iw_psi[i];
    }
    if (m.is_wave_sim() && iw == 3 && in->n_iw_xy < 1)
        fail(MT_ERR_INVALID_ARG, "a user-defined incident wave needs its position in iw_x/iw_y");
    for (int i = 0; i < in->n_iw_xy; i++) {
        m.iw_x.push_back((float)in->iw_x[i]);
        m.iw_y.push_back((float)in->iw_y[i]);
    }

    m.E_0 = (float)in->E_0;
    m.theta = (float)((float)in->theta * kDeg);
    m.phi = (float)((float)in->phi * kDeg);
    // ilc_multem.cu:338-347 and validate_parameters (src/input_multislice.cuh:655-660)
    if (m.is_PED() || m.is_HCTEM()) {
        m.theta = (float)((float)(m.is_PED() ? in->ped_theta : in->hci_theta) * kDeg);
        m.nrot = std::max(1, (int)(float)(m.is_PED() ? in->ped_nrot : in->hci_nrot));
        m.dp_shift = m.is_PED();
    }

    m.cond_lens.from_input(in->cond_lens);
    m.cond_lens.set_input_data(m.E_0, m.grid);
    m.illumination_model = in->illumination_model;
    m.temporal_spatial_incoh = in->temporal_spatial_incoh;
    mt_lens obj = in->obj_lens;
    obj.si_sigma = in->cond_lens.si_sigma;  // ilc_multem.cu:251 reads the condenser's value
    m.obj_lens.from_input(obj);
    m.obj_lens.set_input_data(m.E_0, m.grid);

    if (m.is_scanning()) {
        // Scanning::set_grid (src/types.cuh:4294-4390), regular grid
        m.scan_type = in->scanning_type;
        m.scan_pbc = in->scanning_periodic != 0;
        m.scan_spxs = in->scanning_square_pxs != 0;
        m.scan_ns = in->scanning_ns;
        m.scan_x0 = (float)in->scanning_x0;
        m.scan_y0 = (float)in->scanning_y0;
        m.scan_xe = (float)in->scanning_xe;
        m.scan_ye = (float)in->scanning_ye;
        if (m.scan_ns <= 0) fail(MT_ERR_INVALID_ARG, "scanning_ns must be positive");
        const int ns = m.scan_ns;
        m.scan_nx = m.scan_ny = ns;
        const float eps_rel = 1e-4f;
        if (m.scan_type == 1) {
            float xu = m.scan_xe - m.scan_x0, yu = m.scan_ye - m.scan_y0;
            float ds = std::sqrt(yu * yu + xu * xu);
            float th = std::atan2(yu, xu);
            float ct = std::cos(th);
            ct = is_zero_f(ct) ? 0.0f : ct;
            float st = std::sin(th);
            m.scan_dRx = ds * ct / (float)(m.scan_pbc ? ns : (ns - 1));
            m.scan_dRy = ds * st / (float)(m.scan_pbc ? ns : (ns - 1));
            for (int i = 0; i < ns; i++) {
                m.scan_x.push_back(m.scan_x0 + i * m.scan_dRx);
                m.scan_y.push_back(m.scan_y0 + i * m.scan_dRy);
            }
            m.scan_nx = 1;
            m.scan_ny = ns;
        } else {
            float xu = m.scan_xe - m.scan_x0, yu = m.scan_ye - m.scan_y0;
            if (std::fabs(xu) > std::fabs(yu)) {
                m.scan_dRx = xu / (float)(m.scan_pbc ? ns : (ns - 1));
                m.scan_dRy = std::copysign(m.scan_dRx, yu);
                m.scan_ny = (int)std::floor(yu / m.scan_dRy + eps_rel + 0.5f);
                m.scan_ny += m.scan_pbc ? 0 : 1;
                if (!m.scan_spxs) m.scan_dRy = yu / (float)(m.scan_pbc ? m.scan_ny : (m.scan_ny - 1));
            } else {
                m.scan_dRy = yu / (float)(m.scan_pbc ? ns : (ns - 1));
                m.scan_dRx = std::copysign(m.scan_dRy, xu);
                m.scan_nx = (int)std::floor(xu / m.scan_dRx + eps_rel + 0.5f);
                m.scan_nx += m.scan_pbc ? 0 : 1;
                if (!m.scan_spxs) m.scan_dRx = xu / (float)(m.scan_pbc ? m.scan_nx : (m.scan_nx - 1));
            }
            for (int ix = 0; ix < m.scan_nx; ix++)
                for (int iy = 0; iy < m.scan_ny; iy++) {
                    m.scan_x.push_back(m.scan_x0 + ix * m.scan_dRx);
                    m.scan_y.push_back(m.scan_y0 + iy * m.scan_dRy);
                }
        }
        if (m.scan_nx <= 0 || m.scan_ny <= 0) fail(MT_ERR_INVALID_ARG, "empty scan");
    }
    if (m.is_STEM()) {
        if (in->detector_type != 1 && in->detector_type != 3)
            fail(MT_ERR_UNSUPPORTED, "only circular (type 1) and matrix (type 3) detectors are implemented");
        m.det_type = in->detector_type;
        float lam = lambda_f(m.E_0);
        if (m.det_type == 1) {
            for (int i = 0; i < in->n_detector; i++) {
                double ia = (double)(float)in->detector_inner_ang[i] * kMrad;
                double oa = (double)(float)in->detector_outer_ang[i] * kMrad;
                m.det_g_inner.push_back((float)(std::sin(ia) / lam));
                m.det_g_outer.push_back((float)(std::sin(oa) / lam));
            }
        } else if (in->n_detector > 0) {
            // matrix detectors: fR as float, fft2-shifted to the FFT order the waves use
            // (Wave_Function::set_input_data, src/wave_function.cuh:55-61)
            if (!in->detector_fR) fail(MT_ERR_INVALID_ARG, "matrix detectors need detector_fR");
            const int nx = m.grid.nx, ny = m.grid.ny, nxh = nx / 2, nyh = ny / 2;
            const size_t nxy = (size_t)nx * ny;
            m.det_fR.assign((size_t)in->n_detector * nxy, 0.0f);
            for (int d = 0; d < in->n_detector; d++) {
                m.det_g_inner.push_back(0.0f);
                m.det_g_outer.push_back(0.0f);
                for (int ix = 0; ix < nx; ix++)
                    for (int iy = 0; iy < ny; iy++)
                        m.det_fR[d * nxy + (size_t)((ix + nxh) % nx) * ny + (iy + nyh) % ny] =
                            (float)in->detector_fR[d * nxy + (size_t)ix * ny + iy];
            }
        }
        if (m.det_g_inner.empty()) fail(MT_ERR_INVALID_ARG, "STEM needs at least one detector");
        if (m.det_g_inner.size() > 8) fail(MT_ERR_UNSUPPORTED, "at most 8 detectors are supported");
    }

    // ---- validate_parameters ----
    if (m.pn_seed < 1) m.clamps.push_back("pn_seed " + std::to_string(m.pn_seed) + " -> 1");
    m.pn_seed = std::max(1, m.pn_seed);
    const int nconf_in = m.pn_nconf;
    m.pn_nconf = (!m.is_frozen_phonon()) ? 1 : std::max(1, m.pn_nconf);
    if (m.pn_nconf != nconf_in) m.clamps.push_back("pn_nconf " + std::to_string(nconf_in) + " -> " + std::to_string(m.pn_nconf));
    m.fp_iconf_0 = (!m.is_frozen_phonon()) ? 1 : (m.pn_single_conf ? m.pn_nconf : 1);
    m.lambda = lambda_f(m.E_0);
    snap_incident_angle(m);
    if (m.is_EW()) m.pn_coh_contrib = true;
    if ((m.is_HCTEM() || m.is_ISTEM()) && m.pn_coh_contrib)
        fail(MT_ERR_UNSUPPORTED, "ISTEM/HCTEM with pn_coh_contrib = 1 (the image of the coherent wave, m2psi_coh) "
                                 "is not implemented; ED, CBED, PED, HRTEM and CBEI have it");
    if (m.pn_z && m.is_frozen_phonon()) m.clamps.push_back("pn_dim: z displacement switched off (no subslicing)");
    m.pn_z = false;  // no subslicing: pn_dim.z is switched off (input_multislice.cuh:705-708)

    // specimen rotation (input_multislice.cuh:707-722): whole-specimen thickness, the atoms rotated
    // by spec_rot_theta about the unit axis u0 through the geometric centre (mean position) or a
    // user point (rotate_atoms, src/atomic_data_mt.hpp:61-74; get_rotation_matrix,
    // src/cgpu_fcns.cuh:185-205; r3d::rotate, src/lin_alg_def.cuh:355-360), all in float
    const float rot_theta = (float)((float)in->spec_rot_theta * kDeg);
    if (!is_zero_f(rot_theta)) {
        m.thick_type = 1;
        float ux = (float)in->spec_rot_u0[0], uy = (float)in->spec_rot_u0[1], uz = (float)in->spec_rot_u0[2];
        const float un = std::sqrt(ux * ux + uy * uy + uz * uz);
        if (!(un > 0)) fail(MT_ERR_INVALID_ARG, "spec_rot_u0 must be a non-zero vector");
        ux /= un;
        uy /= un;
        uz /= un;
        float px = (float)in->spec_rot_center_p[0], py = (float)in->spec_rot_center_p[1], pz = (float)in->spec_rot_center_p[2];
        if (in->spec_rot_center_type == 1) {
            float sx = 0, sy = 0, sz = 0;
            for (size_t i = 0; i < A.size(); i++) {
                sx += A.x[i];
                sy += A.y[i];
                sz += A.z[i];
            }
            px = sx / (float)A.size();
            py = sy / (float)A.size();
            pz = sz / (float)A.size();
        }
        float alpha = 1.0f - std::cos(rot_theta);
        alpha = is_zero_f(alpha) ? 0.0f : alpha;
        float beta = std::sin(rot_theta);
        beta = is_zero_f(beta) ? 0.0f : beta;
        const float R[9] = {1.0f + alpha * (ux * ux - 1), uy * ux * alpha + uz * beta, uz * ux * alpha - uy * beta,
                            ux * uy * alpha - uz * beta, 1.0f + alpha * (uy * uy - 1), uz * uy * alpha + ux * beta,
                            ux * uz * alpha + uy * beta, uy * uz * alpha - ux * beta, 1.0f + alpha * (uz * uz - 1)};
        for (size_t i = 0; i < A.size(); i++) {
            const float x = A.x[i] - px, y = A.y[i] - py, z = A.z[i] - pz;
            A.x[i] = (R[0] * x + R[3] * y + R[6] * z) + px;
            A.y[i] = (R[1] * x + R[4] * y + R[7] * z) + py;
            A.z[i] = (R[2] * x + R[5] * y + R[8] * z) + pz;
        }
        A.statistic(nullptr);
    }

    // "temporal fix for phase object" (src/input_multislice.cuh:724-728)
    if (!m.is_multislice() && m.thick_type == 1) m.potential_slicing = 2;

    // Slicing::match_thickness (src/slicing.hpp:53-71)
    if (m.thick_type == 1) {
        m.thick.assign(1, A.z_max);
    } else {
        auto zp = z_planes(m.potential_slicing, A);
        if (m.thick_type == 3) zp = z_slices(m.potential_slicing, zp, A);
        const std::vector<float> req = m.thick;
        match_thick(zp, m.thick, (float)(0.25 * A.dz));
        if (m.thick.empty()) fail(MT_ERR_INVALID_ARG, "no requested thickness lies within the specimen");
        if (m.thick != req) {
            std::string r = "thick [";
            for (size_t i = 0; i < req.size(); i++) r += (i ? ", " : "") + std::to_string(req[i]);
            r += "] -> [";
            for (size_t i = 0; i < m.thick.size(); i++) r += (i ? ", " : "") + std::to_string(m.thick[i]);
            m.clamps.push_back(r + "] (matched to slice planes)");
        }
    }

    // remove atoms outside the thickness range (input_multislice.cuh:733-744)
    {
        const float ee_z = 0.1f;
        const float z_e = m.thick.back() + ee_z;
        if (A.z_max > z_e) {
            const float z_0 = A.z_min - ee_z;
            AtomsF B = A;
            size_t k = 0;
            for (size_t i = 0; i < A.size(); i++) {
                if ((z_0 < A.z[i]) && (A.z[i] < z_e)) {
                    B.Z[k] = A.Z[i]; B.x[k] = A.x[i]; B.y[k] = A.y[i]; B.z[k] = A.z[i];
                    B.sigma[k] = A.sigma[i]; B.occ[k] = A.occ[i]; B.region[k] = A.region[i]; B.charge[k] = A.charge[i];
                    k++;
                }
            }
            B.resize(k);
            m.clamps.push_back(std::to_string(A.size() - k) + " atoms beyond the last thickness removed");
            A = B;
            A.statistic(nullptr);
        }
    }

    // illumination (src/input_multislice.cuh:672-676, 747-776): exit waves are coherent; without
    // full integration, or with spatial incoherence only, the condenser has one defocus point
    if (m.is_EW()) m.illumination_model = 1;
    if ((m.is_CBED() || m.is_CBEI()) && m.illumination_model != 4) m.illumination_model = 1;
    if (is_zero_f(m.cond_lens.si_sigma)) m.temporal_spatial_incoh = 2;
    const bool full_integration = (m.illumination_model == 4);
    if (!full_integration || m.temporal_spatial_incoh == 3) m.cond_lens.ti_npts = 1;
    if (!full_integration || m.temporal_spatial_incoh == 2) m.cond_lens.si_rad_npts = m.cond_lens.si_azm_npts = 1;
    m.cond_lens.set_input_data(m.E_0, m.grid);
    if (!full_integration || m.temporal_spatial_incoh == 3) m.obj_lens.ti_npts = 1;
    m.obj_lens.set_input_data(m.E_0, m.grid);
    if (m.is_imaging()) hrtem_ctf_points(m);
    // Multislice::STEM_ISTEM integrates the defocus spread only under full integration, and not
    // in its coherent-contribution branch, which comes first (src/tem_simulation.cuh:115-176)
    if (m.is_scanning() && full_integration && !m.pn_coh_contrib) temporal_quadrature(m.cond_lens, m.ti_x, m.ti_w);
    // CBED/CBEI under full integration: every configuration runs every (source point, defocus
    // point) pair with the beams moved by the source offset (Multislice::CBED_CBEI,
    // src/tem_simulation.cuh:203-259)
    if ((m.is_CBED() || m.is_CBEI()) && full_integration) {
        temporal_quadrature(m.cond_lens, m.ti_x, m.ti_w);
        spatial_quadrature(m.cond_lens, m.si_x, m.si_y, m.si_w);
    }
    m.cond_lens.zero_defocus_plane = A.size() ? m.cond_lens.get_zero_defocus_plane(A.z_min, A.z_max) : 0.0f;
    m.cond_lens.zero_defocus_type = 4;
    m.obj_lens.set_input_data(m.E_0, m.grid);

    // validate_output_area (src/input_multislice.cuh:823-860)
    m.out_ix_0 = in->output_area_ix_0 - 1;
    m.out_iy_0 = in->output_area_iy_0 - 1;
    m.out_ix_e = in->output_area_ix_e - 1;
    m.out_iy_e = in->output_area_iy_e - 1;
    if (m.is_STEM() || m.out_ix_0 == m.out_ix_e) {
        m.out_ix_0 = 0;
        m.out_ix_e = m.grid.nx;
    }
    if (m.is_STEM() || m.out_iy_0 == m.out_iy_e) {
        m.out_iy_0 = 0;
        m.out_iy_e = m.grid.ny;
    }
    if (m.out_ix_0 > m.out_ix_e) std::swap(m.out_ix_0, m.out_ix_e);
    if (m.out_iy_0 > m.out_iy_e) std::swap(m.out_iy_0, m.out_iy_e);
    m.out_ix_0 = std::max(0, std::min(m.grid.nx, m.out_ix_0));
    m.out_ix_e = std::max(0, std::min(m.grid.nx, m.out_ix_e));
    m.out_iy_0 = std::max(0, std::min(m.grid.ny, m.out_iy_0));
    m.out_iy_e = std::max(0, std::min(m.grid.ny, m.out_iy_e));
    // an area given by the caller (not the "whole grid" default ix_0 == ix_e) that had to be
    // reordered or clipped
    const bool area_given = in->output_area_ix_0 != in->output_area_ix_e || in->output_area_iy_0 != in->output_area_iy_e;
    if ((m.is_wave_sim() || m.is_ISTEM()) && area_given &&
        (m.out_ix_0 != in->output_area_ix_0 - 1 || m.out_ix_e != in->output_area_ix_e - 1 ||
         m.out_iy_0 != in->output_area_iy_0 - 1 || m.out_iy_e != in->output_area_iy_e - 1))
        m.clamps.push_back("output_area -> ix [" + std::to_string(m.out_ix_0 + 1) + ", " + std::to_string(m.out_ix_e + 1) +
                           "], iy [" + std::to_string(m.out_iy_0 + 1) + ", " + std::to_string(m.out_iy_e + 1) + "]");
    return m;
}

// ---------------------------------------------------------------------------------------------
// Spec::set_input_data (src/spec.hpp:44-82)
Specimen::Specimen(const Model& m, const std::vector<float>& R_max_of_Z) : m_(m), R_max_of_Z_(R_max_of_Z) {
    const AtomsF& in = m.atoms_in;
    // Atom_Data::set_atoms(atoms, pbc_xy = true, atom_type) (src/atomic_data_mt.hpp:353-405)
    atoms_u_ = AtomsF();
    atoms_u_.l_x = in.l_x;
    atoms_u_.l_y = in.l_y;
    atoms_u_.l_z = in.l_z;
    atoms_u_.dz = in.dz;
    const float dl = 1e-04f;
    const float lx_b = in.l_x - dl, ly_b = in.l_y - dl;
    for (size_t i = 0; i < in.size(); i++) {
        if ((in.x[i] < lx_b) && (in.y[i] < ly_b)) {
            atoms_u_.Z.push_back(in.Z[i]);
            atoms_u_.x.push_back(in.x[i]);
            atoms_u_.y.push_back(in.y[i]);
            atoms_u_.z.push_back(in.z[i]);
            atoms_u_.sigma.push_back(in.sigma[i]);
            atoms_u_.occ.push_back(in.occ[i]);
            atoms_u_.region.push_back(in.region[i]);
            atoms_u_.charge.push_back(in.charge[i]);
        }
    }
    atoms_u_.amorp = in.amorp;
    if (atoms_u_.size() == 0) fail(MT_ERR_INVALID_ARG, "no atoms inside the simulation box");
    atoms_u_.statistic(R_max_of_Z_.data());
    atoms_u_.sort_by_z();
    z_plane_ = z_planes(m.potential_slicing, atoms_u_);
    grid_dz_ = m.grid.dz;
    // phase-object switch (src/spec.hpp:65-77): a phase object requested, or a specimen thinner
    // than two slices, or a single plane under plane slicing, is transmitted without propagation,
    // one slice per thickness (the weak phase object uses the same slicing, Slicing::get_thick /
    // get_slicing branch on !is_multislice, src/slicing.hpp:326-356)
    thick_type_ = m.thick_type;
    if ((m.interaction_model == 2) || (atoms_u_.s_z_int < 2.0f * grid_dz_) ||
        ((z_plane_.size() == 1) && m.potential_slicing == 1)) {
        phase_object_ = true;
        grid_dz_ = atoms_u_.s_z_int;
        atoms_u_.dz = grid_dz_;
        if (thick_type_ == 3) thick_type_ = 2;
    }
    phase_object_ = phase_object_ || !m.is_multislice();
    atoms_ = atoms_u_;
    atoms_.statistic(R_max_of_Z_.data());
    calculate();
}

// Spec::move_atoms (src/spec.hpp:85-127) with Randn_3d<float, e_host> (src/cgpu_rand.cuh:308-395)
void Specimen::move_atoms(int iconf) {
    std::mt19937_64 gen_u, gen_x, gen_y, gen_z;
    std::uniform_int_distribution<int> rand_u(1);
    std::normal_distribution<float> randn_x(0.0f, 1.0f), randn_y(0.0f, 1.0f), randn_z(0.0f, 1.0f);
    const bool fp = m_.is_frozen_phonon();
    if (fp) {
        int n_iter = std::max(1, iconf);
        gen_u.seed(m_.pn_seed);
        rand_u.reset();
        unsigned int sx = 0, sy = 0, sz = 0;
        for (int ic = 0; ic < n_iter; ic++) {
            sx = rand_u(gen_u);
            sy = rand_u(gen_u);
            sz = rand_u(gen_u);
        }
        gen_x.seed(sx);
        randn_x.reset();
        gen_y.seed(sy);
        randn_y.reset();
        gen_z.seed(sz);
        randn_z.reset();
    }
    for (size_t i = 0; i < atoms_u_.size(); i++) {
        atoms_.Z[i] = atoms_u_.Z[i];
        float x = atoms_u_.x[i], y = atoms_u_.y[i], z = atoms_u_.z[i];
        if (fp) {
            float s = atoms_u_.sigma[i];
            float dx = m_.pn_x ? s * randn_x(gen_x) : 0.0f;
            float dy = m_.pn_y ? s * randn_y(gen_y) : 0.0f;
            float dzv = m_.pn_z ? s * randn_z(gen_z) : 0.0f;
            x += dx;
            y += dy;
            z += dzv;
        }
        atoms_.x[i] = x;
        atoms_.y[i] = y;
        atoms_.z[i] = z;
        atoms_.sigma[i] = atoms_u_.sigma[i];
        atoms_.occ[i] = atoms_u_.occ[i];
        atoms_.region[i] = atoms_u_.region[i];
        atoms_.charge[i] = atoms_u_.charge[i];
    }
    if (m_.pn_z) atoms_.sort_by_z();
    atoms_.statistic(R_max_of_Z_.data());
    calculate();
}

void Specimen::still_atoms() {
    atoms_ = atoms_u_;
    atoms_.statistic(R_max_of_Z_.data());
    calculate();
}

// Slicing::calculate (src/slicing.hpp:93-100) = get_z_slice + get_thick + get_slicing
void Specimen::calculate() {
    z_slice_ = z_slices(m_.potential_slicing, z_plane_, atoms_);

    // get_thick (src/slicing.hpp:253-336), thickness atoms from the undisplaced specimen
    const auto& zr = atoms_u_.z;
    thick_.assign(m_.thick.size(), ThickF());
    for (size_t ik = 0; ik < thick_.size(); ik++) {
        ThickF& t = thick_[ik];
        t.z = m_.thick[ik];
        int islice = 0;
        if (thick_type_ == 3) {
            for (size_t i = 0; i + 1 < z_slice_.size(); i++)
                if (std::fabs(z_slice_[i + 1] - t.z) < 1e-4f) { islice = (int)i; break; }
        } else {
            for (size_t i = 0; i + 1 < z_slice_.size(); i++)
                if ((z_slice_[i] < t.z) && (t.z <= z_slice_[i + 1])) { islice = (int)i; break; }
        }
        t.islice = islice;
        t.iatom_e = last_atom_below(zr, z_slice_[islice + 1]);
        float za = zr[0], zb = zr[std::max(0, t.iatom_e)];
        t.z_zero_def_plane = m_.obj_lens.get_zero_defocus_plane(za, zb);
        if (thick_type_ == 3) {
            t.z_back_prop = 0;
        } else {
            t.z_back_prop = (float)(t.z_zero_def_plane - 0.5 * (z_slice_[islice] + z_slice_[islice + 1]));
            if (std::fabs(t.z_back_prop) < 1e-4f) t.z_back_prop = 0;
        }
    }
    if (phase_object_) {
        // one slice per thickness, back-propagated from the thickness plane
        for (size_t ik = 0; ik < thick_.size(); ik++) {
            thick_[ik].islice = (int)ik;
            thick_[ik].z_back_prop = thick_[ik].z_zero_def_plane - thick_[ik].z;
        }
        slice_.assign(thick_.size(), SliceF());
        for (size_t i = 0; i < slice_.size(); i++) {
            SliceF& s = slice_[i];
            s.z_0 = (i == 0) ? atoms_.z_int_min : thick_[i - 1].z;
            s.z_e = (thick_.size() == 1) ? atoms_.z_int_max : thick_[i].z;
            s.z_int_0 = s.z_0;
            s.z_int_e = s.z_e;
            s.iatom_0 = (i == 0) ? 0 : thick_[i - 1].iatom_e + 1;
            s.iatom_e = thick_[i].iatom_e;
            s.ithk = (int)i;
        }
        return;
    }

    // get_slicing (src/slicing.hpp:339-403)
    slice_.assign(z_slice_.size() - 1, SliceF());
    for (size_t i = 0; i < slice_.size(); i++) {
        SliceF& s = slice_[i];
        s.z_0 = z_slice_[i];
        s.z_e = z_slice_[i + 1];
        s.z_int_0 = s.z_0;
        s.z_int_e = s.z_e;
        atoms_in_range(atoms_.z, s.z_int_0, s.z_int_e, s.iatom_0, s.iatom_e);
        s.ithk = -1;
    }
    for (size_t ithk = 0; ithk < thick_.size(); ithk++) slice_[thick_[ithk].islice].ithk = (int)ithk;
}

// Spec::dz (src/spec.hpp:129-132)
float Specimen::dz(int islice) const {
    if (phase_object_) return 0.0f;  // transmission only (Wave_Function::psi_slice, src/wave_function.cuh:230-238)
    float d = (islice < (int)slice_.size()) ? slice_[islice].z_e - slice_[islice].z_0 : 0.0f;
    return d / std::cos(m_.theta);
}

}  // namespace mtb
