// Multislice engine: the batched slice loop on the device.
//
// Control flow follows Multislice::STEM_ISTEM / EWFS_EWRS (src/tem_simulation.cuh:101-200,
// 304-325): for every frozen-phonon configuration, displace the atoms (host), build the
// transmission functions of all slices (device splat), then push the incident waves through the
// slices and reduce them at every requested thickness. The reference does one probe at a time,
// four launches per slice and a host round trip per detector and thickness; here a batch of probes
// advances slice by slice together (two passes per slice over the whole batch, the transmission
// function of a slice shared from L2 by all probes), and detector sums stay on the device in FP64
// until the end of the run.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "common.hpp"
#include "engine.hpp"

namespace mtb {

namespace {

bool is_zero_f(float a) {
    float d = std::fabs(a);
    return d <= 1e-5f;
}

int env_int(const char* name, int dflt) {
    const char* v = std::getenv(name);
    return v ? std::atoi(v) : dflt;
}

}  // namespace

GridDev grid_dev(const GridF& g) {
    GridDev d{};
    d.nx = g.nx;
    d.ny = g.ny;
    d.nxh = g.nxh;
    d.nyh = g.nyh;
    d.lx = g.lx;
    d.ly = g.ly;
    d.dRx = g.dRx;
    d.dRy = g.dRy;
    d.Rx_0 = g.Rx_0;
    d.Ry_0 = g.Ry_0;
    d.dgx = g.dgx;
    d.dgy = g.dgy;
    return d;
}

Engine::Engine(const mt_system_conf* conf, const mt_input_multislice* in) {
    if (conf) {
        if (conf->precision != 1)
            fail(MT_ERR_UNSUPPORTED, "this engine computes in FP32 (system_conf.precision must be 1)");
        if (conf->device != 2) fail(MT_ERR_UNSUPPORTED, "this engine runs on the GPU (system_conf.device must be 2)");
        device_ = conf->gpu_device;
    }
    // the input is validated on the host first, so its errors do not depend on a GPU
    m_ = build_model(in);
    if (!m_.clamps.empty() && env_int("MTB_STRICT", 0) != 0) {
        std::string r = "MTB_STRICT: the input needs changes the reference would apply silently:";
        for (const auto& c : m_.clamps) r += " " + c + ";";
        fail(MT_ERR_INVALID_ARG, r);
    }
    int ndev = 0;
    MTB_CUDA(cudaGetDeviceCount(&ndev));
    if (device_ < 0 || device_ >= ndev) fail(MT_ERR_INVALID_ARG, "gpu_device out of range");
    MTB_CUDA(cudaSetDevice(device_));
    MTB_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));

    const int nx = m_.grid.nx, ny = m_.grid.ny;
    if (!line_size_supported(nx) || !line_size_supported(ny))
        fail(MT_ERR_UNSUPPORTED, "nx and ny must be one of 64, 128, 256, 384, 512, 1024, 2048");

    gdev_ = grid_dev(m_.grid);

    build_types();
    std::vector<float> rmax_of_Z(103, 0.0f);
    for (size_t t = 0; t < Z_of_type_.size(); t++) rmax_of_Z[Z_of_type_[t] - 1] = R_max_f_[t];
    spec_.reset(new Specimen(m_, rmax_of_Z));

    const size_t nxy = (size_t)nx * ny;
    const int n_thk = (int)m_.thick.size();
    if (m_.is_scanning()) {
        // 64 Mi complex values (512 MiB) per batch, a multiple of the row pipeline's 8 groups
        int bdef = std::max(1, (int)((size_t)1 << 26) / (int)nxy);
        if (bdef >= 8) bdef -= bdef % 8;
        int bmax = env_int("MTB_BATCH", bdef);
        batch_ = std::max(1, std::min(bmax, m_.n_scan()));
        const int n_det = (int)m_.det_g_inner.size();
        if (m_.is_STEM()) {
            d_image_.alloc((size_t)n_thk * n_det * m_.n_scan());
            d_partial_.alloc((size_t)n_thk * batch_ * col_tiles(nx, ny) * n_det);
        } else {
            // ISTEM: one image per thickness, the images of every probe summed
            const size_t onxy = (size_t)(m_.out_ix_e - m_.out_ix_0) * (m_.out_iy_e - m_.out_iy_0);
            d_ew_m2_.alloc((size_t)n_thk * onxy);
            d_tmp_.alloc((size_t)batch_ * nxy);
        }
        std::vector<float2> beam(m_.n_scan());
        std::vector<int> idx(m_.n_scan());
        for (int i = 0; i < m_.n_scan(); i++) {
            beam[i] = make_float2(m_.grid.exp_factor_Rx(m_.scan_x[i]), m_.grid.exp_factor_Ry(m_.scan_y[i]));
            idx[i] = i;
        }
        d_beam_.upload(beam.data(), beam.size(), stream_);
        if (m_.det_type == 3) d_detmat_.upload(m_.det_fR.data(), m_.det_fR.size(), stream_);
        if (m_.pn_coh_contrib) {
            // the coherent part keeps every probe's transformed wave summed over configurations
            const size_t n = (size_t)n_thk * m_.n_scan() * nxy;
            if (n * sizeof(float2) > ((size_t)96 << 30))
                fail(MT_ERR_UNSUPPORTED, "pn_coh_contrib: the probes' coherent waves need more than 96 GiB");
            d_coh_.alloc(n);
            d_image_coh_.alloc((size_t)n_thk * n_det * m_.n_scan());
        }
        d_scan_idx_.upload(idx.data(), idx.size(), stream_);
        probe_norm_ = aperture_norm();
        niter_ = m_.n_scan() * m_.number_conf() * (int)m_.ti_x.size();
    } else {
        batch_ = 1;
        const size_t onxy = (size_t)(m_.out_ix_e - m_.out_ix_0) * (m_.out_iy_e - m_.out_iy_0);
        if (m_.is_EW()) d_ew_psi_.alloc((size_t)n_thk * onxy * 2);
        if (m_.pn_coh_contrib && !m_.is_EW() && !m_.is_imaging()) d_ew_cohpsi_.alloc((size_t)n_thk * onxy * 2);
        if (m_.pn_coh_contrib && m_.is_imaging()) {
            d_coh_img_.alloc((size_t)n_thk * nxy);
            d_coh_m2_.alloc((size_t)n_thk * onxy);
        }
        d_ew_m2_.alloc((size_t)n_thk * onxy);
        // frozen-phonon configurations advance together (one launch per pass for all of them) where
        // every configuration runs the same sequence of passes: a plane incident wave, one beam
        // rotation, no source or defocus quadrature; the transmission functions of all of them are
        // held at once (at most 32 GiB)
        const bool batchable = !m_.is_convergent_wave() && !m_.is_user_wave() && m_.nrot == 1 &&
                               m_.si_x.size() * m_.ti_x.size() == 1;
        const size_t trans_bytes = spec_->slices().size() * nxy * sizeof(float2);
        int eb = batchable ? std::min(8, m_.number_conf()) : 1;
        while (eb > 1 && (size_t)eb * trans_bytes > ((size_t)32 << 30)) eb--;
        ew_batch_ = batchable ? std::max(1, std::min(env_int("MTB_EW_BATCH", eb), m_.number_conf())) : 1;
        d_tmp_.alloc((size_t)ew_batch_ * nxy);
        niter_ = m_.number_conf() * m_.nrot * (int)(m_.si_x.size() * m_.ti_x.size());
        if (m_.is_convergent_wave()) {
            // convergent beams at iw_x/iw_y, summed (Incident_Wave::operator(), src/incident_wave.cuh:72-90);
            // one set of beams per source point (beam_x = iw_x + qs.x in the working precision,
            // src/tem_simulation.cuh:233-237), one source point without full integration
            const int nb = (int)m_.iw_x.size();
            if (nb <= 0 || m_.iw_y.size() != m_.iw_x.size()) fail(MT_ERR_INVALID_ARG, "convergent wave needs iw_x/iw_y");
            const size_t ns = m_.si_x.size();
            std::vector<float2> beam(ns * nb);
            for (size_t s = 0; s < ns; s++)
                for (int i = 0; i < nb; i++) {
                    const float bx = (float)((double)m_.iw_x[i] + m_.si_x[s]);
                    const float by = (float)((double)m_.iw_y[i] + m_.si_y[s]);
                    beam[s * nb + i] = make_float2(m_.grid.exp_factor_Rx(bx), m_.grid.exp_factor_Ry(by));
                }
            d_beam_.upload(beam.data(), beam.size(), stream_);
            if (nb > 1) d_beams_psi_.alloc((size_t)nb * nxy);
            probe_norm_ = aperture_norm();
        }
    }
    d_psi_.alloc((size_t)std::max(batch_, ew_batch_) * nxy);
    slot_.resize(2 * (size_t)ew_batch_);
    if (m_.grid.bwl) build_bwl();
    if (m_.is_imaging()) build_ctf_tables();
    if (m_.tilted()) {
        build_tilt_ramp();
        // STEM outputs at intermediate thicknesses apply the ramp to a copy of the batch
        if (m_.is_scanning() && n_thk > 1) d_tmp_.alloc((size_t)batch_ * nxy);
        if (m_.is_ISTEM() && n_thk > 1) d_tmp2_.alloc((size_t)batch_ * nxy);
    }
    d_trans_.alloc((size_t)ew_batch_ * spec_->slices().size() * nxy);
    d_err_.alloc(1);
    MTB_CUDA(cudaMemsetAsync(d_err_.p, 0, sizeof(int), stream_));
    // line-pass variants: MTB_PIPE pins them (bit 0 rows, bit 1 columns: bulk-copy fed) and
    // MTB_SHAPE the pipeline shapes of the slice step (bits 0-1 rows, bits 2-3 columns: 0 default,
    // 1 or 2 alternatives), else the autotuner picks them and the probes per launch
    pipe_ = env_int("MTB_PIPE", -1);
    graphs_ = env_int("MTB_GRAPH", 1) != 0;
    tune_ = pipe_ < 0;
    if (tune_) pipe_ = 3;
    shape_ = tune_ ? 0 : env_int("MTB_SHAPE", 0) & 15;
    run_batch_ = batch_;
    if (m_.is_wave_sim() && m_.is_user_wave()) build_user_wave();
    reset();
}

Engine::~Engine() {
    if (stream_) {
        cudaStreamSynchronize(stream_);
        // everything below was used on stream_ only: return it to the pool without a device-wide wait
        for (auto& cd : confs_) cd.release_idle();
        for (auto& cd : slot_) cd.release_idle();
        for (auto& g : graph_)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        if (range_graph_.exec) cudaGraphExecDestroy(range_graph_.exec);
        for (auto* b : {&d_tab_, &d_Rmax_}) b->release_idle();
        for (auto* b : {&d_psi_, &d_trans_, &d_tmp_, &d_beam_, &d_prop_bp_, &d_ramp_}) b->release_idle();
        d_detmat_.release_idle();
        d_ctf_.release_idle();
        d_beams_psi_.release_idle();
        d_user_wave_.release_idle();
        d_tmp2_.release_idle();
        for (auto* b : {&d_bwl_, &d_one_, &d_p0_}) b->release_idle();
        d_coh_.release_idle();
        d_image_coh_.release_idle();
        for (auto* b : {&d_partial_, &d_image_, &d_ew_psi_, &d_ew_m2_}) b->release_idle();
        d_err_.release_idle();
        d_scan_idx_.release_idle();
        for (auto& t : tl_) {
            cudaEventDestroy(t.a);
            cudaEventDestroy(t.b);
        }
        if (conf_done_) cudaEventDestroy(conf_done_);
        if (run_a_) cudaEventDestroy(run_a_);
        if (run_b_) cudaEventDestroy(run_b_);
        cudaStreamDestroy(stream_);
    }
}

void Engine::synchronize() {
    MTB_CUDA(cudaStreamSynchronize(stream_));
    if (d_err_.p) {
        int e = 0;
        MTB_CUDA(cudaMemcpy(&e, d_err_.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (e) {
            MTB_CUDA(cudaMemset(d_err_.p, 0, sizeof(int)));
            fail(MT_ERR_TIMEOUT, "a line pass timed out waiting for its bulk copies; results are invalid");
        }
    }
}

void Engine::reset() {
    zero_accumulators();
    iter_ = 0;
    cancel_ = false;
    synchronize();
}

void Engine::zero_accumulators() {
    if (d_image_.p) MTB_CUDA(cudaMemsetAsync(d_image_.p, 0, sizeof(double) * d_image_.n, stream_));
    if (d_coh_.p) MTB_CUDA(cudaMemsetAsync(d_coh_.p, 0, sizeof(float2) * d_coh_.n, stream_));
    if (d_ew_psi_.p) MTB_CUDA(cudaMemsetAsync(d_ew_psi_.p, 0, sizeof(double) * d_ew_psi_.n, stream_));
    if (d_ew_m2_.p) MTB_CUDA(cudaMemsetAsync(d_ew_m2_.p, 0, sizeof(double) * d_ew_m2_.n, stream_));
    if (d_ew_cohpsi_.p) MTB_CUDA(cudaMemsetAsync(d_ew_cohpsi_.p, 0, sizeof(double) * d_ew_cohpsi_.n, stream_));
    if (d_coh_img_.p) MTB_CUDA(cudaMemsetAsync(d_coh_img_.p, 0, sizeof(float2) * d_coh_img_.n, stream_));
}

// Element spline tables for the elements present (Spec::set_input_data builds all 103,
// src/spec.hpp:49-55; only the present ones are ever read).
// One table per (element, charge) in the specimen; an ion without its own coefficients shares its
// element's neutral table. Atoms carry the table index (atom_type(Z, charge)).
int Engine::atom_type(int Z, int charge) const {
    const int q = effective_charge(Z, charge);
    return type_of_Zq_[(size_t)(Z - 1) * kChargeSlots + (q + kChargeSlots / 2)];
}

void Engine::build_types() {
    type_of_Zq_.assign((size_t)103 * kChargeSlots, -1);
    Z_of_type_.clear();
    charge_of_type_.clear();
    const auto& A = m_.atoms_in;
    for (size_t i = 0; i < A.Z.size(); i++) {
        const int Z = A.Z[i] % 1000;
        const int q = effective_charge(Z, A.charge[i]);
        int& t = type_of_Zq_[(size_t)(Z - 1) * kChargeSlots + (q + kChargeSlots / 2)];
        if (t < 0) {
            t = (int)Z_of_type_.size();
            Z_of_type_.push_back(Z);
            charge_of_type_.push_back(q);
        }
    }
    if ((int)Z_of_type_.size() > kMaxTypes) fail(MT_ERR_UNSUPPORTED, "more than 16 (element, charge) types in one specimen");
    d_tab_.alloc((size_t)Z_of_type_.size() * 5 * m_.nR);
    heads_.clear();
    for (int Z : Z_of_type_) heads_.push_back(element_head(Z, m_.potential_type, m_.grid.dR_min(), m_.Vrl));
    build_tables(Z_of_type_, m_.potential_type, heads_, m_.nR, d_tab_.p, stream_, charge_of_type_);
    R_max_f_.resize(Z_of_type_.size());
    for (size_t t = 0; t < Z_of_type_.size(); t++) R_max_f_[t] = (float)heads_[t].R_max;
    d_Rmax_.upload(R_max_f_.data(), R_max_f_.size(), stream_);
    synchronize();
}

// Tilted beam: Wave_Function::get_psi (src/wave_function.cuh:96-105) multiplies the wave by
// exp(i*(gx*Rx + gy*Ry)), gx = 2*pi*(-gx_0), gy = 2*pi*(-gy_0), before the output propagation
// (phase_multiplication :77-94, exp_r_factor_2d src/cgpu_fcns.cuh:1869-1878, unscaled), with
// Rx = Rx_shift(ix) - Rx_c and Rx_c = int(lx/2) (Grid_2d::Rx_c returns an int, src/types.cuh:2284).
// Applied as a row step whose "transmission" is this table; the table carries the row pass's 1/ny
// so the result is in the layout the output propagator tables expect. Stored [ix][iy], one table
// per beam rotation that needs one (launch_tilt_ramp).
void Engine::build_tilt_ramp() {
    const GridF& g = m_.grid;
    const size_t nxy = (size_t)g.nx * g.ny;
    d_ramp_.alloc(nxy * m_.nrot);
    const float rxc = (float)(int)(g.Rx_0 + 0.5f * g.lx), ryc = (float)(int)(g.Ry_0 + 0.5f * g.ly);
    for (int r = 0; r < m_.nrot; r++) {
        if (!m_.ramp_needed(r)) continue;
        const float gx = (float)(2.0 * 3.141592653589793238463 * (double)(-m_.gx_0(r)));
        const float gy = (float)(2.0 * 3.141592653589793238463 * (double)(-m_.gy_0(r)));
        launch_tilt_ramp(gdev_, gx, gy, rxc, ryc, d_ramp_.p + r * nxy, stream_);
    }
}

// Band-width limit (bwl = 1): Grid_2d::bwl_factor_shift (src/types.cuh:2588-2598), the Fermi cut-off
// 1/(1 + exp(alpha (g^2 - gl2_max))) at two thirds of g_max, in float as the reference. The
// propagator multiplies by it (propagate, src/cgpu_fcns.cuh:1837-1845) and so do the transmission
// functions (Transmission_Function::trans, src/transmission_function.cuh:72-82); here it is the
// column passes' [nx][ny] factor (ColArgs::P2).
void Engine::build_bwl() {
    const GridF& g = m_.grid;
    const int nx = g.nx, ny = g.ny;
    std::vector<float2> f((size_t)nx * ny);
    for (int ix = 0; ix < nx; ix++) {
        const float gx = (float)((ix < g.nxh) ? ix : ix - nx) * g.dgx;
        for (int iy = 0; iy < ny; iy++) {
            const float gy = (float)((iy < g.nyh) ? iy : iy - ny) * g.dgy;
            const float g2 = gx * gx + gy * gy;
            const float e = std::exp(g.alpha * (g2 - g.gl2_max));
            f[(size_t)ix * ny + iy] = make_float2((float)(1.0 / (1.0 + (double)e)), 0.0f);
        }
    }
    d_bwl_.upload(f.data(), f.size(), stream_);
    std::vector<float2> ones((size_t)nx * ny, make_float2(1.0f, 0.0f));
    d_one_.upload(ones.data(), ones.size(), stream_);
    std::vector<float2> p0((size_t)nx + ny);
    mtb::prop_tables(m_, 0.0f, p0.data(), p0.data() + nx, false);
    d_p0_.upload(p0.data(), p0.size(), stream_);
    synchronize();
}

// bwl = 1: T <- IFFT(bwl_factor/N * FFT(T)) for the slices of a configuration, as three line passes
// over all slices at once (a real-space row pass, the column pass with the cut-off, the inverse row
// pass).
void Engine::band_limit_trans(const ConfData& cd, float2* trans) {
    const int nx = m_.grid.nx, ny = m_.grid.ny;
    const int ns = cd.last_slice + 1;
    RowArgs ra{};
    ra.in = trans;
    ra.out = trans;
    ra.trans = d_one_.p;
    ra.nx = nx;
    ra.nprobe = ns;
    ra.scale = 1.0f;
    rows(ROW_FIRST_REAL, ra);
    ColArgs ca{};
    ca.in = trans;
    ca.out = trans;
    ca.ny = ny;
    ca.nprobe = ns;
    ca.g = gdev_;
    ca.Px = d_p0_.p;
    ca.Py = d_p0_.p + nx;
    ca.P2 = d_bwl_.p;
    ca.det_w = col_det_width(nx);
    cols(COL_LOAD | COL_PROP | COL_INVERSE | COL_STORE, ca);
    RowArgs rb = ra;
    rows(ROW_INVERSE, rb);
}

// HRTEM: the objective's transfer function per defocus point (Microscope_Effects, see
// hrtem_ctf_points), as [nx][ny] tables in FFT order that the output column pass multiplies in
// after the back-propagation factors (get_psi then apply_CTF / apply_PCTF).
void Engine::build_ctf_tables() {
    const size_t nxy = (size_t)m_.grid.nx * m_.grid.ny;
    const size_t np = m_.obj_c10.size();
    d_ctf_.alloc(np * nxy);
    // the output propagation's band-width limit rides on the transfer function
    for (size_t j = 0; j < np; j++) {
        LensF L = m_.obj_lens;
        if (m_.ctf_mode == 2) {
            // PCTF_LI_WPO_TEM (src/microscope_effects.cuh:124-151): temporal only drops the
            // source spread, spatial only the defocus spread
            const float si = (m_.temporal_spatial_incoh == 2) ? 0.0f : L.si_sigma;
            const float ti = (m_.temporal_spatial_incoh == 3) ? 0.0f : L.ti_sigma;
            PctfArgs p{};
            p.g2_min = L.g2_min;
            p.g2_max = L.g2_max;
            p.c_c_10 = L.c_c_10;
            p.c_c_30 = L.c_c_30;
            p.c_10 = L.c_10;
            p.c_30 = L.c_30;
            p.lambda = L.lambda;
            p.lambda2 = (float)std::pow((double)L.lambda, 2);
            p.ti_iehwgd = (float)(1.414213562373095048802 * (double)ti);
            p.si_theta_c = std::asin((float)(1.414213562373095048802 * (double)si) * L.lambda);
            launch_pctf_table(p, gdev_, d_ctf_.p + j * nxy, stream_);
        } else {
            L.set_defocus(m_.obj_c10[j]);
            ProbeDev pr{};
            pr.c_c_10 = L.c_c_10;
            pr.nz_c10 = !is_zero_f(L.c_10);
            pr.c_c_30 = L.c_c_30;
            pr.nz_c30 = !is_zero_f(L.c_30);
            pr.c_c_50 = L.c_c_50;
            pr.nz_c50 = !is_zero_f(L.c_50);
            pr.g2_min = L.g2_min;
            pr.g2_max = L.g2_max;
            pr.norm = 1.0f;
            pr.phi_required = L.is_phi_required();
            pr.m = L.m;
            pr.c_c_12 = L.c_c_12; pr.phi_12 = L.phi_12;
            pr.c_c_21 = L.c_c_21; pr.phi_21 = L.phi_21;
            pr.c_c_23 = L.c_c_23; pr.phi_23 = L.phi_23;
            pr.c_c_32 = L.c_c_32; pr.phi_32 = L.phi_32;
            pr.c_c_34 = L.c_c_34; pr.phi_34 = L.phi_34;
            pr.c_c_41 = L.c_c_41; pr.phi_41 = L.phi_41;
            pr.c_c_43 = L.c_c_43; pr.phi_43 = L.phi_43;
            pr.c_c_45 = L.c_c_45; pr.phi_45 = L.phi_45;
            pr.c_c_52 = L.c_c_52; pr.phi_52 = L.phi_52;
            pr.c_c_54 = L.c_c_54; pr.phi_54 = L.phi_54;
            pr.c_c_56 = L.c_c_56; pr.phi_56 = L.phi_56;
            launch_ctf_table(pr, gdev_, d_ctf_.p + j * nxy, stream_);
        }
        if (d_bwl_.p) launch_mul_tables(d_ctf_.p + j * nxy, d_bwl_.p, nxy, stream_);
    }
}

// Fresnel propagator factors for distance dz, separable in x and y:
// P(ix, iy) = exp(i*w*(gx^2 + gy^2))/N, w = -pi*lambda*dz (propagate, src/cgpu_fcns.cuh:1837-1845;
// get_propagator_factor, src/input_multislice.cuh:909-912). Phases in double, stored as float.
void prop_tables(const Model& m_, float dz, float2* px, float2* py, bool output, int irot) {
    const int nx = m_.grid.nx, ny = m_.grid.ny;
    const double w = (double)m_.propagator_factor(dz);
    // Between passes the wave is kept as F_y(psi)/ny (the unnormalised row transforms of one step
    // multiply by ny, the column transforms by nx). Inside the loop P carries the reference's 1/N;
    // the output tables (back-propagation to the zero-defocus plane) carry 1/nx so that the
    // materialised wave is psi (or FFT2(psi)*P) itself.
    const double m = output ? 1.0 / (double)nx : (double)(1.0f / (float)(nx * ny));
    const double gx0 = m_.gx_0(irot), gy0 = m_.gy_0(irot);
    for (int ix = 0; ix < nx; ix++) {
        double gx = (double)((float)((ix < m_.grid.nxh) ? ix : ix - nx) * m_.grid.dgx) - gx0;
        double th = w * gx * gx;
        px[ix] = make_float2((float)(m * std::cos(th)), (float)(m * std::sin(th)));
    }
    for (int iy = 0; iy < ny; iy++) {
        double gy = (double)((float)((iy < m_.grid.nyh) ? iy : iy - ny) * m_.grid.dgy) - gy0;
        double th = w * gy * gy;
        py[iy] = make_float2((float)std::cos(th), (float)std::sin(th));
    }
}

void Engine::prop_tables(float dz, float2* px, float2* py, bool output, int irot) const {
    mtb::prop_tables(m_, dz, px, py, output, irot);
}

// gxu/gyu: the beam-tilt offset of exp_i_chi (src/cgpu_fcns.cuh:1950-1980). The simulations build
// their probes with gxu = gyu = 0 (Wave_Function::set_incident_wave, src/wave_function.cuh:300-307);
// only the incident-wave operator passes gx_0/gy_0 (Incident_Wave::operator(), src/incident_wave.cuh:117-121).
ProbeDev Engine::probe_params(float c_c_10, int nz_c10, bool tilt_offset) const {
    const LensF& L = m_.cond_lens;
    ProbeDev p{};
    p.c_c_10 = c_c_10;
    p.nz_c10 = nz_c10;
    p.c_c_30 = L.c_c_30;
    p.nz_c30 = !is_zero_f(L.c_30);
    p.c_c_50 = L.c_c_50;
    p.nz_c50 = !is_zero_f(L.c_50);
    p.g2_min = L.g2_min;
    p.g2_max = L.g2_max;
    p.gxu = tilt_offset ? m_.gx_0() : 0.0f;
    p.gyu = tilt_offset ? m_.gy_0() : 0.0f;
    p.norm = probe_norm_;
    p.phi_required = L.is_phi_required();
    p.m = L.m;
    p.c_c_12 = L.c_c_12; p.phi_12 = L.phi_12;
    p.c_c_21 = L.c_c_21; p.phi_21 = L.phi_21;
    p.c_c_23 = L.c_c_23; p.phi_23 = L.phi_23;
    p.c_c_32 = L.c_c_32; p.phi_32 = L.phi_32;
    p.c_c_34 = L.c_c_34; p.phi_34 = L.phi_34;
    p.c_c_41 = L.c_c_41; p.phi_41 = L.phi_41;
    p.c_c_43 = L.c_c_43; p.phi_43 = L.phi_43;
    p.c_c_45 = L.c_c_45; p.phi_45 = L.phi_45;
    p.c_c_52 = L.c_c_52; p.phi_52 = L.phi_52;
    p.c_c_54 = L.c_c_54; p.phi_54 = L.phi_54;
    p.c_c_56 = L.c_c_56; p.phi_56 = L.phi_56;
    return p;
}

// Host part of one configuration: Spec::move_atoms, slicing, tables; uploads on the stream.
void Engine::prepare_conf(ConfData& cd, int iconf) {
    ConfStage st;
    prepare_conf_host(cd, iconf, st);
    prepare_conf_device(cd, st);
}

// Host part of a configuration's set-up: phonon displacement (host generator), slicing, propagator
// tables and probe defocus into cd's host fields and the staging vectors of st. Runs while the
// GPU works on earlier configurations; touches no device buffer of cd.
void Engine::prepare_conf_host(ConfData& cd, int iconf, ConfStage& st) {
    // pn_rng 1: the undisplaced atoms and their slicing once, the displacements on the device
    const bool device_rng = m_.pn_rng == 1 && m_.is_frozen_phonon();
    if (!device_rng)
        spec_->move_atoms(iconf);
    else if (!d_atoms_u_.p)
        spec_->still_atoms();
    const auto& A = spec_->atoms();
    const auto& S = spec_->slices();
    const int nx = m_.grid.nx, ny = m_.grid.ny;
    cd.iconf = iconf;
    cd.n_slice = (int)S.size();
    std::vector<float4>& at = st.at;
    at.clear();
    st.n_atoms = A.size();
    if (!device_rng || !d_atoms_u_.p) {
        at.resize(A.size());
        for (size_t i = 0; i < A.size(); i++) {
            int t = atom_type(A.Z[i] % 1000, A.charge[i]);
            float tf;
            std::memcpy(&tf, &t, sizeof(float));
            at[i] = make_float4(A.x[i], A.y[i], A.occ[i], tf);
        }
    }
    if (device_rng && !d_atoms_u_.p) {
        d_atoms_u_.upload(at.data(), at.size(), stream_);
        d_sigma_.upload(A.sigma.data(), A.size(), stream_);
    }
    std::vector<int2>& rg = st.rg;
    rg.resize(S.size());
    cd.slice_ithk.resize(S.size());
    cd.last_slice = -1;
    for (size_t k = 0; k < S.size(); k++) {
        rg[k] = make_int2(S[k].iatom_0, S[k].iatom_e);
        cd.slice_ithk[k] = S[k].ithk;
        if (S[k].ithk >= 0) cd.last_slice = (int)k;
    }
    if (cd.last_slice < 0) fail(MT_ERR_INTERNAL, "no slice carries a thickness");
    const auto& TH = spec_->thicks();
    cd.thick_z_back_prop.resize(TH.size());
    for (size_t t = 0; t < TH.size(); t++) cd.thick_z_back_prop[t] = TH[t].z_back_prop;
    const size_t pl = (size_t)nx + ny;
    const size_t rb = (S.size() + TH.size()) * pl;  // one block per beam rotation
    // the tables depend on the slice thicknesses and back-propagation distances only, which the
    // phonon displacements (x and y) do not change: computed once and reused while they match
    std::vector<float> key;
    key.reserve(S.size() + TH.size());
    for (size_t k = 0; k < S.size(); k++) key.push_back(spec_->dz((int)k));
    for (size_t t = 0; t < TH.size(); t++) key.push_back(TH[t].z_back_prop);
    if (key != prop_key_ || prop_cache_.size() != rb * m_.nrot) {
        prop_cache_.assign(rb * m_.nrot, make_float2(0.0f, 0.0f));
        for (int r = 0; r < m_.nrot; r++) {
            float2* q = prop_cache_.data() + r * rb;
            for (size_t k = 0; k < S.size(); k++) prop_tables(spec_->dz((int)k), q + k * pl, q + k * pl + nx, false, r);
            for (size_t t = 0; t < TH.size(); t++)
                prop_tables(TH[t].z_back_prop, q + (S.size() + t) * pl, q + (S.size() + t) * pl + nx, true, r);
        }
        prop_key_ = std::move(key);
    }
    st.prop = prop_cache_;
    // incident-wave defocus relative to the first slice (Incident_Wave::operator(),
    // src/incident_wave.cuh:54-72): f_s = c_10 - (zero_defocus_plane - z_m(0)), with c_10 moved
    // by each defocus-spread point (cond_lens.set_defocus(c_10_0 + qt.x), src/tem_simulation.cuh:155-157)
    const float z_init = (float)(0.5 * (S[0].z_0 + S[0].z_e));
    cd.probe_c_c_10.clear();
    cd.probe_nz_c10.clear();
    for (double dx : m_.ti_x) {
        const float c_10 = (float)((double)m_.cond_lens.c_10 + dx);
        const float f_s = c_10 - (m_.cond_lens.zero_defocus_plane - z_init);
        LensF L = m_.cond_lens;
        L.set_defocus(f_s);
        cd.probe_c_c_10.push_back(L.c_c_10);
        cd.probe_nz_c10.push_back(!is_zero_f(f_s));
    }
}

// Device part: the configuration's atoms (uploaded, or displaced on the device), slice ranges and
// propagator tables into cd's buffers. The uploads wait for the stream's earlier work.
void Engine::prepare_conf_device(ConfData& cd, ConfStage& st) {
    const bool device_rng = m_.pn_rng == 1 && m_.is_frozen_phonon();
    if (device_rng) {
        cd.atoms.alloc(st.n_atoms);
        launch_phonon_displace(d_atoms_u_.p, d_sigma_.p, (int)st.n_atoms, (uint32_t)m_.pn_seed, cd.iconf, m_.pn_x,
                               m_.pn_y, cd.atoms.p, stream_);
    } else {
        cd.atoms.upload(st.at.data(), st.at.size(), stream_);
    }
    cd.ranges.upload(st.rg.data(), st.rg.size(), stream_);
    cd.prop.upload(st.prop.data(), st.prop.size(), stream_);
    synchronize();  // the staging vectors may be reused
}

ConfData* Engine::find_conf(int iconf) {
    for (auto& c : confs_)
        if (c.iconf == iconf) return &c;
    return nullptr;
}

void Engine::prepare_confs(int c0, int c1) {
    for (int c = c0; c <= c1; c++) {
        if (find_conf(c)) continue;
        confs_.emplace_back();
        prepare_conf(confs_.back(), c);
    }
}

void Engine::check_cancel() {
    if (cancel_ && !capturing_) {
        synchronize();
        fail(MT_ERR_CANCELLED, "run cancelled");
    }
}

// Prepared configurations [c0, c1]: with graphs (and no per-launch timing) the whole range is one
// CUDA graph, captured before the run's start event (so the capture is not in the device time)
// and replayed while the range and every configuration's launch signature match; else direct
// launches.
void Engine::run_prepared(int c0, int c1) {
    if (c0 < m_.fp_iconf_0 || c1 > m_.pn_nconf || c0 > c1) fail(MT_ERR_INVALID_ARG, "configuration range out of bounds");
    for (int c = c0; c <= c1; c++)
        if (!find_conf(c)) fail(MT_ERR_INVALID_ARG, "configuration not prepared");
    long long l0 = launches_issued();
    tl_used_ = 0;
    if (!run_a_) {
        MTB_CUDA(cudaEventCreate(&run_a_));
        MTB_CUDA(cudaEventCreate(&run_b_));
    }
    const bool graph = graphs_ && !timing_;
    if (graph) {
        ConfData* cd0 = find_conf(c0);
        if (tune_) tune(*cd0);
        std::vector<char> sig;
        const int range[2] = {c0, c1};
        sig.insert(sig.end(), (const char*)range, (const char*)range + sizeof(range));
        for (int c = c0; c <= c1; c++) {
            std::vector<char> s = graph_signature(*find_conf(c));
            sig.insert(sig.end(), s.begin(), s.end());
        }
        if (!range_graph_.exec || sig != range_graph_.sig) {
            if (range_graph_.exec) {
                MTB_CUDA(cudaGraphExecDestroy(range_graph_.exec));
                range_graph_.exec = nullptr;
            }
            const int it0 = iter_;
            const long long la = launches_issued();
            cudaGraph_t g = nullptr;
            MTB_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
            capturing_ = true;
            try {
                run_prepared_range(c0, c1);
            } catch (...) {
                capturing_ = false;
                cudaStreamEndCapture(stream_, &g);
                if (g) cudaGraphDestroy(g);
                iter_ = it0;
                throw;
            }
            capturing_ = false;
            MTB_CUDA(cudaStreamEndCapture(stream_, &g));
            cudaError_t e = cudaGraphInstantiate(&range_graph_.exec, g, 0);
            cudaGraphDestroy(g);
            MTB_CUDA(e);
            range_graph_.sig = std::move(sig);
            range_graph_.iters = iter_ - it0;
            range_graph_.launches = launches_issued() - la;
            iter_ = it0;
            add_launches(-range_graph_.launches);
        }
    }
    l0 = launches_issued();
    MTB_CUDA(cudaEventRecord(run_a_, stream_));
    if (graph) {
        MTB_CUDA(cudaGraphLaunch(range_graph_.exec, stream_));
        iter_ += range_graph_.iters;
        add_launches(range_graph_.launches);
    } else {
        run_prepared_range(c0, c1);
    }
    MTB_CUDA(cudaEventRecord(run_b_, stream_));
    launches_ = launches_issued() - l0;
    synchronize();
}

// ---- device timing ----
void Engine::tl_begin(int kind) {
    if (!timing_) return;
    if (tl_used_ == tl_.size()) {
        TimedLaunch t{};
        MTB_CUDA(cudaEventCreate(&t.a));
        MTB_CUDA(cudaEventCreate(&t.b));
        tl_.push_back(t);
    }
    tl_[tl_used_].kind = kind;
    MTB_CUDA(cudaEventRecord(tl_[tl_used_].a, stream_));
}

void Engine::tl_end() {
    if (!timing_) return;
    MTB_CUDA(cudaEventRecord(tl_[tl_used_].b, stream_));
    tl_used_++;
}

// Passes get the engine's error flag, which selects the bulk-copy-fed kernels where they fit.
void Engine::rows(RowMode mode, const RowArgs& a) {
    RowArgs b = a;
    b.err = (pipe_ & 1) ? d_err_.p : nullptr;
    b.wait_ns = wait_ns_;
    b.shape = shape_ & 3;
    tl_begin(0);
    launch_rows(m_.grid.ny, mode, b, 0, stream_);
    tl_end();
}

void Engine::cols(int flags, const ColArgs& a) {
    ColArgs b = a;
    b.err = (pipe_ & 2) ? d_err_.p : nullptr;
    b.wait_ns = wait_ns_;
    b.shape = (shape_ >> 2) & 3;
    tl_begin(1);
    launch_cols(m_.grid.nx, flags, b, 0, stream_);
    tl_end();
}

void Engine::timing(double* total_ms, double* rows_ms, long long* n_rows, double* cols_ms, long long* n_cols) {
    synchronize();
    float ms = 0;
    *total_ms = 0;
    if (run_a_) {
        MTB_CUDA(cudaEventElapsedTime(&ms, run_a_, run_b_));
        *total_ms = ms;
    }
    *rows_ms = *cols_ms = 0;
    *n_rows = *n_cols = 0;
    for (size_t i = 0; i < tl_used_; i++) {
        MTB_CUDA(cudaEventElapsedTime(&ms, tl_[i].a, tl_[i].b));
        if (tl_[i].kind == 0) {
            *rows_ms += ms;
            (*n_rows)++;
        } else {
            *cols_ms += ms;
            (*n_cols)++;
        }
    }
}

void Engine::run_confs(int c0, int c1) {
    if (c0 < m_.fp_iconf_0 || c1 > m_.pn_nconf || c0 > c1) fail(MT_ERR_INVALID_ARG, "configuration range out of bounds");
    long long l0 = launches_issued();
    // every configuration as its slot's CUDA graph: captured twice (once per slot) and replayed
    // while the launch sequence and its arguments match
    const int B = ew_batch_;
    if (graphs_ && !timing_) {
        // batch k of B configurations is prepared in slot group k % 2 (prepare_conf waits for the
        // stream, so the group's previous user, batch k - 2, has finished) and runs as that group's
        // graph
        // the host part of batch k + 1 runs while batch k's graph executes
        std::vector<ConfData*> cds(B);
        std::vector<ConfStage> st(B);
        auto stage = [&](int c, int k) {
            const int nb = std::min(B, c1 - c + 1);
            for (int b = 0; b < nb; b++) prepare_conf_host(slot_[(size_t)(k & 1) * B + b], c + b, st[b]);
        };
        stage(c0, 0);
        for (int c = c0, k = 0; c <= c1; c += B, k++) {
            const int nb = std::min(B, c1 - c + 1);
            for (int b = 0; b < nb; b++) {
                cds[b] = &slot_[(size_t)(k & 1) * B + b];
                prepare_conf_device(*cds[b], st[b]);
            }
            run_conf_graph(cds.data(), nb, graph_[k & 1]);
            if (c + B <= c1) stage(c + B, k + 1);
        }
        launches_ = launches_issued() - l0;
        synchronize();
        return;
    }
    // configuration c is prepared on the host while c-1 runs; c-1's buffers go back to the pool once
    // its last launch has completed
    if (!conf_done_) MTB_CUDA(cudaEventCreateWithFlags(&conf_done_, cudaEventDisableTiming));
    std::vector<ConfData> prev;
    for (int c = c0; c <= c1; c += B) {
        const int nb = std::min(B, c1 - c + 1);
        std::vector<ConfData> cur(nb);
        std::vector<ConfData*> cds(nb);
        for (int b = 0; b < nb; b++) {
            prepare_conf(cur[b], c + b);
            cds[b] = &cur[b];
        }
        run_conf_batch(cds.data(), nb);
        if (!prev.empty()) {
            MTB_CUDA(cudaEventSynchronize(conf_done_));
            for (auto& cd : prev) cd.release_idle();
        }
        MTB_CUDA(cudaEventRecord(conf_done_, stream_));
        prev = std::move(cur);
    }
    launches_ = launches_issued() - l0;
    synchronize();
    for (auto& cd : prev) cd.release_idle();
}

// Configurations c0..c1 (prepared) run in batches of ew_batch_.
static void for_batches(int c0, int c1, int B, const std::function<void(int, int)>& f) {
    for (int c = c0; c <= c1; c += B) f(c, std::min(B, c1 - c + 1));
}

void Engine::run_prepared_range(int c0, int c1) {
    for_batches(c0, c1, ew_batch_, [&](int c, int nb) {
        std::vector<ConfData*> cds(nb);
        for (int b = 0; b < nb; b++) cds[b] = find_conf(c + b);
        run_conf_batch(cds.data(), nb);
    });
}

void Engine::prepare_run() {
    const int c0 = m_.fp_iconf_0, c1 = m_.pn_nconf;
    prepare_confs(c0, c1);
    ConfData* cd = find_conf(c0);
    if (tune_ && cd) tune(*cd);
    synchronize();
}

void Engine::record_run() {
    zero_accumulators();
    iter_ = 0;
    cancel_ = false;
    capturing_ = true;  // no host synchronisation (check_cancel) while the work is recorded
    try {
        for_batches(m_.fp_iconf_0, m_.pn_nconf, ew_batch_, [&](int c, int nb) {
            std::vector<ConfData*> cds(nb);
            for (int b = 0; b < nb; b++) {
                cds[b] = find_conf(c + b);
                if (!cds[b]) fail(MT_ERR_INTERNAL, "configuration not prepared before recording");
            }
            run_conf_batch(cds.data(), nb);
        });
    } catch (...) {
        capturing_ = false;
        throw;
    }
    capturing_ = false;
}

// Everything a captured run_conf bakes into its launches besides the engine's own buffers.
std::vector<char> Engine::graph_signature(const ConfData& cd) const {
    std::vector<char> sig;
    auto put = [&](const void* p, size_t n) { sig.insert(sig.end(), (const char*)p, (const char*)p + n); };
    const void* ptrs[3] = {cd.atoms.p, cd.ranges.p, cd.prop.p};
    put(ptrs, sizeof(ptrs));
    const int ints[5] = {cd.n_slice, cd.last_slice, pipe_, shape_, run_batch_};
    put(ints, sizeof(ints));
    put(&wait_ns_, sizeof(wait_ns_));
    put(cd.probe_nz_c10.data(), cd.probe_nz_c10.size() * sizeof(int));
    put(cd.probe_c_c_10.data(), cd.probe_c_c_10.size() * sizeof(float));
    put(cd.slice_ithk.data(), cd.slice_ithk.size() * sizeof(int));
    // the back-propagation distances live in the device tables; only whether each is zero
    // changes the launches (run_ew)
    for (float z : cd.thick_z_back_prop) sig.push_back(z != 0.0f);
    return sig;
}

// run_conf as a CUDA graph: captured once, then replayed for every configuration with the same
// launch sequence and arguments (same slot buffers, slice count, thickness map and probe defocus).
// The line-pass autotuner runs before the capture (it times launches and waits for them).
void Engine::run_conf_graph(ConfData* const* cds, int nb, ConfGraph& g) {
    if (tune_) tune(*cds[0]);
    std::vector<char> sig;
    sig.insert(sig.end(), (const char*)&nb, (const char*)&nb + sizeof(nb));
    for (int b = 0; b < nb; b++) {
        std::vector<char> s = graph_signature(*cds[b]);
        sig.insert(sig.end(), s.begin(), s.end());
    }
    if (!g.exec || sig != g.sig) {
        if (g.exec) {
            MTB_CUDA(cudaGraphExecDestroy(g.exec));
            g.exec = nullptr;
        }
        const int it0 = iter_;
        const long long l0 = launches_issued();
        cudaGraph_t graph = nullptr;
        MTB_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        capturing_ = true;
        try {
            run_conf_batch(cds, nb);
        } catch (...) {
            capturing_ = false;
            cudaStreamEndCapture(stream_, &graph);
            if (graph) cudaGraphDestroy(graph);
            iter_ = it0;
            throw;
        }
        capturing_ = false;
        MTB_CUDA(cudaStreamEndCapture(stream_, &graph));
        cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        MTB_CUDA(e);
        g.sig = std::move(sig);
        g.iters = iter_ - it0;
        g.launches = launches_issued() - l0;
        iter_ = it0;
        add_launches(-g.launches);
    }
    MTB_CUDA(cudaGraphLaunch(g.exec, stream_));
    iter_ += g.iters;
    add_launches(g.launches);
    check_cancel();
}

void Engine::run_conf(ConfData& cd) {
    ConfData* p = &cd;
    run_conf_batch(&p, 1);
}

void Engine::run_conf_batch(ConfData* const* cds, int nb) {
    if (nb < 1 || nb > ew_batch_ || (nb > 1 && m_.is_scanning())) fail(MT_ERR_INTERNAL, "bad configuration batch");
    const size_t tstride = (size_t)spec_->slices().size() * m_.grid.nx * m_.grid.ny;
    for (int b = 1; b < nb; b++)
        if (cds[b]->n_slice != cds[0]->n_slice || cds[b]->last_slice != cds[0]->last_slice ||
            cds[b]->slice_ithk != cds[0]->slice_ithk)
            fail(MT_ERR_INTERNAL, "configurations of a batch must share their slicing");
    for (int b = 0; b < nb; b++) {
        const ConfData& cd = *cds[b];
        float2* trans = d_trans_.p + b * tstride;
        // transmission functions of the slices up to the last output thickness
        SplatArgs sa{};
        sa.g = gdev_;
        sa.atoms = cd.atoms.p;
        sa.slice_range = cd.ranges.p;
        sa.tab = d_tab_.p;
        sa.R_max = d_Rmax_.p;
        sa.n_types = (int)Z_of_type_.size();
        sa.nR = m_.nR;
        sa.w = m_.Vr_factor();
        sa.wpo = (m_.interaction_model == 3);
        sa.trans = trans;
        sa.V = nullptr;
        launch_splat(sa, 0, cd.last_slice + 1, stream_);
        if (d_bwl_.p) band_limit_trans(cd, trans);
    }
    if (m_.is_scanning()) run_stem(*cds[0]); else run_ew(cds, nb);
}

// Autotuner of the line passes. For each (nx, ny, allocated probes per launch) the process times,
// once, on this engine's probe buffer, transmission function and propagator (one warm-up and three
// timed launches each): the row pass and the column pass of the slice step in each variant (per-
// thread loads; bulk-copy fed; bulk-copy fed in the alternative pipeline shapes RowPipeShape<N, 1|2>
// and ColPipeShape<N, 1|2>: narrower groups, and early issue with full exchange buffers in as many
// groups as shared memory holds), keeping the fastest of each; then, for STEM batches of at least 16
// probes, the chosen step at the full and at half the batch, keeping the batch with the lower
// time per probe. Every variant computes the same transforms with the same rounding, so the
// choice changes only the speed (the FP64 detector partials of other tile widths are added in
// another order).
Engine::Tuning Engine::tune_passes(int nprobe, ConfData& cd) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, int>, Tuning> chosen;
    const int nx = m_.grid.nx, ny = m_.grid.ny;
    const auto key = std::make_tuple(nx, ny, nprobe);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = chosen.find(key);
        if (it != chosen.end()) return it->second;
    }
    const size_t nxy = (size_t)nx * ny;
    MTB_CUDA(cudaMemsetAsync(d_psi_.p, 0, sizeof(float2) * nxy * nprobe, stream_));
    cudaEvent_t a, b;
    MTB_CUDA(cudaEventCreate(&a));
    MTB_CUDA(cudaEventCreate(&b));
    auto time_of = [&](auto launch) {
        launch();
        MTB_CUDA(cudaEventRecord(a, stream_));
        for (int i = 0; i < 3; i++) launch();
        MTB_CUDA(cudaEventRecord(b, stream_));
        MTB_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        MTB_CUDA(cudaEventElapsedTime(&ms, a, b));
        return ms;
    };
    RowArgs ra{};
    ra.in = d_psi_.p;
    ra.out = d_psi_.p;
    ra.trans = d_trans_.p;
    ra.nx = nx;
    ra.scale = 1.0f;
    ra.wait_ns = wait_ns_;
    ColArgs ca{};
    ca.in = d_psi_.p;
    ca.out = d_psi_.p;
    ca.ny = ny;
    ca.g = gdev_;
    ca.Px = cd.prop.p;
    ca.Py = cd.prop.p + nx;
    ca.det_w = col_det_width(nx);
    ca.wait_ns = wait_ns_;
    const int step = COL_LOAD | COL_PROP | COL_INVERSE | COL_STORE;
    // variant v: 0 per-thread loads, 1 bulk-copy fed, 2 and 3 bulk-copy fed in the alternative
    // pipeline shapes 1 and 2 (a shape that does not fit this length runs the default one)
    auto rows_t = [&](int v, int nb) {
        ra.nprobe = nb;
        ra.err = v ? d_err_.p : nullptr;
        ra.shape = v > 1 ? v - 1 : 0;
        return time_of([&] { launch_rows(ny, ROW_STEP, ra, 0, stream_); });
    };
    auto cols_t = [&](int v, int nb) {
        ca.nprobe = nb;
        ca.err = v ? d_err_.p : nullptr;
        ca.shape = v > 1 ? v - 1 : 0;
        return time_of([&] { launch_cols(nx, step, ca, 0, stream_); });
    };
    constexpr int NV = 4;
    float tr[NV], tc[NV];
    for (int v = 0; v < NV; v++) {
        tr[v] = rows_t(v, nprobe);
        tc[v] = cols_t(v, nprobe);
    }
    int vr = 0, vc = 0;
    for (int v = 1; v < NV; v++) {
        if (tr[v] < tr[vr]) vr = v;
        if (tc[v] < tc[vc]) vc = v;
    }
    Tuning t{(vr ? 1 : 0) | (vc ? 2 : 0), (vr > 1 ? vr - 1 : 0) | ((vc > 1 ? vc - 1 : 0) << 2), nprobe};
    if (m_.is_scanning() && nprobe >= 16 && (nprobe / 2) % 8 == 0) {
        const float full = tr[vr] + tc[vc];
        const float half = rows_t(vr, nprobe / 2) + cols_t(vc, nprobe / 2);
        if (2.0f * half < 0.99f * full) t.nprobe = nprobe / 2;
    }
    MTB_CUDA(cudaEventDestroy(a));
    MTB_CUDA(cudaEventDestroy(b));
    synchronize();
    std::lock_guard<std::mutex> lk(mu);
    return chosen.emplace(key, t).first->second;
}

void Engine::tune(ConfData& cd) {
    const int nprobe = m_.is_scanning() ? std::min(batch_, m_.n_scan()) : ew_batch_;
    const Tuning t = tune_passes(nprobe, cd);
    pipe_ = t.pipe;
    shape_ = t.shape;
    run_batch_ = m_.is_scanning() ? std::max(1, std::min(t.nprobe, batch_)) : batch_;
}

void Engine::tuning(int* rows_variant, int* cols_variant, int* probes_per_launch) const {
    *rows_variant = (pipe_ & 1) ? 1 + (shape_ & 3) : 0;
    *cols_variant = (pipe_ & 2) ? 1 + ((shape_ >> 2) & 3) : 0;
    *probes_per_launch = run_batch_;
}

// User-defined incident wave (Incident_Wave, src/incident_wave.cuh:48-52 and 92-110): the wave
// iw_psi, fft2-shifted, moved by (iw_x[0] - lx/2, iw_y[0] - ly/2) through the Fourier phase
// exp(i (Rx gx + Ry gy)), Rx = exp_factor_Rx(iw_x[0]) (applied here as separable x and y factors
// with the loop's 1/N), in the layout the first row step reads. Built once per engine: the wave is
// the same for every configuration.
void Engine::build_user_wave() {
    const GridF& g = m_.grid;
    const int nx = g.nx, ny = g.ny;
    const size_t nxy = (size_t)nx * ny;
    std::vector<float2> h(nxy);
    for (int ix = 0; ix < nx; ix++)
        for (int iy = 0; iy < ny; iy++) {
            const size_t src = (size_t)ix * ny + iy;
            const size_t dst = (size_t)((ix + g.nxh) % nx) * ny + (iy + g.nyh) % ny;
            h[dst] = make_float2(m_.iw_psi[2 * src], m_.iw_psi[2 * src + 1]);
        }
    const float Rx = g.exp_factor_Rx(m_.iw_x[0]), Ry = g.exp_factor_Ry(m_.iw_y[0]);
    const double mnorm = (double)(1.0f / (float)(nx * ny));
    std::vector<float2> tab((size_t)nx + ny);
    for (int ix = 0; ix < nx; ix++) {
        const double th = (double)(Rx * ((float)((ix < g.nxh) ? ix : ix - nx) * g.dgx));
        tab[ix] = make_float2((float)(mnorm * std::cos(th)), (float)(mnorm * std::sin(th)));
    }
    for (int iy = 0; iy < ny; iy++) {
        const double th = (double)(Ry * ((float)((iy < g.nyh) ? iy : iy - ny) * g.dgy));
        tab[nx + iy] = make_float2((float)std::cos(th), (float)std::sin(th));
    }
    std::vector<float2> ones(nxy, make_float2(1.0f, 0.0f));
    DevBuf<float2> d_one, d_tab;
    d_user_wave_.upload(h.data(), nxy, stream_);
    d_one.upload(ones.data(), nxy, stream_);
    d_tab.upload(tab.data(), tab.size(), stream_);
    RowArgs ra{};
    ra.in = d_user_wave_.p;
    ra.out = d_user_wave_.p;
    ra.trans = d_one.p;
    ra.nx = nx;
    ra.nprobe = 1;
    ra.scale = 1.0f;
    rows(ROW_FIRST_REAL, ra);
    ColArgs ca{};
    ca.in = d_user_wave_.p;
    ca.out = d_user_wave_.p;
    ca.ny = ny;
    ca.nprobe = 1;
    ca.g = gdev_;
    ca.Px = d_tab.p;
    ca.Py = d_tab.p + nx;
    ca.det_w = col_det_width(nx);
    cols(COL_LOAD | COL_PROP | COL_INVERSE | COL_STORE, ca);
    synchronize();
}

// Probe normalisation: the reference scales each probe by sqrt(1/sum|psi_hat|^2)
// (src/gpu_fcns.cuh:1612-1624); |exp(i chi)| = 1 inside the aperture, so the sum is the
// aperture's pixel count (aperture test in the kernel's float arithmetic; no tilt offset in the
// simulations' probes).
float Engine::aperture_norm() const {
    const LensF& L = m_.cond_lens;
    const int nx = m_.grid.nx, ny = m_.grid.ny;
    double count = 0;
    for (int ix = 0; ix < nx; ix++) {
        float gx = (float)((ix < m_.grid.nxh) ? ix : ix - nx) * m_.grid.dgx;
        for (int iy = 0; iy < ny; iy++) {
            float gy = (float)((iy < m_.grid.nyh) ? iy : iy - ny) * m_.grid.dgy;
            float g2 = gx * gx + gy * gy;
            if ((L.g2_min <= g2) && (g2 < L.g2_max)) count += 1.0;
        }
    }
    if (count <= 0) fail(MT_ERR_INVALID_ARG, "condenser aperture contains no Fourier pixel");
    return (float)std::sqrt(1.0 / (double)(float)count);
}

ColArgs Engine::det_args() const {
    ColArgs ca{};
    ca.ny = m_.grid.ny;
    ca.g = gdev_;
    ca.n_det = (int)m_.det_g_inner.size();
    for (int d = 0; d < ca.n_det; d++) {
        // sum_square_over_Det bounds: g2 = pow(g, 2) stored as float (src/cpu_fcns.hpp:1168-1169)
        ca.det_g2_min[d] = (float)std::pow((double)m_.det_g_inner[d], 2);
        ca.det_g2_max[d] = (float)std::pow((double)m_.det_g_outer[d], 2);
    }
    ca.gx_0 = 0;
    ca.gy_0 = 0;
    ca.det_mat = d_detmat_.p;
    return ca;
}


void Engine::run_stem(ConfData& cd) {
    const int nx = m_.grid.nx, ny = m_.grid.ny;
    const size_t nxy = (size_t)nx * ny;
    const int n_det = (int)m_.det_g_inner.size();
    const int n_scan = m_.n_scan();
    const int n_thk = (int)m_.thick.size();
    const int tiles = col_tiles(nx, ny);
    const size_t pl = (size_t)nx + ny;
    ColArgs ca = det_args();
    ca.det_w = col_det_width(nx);
    ca.coh_w = (float)m_.phonon_weight();
    ca.P2 = d_bwl_.p;  // band-width limit of every propagation (NULL without bwl)
    const bool tilt = d_ramp_.p != nullptr;
    const bool istem = m_.is_ISTEM();
    // the detectors get their own output pass when the output needs more than the last slice's
    // column pass: a phase ramp (tilt) or a second band-width limit (bwl)
    const bool sep_out = tilt || d_bwl_.p != nullptr;
    RowArgs ra{};
    ra.nx = nx;
    ra.scale = 1.0f;

    if (tune_) tune(cd);
    // defocus-spread points (one without full integration), each over every probe, weighted
    // w_pr_0 * qt.w as a float (Multislice::STEM_ISTEM, src/tem_simulation.cuh:146-176)
    for (size_t it = 0; it < m_.ti_x.size(); it++) {
    ca.probe = probe_params(cd.probe_c_c_10[it], cd.probe_nz_c10[it], false);
    const double w = (double)(float)((double)m_.phonon_weight() * m_.ti_w[it]);
    for (int p0 = 0; p0 < n_scan; p0 += run_batch_) {
        const int nb = std::min(run_batch_, n_scan - p0);
        ca.nprobe = nb;
        ra.nprobe = nb;
        // incident probes, generated in Fourier space and brought to the hybrid layout
        ca.in = nullptr;
        ca.out = d_psi_.p;
        ca.beam = d_beam_.p + p0;
        ca.Px = nullptr;
        ca.Py = nullptr;
        cols(COL_INVERSE | COL_STORE, ca);
        for (int k = 0; k <= cd.last_slice; k++) {
            ra.in = d_psi_.p;
            ra.out = d_psi_.p;
            ra.trans = d_trans_.p + (size_t)k * nxy;
            rows(ROW_STEP, ra);
            const int ithk = cd.slice_ithk[k];
            int flags = COL_LOAD | COL_PROP;
            if (ithk >= 0 && !sep_out && !istem) flags |= COL_DETECT;
            if (k < cd.last_slice || sep_out || istem) flags |= COL_INVERSE | COL_STORE;
            ca.in = d_psi_.p;
            ca.out = d_psi_.p;
            ca.Px = cd.prop.p + (size_t)k * pl;
            ca.Py = ca.Px + nx;
            ca.det_partial = d_partial_.p + (size_t)(ithk >= 0 ? ithk : 0) * batch_ * tiles * n_det;
            ca.coh = (d_coh_.p && ithk >= 0) ? d_coh_.p + ((size_t)ithk * n_scan + p0) * nxy : nullptr;
            cols(flags, ca);
            if (istem && ithk >= 0) {
                // ISTEM: each probe's wave through the objective lens (get_psi, then
                // Microscope_Effects), |psi|^2 of the batch summed into the thickness's image
                // (set_m2psi_tot_psi_coh, src/wave_function.cuh:166-170)
                const float2* src = d_psi_.p;
                if (tilt) {
                    // the ramped batch goes where the next slices do not need it
                    RowArgs rr = ra;
                    rr.out = (k < cd.last_slice) ? d_tmp2_.p : d_psi_.p;
                    rr.trans = d_ramp_.p;
                    rows(ROW_STEP, rr);
                    src = rr.out;
                }
                for (size_t j = 0; j < m_.obj_c10.size(); j++) {
                    ColArgs cj = ca;
                    cj.in = src;
                    cj.out = d_tmp_.p;
                    cj.Px = cd.prop.p + (size_t)(cd.n_slice + ithk) * pl;
                    cj.Py = cj.Px + nx;
                    cj.P2 = d_ctf_.p + j * nxy;
                    cols(COL_LOAD | COL_PROP | COL_INVERSE | COL_STORE, cj);
                    RowArgs rb = ra;
                    rb.in = d_tmp_.p;
                    rb.out = d_tmp_.p;
                    rows(ROW_INVERSE, rb);
                    launch_ew_accumulate(d_tmp_.p, nx, ny, m_.out_ix_0, m_.out_ix_e, m_.out_iy_0, m_.out_iy_e,
                                         (double)(float)(w * m_.obj_w[j]), 0, nullptr,
                                         d_ew_m2_.p + (size_t)ithk * ((size_t)(m_.out_ix_e - m_.out_ix_0) *
                                                                      (m_.out_iy_e - m_.out_iy_0)),
                                         stream_, nb);
                }
                continue;
            }
            if (sep_out && ithk >= 0) {
                // get_psi: phase ramp (tilted beam), then the detectors on the transform after
                // the output propagation (its phase does not change |psi_hat|^2; its band-width
                // limit does)
                float2* src = d_psi_.p;
                if (tilt) {
                    RowArgs rr = ra;
                    rr.out = (k < cd.last_slice) ? d_tmp_.p : d_psi_.p;
                    rr.trans = d_ramp_.p;
                    rows(ROW_STEP, rr);
                    src = rr.out;
                }
                ColArgs cc = ca;
                cc.in = src;
                cc.out = src;
                cc.Px = cd.prop.p + (size_t)(cd.n_slice + ithk) * pl;
                cc.Py = cc.Px + nx;
                cols(COL_LOAD | COL_PROP | COL_DETECT, cc);
            }
        }
        for (int t = 0; t < n_thk && !istem; t++)
            launch_det_reduce(d_partial_.p + (size_t)t * batch_ * tiles * n_det, nb, tiles, n_det, d_scan_idx_.p + p0, w,
                              d_image_.p + (size_t)t * n_det * n_scan, n_scan, stream_);
        iter_ += nb;
        check_cancel();
    }
    }
}

// nb configurations of the batch advance together: their waves are the nb "probes" of every pass,
// each row pass multiplying wave b by its own transmission functions (trans_stride), and the
// outputs of each thickness are accumulated wave by wave in configuration order, as nb separate
// configurations would be.
void Engine::run_ew(ConfData* const* cds, int nb) {
    const ConfData& cd = *cds[0];
    const int nx = m_.grid.nx, ny = m_.grid.ny;
    const size_t nxy = (size_t)nx * ny;
    const size_t pl = (size_t)nx + ny;
    const int ox = m_.out_ix_e - m_.out_ix_0, oy = m_.out_iy_e - m_.out_iy_0;
    const size_t onxy = (size_t)ox * oy;
    const double w = (double)m_.phonon_weight();
    const bool sc = m_.is_EW_SC();

    RowArgs ra{};
    ra.nx = nx;
    ra.nprobe = nb;
    ra.scale = 1.0f;
    ra.trans_stride = nb > 1 ? (size_t)spec_->slices().size() * nxy : 0;
    ColArgs ca{};
    ca.ny = ny;
    ca.nprobe = nb;
    ca.g = gdev_;
    ca.n_det = 0;
    ca.P2 = d_bwl_.p;  // band-width limit of every propagation (NULL without bwl)
    if (tune_) tune(*cds[0]);
    const bool conv = m_.is_convergent_wave();
    const bool user = m_.is_user_wave();
    if (nb > 1 && (conv || user || m_.nrot != 1)) fail(MT_ERR_INTERNAL, "this incident wave runs one configuration at a time");
    const size_t rblock = (size_t)(cd.n_slice + (int)cd.thick_z_back_prop.size()) * pl;
    // beam rotations of PED / HCTEM (Multislice::PED_HCTEM, src/tem_simulation.cuh:274-300); one
    // pass otherwise
    // CBED/CBEI under full integration: every (source point, defocus point) pair is a slice loop of
    // its own, weighted by the product of the two quadrature weights (Multislice::CBED_CBEI,
    // src/tem_simulation.cuh:226-251); one pass with the configuration's weight otherwise
    const int n_si = (int)m_.si_x.size(), n_ti = (int)m_.ti_x.size();
    const bool full = conv && (n_si * n_ti > 1);
    const double w_pr = w;
    for (int r = 0; r < m_.nrot; r++) {
    for (int ip = 0; ip < (full ? n_si * n_ti : 1); ip++) {
    const int is = ip / n_ti, it = ip % n_ti;
    const double w = full ? (double)(float)(w_pr * m_.si_w[is] * m_.ti_w[it]) : w_pr;
    const float2* prop = cd.prop.p + (size_t)r * rblock;
    const float2* ramp = m_.ramp_needed(r) ? d_ramp_.p + (size_t)r * nxy : nullptr;
    if (conv) {
        // the beams' probes, generated in Fourier space and brought to the hybrid layout, summed
        const int nb = (int)m_.iw_x.size();
        ColArgs cp = ca;
        cp.nprobe = nb;
        cp.in = nullptr;
        cp.out = (nb > 1) ? d_beams_psi_.p : d_psi_.p;
        cp.beam = d_beam_.p + (size_t)is * nb;
        cp.probe = probe_params(cd.probe_c_c_10[it], cd.probe_nz_c10[it], false);
        cols(COL_INVERSE | COL_STORE, cp);
        if (nb > 1) launch_sum_waves(d_beams_psi_.p, nb, nxy, d_psi_.p, stream_);
    }
    for (int k = 0; k <= cd.last_slice; k++) {
        ra.in = (k == 0 && user) ? d_user_wave_.p : d_psi_.p;
        ra.out = d_psi_.p;
        ra.trans = d_trans_.p + (size_t)k * nxy;
        rows((k == 0 && !conv && !user) ? ROW_FIRST_ONE : ROW_STEP, ra);
        ca.in = d_psi_.p;
        ca.out = d_psi_.p;
        ca.Px = prop + (size_t)k * pl;
        ca.Py = ca.Px + nx;
        cols(COL_LOAD | COL_PROP | COL_INVERSE | COL_STORE, ca);
        const int ithk = cd.slice_ithk[k];
        if (ithk < 0) continue;
        // wave at this thickness (Wave_Function::get_psi, src/wave_function.cuh:96-105)
        const float zbp = cd.thick_z_back_prop[ithk];
        float2* src = d_psi_.p;
        if (ramp) {
            // tilted beam: phase ramp before the output propagation
            RowArgs rr = ra;
            rr.in = d_psi_.p;
            rr.out = d_tmp_.p;
            rr.trans = ramp;
            rr.trans_stride = 0;  // one ramp for every wave
            rows(ROW_STEP, rr);
            src = d_tmp_.p;
        }
        ColArgs cb = ca;
        cb.in = src;
        cb.out = d_tmp_.p;
        cb.Px = prop + (size_t)(cd.n_slice + ithk) * pl;
        cb.Py = cb.Px + nx;
        if (m_.is_imaging()) {
            // coherent contribution: the weighted wave of this thickness, imaged once at output
            // (add_scale_psi_coh then set_m2psi_coh, src/wave_function.cuh:166-172, 210-218)
            if (d_coh_img_.p)
                for (int b = 0; b < nb; b++)
                    launch_axpy_wave(src + b * nxy, (float)w, nxy, d_coh_img_.p + (size_t)ithk * nxy, stream_);
            // image formation: transfer function per defocus point, inverse transform, |psi|^2
            // weighted (Microscope_Effects::operator(), src/microscope_effects.cuh:56-85)
            for (size_t j = 0; j < m_.obj_c10.size(); j++) {
                ColArgs cj = cb;
                cj.P2 = d_ctf_.p + j * nxy;
                cols(COL_LOAD | COL_PROP | COL_INVERSE | COL_STORE, cj);
                RowArgs rb = ra;
                rb.in = d_tmp_.p;
                rb.out = d_tmp_.p;
                rb.scale = 1.0f;
                rows(ROW_INVERSE, rb);
                for (int b = 0; b < nb; b++)
                    launch_ew_accumulate(d_tmp_.p + b * nxy, nx, ny, m_.out_ix_0, m_.out_ix_e, m_.out_iy_0,
                                         m_.out_iy_e, (double)(float)(w * m_.obj_w[j]), 0, nullptr,
                                         d_ew_m2_.p + (size_t)ithk * onxy, stream_);
            }
            continue;
        }
        if (m_.is_EWRS()) {
            RowArgs rb = ra;
            if (zbp != 0.0f || d_bwl_.p) {
                cols(COL_LOAD | COL_PROP | COL_INVERSE | COL_STORE, cb);
                rb.in = d_tmp_.p;
                rb.scale = 1.0f;
            } else {
                rb.in = src;
                rb.scale = 1.0f;
            }
            rb.out = d_tmp_.p;
            rows(ROW_INVERSE, rb);
        } else {
            cols(COL_LOAD | COL_PROP | COL_STORE, cb);
        }
        for (int b = 0; b < nb; b++) {
            const float2* wave = d_tmp_.p + b * nxy;
            // ED and CBED keep only |psi_hat|^2 (add_scale_crop_shift_m2psi_tot_from_psi, wave_function.cuh:172-184)
            launch_ew_accumulate(wave, nx, ny, m_.out_ix_0, m_.out_ix_e, m_.out_iy_0, m_.out_iy_e, w, sc ? 1 : 0,
                                 m_.is_EW() ? d_ew_psi_.p + (size_t)ithk * onxy * 2 : nullptr,
                                 sc ? nullptr : d_ew_m2_.p + (size_t)ithk * onxy, stream_);
            // coherent contribution of ED / CBED / PED: the configuration-weighted wave (add_scale_psi_coh,
            // src/output_multislice.hpp:770-780), kept cropped and shifted like the intensity
            if (d_ew_cohpsi_.p)
                launch_ew_accumulate(wave, nx, ny, m_.out_ix_0, m_.out_ix_e, m_.out_iy_0, m_.out_iy_e, w, 0,
                                     d_ew_cohpsi_.p + (size_t)ithk * onxy * 2, nullptr, stream_);
        }
    }
    iter_ += nb;
    }
    }
    check_cancel();
}

mt_output_dims Engine::dims() const { return output_dims(m_); }

// Output_Multislice::set_input_data sizes (src/output_multislice.hpp:415-520); host only.
mt_output_dims output_dims(const Model& m_) {
    mt_output_dims d{};
    d.n_thick = (int)m_.thick.size();
    if (m_.is_STEM()) {
        d.n_detector = (int)m_.det_g_inner.size();
        d.nx = m_.scan_nx;
        d.ny = m_.scan_ny;
        d.has_image_tot = 1;
        d.has_image_coh = m_.pn_coh_contrib ? 1 : 0;
        d.n_x = (int)m_.scan_x.size();
        d.n_y = (int)m_.scan_y.size();
    } else {
        d.nx = m_.out_ix_e - m_.out_ix_0;
        d.ny = m_.out_iy_e - m_.out_iy_0;
        d.has_psi_coh = m_.is_EW() ? 1 : 0;
        d.has_m2psi_coh = (m_.pn_coh_contrib && m_.is_wave_sim() && !m_.is_EW()) ? 1 : 0;
        d.has_m2psi_tot = m_.is_EW_SC() ? 0 : 1;
        d.n_x = d.nx;
        d.n_y = d.ny;
    }
    return d;
}

void Engine::read_stem(double* image_tot, size_t n) {
    if (!m_.is_STEM()) fail(MT_ERR_INVALID_ARG, "not a STEM engine");
    if (n < d_image_.n) fail(MT_ERR_INVALID_ARG, "image buffer too small");
    MTB_CUDA(cudaMemcpyAsync(image_tot, d_image_.p, sizeof(double) * d_image_.n, cudaMemcpyDeviceToHost, stream_));
    synchronize();
}

// Output_Multislice::set_output_grid + gather (src/output_multislice.hpp:1207-1245) and
// set_struct_multislice (mex_files_multem/ilc_multem.cu:382-481).
void Engine::write_output(mt_output_multislice* out) {
    if (!out) return;
    synchronize();
    const mt_output_dims d = dims();
    if (out->thick)
        for (int i = 0; i < d.n_thick; i++) out->thick[i] = m_.thick[i];
    if (m_.is_STEM()) {
        out->dx = m_.scan_dRx;
        out->dy = m_.scan_dRy;
        if (out->x)
            for (size_t i = 0; i < m_.scan_x.size(); i++) out->x[i] = m_.scan_x[i];
        if (out->y)
            for (size_t i = 0; i < m_.scan_y.size(); i++) out->y[i] = m_.scan_y[i];
        if (out->image_tot)
            MTB_CUDA(cudaMemcpy(out->image_tot, d_image_.p, sizeof(double) * d_image_.n, cudaMemcpyDeviceToHost));
        if (out->image_coh && d_coh_.p) {
            launch_coh_detect(d_coh_.p, (int)m_.thick.size(), m_.n_scan(), det_args(), d_image_coh_.p, stream_);
            synchronize();
            MTB_CUDA(cudaMemcpy(out->image_coh, d_image_coh_.p, sizeof(double) * d_image_coh_.n, cudaMemcpyDeviceToHost));
        }
    } else {
        const bool rs = !m_.is_grid_FS();
        out->dx = rs ? m_.grid.dRx : m_.grid.dgx;
        out->dy = rs ? m_.grid.dRy : m_.grid.dgy;
        if (out->x)
            for (int ix = m_.out_ix_0; ix < m_.out_ix_e; ix++)
                out->x[ix - m_.out_ix_0] = rs ? m_.grid.Rx(ix) : m_.grid.gx(ix);
        if (out->y)
            for (int iy = m_.out_iy_0; iy < m_.out_iy_e; iy++)
                out->y[iy - m_.out_iy_0] = rs ? m_.grid.Ry(iy) : m_.grid.gy(iy);
        if (out->psi_coh && d.has_psi_coh)
            MTB_CUDA(cudaMemcpy(out->psi_coh, d_ew_psi_.p, sizeof(double) * d_ew_psi_.n, cudaMemcpyDeviceToHost));
        if (out->m2psi_tot && d.has_m2psi_tot)
            MTB_CUDA(cudaMemcpy(out->m2psi_tot, d_ew_m2_.p, sizeof(double) * d_ew_m2_.n, cudaMemcpyDeviceToHost));
        if (out->m2psi_coh && d.has_m2psi_coh && d_coh_img_.p) {
            coherent_image();
            MTB_CUDA(cudaMemcpy(out->m2psi_coh, d_coh_m2_.p, sizeof(double) * d_coh_m2_.n, cudaMemcpyDeviceToHost));
        } else if (out->m2psi_coh && d.has_m2psi_coh) {
            // |configuration-averaged wave|^2 of the output window (set_m2psi_coh's last branch,
            // src/wave_function.cuh:219-226: the crop and shift commute with the average)
            std::vector<double> h(d_ew_cohpsi_.n);
            MTB_CUDA(cudaMemcpy(h.data(), d_ew_cohpsi_.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < h.size() / 2; i++) out->m2psi_coh[i] = h[2 * i] * h[2 * i] + h[2 * i + 1] * h[2 * i + 1];
        }
    }
}

// HRTEM / CBEI with pn_coh_contrib: the configuration-weighted wave of each thickness through the
// objective, the same passes run_ew applies to each configuration's wave (back-propagation,
// transfer function per defocus point, inverse transform, weighted |psi|^2), with weight 1 (the
// ISTEM_CBEI_HRTEM branch of set_m2psi_coh, src/wave_function.cuh:210-218). The back-propagation
// distance of a thickness does not depend on the configuration (z is never displaced).
void Engine::coherent_image() {
    const int nx = m_.grid.nx, ny = m_.grid.ny;
    const size_t nxy = (size_t)nx * ny;
    const size_t onxy = (size_t)(m_.out_ix_e - m_.out_ix_0) * (m_.out_iy_e - m_.out_iy_0);
    MTB_CUDA(cudaMemsetAsync(d_coh_m2_.p, 0, sizeof(double) * d_coh_m2_.n, stream_));
    const auto& TH = spec_->thicks();
    // back-propagation factors of every thickness, uploaded once
    const size_t pl = (size_t)nx + ny;
    std::vector<float2> tab(pl * TH.size());
    for (size_t t = 0; t < TH.size(); t++) prop_tables(TH[t].z_back_prop, &tab[t * pl], &tab[t * pl] + nx, true, 0);
    DevBuf<float2> d_bp;
    d_bp.upload(tab.data(), tab.size(), stream_);
    for (size_t t = 0; t < TH.size(); t++) {
        for (size_t j = 0; j < m_.obj_c10.size(); j++) {
            ColArgs cj{};
            cj.ny = ny;
            cj.nprobe = 1;
            cj.g = gdev_;
            cj.n_det = 0;
            cj.in = d_coh_img_.p + t * nxy;
            cj.out = d_tmp_.p;
            cj.Px = d_bp.p + t * pl;
            cj.Py = cj.Px + nx;
            cj.P2 = d_ctf_.p + j * nxy;
            cols(COL_LOAD | COL_PROP | COL_INVERSE | COL_STORE, cj);
            RowArgs rb{};
            rb.nx = nx;
            rb.nprobe = 1;
            rb.scale = 1.0f;
            rb.in = d_tmp_.p;
            rb.out = d_tmp_.p;
            rows(ROW_INVERSE, rb);
            launch_ew_accumulate(d_tmp_.p, nx, ny, m_.out_ix_0, m_.out_ix_e, m_.out_iy_0, m_.out_iy_e,
                                 (double)(float)m_.obj_w[j], 0, nullptr, d_coh_m2_.p + t * onxy, stream_);
        }
    }
    synchronize();  // before the tables' device buffer is released
}

// Projected potential / transmission of one slice, reference stored layout.
void Engine::projected_potential(int iconf, int islice, double* V, double* trans) {
    ConfData cd;
    prepare_conf(cd, iconf);
    if (islice < 0 || islice >= cd.n_slice) fail(MT_ERR_INVALID_ARG, "islice out of range");
    const size_t nxy = (size_t)m_.grid.nx * m_.grid.ny;
    DevBuf<float> dV;
    DevBuf<float2> dT;
    dV.alloc(nxy);
    dT.alloc(nxy);
    SplatArgs sa{};
    sa.g = gdev_;
    sa.atoms = cd.atoms.p;
    sa.slice_range = cd.ranges.p + islice;
    sa.tab = d_tab_.p;
    sa.R_max = d_Rmax_.p;
    sa.n_types = (int)Z_of_type_.size();
    sa.nR = m_.nR;
    sa.w = m_.Vr_factor();
    sa.wpo = (m_.interaction_model == 3);
    sa.trans = dT.p;
    sa.V = dV.p;
    launch_splat(sa, 0, 1, stream_);
    std::vector<float> hV(nxy);
    std::vector<float2> hT(nxy);
    MTB_CUDA(cudaMemcpyAsync(hV.data(), dV.p, sizeof(float) * nxy, cudaMemcpyDeviceToHost, stream_));
    MTB_CUDA(cudaMemcpyAsync(hT.data(), dT.p, sizeof(float2) * nxy, cudaMemcpyDeviceToHost, stream_));
    synchronize();
    if (V)
        for (size_t i = 0; i < nxy; i++) V[i] = hV[i];
    if (trans)
        for (size_t i = 0; i < nxy; i++) {
            trans[2 * i] = hT[i].x;
            trans[2 * i + 1] = hT[i].y;
        }
}

// Incident_Wave::operator()(space, output) (src/incident_wave.cuh:98-116): convergent probe(s) at
// iw_x/iw_y, defocus referred to z = 0; space 1 real, 2 reciprocal.
void Engine::incident_wave(int space, double* psi) {
    if (!m_.is_convergent_wave()) fail(MT_ERR_UNSUPPORTED, "incident_wave implements the convergent wave");
    const int nx = m_.grid.nx, ny = m_.grid.ny;
    const size_t nxy = (size_t)nx * ny;
    const int nb = (int)m_.iw_x.size();
    if (nb <= 0) fail(MT_ERR_INVALID_ARG, "iw_x/iw_y are empty");
    // probe normalisation as in the STEM constructor, with the tilt offset of this operator
    const LensF& L = m_.cond_lens;
    double count = 0;
    for (int ix = 0; ix < nx; ix++) {
        float gx = (float)((ix < m_.grid.nxh) ? ix : ix - nx) * m_.grid.dgx + m_.gx_0();
        for (int iy = 0; iy < ny; iy++) {
            float gy = (float)((iy < m_.grid.nyh) ? iy : iy - ny) * m_.grid.dgy + m_.gy_0();
            float g2 = gx * gx + gy * gy;
            if ((L.g2_min <= g2) && (g2 < L.g2_max)) count += 1.0;
        }
    }
    const float norm = (float)std::sqrt(1.0 / (double)(float)count);
    const float f_s = m_.cond_lens.c_10 - (m_.cond_lens.zero_defocus_plane - 0.0f);
    LensF Lp = m_.cond_lens;
    Lp.set_defocus(f_s);
    std::vector<float2> beam(nb);
    for (int i = 0; i < nb; i++) beam[i] = make_float2(m_.grid.exp_factor_Rx(m_.iw_x[i]), m_.grid.exp_factor_Ry(m_.iw_y[i]));
    DevBuf<float2> dbeam, dpsi;
    dbeam.upload(beam.data(), nb, stream_);
    dpsi.alloc(nxy * nb);
    ColArgs ca{};
    ca.ny = ny;
    ca.nprobe = nb;
    ca.g = gdev_;
    ca.beam = dbeam.p;
    ca.probe = probe_params(Lp.c_c_10, !is_zero_f(f_s), true);
    ca.probe.norm = norm;
    ca.out = dpsi.p;
    if (space == 2) {
        cols(COL_STORE, ca);
    } else {
        cols(COL_INVERSE | COL_STORE, ca);
        RowArgs ra{};
        ra.in = dpsi.p;
        ra.out = dpsi.p;
        ra.nx = nx;
        ra.nprobe = nb;
        ra.scale = 1.0f;
        rows(ROW_INVERSE, ra);
    }
    std::vector<float2> h(nxy * nb);
    MTB_CUDA(cudaMemcpyAsync(h.data(), dpsi.p, sizeof(float2) * h.size(), cudaMemcpyDeviceToHost, stream_));
    synchronize();
    for (size_t i = 0; i < nxy; i++) {
        double re = 0, im = 0;
        for (int b = 0; b < nb; b++) {
            re += h[b * nxy + i].x;
            im += h[b * nxy + i].y;
        }
        psi[2 * i] = re;
        psi[2 * i + 1] = im;
    }
}

// ilc_propagate (mex_files_multem/ilc_propagate.cu:125-147; Propagator::operator(),
// src/propagator.cuh:51-103): the user wave iw_psi is fft-shifted in, Fourier transformed, multiplied
// by the Fresnel propagator of distance z (tilt offset g0 from theta/phi, 1/N folded in) and, for
// real-space output, transformed back; then shifted back. With |z| <= 1e-5 (isZero) the real-space
// result is the wave itself and the reciprocal one FFT2(psi)/N. One wave runs through the same line
// passes as a multislice step with a transmission function of ones: row pass F_y, column pass
// F_x * P (* F_x^-1), row pass F_y^-1.
void propagate_wave(const mt_system_conf* conf, const mt_input_multislice* in, int space, double z, double* psi_out) {
    if (space != 1 && space != 2) fail(MT_ERR_INVALID_ARG, "space must be 1 (real) or 2 (reciprocal)");
    if (!psi_out) fail(MT_ERR_INVALID_ARG, "psi_out is NULL");
    int device = 0;
    if (conf) {
        if (conf->precision != 1) fail(MT_ERR_UNSUPPORTED, "this engine computes in FP32 (system_conf.precision must be 1)");
        if (conf->device != 2) fail(MT_ERR_UNSUPPORTED, "this engine runs on the GPU (system_conf.device must be 2)");
        device = conf->gpu_device;
    }
    const Model m = build_prop_model(in);
    const int nx = m.grid.nx, ny = m.grid.ny;
    const size_t nxy = (size_t)nx * ny;
    std::vector<float2> h(nxy);
    for (int ix = 0; ix < nx; ix++)
        for (int iy = 0; iy < ny; iy++) {
            const size_t src = (size_t)ix * ny + iy;
            const size_t dst = (size_t)((ix + m.grid.nxh) % nx) * ny + (iy + m.grid.nyh) % ny;
            h[dst] = make_float2(m.iw_psi[2 * src], m.iw_psi[2 * src + 1]);
        }
    auto write_out = [&](const std::vector<float2>& v) {
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                const size_t src = (size_t)((ix + m.grid.nxh) % nx) * ny + (iy + m.grid.nyh) % ny;
                const size_t dst = (size_t)ix * ny + iy;
                psi_out[2 * dst] = v[src].x;
                psi_out[2 * dst + 1] = v[src].y;
            }
    };
    const bool zero = is_zero_f((float)z);
    if (zero && space == 1) {
        write_out(h);
        return;
    }
    int ndev = 0;
    MTB_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) fail(MT_ERR_INVALID_ARG, "gpu_device out of range");
    MTB_CUDA(cudaSetDevice(device));
    cudaStream_t st;
    MTB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } guard{st};
    std::vector<float2> ones(nxy, make_float2(1.0f, 0.0f));
    std::vector<float2> prop((size_t)nx + ny);
    prop_tables(m, zero ? 0.0f : (float)z, prop.data(), prop.data() + nx, false);
    DevBuf<float2> d_psi, d_out, d_one, d_prop;
    d_psi.upload(h.data(), nxy, st);
    d_one.upload(ones.data(), nxy, st);
    d_prop.upload(prop.data(), prop.size(), st);
    d_out.alloc(nxy);
    RowArgs ra{};
    ra.in = d_psi.p;
    ra.out = d_psi.p;
    ra.trans = d_one.p;
    ra.nx = nx;
    ra.nprobe = 1;
    ra.scale = 1.0f;
    launch_rows(ny, ROW_FIRST_REAL, ra, 0, st);
    ColArgs ca{};
    ca.in = d_psi.p;
    ca.out = d_psi.p;
    ca.ny = ny;
    ca.nprobe = 1;
    ca.g = grid_dev(m.grid);
    ca.Px = d_prop.p;
    ca.Py = d_prop.p + nx;
    ca.det_w = 1;
    launch_cols(nx, space == 1 ? (COL_LOAD | COL_PROP | COL_INVERSE | COL_STORE) : (COL_LOAD | COL_PROP | COL_STORE), ca, 0,
                st);
    const float2* res = d_psi.p;
    if (space == 1) {
        RowArgs rb{};
        rb.in = d_psi.p;
        rb.out = d_out.p;
        rb.nx = nx;
        rb.nprobe = 1;
        rb.scale = 1.0f;
        launch_rows(ny, ROW_INVERSE, rb, 0, st);
        res = d_out.p;
    }
    MTB_CUDA(cudaMemcpyAsync(h.data(), res, sizeof(float2) * nxy, cudaMemcpyDeviceToHost, st));
    MTB_CUDA(cudaStreamSynchronize(st));
    write_out(h);
}

}  // namespace mtb
