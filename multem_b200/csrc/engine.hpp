// Multislice engine: device state and the batched slice loop.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <memory>
#include <vector>

#include "devmem.hpp"
#include "host_model.hpp"
#include "kernels.cuh"
#include "multem_b200.h"
#include "tables.hpp"

namespace mtb {

// Device array from the library's memory pool (devmem.hpp).
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    int dev = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), dev(o.dev) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        std::swap(p, o.p);
        std::swap(n, o.n);
        std::swap(dev, o.dev);
        return *this;
    }
    ~DevBuf() { if (p) dev_free(p, dev); }
    void alloc(size_t count) {
        if (count <= n && p) return;
        if (p) dev_free(p, dev);
        p = nullptr;
        n = 0;
        p = static_cast<T*>(dev_alloc(sizeof(T) * (count ? count : 1), &dev));
        n = count;
    }
    // free now; the owner has synchronised every stream that used the buffer
    void release_idle() {
        if (p) dev_free_idle(p, dev);
        p = nullptr;
        n = 0;
    }
    void upload(const T* h, size_t count, cudaStream_t s) {
        alloc(count);
        if (count) cuda_check(cudaMemcpyAsync(p, h, sizeof(T) * count, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync H2D");
    }
};

GridDev grid_dev(const GridF& g);
// Fresnel propagator factors Px[nx], Py[ny] of distance dz (see engine.cu).
void prop_tables(const Model& m, float dz, float2* px, float2* py, bool output, int irot = 0);
// mt_propagate: the user wave in->iw_psi propagated by z (space 1 real, 2 reciprocal).
void propagate_wave(const mt_system_conf* conf, const mt_input_multislice* in, int space, double z, double* psi_out);

// Per phonon configuration: displaced atoms, slice ranges, propagator tables, probe defocus.
struct ConfData {
    int iconf = 0;
    int n_slice = 0;
    int last_slice = 0;             // last slice that carries a thickness
    std::vector<int> slice_ithk;    // per slice
    std::vector<float> thick_z_back_prop;
    std::vector<float> probe_c_c_10;  // per point of the defocus-spread quadrature
    std::vector<int> probe_nz_c10;
    DevBuf<float4> atoms;
    DevBuf<int2> ranges;
    DevBuf<float2> prop;            // per rotation, per slice then per thickness: Px[nx] then Py[ny]
    void release_idle() {
        atoms.release_idle();
        ranges.release_idle();
        prop.release_idle();
    }
};

mt_output_dims output_dims(const Model& m);

class Engine {
  public:
    Engine(const mt_system_conf* conf, const mt_input_multislice* in);
    ~Engine();

    const Model& model() const { return m_; }
    Specimen& specimen() { return *spec_; }

    mt_output_dims dims() const;
    void reset();
    void prepare_confs(int c0, int c1);      // host RNG + slicing + uploads
    void run_prepared(int c0, int c1);       // device-only work for prepared confs
    void run_confs(int c0, int c1);          // prepare + run
    // Whole-run recording, for one CUDA graph over a batch of engines: prepare_run prepares every
    // configuration of the run in its own buffers and chooses the pass variants (host work, with
    // synchronisation); record_run then issues all of the run's device work on this engine's
    // stream without any host synchronisation (the caller has the stream in a capture); after the
    // graph has run, write_output reads the results.
    void prepare_run();
    void record_run();
    void write_output(mt_output_multislice* out);
    void read_stem(double* image_tot, size_t n);
    void cancel() { cancel_ = true; }
    void progress(int* iter, int* niter) const { *iter = iter_; *niter = niter_; }
    long long launches() const { return launches_; }
    void synchronize();

    // operator-level entries
    void projected_potential(int iconf, int islice, double* V, double* trans);
    void incident_wave(int space, double* psi);

    cudaStream_t stream() const { return stream_; }
    int batch_size() const { return batch_; }

    // device timing
    void set_timing(bool on) { timing_ = on; }
    // Bound of each wait of a line pass for its bulk copies (ns); 0: a copy that has not landed at
    // the first check is a timeout.
    void set_wait_limit(long long ns) { wait_ns_ = ns < 0 ? 0 : ns; }
    int pass_variants() const { return pipe_; }
    // The autotuner's choice: row and column pass variant (0 per-thread loads, 1 bulk-copy fed,
    // 2 and 3 bulk-copy fed in the alternative pipeline shapes 1 and 2) and probes per launch.
    void tuning(int* rows_variant, int* cols_variant, int* probes_per_launch) const;
    void timing(double* total_ms, double* rows_ms, long long* n_rows, double* cols_ms, long long* n_cols);

  private:
    bool timing_ = false;
    struct TimedLaunch {
        cudaEvent_t a, b;
        int kind;  // 0 rows, 1 cols
    };
    std::vector<TimedLaunch> tl_;
    size_t tl_used_ = 0;
    cudaEvent_t run_a_ = nullptr, run_b_ = nullptr;
    cudaEvent_t conf_done_ = nullptr;  // last launch of the previous configuration in run_confs
    void tl_begin(int kind);
    void tl_end();
    void rows(RowMode mode, const RowArgs& a);
    void cols(int flags, const ColArgs& a);
    Model m_;
    std::unique_ptr<Specimen> spec_;
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    std::atomic<bool> cancel_{false};
    int iter_ = 0, niter_ = 0;
    long long launches_ = 0;

    // element tables
    static constexpr int kChargeSlots = 15;  // charges -7..7, the reference's ionic range
    std::vector<int> type_of_Zq_;    // (Z-1)*kChargeSlots + charge+7 -> table index or -1
    std::vector<int> Z_of_type_;
    std::vector<int> charge_of_type_;
    int atom_type(int Z, int charge) const;
    std::vector<float> R_max_f_;     // per type
    std::vector<TableHead> heads_;
    DevBuf<float> d_tab_;
    DevBuf<float> d_Rmax_;

    // wave state
    int batch_ = 1;
    DevBuf<int> d_err_;              // set by a line pass whose bounded wait gave up
    int pipe_ = 3;                   // bulk-copy-fed line passes where they fit (bit 0 rows, bit 1 cols)
    long long wait_ns_ = 2000000000ll;  // bound of the line passes' waits for their copies
    bool tune_ = true;               // choose pipe_, shape_, run_batch_ per shape with tune (MTB_PIPE unset)
    int shape_ = 0;                  // pipeline shapes of the step passes (bits 0-1 rows, bits 2-3 cols)
    int run_batch_ = 1;              // probes per launch (<= batch_, the allocated batch)
    // exit-wave family (EW, ED, HRTEM) with frozen phonons: configurations whose waves advance
    // through the slices together, one launch per pass for all of them, each with its own
    // transmission functions (1: one configuration at a time)
    int ew_batch_ = 1;
    DevBuf<float2> d_psi_;
    DevBuf<float2> d_trans_;
    DevBuf<float2> d_tmp_;
    DevBuf<float2> d_beam_;          // all scan positions (exp factors)
    DevBuf<int> d_scan_idx_;
    DevBuf<double> d_partial_;
    DevBuf<double> d_image_;         // [n_thk][n_det][n_scan]
    DevBuf<double> d_ew_psi_;        // [n_thk][out_nxy][2]
    DevBuf<double> d_ew_m2_;         // [n_thk][out_nxy]
    DevBuf<double> d_ew_cohpsi_;     // ED/CBED/PED with pn_coh_contrib: weighted wave sum [n_thk][out_nxy][2]
    DevBuf<float2> d_coh_img_;       // HRTEM/CBEI with pn_coh_contrib: weighted wave sum, row-pass layout [n_thk][nx*ny]
    DevBuf<double> d_coh_m2_;        // its image through the objective [n_thk][out_nxy]
    void coherent_image();
    DevBuf<float2> d_prop_bp_;       // back-propagation tables per thickness
    DevBuf<float2> d_ramp_;          // tilted beam: output phase ramp / ny per rotation (else empty)
    DevBuf<float> d_detmat_;         // matrix detectors [n_det][nx][ny] (else empty)
    DevBuf<float2> d_ctf_;           // HRTEM transfer functions, one [nx][ny] table per defocus point
    DevBuf<float2> d_beams_psi_;     // convergent incident wave of several beams: one wave per beam
    DevBuf<float2> d_user_wave_;     // user-defined incident wave, in the row pass's input layout
    DevBuf<float2> d_tmp2_;          // tilted ISTEM with several thicknesses: the ramped batch
    DevBuf<float2> d_bwl_;           // band-width limit factor [nx][ny] (bwl = 1), else empty
    DevBuf<float2> d_one_;           // ones [nx][ny]: the row pass that transforms the transmission functions
    DevBuf<float2> d_p0_;            // zero-distance propagator factors (1/N only), Px then Py
    DevBuf<float2> d_coh_;           // STEM with pn_coh_contrib: psi_coh [n_thk][n_scan][nx][ny]
    DevBuf<double> d_image_coh_;     // [n_thk][n_det][n_scan]
    DevBuf<float4> d_atoms_u_;       // pn_rng 1: undisplaced atoms (x, y, occ, type), z-sorted
    DevBuf<float> d_sigma_;          // pn_rng 1: per-atom displacement sigma
    ColArgs det_args() const;        // detector description for the column pass
    std::vector<ConfData> confs_;
    GridDev gdev_{};
    float probe_norm_ = 1.0f;

    void build_types();
    void build_tilt_ramp();
    void prepare_conf(ConfData& cd, int iconf);
    struct ConfStage {                // host staging of a configuration's device data
        std::vector<float4> at;
        std::vector<int2> rg;
        std::vector<float2> prop;
        size_t n_atoms = 0;
    };
    void prepare_conf_host(ConfData& cd, int iconf, ConfStage& st);
    std::vector<float> prop_key_;     // slice thicknesses and back-propagation distances of prop_cache_
    std::vector<float2> prop_cache_;  // propagator tables of every rotation (per slice, then per thickness)
    void prepare_conf_device(ConfData& cd, ConfStage& st);
    void run_conf(ConfData& cd);
    // the splats of nb configurations (into consecutive transmission blocks) and their slice loop
    // (nb > 1: exit-wave family only, configurations with identical slicing)
    void run_conf_batch(ConfData* const* cds, int nb);
    void run_prepared_range(int c0, int c1);  // prepared configurations c0..c1 in batches of ew_batch_
    struct Tuning {
        int pipe, shape, nprobe;
    };
    Tuning tune_passes(int nprobe, ConfData& cd);
    void tune(ConfData& cd);         // tune_passes for this engine's shape; sets pipe_, shape_, run_batch_
    void run_stem(ConfData& cd);
    void run_ew(ConfData* const* cds, int nb);
    void prop_tables(float dz, float2* px, float2* py, bool output, int irot = 0) const;
    ProbeDev probe_params(float c_c_10, int nz_c10, bool tilt_offset) const;
    void build_ctf_tables();
    float aperture_norm() const;
    void build_user_wave();
    void build_bwl();
    void band_limit_trans(const ConfData& cd, float2* trans);
    void check_cancel();
    void zero_accumulators();        // the accumulators' memsets on the stream (no synchronisation)
    ConfData* find_conf(int iconf);

    // CUDA graphs of run_conf_batch, one per group of configuration slots (run_confs alternates two
    // groups of ew_batch_ slots whose buffers keep their addresses), replayed while the launch
    // sequence and its arguments match
    struct ConfGraph {
        cudaGraphExec_t exec = nullptr;
        std::vector<char> sig;  // launch-shaping data the graph was captured with
        int iters = 0;          // progress iterations it advances
        long long launches = 0;  // kernel launches it holds
    };
    bool graphs_ = true;
    bool capturing_ = false;
    std::vector<ConfData> slot_;     // 2 x ew_batch_
    ConfGraph graph_[2];
    ConfGraph range_graph_;  // run_prepared: one graph over a range of prepared configurations
    std::vector<char> graph_signature(const ConfData& cd) const;
    void run_conf_graph(ConfData* const* cds, int nb, ConfGraph& g);
};

}  // namespace mtb
