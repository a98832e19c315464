// extern "C" entry points declared in include/multem_b200.h.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>
#include <exception>
#include <memory>
#include <string>

#include "common.hpp"
#include "devmem.hpp"
#include "engine.hpp"
#include "matio.hpp"
#include "multem_b200.h"

struct mt_engine {
    std::unique_ptr<mtb::Engine> eng;
};

struct mt_mat_input {
    std::unique_ptr<mtb::matio::Input> h;
};

namespace {

thread_local std::string g_last_error;

template <class F>
mt_status guarded(F fn) {
    try {
        fn();
        g_last_error.clear();
        return MT_OK;
    } catch (const mtb::Error& e) {
        g_last_error = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return MT_ERR_OOM;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return MT_ERR_INTERNAL;
    } catch (...) {
        g_last_error = "unknown error";
        return MT_ERR_INTERNAL;
    }
}

mt_system_conf default_conf() {
    mt_system_conf c{};
    c.precision = 1;
    c.device = 2;
    c.cpu_nthread = 1;
    c.gpu_device = 0;
    return c;
}

}  // namespace

extern "C" {

int mt_abi_version(void) { return MT_ABI_VERSION; }

const char* mt_last_error(void) { return g_last_error.c_str(); }

mt_status mt_device_alloc_count(long long* count) {
    return guarded([&] {
        if (!count) mtb::fail(MT_ERR_INVALID_ARG, "count is NULL");
        *count = mtb::dev_alloc_count();
    });
}

mt_status mt_output_query(const mt_input_multislice* in, mt_output_dims* dims) {
    return guarded([&] {
        if (!dims) mtb::fail(MT_ERR_INVALID_ARG, "dims is NULL");
        *dims = mtb::output_dims(mtb::build_model(in));
    });
}

mt_status mt_engine_create(const mt_system_conf* conf, const mt_input_multislice* in, mt_engine** eng) {
    return guarded([&] {
        if (!eng) mtb::fail(MT_ERR_INVALID_ARG, "eng is NULL");
        *eng = nullptr;
        mt_system_conf c = conf ? *conf : default_conf();
        auto h = std::unique_ptr<mt_engine>(new mt_engine);
        h->eng.reset(new mtb::Engine(&c, in));
        *eng = h.release();
    });
}

mt_status mt_engine_destroy(mt_engine* eng) {
    return guarded([&] { delete eng; });
}

mt_status mt_engine_run(mt_engine* eng, mt_output_multislice* out) {
    return guarded([&] {
        if (!eng) mtb::fail(MT_ERR_INVALID_ARG, "eng is NULL");
        auto& e = *eng->eng;
        e.reset();
        e.run_confs(e.model().fp_iconf_0, e.model().pn_nconf);
        e.write_output(out);
    });
}

mt_status mt_engine_run_confs(mt_engine* eng, int iconf_0, int iconf_e) {
    return guarded([&] {
        if (!eng) mtb::fail(MT_ERR_INVALID_ARG, "eng is NULL");
        eng->eng->run_confs(iconf_0, iconf_e);
    });
}

mt_status mt_engine_reset(mt_engine* eng) {
    return guarded([&] {
        if (!eng) mtb::fail(MT_ERR_INVALID_ARG, "eng is NULL");
        eng->eng->reset();
    });
}

mt_status mt_engine_read_stem(mt_engine* eng, double* image_tot, size_t n) {
    return guarded([&] {
        if (!eng || !image_tot) mtb::fail(MT_ERR_INVALID_ARG, "NULL argument");
        eng->eng->read_stem(image_tot, n);
    });
}

mt_status mt_engine_cancel(mt_engine* eng) {
    return guarded([&] {
        if (!eng) mtb::fail(MT_ERR_INVALID_ARG, "eng is NULL");
        eng->eng->cancel();
    });
}

mt_status mt_engine_set_wait_limit(mt_engine* eng, double seconds) {
    return guarded([&] {
        if (!eng) mtb::fail(MT_ERR_INVALID_ARG, "eng is NULL");
        if (!(seconds >= 0.0) || seconds > 60.0) mtb::fail(MT_ERR_INVALID_ARG, "seconds must be in [0, 60]");
        eng->eng->set_wait_limit((long long)(seconds * 1e9));
    });
}

mt_status mt_engine_progress(mt_engine* eng, int* iter, int* niter) {
    return guarded([&] {
        if (!eng || !iter || !niter) mtb::fail(MT_ERR_INVALID_ARG, "NULL argument");
        eng->eng->progress(iter, niter);
    });
}

mt_status mt_engine_prepare_confs(mt_engine* eng, int iconf_0, int iconf_e) {
    return guarded([&] {
        if (!eng) mtb::fail(MT_ERR_INVALID_ARG, "eng is NULL");
        eng->eng->prepare_confs(iconf_0, iconf_e);
    });
}

mt_status mt_engine_run_prepared(mt_engine* eng, int iconf_0, int iconf_e) {
    return guarded([&] {
        if (!eng) mtb::fail(MT_ERR_INVALID_ARG, "eng is NULL");
        eng->eng->run_prepared(iconf_0, iconf_e);
    });
}

mt_status mt_engine_launch_count(mt_engine* eng, long long* n) {
    return guarded([&] {
        if (!eng || !n) mtb::fail(MT_ERR_INVALID_ARG, "NULL argument");
        *n = eng->eng->launches();
    });
}

mt_status mt_engine_pass_variants(mt_engine* eng, int* variants) {
    return guarded([&] {
        if (!eng || !variants) mtb::fail(MT_ERR_INVALID_ARG, "NULL argument");
        *variants = eng->eng->pass_variants();
    });
}

mt_status mt_engine_tuning(mt_engine* eng, int* rows_variant, int* cols_variant, int* probes_per_launch) {
    return guarded([&] {
        if (!eng || !rows_variant || !cols_variant || !probes_per_launch) mtb::fail(MT_ERR_INVALID_ARG, "NULL argument");
        eng->eng->tuning(rows_variant, cols_variant, probes_per_launch);
    });
}

mt_status mt_engine_set_timing(mt_engine* eng, int on) {
    return guarded([&] {
        if (!eng) mtb::fail(MT_ERR_INVALID_ARG, "eng is NULL");
        eng->eng->set_timing(on != 0);
    });
}

mt_status mt_engine_timing(mt_engine* eng, double* total_ms, double* rows_ms, long long* n_rows, double* cols_ms,
                           long long* n_cols) {
    return guarded([&] {
        if (!eng || !total_ms || !rows_ms || !n_rows || !cols_ms || !n_cols) mtb::fail(MT_ERR_INVALID_ARG, "NULL argument");
        eng->eng->timing(total_ms, rows_ms, n_rows, cols_ms, n_cols);
    });
}

mt_status mt_input_report(const mt_input_multislice* in, char* buf, size_t n, int* n_changes) {
    return guarded([&] {
        const mtb::Model m = mtb::build_model(in);
        std::string r;
        for (const auto& c : m.clamps) r += c + "\n";
        if (n_changes) *n_changes = (int)m.clamps.size();
        if (buf && n > 0) {
            const size_t k = std::min(n - 1, r.size());
            std::memcpy(buf, r.data(), k);
            buf[k] = '\0';
        }
    });
}

mt_status mt_multislice_run(const mt_system_conf* conf, const mt_input_multislice* in, mt_output_multislice* out) {
    return guarded([&] {
        mt_system_conf c = conf ? *conf : default_conf();
        mtb::Engine e(&c, in);
        e.run_confs(e.model().fp_iconf_0, e.model().pn_nconf);
        e.write_output(out);
    });
}

mt_status mt_mat_input_open(const char* path, const char* var, mt_mat_input** handle, mt_system_conf* conf,
                            mt_input_multislice* in) {
    return guarded([&] {
        if (!path || !handle || !in) mtb::fail(MT_ERR_INVALID_ARG, "NULL argument");
        *handle = nullptr;
        auto h = std::make_unique<mt_mat_input>();
        h->h = mtb::matio::read_input(path, var ? var : "");
        *in = h->h->in;
        if (conf) *conf = h->h->conf;
        *handle = h.release();
    });
}

mt_status mt_mat_input_close(mt_mat_input* handle) {
    delete handle;
    return MT_OK;
}

mt_status mt_mat_output_write(const char* path, const char* var, const mt_input_multislice* in,
                              const mt_output_multislice* out, int compress) {
    return guarded([&] {
        if (!path || !in || !out) mtb::fail(MT_ERR_INVALID_ARG, "NULL argument");
        const mt_output_dims d = mtb::output_dims(mtb::build_model(in));
        mtb::matio::write_output(path, var ? var : "", d, *out, compress != 0);
    });
}

mt_status mt_multislice_run_mat(const char* in_path, const char* var, const char* out_path, int compress) {
    return guarded([&] {
        if (!in_path || !out_path) mtb::fail(MT_ERR_INVALID_ARG, "NULL path");
        auto h = mtb::matio::read_input(in_path, var ? var : "");
        const mt_input_multislice& in = h->in;
        const mt_output_dims d = mtb::output_dims(mtb::build_model(&in));
        const size_t nxy = (size_t)d.nx * d.ny;
        std::vector<double> x(std::max(1, d.n_x)), y(std::max(1, d.n_y)), th(std::max(1, d.n_thick));
        std::vector<double> itot, icoh, m2, psi, m2c;
        mt_output_multislice out{};
        out.x = x.data();
        out.y = y.data();
        out.thick = th.data();
        auto sized = [](std::vector<double>& v, size_t n) { v.assign(std::max<size_t>(1, n), 0.0); return v.data(); };
        if (d.has_image_tot) out.image_tot = sized(itot, (size_t)d.n_thick * d.n_detector * nxy);
        if (d.has_image_coh) out.image_coh = sized(icoh, (size_t)d.n_thick * d.n_detector * nxy);
        if (d.has_m2psi_tot) out.m2psi_tot = sized(m2, (size_t)d.n_thick * nxy);
        if (d.has_psi_coh) out.psi_coh = sized(psi, 2 * (size_t)d.n_thick * nxy);
        if (d.has_m2psi_coh) out.m2psi_coh = sized(m2c, (size_t)d.n_thick * nxy);
        mtb::Engine e(&h->conf, &in);
        e.run_confs(e.model().fp_iconf_0, e.model().pn_nconf);
        e.write_output(&out);
        mtb::matio::write_output(out_path, "", d, out, compress != 0);
    });
}

// The whole batch as one CUDA graph: every input's engine is created (on `workers` host threads)
// and prepares all of its configurations, then one capture records each engine's complete run on
// the engine's own stream, forked from and joined back into one origin stream, so that a single
// graph launch advances every specimen, configuration and probe batch, the GPU running the
// specimens' independent branches concurrently. An input whose engine cannot be set up gets its
// status in st/msg and is left out of the graph; the others run. Returns false (nothing run, st
// cleared) when the engines do not fit in device memory together; the caller then runs the inputs
// on host workers instead.
static bool run_batch_graph(const mt_system_conf& c, int n, const mt_input_multislice* in, mt_output_multislice* out,
                            const std::vector<int>& order, int workers, std::vector<mt_status>& st,
                            std::vector<std::string>& msg) {
    std::vector<std::unique_ptr<mtb::Engine>> eng(n);
    std::atomic<int> next{0};
    std::atomic<bool> oom{false};
    const bool prof = std::getenv("MTB_BATCH_PROFILE") != nullptr;  // phase times on stderr
    auto now = [] { return std::chrono::steady_clock::now(); };
    auto secs = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
        return std::chrono::duration<double>(b - a).count();
    };
    const auto t0 = now();
    auto build = [&] {
        for (;;) {
            const int k = next++;
            if (k >= n || oom) break;
            const int i = order[k];
            st[i] = guarded([&] {
                MTB_CUDA(cudaSetDevice(c.gpu_device));
                eng[i].reset(new mtb::Engine(&c, &in[i]));
                eng[i]->prepare_run();
            });
            if (st[i] == MT_ERR_OOM) oom = true;
            if (st[i] != MT_OK) msg[i] = g_last_error;
        }
    };
    {
        std::vector<std::thread> pool;
        for (int t = 1; t < workers; t++) pool.emplace_back(build);
        build();
        for (auto& t : pool) t.join();
    }
    if (oom) {  // the engines are released here; the host-worker path runs the batch
        for (int i = 0; i < n; i++) {
            st[i] = MT_OK;
            msg[i].clear();
        }
        return false;
    }
    std::vector<int> ok;
    for (int k = 0; k < n; k++)
        if (st[order[k]] == MT_OK) ok.push_back(order[k]);
    if (ok.empty()) return true;
    const auto t1 = now();
    MTB_CUDA(cudaSetDevice(c.gpu_device));
    cudaStream_t origin = nullptr;
    MTB_CUDA(cudaStreamCreateWithFlags(&origin, cudaStreamNonBlocking));
    const int m = (int)ok.size();
    std::vector<cudaEvent_t> ev(m + 1, nullptr);
    for (auto& e : ev) MTB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    auto cleanup = [&] {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto& e : ev) cudaEventDestroy(e);
        cudaStreamDestroy(origin);
    };
    try {
        MTB_CUDA(cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal));
        try {
            MTB_CUDA(cudaEventRecord(ev[m], origin));
            for (int k = 0; k < m; k++) {
                mtb::Engine& e = *eng[ok[k]];
                MTB_CUDA(cudaStreamWaitEvent(e.stream(), ev[m], 0));  // fork: the engine's stream joins the capture
                e.record_run();
                MTB_CUDA(cudaEventRecord(ev[k], e.stream()));
                MTB_CUDA(cudaStreamWaitEvent(origin, ev[k], 0));      // join
            }
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(origin, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        MTB_CUDA(cudaStreamEndCapture(origin, &graph));
        const auto t2 = now();
        MTB_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        const auto t3 = now();
        MTB_CUDA(cudaGraphLaunch(exec, origin));
        MTB_CUDA(cudaStreamSynchronize(origin));
        const auto t4 = now();
        if (prof) {
            size_t nodes = 0;
            cudaGraphGetNodes(graph, nullptr, &nodes);
            std::fprintf(stderr, "batch graph: %d inputs, %zu nodes; set-up %.3f s, capture %.3f s, instantiate %.3f s, run %.3f s\n",
                         m, nodes, secs(t0, t1), secs(t1, t2), secs(t2, t3), secs(t3, t4));
        }
        for (int i : ok) {
            st[i] = guarded([&] { eng[i]->write_output(&out[i]); });
            if (st[i] != MT_OK) msg[i] = g_last_error;
        }
    } catch (...) {
        cleanup();
        throw;
    }
    cleanup();
    return true;
}

mt_status mt_multislice_run_batch(const mt_system_conf* conf, int n, const mt_input_multislice* in,
                                  mt_output_multislice* out, mt_status* status) {
    std::vector<mt_status> st(n > 0 ? n : 0, MT_OK);
    std::vector<std::string> msg(st.size());
    mt_status rc = guarded([&] {
        if (n < 0 || (n > 0 && (!in || !out))) mtb::fail(MT_ERR_INVALID_ARG, "bad batch arguments");
        const mt_system_conf c = conf ? *conf : default_conf();
        // largest first: grid points x probes x configurations x slices (from the box depth)
        std::vector<double> cost(n);
        for (int i = 0; i < n; i++) {
            const mt_input_multislice& q = in[i];
            double probes = (q.simulation_type == 11) ? (double)std::max(1, q.scanning_ns) * std::max(1, q.scanning_ns) : 1;
            double slices = (q.spec_dz > 0 && q.spec_lz > 0) ? q.spec_lz / q.spec_dz : 1;
            cost[i] = (double)q.nx * q.ny * probes * std::max(1, q.pn_nconf) * slices;
        }
        std::vector<int> order(n);
        for (int i = 0; i < n; i++) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
        const char* w = std::getenv("MTB_BATCH_WORKERS");
        const int workers = std::max(1, std::min(n, w ? std::atoi(w) : 4));
        const char* mode = std::getenv("MTB_BATCH_MODE");
        const bool graph = n > 1 && !(mode && std::strcmp(mode, "threads") == 0) &&
                           run_batch_graph(c, n, in, out, order, workers, st, msg);
        std::atomic<int> next{graph ? n : 0};
        auto work = [&] {
            for (;;) {
                const int k = next++;
                if (k >= n) break;
                const int i = order[k];
                st[i] = guarded([&] {
                    MTB_CUDA(cudaSetDevice(c.gpu_device));
                    mtb::Engine e(&c, &in[i]);
                    e.run_confs(e.model().fp_iconf_0, e.model().pn_nconf);
                    e.write_output(&out[i]);
                });
                if (st[i] != MT_OK) msg[i] = g_last_error;
            }
        };
        std::vector<std::thread> pool;
        for (int t = 1; t < workers; t++) pool.emplace_back(work);
        work();
        for (auto& t : pool) t.join();
        for (int i = 0; i < n; i++)
            if (st[i] != MT_OK) throw mtb::Error(st[i], "input " + std::to_string(i) + ": " + msg[i]);
    });
    if (status)
        for (int i = 0; i < n; i++) status[i] = st[i];
    return rc;
}

mt_status mt_projected_potential(const mt_system_conf* conf, const mt_input_multislice* in, int iconf, int islice,
                                 double* V) {
    return guarded([&] {
        if (!V) mtb::fail(MT_ERR_INVALID_ARG, "V is NULL");
        mt_system_conf c = conf ? *conf : default_conf();
        mtb::Engine e(&c, in);
        e.projected_potential(iconf, islice, V, nullptr);
    });
}

mt_status mt_transmission_function(const mt_system_conf* conf, const mt_input_multislice* in, int iconf, int islice,
                                   double* trans) {
    return guarded([&] {
        if (!trans) mtb::fail(MT_ERR_INVALID_ARG, "trans is NULL");
        mt_system_conf c = conf ? *conf : default_conf();
        mtb::Engine e(&c, in);
        e.projected_potential(iconf, islice, nullptr, trans);
    });
}

mt_status mt_propagate(const mt_system_conf* conf, const mt_input_multislice* in, int space, double z,
                       double* psi_out) {
    return guarded([&] {
        mt_system_conf c = conf ? *conf : default_conf();
        mtb::propagate_wave(&c, in, space, z, psi_out);
    });
}

mt_status mt_incident_wave(const mt_system_conf* conf, const mt_input_multislice* in, int space, double* psi_out) {
    return guarded([&] {
        if (!psi_out) mtb::fail(MT_ERR_INVALID_ARG, "psi_out is NULL");
        mt_system_conf c = conf ? *conf : default_conf();
        mtb::Engine e(&c, in);
        e.incident_wave(space, psi_out);
    });
}

mt_status mt_spline_tables(const mt_system_conf* conf, const int* Z, int n, double dR_min, double Vrl, int nR,
                           double* heads, float* tab) {
    return mt_spline_tables_ex(conf, 6, Z, nullptr, n, dR_min, Vrl, nR, heads, tab);
}

mt_status mt_spline_tables_ex(const mt_system_conf* conf, int potential_type, const int* Z, const int* charge, int n,
                              double dR_min, double Vrl, int nR, double* heads, float* tab) {
    return guarded([&] {
        if (!Z || n <= 0 || !tab || nR < 2) mtb::fail(MT_ERR_INVALID_ARG, "bad arguments");
        if (!mtb::potential_type_supported(potential_type))
            mtb::fail(MT_ERR_UNSUPPORTED, "potential_type must be 1-4 or 6");
        for (int i = 0; i < n; i++)
            if (Z[i] < 1 || Z[i] > 103) mtb::fail(MT_ERR_INVALID_ARG, "Z out of range 1..103");
        const int dev = conf ? conf->gpu_device : 0;
        MTB_CUDA(cudaSetDevice(dev));
        cudaStream_t s;
        MTB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        std::vector<int> zs(Z, Z + n);
        std::vector<mtb::TableHead> hd;
        for (int z : zs) hd.push_back(mtb::element_head(z, potential_type, (float)dR_min, (float)Vrl));
        mtb::DevBuf<float> d_tab;
        d_tab.alloc((size_t)n * 5 * nR);
        std::vector<int> qs;
        if (charge) qs.assign(charge, charge + n);
        mtb::build_tables(zs, potential_type, hd, nR, d_tab.p, s, qs);
        MTB_CUDA(cudaMemcpyAsync(tab, d_tab.p, sizeof(float) * (size_t)n * 5 * nR, cudaMemcpyDeviceToHost, s));
        MTB_CUDA(cudaStreamSynchronize(s));
        MTB_CUDA(cudaStreamDestroy(s));
        if (heads)
            for (int i = 0; i < n; i++) {
                heads[4 * i] = hd[i].R_min;
                heads[4 * i + 1] = hd[i].R_max;
                heads[4 * i + 2] = hd[i].R_tap;
                heads[4 * i + 3] = hd[i].tap_cf;
            }
    });
}

mt_status mt_spline_tables_noalloc(const int* Z, int n, double dR_min, double Vrl, int nR, double* heads,
                                   float* d_tab, void* stream) {
    return mt_spline_tables_noalloc_ex(6, Z, nullptr, n, dR_min, Vrl, nR, heads, d_tab, stream);
}

mt_status mt_spline_tables_noalloc_ex(int potential_type, const int* Z, const int* charge, int n, double dR_min,
                                      double Vrl, int nR, double* heads, float* d_tab, void* stream) {
    return guarded([&] {
        if (!mtb::potential_type_supported(potential_type))
            mtb::fail(MT_ERR_UNSUPPORTED, "potential_type must be 1-4 or 6");
        if (!Z || !d_tab) mtb::fail(MT_ERR_INVALID_ARG, "Z and d_tab must not be NULL");
        if (n < 1) mtb::fail(MT_ERR_INVALID_ARG, "n must be positive");
        for (int i = 0; i < n; i++)
            if (Z[i] < 1 || Z[i] > 103) mtb::fail(MT_ERR_INVALID_ARG, "Z out of range 1..103");
        std::vector<int> zs(Z, Z + n);
        std::vector<mtb::TableHead> hd;
        for (int z : zs) hd.push_back(mtb::element_head(z, potential_type, (float)dR_min, (float)Vrl));
        std::vector<int> qs;
        if (charge) qs.assign(charge, charge + n);
        mtb::build_tables_noalloc(zs, potential_type, hd, nR, d_tab, static_cast<cudaStream_t>(stream), qs);
        if (heads)
            for (int i = 0; i < n; i++) {
                heads[4 * i] = hd[i].R_min;
                heads[4 * i + 1] = hd[i].R_max;
                heads[4 * i + 2] = hd[i].R_tap;
                heads[4 * i + 3] = hd[i].tap_cf;
            }
    });
}

// Host-only parity helpers: no GPU needed.
namespace {
struct HostSpec {
    mtb::Model m;
    std::unique_ptr<mtb::Specimen> spec;
    explicit HostSpec(const mt_input_multislice* in) : m(mtb::build_model(in)) {
        std::vector<float> rmax(103, 0.0f);
        for (int Zr : m.atoms_in.Z) {
            int Z = Zr % 1000;
            if (rmax[Z - 1] == 0.0f)
                rmax[Z - 1] = (float)mtb::element_head(Z, m.potential_type, m.grid.dR_min(), m.Vrl).R_max;
        }
        spec.reset(new mtb::Specimen(m, rmax));
    }
};
}  // namespace

mt_status mt_specimen_info(const mt_input_multislice* in, int iconf, int* n_atoms, int* n_slice, int* n_thick) {
    return guarded([&] {
        HostSpec h(in);
        h.spec->move_atoms(iconf);
        if (n_atoms) *n_atoms = (int)h.spec->atoms().size();
        if (n_slice) *n_slice = (int)h.spec->slices().size();
        if (n_thick) *n_thick = (int)h.spec->thicks().size();
    });
}

mt_status mt_specimen_atoms(const mt_input_multislice* in, int iconf, int* Z, double* xyz, int n) {
    return guarded([&] {
        HostSpec h(in);
        h.spec->move_atoms(iconf);
        const auto& A = h.spec->atoms();
        if (n < (int)A.size()) mtb::fail(MT_ERR_INVALID_ARG, "buffer too small");
        for (size_t i = 0; i < A.size(); i++) {
            Z[i] = A.Z[i];
            xyz[3 * i] = A.x[i];
            xyz[3 * i + 1] = A.y[i];
            xyz[3 * i + 2] = A.z[i];
        }
    });
}

mt_status mt_phonon_atoms(const mt_system_conf* conf, const mt_input_multislice* in, int iconf, int* Z, double* xyz,
                          int n) {
    return guarded([&] {
        HostSpec h(in);
        if (!(h.m.pn_rng == 1 && h.m.is_frozen_phonon())) {
            h.spec->move_atoms(iconf);
        } else {
            h.spec->still_atoms();
        }
        const auto& A = h.spec->atoms();
        if (n < (int)A.size()) mtb::fail(MT_ERR_INVALID_ARG, "buffer too small");
        std::vector<float> x(A.x), y(A.y);
        if (h.m.pn_rng == 1 && h.m.is_frozen_phonon() && A.size()) {
            if (iconf < 1 || iconf > h.m.pn_nconf) mtb::fail(MT_ERR_INVALID_ARG, "iconf out of range 1..pn_nconf");
            MTB_CUDA(cudaSetDevice(conf ? conf->gpu_device : 0));
            cudaStream_t s;
            MTB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
            std::vector<float4> base(A.size());
            for (size_t i = 0; i < A.size(); i++) base[i] = make_float4(A.x[i], A.y[i], A.occ[i], 0.0f);
            mtb::DevBuf<float4> d_base, d_out;
            mtb::DevBuf<float> d_sigma;
            d_base.upload(base.data(), base.size(), s);
            d_sigma.upload(A.sigma.data(), A.size(), s);
            d_out.alloc(A.size());
            mtb::launch_phonon_displace(d_base.p, d_sigma.p, (int)A.size(), (uint32_t)h.m.pn_seed, iconf, h.m.pn_x,
                                        h.m.pn_y, d_out.p, s);
            MTB_CUDA(cudaMemcpyAsync(base.data(), d_out.p, sizeof(float4) * A.size(), cudaMemcpyDeviceToHost, s));
            MTB_CUDA(cudaStreamSynchronize(s));
            MTB_CUDA(cudaStreamDestroy(s));
            for (size_t i = 0; i < A.size(); i++) {
                x[i] = base[i].x;
                y[i] = base[i].y;
            }
        }
        for (size_t i = 0; i < A.size(); i++) {
            Z[i] = A.Z[i];
            xyz[3 * i] = x[i];
            xyz[3 * i + 1] = y[i];
            xyz[3 * i + 2] = A.z[i];
        }
    });
}

mt_status mt_philox4x32_10(const unsigned* ctr, const unsigned* key, int n, unsigned* out) {
    return guarded([&] {
        if (n < 1 || !ctr || !key || !out) mtb::fail(MT_ERR_INVALID_ARG, "bad arguments");
        cudaStream_t s;
        MTB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        mtb::DevBuf<uint4> d_ctr, d_out;
        mtb::DevBuf<uint2> d_key;
        d_ctr.upload(reinterpret_cast<const uint4*>(ctr), n, s);
        d_key.upload(reinterpret_cast<const uint2*>(key), n, s);
        d_out.alloc(n);
        mtb::launch_philox(d_ctr.p, d_key.p, n, d_out.p, s);
        MTB_CUDA(cudaMemcpyAsync(out, d_out.p, sizeof(uint4) * n, cudaMemcpyDeviceToHost, s));
        MTB_CUDA(cudaStreamSynchronize(s));
        MTB_CUDA(cudaStreamDestroy(s));
    });
}

mt_status mt_specimen_slices(const mt_input_multislice* in, int iconf, double* z_0, double* z_e, int* iatom_0,
                             int* iatom_e, int* ithk, int n) {
    return guarded([&] {
        HostSpec h(in);
        if (h.m.pn_rng == 1 && h.m.is_frozen_phonon())
            h.spec->still_atoms();  // the slicing every device-generated configuration uses
        else
            h.spec->move_atoms(iconf);
        const auto& S = h.spec->slices();
        if (n < (int)S.size()) mtb::fail(MT_ERR_INVALID_ARG, "buffer too small");
        for (size_t i = 0; i < S.size(); i++) {
            z_0[i] = S[i].z_0;
            z_e[i] = S[i].z_e;
            iatom_0[i] = S[i].iatom_0;
            iatom_e[i] = S[i].iatom_e;
            ithk[i] = S[i].ithk;
        }
    });
}

}  // extern "C"
