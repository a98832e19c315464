// FFTW-API shim for building the reference's CPU path (test/baseline infrastructure only).
//
// The reference's host FFT wrapper (src/fft.cuh:37-361, classes FFT<float,e_host> and
// FFT<double,e_host>) calls the public FFTW 3 C API: fftw(f)_plan_dft_1d/2d, fftw(f)_plan_many_dft,
// fftw(f)_execute_dft, fftw(f)_destroy_plan, fftw(f)_plan_with_nthreads, fftw(f)_init_threads,
// fftw(f)_cleanup_threads and the wisdom import/export calls. FFTW itself is not installed in this
// image, so this file provides those entry points with its own implementation:
//
//   * 1-D transforms: iterative Stockham autosort FFT, radices 4/2/3/5 and a direct DFT for any
//     remaining prime factor; twiddles computed in double and rounded once to the working type;
//     unnormalised in both directions, sign convention exp(sign * 2*pi*i*j*k/n) as in FFTW.
//   * 2-D/batched transforms: rows (contiguous) then columns (gathered in blocks of 16 into a
//     contiguous scratch buffer), each split over plan_with_nthreads threads of one persistent
//     worker pool (started on first use, as FFTW's threads are, rather than per execute).
//
// Wisdom calls are accepted and do nothing. Nothing in the product links this file; it exists
// only so that oracle/_ref can be compiled from the reference sources.
#include <cmath>
#include <complex>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>
#include <algorithm>

namespace {

int g_nthreads = 1;

// Persistent workers: run(n, f) calls f(0) on the caller and f(1..n-1) on workers, and returns when
// all are done. One parallel region at a time (callers from several threads take turns).
class Pool {
public:
    void run(int n, const std::function<void(int)>& f) {
        std::lock_guard<std::mutex> call(call_mu_);
        {
            std::lock_guard<std::mutex> lk(mu_);
            while ((int)th_.size() < n - 1) {
                const int id = (int)th_.size() + 1;
                th_.emplace_back([this, id] { loop(id); });
            }
            task_ = &f;
            active_ = n;
            pending_ = n - 1;
            ++gen_;
        }
        start_.notify_all();
        f(0);
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [&] { return pending_ == 0; });
        task_ = nullptr;
    }

private:
    void loop(int id) {
        unsigned long seen = 0;
        for (;;) {
            const std::function<void(int)>* t = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu_);
                start_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
                if (id >= active_) continue;
                t = task_;
            }
            (*t)(id);
            std::lock_guard<std::mutex> lk(mu_);
            if (--pending_ == 0) done_.notify_one();
        }
    }
    std::mutex call_mu_, mu_;
    std::condition_variable start_, done_;
    std::vector<std::thread> th_;
    const std::function<void(int)>* task_ = nullptr;
    int active_ = 0, pending_ = 0;
    unsigned long gen_ = 0;
};

// never destroyed: the workers live until the process exits, like FFTW's
Pool& pool() {
    static Pool* p = new Pool();
    return *p;
}

template <class T>
struct Fft1d {
    using C = std::complex<T>;
    int n = 0;
    std::vector<int> radices;
    std::vector<std::vector<C>> twiddles;  // per stage: (R-1) * (n/R) entries
    std::vector<C> prime_w;                // for a direct-DFT stage of prime order

    explicit Fft1d(int n_) : n(n_) {
        int m = n;
        while (m % 4 == 0) { radices.push_back(4); m /= 4; }
        while (m % 2 == 0) { radices.push_back(2); m /= 2; }
        while (m % 3 == 0) { radices.push_back(3); m /= 3; }
        while (m % 5 == 0) { radices.push_back(5); m /= 5; }
        for (int p = 7; m > 1; p += 2) {
            while (m % p == 0) { radices.push_back(p); m /= p; }
        }
        // Stockham stage s with radix R and Ns = product of the earlier radices:
        //   for j in [0, n/R): k = j % Ns, v_r = x[j + r*n/R] * w^{r*k}, DFT_R(v),
        //   y[(j/Ns)*Ns*R + k + r*Ns] = v_r, with w = exp(-2*pi*i/(Ns*R)).
        int Ns = 1;
        for (int R : radices) {
            std::vector<C> tw((size_t)(R - 1) * Ns);
            for (int k = 0; k < Ns; ++k)
                for (int r = 1; r < R; ++r) {
                    double a = -2.0 * M_PI * (double)(r * k) / (double)(Ns * R);
                    tw[(size_t)k * (R - 1) + (r - 1)] = C((T)std::cos(a), (T)std::sin(a));
                }
            twiddles.push_back(std::move(tw));
            Ns *= R;
        }
    }

    // sign = -1 forward, +1 backward. Output returned in `x`; `work` has n entries.
    void run(C* x, C* work, int sign) const {
        if (n == 1) return;
        C* a = x;
        C* b = work;
        int Ns = 1;
        const int nstage = (int)radices.size();
        for (int s = 0; s < nstage; ++s) {
            const int R = radices[s];
            const int L = n / R;
            const C* tw = twiddles[s].data();
            for (int j = 0; j < L; ++j) {
                const int k = j % Ns;
                C v[64];
                C vv[64];
                for (int r = 0; r < R; ++r) {
                    C t = a[j + r * L];
                    if (r > 0 && k > 0) {
                        C w = tw[(size_t)k * (R - 1) + (r - 1)];
                        if (sign > 0) w = std::conj(w);
                        t *= w;
                    }
                    v[r] = t;
                }
                butterfly(R, v, vv, sign);
                const int base = (j / Ns) * Ns * R + k;
                for (int r = 0; r < R; ++r) b[base + r * Ns] = vv[r];
            }
            std::swap(a, b);
            Ns *= R;
        }
        if (a != x) std::memcpy(x, a, sizeof(C) * (size_t)n);
    }

    static void butterfly(int R, const C* v, C* o, int sign) {
        const T s = (T)sign;
        if (R == 2) {
            o[0] = v[0] + v[1];
            o[1] = v[0] - v[1];
        } else if (R == 4) {
            C t0 = v[0] + v[2], t1 = v[0] - v[2];
            C t2 = v[1] + v[3], t3 = v[1] - v[3];
            C jt3(-s * t3.imag(), s * t3.real());  // sign*i*t3
            o[0] = t0 + t2;
            o[2] = t0 - t2;
            o[1] = t1 + jt3;
            o[3] = t1 - jt3;
        } else {
            for (int q = 0; q < R; ++q) {
                C acc(0, 0);
                for (int r = 0; r < R; ++r) {
                    double a = sign * 2.0 * M_PI * (double)((r * q) % R) / (double)R;
                    acc += v[r] * C((T)std::cos(a), (T)std::sin(a));
                }
                o[q] = acc;
            }
        }
    }
};

template <class T>
struct Plan {
    using C = std::complex<T>;
    int rank = 1;
    int n0 = 1, n1 = 1;       // rank 2: n0 slow, n1 fast (row-major)
    int howmany = 1, idist = 0;
    int sign = -1;
    int nthreads = 1;
    Fft1d<T>* f0 = nullptr;   // length n0
    Fft1d<T>* f1 = nullptr;   // length n1

    ~Plan() {
        delete f1;
        if (f0 != f1) delete f0;
    }

    void exec(C* data) const {
        for (int h = 0; h < howmany; ++h) exec_one(data + (size_t)h * idist);
    }

    template <class F>
    void parallel(int count, F fn) const {
        int nt = std::max(1, std::min(nthreads, count));
        if (nt == 1) { fn(0, count); return; }
        const int chunk = (count + nt - 1) / nt;
        pool().run(nt, [&](int t) {
            const int b = t * chunk, e = std::min(count, b + chunk);
            if (b < e) fn(b, e);
        });
    }

    void exec_one(C* d) const {
        if (rank == 1) {
            std::vector<C> w(n1);
            f1->run(d, w.data(), sign);
            return;
        }
        // rows: n0 contiguous lines of length n1
        parallel(n0, [&](int b, int e) {
            std::vector<C> w(n1);
            for (int i = b; i < e; ++i) f1->run(d + (size_t)i * n1, w.data(), sign);
        });
        // columns: n1 strided lines of length n0, gathered 16 at a time
        const int BW = 16;
        int nblk = (n1 + BW - 1) / BW;
        parallel(nblk, [&](int b, int e) {
            std::vector<C> buf((size_t)BW * n0), w(n0);
            for (int blk = b; blk < e; ++blk) {
                int c0 = blk * BW, cw = std::min(BW, n1 - c0);
                for (int i = 0; i < n0; ++i)
                    for (int c = 0; c < cw; ++c) buf[(size_t)c * n0 + i] = d[(size_t)i * n1 + c0 + c];
                for (int c = 0; c < cw; ++c) f0->run(buf.data() + (size_t)c * n0, w.data(), sign);
                for (int i = 0; i < n0; ++i)
                    for (int c = 0; c < cw; ++c) d[(size_t)i * n1 + c0 + c] = buf[(size_t)c * n0 + i];
            }
        });
    }
};

template <class T>
Plan<T>* make_plan(int rank, const int* n, int howmany, int idist, int sign) {
    auto* p = new Plan<T>();
    p->rank = rank;
    p->sign = sign;
    p->nthreads = g_nthreads;
    p->howmany = std::max(1, howmany);
    if (rank == 1) {
        p->n1 = n[0];
        p->f1 = new Fft1d<T>(n[0]);
        p->idist = idist ? idist : n[0];
    } else {
        p->n0 = n[0];
        p->n1 = n[1];
        p->f1 = new Fft1d<T>(n[1]);
        p->f0 = (n[0] == n[1]) ? p->f1 : new Fft1d<T>(n[0]);
        p->idist = idist ? idist : n[0] * n[1];
    }
    return p;
}

}  // namespace

extern "C" {

typedef double fftw_complex[2];
typedef float fftwf_complex[2];
typedef void* fftw_plan;
typedef void* fftwf_plan;

// ---- double precision ----
int fftw_init_threads(void) { return 1; }
void fftw_cleanup_threads(void) {}
void fftw_plan_with_nthreads(int n) { g_nthreads = std::max(1, n); }
int fftw_import_wisdom_from_filename(const char*) { return 0; }
int fftw_export_wisdom_to_filename(const char*) { return 1; }

fftw_plan fftw_plan_dft_1d(int n, fftw_complex*, fftw_complex*, int sign, unsigned) {
    return make_plan<double>(1, &n, 1, 0, sign);
}
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex*, fftw_complex*, int sign, unsigned) {
    int n[2] = {n0, n1};
    return make_plan<double>(2, n, 1, 0, sign);
}
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex*, const int*, int, int idist,
                             fftw_complex*, const int*, int, int, int sign, unsigned) {
    return make_plan<double>(rank, n, howmany, idist, sign);
}
void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out) {
    auto* pl = static_cast<Plan<double>*>(p);
    size_t total = (size_t)pl->howmany * pl->idist;
    if (in != out) std::memcpy(out, in, sizeof(fftw_complex) * total);
    pl->exec(reinterpret_cast<std::complex<double>*>(out));
}
void fftw_destroy_plan(fftw_plan p) { delete static_cast<Plan<double>*>(p); }

// ---- single precision ----
int fftwf_init_threads(void) { return 1; }
void fftwf_cleanup_threads(void) {}
void fftwf_plan_with_nthreads(int n) { g_nthreads = std::max(1, n); }
int fftwf_import_wisdom_from_filename(const char*) { return 0; }
int fftwf_export_wisdom_to_filename(const char*) { return 1; }

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex*, fftwf_complex*, int sign, unsigned) {
    return make_plan<float>(1, &n, 1, 0, sign);
}
fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex*, fftwf_complex*, int sign, unsigned) {
    int n[2] = {n0, n1};
    return make_plan<float>(2, n, 1, 0, sign);
}
fftwf_plan fftwf_plan_many_dft(int rank, const int* n, int howmany, fftwf_complex*, const int*, int, int idist,
                               fftwf_complex*, const int*, int, int, int sign, unsigned) {
    return make_plan<float>(rank, n, howmany, idist, sign);
}
void fftwf_execute_dft(const fftwf_plan p, fftwf_complex* in, fftwf_complex* out) {
    auto* pl = static_cast<Plan<float>*>(p);
    size_t total = (size_t)pl->howmany * pl->idist;
    if (in != out) std::memcpy(out, in, sizeof(fftwf_complex) * total);
    pl->exec(reinterpret_cast<std::complex<float>*>(out));
}
void fftwf_destroy_plan(fftwf_plan p) { delete static_cast<Plan<float>*>(p); }

}  // extern "C"
