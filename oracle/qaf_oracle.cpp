// qaf_oracle.cpp — FP64 host oracle (test infrastructure; see qaf_oracle.h).
// Every routine cites the reference lines it restates. Compiled with
// -ffp-contract=off so that no FMA contraction changes the rounding between
// builds of the oracle. Row and column loops of the 2D transforms run on
// std::threads (QAF_ORACLE_THREADS, default: all hardware threads); each
// row/column is computed identically whatever the thread count.

#include "qaf_oracle.h"
#include "qaf_init.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <cstdlib>
#include <algorithm>
#include <condition_variable>
#include <functional>
#include <vector>

namespace {

using cplx = std::complex<double>;

int oracle_threads() {
    static int n = [] {
        const char* e = std::getenv("QAF_ORACLE_THREADS");
        int v = e ? std::atoi(e) : (int)std::thread::hardware_concurrency();
        return v < 1 ? 1 : v;
    }();
    return n;
}

// A fixed pool of worker threads; parallel_for(count, body) runs body(lo, hi)
// on contiguous chunks of [0, count) and returns when all chunks are done.
class Pool {
  public:
    static Pool& get() { static Pool p(oracle_threads()); return p; }
    template <class F>
    void run(int count, F& body) {
        int nt = std::min(nthreads_, count);
        if (nt <= 1) { body(0, count); return; }
        std::unique_lock<std::mutex> lk(mu_);
        job_ = [&body](int lo, int hi) { body(lo, hi); };
        count_ = count; chunks_ = nt; next_ = 0; done_ = 0; ++gen_;
        cv_.notify_all();
        lk.unlock();
        work();
        lk.lock();
        done_cv_.wait(lk, [&] { return done_ == chunks_; });
        job_ = nullptr;
    }
    ~Pool() {
        { std::lock_guard<std::mutex> g(mu_); stop_ = true; ++gen_; }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }

  private:
    explicit Pool(int n) : nthreads_(n) {
        for (int t = 1; t < n; ++t) th_.emplace_back([this] { loop(); });
    }
    void work() {
        for (;;) {
            int c;
            { std::lock_guard<std::mutex> g(mu_); if (next_ >= chunks_) return; c = next_++; }
            int chunk = (count_ + chunks_ - 1) / chunks_;
            int lo = c * chunk, hi = std::min(count_, lo + chunk);
            if (lo < hi) job_(lo, hi);
            { std::lock_guard<std::mutex> g(mu_); if (++done_ == chunks_) done_cv_.notify_all(); }
        }
    }
    void loop() {
        unsigned long long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
                if (stop_) return;
            }
            work();
        }
    }
    int nthreads_;
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    std::function<void(int, int)> job_;
    int count_ = 0, chunks_ = 0, next_ = 0, done_ = 0;
    unsigned long long gen_ = 0;
    bool stop_ = false;
};

template <class F>
void parallel_for(int count, F body) { Pool::get().run(count, body); }

// ---------------------------------------------------------------------------
// 1D mixed-radix FFT: iterative Stockham autosort (out-of-place, ping-pong),
// any length whose prime factors are small. Twiddles W_n^t = exp(-2 pi i t/n)
// from long-double cosl/sinl.
// ---------------------------------------------------------------------------
struct Plan1D {
    int n;
    std::vector<int> factors;
    std::vector<cplx> tw;  // tw[t] = exp(-2 pi i t / n)
    explicit Plan1D(int n_) : n(n_) {
        int m = n;
        for (int r : {4, 2, 3, 5, 7}) while (m % r == 0) { factors.push_back(r); m /= r; }
        for (int r = 11; m > 1; r += 2) while (m % r == 0) { factors.push_back(r); m /= r; }
        tw.resize(n);
        const long double pi = 3.141592653589793238462643383279502884L;
        for (int t = 0; t < n; ++t) {
            long double a = -2.0L * pi * (long double)t / (long double)n;
            tw[t] = cplx((double)cosl(a), (double)sinl(a));
        }
    }
};

const Plan1D& plan_for(int n) {
    static std::mutex mu;
    static std::map<int, std::unique_ptr<Plan1D>> cache;
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find(n);
    if (it == cache.end()) it = cache.emplace(n, std::make_unique<Plan1D>(n)).first;
    return *it->second;
}

// Stockham pass with radix R: for L = product of the radices already applied
// and m = n / (L R), input element x[(q m + j) L + k]... written out below as
//   y[(j R + r) L + k] = sum_q x[(q m + j) L + k] * W_{R}^{q r} * W_{L R}^{q k}
// (decimation in frequency form with the twiddle applied on the way out).
void stockham(const cplx* x, cplx* y, cplx* work, int n, bool inverse) {
    const Plan1D& p = plan_for(n);
    const cplx* src = x;
    cplx* bufs[2] = {y, work};
    int which = (p.factors.size() % 2 == 0) ? 1 : 0;  // so that the last pass lands in y
    int L = 1;
    for (size_t f = 0; f < p.factors.size(); ++f) {
        const int R = p.factors[f];
        const int m = n / (L * R);
        cplx* dst = bufs[which];
        cplx abuf[16];
        std::vector<cplx> av;
        cplx* a = abuf;
        if (R > 16) { av.resize(R); a = av.data(); }
        // the R x R DFT matrix of this pass, W_R^{q r} = W_n^{(q r mod R) n/R}
        cplx dft[16 * 16];
        std::vector<cplx> dftv;
        cplx* D = dft;
        if (R > 16) { dftv.resize((size_t)R * R); D = dftv.data(); }
        for (int q = 0; q < R; ++q)
            for (int r = 0; r < R; ++r) {
                cplx w = p.tw[(size_t)(q * r % R) * (n / R)];
                D[q * R + r] = inverse ? std::conj(w) : w;
            }
        // pass: sub-transforms of length L*R built from R interleaved ones of length L
        for (int j = 0; j < m; ++j)
            for (int k = 0; k < L; ++k) {
                for (int q = 0; q < R; ++q) {
                    cplx v = src[(size_t)(j + q * m) * L + k];
                    // twiddle W_{L R}^{q k} = W_n^{q k m}; q k m < R L m = n
                    cplx w = p.tw[(size_t)q * k * m];
                    a[q] = v * (inverse ? std::conj(w) : w);
                }
                for (int r = 0; r < R; ++r) {
                    cplx s = a[0];
                    for (int q = 1; q < R; ++q) s += a[q] * D[q * R + r];
                    dst[(size_t)(j * L) * R + r * L + k] = s;
                }
            }
        src = dst;
        which ^= 1;
        L *= R;
    }
    if (p.factors.empty()) y[0] = x[0];
}

// unnormalised forward (inverse=false: e^{-i}) or backward (e^{+i}) DFT, out-of-place
void fft1d(const cplx* x, cplx* y, int n, bool inverse) {
    thread_local std::vector<cplx> work;
    if ((int)work.size() < n) work.resize(n);
    stockham(x, y, work.data(), n, inverse);
}

// ---------------------------------------------------------------------------
// 2D transforms in the reference's layouts.
// ---------------------------------------------------------------------------
// R2C (cufftExecD2Z, QFldfuncs.cuh:45-48): row R2C along x, then column C2C along y.
void fwd2d(int nx, int ny, const double* phys, cplx* spec) {
    const int nxh = nx / 2 + 1;
    parallel_for(ny, [&](int lo, int hi) {
        std::vector<cplx> a(nx), b(nx);
        for (int j = lo; j < hi; ++j) {
            for (int i = 0; i < nx; ++i) a[i] = cplx(phys[i + (size_t)j * nx], 0.0);
            fft1d(a.data(), b.data(), nx, false);
            for (int i = 0; i < nxh; ++i) spec[i + (size_t)j * nxh] = b[i];
        }
    });
    parallel_for(nxh, [&](int lo, int hi) {
        std::vector<cplx> a(ny), b(ny);
        for (int i = lo; i < hi; ++i) {
            for (int j = 0; j < ny; ++j) a[j] = spec[i + (size_t)j * nxh];
            fft1d(a.data(), b.data(), ny, false);
            for (int j = 0; j < ny; ++j) spec[i + (size_t)j * nxh] = b[j];
        }
    });
}

// C2R (cufftExecZ2D + coeff, QFldfuncs.cuh:50-55 and :8-16): column C2C along
// y, then a row C2R that takes the real parts of the DC and Nyquist terms, then
// the 1/(nx ny) scaling of coeff.
void bwd2d(int nx, int ny, const cplx* spec, double* phys) {
    const int nxh = nx / 2 + 1;
    std::vector<cplx> tmp((size_t)nxh * ny);
    parallel_for(nxh, [&](int lo, int hi) {
        std::vector<cplx> a(ny), b(ny);
        for (int i = lo; i < hi; ++i) {
            for (int j = 0; j < ny; ++j) a[j] = spec[i + (size_t)j * nxh];
            fft1d(a.data(), b.data(), ny, true);
            for (int j = 0; j < ny; ++j) tmp[i + (size_t)j * nxh] = b[j];
        }
    });
    const double scale = 1.0 / ((double)nx * (double)ny);
    parallel_for(ny, [&](int lo, int hi) {
        std::vector<cplx> a(nx), b(nx);
        for (int j = lo; j < hi; ++j) {
            const cplx* row = &tmp[(size_t)j * nxh];
            a[0] = cplx(row[0].real(), 0.0);
            for (int i = 1; i < nxh; ++i) {
                if (2 * i == nx) { a[i] = cplx(row[i].real(), 0.0); continue; }
                a[i] = row[i];
                a[nx - i] = std::conj(row[i]);
            }
            fft1d(a.data(), b.data(), nx, true);
            for (int i = 0; i < nx; ++i) phys[i + (size_t)j * nx] = b[i].real() * scale;
        }
    });
}

// symmetry_func (QFldfuncs.cuh:18-44): for i == 0 and 0 < j < ny/2 replace the
// pair (j, ny-j) by their conjugate-symmetric mean, in place.
void symmetrise(int nx, int ny, cplx* spec) {
    const int nxh = nx / 2 + 1;
    for (int j = 1; j < ny / 2; ++j) {
        cplx& a = spec[(size_t)j * nxh];
        cplx& b = spec[(size_t)(ny - j) * nxh];
        cplx mean = 0.5 * (a + std::conj(b));
        a = mean;
        b = std::conj(mean);
    }
}

// ---------------------------------------------------------------------------
// Mesh tables (Mesh.cuh:6-46).
// ---------------------------------------------------------------------------
struct Mesh {
    int nx, ny, nxh;
    double lx, ly, dx, dy;
    std::vector<double> kx, ky, k2, cutoff;
    explicit Mesh(const oracle_params* p) : nx(p->nx), ny(p->ny), nxh(p->nx / 2 + 1), lx(p->lx), ly(p->ly) {
        dx = lx / nx; dy = ly / ny;
        size_t ns = (size_t)nxh * ny;
        kx.resize(ns); ky.resize(ns); k2.resize(ns); cutoff.resize(ns);
        for (int i = 0; i < nxh; ++i)
            for (int j = 0; j < ny; ++j) {
                size_t idx = i + (size_t)j * nxh;
                ky[idx] = (j < ny / 2 + 1) ? 2 * M_PI / ly * j : 2 * M_PI / ly * (j - ny);
                kx[idx] = 2 * M_PI / lx * i;
                k2[idx] = kx[idx] * kx[idx] + ky[idx] * ky[idx];
                bool keep = (i < (nxh - 1) * 2 / 3 + 1) && ((j < ny / 3 + 1) || ((ny - j) < ny / 3));
                cutoff[idx] = keep ? 1.0 : 0.0;
            }
    }
    size_t ns() const { return (size_t)nxh * ny; }
    size_t np() const { return (size_t)nx * ny; }
};

// A (spectral, physical) pair, as the reference's Field (Mesh.cuh:115-129).
struct Field {
    std::vector<cplx> spec;
    std::vector<double> phys;
    explicit Field(const Mesh& m) : spec(m.ns()), phys(m.np()) {}
};

struct Ctx {
    const oracle_params* p;
    Mesh m;
    explicit Ctx(const oracle_params* p_) : p(p_), m(p_) {}

    void Fwd(std::vector<cplx>& ft, const std::vector<double>& f) { fwd2d(m.nx, m.ny, f.data(), ft.data()); }
    // BwdTrans: transform a copy; symmetrise the caller's buffer in place.
    void Bwd(std::vector<double>& f, std::vector<cplx>& ft) {
        std::vector<cplx> copy = ft;
        if (p->emulate_symmetry) symmetrise(m.nx, m.ny, ft.data());
        bwd2d(m.nx, m.ny, copy.data(), f.data());
    }
    // xDeriv / yDeriv / Laplacian (QFldfuncs.cuh:165-202)
    void xDeriv(std::vector<cplx>& out, const std::vector<cplx>& in) {
        for (size_t k = 0; k < m.ns(); ++k) out[k] = cplx(0, 1) * m.kx[k] * in[k];
    }
    void yDeriv(std::vector<cplx>& out, const std::vector<cplx>& in) {
        for (size_t k = 0; k < m.ns(); ++k) out[k] = cplx(0, 1) * m.ky[k] * in[k];
    }
    void Laplacian(std::vector<cplx>& out, const std::vector<cplx>& in) {
        for (size_t k = 0; k < m.ns(); ++k) out[k] = -1.0 * m.k2[k] * in[k];
    }
    // vel_func (QFldfuncs.cuh:204-224)
    void vel(const std::vector<cplx>& w, std::vector<cplx>& u, std::vector<cplx>& v) {
        for (size_t k = 0; k < m.ns(); ++k) {
            if (k == 0) { u[k] = 0; v[k] = 0; continue; }
            u[k] = m.ky[k] * cplx(0, 1) * w[k] / m.k2[k];
            v[k] = -1.0 * m.kx[k] * cplx(0, 1) * w[k] / m.k2[k];
        }
    }
};

// ---------------------------------------------------------------------------
// Nonlinear terms (friction/Qsolver.cuh:63-312).
// ---------------------------------------------------------------------------
struct Work {
    Field wcurr, r1curr, r2curr, u, v, S, p11, p12, p21, aux, aux1, wnonl, r1nonl, r2nonl;
    std::vector<double> Ra;
    explicit Work(const Mesh& m)
        : wcurr(m), r1curr(m), r2curr(m), u(m), v(m), S(m), p11(m), p12(m), p21(m), aux(m), aux1(m),
          wnonl(m), r1nonl(m), r2nonl(m), Ra(m.np()) {}
};

// curr_func (Qsolver.cuh:302-312)
void curr_func(Ctx& c, Work& W) {
    c.Bwd(W.r1curr.phys, W.r1curr.spec);
    c.Bwd(W.r2curr.phys, W.r2curr.spec);
    c.Bwd(W.wcurr.phys, W.wcurr.spec);
    for (size_t k = 0; k < c.m.np(); ++k)   // S_func :63-71
        W.S.phys[k] = 2 * std::sqrt(W.r1curr.phys[k] * W.r1curr.phys[k] + W.r2curr.phys[k] * W.r2curr.phys[k]);
    c.vel(W.wcurr.spec, W.u.spec, W.v.spec);
    c.Bwd(W.u.phys, W.u.spec);
    c.Bwd(W.v.phys, W.v.spec);
}

// single (:95-105): s0 = -lambda S Lap(r) + lambda S (S^2-1) r
void single(Ctx& c, Field& s0, Field& r, const Field& S, double lambda) {
    c.Laplacian(s0.spec, r.spec);
    c.Bwd(s0.phys, s0.spec);
    for (size_t k = 0; k < c.m.np(); ++k) s0.phys[k] = -1.0 * lambda * s0.phys[k] * S.phys[k];
    for (size_t k = 0; k < c.m.np(); ++k)
        s0.phys[k] = s0.phys[k] + lambda * S.phys[k] * (S.phys[k] * S.phys[k] - 1.0) * r.phys[k];
}

// cross (:107-122): cs = 2 Lap(a) b - 2 a Lap(b)
void cross(Ctx& c, Field& cs, Field& a, Field& b, Field& aux) {
    c.Laplacian(cs.spec, a.spec);
    c.Bwd(cs.phys, cs.spec);
    for (size_t k = 0; k < c.m.np(); ++k) cs.phys[k] = 2.0 * cs.phys[k] * b.phys[k];
    c.Laplacian(aux.spec, b.spec);
    c.Bwd(aux.phys, aux.spec);
    for (size_t k = 0; k < c.m.np(); ++k) aux.phys[k] = -2.0 * a.phys[k] * aux.phys[k];
    for (size_t k = 0; k < c.m.np(); ++k) cs.phys[k] = 1.0 * cs.phys[k] + 1.0 * aux.phys[k];
}

void rar(Ctx& c, Field& x, const Field& r, const std::vector<double>& Ra) {   // Rar :75-83
    for (size_t k = 0; k < c.m.np(); ++k) x.phys[k] = x.phys[k] - Ra[k] * r.phys[k];
}

// wnonl_func (:166-201)
void wnonl_func(Ctx& c, Work& W) {
    const double lambda = c.p->lambda;
    const size_t np = c.m.np(), ns = c.m.ns();
    if (c.p->advect_omega) {
        for (size_t k = 0; k < np; ++k) W.wnonl.phys[k] = -1.0 * W.u.phys[k] * W.wcurr.phys[k];
        c.Fwd(W.wnonl.spec, W.wnonl.phys);
        c.xDeriv(W.wnonl.spec, W.wnonl.spec);
        c.Bwd(W.wnonl.phys, W.wnonl.spec);
        for (size_t k = 0; k < np; ++k) W.aux.phys[k] = -1.0 * W.v.phys[k] * W.wcurr.phys[k];
        c.Fwd(W.aux.spec, W.aux.phys);
        c.yDeriv(W.aux.spec, W.aux.spec);
        c.Bwd(W.aux.phys, W.aux.spec);
        for (size_t k = 0; k < np; ++k) W.wnonl.phys[k] = 1.0 * W.wnonl.phys[k] + 1.0 * W.aux.phys[k];
    } else {
        // the advection-free variant sets the physical term to zero (beginning2/Qsolver.cuh)
        for (size_t k = 0; k < np; ++k) W.wnonl.phys[k] = 0.0;
    }
    c.Fwd(W.wnonl.spec, W.wnonl.phys);
    // p11func (:124-131)
    single(c, W.p11, W.r1curr, W.S, lambda);
    rar(c, W.p11, W.r1curr, W.Ra);
    c.Fwd(W.p11.spec, W.p11.phys);
    // p12func (:133-141)
    single(c, W.p12, W.r2curr, W.S, lambda);
    cross(c, W.aux, W.r1curr, W.r2curr, W.aux1);
    for (size_t k = 0; k < np; ++k) W.p12.phys[k] = 1.0 * W.p12.phys[k] + 1.0 * W.aux.phys[k];
    rar(c, W.p12, W.r2curr, W.Ra);
    c.Fwd(W.p12.spec, W.p12.phys);
    // p21func (:143-151)
    single(c, W.p21, W.r2curr, W.S, lambda);
    cross(c, W.aux, W.r2curr, W.r1curr, W.aux1);
    for (size_t k = 0; k < np; ++k) W.p21.phys[k] = 1.0 * W.p21.phys[k] + 1.0 * W.aux.phys[k];
    rar(c, W.p21, W.r2curr, W.Ra);
    c.Fwd(W.p21.spec, W.p21.phys);
    // PiDeriv (:154-164)
    const double ce = 1.0 / (c.p->er * c.p->re);
    for (size_t k = 0; k < ns; ++k) {
        const double kx = c.m.kx[k], ky = c.m.ky[k];
        W.wnonl.spec[k] = W.wnonl.spec[k] + ce * (-1.0 * kx * kx * W.p12.spec[k] + 2.0 * kx * ky * W.p11.spec[k]
                                                  + ky * ky * W.p21.spec[k]);
    }
}

// r1nonl_func (:217-255)
void r1nonl_func(Ctx& c, Work& W) {
    const double lambda = c.p->lambda;
    const size_t np = c.m.np(), ns = c.m.ns();
    for (size_t k = 0; k < np; ++k) W.r1nonl.phys[k] = -1.0 * W.wcurr.phys[k] * W.r2curr.phys[k];
    for (size_t k = 0; k < np; ++k) W.r1nonl.phys[k] = W.r1nonl.phys[k] - W.S.phys[k] * W.S.phys[k] * W.r1curr.phys[k];
    c.Fwd(W.r1nonl.spec, W.r1nonl.phys);
    for (size_t k = 0; k < np; ++k) W.aux.phys[k] = -1.0 * W.u.phys[k] * W.r1curr.phys[k];
    c.Fwd(W.aux.spec, W.aux.phys);
    c.xDeriv(W.aux.spec, W.aux.spec);
    for (size_t k = 0; k < np; ++k) W.aux1.phys[k] = -1.0 * W.v.phys[k] * W.r1curr.phys[k];
    c.Fwd(W.aux1.spec, W.aux1.phys);
    c.yDeriv(W.aux1.spec, W.aux1.spec);
    for (size_t k = 0; k < ns; ++k) W.aux.spec[k] = 1.0 * W.aux.spec[k] + 1.0 * W.aux1.spec[k];
    for (size_t k = 0; k < ns; ++k) W.r1nonl.spec[k] = 1.0 * W.r1nonl.spec[k] + 1.0 * W.aux.spec[k];
    c.xDeriv(W.aux.spec, W.u.spec);
    c.Bwd(W.aux.phys, W.aux.spec);
    for (size_t k = 0; k < np; ++k) W.aux.phys[k] = lambda * W.S.phys[k] * W.aux.phys[k];
    c.Fwd(W.aux.spec, W.aux.phys);
    for (size_t k = 0; k < ns; ++k) W.r1nonl.spec[k] = 1.0 * W.r1nonl.spec[k] + 1.0 * W.aux.spec[k];
}

// r2nonl_func (:257-300)
void r2nonl_func(Ctx& c, Work& W) {
    const double lambda = c.p->lambda;
    const size_t np = c.m.np(), ns = c.m.ns();
    for (size_t k = 0; k < np; ++k) W.r2nonl.phys[k] = 1.0 * W.wcurr.phys[k] * W.r1curr.phys[k];
    for (size_t k = 0; k < np; ++k) W.r2nonl.phys[k] = W.r2nonl.phys[k] - W.S.phys[k] * W.S.phys[k] * W.r2curr.phys[k];
    c.Fwd(W.r2nonl.spec, W.r2nonl.phys);
    for (size_t k = 0; k < np; ++k) W.aux.phys[k] = -1.0 * W.u.phys[k] * W.r2curr.phys[k];
    c.Fwd(W.aux.spec, W.aux.phys);
    c.xDeriv(W.aux.spec, W.aux.spec);
    for (size_t k = 0; k < np; ++k) W.aux1.phys[k] = -1.0 * W.v.phys[k] * W.r2curr.phys[k];
    c.Fwd(W.aux1.spec, W.aux1.phys);
    c.yDeriv(W.aux1.spec, W.aux1.spec);
    for (size_t k = 0; k < ns; ++k) W.aux.spec[k] = 1.0 * W.aux.spec[k] + 1.0 * W.aux1.spec[k];
    for (size_t k = 0; k < ns; ++k) W.r2nonl.spec[k] = 1.0 * W.r2nonl.spec[k] + 1.0 * W.aux.spec[k];
    c.yDeriv(W.aux.spec, W.u.spec);
    c.xDeriv(W.aux1.spec, W.v.spec);
    for (size_t k = 0; k < ns; ++k) W.aux.spec[k] = 1.0 * W.aux.spec[k] + 1.0 * W.aux1.spec[k];
    c.Bwd(W.aux.phys, W.aux.spec);
    for (size_t k = 0; k < np; ++k) W.aux.phys[k] = 0.5 * lambda * W.S.phys[k] * W.aux.phys[k];
    c.Fwd(W.aux.spec, W.aux.phys);
    for (size_t k = 0; k < ns; ++k) W.r2nonl.spec[k] = 1.0 * W.r2nonl.spec[k] + 1.0 * W.aux.spec[k];
}

void all_nonlinear(Ctx& c, Work& W) {
    curr_func(c, W);
    wnonl_func(c, W);
    r1nonl_func(c, W);
    r2nonl_func(c, W);
}

// IF tables (wlin_func / r1lin_func / r2lin_func, Qsolver.cuh:20-54)
void if_tables(const Ctx& c, int which, double dt, std::vector<double>& IF, std::vector<double>& IFh) {
    IF.resize(c.m.ns()); IFh.resize(c.m.ns());
    for (size_t k = 0; k < c.m.ns(); ++k) {
        double a = (which == 0) ? 1.0 / c.p->re * (-1.0 * c.m.k2[k] - c.p->rf) : (-1.0 * c.m.k2[k] + c.p->q_lin);
        IF[k] = std::exp(a * dt);
        IFh[k] = std::exp(a * dt * 0.5);
    }
}

void set_ra(const Ctx& c, Work& W, const double* alpha_field) {
    for (size_t k = 0; k < c.m.np(); ++k) W.Ra[k] = alpha_field ? alpha_field[k] : c.p->alpha;
}

cplx* as_cplx(double* p) { return reinterpret_cast<cplx*>(p); }
const cplx* as_cplx(const double* p) { return reinterpret_cast<const cplx*>(p); }

bool valid(const oracle_params* p) {
    return p && p->nx >= 2 && p->ny >= 2 && p->nx % 2 == 0 && p->lx > 0 && p->ly > 0;
}

} // namespace

// ---------------------------------------------------------------------------
// Tangent-linear model of the nonlinear terms: the derivative of
// all_nonlinear along (dw, dr1, dr2, dRa), operation by operation in the same
// sequence (every transform and multiplier is linear; the products take the
// product rule). W holds the forward evaluation at the same stage input
// (all_nonlinear already run on it); D.{w,r1,r2}curr.spec hold the tangent
// input and D.Ra the tangent activity; the tangent terms land in
// D.{w,r1,r2}nonl.spec.
// ---------------------------------------------------------------------------
void all_nonlinear_tlm(Ctx& c, Work& W, Work& D) {
    const double lambda = c.p->lambda;
    const size_t np = c.m.np(), ns = c.m.ns();
    // forward fields the products need besides W's current ones
    Field L1(c.m), L2(c.m), ux(c.m), sh(c.m), t1(c.m), t2(c.m);
    c.Laplacian(L1.spec, W.r1curr.spec); c.Bwd(L1.phys, L1.spec);
    c.Laplacian(L2.spec, W.r2curr.spec); c.Bwd(L2.phys, L2.spec);
    c.xDeriv(ux.spec, W.u.spec); c.Bwd(ux.phys, ux.spec);
    c.yDeriv(t1.spec, W.u.spec); c.xDeriv(t2.spec, W.v.spec);
    for (size_t k = 0; k < ns; ++k) sh.spec[k] = t1.spec[k] + t2.spec[k];
    c.Bwd(sh.phys, sh.spec);
    const auto& w = W.wcurr.phys; const auto& r1 = W.r1curr.phys; const auto& r2 = W.r2curr.phys;
    const auto& u = W.u.phys; const auto& v = W.v.phys; const auto& S = W.S.phys;
    // tangent curr_func
    c.Bwd(D.r1curr.phys, D.r1curr.spec);
    c.Bwd(D.r2curr.phys, D.r2curr.spec);
    c.Bwd(D.wcurr.phys, D.wcurr.spec);
    for (size_t k = 0; k < np; ++k)
        D.S.phys[k] = S[k] > 0 ? 4.0 * (r1[k] * D.r1curr.phys[k] + r2[k] * D.r2curr.phys[k]) / S[k] : 0.0;
    c.vel(D.wcurr.spec, D.u.spec, D.v.spec);
    c.Bwd(D.u.phys, D.u.spec);
    c.Bwd(D.v.phys, D.v.spec);
    const auto& dw = D.wcurr.phys; const auto& dr1 = D.r1curr.phys; const auto& dr2 = D.r2curr.phys;
    const auto& du = D.u.phys; const auto& dv = D.v.phys; const auto& dS = D.S.phys;
    Field dL1(c.m), dL2(c.m), dux(c.m), dsh(c.m);
    c.Laplacian(dL1.spec, D.r1curr.spec); c.Bwd(dL1.phys, dL1.spec);
    c.Laplacian(dL2.spec, D.r2curr.spec); c.Bwd(dL2.phys, dL2.spec);
    c.xDeriv(dux.spec, D.u.spec); c.Bwd(dux.phys, dux.spec);
    c.yDeriv(t1.spec, D.u.spec); c.xDeriv(t2.spec, D.v.spec);
    for (size_t k = 0; k < ns; ++k) dsh.spec[k] = t1.spec[k] + t2.spec[k];
    c.Bwd(dsh.phys, dsh.spec);

    // wnonl_func
    if (c.p->advect_omega) {
        for (size_t k = 0; k < np; ++k) D.wnonl.phys[k] = -(du[k] * w[k] + u[k] * dw[k]);
        c.Fwd(D.wnonl.spec, D.wnonl.phys);
        c.xDeriv(D.wnonl.spec, D.wnonl.spec);
        c.Bwd(D.wnonl.phys, D.wnonl.spec);
        for (size_t k = 0; k < np; ++k) D.aux.phys[k] = -(dv[k] * w[k] + v[k] * dw[k]);
        c.Fwd(D.aux.spec, D.aux.phys);
        c.yDeriv(D.aux.spec, D.aux.spec);
        c.Bwd(D.aux.phys, D.aux.spec);
        for (size_t k = 0; k < np; ++k) D.wnonl.phys[k] = D.wnonl.phys[k] + D.aux.phys[k];
    } else {
        for (size_t k = 0; k < np; ++k) D.wnonl.phys[k] = 0.0;
    }
    c.Fwd(D.wnonl.spec, D.wnonl.phys);
    // single: -lambda S L + lambda S (S^2 - 1) r; Rar: -Ra r; cross: 2 La b - 2 a Lb
    auto dsingle = [&](size_t k, double L, double dL, double r, double dr) {
        return -lambda * (dS[k] * L + S[k] * dL) + lambda * (3.0 * S[k] * S[k] - 1.0) * dS[k] * r +
               lambda * S[k] * (S[k] * S[k] - 1.0) * dr;
    };
    for (size_t k = 0; k < np; ++k) {
        const double dcross12 = 2.0 * (dL1.phys[k] * r2[k] + L1.phys[k] * dr2[k]) - 2.0 * (dr1[k] * L2.phys[k] + r1[k] * dL2.phys[k]);
        D.p11.phys[k] = dsingle(k, L1.phys[k], dL1.phys[k], r1[k], dr1[k]) - (D.Ra[k] * r1[k] + W.Ra[k] * dr1[k]);
        D.p12.phys[k] = dsingle(k, L2.phys[k], dL2.phys[k], r2[k], dr2[k]) + dcross12 - (D.Ra[k] * r2[k] + W.Ra[k] * dr2[k]);
        D.p21.phys[k] = dsingle(k, L2.phys[k], dL2.phys[k], r2[k], dr2[k]) - dcross12 - (D.Ra[k] * r2[k] + W.Ra[k] * dr2[k]);
    }
    c.Fwd(D.p11.spec, D.p11.phys);
    c.Fwd(D.p12.spec, D.p12.phys);
    c.Fwd(D.p21.spec, D.p21.phys);
    const double ce = 1.0 / (c.p->er * c.p->re);
    for (size_t k = 0; k < ns; ++k) {
        const double kx = c.m.kx[k], ky = c.m.ky[k];
        D.wnonl.spec[k] = D.wnonl.spec[k] + ce * (-1.0 * kx * kx * D.p12.spec[k] + 2.0 * kx * ky * D.p11.spec[k]
                                                  + ky * ky * D.p21.spec[k]);
    }
    // r1nonl_func, r2nonl_func
    for (int f = 0; f < 2; ++f) {
        const auto& ra = f == 0 ? r1 : r2;   // the field advanced
        const auto& dra = f == 0 ? dr1 : dr2;
        Field& out = f == 0 ? D.r1nonl : D.r2nonl;
        for (size_t k = 0; k < np; ++k) {
            const double rot = f == 0 ? -(dw[k] * r2[k] + w[k] * dr2[k]) : (dw[k] * r1[k] + w[k] * dr1[k]);
            out.phys[k] = rot - (2.0 * S[k] * dS[k] * ra[k] + S[k] * S[k] * dra[k]);
        }
        c.Fwd(out.spec, out.phys);
        for (size_t k = 0; k < np; ++k) D.aux.phys[k] = -(du[k] * ra[k] + u[k] * dra[k]);
        c.Fwd(D.aux.spec, D.aux.phys);
        c.xDeriv(D.aux.spec, D.aux.spec);
        for (size_t k = 0; k < np; ++k) D.aux1.phys[k] = -(dv[k] * ra[k] + v[k] * dra[k]);
        c.Fwd(D.aux1.spec, D.aux1.phys);
        c.yDeriv(D.aux1.spec, D.aux1.spec);
        for (size_t k = 0; k < ns; ++k) out.spec[k] = out.spec[k] + (D.aux.spec[k] + D.aux1.spec[k]);
        for (size_t k = 0; k < np; ++k)
            D.aux.phys[k] = f == 0 ? lambda * (dS[k] * ux.phys[k] + S[k] * dux.phys[k])
                                   : 0.5 * lambda * (dS[k] * sh.phys[k] + S[k] * dsh.phys[k]);
        c.Fwd(D.aux.spec, D.aux.phys);
        for (size_t k = 0; k < ns; ++k) out.spec[k] = out.spec[k] + D.aux.spec[k];
    }
}

// enstrophy 0.5 mean(w^2) of a spectral vorticity and its derivative along dw
void enstrophy_tlm(Ctx& c, const cplx* ws, const cplx* dws, double* z, double* dz) {
    const size_t ns = c.m.ns(), np = c.m.np();
    std::vector<cplx> a(ws, ws + ns), b(dws, dws + ns);
    std::vector<double> wp(np), dwp(np);
    bwd2d(c.m.nx, c.m.ny, a.data(), wp.data());
    bwd2d(c.m.nx, c.m.ny, b.data(), dwp.data());
    double s = 0, ds = 0;
    for (size_t k = 0; k < np; ++k) { s += wp[k] * wp[k]; ds += wp[k] * dwp[k]; }
    *z = 0.5 * s / (double)np;
    *dz = ds / (double)np;
}

extern "C" {

int oracle_tables(const oracle_params* p, double* kx, double* ky, double* k2, double* cutoff) {
    if (!valid(p)) return 1;
    Mesh m(p);
    size_t ns = m.ns();
    if (kx) std::memcpy(kx, m.kx.data(), ns * sizeof(double));
    if (ky) std::memcpy(ky, m.ky.data(), ns * sizeof(double));
    if (k2) std::memcpy(k2, m.k2.data(), ns * sizeof(double));
    if (cutoff) std::memcpy(cutoff, m.cutoff.data(), ns * sizeof(double));
    return 0;
}

int oracle_fwd(int nx, int ny, const double* phys, double* spec) {
    if (nx < 2 || ny < 1 || nx % 2) return 1;
    fwd2d(nx, ny, phys, as_cplx(spec));
    return 0;
}

int oracle_bwd(int nx, int ny, const double* spec, double* phys) {
    if (nx < 2 || ny < 1 || nx % 2) return 1;
    bwd2d(nx, ny, as_cplx(spec), phys);
    return 0;
}

int oracle_bwd_mutating(int nx, int ny, double* spec, double* phys) {
    if (nx < 2 || ny < 1 || nx % 2) return 1;
    size_t ns = (size_t)(nx / 2 + 1) * ny;
    std::vector<cplx> copy(as_cplx(spec), as_cplx(spec) + ns);
    symmetrise(nx, ny, as_cplx(spec));
    bwd2d(nx, ny, copy.data(), phys);
    return 0;
}

int oracle_xderiv(const oracle_params* p, const double* in, double* out) {
    if (!valid(p)) return 1;
    Ctx c(p);
    std::vector<cplx> a(as_cplx(in), as_cplx(in) + c.m.ns()), b(c.m.ns());
    c.xDeriv(b, a);
    std::memcpy(out, b.data(), b.size() * sizeof(cplx));
    return 0;
}

int oracle_yderiv(const oracle_params* p, const double* in, double* out) {
    if (!valid(p)) return 1;
    Ctx c(p);
    std::vector<cplx> a(as_cplx(in), as_cplx(in) + c.m.ns()), b(c.m.ns());
    c.yDeriv(b, a);
    std::memcpy(out, b.data(), b.size() * sizeof(cplx));
    return 0;
}

int oracle_laplacian(const oracle_params* p, const double* in, double* out) {
    if (!valid(p)) return 1;
    Ctx c(p);
    std::vector<cplx> a(as_cplx(in), as_cplx(in) + c.m.ns()), b(c.m.ns());
    c.Laplacian(b, a);
    std::memcpy(out, b.data(), b.size() * sizeof(cplx));
    return 0;
}

int oracle_vel(const oracle_params* p, const double* w, double* u, double* v) {
    if (!valid(p)) return 1;
    Ctx c(p);
    std::vector<cplx> a(as_cplx(w), as_cplx(w) + c.m.ns()), uu(c.m.ns()), vv(c.m.ns());
    c.vel(a, uu, vv);
    std::memcpy(u, uu.data(), uu.size() * sizeof(cplx));
    std::memcpy(v, vv.data(), vv.size() * sizeof(cplx));
    return 0;
}

// whether the step truncates field f by the 2/3 mask: all three fields
// (friction.cu:253-255), none (no_dealias 1, couple.cu:179-215) or w only
// (no_dealias 2, dealias/couple.cu:226-229)
static bool truncates(const oracle_params* p, int f) {
    return p->no_dealias == 0 || (p->no_dealias == 2 && f == 0);
}

int oracle_dealias(const oracle_params* p, double* spec) {   // dealias (Qsolver.cuh:314-322)
    if (!valid(p)) return 1;
    Mesh m(p);
    cplx* s = as_cplx(spec);
    for (size_t k = 0; k < m.ns(); ++k) s[k] = s[k] * m.cutoff[k];
    return 0;
}

int oracle_if_tables(const oracle_params* p, int which, double dt, double* IF, double* IFh) {
    if (!valid(p) || (which != 0 && which != 1)) return 1;
    Ctx c(p);
    std::vector<double> a, b;
    if_tables(c, which, dt, a, b);
    if (IF) std::memcpy(IF, a.data(), a.size() * sizeof(double));
    if (IFh) std::memcpy(IFh, b.data(), b.size() * sizeof(double));
    return 0;
}

int oracle_nonlinear(const oracle_params* p, const double* alpha_field, const double* w, const double* r1,
                     const double* r2, double* wn, double* r1n, double* r2n, double* phys_out) {
    if (!valid(p)) return 1;
    Ctx c(p);
    Work W(c.m);
    set_ra(c, W, alpha_field);
    size_t ns = c.m.ns(), np = c.m.np();
    std::memcpy(W.wcurr.spec.data(), w, ns * sizeof(cplx));
    std::memcpy(W.r1curr.spec.data(), r1, ns * sizeof(cplx));
    std::memcpy(W.r2curr.spec.data(), r2, ns * sizeof(cplx));
    all_nonlinear(c, W);
    if (wn) std::memcpy(wn, W.wnonl.spec.data(), ns * sizeof(cplx));
    if (r1n) std::memcpy(r1n, W.r1nonl.spec.data(), ns * sizeof(cplx));
    if (r2n) std::memcpy(r2n, W.r2nonl.spec.data(), ns * sizeof(cplx));
    if (phys_out) {
        const std::vector<double>* f[9] = {&W.wcurr.phys, &W.r1curr.phys, &W.r2curr.phys, &W.u.phys, &W.v.phys,
                                           &W.S.phys, &W.p11.phys, &W.p12.phys, &W.p21.phys};
        for (int q = 0; q < 9; ++q) std::memcpy(phys_out + q * np, f[q]->data(), np * sizeof(double));
    }
    return 0;
}

// Step drivers. RK4 follows friction.cu:212-259 with the stage kernels of
// RK4.cuh:12-74; IF-RK2 uses IFRK2.cuh:16-51 with the full-step factor passed
// as the curr factor (so the second stage sits at t + dt, Lawson-Heun); IF-Euler
// uses IFE.cuh:15-25. Every step ends with dealias of new and old <- new.
int oracle_step(const oracle_params* p, int integrator, const double* alpha_field, double* w, double* r1,
                double* r2, int nsteps) {
    if (!valid(p) || nsteps < 0) return 1;
    if (integrator != ORACLE_IFE && integrator != ORACLE_IFRK2 && integrator != ORACLE_IFRK4) return 1;
    Ctx c(p);
    Work W(c.m);
    set_ra(c, W, alpha_field);
    const size_t ns = c.m.ns();
    const double dt = p->dt;
    std::vector<double> IFw, IFwh, IFq, IFqh;
    if_tables(c, 0, dt, IFw, IFwh);
    if_tables(c, 1, dt, IFq, IFqh);
    cplx* old[3] = {as_cplx(w), as_cplx(r1), as_cplx(r2)};
    std::vector<cplx>* curr[3] = {&W.wcurr.spec, &W.r1curr.spec, &W.r2curr.spec};
    std::vector<cplx>* nonl[3] = {&W.wnonl.spec, &W.r1nonl.spec, &W.r2nonl.spec};
    std::vector<cplx> nw[3] = {std::vector<cplx>(ns), std::vector<cplx>(ns), std::vector<cplx>(ns)};
    const std::vector<double>* E[3] = {&IFw, &IFq, &IFq};
    const std::vector<double>* Eh[3] = {&IFwh, &IFqh, &IFqh};

    for (int s = 0; s < nsteps; ++s) {
        if (integrator == ORACLE_IFRK4) {
            for (int f = 0; f < 3; ++f)   // integrate_func0D
                for (size_t k = 0; k < ns; ++k) { nw[f][k] = old[f][k] * (*E[f])[k]; (*curr[f])[k] = old[f][k]; }
            all_nonlinear(c, W);
            for (int f = 0; f < 3; ++f)   // integrate_func1D
                for (size_t k = 0; k < ns; ++k) {
                    cplx an = (*nonl[f])[k] * dt;
                    nw[f][k] = nw[f][k] + 1.0 / 6.0 * ((*E[f])[k]) * an;
                    (*curr[f])[k] = (old[f][k] + an / 2.0) * ((*Eh[f])[k]);
                }
            all_nonlinear(c, W);
            for (int f = 0; f < 3; ++f)   // integrate_func2D
                for (size_t k = 0; k < ns; ++k) {
                    cplx bn = (*nonl[f])[k] * dt;
                    nw[f][k] = nw[f][k] + 1.0 / 3.0 * (*Eh[f])[k] * bn;
                    (*curr[f])[k] = old[f][k] * ((*Eh[f])[k]) + bn / 2.0;
                }
            all_nonlinear(c, W);
            for (int f = 0; f < 3; ++f)   // integrate_func3D
                for (size_t k = 0; k < ns; ++k) {
                    cplx cn = (*nonl[f])[k] * dt;
                    nw[f][k] = nw[f][k] + 1.0 / 3.0 * (*Eh[f])[k] * cn;
                    (*curr[f])[k] = old[f][k] * (*E[f])[k] + cn * (*Eh[f])[k];
                }
            all_nonlinear(c, W);
            for (int f = 0; f < 3; ++f)   // integrate_func4D
                for (size_t k = 0; k < ns; ++k) {
                    cplx dn = (*nonl[f])[k] * dt;
                    nw[f][k] = nw[f][k] + 1.0 / 6.0 * dn;
                }
        } else if (integrator == ORACLE_IFRK2) {
            for (int f = 0; f < 3; ++f)   // IF::IFRK2::integrate_func0D
                for (size_t k = 0; k < ns; ++k) { nw[f][k] = old[f][k] * (*E[f])[k]; (*curr[f])[k] = old[f][k]; }
            all_nonlinear(c, W);
            for (int f = 0; f < 3; ++f)   // IF::IFRK2::integrate_func1D, curr factor = full step
                for (size_t k = 0; k < ns; ++k) {
                    cplx an = (*nonl[f])[k] * dt;
                    nw[f][k] = nw[f][k] + 1.0 / 2.0 * ((*E[f])[k]) * an;
                    (*curr[f])[k] = (old[f][k] + an) * ((*E[f])[k]);
                }
            all_nonlinear(c, W);
            for (int f = 0; f < 3; ++f)   // IF::IFRK2::integrate_func2D
                for (size_t k = 0; k < ns; ++k) {
                    cplx bn = (*nonl[f])[k] * dt;
                    nw[f][k] = nw[f][k] + 1.0 / 2.0 * bn;
                }
        } else {
            for (int f = 0; f < 3; ++f)
                for (size_t k = 0; k < ns; ++k) (*curr[f])[k] = old[f][k];
            all_nonlinear(c, W);
            for (int f = 0; f < 3; ++f)   // IF::IFE::integrate_func1D
                for (size_t k = 0; k < ns; ++k) {
                    cplx an = (*nonl[f])[k] * dt;
                    nw[f][k] = (old[f][k] + an) * (*E[f])[k];
                }
        }
        for (int f = 0; f < 3; ++f) {     // dealias + SpecSet(old <- new)
            const bool tr = truncates(c.p, f);
            for (size_t k = 0; k < ns; ++k) old[f][k] = tr ? nw[f][k] * c.m.cutoff[k] : nw[f][k];
        }
    }
    return 0;
}

int oracle_diagnostics(const oracle_params* p, const double* w, double* energy, double* enstrophy,
                       double* spectrum, int nshells) {
    if (!valid(p)) return 1;
    Ctx c(p);
    const size_t ns = c.m.ns(), np = c.m.np();
    std::vector<cplx> ws(as_cplx(w), as_cplx(w) + ns), us(ns), vs(ns), wr(ns);
    std::vector<double> wp(np), up(np), vp(np);
    bwd2d(c.m.nx, c.m.ny, ws.data(), wp.data());
    fwd2d(c.m.nx, c.m.ny, wp.data(), wr.data());
    c.vel(wr, us, vs);
    if (energy) {
        bwd2d(c.m.nx, c.m.ny, us.data(), up.data());
        bwd2d(c.m.nx, c.m.ny, vs.data(), vp.data());
        double e = 0;
        for (size_t k = 0; k < np; ++k) e += (up[k] * up[k] + vp[k] * vp[k]) * 0.5 * c.m.dx * c.m.dy;
        *energy = e / (c.m.lx * c.m.ly);
    }
    if (enstrophy) {
        double z = 0;
        for (size_t k = 0; k < np; ++k) z += wp[k] * wp[k];
        *enstrophy = 0.5 * z / (double)np;
    }
    if (spectrum && nshells > 0) {
        // shells [k, k + dk) with k advanced by repeated addition, k += dk, as the
        // post-processor loops (EnergySpec.cu:194-204), so consecutive shells tile
        const double dk = 2 * M_PI / c.m.lx;
        const double norm = 2.0 * dk * (double)c.m.nx * c.m.ny * (double)c.m.nx * c.m.ny;
        double k0 = 0.0;
        for (int s = 0; s < nshells; ++s) {
            double e = 0;
            for (size_t k = 0; k < ns; ++k) {
                double mod = c.m.kx[k] * c.m.kx[k] + c.m.ky[k] * c.m.ky[k];
                if (mod < (k0 + dk) * (k0 + dk) && mod >= k0 * k0) e += std::norm(us[k]) + std::norm(vs[k]);
            }
            spectrum[s] = e / norm;
            k0 += dk;
        }
    }
    return 0;
}

void oracle_random_q_init(unsigned long long seed, int nx, int ny, double lo, double hi, double* w, double* r1,
                          double* r2) {
    qaf_random_q_init(seed, nx, ny, lo, hi, w, r1, r2);
}

void oracle_couple_init(unsigned long long seed, int n, double L, double amp, double* w, double* r1, double* r2) {
    qaf_couple_init(seed, n, n, L, L, amp, w, r1, r2);
}


// IF-RK4 (friction.cu:212-259) advanced together with its tangent-linear model.
int oracle_step_tlm(const oracle_params* p, const double* alpha_field, const double* dalpha_field, double* w,
                    double* r1, double* r2, double* dw, double* dr1, double* dr2, int nsteps, int loss_window,
                    double* loss, double* dloss) {
    if (!valid(p) || nsteps < 0 || loss_window < 0 || loss_window > nsteps) return 1;
    Ctx c(p);
    Work W(c.m), D(c.m);
    set_ra(c, W, alpha_field);
    for (size_t k = 0; k < c.m.np(); ++k) D.Ra[k] = dalpha_field ? dalpha_field[k] : 0.0;
    const size_t ns = c.m.ns();
    const double dt = p->dt;
    std::vector<double> IFw, IFwh, IFq, IFqh;
    if_tables(c, 0, dt, IFw, IFwh);
    if_tables(c, 1, dt, IFq, IFqh);
    cplx* old[3] = {as_cplx(w), as_cplx(r1), as_cplx(r2)};
    cplx* dold[3] = {as_cplx(dw), as_cplx(dr1), as_cplx(dr2)};
    std::vector<cplx>* curr[3] = {&W.wcurr.spec, &W.r1curr.spec, &W.r2curr.spec};
    std::vector<cplx>* dcurr[3] = {&D.wcurr.spec, &D.r1curr.spec, &D.r2curr.spec};
    std::vector<cplx>* nonl[3] = {&W.wnonl.spec, &W.r1nonl.spec, &W.r2nonl.spec};
    std::vector<cplx>* dnonl[3] = {&D.wnonl.spec, &D.r1nonl.spec, &D.r2nonl.spec};
    std::vector<cplx> nw[3] = {std::vector<cplx>(ns), std::vector<cplx>(ns), std::vector<cplx>(ns)};
    std::vector<cplx> dnw[3] = {std::vector<cplx>(ns), std::vector<cplx>(ns), std::vector<cplx>(ns)};
    const std::vector<double>* E[3] = {&IFw, &IFq, &IFq};
    const std::vector<double>* Eh[3] = {&IFwh, &IFqh, &IFqh};
    auto eval = [&]() {
        // the forward's Bwd may symmetrise curr in place; evaluate the tangent on the same inputs
        all_nonlinear(c, W);
        all_nonlinear_tlm(c, W, D);
    };
    double L = 0, dL = 0;
    for (int s = 0; s < nsteps; ++s) {
        for (int f = 0; f < 3; ++f)
            for (size_t k = 0; k < ns; ++k) {
                nw[f][k] = old[f][k] * (*E[f])[k]; (*curr[f])[k] = old[f][k];
                dnw[f][k] = dold[f][k] * (*E[f])[k]; (*dcurr[f])[k] = dold[f][k];
            }
        eval();
        for (int f = 0; f < 3; ++f)
            for (size_t k = 0; k < ns; ++k) {
                cplx an = (*nonl[f])[k] * dt, dan = (*dnonl[f])[k] * dt;
                nw[f][k] = nw[f][k] + 1.0 / 6.0 * ((*E[f])[k]) * an;
                dnw[f][k] = dnw[f][k] + 1.0 / 6.0 * ((*E[f])[k]) * dan;
                (*curr[f])[k] = (old[f][k] + an / 2.0) * ((*Eh[f])[k]);
                (*dcurr[f])[k] = (dold[f][k] + dan / 2.0) * ((*Eh[f])[k]);
            }
        eval();
        for (int f = 0; f < 3; ++f)
            for (size_t k = 0; k < ns; ++k) {
                cplx bn = (*nonl[f])[k] * dt, dbn = (*dnonl[f])[k] * dt;
                nw[f][k] = nw[f][k] + 1.0 / 3.0 * (*Eh[f])[k] * bn;
                dnw[f][k] = dnw[f][k] + 1.0 / 3.0 * (*Eh[f])[k] * dbn;
                (*curr[f])[k] = old[f][k] * ((*Eh[f])[k]) + bn / 2.0;
                (*dcurr[f])[k] = dold[f][k] * ((*Eh[f])[k]) + dbn / 2.0;
            }
        eval();
        for (int f = 0; f < 3; ++f)
            for (size_t k = 0; k < ns; ++k) {
                cplx cn = (*nonl[f])[k] * dt, dcn = (*dnonl[f])[k] * dt;
                nw[f][k] = nw[f][k] + 1.0 / 3.0 * (*Eh[f])[k] * cn;
                dnw[f][k] = dnw[f][k] + 1.0 / 3.0 * (*Eh[f])[k] * dcn;
                (*curr[f])[k] = old[f][k] * (*E[f])[k] + cn * (*Eh[f])[k];
                (*dcurr[f])[k] = dold[f][k] * (*E[f])[k] + dcn * (*Eh[f])[k];
            }
        eval();
        for (int f = 0; f < 3; ++f)
            for (size_t k = 0; k < ns; ++k) {
                cplx dn = (*nonl[f])[k] * dt, ddn = (*dnonl[f])[k] * dt;
                nw[f][k] = nw[f][k] + 1.0 / 6.0 * dn;
                dnw[f][k] = dnw[f][k] + 1.0 / 6.0 * ddn;
            }
        for (int f = 0; f < 3; ++f)
            for (size_t k = 0; k < ns; ++k) {
                const double keep = truncates(c.p, f) ? c.m.cutoff[k] : 1.0;
                old[f][k] = nw[f][k] * keep;
                dold[f][k] = dnw[f][k] * keep;
            }
        if (s >= nsteps - loss_window) {
            double z, dz;
            enstrophy_tlm(c, old[0], dold[0], &z, &dz);
            L += z / loss_window;
            dL += dz / loss_window;
        }
    }
    if (loss) *loss = L;
    if (dloss) *dloss = dL;
    return 0;
}

} // extern "C"
