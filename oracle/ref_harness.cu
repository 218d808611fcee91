// ref_harness.cu — a project-written driver around the reference's UNMODIFIED
// solver headers (InertialFriction/friction/Qsolver.cuh, TimeIntegration/RK4.cuh,
// FldOp/QFldfuncs.cuh, Basic/Mesh.cuh), compiled from where they lie by
// oracle/Makefile into oracle/_ref/. It is test infrastructure: the tests and
// bench.py's reference arm run it to pin the FP64 host oracle and to time the
// reference's own CUDA build on the same GPU. No reference source is copied;
// this file only calls the reference's public functions and kernels, in the
// order of the reference driver InertialFriction/friction/friction.cu:212-259.
//
// Modes (first argument):
//   run        step the coupled (w, r1, r2) system with IF-RK4 and dump the
//              spectral state (reference layout i + j*Nxh) at chosen steps
//   nonlinear  evaluate curr_func + wnonl_func + r1nonl_func + r2nonl_func once
//              on the initial state and dump the three nonlinear spectra
//   time       warm up, then time K steps with CUDA events; print one JSON line
//   probe      feed random non-Hermitian spectra to the reference's BwdTrans
//              and report how its C2R treats the non-Hermitian part
//
// Built twice: FP64 (the reference as shipped) and FP32 (QAF_REF_FP32), the
// latter through the macro shim below, which retargets the reference's
// hard-coded double types and cuFFT D2Z/Z2D calls to float/R2C/C2R without
// editing any reference file.

#ifdef QAF_REF_FP32
#include <cuComplex.h>
#include <cufft.h>
#define __QACTFLOWDEF_CUH
typedef float Qreal;
typedef cuComplex Qcomp;
#include <Basic/cuComplexBinOp.cuh>
#define im imf
#define make_cuDoubleComplex make_cuComplex
#define cuConj cuConjf
#define cufftExecD2Z cufftExecR2C
#define cufftExecZ2D cufftExecC2R
#define CUFFT_D2Z CUFFT_R2C
#define CUFFT_Z2D CUFFT_C2R
#endif

#include "Qsolver.cuh"
#include <TimeIntegration/RK4.cuh>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <vector>
#include <string>
#include <set>
#include <chrono>

#include "qaf_init.h"

namespace {

struct Opts {
    std::string mode = "run";
    int n = 128;               // nx (and ny unless --ny is given)
    int ny = 0;                // 0: the same as n
    double L = 16.0 * M_PI;    // Lx (and Ly unless --Ly is given)
    double Ly = 0;
    double re = 1.0, er = 1.0, rf = 0.1, lambda = 0.1, alpha = 1.0, dt = 1e-3;
    int steps = 10;
    std::set<int> dumps;
    std::string init = "random";
    uint64_t seed = 0;
    std::string out = "ref";
    int warmup = 3, timed = 10;
    int dealias = 1;   // 0: the coupled runs' step, no truncation (couple.cu:179-215);
                       // 2: dealias/couple.cu:226-229's, wnew truncated (three times) and r1, r2 not
};

void die(const char* msg) { std::fprintf(stderr, "ref_harness: %s\n", msg); std::exit(2); }

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) { std::fprintf(stderr, "ref_harness: %s: %s\n", what, cudaGetErrorString(e)); std::exit(3); }
}

Opts parse(int argc, char** argv) {
    Opts o;
    if (argc < 2) die("usage: ref_harness run|nonlinear|time|probe [--key value]...");
    o.mode = argv[1];
    for (int a = 2; a + 1 < argc; a += 2) {
        std::string k = argv[a]; const char* v = argv[a + 1];
        if (k == "--n") o.n = std::atoi(v);
        else if (k == "--ny") o.ny = std::atoi(v);
        else if (k == "--L") o.L = std::atof(v);
        else if (k == "--Ly") o.Ly = std::atof(v);
        else if (k == "--re") o.re = std::atof(v);
        else if (k == "--er") o.er = std::atof(v);
        else if (k == "--rf") o.rf = std::atof(v);
        else if (k == "--lambda") o.lambda = std::atof(v);
        else if (k == "--alpha") o.alpha = std::atof(v);
        else if (k == "--dt") o.dt = std::atof(v);
        else if (k == "--steps") o.steps = std::atoi(v);
        else if (k == "--init") o.init = v;
        else if (k == "--seed") o.seed = std::strtoull(v, nullptr, 10);
        else if (k == "--out") o.out = v;
        else if (k == "--warmup") o.warmup = std::atoi(v);
        else if (k == "--timed") o.timed = std::atoi(v);
        else if (k == "--dealias") o.dealias = std::atoi(v);
        else if (k == "--dumps") {
            std::string s = v; size_t p = 0;
            while (p < s.size()) { size_t q = s.find(',', p); if (q == std::string::npos) q = s.size();
                o.dumps.insert(std::atoi(s.substr(p, q - p).c_str())); p = q + 1; }
        } else die(("unknown option " + k).c_str());
    }
    return o;
}

// Analytic initial fields of the reference's unit tests (UnitTest/Nonlinear/
// nlterms0-4.cu, UnitTest/TimeIntegration/Taylor/Taylor.cu), restated.
void analytic(const std::string& kind, double x, double y, double& w, double& r1, double& r2) {
    if (kind == "kat0") { w = -2 * std::sin(x + y); r1 = std::sin(x); r2 = std::cos(x); }
    else if (kind == "kat1") { w = -2 * std::sin(x + y); r1 = std::cos(x + y); r2 = std::sin(x + y); }
    else if (kind == "kat2") { w = -5 * std::sin(2 * x + y); r1 = std::cos(x + y); r2 = std::sin(x + y); }
    else if (kind == "kat3") { w = -298 * std::sin(17 * x + 3 * y); r1 = std::cos(5 * x + y); r2 = std::sin(5 * x + y); }
    else if (kind == "kat4") { w = -13 * std::sin(2 * x + 3 * y); r1 = std::cos(3 * x + 2 * y); r2 = std::sin(3 * x + 2 * y); }
    else if (kind == "taylor") { w = -2 * std::cos(x) * std::cos(y); r1 = 0; r2 = 0; }
    else die("unknown --init");
}

void make_init(const Opts& o, std::vector<double>& w, std::vector<double>& r1, std::vector<double>& r2) {
    int n = o.n, ny = o.ny; size_t np = (size_t)n * ny;
    w.assign(np, 0); r1.assign(np, 0); r2.assign(np, 0);
    if (o.init == "random") { qaf_random_q_init(o.seed, n, ny, -0.01, 0.01, w.data(), r1.data(), r2.data()); return; }
    if (ny != n) die("--ny != --n: only --init random");
    if (o.init == "couple") { qaf_couple_init(o.seed, n, n, o.L, o.L, 1e-3, w.data(), r1.data(), r2.data()); return; }
    double dx = o.L / n;
    for (int j = 0; j < n; ++j) for (int i = 0; i < n; ++i) {
        size_t idx = (size_t)i + (size_t)j * n;
        analytic(o.init, i * dx, j * dx, w[idx], r1[idx], r2[idx]);
    }
}

// Binary dump: "QAFDUMP1", int32 nx, ny, nxh, real_bytes, nfields, kind (0 spectral, 1 physical),
// int64 step, then the fields back to back in the reference's layout.
void dump(const std::string& path, int n, int ny, int kind, long long step, const std::vector<const void*>& dev,
          size_t bytes_each) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) die(("cannot write " + path).c_str());
    int32_t hdr[6] = { n, ny, n / 2 + 1, (int32_t)sizeof(Qreal), (int32_t)dev.size(), kind };
    std::fwrite("QAFDUMP1", 1, 8, f);
    std::fwrite(hdr, sizeof(hdr), 1, f);
    int64_t s = step; std::fwrite(&s, sizeof(s), 1, f);
    std::vector<char> host(bytes_each);
    for (const void* p : dev) {
        check(cudaMemcpy(host.data(), p, bytes_each, cudaMemcpyDeviceToHost), "dump memcpy");
        std::fwrite(host.data(), 1, bytes_each, f);
    }
    std::fclose(f);
}

struct Solver {
    Mesh* mesh;
    Field *wold, *wcurr, *wnew, *wnonl, *u, *v;
    Field *r1old, *r1curr, *r1new, *r1nonl, *r2old, *r2curr, *r2new, *r2nonl, *S;
    Field *p11, *p12, *p21, *Ra, *aux, *aux1;
    Qreal *IFw, *IFwh, *IFr1, *IFr1h, *IFr2, *IFr2h;
    Qreal re, er, rf, lambda, dt;
    int Nxh, Ny, BSZ, do_dealias;

    Solver(const Opts& o) {
        const int BSZ_ = 16;
        mesh = new Mesh(o.n, o.ny, o.L, o.Ly, BSZ_);
        Nxh = mesh->Nxh; Ny = mesh->Ny; BSZ = BSZ_;
        re = o.re; er = o.er; rf = o.rf; lambda = o.lambda; dt = o.dt; do_dealias = o.dealias;
        wold = new Field(mesh); wcurr = new Field(mesh); wnew = new Field(mesh); wnonl = new Field(mesh);
        u = new Field(mesh); v = new Field(mesh);
        r1old = new Field(mesh); r1curr = new Field(mesh); r1new = new Field(mesh); r1nonl = new Field(mesh);
        r2old = new Field(mesh); r2curr = new Field(mesh); r2new = new Field(mesh); r2nonl = new Field(mesh);
        S = new Field(mesh);
        p11 = new Field(mesh); p12 = new Field(mesh); p21 = new Field(mesh);
        Ra = new Field(mesh); aux = new Field(mesh); aux1 = new Field(mesh);

        std::vector<double> w0, r10, r20;
        make_init(o, w0, r10, r20);
        load(wold, w0); load(r1old, r10); load(r2old, r20);
        std::vector<double> ra((size_t)o.n * o.ny, o.alpha);
        std::vector<Qreal> rah(ra.begin(), ra.end());
        check(cudaMemcpy(Ra->phys, rah.data(), mesh->physsize, cudaMemcpyHostToDevice), "Ra");

        check(cudaMalloc((void**)&IFw, mesh->wavesize), "IF"); check(cudaMalloc((void**)&IFwh, mesh->wavesize), "IF");
        check(cudaMalloc((void**)&IFr1, mesh->wavesize), "IF"); check(cudaMalloc((void**)&IFr1h, mesh->wavesize), "IF");
        check(cudaMalloc((void**)&IFr2, mesh->wavesize), "IF"); check(cudaMalloc((void**)&IFr2h, mesh->wavesize), "IF");
        wlin_func<<<mesh->dimGridsp, mesh->dimBlocksp>>>(IFw, IFwh, mesh->k_squared, re, rf, dt, Nxh, Ny, BSZ);
        r1lin_func<<<mesh->dimGridsp, mesh->dimBlocksp>>>(IFr1, IFr1h, mesh->k_squared, dt, Nxh, Ny, BSZ);
        r2lin_func<<<mesh->dimGridsp, mesh->dimBlocksp>>>(IFr2, IFr2h, mesh->k_squared, dt, Nxh, Ny, BSZ);
        check(cudaDeviceSynchronize(), "setup");
    }

    // Physical field -> device, then the Fwd/Bwd round trip the reference driver
    // applies to its initial fields (friction.cu:165-167).
    void load(Field* f, const std::vector<double>& h) {
        std::vector<Qreal> hr(h.begin(), h.end());
        check(cudaMemcpy(f->phys, hr.data(), mesh->physsize, cudaMemcpyHostToDevice), "load");
        FwdTrans(f->spec, f->phys, mesh);
        BwdTrans(f->phys, f->spec, mesh);
    }

    void nonlinear() {
        curr_func(r1curr, r2curr, wcurr, u, v, S);
        wnonl_func(wnonl, wcurr, u, v, r1curr, r2curr, Ra, S, p11, p12, p21, re, er, lambda, aux, aux1);
        r1nonl_func(r1nonl, wcurr, u, v, r1curr, r2curr, S, lambda, aux, aux1);
        r2nonl_func(r2nonl, wcurr, u, v, r1curr, r2curr, S, lambda, aux, aux1);
    }

    // One IF-RK4 step in the order of friction.cu:213-259; without the dealias
    // kernels it is the step of the coupled runs (couple.cu:179-215).
    void step() {
        dim3 g = mesh->dimGridsp, b = mesh->dimBlocksp;
        integrate_func0D<<<g, b>>>(wold->spec, wcurr->spec, wnew->spec, IFw, IFwh, Nxh, Ny, BSZ, dt);
        integrate_func0D<<<g, b>>>(r1old->spec, r1curr->spec, r1new->spec, IFr1, IFr1h, Nxh, Ny, BSZ, dt);
        integrate_func0D<<<g, b>>>(r2old->spec, r2curr->spec, r2new->spec, IFr2, IFr2h, Nxh, Ny, BSZ, dt);
        nonlinear();
        integrate_func1D<<<g, b>>>(wold->spec, wcurr->spec, wnew->spec, wnonl->spec, IFw, IFwh, Nxh, Ny, BSZ, dt);
        integrate_func1D<<<g, b>>>(r1old->spec, r1curr->spec, r1new->spec, r1nonl->spec, IFr1, IFr1h, Nxh, Ny, BSZ, dt);
        integrate_func1D<<<g, b>>>(r2old->spec, r2curr->spec, r2new->spec, r2nonl->spec, IFr2, IFr2h, Nxh, Ny, BSZ, dt);
        nonlinear();
        integrate_func2D<<<g, b>>>(wold->spec, wcurr->spec, wnew->spec, wnonl->spec, IFw, IFwh, Nxh, Ny, BSZ, dt);
        integrate_func2D<<<g, b>>>(r1old->spec, r1curr->spec, r1new->spec, r1nonl->spec, IFr1, IFr1h, Nxh, Ny, BSZ, dt);
        integrate_func2D<<<g, b>>>(r2old->spec, r2curr->spec, r2new->spec, r2nonl->spec, IFr2, IFr2h, Nxh, Ny, BSZ, dt);
        nonlinear();
        integrate_func3D<<<g, b>>>(wold->spec, wcurr->spec, wnew->spec, wnonl->spec, IFw, IFwh, Nxh, Ny, BSZ, dt);
        integrate_func3D<<<g, b>>>(r1old->spec, r1curr->spec, r1new->spec, r1nonl->spec, IFr1, IFr1h, Nxh, Ny, BSZ, dt);
        integrate_func3D<<<g, b>>>(r2old->spec, r2curr->spec, r2new->spec, r2nonl->spec, IFr2, IFr2h, Nxh, Ny, BSZ, dt);
        nonlinear();
        integrate_func4D<<<g, b>>>(wold->spec, wcurr->spec, wnew->spec, wnonl->spec, IFw, IFwh, Nxh, Ny, BSZ, dt);
        integrate_func4D<<<g, b>>>(r1old->spec, r1curr->spec, r1new->spec, r1nonl->spec, IFr1, IFr1h, Nxh, Ny, BSZ, dt);
        integrate_func4D<<<g, b>>>(r2old->spec, r2curr->spec, r2new->spec, r2nonl->spec, IFr2, IFr2h, Nxh, Ny, BSZ, dt);
        if (do_dealias == 1) {
            dealias<<<g, b>>>(wnew->spec, mesh->cutoff, Nxh, Ny, BSZ);
            dealias<<<g, b>>>(r1new->spec, mesh->cutoff, Nxh, Ny, BSZ);
            dealias<<<g, b>>>(r2new->spec, mesh->cutoff, Nxh, Ny, BSZ);
        } else if (do_dealias == 2) {
            for (int k = 0; k < 3; ++k) dealias<<<g, b>>>(wnew->spec, mesh->cutoff, Nxh, Ny, BSZ);
        }
        SpecSet<<<g, b>>>(wold->spec, wnew->spec, Nxh, Ny, BSZ);
        SpecSet<<<g, b>>>(r1old->spec, r1new->spec, Nxh, Ny, BSZ);
        SpecSet<<<g, b>>>(r2old->spec, r2new->spec, Nxh, Ny, BSZ);
    }

    // In the reference's stage-1 the nonlinear terms read the *curr* fields,
    // which integrate_func0D set equal to old; for a standalone evaluation copy
    // old into curr first.
    void set_curr_from_old() {
        dim3 g = mesh->dimGridsp, b = mesh->dimBlocksp;
        SpecSet<<<g, b>>>(wcurr->spec, wold->spec, Nxh, Ny, BSZ);
        SpecSet<<<g, b>>>(r1curr->spec, r1old->spec, Nxh, Ny, BSZ);
        SpecSet<<<g, b>>>(r2curr->spec, r2old->spec, Nxh, Ny, BSZ);
    }
};

std::string stepname(const std::string& out, int s) { return out + "_s" + std::to_string(s) + ".bin"; }

int run(const Opts& o) {
    Solver sv(o);
    size_t sb = sv.mesh->specsize;
    if (o.dumps.count(0)) dump(stepname(o.out, 0), o.n, o.ny, 0, 0, {sv.wold->spec, sv.r1old->spec, sv.r2old->spec}, sb);
    for (int m = 1; m <= o.steps; ++m) {
        sv.step();
        if (o.dumps.count(m)) dump(stepname(o.out, m), o.n, o.ny, 0, m, {sv.wold->spec, sv.r1old->spec, sv.r2old->spec}, sb);
    }
    check(cudaDeviceSynchronize(), "run");
    std::printf("{\"mode\": \"run\", \"n\": %d, \"steps\": %d, \"ok\": true}\n", o.n, o.steps);
    return 0;
}

int nonlinear(const Opts& o) {
    Solver sv(o);
    sv.set_curr_from_old();
    sv.nonlinear();
    check(cudaDeviceSynchronize(), "nonlinear");
    size_t sb = sv.mesh->specsize;
    dump(o.out + "_nl.bin", o.n, o.ny, 0, 0, {sv.wnonl->spec, sv.r1nonl->spec, sv.r2nonl->spec}, sb);
    dump(o.out + "_in.bin", o.n, o.ny, 0, 0, {sv.wold->spec, sv.r1old->spec, sv.r2old->spec}, sb);
    std::printf("{\"mode\": \"nonlinear\", \"n\": %d, \"ok\": true}\n", o.n);
    return 0;
}

int timeit(const Opts& o) {
    Solver sv(o);
    for (int m = 0; m < o.warmup; ++m) sv.step();
    check(cudaDeviceSynchronize(), "warmup");
    cudaEvent_t a, b;
    check(cudaEventCreate(&a), "event"); check(cudaEventCreate(&b), "event");
    check(cudaEventRecord(a), "record");
    for (int m = 0; m < o.timed; ++m) sv.step();
    check(cudaEventRecord(b), "record");
    check(cudaEventSynchronize(b), "sync");
    float ms = 0; check(cudaEventElapsedTime(&ms, a, b), "elapsed");
    check(cudaGetLastError(), "launch");
    double per = ms / o.timed;
    std::printf("{\"mode\": \"time\", \"n\": %d, \"real_bytes\": %d, \"warmup\": %d, \"timed\": %d, "
                "\"ms_total\": %.6f, \"ms_per_step\": %.6f}\n",
                o.n, (int)sizeof(Qreal), o.warmup, o.timed, (double)ms, per);
    return 0;
}

// ---- C2R convention probe -------------------------------------------------
// The C2R of the reference (BwdTrans, QFldfuncs.cuh:50-55) receives spectra
// that are not Hermitian in the kx = 0 and kx = Nx/2 columns. Hypothesis H:
// the physical result is Re(IDFT_y) on those two columns (i.e. their Hermitian
// part), which is what a column C2C followed by a row C2R that ignores the
// imaginary parts of the row's DC and Nyquist terms computes. The probe fits
// the deviation from H onto the four leak patterns Im(y0), Im(y0)(-1)^m,
// Im(yN), Im(yN)(-1)^m and reports the fit and its residual.
int probe(const Opts& o) {
    Solver sv(o);
    int n = o.n, nxh = n / 2 + 1;
    std::vector<double> re(nxh * (size_t)n), imv(nxh * (size_t)n);
    for (size_t k = 0; k < re.size(); ++k) { re[k] = qaf_uniform_at(o.seed + 77, 2 * k, -1, 1); imv[k] = qaf_uniform_at(o.seed + 77, 2 * k + 1, -1, 1); }
    std::vector<Qcomp> hs(re.size());
    for (size_t k = 0; k < re.size(); ++k) { hs[k].x = (Qreal)re[k]; hs[k].y = (Qreal)imv[k]; re[k] = hs[k].x; imv[k] = hs[k].y; }
    check(cudaMemcpy(sv.aux->spec, hs.data(), sv.mesh->specsize, cudaMemcpyHostToDevice), "probe in");
    BwdTrans(sv.aux->phys, sv.aux->spec, sv.mesh);
    std::vector<Qreal> out((size_t)n * n);
    check(cudaMemcpy(out.data(), sv.aux->phys, sv.mesh->physsize, cudaMemcpyDeviceToHost), "probe out");

    std::vector<double> cs(n), sn(n);
    for (int k = 0; k < n; ++k) { long double a = 2.0L * 3.14159265358979323846264338327950288L * k / n; cs[k] = (double)cosl(a); sn[k] = (double)sinl(a); }
    // column IDFT along y for every stored column i
    std::vector<double> yr(nxh * (size_t)n), yi(nxh * (size_t)n);
    for (int i = 0; i < nxh; ++i)
        for (int m = 0; m < n; ++m) {
            double sr = 0, si = 0;
            for (int j = 0; j < n; ++j) {
                int t = (int)(((long long)j * m) % n);
                double xr = re[i + (size_t)j * nxh], xi = imv[i + (size_t)j * nxh];
                sr += xr * cs[t] - xi * sn[t]; si += xr * sn[t] + xi * cs[t];
            }
            yr[i + (size_t)m * nxh] = sr; yi[i + (size_t)m * nxh] = si;
        }
    double inv = 1.0 / ((double)n * n);
    double num[4][4] = {{0}}, rhs[4] = {0}, dev2 = 0, out2 = 0;
    std::vector<double> h((size_t)n * n);
    for (int m = 0; m < n; ++m)            // y index
        for (int p = 0; p < n; ++p) {      // x index
            double s = yr[0 + (size_t)m * nxh] + yr[nxh - 1 + (size_t)m * nxh] * ((p & 1) ? -1.0 : 1.0);
            for (int i = 1; i < nxh - 1; ++i) {
                int t = (int)(((long long)i * p) % n);
                s += 2.0 * (yr[i + (size_t)m * nxh] * cs[t] - yi[i + (size_t)m * nxh] * sn[t]);
            }
            double hv = s * inv, cv = out[p + (size_t)m * n];
            double sg = (p & 1) ? -1.0 : 1.0;
            double b[4] = { yi[0 + (size_t)m * nxh] * inv, yi[0 + (size_t)m * nxh] * sg * inv,
                            yi[nxh - 1 + (size_t)m * nxh] * inv, yi[nxh - 1 + (size_t)m * nxh] * sg * inv };
            double d = cv - hv;
            dev2 += d * d; out2 += cv * cv;
            for (int r = 0; r < 4; ++r) { rhs[r] += b[r] * d; for (int c = 0; c < 4; ++c) num[r][c] += b[r] * b[c]; }
            h[p + (size_t)m * n] = d;
        }
    // solve the 4x4 normal equations (Gaussian elimination, no pivoting needed: SPD)
    double A[4][5];
    for (int r = 0; r < 4; ++r) { for (int c = 0; c < 4; ++c) A[r][c] = num[r][c]; A[r][4] = rhs[r]; }
    for (int c = 0; c < 4; ++c) for (int r = c + 1; r < 4; ++r) { double f = A[r][c] / A[c][c]; for (int k = c; k < 5; ++k) A[r][k] -= f * A[c][k]; }
    double coef[4];
    for (int r = 3; r >= 0; --r) { double s = A[r][4]; for (int c = r + 1; c < 4; ++c) s -= A[r][c] * coef[c]; coef[r] = s / A[r][r]; }
    double res2 = 0;
    for (int m = 0; m < n; ++m) for (int p = 0; p < n; ++p) {
        double sg = (p & 1) ? -1.0 : 1.0;
        double fit = coef[0] * yi[0 + (size_t)m * nxh] * inv + coef[1] * yi[0 + (size_t)m * nxh] * sg * inv
                   + coef[2] * yi[nxh - 1 + (size_t)m * nxh] * inv + coef[3] * yi[nxh - 1 + (size_t)m * nxh] * sg * inv;
        double r = h[p + (size_t)m * n] - fit; res2 += r * r;
    }
    std::printf("{\"mode\": \"probe\", \"n\": %d, \"real_bytes\": %d, \"rel_dev_from_hermitian_projection\": %.3e, "
                "\"leak_coef\": [%.6f, %.6f, %.6f, %.6f], \"rel_residual_after_fit\": %.3e}\n",
                n, (int)sizeof(Qreal), std::sqrt(dev2 / out2), coef[0], coef[1], coef[2], coef[3], std::sqrt(res2 / out2));
    return 0;
}

} // namespace

int main(int argc, char** argv) {
    Opts o = parse(argc, argv);
    if (o.ny == 0) o.ny = o.n;
    if (o.Ly == 0) o.Ly = o.L;
    if (o.n < 4 || (o.n % 2) || o.ny < 4) die("--n must be even and >= 4, --ny >= 4");
    if (o.mode == "run") return run(o);
    if (o.mode == "nonlinear") return nonlinear(o);
    if (o.mode == "time") return timeit(o);
    if (o.mode == "probe") return probe(o);
    die("unknown mode");
    return 2;
}
