// qaf_api.cu — the C ABI of include/qaf.h: meshes, workspaces, launch
// configuration per grid size and precision, and the step driver.
#include "qaf.h"
#include "qaf_init.h"

#include <cudaTypedefs.h>   // PFN_cuTensorMapEncodeTiled
#include "qaf_internal.cuh"
#include "qaf_adjoint.cuh"

#include <cmath>
#include <cstdio>
#include <algorithm>
#include <atomic>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <tuple>
#include <string>
#include <type_traits>
#include <vector>

using namespace qaf;
using namespace qaf::detail;

namespace {

thread_local std::string g_last_error;

}  // namespace

namespace qaf {
namespace detail {

qaf_status fail(qaf_status st, const std::string& msg) {
    g_last_error = msg;
    return st;
}
std::mutex g_setup_mu;

}  // namespace detail
}  // namespace qaf

namespace {

template <typename real>
struct Workspace {
    int N = 0;
    cplx<real>* block = nullptr;  // one allocation for everything below
    cplx<real>* old_m[3];
    cplx<real>* old_n[3];
    cplx<real>* acc_m[3];
    cplx<real>* acc_n[3];
    cplx<real>* Y;
    cplx<real>* D;
    cplx<real>* G;
    cplx<real>* Ed;
    cplx<real>* T;     // transform scratch
    cplx<real>* tw;    // twiddles of length nx (row transforms)
    cplx<real>* tw_y;  // twiddles of length ny (column transforms; == tw when nx == ny)
    real* ex;
    real* ey;
    double* diag;      // [0] energy sum, [1] enstrophy sum, [2..] spectrum shells (scratch)
    unsigned* flags;
    int* queue;        // work counter of the persistent column kernel
    CUtensorMap tm_G;  // TMA view of the G arrays
    double cached[5] = {NAN, NAN, NAN, NAN, NAN};   // dt, re, rf, q_lin, unused -> IF tables valid for
    real e0[4];
};

size_t align_up(size_t x) { return (x + 31) & ~size_t(31); }

// TMA descriptor of the G arrays: [NG*ny rows][nx/2 columns] of 8-byte
// elements (two per FP64 complex), boxes of TW columns x g_box_rows(ny) rows
// (rows: the total row count when several instances follow each other).
template <typename real>
qaf_status encode_g_map(CUtensorMap* tm, const cplx<real>* G, int nx, int ny, size_t rows = 0) {
    // looked up once per process (a function-local static: thread-safe)
    static const PFN_cuTensorMapEncodeTiled_v12000 encode = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    if (!encode) return fail(QAF_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    const int H = nx / 2;
    const cuuint64_t cpe = sizeof(cplx<real>) / 8;
    cuuint64_t dims[2] = {(cuuint64_t)H * cpe, (cuuint64_t)(rows ? rows : (size_t)NG * ny)};
    cuuint64_t strides[1] = {(cuuint64_t)H * cpe * 8};
    cuuint32_t box[2] = {(cuuint32_t)(TW * cpe), (cuuint32_t)g_box_rows(ny)};   // the column kernel's BOXR
    cuuint32_t estr[2] = {1, 1};
    CUresult r = encode(tm, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<cplx<real>*>(G), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(QAF_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    return QAF_OK;
}

}  // namespace

struct qaf_mesh {
    qaf_mesh_desc desc;
    int nxh;
    double dkx, dky;
    Workspace<float> wf;
    Workspace<double> wd;
    int device;
    bool loaded = false;    // the resident state holds a loaded spectral state
    bool y_valid = false;   // the Y/D arrays hold the inverse transforms of that state
    uint64_t launches = 0;
};

namespace {

template <typename real>
Workspace<real>& ws(qaf_mesh* m);
template <> Workspace<float>& ws<float>(qaf_mesh* m) { return m->wf; }
template <> Workspace<double>& ws<double>(qaf_mesh* m) { return m->wd; }

// twiddles exp(-2 pi i m / N), from long double
template <typename real>
std::vector<cplx<real>> host_twiddles(int N) {
    std::vector<cplx<real>> tw(N);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < N; ++k) {
        long double a = -2.0L * pi * (long double)k / (long double)N;
        tw[k] = mk<real>((real)cosl(a), (real)sinl(a));
    }
    return tw;
}

// Separable integrating factors: exp(L dt) with L_w = (-kx^2 - ky^2 - Rf)/Re
// and L_Q = -kx^2 - ky^2 + q_lin factor into exp(-c kx^2 dt) exp(-c ky^2 dt) exp(c0 dt).
// ex/ey hold the kx/ky factors for the classes {w full, w half, Q full, Q half} step.
template <typename real>
void host_if_tables(int nx, int ny, double dkx, double dky, double dt, double re, std::vector<real>& ex,
                    std::vector<real>& ey) {
    const int H = nx / 2, N = ny;
    ex.assign(4 * (H + 1), 0);
    ey.assign(4 * (size_t)N, 0);
    const double steps[4] = {dt, 0.5 * dt, dt, 0.5 * dt};
    const double visc[4] = {1.0 / re, 1.0 / re, 1.0, 1.0};
    for (int c = 0; c < 4; ++c) {
        for (int i = 0; i <= H; ++i) {
            long double kx = (long double)dkx * i;
            ex[c * (H + 1) + i] = (real)expl(-(long double)visc[c] * kx * kx * (long double)steps[c]);
        }
        for (int j = 0; j < N; ++j) {
            long double ky = (long double)dky * (j < N / 2 + 1 ? j : j - N);
            ey[c * N + j] = (real)expl(-(long double)visc[c] * ky * ky * (long double)steps[c]);
        }
    }
}

// the constant parts exp(-Rf/Re dt), exp(-Rf/Re dt/2), exp(q_lin dt), exp(q_lin dt/2)
template <typename real>
void host_if_e0(double dt, double re, double rf, double q_lin, real* e0) {
    e0[0] = (real)expl(-(long double)rf / re * dt);
    e0[1] = (real)expl(-(long double)rf / re * dt * 0.5L);
    e0[2] = (real)expl((long double)q_lin * dt);
    e0[3] = (real)expl((long double)q_lin * dt * 0.5L);
}

template <typename real>
qaf_status ensure_ws(qaf_mesh* m) {
    Workspace<real>& w = ws<real>(m);
    if (w.block) return QAF_OK;
    // columns of length N = ny, H = nx / 2 of them (the state's main part)
    const int NXg = m->desc.nx, N = m->desc.ny, H = NXg / 2;
    const size_t plane = (size_t)N * H;
    // element counts (complex)
    size_t off = 0;
    auto take = [&](size_t n) { size_t o = off; off += align_up(n); return o; };
    size_t o_old_m[3], o_old_n[3], o_acc_m[3], o_acc_n[3];
    for (int f = 0; f < 3; ++f) { o_old_m[f] = take(plane); o_old_n[f] = take(N); }
    for (int f = 0; f < 3; ++f) { o_acc_m[f] = take(plane); o_acc_n[f] = take(N); }
    size_t oY = take(NY * plane), oD = take((size_t)PF_COUNT * N), oG = take(NG * plane), oE = take((size_t)NE * N);
    size_t oT = take(plane), otw = take(NXg), otwy = take(N);
    // real tables stored in complex slots
    size_t oex = take((4 * (H + 1) + 1) / 2 + 1), oey = take((4 * N + 1) / 2 + 1);
    // [0, 2) step sums, [2, 4) diagnostics, [4, 516) spectrum, [516, 1029) shell bounds, [1029, 1031) async copy-out
    size_t odiag = take((4 + 512 + 513 + 2) * sizeof(double) / sizeof(cplx<real>) + 1);
    size_t oflags = take(1);
    size_t oqueue = take(1);
    cplx<real>* b = nullptr;
    cudaError_t e = cudaMalloc((void**)&b, off * sizeof(cplx<real>));
    if (e != cudaSuccess) return fail(QAF_ERR_ALLOC, std::string("workspace cudaMalloc: ") + cudaGetErrorString(e));
    w.block = b;
    w.N = N;
    for (int f = 0; f < 3; ++f) {
        w.old_m[f] = b + o_old_m[f]; w.old_n[f] = b + o_old_n[f];
        w.acc_m[f] = b + o_acc_m[f]; w.acc_n[f] = b + o_acc_n[f];
    }
    w.Y = b + oY; w.D = b + oD; w.G = b + oG; w.Ed = b + oE; w.T = b + oT; w.tw = b + otw; w.tw_y = b + otwy;
    w.ex = reinterpret_cast<real*>(b + oex);
    w.ey = reinterpret_cast<real*>(b + oey);
    w.diag = reinterpret_cast<double*>(b + odiag);
    w.flags = reinterpret_cast<unsigned*>(b + oflags);
    w.queue = reinterpret_cast<int*>(b + oqueue);
    const std::vector<cplx<real>> tw = host_twiddles<real>(NXg), twy = host_twiddles<real>(N);
    QAF_CUDA(cudaMemcpy(w.tw, tw.data(), NXg * sizeof(cplx<real>), cudaMemcpyHostToDevice));
    QAF_CUDA(cudaMemcpy(w.tw_y, twy.data(), N * sizeof(cplx<real>), cudaMemcpyHostToDevice));
    QAF_TRY(encode_g_map<real>(&w.tm_G, w.G, NXg, N));
    QAF_CUDA(cudaMemset(w.flags, 0, sizeof(unsigned)));
    QAF_CUDA(cudaMemset(w.diag, 0, 2 * sizeof(double)));
    return QAF_OK;
}

template <typename real>
qaf_status ensure_if(qaf_mesh* m, const qaf_params* p, cudaStream_t st) {
    Workspace<real>& w = ws<real>(m);
    if (w.cached[0] == p->dt && w.cached[1] == p->re && w.cached[2] == p->rf && w.cached[3] == p->q_lin) return QAF_OK;
    std::vector<real> ex, ey;
    host_if_tables<real>(m->desc.nx, m->desc.ny, m->dkx, m->dky, p->dt, p->re, ex, ey);
    host_if_e0<real>(p->dt, p->re, p->rf, p->q_lin, w.e0);
    QAF_CUDA(cudaMemcpyAsync(w.ex, ex.data(), ex.size() * sizeof(real), cudaMemcpyHostToDevice, st));
    QAF_CUDA(cudaMemcpyAsync(w.ey, ey.data(), ey.size() * sizeof(real), cudaMemcpyHostToDevice, st));
    QAF_CUDA(cudaStreamSynchronize(st));   // host vectors go out of scope
    w.cached[0] = p->dt; w.cached[1] = p->re; w.cached[2] = p->rf; w.cached[3] = p->q_lin;
    return QAF_OK;
}

// the step's truncation of the new state by the 2/3 mask (keep i <= kx_keep
// && (j <= ky_lo || j >= ky_hi)) after stage 4, per field: all three
// (no_dealias 0, friction.cu:253-255), none (1, the coupled runs,
// couple.cu:179-215) or w only (2, dealias/couple.cu:226-229)
template <class Args>
void set_mask(Args& a, int nx, int ny, int no_dealias) {
    a.kx_keep = (nx / 2) * 2 / 3; a.ky_lo = ny / 3; a.ky_hi = ny - ny / 3 + 1;
    a.trunc = no_dealias == 0 ? 7 : (no_dealias == 2 ? 1 : 0);
}

template <typename real>
StageArgs<real> make_args(qaf_mesh* m, const qaf_params* p) {
    Workspace<real>& w = ws<real>(m);
    StageArgs<real> a;
    std::memset(&a, 0, sizeof(a));
    a.nx = m->desc.nx; a.ny = m->desc.ny;
    a.dkx = (real)m->dkx; a.dky = (real)m->dky;
    a.lambda = (real)p->lambda; a.ce = (real)(1.0 / (p->er * p->re)); a.alpha = (real)p->alpha;
    a.alpha_field = reinterpret_cast<const real*>(p->alpha_field);
    a.dt = (real)p->dt; a.advect = p->advect_omega ? 1 : 0;
    set_mask(a, a.nx, a.ny, p->no_dealias);
    for (int f = 0; f < 3; ++f) {
        a.old_m[f] = w.old_m[f]; a.old_n[f] = w.old_n[f]; a.acc_m[f] = w.acc_m[f]; a.acc_n[f] = w.acc_n[f];
        a.nl_m[f] = w.acc_m[f]; a.nl_n[f] = w.acc_n[f];
    }
    a.Y = w.Y; a.D = w.D; a.G = w.G; a.Ed = w.Ed; a.tw = w.tw; a.tw_y = w.tw_y; a.ex = w.ex; a.ey = w.ey;
    for (int c = 0; c < 4; ++c) a.e0[c] = w.e0[c];
    a.diag = w.diag; a.flags = w.flags; a.queue = w.queue;
    a.tm_G = w.tm_G;
    a.ninst = 1;
    return a;
}

// ---------------------------------------------------------------------------
// launch-shape choices (autotuner): per (precision, grid size, batched) the
// column and row variants to use instead of the built-in shapes; -1 = built in
// ---------------------------------------------------------------------------
struct TuneChoice {
    int col = -1, row = -1;
    double us = 0;
};
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, TuneChoice> g_tune;

int variant_list(int dtype, int n, StepVariant<float>** out) {
    *out = nullptr;
    return dtype == QAF_F32 ? step_variants_f32(n, out) : 0;
}

// set-up of each variant per device: resident column CTAs (column variants)
// or 1 (row variants, attributes only), keyed by (variant, device)
std::map<std::pair<const StepVariant<float>*, int>, int> g_variant_setup;

}  // namespace

namespace qaf {
namespace detail {

// the variant to launch for kind (0 column, 1 row), or nullptr for the
// built-in shape; *slots receives its persistent grid size on this device
StepVariant<float>* tuned_variant(int n, int kind, bool batched, int* slots) {
    int idx = -1;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (g_tune.empty()) return nullptr;
    auto it = g_tune.find(std::make_tuple((int)QAF_F32, n, batched ? 1 : 0));
    if (it == g_tune.end()) return nullptr;
    idx = kind == 0 ? it->second.col : it->second.row;
    if (idx < 0) return nullptr;
    StepVariant<float>* v = nullptr;
    const int cnt = step_variants_f32(n, &v);
    if (idx >= cnt) return nullptr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    const auto key = std::make_pair((const StepVariant<float>*)&v[idx], dev);
    auto s = g_variant_setup.find(key);
    if (s == g_variant_setup.end()) {
        int got = 0;
        if (v[idx].setup(&got) != cudaSuccess) return nullptr;
        if (v[idx].kind == 0 && got < 1) return nullptr;
        s = g_variant_setup.emplace(key, v[idx].kind == 0 ? got : 1).first;
    }
    *slots = s->second;
    return &v[idx];
}

// test hook of qaf_test_lose_copy: consumed by the next column launch
std::atomic<int> g_test_drop{0};        // slab + 1, 0: off
std::atomic<unsigned> g_test_polls{0};

}  // namespace detail
}  // namespace qaf

namespace {

// ---------------------------------------------------------------------------
// per-size launchers
// ---------------------------------------------------------------------------
// Calls f(std::integral_constant<int, N>) for a supported transform length N.
template <class F>
qaf_status with_n(int N, F&& f) {
#ifdef QAF_ONLY_N
    if (N == QAF_ONLY_N) return f(std::integral_constant<int, QAF_ONLY_N>{});
    return fail(QAF_ERR_UNSUPPORTED, "no kernels for this grid size (a build for one size only)");
#endif
    switch (N) {
        case 16: return f(std::integral_constant<int, 16>{});
        case 32: return f(std::integral_constant<int, 32>{});
        case 64: return f(std::integral_constant<int, 64>{});
        case 128: return f(std::integral_constant<int, 128>{});
        case 256: return f(std::integral_constant<int, 256>{});
        case 512: return f(std::integral_constant<int, 512>{});
        case 1024: return f(std::integral_constant<int, 1024>{});
        case 48: return f(std::integral_constant<int, 48>{});
        case 96: return f(std::integral_constant<int, 96>{});
        case 192: return f(std::integral_constant<int, 192>{});
        case 384: return f(std::integral_constant<int, 384>{});
        case 768: return f(std::integral_constant<int, 768>{});
        default: return fail(QAF_ERR_UNSUPPORTED, "no kernels for this grid size");
    }
}

// Runtime-size launches on an nx x ny grid: the row kernel and the row
// transforms are the nx-point kernels, the column ones the ny-point kernels.
template <typename real>
qaf_status setup_grid(int nx, int ny) {
    QAF_TRY(with_n(nx, [](auto n) -> qaf_status { return Launch<real, decltype(n)::value>::setup(); }));
    if (ny != nx) QAF_TRY(with_n(ny, [](auto n) -> qaf_status { return Launch<real, decltype(n)::value>::setup(); }));
    return QAF_OK;
}
template <typename real>
void launch_row(const StageArgs<real>& a, cudaStream_t st) {
    with_n(a.nx, [&](auto n) -> qaf_status { Launch<real, decltype(n)::value>::row(a, st); return QAF_OK; });
}
template <typename real>
void launch_col(const StageArgs<real>& a, cudaStream_t st) {
    with_n(a.ny, [&](auto n) -> qaf_status { Launch<real, decltype(n)::value>::col(a, st); return QAF_OK; });
}

// Calls F::template run<real>(args...) for the mesh's precision, after
// checking that both grid sizes have kernels (the operation's launches take
// the sizes at run time: launch_row / launch_col, Launch<real, N>::col_*/row_*).
template <class F, class... A>
qaf_status dispatch_grid(const qaf_mesh* m, A&&... args) {
    if (!size_supported(m->desc.nx) || !size_supported(m->desc.ny))
        return fail(QAF_ERR_UNSUPPORTED, "no kernels for this grid size (nx and ny each a power of two in "
                                         "[16, 1024] or 3 * 2^k in [48, 768])");
#ifdef QAF_ONLY_N
    if (m->desc.nx != QAF_ONLY_N || m->desc.ny != QAF_ONLY_N)
        return fail(QAF_ERR_UNSUPPORTED, "no kernels for this grid size (a build for one size only)");
#endif
    return m->desc.dtype == QAF_F64 ? F::template run<double>(std::forward<A>(args)...)
                                    : F::template run<float>(std::forward<A>(args)...);
}

// Calls F::template run<real, N>(args...) for the mesh's precision and size
// (square grids: noalloc step, adjoint).
template <class F, class... A>
qaf_status dispatch(const qaf_mesh* m, A&&... args) {
    const int N = m->desc.nx;
    if (m->desc.ny != N) return fail(QAF_ERR_UNSUPPORTED, "this operation needs nx == ny");
    const bool f64 = m->desc.dtype == QAF_F64;
#define QAF_CASE(n)                                                                       \
    case n:                                                                               \
        return f64 ? F::template run<double, n>(std::forward<A>(args)...)                \
                   : F::template run<float, n>(std::forward<A>(args)...);
    switch (N) {
#ifdef QAF_ONLY_N
        QAF_CASE(QAF_ONLY_N)
#else
        QAF_CASE(16) QAF_CASE(32) QAF_CASE(64) QAF_CASE(128) QAF_CASE(256) QAF_CASE(512) QAF_CASE(1024)
        QAF_CASE(48) QAF_CASE(96) QAF_CASE(192) QAF_CASE(384) QAF_CASE(768)
#endif
        default: break;
    }
#undef QAF_CASE
    return fail(QAF_ERR_UNSUPPORTED, "no kernels for this grid size (need nx == ny, a power of two in [16, 1024] "
                                     "or 3 * 2^k in [48, 768])");
}

qaf_status check_mesh(const qaf_mesh* m) {
    if (!m) return fail(QAF_ERR_INVALID, "null mesh");
    return QAF_OK;
}

size_t spec_elems(const qaf_mesh* m) { return (size_t)m->nxh * m->desc.ny; }
size_t phys_elems(const qaf_mesh* m) { return (size_t)m->desc.nx * m->desc.ny; }
size_t real_bytes(const qaf_mesh* m) { return m->desc.dtype == QAF_F64 ? 8 : 4; }

Geo geo(const qaf_mesh* m) { return Geo{m->desc.nx, m->desc.ny, m->nxh, m->dkx, m->dky}; }
int grid_for(size_t n) { size_t g = (n + 255) / 256; return (int)(g > 148 * 16 ? 148 * 16 : (g < 1 ? 1 : g)); }

qaf_status post_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(QAF_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return QAF_OK;
}

// ---------------------------------------------------------------------------
// operations
// ---------------------------------------------------------------------------
// BwdTrans: the ny-point column inverse transforms of the nx/2 columns, then
// the nx-point row C2Rs of the ny rows
struct OpBwd {
    template <typename real>
    static qaf_status run(qaf_mesh* m, const void* spec, void* phys, cudaStream_t st) {
        QAF_TRY(ensure_ws<real>(m));
        const int nx = m->desc.nx, ny = m->desc.ny;
        QAF_TRY(setup_grid<real>(nx, ny));
        Workspace<real>& w = ws<real>(m);
        QAF_TRY(with_n(ny, [&](auto n) -> qaf_status {
            Launch<real, decltype(n)::value>::col_ifft(reinterpret_cast<const cplx<real>*>(spec), w.T, w.tw_y, nx, st);
            return QAF_OK;
        }));
        QAF_TRY(with_n(nx, [&](auto n) -> qaf_status {
            Launch<real, decltype(n)::value>::row_c2r(w.T, reinterpret_cast<real*>(phys), w.tw, ny, st);
            return QAF_OK;
        }));
        return post_launch("BwdTrans");
    }
};

struct OpFwd {
    template <typename real>
    static qaf_status run(qaf_mesh* m, const void* phys, void* spec, cudaStream_t st) {
        QAF_TRY(ensure_ws<real>(m));
        const int nx = m->desc.nx, ny = m->desc.ny;
        QAF_TRY(setup_grid<real>(nx, ny));
        Workspace<real>& w = ws<real>(m);
        QAF_TRY(with_n(nx, [&](auto n) -> qaf_status {
            Launch<real, decltype(n)::value>::row_r2c(reinterpret_cast<const real*>(phys), w.T, w.tw, ny, st);
            return QAF_OK;
        }));
        QAF_TRY(with_n(ny, [&](auto n) -> qaf_status {
            Launch<real, decltype(n)::value>::col_fft(w.T, reinterpret_cast<cplx<real>*>(spec), w.tw_y, nx, st);
            return QAF_OK;
        }));
        return post_launch("FwdTrans");
    }
};

template <typename real>
void to_internal(qaf_mesh* m, const void* ref, int f, cudaStream_t st) {
    Workspace<real>& w = ws<real>(m);
    ref_to_internal<real><<<grid_for(spec_elems(m)), 256, 0, st>>>(reinterpret_cast<const cplx<real>*>(ref), w.old_m[f], w.old_n[f],
                                                                    m->desc.nx, m->desc.ny);
}

template <typename real>
void from_internal(qaf_mesh* m, cplx<real>* mm, cplx<real>* nq, void* ref, cudaStream_t st) {
    internal_to_ref<real><<<grid_for(spec_elems(m)), 256, 0, st>>>(mm, nq, reinterpret_cast<cplx<real>*>(ref), m->desc.nx,
                                                                    m->desc.ny);
}

struct OpNonlinear {
    template <typename real>
    static qaf_status run(qaf_mesh* m, const qaf_params* p, const void* const* in, void* const* out, void* phys_out,
                          cudaStream_t st) {
        QAF_TRY(ensure_ws<real>(m));
        QAF_TRY(setup_grid<real>(m->desc.nx, m->desc.ny));
        Workspace<real>& w = ws<real>(m);
        for (int f = 0; f < 3; ++f) to_internal<real>(m, in[f], f, st);
        m->loaded = true;      // the nonlinear evaluation reuses the state buffers
        m->y_valid = false;
        m->launches += 9;
        StageArgs<real> a = make_args<real>(m, p);
        a.phys_out = static_cast<real*>(phys_out);
        a.phys_all = 1;
        a.mode = MODE_PROLOGUE; a.do_inverse = 1;
        QAF_CUDA(cudaMemsetAsync(w.queue, 0, sizeof(int), st));
        launch_col<real>(a, st);
        launch_row<real>(a, st);
        a.mode = MODE_NONL; a.do_inverse = 0;
        launch_col<real>(a, st);
        for (int f = 0; f < 3; ++f) from_internal<real>(m, w.acc_m[f], w.acc_n[f], out[f], st);
        return post_launch("qaf_nonlinear");
    }
};

struct OpLoad {
    template <typename real>
    static qaf_status run(qaf_mesh* m, void* const* state, cudaStream_t st) {
        QAF_TRY(ensure_ws<real>(m));
        for (int f = 0; f < 3; ++f) to_internal<real>(m, state[f], f, st);
        m->launches += 3;
        m->loaded = true;
        m->y_valid = false;
        return post_launch("qaf_state_load");
    }
};

struct OpStore {
    template <typename real>
    static qaf_status run(qaf_mesh* m, void* const* state, cudaStream_t st) {
        Workspace<real>& w = ws<real>(m);
        for (int f = 0; f < 3; ++f) from_internal<real>(m, w.old_m[f], w.old_n[f], state[f], st);
        m->launches += 3;
        return post_launch("qaf_state_store");
    }
};

// Events around every row/column launch when `ev` is given (timed variant).
struct KernelTimer {
    std::vector<cudaEvent_t> ev;
    std::vector<int> kind;    // 0 row, 1 column
};

struct OpAdvance {
    template <typename real>
    static qaf_status run(qaf_mesh* m, const qaf_params* p, int integ, int nsteps, bool final_inverse, KernelTimer* timer,
                          cudaStream_t st) {
        QAF_TRY(ensure_ws<real>(m));
        QAF_TRY(setup_grid<real>(m->desc.nx, m->desc.ny));
        QAF_TRY(ensure_if<real>(m, p, st));
        Workspace<real>& w = ws<real>(m);
        StageArgs<real> a = make_args<real>(m, p);
        a.integrator = integ;
        const int nst = integ == QAF_IFRK4 ? 4 : (integ == QAF_IFRK2 ? 2 : 1);
        auto launch = [&](int kind) {
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            if (timer) {
                cudaEventCreate(&e0); cudaEventCreate(&e1);
                cudaEventRecord(e0, st);
            }
            if (kind == 0) launch_row<real>(a, st); else launch_col<real>(a, st);
            if (timer) {
                cudaEventRecord(e1, st);
                timer->ev.push_back(e0); timer->ev.push_back(e1); timer->kind.push_back(kind);
            }
            m->launches += 1;
        };
        if (!m->y_valid) {
            a.mode = MODE_PROLOGUE; a.do_inverse = 1;
            QAF_CUDA(cudaMemsetAsync(w.queue, 0, sizeof(int), st));
            launch_col<real>(a, st);
            m->launches += 1;
        }
        a.mode = MODE_STAGE;
        for (int s = 0; s < nsteps; ++s) {
            const bool last_step = s == nsteps - 1;
            if (last_step) {
                QAF_CUDA(cudaMemsetAsync(w.diag, 0, 2 * sizeof(double), st));
                m->launches += 1;
            }
            for (int k = 1; k <= nst; ++k) {
                a.stage = k;
                a.last_stage = k == nst;
                a.do_inverse = !(last_step && k == nst && !final_inverse);
                a.diag = (last_step && k == nst) ? w.diag : nullptr;
                launch(0);
                launch(1);
            }
        }
        m->y_valid = final_inverse;
        return post_launch("qaf_state_advance");
    }
};

template <typename real>
qaf_status diag_impl(qaf_mesh* m, const void* wspec, double* energy, double* enstrophy, double* spectrum, int nshells,
                     cudaStream_t st) {
    QAF_TRY(ensure_ws<real>(m));
    Workspace<real>& w = ws<real>(m);
    if (nshells > 512) return fail(QAF_ERR_INVALID, "at most 512 spectrum shells");
    QAF_CUDA(cudaMemsetAsync(w.diag + 2, 0, (2 + (size_t)(nshells > 0 ? nshells : 0)) * sizeof(double), st));
    // shell bounds k_0 = 0, k_{s+1} = k_s + dk, by repeated addition as the post-processor does
    std::vector<double> bounds(nshells + 1 > 0 ? nshells + 1 : 1, 0.0);
    const double dk = 2 * M_PI / m->desc.lx;
    for (int s = 1; s <= nshells; ++s) bounds[s] = bounds[s - 1] + dk;
    double* dbounds = w.diag + 4 + 512;
    QAF_CUDA(cudaMemcpyAsync(dbounds, bounds.data(), bounds.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    diag_kernel<real><<<grid_for(spec_elems(m)), 256, 0, st>>>(geo(m), reinterpret_cast<const cplx<real>*>(wspec),
                                                               w.diag + 2, dbounds, nshells);
    QAF_TRY(post_launch("qaf_diagnostics"));
    std::vector<double> h(2 + (nshells > 0 ? nshells : 0));
    QAF_CUDA(cudaMemcpyAsync(h.data(), w.diag + 2, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    QAF_CUDA(cudaStreamSynchronize(st));   // also keeps `bounds` alive until the copy is done
    const double n4 = (double)m->desc.nx * m->desc.ny * (double)m->desc.nx * m->desc.ny;
    if (energy) *energy = 0.5 * h[0] / n4;
    if (enstrophy) *enstrophy = 0.5 * h[1] / n4;
    if (spectrum && nshells > 0) {
        const double dk = 2 * M_PI / m->desc.lx;
        const double norm = 2.0 * dk * n4;
        for (int s = 0; s < nshells; ++s) spectrum[s] = h[2 + s] / norm;
    }
    return QAF_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* qaf_version(void) { return "qaf-b200 0.1 (sm_100a)"; }
const char* qaf_last_error(void) { return g_last_error.c_str(); }

int qaf_supported(int n, qaf_dtype dtype) {
    return (dtype == QAF_F32 || dtype == QAF_F64) && size_supported(n);
}

qaf_status qaf_mesh_create(const qaf_mesh_desc* desc, qaf_mesh** out) {
    if (!desc || !out) return fail(QAF_ERR_INVALID, "null argument");
    *out = nullptr;
    if (desc->nx < 4 || desc->ny < 4 || desc->nx % 2) return fail(QAF_ERR_INVALID, "nx, ny must be >= 4 and nx even");
    if (!(desc->lx > 0) || !(desc->ly > 0)) return fail(QAF_ERR_INVALID, "lx, ly must be positive");
    if (desc->dtype != QAF_F32 && desc->dtype != QAF_F64) return fail(QAF_ERR_INVALID, "bad dtype");
    qaf_mesh* m = new qaf_mesh();
    m->desc = *desc;
    m->nxh = desc->nx / 2 + 1;
    m->dkx = 2 * M_PI / desc->lx;   // waveinit, Mesh.cuh:6-21
    m->dky = 2 * M_PI / desc->ly;
    cudaGetDevice(&m->device);
    *out = m;
    return QAF_OK;
}

qaf_status qaf_mesh_destroy(qaf_mesh* m) {
    if (!m) return QAF_OK;
    if (m->wf.block) cudaFree(m->wf.block);
    if (m->wd.block) cudaFree(m->wd.block);
    delete m;
    return QAF_OK;
}

qaf_status qaf_mesh_sizes(const qaf_mesh* m, size_t* phys_bytes, size_t* spec_bytes) {
    QAF_TRY(check_mesh(m));
    if (phys_bytes) *phys_bytes = phys_elems(m) * real_bytes(m);
    if (spec_bytes) *spec_bytes = spec_elems(m) * 2 * real_bytes(m);
    return QAF_OK;
}

qaf_status qaf_field_alloc(const qaf_mesh* m, void** phys, void** spec) {
    QAF_TRY(check_mesh(m));
    if (phys) { *phys = nullptr; QAF_CUDA(cudaMalloc(phys, phys_elems(m) * real_bytes(m))); }
    if (spec) { *spec = nullptr; QAF_CUDA(cudaMalloc(spec, spec_elems(m) * 2 * real_bytes(m))); }
    return QAF_OK;
}

qaf_status qaf_field_free(void* phys, void* spec) {
    if (phys) cudaFree(phys);
    if (spec) cudaFree(spec);
    return QAF_OK;
}

qaf_status qaf_mesh_tables(const qaf_mesh* m, void* kx, void* ky, void* k2, void* cutoff) {
    QAF_TRY(check_mesh(m));
    const int nxh = m->nxh, ny = m->desc.ny;
    const bool f64 = m->desc.dtype == QAF_F64;
    for (int i = 0; i < nxh; ++i)
        for (int j = 0; j < ny; ++j) {
            const size_t idx = i + (size_t)j * nxh;
            const double kyv = (j < ny / 2 + 1) ? 2 * M_PI / m->desc.ly * j : 2 * M_PI / m->desc.ly * (j - ny);
            const double kxv = 2 * M_PI / m->desc.lx * i;
            const double k2v = kxv * kxv + kyv * kyv;
            const double cut = ((i < (nxh - 1) * 2 / 3 + 1) && ((j < ny / 3 + 1) || ((ny - j) < ny / 3))) ? 1.0 : 0.0;
            const double vals[4] = {kxv, kyv, k2v, cut};
            void* dst[4] = {kx, ky, k2, cutoff};
            for (int q = 0; q < 4; ++q) {
                if (!dst[q]) continue;
                if (f64) static_cast<double*>(dst[q])[idx] = vals[q];
                else static_cast<float*>(dst[q])[idx] = (float)vals[q];
            }
        }
    return QAF_OK;
}

qaf_status qaf_bwd_trans(qaf_mesh* m, const void* spec, void* phys, void* stream) {
    QAF_TRY(check_mesh(m));
    if (!spec || !phys) return fail(QAF_ERR_INVALID, "null pointer");
    return dispatch_grid<OpBwd>(m, m, spec, phys, (cudaStream_t)stream);
}

qaf_status qaf_fwd_trans(qaf_mesh* m, const void* phys, void* spec, void* stream) {
    QAF_TRY(check_mesh(m));
    if (!spec || !phys) return fail(QAF_ERR_INVALID, "null pointer");
    return dispatch_grid<OpFwd>(m, m, phys, spec, (cudaStream_t)stream);
}

#define QAF_BY_DTYPE(m, KERNEL_F32, KERNEL_F64) \
    do { if ((m)->desc.dtype == QAF_F64) { KERNEL_F64; } else { KERNEL_F32; } } while (0)

qaf_status qaf_symmetrize(qaf_mesh* m, void* spec, void* stream) {
    QAF_TRY(check_mesh(m));
    if (!spec) return fail(QAF_ERR_INVALID, "null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    QAF_BY_DTYPE(m, (symmetrize_kernel<float><<<grid_for(m->desc.ny), 256, 0, st>>>(geo(m), (cplx<float>*)spec)),
                    (symmetrize_kernel<double><<<grid_for(m->desc.ny), 256, 0, st>>>(geo(m), (cplx<double>*)spec)));
    return post_launch("qaf_symmetrize");
}

static qaf_status unary(qaf_mesh* m, int op, const void* in, void* out, void* stream) {
    QAF_TRY(check_mesh(m));
    if (!in || !out) return fail(QAF_ERR_INVALID, "null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    int g = grid_for(spec_elems(m));
    QAF_BY_DTYPE(m, (spec_unary_kernel<float><<<g, 256, 0, st>>>(geo(m), op, (const cplx<float>*)in, (cplx<float>*)out)),
                    (spec_unary_kernel<double><<<g, 256, 0, st>>>(geo(m), op, (const cplx<double>*)in, (cplx<double>*)out)));
    return post_launch("spectral operator");
}

qaf_status qaf_xderiv(qaf_mesh* m, const void* in, void* out, void* stream) { return unary(m, 0, in, out, stream); }
qaf_status qaf_yderiv(qaf_mesh* m, const void* in, void* out, void* stream) { return unary(m, 1, in, out, stream); }
qaf_status qaf_laplacian(qaf_mesh* m, const void* in, void* out, void* stream) { return unary(m, 2, in, out, stream); }

qaf_status qaf_vel(qaf_mesh* m, const void* w, void* u, void* v, void* stream) {
    QAF_TRY(check_mesh(m));
    if (!w || !u || !v) return fail(QAF_ERR_INVALID, "null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    int g = grid_for(spec_elems(m));
    QAF_BY_DTYPE(m, (vel_kernel<float><<<g, 256, 0, st>>>(geo(m), (const cplx<float>*)w, (cplx<float>*)u, (cplx<float>*)v)),
                    (vel_kernel<double><<<g, 256, 0, st>>>(geo(m), (const cplx<double>*)w, (cplx<double>*)u, (cplx<double>*)v)));
    return post_launch("qaf_vel");
}

qaf_status qaf_dealias(qaf_mesh* m, void* spec, void* stream) {
    QAF_TRY(check_mesh(m));
    if (!spec) return fail(QAF_ERR_INVALID, "null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    int g = grid_for(spec_elems(m));
    QAF_BY_DTYPE(m, (dealias_kernel<float><<<g, 256, 0, st>>>(geo(m), (cplx<float>*)spec)),
                    (dealias_kernel<double><<<g, 256, 0, st>>>(geo(m), (cplx<double>*)spec)));
    return post_launch("qaf_dealias");
}

qaf_status qaf_if_tables(qaf_mesh* m, const qaf_params* p, int which, void* IF, void* IFh, void* stream) {
    QAF_TRY(check_mesh(m));
    if (!p || !IF || !IFh || (which != 0 && which != 1)) return fail(QAF_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    int g = grid_for(spec_elems(m));
    QAF_BY_DTYPE(m, (if_table_kernel<float><<<g, 256, 0, st>>>(geo(m), which, p->re, p->rf, p->q_lin, p->dt, (float*)IF, (float*)IFh)),
                    (if_table_kernel<double><<<g, 256, 0, st>>>(geo(m), which, p->re, p->rf, p->q_lin, p->dt, (double*)IF, (double*)IFh)));
    return post_launch("qaf_if_tables");
}

qaf_status qaf_integrate(qaf_mesh* m, qaf_integrator integ, int stage, const void* old_spec, void* curr_spec,
                         void* new_spec, const void* nonl_spec, const void* IF, const void* IFh, double dt, void* stream) {
    QAF_TRY(check_mesh(m));
    const int max_stage = integ == QAF_IFRK4 ? 4 : (integ == QAF_IFRK2 ? 2 : 1);
    const int min_stage = integ == QAF_IFE ? 1 : 0;
    if (stage < min_stage || stage > max_stage) return fail(QAF_ERR_INVALID, "bad stage for this integrator");
    if (!old_spec || !new_spec || !IF || !IFh || (stage > 0 && !nonl_spec) || (integ != QAF_IFE && !curr_spec))
        return fail(QAF_ERR_INVALID, "null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = spec_elems(m);
    int g = grid_for(n);
    QAF_BY_DTYPE(m,
        (integrate_kernel<float><<<g, 256, 0, st>>>(n, (int)integ, stage, (const cplx<float>*)old_spec, (cplx<float>*)curr_spec,
            (cplx<float>*)new_spec, (const cplx<float>*)nonl_spec, (const float*)IF, (const float*)IFh, (float)dt)),
        (integrate_kernel<double><<<g, 256, 0, st>>>(n, (int)integ, stage, (const cplx<double>*)old_spec, (cplx<double>*)curr_spec,
            (cplx<double>*)new_spec, (const cplx<double>*)nonl_spec, (const double*)IF, (const double*)IFh, dt)));
    return post_launch("qaf_integrate");
}

static qaf_status check_params(const qaf_params* p) {
    if (!p) return fail(QAF_ERR_INVALID, "null params");
    if (!(p->re > 0) || !(p->er > 0)) return fail(QAF_ERR_INVALID, "re and er must be positive");
    if (p->no_dealias < 0 || p->no_dealias > 2) return fail(QAF_ERR_INVALID, "no_dealias must be 0, 1 or 2");
    if (!std::isfinite(p->dt) || !std::isfinite(p->lambda) || !std::isfinite(p->rf) || !std::isfinite(p->alpha) ||
        !std::isfinite(p->q_lin))
        return fail(QAF_ERR_INVALID, "non-finite parameter");
    return QAF_OK;
}

qaf_status qaf_nonlinear_dbg(qaf_mesh* m, const qaf_params* p, const void* w, const void* r1, const void* r2,
                             void* w_nl, void* r1_nl, void* r2_nl, void* phys_out, void* stream);

qaf_status qaf_nonlinear(qaf_mesh* m, const qaf_params* p, const void* w, const void* r1, const void* r2,
                         void* w_nl, void* r1_nl, void* r2_nl, void* stream) {
    return qaf_nonlinear_dbg(m, p, w, r1, r2, w_nl, r1_nl, r2_nl, nullptr, stream);
}

// qaf_nonlinear with an optional dump of the 13 physical fields of the row
// pass (w r1 r2 u v du/dx du/dy+dv/dx Lap r1 Lap r2 S p11 p12 p21), for tests.
qaf_status qaf_nonlinear_dbg(qaf_mesh* m, const qaf_params* p, const void* w, const void* r1, const void* r2,
                             void* w_nl, void* r1_nl, void* r2_nl, void* phys_out, void* stream) {
    QAF_TRY(check_mesh(m));
    QAF_TRY(check_params(p));
    if (!w || !r1 || !r2 || !w_nl || !r1_nl || !r2_nl) return fail(QAF_ERR_INVALID, "null pointer");
    const void* in[3] = {w, r1, r2};
    void* out[3] = {w_nl, r1_nl, r2_nl};
    return dispatch_grid<OpNonlinear>(m, m, p, (const void* const*)in, (void* const*)out, phys_out, (cudaStream_t)stream);
}

static qaf_status check_advance(qaf_mesh* m, const qaf_params* p, qaf_integrator integ, int nsteps) {
    QAF_TRY(check_mesh(m));
    QAF_TRY(check_params(p));
    if (integ != QAF_IFE && integ != QAF_IFRK2 && integ != QAF_IFRK4) return fail(QAF_ERR_INVALID, "bad integrator");
    if (nsteps < 0) return fail(QAF_ERR_INVALID, "nsteps < 0");
    return QAF_OK;
}

qaf_status qaf_state_load(qaf_mesh* m, const void* w, const void* r1, const void* r2, void* stream) {
    QAF_TRY(check_mesh(m));
    if (!w || !r1 || !r2) return fail(QAF_ERR_INVALID, "null pointer");
    void* st[3] = {const_cast<void*>(w), const_cast<void*>(r1), const_cast<void*>(r2)};
    return dispatch_grid<OpLoad>(m, m, (void* const*)st, (cudaStream_t)stream);
}

qaf_status qaf_state_store(qaf_mesh* m, void* w, void* r1, void* r2, void* stream) {
    QAF_TRY(check_mesh(m));
    if (!w || !r1 || !r2) return fail(QAF_ERR_INVALID, "null pointer");
    if (!m->loaded) return fail(QAF_ERR_INVALID, "no state loaded on this mesh");
    void* st[3] = {w, r1, r2};
    return dispatch_grid<OpStore>(m, m, (void* const*)st, (cudaStream_t)stream);
}

qaf_status qaf_state_advance(qaf_mesh* m, const qaf_params* p, qaf_integrator integ, int nsteps, void* stream) {
    QAF_TRY(check_advance(m, p, integ, nsteps));
    if (!m->loaded) return fail(QAF_ERR_INVALID, "no state loaded on this mesh");
    if (nsteps == 0) return QAF_OK;
    return dispatch_grid<OpAdvance>(m, m, p, (int)integ, nsteps, true, (KernelTimer*)nullptr, (cudaStream_t)stream);
}

qaf_status qaf_state_advance_timed(qaf_mesh* m, const qaf_params* p, qaf_integrator integ, int nsteps, double out_ms[3],
                                   void* stream) {
    QAF_TRY(check_advance(m, p, integ, nsteps));
    if (!m->loaded) return fail(QAF_ERR_INVALID, "no state loaded on this mesh");
    if (!out_ms) return fail(QAF_ERR_INVALID, "null pointer");
    KernelTimer timer;
    qaf_status s = nsteps ? dispatch_grid<OpAdvance>(m, m, p, (int)integ, nsteps, true, &timer, (cudaStream_t)stream) : QAF_OK;
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    double sum[2] = {0, 0};
    int cnt[2] = {0, 0};
    for (size_t k = 0; k < timer.kind.size(); ++k) {
        float ms = 0;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, timer.ev[2 * k], timer.ev[2 * k + 1]);
        sum[timer.kind[k]] += ms;
        cnt[timer.kind[k]] += 1;
    }
    for (cudaEvent_t ev : timer.ev) cudaEventDestroy(ev);
    if (s != QAF_OK) return s;
    if (e != cudaSuccess) return fail(QAF_ERR_CUDA, std::string("qaf_state_advance_timed: ") + cudaGetErrorString(e));
    out_ms[0] = cnt[0] ? sum[0] / cnt[0] : 0.0;
    out_ms[1] = cnt[1] ? sum[1] / cnt[1] : 0.0;
    out_ms[2] = (double)(cnt[0] + cnt[1]);
    return QAF_OK;
}

uint64_t qaf_launch_count(const qaf_mesh* m) { return m ? m->launches : 0; }

qaf_status qaf_test_lose_copy(int slab, unsigned polls) {
    if (slab < 0 || polls < 1) return fail(QAF_ERR_INVALID, "qaf_test_lose_copy: slab >= 0 and polls >= 1");
    g_test_polls.store(polls);
    g_test_drop.store(slab + 1);
    return QAF_OK;
}

qaf_status qaf_step(qaf_mesh* m, const qaf_params* p, qaf_integrator integ, void* w, void* r1, void* r2, int nsteps,
                    void* stream) {
    QAF_TRY(check_advance(m, p, integ, nsteps));
    if (!w || !r1 || !r2) return fail(QAF_ERR_INVALID, "null pointer");
    if (nsteps == 0) return QAF_OK;
    void* st[3] = {w, r1, r2};
    cudaStream_t s = (cudaStream_t)stream;
    QAF_TRY(dispatch_grid<OpLoad>(m, m, (void* const*)st, s));
    QAF_TRY(dispatch_grid<OpAdvance>(m, m, p, (int)integ, nsteps, false, (KernelTimer*)nullptr, s));
    return dispatch_grid<OpStore>(m, m, (void* const*)st, s);
}

qaf_status qaf_step_host(qaf_mesh* m, const qaf_params* p, qaf_integrator integ, void* w, void* r1, void* r2,
                         int nsteps) {
    QAF_TRY(check_mesh(m));
    if (!w || !r1 || !r2) return fail(QAF_ERR_INVALID, "null pointer");
    const size_t bytes = spec_elems(m) * 2 * real_bytes(m);
    void* d = nullptr;
    QAF_CUDA(cudaMalloc(&d, 3 * bytes));
    char* dc = static_cast<char*>(d);
    void* host[3] = {w, r1, r2};
    qaf_status s = QAF_OK;
    for (int f = 0; f < 3 && s == QAF_OK; ++f) {
        cudaError_t e = cudaMemcpy(dc + f * bytes, host[f], bytes, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) s = fail(QAF_ERR_CUDA, std::string("H2D: ") + cudaGetErrorString(e));
    }
    if (s == QAF_OK) s = qaf_step(m, p, integ, dc, dc + bytes, dc + 2 * bytes, nsteps, nullptr);
    for (int f = 0; f < 3 && s == QAF_OK; ++f) {
        cudaError_t e = cudaMemcpy(host[f], dc + f * bytes, bytes, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) s = fail(QAF_ERR_CUDA, std::string("D2H: ") + cudaGetErrorString(e));
    }
    cudaFree(d);
    return s;
}

qaf_status qaf_last_diagnostics(qaf_mesh* m, double out[2]) {
    QAF_TRY(check_mesh(m));
    if (!out) return fail(QAF_ERR_INVALID, "null pointer");
    double h[2] = {0, 0};
    unsigned flags = 0;
    if (m->desc.dtype == QAF_F64) {
        if (!m->wd.block) return fail(QAF_ERR_INVALID, "no step has run on this mesh");
        QAF_CUDA(cudaMemcpy(h, m->wd.diag, sizeof(h), cudaMemcpyDeviceToHost));
        QAF_CUDA(cudaMemcpy(&flags, m->wd.flags, sizeof(flags), cudaMemcpyDeviceToHost));
    } else {
        if (!m->wf.block) return fail(QAF_ERR_INVALID, "no step has run on this mesh");
        QAF_CUDA(cudaMemcpy(h, m->wf.diag, sizeof(h), cudaMemcpyDeviceToHost));
        QAF_CUDA(cudaMemcpy(&flags, m->wf.flags, sizeof(flags), cudaMemcpyDeviceToHost));
    }
    const double n4 = (double)m->desc.nx * m->desc.ny * (double)m->desc.nx * m->desc.ny;
    out[0] = 0.5 * h[1] / n4;   // energy: sum |w|^2 / k^2
    out[1] = 0.5 * h[0] / n4;   // enstrophy: sum |w|^2
    if (flags & FLAG_WAIT_TIMEOUT) return fail(QAF_ERR_CUDA, "a kernel's wait for its own copy timed out");
    if (flags) return fail(QAF_ERR_NONFINITE, "a step produced a non-finite value");
    return QAF_OK;
}

// Checkpoint file: "QAFSTAT1", int32 nx, ny, dtype (0 f32, 1 f64), pad, double lx, ly,
// uint64 step, then the w, r1, r2 spectra in the reference layout (i + j*(nx/2+1)),
// interleaved (re, im), little-endian as the host writes them.
qaf_status qaf_state_save(qaf_mesh* m, const char* path, uint64_t step, void* stream) {
    QAF_TRY(check_mesh(m));
    if (!path) return fail(QAF_ERR_INVALID, "null path");
    if (!m->loaded) return fail(QAF_ERR_INVALID, "no state loaded on this mesh");
    const size_t nb = spec_elems(m) * 2 * real_bytes(m);
    void* d = nullptr;
    QAF_CUDA(cudaMalloc(&d, 3 * nb));
    char* dc = static_cast<char*>(d);
    std::vector<char> h(3 * nb);
    qaf_status s = qaf_state_store(m, dc, dc + nb, dc + 2 * nb, stream);
    cudaError_t e = cudaSuccess;
    if (s == QAF_OK) e = cudaMemcpyAsync(h.data(), d, 3 * nb, cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    cudaFree(d);
    if (s != QAF_OK) return s;
    if (e != cudaSuccess) return fail(QAF_ERR_CUDA, std::string("qaf_state_save: ") + cudaGetErrorString(e));
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(QAF_ERR_INVALID, std::string("cannot write ") + path);
    const int32_t hdr[4] = {m->desc.nx, m->desc.ny, m->desc.dtype == QAF_F64 ? 1 : 0, 0};
    const double geo2[2] = {m->desc.lx, m->desc.ly};
    bool ok = std::fwrite("QAFSTAT1", 1, 8, f) == 8 && std::fwrite(hdr, sizeof(hdr), 1, f) == 1 &&
              std::fwrite(geo2, sizeof(geo2), 1, f) == 1 && std::fwrite(&step, sizeof(step), 1, f) == 1 &&
              std::fwrite(h.data(), 1, h.size(), f) == h.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? QAF_OK : fail(QAF_ERR_INVALID, std::string("short write to ") + path);
}

qaf_status qaf_state_restore(qaf_mesh* m, const char* path, uint64_t* step, void* stream) {
    QAF_TRY(check_mesh(m));
    if (!path) return fail(QAF_ERR_INVALID, "null path");
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(QAF_ERR_INVALID, std::string("cannot read ") + path);
    char magic[8];
    int32_t hdr[4];
    double geo2[2];
    uint64_t st = 0;
    const size_t nb = spec_elems(m) * 2 * real_bytes(m);
    std::vector<char> h(3 * nb);
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "QAFSTAT1", 8) == 0 &&
              std::fread(hdr, sizeof(hdr), 1, f) == 1 && std::fread(geo2, sizeof(geo2), 1, f) == 1 &&
              std::fread(&st, sizeof(st), 1, f) == 1;
    if (!ok) { std::fclose(f); return fail(QAF_ERR_INVALID, std::string(path) + ": not a qaf state file"); }
    if (hdr[0] != m->desc.nx || hdr[1] != m->desc.ny || hdr[2] != (m->desc.dtype == QAF_F64 ? 1 : 0) ||
        geo2[0] != m->desc.lx || geo2[1] != m->desc.ly) {
        std::fclose(f);
        return fail(QAF_ERR_INVALID, std::string(path) + ": grid, precision or domain differ from the mesh");
    }
    ok = std::fread(h.data(), 1, h.size(), f) == h.size();
    std::fclose(f);
    if (!ok) return fail(QAF_ERR_INVALID, std::string(path) + ": truncated");
    void* d = nullptr;
    QAF_CUDA(cudaMalloc(&d, 3 * nb));
    char* dc = static_cast<char*>(d);
    cudaError_t e = cudaMemcpyAsync(d, h.data(), 3 * nb, cudaMemcpyHostToDevice, (cudaStream_t)stream);
    qaf_status s = e == cudaSuccess ? qaf_state_load(m, dc, dc + nb, dc + 2 * nb, stream)
                                    : fail(QAF_ERR_CUDA, cudaGetErrorString(e));
    if (s == QAF_OK) {
        e = cudaStreamSynchronize((cudaStream_t)stream);   // h and d go out of scope
        if (e != cudaSuccess) s = fail(QAF_ERR_CUDA, cudaGetErrorString(e));
    }
    cudaFree(d);
    if (s == QAF_OK && step) *step = st;
    return s;
}

qaf_status qaf_last_diagnostics_async(qaf_mesh* m, double* out, void* stream) {
    QAF_TRY(check_mesh(m));
    if (!out) return fail(QAF_ERR_INVALID, "null pointer");
    double* diag = m->desc.dtype == QAF_F64 ? m->wd.diag : m->wf.diag;
    if (!diag) return fail(QAF_ERR_INVALID, "no step has run on this mesh");
    cudaStream_t st = (cudaStream_t)stream;
    const double n4 = (double)m->desc.nx * m->desc.ny * (double)m->desc.nx * m->desc.ny;
    // The kernel stores the two values where the device can address `out`
    // directly: device memory of the current device, or page-locked host
    // memory mapped into the device's address space (the same pointer under
    // unified addressing). A copy operation in the stream would hold the
    // stream's next kernel back for a PCIe round trip (~20-30 us per step);
    // plain stores from the kernel are posted and visible to the host once
    // the stream has been synchronised. Other memory takes the staged copy.
    double* direct = nullptr;
    int dev = 0;
    cudaPointerAttributes pa;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaPointerGetAttributes(&pa, out) == cudaSuccess) {
        if (pa.type == cudaMemoryTypeDevice && pa.device == dev) direct = out;
        else if (pa.type == cudaMemoryTypeHost && pa.devicePointer) direct = static_cast<double*>(pa.devicePointer);
    }
    cudaGetLastError();   // an unregistered host pointer leaves an error behind
    if (direct) {
        diag_finalize_kernel<<<1, 32, 0, st>>>(diag, direct, n4);
        return post_launch("qaf_last_diagnostics_async");
    }
    double* staged = diag + 4 + 512 + 513;
    diag_finalize_kernel<<<1, 32, 0, st>>>(diag, staged, n4);
    QAF_TRY(post_launch("qaf_last_diagnostics_async"));
    QAF_CUDA(cudaMemcpyAsync(out, staged, 2 * sizeof(double), cudaMemcpyDefault, st));
    return QAF_OK;
}

qaf_status qaf_check_finite(qaf_mesh* m, void* stream) {
    QAF_TRY(check_mesh(m));
    QAF_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    unsigned* fp = m->desc.dtype == QAF_F64 ? m->wd.flags : m->wf.flags;
    if (!fp) return QAF_OK;
    unsigned flags = 0;
    QAF_CUDA(cudaMemcpy(&flags, fp, sizeof(flags), cudaMemcpyDeviceToHost));
    QAF_CUDA(cudaMemset(fp, 0, sizeof(unsigned)));
    if (flags & FLAG_WAIT_TIMEOUT) return fail(QAF_ERR_CUDA, "a kernel's wait for its own copy timed out");
    if (flags) return fail(QAF_ERR_NONFINITE, "a step produced a non-finite value");
    return QAF_OK;
}

qaf_status qaf_diagnostics(qaf_mesh* m, const void* w, double* energy, double* enstrophy, double* spectrum, int nshells,
                           void* stream) {
    QAF_TRY(check_mesh(m));
    if (!w) return fail(QAF_ERR_INVALID, "null pointer");
    if (m->desc.dtype == QAF_F64) return diag_impl<double>(m, w, energy, enstrophy, spectrum, nshells, (cudaStream_t)stream);
    return diag_impl<float>(m, w, energy, enstrophy, spectrum, nshells, (cudaStream_t)stream);
}

qaf_status qaf_init_random_q(qaf_mesh* m, uint64_t seed, double lo, double hi, void* w, void* r1, void* r2,
                             void* stream) {
    QAF_TRY(check_mesh(m));
    if (!w || !r1 || !r2) return fail(QAF_ERR_INVALID, "null pointer");
    if (!(hi >= lo)) return fail(QAF_ERR_INVALID, "need lo <= hi");
    const size_t np = phys_elems(m);
    std::vector<double> hw(np), h1(np), h2(np);
    qaf_random_q_init(seed, m->desc.nx, m->desc.ny, lo, hi, hw.data(), h1.data(), h2.data());
    const size_t rb = real_bytes(m);
    void* d = nullptr;
    QAF_CUDA(cudaMalloc(&d, np * rb));
    void* out[3] = {w, r1, r2};
    const std::vector<double>* src[3] = {&hw, &h1, &h2};
    qaf_status st = QAF_OK;
    std::vector<float> tmp;
    for (int f = 0; f < 3 && st == QAF_OK; ++f) {
        const void* hp = src[f]->data();
        if (rb == 4) { tmp.assign(src[f]->begin(), src[f]->end()); hp = tmp.data(); }
        cudaError_t e = cudaMemcpy(d, hp, np * rb, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { st = fail(QAF_ERR_CUDA, std::string("qaf_init_random_q: ") + cudaGetErrorString(e)); break; }
        st = qaf_fwd_trans(m, d, out[f], stream);
        if (st == QAF_OK) {
            e = cudaStreamSynchronize((cudaStream_t)stream);
            if (e != cudaSuccess) st = fail(QAF_ERR_CUDA, std::string("qaf_init_random_q: ") + cudaGetErrorString(e));
        }
    }
    cudaFree(d);
    return st;
}

}  // extern "C"

// ===========================================================================
// Allocation-free step
//
// Some callers cannot allocate device memory at the moment they want to step:
// code that runs while a stream is being captured into a CUDA graph (where
// cudaMalloc is not allowed), hosts whose device memory is owned by a pool or
// arena that a plugin must not bypass, and control loops that must not
// allocate once they are running. qaf_step_noalloc serves them: it runs the
// same fused kernels as qaf_step, with all of its scratch — the working copy of
// the state, the row/column intermediates, twiddles, integrating-factor tables,
// diagnostics and status flags — in one file-scope device array of fixed size
// that every GPU loading this library holds until the process exits. The
// tables are built on the device; nothing is allocated, on the device or on
// the host, on the success path.
// ===========================================================================
namespace {

// Holds the workspace of one grid up to 128 x 128, FP32 or FP64.
constexpr int kNoAllocMaxN = 128;
constexpr size_t kNoAllocBytes = 4u << 20;   // 4 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch per device, looked up once per device
// (with that device current) on the first call made on it.
unsigned char* g_noalloc_ptr[kMaxDevices] = {};
std::mutex g_noalloc_mu;

qaf_status noalloc_scratch(unsigned char** out) {
    int dev = 0;
    QAF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(QAF_ERR_UNSUPPORTED, "qaf_step_noalloc: device index out of range");
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        unsigned char* ptr = nullptr;
        QAF_CUDA(cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch));
        g_noalloc_ptr[dev] = ptr;
    }
    *out = g_noalloc_ptr[dev];
    return QAF_OK;
}

// Workspace element layout inside the fixed array (the same buffers that
// ensure_ws allocates for a mesh), in complex elements of the precision.
template <typename real>
size_t noalloc_carve(Workspace<real>& w, cplx<real>* b, int N) {
    const int H = N / 2;
    const size_t plane = (size_t)N * H;
    size_t off = 0;
    auto take = [&](size_t n) { size_t o = off; off += align_up(n); return o; };
    for (int f = 0; f < 3; ++f) { w.old_m[f] = b + take(plane); w.old_n[f] = b + take(N); }
    for (int f = 0; f < 3; ++f) { w.acc_m[f] = b + take(plane); w.acc_n[f] = b + take(N); }
    w.Y = b + take(NY * plane);
    w.D = b + take((size_t)PF_COUNT * N);
    w.G = b + take(NG * plane);
    w.Ed = b + take((size_t)NE * N);
    w.T = b + take(plane);
    w.tw = b + take(N);
    w.tw_y = w.tw;
    w.ex = reinterpret_cast<real*>(b + take((4 * (H + 1) + 1) / 2 + 1));
    w.ey = reinterpret_cast<real*>(b + take((4 * N + 1) / 2 + 1));
    w.diag = reinterpret_cast<double*>(b + take(4 * sizeof(double) / sizeof(cplx<real>) + 1));
    w.flags = reinterpret_cast<unsigned*>(b + take(1));
    w.queue = reinterpret_cast<int*>(b + take(1));
    w.block = b;
    w.N = N;
    return off * sizeof(cplx<real>);
}

// Twiddles exp(-2 pi i m / N) and the separable integrating factors, built on
// the device (sincospi / exp in double, rounded to the working precision).
template <typename real>
__global__ void noalloc_tables_kernel(cplx<real>* tw, real* ex, real* ey, int N, double dkx, double dky, double dt,
                                      double re) {
    const int H = N / 2;
    const int total = N + 4 * (H + 1) + 4 * N;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        if (k < N) {
            double sn, cs;
            sincospi(-2.0 * (double)k / (double)N, &sn, &cs);
            tw[k] = mk<real>((real)cs, (real)sn);
            continue;
        }
        const bool is_x = k < N + 4 * (H + 1);
        const int r = is_x ? k - N : k - N - 4 * (H + 1);
        const int per = is_x ? H + 1 : N;
        const int c = r / per, idx = r % per;
        const double step = (c == 0 || c == 2) ? dt : 0.5 * dt;
        const double visc = c < 2 ? 1.0 / re : 1.0;
        const double kk = is_x ? dkx * idx : dky * (idx < N / 2 + 1 ? idx : idx - N);
        const real val = (real)exp(-visc * kk * kk * step);
        if (is_x) ex[r] = val; else ey[r] = val;
    }
}

struct OpStepNoAlloc {
    template <typename real, int N>
    static qaf_status run(qaf_mesh* m, unsigned char* scratch, const qaf_params* p, int integ, void* const* state,
                          int nsteps, void* status, cudaStream_t st) {
        if (N > kNoAllocMaxN) return fail(QAF_ERR_INVALID, "qaf_step_noalloc: grid larger than 128 x 128");
        Workspace<real>& w = ws<real>(m);
        const size_t need = noalloc_carve<real>(w, reinterpret_cast<cplx<real>*>(scratch), N);
        if (need > kNoAllocBytes) return fail(QAF_ERR_INVALID, "qaf_step_noalloc: workspace exceeds the fixed scratch");
        QAF_TRY(encode_g_map<real>(&w.tm_G, w.G, N, N));
        QAF_TRY((Launch<real, N>::setup()));
        noalloc_tables_kernel<real><<<8, 256, 0, st>>>(w.tw, w.ex, w.ey, N, m->dkx, m->dky, p->dt, p->re);
        // the array keeps the previous call's contents: clear the status flags
        QAF_CUDA(cudaMemsetAsync(w.flags, 0, sizeof(unsigned), st));
        w.e0[0] = (real)exp(-p->rf / p->re * p->dt);
        w.e0[1] = (real)exp(-p->rf / p->re * p->dt * 0.5);
        w.e0[2] = (real)exp(p->q_lin * p->dt);
        w.e0[3] = (real)exp(p->q_lin * p->dt * 0.5);
        for (int f = 0; f < 3; ++f)
            ref_to_internal<real><<<grid_for(spec_elems(m)), 256, 0, st>>>(
                reinterpret_cast<const cplx<real>*>(state[f]), w.old_m[f], w.old_n[f], N, N);
        StageArgs<real> a = make_args<real>(m, p);
        a.integrator = integ;
        const int nst = integ == QAF_IFRK4 ? 4 : (integ == QAF_IFRK2 ? 2 : 1);
        a.mode = MODE_PROLOGUE;
        a.do_inverse = 1;
        QAF_CUDA(cudaMemsetAsync(w.queue, 0, sizeof(int), st));
        Launch<real, N>::col(a, st);
        a.mode = MODE_STAGE;
        for (int s = 0; s < nsteps; ++s) {
            const bool last_step = s == nsteps - 1;
            if (last_step) QAF_CUDA(cudaMemsetAsync(w.diag, 0, 2 * sizeof(double), st));
            for (int k = 1; k <= nst; ++k) {
                a.stage = k;
                a.last_stage = k == nst;
                a.do_inverse = !(last_step && k == nst);
                a.diag = (last_step && k == nst) ? w.diag : nullptr;
                Launch<real, N>::row(a, st);
                Launch<real, N>::col(a, st);
            }
        }
        for (int f = 0; f < 3; ++f)
            from_internal<real>(m, w.old_m[f], w.old_n[f], state[f], st);
        QAF_TRY(post_launch("qaf_step_noalloc"));
        // the call's status flags, in stream order, for the caller to read
        // once the stream has reached this point
        if (status) QAF_CUDA(cudaMemcpyAsync(status, w.flags, sizeof(unsigned), cudaMemcpyDefault, st));
        return QAF_OK;
    }
};

}  // namespace

extern "C" qaf_status qaf_step_noalloc(int n, double lx, double ly, qaf_dtype dtype, const qaf_params* p,
                                       qaf_integrator integ, void* w, void* r1, void* r2, int nsteps, void* status,
                                       void* stream) {
    if (!p || !w || !r1 || !r2) return fail(QAF_ERR_INVALID, "qaf_step_noalloc: null pointer");
    if (n < 16 || n > kNoAllocMaxN || (n & (n - 1)))
        return fail(QAF_ERR_INVALID, "qaf_step_noalloc: n must be a power of two in [16, 128] "
                                     "(the fixed scratch holds the workspace of a 128 x 128 grid)");
    if (dtype != QAF_F32 && dtype != QAF_F64) return fail(QAF_ERR_INVALID, "qaf_step_noalloc: bad dtype");
    if (!(lx > 0) || !(ly > 0)) return fail(QAF_ERR_INVALID, "qaf_step_noalloc: lx, ly must be positive");
    QAF_TRY(check_params(p));
    if (integ != QAF_IFE && integ != QAF_IFRK2 && integ != QAF_IFRK4) return fail(QAF_ERR_INVALID, "bad integrator");
    if (nsteps < 0) return fail(QAF_ERR_INVALID, "nsteps < 0");
    if (nsteps == 0) {
        if (status) QAF_CUDA(cudaMemsetAsync(status, 0, sizeof(unsigned), (cudaStream_t)stream));
        return QAF_OK;
    }
    unsigned char* scratch = nullptr;
    QAF_TRY(noalloc_scratch(&scratch));
    // a mesh description on the stack whose workspace points into the fixed array
    qaf_mesh m;
    m.desc = qaf_mesh_desc{n, n, lx, ly, dtype};
    m.nxh = n / 2 + 1;
    m.dkx = 2 * M_PI / lx;
    m.dky = 2 * M_PI / ly;
    QAF_CUDA(cudaGetDevice(&m.device));
    void* st[3] = {w, r1, r2};
    return dispatch<OpStepNoAlloc>(&m, &m, scratch, p, (int)integ, (void* const*)st, nsteps, status,
                                   (cudaStream_t)stream);
}

// ===========================================================================
// Ensembles: many independent instances of mixed grid size and parameters,
// advanced together. Instances of one grid size form a group whose buffers
// share one allocation with a fixed per-instance stride, so each row or
// column launch serves the whole group (the row grid spans every instance's
// rows, the persistent column kernel's queue every instance's tiles). One
// step of all groups is captured once into a CUDA graph, the groups as
// parallel branches, and replayed per step.
// ===========================================================================
namespace {

template <typename real>
struct EnsGroup {
    int N = 0, ninst = 0;
    std::vector<int> members;       // ensemble instance ids in group order
    size_t istride = 0;             // complex elements per instance
    cplx<real>* block = nullptr;    // ninst * istride: per-instance buffers
    void* shared = nullptr;         // tables, per-instance parameters, diagnostics, status
    Workspace<real> w;              // instance-0 pointers and the shared tables
    real* inst_alpha = nullptr;
    real* inst_e0 = nullptr;
    double* diag = nullptr;         // 2 per instance
    real* alpha_fields = nullptr;   // per-instance activity fields (N*N each), or nullptr: inst_alpha
};

// per-instance buffer layout (complex elements), returned size rounded up to
// a multiple of H so that instance k's G rows start at row k*istride/H
template <typename real>
size_t carve_instance(Workspace<real>& w, cplx<real>* b, int N) {
    const int H = N / 2;
    const size_t plane = (size_t)N * H;
    size_t off = 0;
    auto take = [&](size_t n) { size_t o = off; off += align_up(n); return o; };
    for (int f = 0; f < 3; ++f) { w.old_m[f] = b + take(plane); w.old_n[f] = b + take(N); }
    for (int f = 0; f < 3; ++f) { w.acc_m[f] = b + take(plane); w.acc_n[f] = b + take(N); }
    w.Y = b + take(NY * plane);
    w.D = b + take((size_t)PF_COUNT * N);
    w.G = b + take(NG * plane);
    w.Ed = b + take((size_t)NE * N);
    // a multiple of H (instance k's G rows start at tensor-map row k * istride / H)
    // and of the 32-element alignment of every buffer
    const size_t unit = (size_t)H / gcd_c(H, 32) * 32;
    return (off + unit - 1) / unit * unit;
}

}  // namespace

struct qaf_ensemble {
    qaf_dtype dtype;
    double lx, ly;
    qaf_params p;
    int ninst;
    std::vector<int> n_of;
    std::vector<std::pair<int, int>> where;   // instance -> (group, slot)
    std::vector<EnsGroup<float>> gf;
    std::vector<EnsGroup<double>> gd;
    bool y_valid = false;
    cudaStream_t cap = nullptr;
    std::vector<cudaStream_t> gstream;
    std::vector<cudaEvent_t> gevent;
    cudaEvent_t fork = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    void* staging = nullptr;          // pinned host copy of the per-instance controls
    size_t staging_bytes = 0;
    cudaEvent_t staged = nullptr;     // the last upload from `staging` has been read
};

namespace {

template <typename real> std::vector<EnsGroup<real>>& groups(qaf_ensemble* e);
template <> std::vector<EnsGroup<float>>& groups<float>(qaf_ensemble* e) { return e->gf; }
template <> std::vector<EnsGroup<double>>& groups<double>(qaf_ensemble* e) { return e->gd; }


template <typename real>
StageArgs<real> group_args(const qaf_ensemble* e, const EnsGroup<real>& g) {
    StageArgs<real> a;
    std::memset(&a, 0, sizeof(a));
    const int N = g.N;
    a.dkx = (real)(2 * M_PI / e->lx); a.dky = (real)(2 * M_PI / e->ly);
    a.lambda = (real)e->p.lambda; a.ce = (real)(1.0 / (e->p.er * e->p.re)); a.alpha = (real)e->p.alpha;
    a.dt = (real)e->p.dt; a.advect = e->p.advect_omega ? 1 : 0;
    a.nx = N; a.ny = N;
    set_mask(a, N, N, e->p.no_dealias);
    for (int f = 0; f < 3; ++f) {
        a.old_m[f] = g.w.old_m[f]; a.old_n[f] = g.w.old_n[f]; a.acc_m[f] = g.w.acc_m[f]; a.acc_n[f] = g.w.acc_n[f];
        a.nl_m[f] = g.w.acc_m[f]; a.nl_n[f] = g.w.acc_n[f];
    }
    a.Y = g.w.Y; a.D = g.w.D; a.G = g.w.G; a.Ed = g.w.Ed; a.tw = g.w.tw; a.tw_y = g.w.tw; a.ex = g.w.ex; a.ey = g.w.ey;
    a.flags = g.w.flags; a.queue = g.w.queue; a.tm_G = g.w.tm_G;
    a.ninst = g.ninst; a.istride = g.istride;
    a.inst_alpha = g.inst_alpha; a.inst_e0 = g.inst_e0;
    if (g.alpha_fields) { a.alpha_field = g.alpha_fields; a.alpha_istride = (size_t)N * N; }
    a.diag = g.diag; a.diag_istride = 2;
    a.integrator = INT_IFRK4;
    return a;
}

template <typename real>
qaf_status build_groups(qaf_ensemble* e, const double* alpha, const double* rf) {
    auto& G = groups<real>(e);
    std::vector<int> sizes(e->n_of);
    std::sort(sizes.begin(), sizes.end());
    sizes.erase(std::unique(sizes.begin(), sizes.end()), sizes.end());
    e->where.assign(e->ninst, {-1, -1});
    for (int N : sizes) {
        EnsGroup<real> g;
        g.N = N;
        for (int k = 0; k < e->ninst; ++k)
            if (e->n_of[k] == N) { e->where[k] = {(int)G.size(), (int)g.members.size()}; g.members.push_back(k); }
        g.ninst = (int)g.members.size();
        Workspace<real> probe;
        g.istride = carve_instance<real>(probe, nullptr, N);
        cplx<real>* blk = nullptr;
        cudaError_t er = cudaMalloc((void**)&blk, g.istride * g.ninst * sizeof(cplx<real>));
        if (er != cudaSuccess) return fail(QAF_ERR_ALLOC, std::string("ensemble cudaMalloc: ") + cudaGetErrorString(er));
        g.block = blk;
        carve_instance<real>(g.w, blk, N);
        // shared: tw (N), ex (4(H+1)), ey (4N), alpha (ninst), e0 (4 ninst), diag (2 ninst), flags, queue
        const int H = N / 2;
        const size_t bytes = N * sizeof(cplx<real>) + (4 * (H + 1) + 4 * N + 5 * (size_t)g.ninst) * sizeof(real) +
                             2 * (size_t)g.ninst * sizeof(double) + 256;
        void* sh = nullptr;
        er = cudaMalloc(&sh, bytes);
        if (er != cudaSuccess) return fail(QAF_ERR_ALLOC, std::string("ensemble cudaMalloc: ") + cudaGetErrorString(er));
        g.shared = sh;
        char* c = static_cast<char*>(sh);
        g.diag = reinterpret_cast<double*>(c); c += 2 * (size_t)g.ninst * sizeof(double);
        g.w.tw = reinterpret_cast<cplx<real>*>(c); c += N * sizeof(cplx<real>);
        g.w.ex = reinterpret_cast<real*>(c); c += 4 * (H + 1) * sizeof(real);
        g.w.ey = reinterpret_cast<real*>(c); c += 4 * (size_t)N * sizeof(real);
        g.inst_alpha = reinterpret_cast<real*>(c); c += g.ninst * sizeof(real);
        g.inst_e0 = reinterpret_cast<real*>(c); c += 4 * (size_t)g.ninst * sizeof(real);
        c = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(c) + 15) & ~uintptr_t(15));
        g.w.flags = reinterpret_cast<unsigned*>(c); c += 16;
        g.w.queue = reinterpret_cast<int*>(c);
        // host-built tables, the same as a single mesh's
        const std::vector<cplx<real>> tw = host_twiddles<real>(N);
        std::vector<real> ex, ey, ia(g.ninst), ie0(4 * (size_t)g.ninst);
        host_if_tables<real>(N, N, 2 * M_PI / e->lx, 2 * M_PI / e->ly, e->p.dt, e->p.re, ex, ey);
        for (int s2 = 0; s2 < g.ninst; ++s2) {
            const int k = g.members[s2];
            ia[s2] = (real)alpha[k];
            host_if_e0<real>(e->p.dt, e->p.re, rf[k], e->p.q_lin, &ie0[4 * (size_t)s2]);
        }
        QAF_CUDA(cudaMemcpy(g.w.tw, tw.data(), tw.size() * sizeof(cplx<real>), cudaMemcpyHostToDevice));
        QAF_CUDA(cudaMemcpy(g.w.ex, ex.data(), ex.size() * sizeof(real), cudaMemcpyHostToDevice));
        QAF_CUDA(cudaMemcpy(g.w.ey, ey.data(), ey.size() * sizeof(real), cudaMemcpyHostToDevice));
        QAF_CUDA(cudaMemcpy(g.inst_alpha, ia.data(), ia.size() * sizeof(real), cudaMemcpyHostToDevice));
        QAF_CUDA(cudaMemcpy(g.inst_e0, ie0.data(), ie0.size() * sizeof(real), cudaMemcpyHostToDevice));
        QAF_CUDA(cudaMemset(g.w.flags, 0, 16));
        QAF_CUDA(cudaMemset(g.diag, 0, 2 * (size_t)g.ninst * sizeof(double)));
        // TMA view of every instance's G arrays
        QAF_TRY(encode_g_map<real>(&g.w.tm_G, g.w.G, N, N, (size_t)(g.ninst - 1) * (g.istride / H) + (size_t)NG * N));
        qaf_status st = with_n(N, [&](auto n) -> qaf_status { return Launch<real, decltype(n)::value>::setup(); });
        if (st != QAF_OK) return st;
        G.push_back(g);
    }
    return QAF_OK;
}

template <typename real>
qaf_status ens_prologue(qaf_ensemble* e, cudaStream_t st) {
    for (auto& g : groups<real>(e)) {
        StageArgs<real> a = group_args<real>(e, g);
        a.mode = MODE_PROLOGUE;
        a.do_inverse = 1;
        QAF_CUDA(cudaMemsetAsync(g.w.queue, 0, sizeof(int), st));
        qaf_status s2 = with_n(g.N, [&](auto n) -> qaf_status {
            Launch<real, decltype(n)::value>::col(a, st);
            return QAF_OK;
        });
        if (s2 != QAF_OK) return s2;
    }
    return post_launch("ensemble prologue");
}

// one IF-RK4 step of every group, each group on its own stream
template <typename real>
qaf_status ens_capture(qaf_ensemble* e) {
    auto& G = groups<real>(e);
    QAF_CUDA(cudaStreamBeginCapture(e->cap, cudaStreamCaptureModeThreadLocal));
    QAF_CUDA(cudaEventRecord(e->fork, e->cap));
    for (size_t gi = 0; gi < G.size(); ++gi) {
        auto& g = G[gi];
        cudaStream_t st = e->gstream[gi];
        QAF_CUDA(cudaStreamWaitEvent(st, e->fork, 0));
        QAF_CUDA(cudaMemsetAsync(g.diag, 0, 2 * (size_t)g.ninst * sizeof(double), st));
        StageArgs<real> a = group_args<real>(e, g);
        a.mode = MODE_STAGE;
        a.do_inverse = 1;
        qaf_status s2 = with_n(g.N, [&](auto n) -> qaf_status {
            for (int k = 1; k <= 4; ++k) {
                a.stage = k;
                a.last_stage = k == 4;
                Launch<real, decltype(n)::value>::row(a, st);
                Launch<real, decltype(n)::value>::col(a, st);
            }
            return QAF_OK;
        });
        if (s2 != QAF_OK) return s2;
        QAF_CUDA(cudaEventRecord(e->gevent[gi], st));
        QAF_CUDA(cudaStreamWaitEvent(e->cap, e->gevent[gi], 0));
    }
    QAF_CUDA(cudaStreamEndCapture(e->cap, &e->graph));
    QAF_CUDA(cudaGraphInstantiate(&e->exec, e->graph, 0));
    return QAF_OK;
}

qaf_status check_ens(const qaf_ensemble* e, int inst) {
    if (!e) return fail(QAF_ERR_INVALID, "null ensemble");
    if (inst < 0 || inst >= e->ninst) return fail(QAF_ERR_INVALID, "instance index out of range");
    return QAF_OK;
}

template <typename real>
qaf_status ens_copy(qaf_ensemble* e, int inst, void* const* st3, bool load, cudaStream_t st) {
    auto& g = groups<real>(e)[e->where[inst].first];
    const size_t io = (size_t)e->where[inst].second * g.istride;
    const size_t n = (size_t)(g.N / 2 + 1) * g.N;
    for (int f = 0; f < 3; ++f) {
        if (load)
            ref_to_internal<real><<<grid_for(n), 256, 0, st>>>(reinterpret_cast<const cplx<real>*>(st3[f]),
                                                             g.w.old_m[f] + io, g.w.old_n[f] + io, g.N, g.N);
        else
            internal_to_ref<real><<<grid_for(n), 256, 0, st>>>(g.w.old_m[f] + io, g.w.old_n[f] + io,
                                                             reinterpret_cast<cplx<real>*>(st3[f]), g.N, g.N);
    }
    if (load) e->y_valid = false;
    return post_launch(load ? "qaf_ensemble_load" : "qaf_ensemble_store");
}

// per-instance alpha and e0 of every group, packed group after group
template <typename real>
qaf_status ens_controls(qaf_ensemble* e, const double* alpha, const double* rf, cudaStream_t st) {
    auto& G = groups<real>(e);
    size_t need = 0;
    for (auto& g : G) need += 5 * (size_t)g.ninst * sizeof(real);
    if (!e->staging) {
        QAF_CUDA(cudaMallocHost(&e->staging, need));
        e->staging_bytes = need;
        QAF_CUDA(cudaEventCreateWithFlags(&e->staged, cudaEventDisableTiming));
    } else {
        QAF_CUDA(cudaEventSynchronize(e->staged));   // the previous upload has left the buffer
    }
    real* h = static_cast<real*>(e->staging);
    for (auto& g : G) {
        real* ha = h;
        real* he = h + g.ninst;
        for (int s2 = 0; s2 < g.ninst; ++s2) {
            const int k = g.members[s2];
            ha[s2] = (real)alpha[k];
            host_if_e0<real>(e->p.dt, e->p.re, rf[k], e->p.q_lin, he + 4 * (size_t)s2);
        }
        QAF_CUDA(cudaMemcpyAsync(g.inst_alpha, ha, g.ninst * sizeof(real), cudaMemcpyHostToDevice, st));
        QAF_CUDA(cudaMemcpyAsync(g.inst_e0, he, 4 * (size_t)g.ninst * sizeof(real), cudaMemcpyHostToDevice, st));
        h += 5 * (size_t)g.ninst;
    }
    QAF_CUDA(cudaEventRecord(e->staged, st));
    return QAF_OK;
}

template <typename real>
void ens_free(qaf_ensemble* e) {
    for (auto& g : groups<real>(e)) {
        if (g.block) cudaFree(g.block);
        if (g.shared) cudaFree(g.shared);
    }
}

}  // namespace

extern "C" {

qaf_status qaf_ensemble_create(int ninst, const int* n, double lx, double ly, qaf_dtype dtype, const qaf_params* p,
                               const double* alpha, const double* rf, qaf_ensemble** out) {
    if (!out || !n || !p || !alpha || !rf) return fail(QAF_ERR_INVALID, "null argument");
    *out = nullptr;
    if (ninst < 1) return fail(QAF_ERR_INVALID, "need at least one instance");
    if (!(lx > 0) || !(ly > 0)) return fail(QAF_ERR_INVALID, "lx, ly must be positive");
    if (dtype != QAF_F32 && dtype != QAF_F64) return fail(QAF_ERR_INVALID, "bad dtype");
    QAF_TRY(check_params(p));
    for (int k = 0; k < ninst; ++k) {
        if (!qaf_supported(n[k], dtype)) return fail(QAF_ERR_UNSUPPORTED, "an instance grid size has no kernels");
        if (!std::isfinite(alpha[k]) || !std::isfinite(rf[k])) return fail(QAF_ERR_INVALID, "non-finite alpha or rf");
    }
    qaf_ensemble* e = new qaf_ensemble();
    e->dtype = dtype; e->lx = lx; e->ly = ly; e->p = *p; e->p.alpha_field = nullptr; e->ninst = ninst;
    e->n_of.assign(n, n + ninst);
    qaf_status s = dtype == QAF_F64 ? build_groups<double>(e, alpha, rf) : build_groups<float>(e, alpha, rf);
    const size_t ng = dtype == QAF_F64 ? e->gd.size() : e->gf.size();
    if (s == QAF_OK) {
        cudaError_t er = cudaStreamCreateWithFlags(&e->cap, cudaStreamNonBlocking);
        if (er == cudaSuccess) er = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming);
        for (size_t gi = 0; gi < ng && er == cudaSuccess; ++gi) {
            cudaStream_t st;
            cudaEvent_t ev;
            er = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
            if (er == cudaSuccess) { e->gstream.push_back(st); er = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming); }
            if (er == cudaSuccess) e->gevent.push_back(ev);
        }
        if (er != cudaSuccess) s = fail(QAF_ERR_CUDA, std::string("ensemble streams: ") + cudaGetErrorString(er));
    }
    if (s == QAF_OK) s = dtype == QAF_F64 ? ens_capture<double>(e) : ens_capture<float>(e);
    if (s != QAF_OK) {
        qaf_ensemble_destroy(e);
        return s;
    }
    *out = e;
    return QAF_OK;
}

qaf_status qaf_ensemble_destroy(qaf_ensemble* e) {
    if (!e) return QAF_OK;
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    for (cudaStream_t st : e->gstream) cudaStreamDestroy(st);
    for (cudaEvent_t ev : e->gevent) cudaEventDestroy(ev);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->cap) cudaStreamDestroy(e->cap);
    if (e->staged) { cudaEventSynchronize(e->staged); cudaEventDestroy(e->staged); }
    if (e->staging) cudaFreeHost(e->staging);
    if (e->dtype == QAF_F64) ens_free<double>(e); else ens_free<float>(e);
    delete e;
    return QAF_OK;
}

qaf_status qaf_ensemble_load(qaf_ensemble* e, int inst, const void* w, const void* r1, const void* r2, void* stream) {
    QAF_TRY(check_ens(e, inst));
    if (!w || !r1 || !r2) return fail(QAF_ERR_INVALID, "null pointer");
    void* st3[3] = {const_cast<void*>(w), const_cast<void*>(r1), const_cast<void*>(r2)};
    return e->dtype == QAF_F64 ? ens_copy<double>(e, inst, st3, true, (cudaStream_t)stream)
                               : ens_copy<float>(e, inst, st3, true, (cudaStream_t)stream);
}

qaf_status qaf_ensemble_store(qaf_ensemble* e, int inst, void* w, void* r1, void* r2, void* stream) {
    QAF_TRY(check_ens(e, inst));
    if (!w || !r1 || !r2) return fail(QAF_ERR_INVALID, "null pointer");
    void* st3[3] = {w, r1, r2};
    return e->dtype == QAF_F64 ? ens_copy<double>(e, inst, st3, false, (cudaStream_t)stream)
                               : ens_copy<float>(e, inst, st3, false, (cudaStream_t)stream);
}

qaf_status qaf_ensemble_advance(qaf_ensemble* e, int nsteps, void* stream) {
    QAF_TRY(check_ens(e, 0));
    if (nsteps < 0) return fail(QAF_ERR_INVALID, "nsteps < 0");
    cudaStream_t st = (cudaStream_t)stream;
    if (!e->y_valid) {
        QAF_TRY(e->dtype == QAF_F64 ? ens_prologue<double>(e, st) : ens_prologue<float>(e, st));
        e->y_valid = true;
    }
    for (int s = 0; s < nsteps; ++s) QAF_CUDA(cudaGraphLaunch(e->exec, st));
    return QAF_OK;
}

qaf_status qaf_ensemble_set_controls(qaf_ensemble* e, const double* alpha, const double* rf, void* stream) {
    QAF_TRY(check_ens(e, 0));
    if (!alpha || !rf) return fail(QAF_ERR_INVALID, "null pointer");
    for (int k = 0; k < e->ninst; ++k)
        if (!std::isfinite(alpha[k]) || !std::isfinite(rf[k])) return fail(QAF_ERR_INVALID, "non-finite alpha or rf");
    return e->dtype == QAF_F64 ? ens_controls<double>(e, alpha, rf, (cudaStream_t)stream)
                               : ens_controls<float>(e, alpha, rf, (cudaStream_t)stream);
}

qaf_status qaf_ensemble_diagnostics(qaf_ensemble* e, double* out, void* stream) {
    QAF_TRY(check_ens(e, 0));
    if (!out) return fail(QAF_ERR_INVALID, "null pointer");
    QAF_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    unsigned flags = 0;
    auto gather = [&](auto& G) -> qaf_status {
        for (auto& g : G) {
            std::vector<double> h(2 * (size_t)g.ninst);
            unsigned fl = 0;
            QAF_CUDA(cudaMemcpy(h.data(), g.diag, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
            QAF_CUDA(cudaMemcpy(&fl, g.w.flags, sizeof(fl), cudaMemcpyDeviceToHost));
            flags |= fl;
            const double n4 = (double)g.N * g.N * (double)g.N * g.N;
            for (int s2 = 0; s2 < g.ninst; ++s2) {
                out[2 * g.members[s2] + 0] = 0.5 * h[2 * s2 + 1] / n4;
                out[2 * g.members[s2] + 1] = 0.5 * h[2 * s2 + 0] / n4;
            }
        }
        return QAF_OK;
    };
    QAF_TRY(e->dtype == QAF_F64 ? gather(e->gd) : gather(e->gf));
    if (flags & FLAG_WAIT_TIMEOUT) return fail(QAF_ERR_CUDA, "a kernel's wait for its own copy timed out");
    if (flags) return fail(QAF_ERR_NONFINITE, "an instance produced a non-finite value");
    return QAF_OK;
}

qaf_status qaf_ensemble_init_random(qaf_ensemble* e, const uint64_t* seeds, double lo, double hi, void* stream) {
    QAF_TRY(check_ens(e, 0));
    if (!seeds) return fail(QAF_ERR_INVALID, "null seeds");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t rb = e->dtype == QAF_F64 ? 8 : 4;
    const int nmax = *std::max_element(e->n_of.begin(), e->n_of.end());
    const size_t smax = (size_t)(nmax / 2 + 1) * nmax * 2 * rb;
    void* buf = nullptr;
    if (cudaMalloc(&buf, 3 * smax) != cudaSuccess) return fail(QAF_ERR_ALLOC, "ensemble init cudaMalloc");
    char* b = static_cast<char*>(buf);
    std::vector<std::pair<int, qaf_mesh*>> meshes;   // one transform mesh per grid size
    qaf_status s = QAF_OK;
    for (int k = 0; k < e->ninst && s == QAF_OK; ++k) {
        const int N = e->n_of[k];
        const size_t sb = (size_t)(N / 2 + 1) * N * 2 * rb;
        qaf_mesh* m = nullptr;
        for (auto& pm : meshes)
            if (pm.first == N) m = pm.second;
        if (!m) {
            qaf_mesh_desc d{N, N, e->lx, e->ly, e->dtype};
            s = qaf_mesh_create(&d, &m);
            if (s != QAF_OK) break;
            meshes.push_back({N, m});
        }
        s = qaf_init_random_q(m, seeds[k], lo, hi, b, b + sb, b + 2 * sb, stream);
        if (s == QAF_OK) s = qaf_ensemble_load(e, k, b, b + sb, b + 2 * sb, stream);
    }
    if (s == QAF_OK) {
        cudaError_t er = cudaStreamSynchronize(st);
        if (er != cudaSuccess) s = fail(QAF_ERR_CUDA, cudaGetErrorString(er));
    }
    cudaFree(buf);
    for (auto& pm : meshes) qaf_mesh_destroy(pm.second);
    return s;
}

}  // extern "C"

// ===========================================================================
// Discrete adjoint of IF-RK4 (gradients of a mean-enstrophy loss and of the
// final state with respect to the initial spectra and the activity field).
// The forward run keeps the state every K steps; the backward sweep, segment
// by segment from the last, reruns the segment's K steps from its checkpoint
// recording each stage input's nine physical fields and the vorticity after
// each step, then walks the steps backwards through the adjoint kernels.
// ===========================================================================
struct qaf_adjoint {
    qaf_mesh* m = nullptr;
    int nsteps = 0, K = 0, window = 0, nseg = 0;
    size_t ns = 0, np = 0, rb = 0;
    unsigned char* blk = nullptr;
    unsigned char *ckpt = nullptr, *wlog = nullptr, *phys = nullptr, *Tg = nullptr, *Tx = nullptr;
    unsigned char *abar = nullptr, *sacc = nullptr, *sbar = nullptr, *edge = nullptr, *agrad = nullptr;
    double* loss = nullptr;
    qaf_params p{};
    bool have_forward = false;
};

namespace {

// what a recording advance keeps
struct AdjRecord {
    void* phys;           // 4 slots of PF_COUNT * N * N reals per step, or nullptr
    void* wlog;           // w after each step (reference layout), or nullptr
    double* loss;         // += weight * enstrophy sum of the state after each step >= loss_from
    int loss_from;
    double loss_weight;
};

// IF-RK4 steps of the resident state, as OpAdvance, with the recording above
struct OpRecord {
    template <typename real, int N>
    static qaf_status run(qaf_mesh* m, const qaf_params* p, int nsteps, const AdjRecord* rec, cudaStream_t st) {
        QAF_TRY(ensure_ws<real>(m));
        QAF_TRY((Launch<real, N>::setup()));
        QAF_TRY(ensure_if<real>(m, p, st));
        Workspace<real>& w = ws<real>(m);
        StageArgs<real> a = make_args<real>(m, p);
        a.integrator = INT_IFRK4;
        if (!m->y_valid) {
            a.mode = MODE_PROLOGUE; a.do_inverse = 1;
            QAF_CUDA(cudaMemsetAsync(w.queue, 0, sizeof(int), st));
            Launch<real, N>::col(a, st);
            m->launches += 1;
        }
        a.mode = MODE_STAGE;
        a.do_inverse = 1;
        const size_t slot = (size_t)PF_COUNT * N * N;
        const size_t ns = (size_t)(N / 2 + 1) * N;
        for (int s = 0; s < nsteps; ++s) {
            const bool lstep = rec->loss && s >= rec->loss_from;
            if (lstep) QAF_CUDA(cudaMemsetAsync(w.diag, 0, 2 * sizeof(double), st));
            for (int k = 1; k <= 4; ++k) {
                a.stage = k;
                a.last_stage = k == 4;
                a.diag = (lstep && k == 4) ? w.diag : nullptr;
                a.phys_out = rec->phys ? static_cast<real*>(rec->phys) + ((size_t)s * 4 + (k - 1)) * slot : nullptr;
                Launch<real, N>::row(a, st);
                Launch<real, N>::col(a, st);
                m->launches += 2;
            }
            if (lstep) { adj_loss_accumulate<<<1, 32, 0, st>>>(w.diag, rec->loss, rec->loss_weight); m->launches += 1; }
            if (rec->wlog) {
                from_internal<real>(m, w.old_m[0], w.old_n[0], static_cast<cplx<real>*>(rec->wlog) + (size_t)s * ns, st);
                m->launches += 1;
            }
        }
        m->y_valid = true;
        return post_launch("adjoint recording advance");
    }
};

template <typename real>
cplx<real>* adj_field(unsigned char* base, size_t ns, int f) { return reinterpret_cast<cplx<real>*>(base) + (size_t)f * ns; }

struct OpAdjForward {
    template <typename real, int N>
    static qaf_status run(qaf_adjoint* A, const void* const* s0, void* const* sT, double* loss, cudaStream_t st) {
        qaf_mesh* m = A->m;
        const size_t ns = A->ns, cb = sizeof(cplx<real>);
        for (int f = 0; f < 3; ++f)
            QAF_CUDA(cudaMemcpyAsync(adj_field<real>(A->ckpt, ns, f), s0[f], ns * cb, cudaMemcpyDeviceToDevice, st));
        QAF_TRY((OpLoad::run<real>(m, const_cast<void* const*>(s0), st)));
        QAF_CUDA(cudaMemsetAsync(A->loss, 0, sizeof(double), st));
        const double n4 = (double)N * N * (double)N * N;
        for (int seg = 0; seg < A->nseg; ++seg) {
            const int t0 = seg * A->K, t1 = std::min(A->nsteps, t0 + A->K);
            AdjRecord rec{nullptr, nullptr, A->window > 0 ? A->loss : nullptr, A->nsteps - A->window - t0,
                          1.0 / ((double)(A->window > 0 ? A->window : 1) * n4)};
            QAF_TRY((OpRecord::run<real, N>(m, &A->p, t1 - t0, &rec, st)));
            if (t1 < A->nsteps) {
                unsigned char* c = A->ckpt + (size_t)(seg + 1) * 3 * ns * cb;
                void* dst[3] = {adj_field<real>(c, ns, 0), adj_field<real>(c, ns, 1), adj_field<real>(c, ns, 2)};
                QAF_TRY((OpStore::run<real>(m, dst, st)));
            }
        }
        if (sT[0] && sT[1] && sT[2]) QAF_TRY((OpStore::run<real>(m, sT, st)));
        double h = 0;
        QAF_CUDA(cudaMemcpyAsync(&h, A->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
        QAF_CUDA(cudaStreamSynchronize(st));
        if (loss) *loss = h;
        return post_launch("qaf_adjoint_forward");
    }
};

struct OpAdjBackward {
    template <typename real, int N>
    static qaf_status run(qaf_adjoint* A, const void* const* gT, double gloss, void* const* g0, void* galpha,
                          cudaStream_t st) {
        using C = Cfg<real, N>;
        constexpr int H = N / 2;
        // column pass: field-parallel (11 transform teams per column, one column per CTA) up to 256^2,
        // W columns per CTA with the transforms in sequence above
        constexpr bool FP = N <= 256;
        // FP32 from 128^2: 2 columns per CTA with 8-value teams (704 threads, 16-byte segments of the
        // T arrays); otherwise one column per CTA with 16-value teams (FP64 keeps its registers)
        constexpr bool W2 = FP && sizeof(real) == 4 && N >= 128;
        constexpr int W = FP ? (W2 ? 2 : 1) : C::W;
        constexpr int P = pow2_size(N);
        constexpr int EC = FP ? fit_e(N, W2 ? P / 32 : (P / 16 > 4 ? P / 16 : 4)) : C::EC;
        constexpr int COL_THREADS = FP ? NGA * W * (N / EC) : W * (N / EC);
        constexpr size_t COL_SMEM = FP ? (size_t)NGA * N * (W > 1 ? W : 2) * sizeof(cplx<real>)
                                       : (size_t)W * N * sizeof(cplx<real>);
        // row pass: field-parallel, teams of H/ER threads (16 from 128^2 up)
        constexpr int ER = fit_e(H, P / 32 < 2 ? 2 : (P / 32 > 16 ? 16 : P / 32));
        constexpr int ROW_THREADS = NGA * (H / ER);
        constexpr size_t ROW_SMEM = (size_t)NGA * H * sizeof(cplx<real>);
        static DeviceOnce attrs;   // kernel attributes, per device
        QAF_TRY(attrs.get(nullptr, [](int*) -> qaf_status {
            if constexpr (FP)
                QAF_CUDA(cudaFuncSetAttribute(adj_colp_kernel<real, N, W, EC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)COL_SMEM));
            else
                QAF_CUDA(cudaFuncSetAttribute(adj_col_kernel<real, N, W, EC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)COL_SMEM));
            QAF_CUDA(cudaFuncSetAttribute(adj_row_kernel<real, N, ER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ROW_SMEM));
            return QAF_OK;
        }));
        qaf_mesh* m = A->m;
        const size_t ns = A->ns, cb = sizeof(cplx<real>);
        const size_t slot = (size_t)PF_COUNT * N * N;
        QAF_TRY(ensure_ws<real>(m));
        QAF_TRY(ensure_if<real>(m, &A->p, st));
        Workspace<real>& w = ws<real>(m);

        AdjArgs<real> a;
        std::memset(&a, 0, sizeof(a));
        a.dkx = (real)m->dkx; a.dky = (real)m->dky; a.dt = (real)A->p.dt; a.lambda = (real)A->p.lambda;
        a.ce = (real)(1.0 / (A->p.er * A->p.re));
        a.advect = A->p.advect_omega ? 1 : 0;
        set_mask(a, N, N, A->p.no_dealias);
        a.tw = w.tw; a.ex = w.ex; a.ey = w.ey;
        for (int c = 0; c < 4; ++c) a.e0[c] = w.e0[c];
        a.Tg = reinterpret_cast<cplx<real>*>(A->Tg); a.Tx = reinterpret_cast<cplx<real>*>(A->Tx);
        for (int f = 0; f < 3; ++f) {
            a.abar[f] = adj_field<real>(A->abar, ns, f);
            a.sacc[f] = adj_field<real>(A->sacc, ns, f);
            a.sbar[f] = adj_field<real>(A->sbar, ns, f);
        }
        a.edge = reinterpret_cast<cplx<real>*>(A->edge);
        a.alpha_field = reinterpret_cast<const real*>(A->p.alpha_field);
        a.alpha = (real)A->p.alpha;
        a.alpha_grad = reinterpret_cast<real*>(A->agrad);
        a.ninst = 1;
        const real lw = (real)(A->window > 0 ? gloss / A->window : 0.0);
        a.loss_w = lw;

        for (int f = 0; f < 3; ++f) {
            if (gT[f]) QAF_CUDA(cudaMemcpyAsync(a.sbar[f], gT[f], ns * cb, cudaMemcpyDeviceToDevice, st));
            else QAF_CUDA(cudaMemsetAsync(a.sbar[f], 0, ns * cb, st));
        }
        QAF_CUDA(cudaMemsetAsync(A->agrad, 0, (size_t)N * N * sizeof(real), st));
        const int T = A->nsteps;
        auto in_window = [&](int n) { return A->window > 0 && gloss != 0.0 && n >= T - A->window + 1; };
        auto col = [&]() {
            if constexpr (FP) adj_colp_kernel<real, N, W, EC><<<H / W + 1, COL_THREADS, COL_SMEM, st>>>(a);
            else adj_col_kernel<real, N, W, EC><<<H / W + 1, COL_THREADS, COL_SMEM, st>>>(a);
            m->launches += 1;
        };
        bool started = false;
        for (int seg = A->nseg - 1; seg >= 0; --seg) {
            const int t0 = seg * A->K, t1 = std::min(T, t0 + A->K);
            unsigned char* c = A->ckpt + (size_t)seg * 3 * ns * cb;
            const void* cs[3] = {adj_field<real>(c, ns, 0), adj_field<real>(c, ns, 1), adj_field<real>(c, ns, 2)};
            QAF_TRY((OpLoad::run<real>(m, const_cast<void* const*>(cs), st)));
            AdjRecord rec{A->phys, A->wlog, nullptr, 0, 0.0};
            QAF_TRY((OpRecord::run<real, N>(m, &A->p, t1 - t0, &rec, st)));
            auto w_at = [&](int n) -> const cplx<real>* {   // w of the state at time n (t0 <= n <= t1)
                if (n == t0) return adj_field<real>(c, ns, 0);
                return reinterpret_cast<const cplx<real>*>(A->wlog) + (size_t)(n - 1 - t0) * ns;
            };
            for (int n = t1 - 1; n >= t0; --n) {
                if (!started) {
                    a.stage = 0; a.emit = 1;
                    a.wstate = in_window(T) ? w_at(T) : nullptr;
                    col();
                    started = true;
                }
                for (int s = 4; s >= 1; --s) {
                    a.phys = reinterpret_cast<const real*>(A->phys) + ((size_t)(n - t0) * 4 + (s - 1)) * slot;
                    adj_row_kernel<real, N, ER><<<N, ROW_THREADS, ROW_SMEM, st>>>(a);
                    m->launches += 1;
                    a.stage = s;
                    a.emit = (s > 1 || n > 0) ? 1 : 0;
                    a.wstate = (s == 1 && in_window(n)) ? w_at(n) : nullptr;
                    col();
                }
            }
        }
        for (int f = 0; f < 3; ++f)
            if (g0[f]) QAF_CUDA(cudaMemcpyAsync(g0[f], a.sbar[f], ns * cb, cudaMemcpyDeviceToDevice, st));
        if (galpha)
            QAF_CUDA(cudaMemcpyAsync(galpha, A->agrad, (size_t)N * N * sizeof(real), cudaMemcpyDeviceToDevice, st));
        return post_launch("qaf_adjoint_backward");
    }
};

}  // namespace

extern "C" {

qaf_status qaf_adjoint_create(qaf_mesh* m, int nsteps, int checkpoint_every, int loss_window, qaf_adjoint** out) {
    QAF_TRY(check_mesh(m));
    if (!out) return fail(QAF_ERR_INVALID, "null output");
    *out = nullptr;
    if (nsteps < 1) return fail(QAF_ERR_INVALID, "nsteps must be >= 1");
    if (checkpoint_every < 1) return fail(QAF_ERR_INVALID, "checkpoint_every must be >= 1");
    if (loss_window < 0 || loss_window > nsteps) return fail(QAF_ERR_INVALID, "loss_window must be in [0, nsteps]");
    if (!qaf_supported(m->desc.nx, m->desc.dtype) || m->desc.nx != m->desc.ny)
        return fail(QAF_ERR_UNSUPPORTED, "no kernels for this grid size");
    qaf_adjoint* A = new qaf_adjoint();
    A->m = m;
    A->nsteps = nsteps;
    A->K = std::min(checkpoint_every, nsteps);
    A->window = loss_window;
    A->nseg = (nsteps + A->K - 1) / A->K;
    const int N = m->desc.nx;
    A->ns = spec_elems(m);
    A->np = phys_elems(m);
    A->rb = real_bytes(m);
    const size_t cb = 2 * A->rb;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
    const size_t o_ck = take((size_t)A->nseg * 3 * A->ns * cb);
    const size_t o_wl = take((size_t)A->K * A->ns * cb);
    const size_t o_ph = take((size_t)A->K * 4 * PF_COUNT * A->np * A->rb);
    const size_t o_tg = take((size_t)NGA * N * (N / 2) * cb);
    const size_t o_tx = take((size_t)PF_COUNT * N * (N / 2) * cb);
    const size_t o_ab = take(3 * A->ns * cb), o_sa = take(3 * A->ns * cb), o_sb = take(3 * A->ns * cb);
    const size_t o_ed = take(6 * (size_t)N * cb);
    const size_t o_ag = take(A->np * A->rb);
    const size_t o_ls = take(sizeof(double));
    cudaError_t e = cudaMalloc((void**)&A->blk, off);
    if (e != cudaSuccess) {
        delete A;
        return fail(QAF_ERR_ALLOC, std::string("qaf_adjoint_create: cudaMalloc of ") + std::to_string(off >> 20) +
                                       " MiB: " + cudaGetErrorString(e));
    }
    A->ckpt = A->blk + o_ck; A->wlog = A->blk + o_wl; A->phys = A->blk + o_ph; A->Tg = A->blk + o_tg;
    A->Tx = A->blk + o_tx; A->abar = A->blk + o_ab; A->sacc = A->blk + o_sa; A->sbar = A->blk + o_sb;
    A->edge = A->blk + o_ed; A->agrad = A->blk + o_ag; A->loss = reinterpret_cast<double*>(A->blk + o_ls);
    *out = A;
    return QAF_OK;
}

qaf_status qaf_adjoint_destroy(qaf_adjoint* A) {
    if (!A) return QAF_OK;
    if (A->blk) cudaFree(A->blk);
    delete A;
    return QAF_OK;
}

qaf_status qaf_adjoint_forward(qaf_adjoint* A, const qaf_params* p, const void* w0, const void* r1_0, const void* r2_0,
                               void* wT, void* r1T, void* r2T, double* loss, void* stream) {
    if (!A) return fail(QAF_ERR_INVALID, "null adjoint");
    QAF_TRY(check_params(p));
    if (!w0 || !r1_0 || !r2_0) return fail(QAF_ERR_INVALID, "null initial state");
    A->p = *p;
    A->have_forward = false;
    const void* s0[3] = {w0, r1_0, r2_0};
    void* sT[3] = {wT, r1T, r2T};
    QAF_TRY(dispatch<OpAdjForward>(A->m, A, (const void* const*)s0, (void* const*)sT, loss, (cudaStream_t)stream));
    A->have_forward = true;
    return QAF_OK;
}

qaf_status qaf_adjoint_backward(qaf_adjoint* A, const void* gwT, const void* gr1T, const void* gr2T, double gloss,
                                void* gw0, void* gr1_0, void* gr2_0, void* galpha, void* stream) {
    if (!A) return fail(QAF_ERR_INVALID, "null adjoint");
    if (!A->have_forward) return fail(QAF_ERR_INVALID, "qaf_adjoint_backward needs a qaf_adjoint_forward first");
    if (!std::isfinite(gloss)) return fail(QAF_ERR_INVALID, "non-finite loss gradient");
    const void* gT[3] = {gwT, gr1T, gr2T};
    void* g0[3] = {gw0, gr1_0, gr2_0};
    return dispatch<OpAdjBackward>(A->m, A, (const void* const*)gT, gloss, (void* const*)g0, galpha,
                                   (cudaStream_t)stream);
}

}  // extern "C"

// ===========================================================================
// Autotuner: times the launch variants of the fused step kernels on a
// synthetic ensemble and keeps the fastest per (precision, grid size,
// batched); the choices persist in a JSON-lines cache.
// ===========================================================================
namespace {

// one IF-RK4 step of every group of the ensemble, launched directly (not the captured graph)
template <typename real>
qaf_status ens_step_direct(qaf_ensemble* e, cudaStream_t st) {
    for (auto& g : groups<real>(e)) {
        StageArgs<real> a = group_args<real>(e, g);
        a.mode = MODE_STAGE;
        a.do_inverse = 1;
        a.diag = nullptr;
        qaf_status s2 = with_n(g.N, [&](auto n) -> qaf_status {
            for (int k = 1; k <= 4; ++k) {
                a.stage = k;
                a.last_stage = k == 4;
                Launch<real, decltype(n)::value>::row(a, st);
                Launch<real, decltype(n)::value>::col(a, st);
            }
            return QAF_OK;
        });
        if (s2 != QAF_OK) return s2;
    }
    return post_launch("autotune step");
}

std::string device_name() {
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        cudaGetLastError();
        return "";
    }
    return prop.name;
}

std::string variant_name(int dtype, int n, int kind, int idx) {
    if (idx < 0) return kind == 0 ? "col:default" : "row:default";
    StepVariant<float>* v = nullptr;
    const int cnt = variant_list(dtype, n, &v);
    return idx < cnt ? v[idx].name : "?";
}

// index of a variant by name: -1 for "<kind>:default" or "default", -2 if unknown
int variant_index(int dtype, int n, int kind, const std::string& name) {
    if (name == "default" || name == (kind == 0 ? "col:default" : "row:default")) return -1;
    StepVariant<float>* v = nullptr;
    const int cnt = variant_list(dtype, n, &v);
    for (int i = 0; i < cnt; ++i)
        if (v[i].kind == kind && name == v[i].name) return i;
    return -2;
}

void set_choice(int dtype, int n, int batched, int col, int row, double us) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    TuneChoice c;
    c.col = col; c.row = row; c.us = us;
    g_tune[std::make_tuple(dtype, n, batched)] = c;
}

// the value of "key": in one JSON-lines record (string or number, as text)
bool json_field(const std::string& line, const std::string& key, std::string& out) {
    const std::string pat = "\"" + key + "\":";
    size_t p = line.find(pat);
    if (p == std::string::npos) return false;
    p += pat.size();
    while (p < line.size() && line[p] == ' ') ++p;
    if (p < line.size() && line[p] == '"') {
        const size_t q = line.find('"', p + 1);
        if (q == std::string::npos) return false;
        out = line.substr(p + 1, q - p - 1);
        return true;
    }
    size_t q = p;
    while (q < line.size() && line[q] != ',' && line[q] != '}') ++q;
    out = line.substr(p, q - p);
    return !out.empty();
}

std::string cache_record(const std::string& dev, int dtype, int n, int batched, int col, int row, double us) {
    std::ostringstream o;
    o << "{\"device\": \"" << dev << "\", \"dtype\": \"" << (dtype == QAF_F64 ? "f64" : "f32") << "\", \"n\": " << n
      << ", \"batched\": " << batched << ", \"col\": \"" << variant_name(dtype, n, 0, col) << "\", \"row\": \""
      << variant_name(dtype, n, 1, row) << "\", \"us_per_step\": " << us << "}";
    return o.str();
}

qaf_status cache_write(const char* path, const std::string& dev, int dtype, int n, int batched, const std::string& rec) {
    std::vector<std::string> keep;
    {
        std::ifstream in(path);
        std::string line;
        while (std::getline(in, line)) {
            std::string d, t, nn, b;
            if (json_field(line, "device", d) && json_field(line, "dtype", t) && json_field(line, "n", nn) &&
                json_field(line, "batched", b) && d == dev && t == (dtype == QAF_F64 ? "f64" : "f32") &&
                std::atoi(nn.c_str()) == n && std::atoi(b.c_str()) == batched)
                continue;   // replaced below
            if (!line.empty()) keep.push_back(line);
        }
    }
    keep.push_back(rec);
    const std::string tmp = std::string(path) + ".tmp";
    {
        std::ofstream out(tmp, std::ios::trunc);
        if (!out) return fail(QAF_ERR_INVALID, std::string("cannot write ") + tmp);
        for (auto& l : keep) out << l << "\n";
    }
    if (std::rename(tmp.c_str(), path) != 0) return fail(QAF_ERR_INVALID, std::string("cannot replace ") + path);
    return QAF_OK;
}

template <typename real>
qaf_status autotune_impl(int n, int ninst, int dtype, double* best_us, int* best_col, int* best_row) {
    std::vector<int> sizes(ninst, n);
    std::vector<double> alpha(ninst, 1.0), rf(ninst, 0.1);
    std::vector<uint64_t> seeds(ninst);
    for (int k = 0; k < ninst; ++k) seeds[k] = 1000 + k;
    qaf_params p{};
    p.re = 1; p.er = 1; p.rf = 0.1; p.lambda = 0.1; p.alpha = 1; p.alpha_field = nullptr; p.dt = 1e-3; p.q_lin = 1;
    p.advect_omega = 1;
    qaf_ensemble* e = nullptr;
    QAF_TRY(qaf_ensemble_create(ninst, sizes.data(), 16 * M_PI, 16 * M_PI, (qaf_dtype)dtype, &p, alpha.data(),
                                rf.data(), &e));
    struct Guard { qaf_ensemble* e; ~Guard() { qaf_ensemble_destroy(e); } } guard{e};
    cudaStream_t st = nullptr;
    QAF_TRY(qaf_ensemble_init_random(e, seeds.data(), -0.01, 0.01, st));
    QAF_TRY(qaf_ensemble_advance(e, 0, st));   // prologue
    const int batched = ninst > 1 ? 1 : 0;
    cudaEvent_t e0, e1;
    QAF_CUDA(cudaEventCreate(&e0));
    QAF_CUDA(cudaEventCreate(&e1));
    auto time_choice = [&](int col, int row, double* us) -> qaf_status {
        set_choice(dtype, n, batched, col, row, 0);
        for (int w = 0; w < 3; ++w) QAF_TRY(ens_step_direct<real>(e, st));
        const int reps = 20;
        QAF_CUDA(cudaEventRecord(e0, st));
        for (int r = 0; r < reps; ++r) QAF_TRY(ens_step_direct<real>(e, st));
        QAF_CUDA(cudaEventRecord(e1, st));
        QAF_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        QAF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        *us = 1e3 * ms / reps;
        return QAF_OK;
    };
    StepVariant<float>* v = nullptr;
    const int cnt = variant_list(dtype, n, &v);
    double t = 0;
    int bc = -1, br = -1;
    qaf_status s = time_choice(-1, -1, &t);
    double bt = t;
    for (int i = 0; i < cnt && s == QAF_OK; ++i) {
        if (v[i].kind != 0) continue;
        s = time_choice(i, -1, &t);
        if (s == QAF_OK && t < bt) { bt = t; bc = i; }
    }
    for (int i = 0; i < cnt && s == QAF_OK; ++i) {
        if (v[i].kind != 1) continue;
        s = time_choice(bc, i, &t);
        if (s == QAF_OK && t < bt) { bt = t; br = i; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s != QAF_OK) {
        set_choice(dtype, n, batched, -1, -1, 0);
        return s;
    }
    set_choice(dtype, n, batched, bc, br, bt);
    *best_us = bt; *best_col = bc; *best_row = br;
    return QAF_OK;
}

}  // namespace

extern "C" {

qaf_status qaf_autotune(int n, qaf_dtype dtype, int ninst, const char* cache_path, char* choice, int choice_len,
                        double* us_per_step) {
    if (!qaf_supported(n, dtype)) return fail(QAF_ERR_UNSUPPORTED, "no kernels for this grid size");
    if (ninst < 1) return fail(QAF_ERR_INVALID, "ninst must be >= 1");
    double us = 0;
    int col = -1, row = -1;
    QAF_TRY(dtype == QAF_F64 ? autotune_impl<double>(n, ninst, dtype, &us, &col, &row)
                             : autotune_impl<float>(n, ninst, dtype, &us, &col, &row));
    const int batched = ninst > 1 ? 1 : 0;
    if (us_per_step) *us_per_step = us;
    if (choice && choice_len > 0) {
        const std::string c = variant_name(dtype, n, 0, col) + " " + variant_name(dtype, n, 1, row);
        std::snprintf(choice, (size_t)choice_len, "%s", c.c_str());
    }
    if (cache_path && *cache_path) {
        const std::string dev = device_name();
        QAF_TRY(cache_write(cache_path, dev, dtype, n, batched, cache_record(dev, dtype, n, batched, col, row, us)));
    }
    return QAF_OK;
}

qaf_status qaf_autotune_load(const char* cache_path) {
    if (!cache_path) return fail(QAF_ERR_INVALID, "null path");
    std::ifstream in(cache_path);
    if (!in) return fail(QAF_ERR_INVALID, std::string("cannot read ") + cache_path);
    const std::string dev = device_name();
    std::string line;
    int used = 0;
    while (std::getline(in, line)) {
        std::string d, t, nn, b, c, r, u;
        if (!(json_field(line, "device", d) && json_field(line, "dtype", t) && json_field(line, "n", nn) &&
              json_field(line, "batched", b) && json_field(line, "col", c) && json_field(line, "row", r)))
            continue;
        if (d != "*" && d != dev) continue;
        const int dtype = t == "f64" ? QAF_F64 : QAF_F32;
        const int n = std::atoi(nn.c_str());
        const int ci = variant_index(dtype, n, 0, c), ri = variant_index(dtype, n, 1, r);
        if (ci < -1 || ri < -1) continue;   // a variant this build does not have
        set_choice(dtype, n, std::atoi(b.c_str()) ? 1 : 0, ci, ri, json_field(line, "us_per_step", u) ? std::atof(u.c_str()) : 0);
        ++used;
    }
    (void)used;
    return QAF_OK;
}

qaf_status qaf_autotune_reset(void) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.clear();
    return QAF_OK;
}

qaf_status qaf_set_variant(int n, qaf_dtype dtype, int batched, const char* col, const char* row) {
    if (!col || !row) return fail(QAF_ERR_INVALID, "null variant name");
    const int ci = variant_index(dtype, n, 0, col), ri = variant_index(dtype, n, 1, row);
    if (ci < -1 || ri < -1) return fail(QAF_ERR_INVALID, "unknown launch variant for this size and precision");
    set_choice(dtype, n, batched ? 1 : 0, ci, ri, 0);
    return QAF_OK;
}

qaf_status qaf_variant_choice(int n, qaf_dtype dtype, int batched, char* buf, int len) {
    if (!buf || len < 1) return fail(QAF_ERR_INVALID, "null buffer");
    int col = -1, row = -1;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(std::make_tuple((int)dtype, n, batched ? 1 : 0));
        if (it != g_tune.end()) { col = it->second.col; row = it->second.row; }
    }
    const std::string c = variant_name(dtype, n, 0, col) + " " + variant_name(dtype, n, 1, row);
    std::snprintf(buf, (size_t)len, "%s", c.c_str());
    return QAF_OK;
}

qaf_status qaf_variant_list(int n, qaf_dtype dtype, char* buf, int len) {
    if (!buf || len < 1) return fail(QAF_ERR_INVALID, "null buffer");
    std::string c = "col:default row:default";
    StepVariant<float>* v = nullptr;
    const int cnt = variant_list(dtype, n, &v);
    for (int i = 0; i < cnt; ++i) c += std::string(" ") + v[i].name;
    std::snprintf(buf, (size_t)len, "%s", c.c_str());
    return QAF_OK;
}

}  // extern "C"

// ===========================================================================
// Batched adjoint: `ninst` instances of one grid size, each with its own
// initial state and activity field, advanced and differentiated together —
// every forward, recompute and adjoint stage is one launch for the whole
// batch (the ensemble's instance-indexed kernels and the instance-indexed
// field-parallel adjoint kernels). Grids up to 256 x 256.
// ===========================================================================
struct qaf_adjoint_batch {
    qaf_ensemble* ens = nullptr;    // ninst instances of size n: forward machinery and tables
    int ninst = 0, n = 0, nsteps = 0, K = 0, window = 0, nseg = 0;
    size_t ns = 0, np = 0;
    unsigned char* blk = nullptr;
    unsigned char *ckpt = nullptr, *wlog = nullptr, *phys = nullptr, *Tg = nullptr, *Tx = nullptr;
    unsigned char *abar = nullptr, *sacc = nullptr, *sbar = nullptr, *agrad = nullptr, *alpha = nullptr, *lossw = nullptr;
    double* loss = nullptr;
    bool have_alpha = false, have_forward = false;
};

namespace {

// spectral arrays of the batch: [field][instance][ns]
template <typename real>
cplx<real>* bfield(unsigned char* base, size_t ns, int ninst, int f) {
    return reinterpret_cast<cplx<real>*>(base) + (size_t)f * ninst * ns;
}

template <typename real>
struct BatchOps {
    static EnsGroup<real>& group(qaf_adjoint_batch* B) { return groups<real>(B->ens)[0]; }

    // load field-major [field][inst][ns] reference-layout spectra into the group's states
    static qaf_status load(qaf_adjoint_batch* B, const cplx<real>* const* src, size_t src_istride, cudaStream_t st) {
        EnsGroup<real>& g = group(B);
        dim3 grid(grid_for(B->ns), B->ninst);
        for (int f = 0; f < 3; ++f)
            ref_to_internal_batch<real><<<grid, 256, 0, st>>>(src[f], src_istride, g.w.old_m[f], g.w.old_n[f], g.istride, B->n);
        B->ens->y_valid = false;
        return post_launch("adjoint batch load");
    }
    static qaf_status store(qaf_adjoint_batch* B, cplx<real>* const* dst, size_t dst_istride, cudaStream_t st) {
        EnsGroup<real>& g = group(B);
        dim3 grid(grid_for(B->ns), B->ninst);
        for (int f = 0; f < 3; ++f)
            internal_to_ref_batch<real><<<grid, 256, 0, st>>>(g.w.old_m[f], g.w.old_n[f], g.istride, dst[f], dst_istride, B->n);
        return post_launch("adjoint batch store");
    }

    // nsteps IF-RK4 steps of the whole batch, recording on request the stage inputs' fields
    // (phys: per step and stage ninst * PF_COUNT * N * N reals), w after the steps from local
    // step wfrom on (wlog: ninst spectra per step, indexed from wfrom) and the loss
    template <int N>
    static qaf_status advance(qaf_adjoint_batch* B, int nsteps, real* phys, cplx<real>* wlog, int wfrom, bool loss,
                              int loss_from, double lweight, cudaStream_t st) {
        qaf_ensemble* e = B->ens;
        EnsGroup<real>& g = group(B);
        if (!e->y_valid) {
            QAF_TRY(ens_prologue<real>(e, st));
            e->y_valid = true;
        }
        StageArgs<real> a = group_args<real>(e, g);
        a.mode = MODE_STAGE;
        a.do_inverse = 1;
        a.phys_istride = (size_t)PF_COUNT * N * N;
        const size_t slot = (size_t)B->ninst * PF_COUNT * N * N;
        for (int s = 0; s < nsteps; ++s) {
            const bool lstep = loss && s >= loss_from;
            if (lstep) QAF_CUDA(cudaMemsetAsync(g.diag, 0, 2 * (size_t)B->ninst * sizeof(double), st));
            for (int k = 1; k <= 4; ++k) {
                a.stage = k;
                a.last_stage = k == 4;
                a.diag = (lstep && k == 4) ? g.diag : nullptr;
                a.phys_out = phys ? phys + ((size_t)s * 4 + (k - 1)) * slot : nullptr;
                Launch<real, N>::row(a, st);
                Launch<real, N>::col(a, st);
            }
            if (lstep) adj_loss_accumulate_batch<<<(B->ninst + 127) / 128, 128, 0, st>>>(g.diag, B->loss, lweight, B->ninst);
            if (wlog && s >= wfrom) {
                dim3 grid(grid_for(B->ns), B->ninst);
                internal_to_ref_batch<real><<<grid, 256, 0, st>>>(g.w.old_m[0], g.w.old_n[0], g.istride,
                                                                  wlog + (size_t)(s - wfrom) * B->ninst * B->ns, B->ns, N);
            }
        }
        return post_launch("adjoint batch advance");
    }
};

template <typename real, int N>
qaf_status batch_forward(qaf_adjoint_batch* B, const void* const* s0, const void* alpha, void* const* sT, double* losses,
                         cudaStream_t st) {
    using O = BatchOps<real>;
    EnsGroup<real>& g = O::group(B);
    const size_t ns = B->ns, cb = sizeof(cplx<real>), ni = (size_t)B->ninst;
    if (alpha) {
        QAF_CUDA(cudaMemcpyAsync(B->alpha, alpha, ni * N * N * sizeof(real), cudaMemcpyDeviceToDevice, st));
        g.alpha_fields = reinterpret_cast<real*>(B->alpha);
        B->have_alpha = true;
    } else {
        g.alpha_fields = nullptr;
        B->have_alpha = false;
    }
    for (int f = 0; f < 3; ++f)   // checkpoint 0: the inputs
        QAF_CUDA(cudaMemcpyAsync(bfield<real>(B->ckpt, ns, B->ninst, f), s0[f], ni * ns * cb, cudaMemcpyDeviceToDevice, st));
    const cplx<real>* src[3] = {bfield<real>(B->ckpt, ns, B->ninst, 0), bfield<real>(B->ckpt, ns, B->ninst, 1),
                                bfield<real>(B->ckpt, ns, B->ninst, 2)};
    QAF_TRY(O::load(B, src, ns, st));
    QAF_CUDA(cudaMemsetAsync(B->loss, 0, ni * sizeof(double), st));
    const double n4 = (double)N * N * (double)N * N;
    const double lweight = 1.0 / ((double)(B->window > 0 ? B->window : 1) * n4);
    for (int seg = 0; seg < B->nseg; ++seg) {
        const int t0 = seg * B->K, t1 = std::min(B->nsteps, t0 + B->K);
        QAF_TRY(O::template advance<N>(B, t1 - t0, nullptr, nullptr, 0, B->window > 0, B->nsteps - B->window - t0,
                                       lweight, st));
        if (t1 < B->nsteps) {
            unsigned char* c = B->ckpt + (size_t)(seg + 1) * 3 * ni * ns * cb;
            cplx<real>* dst[3] = {bfield<real>(c, ns, B->ninst, 0), bfield<real>(c, ns, B->ninst, 1),
                                  bfield<real>(c, ns, B->ninst, 2)};
            QAF_TRY(O::store(B, dst, ns, st));
        }
    }
    if (sT[0] && sT[1] && sT[2]) {
        cplx<real>* dst[3] = {static_cast<cplx<real>*>(sT[0]), static_cast<cplx<real>*>(sT[1]),
                              static_cast<cplx<real>*>(sT[2])};
        QAF_TRY(O::store(B, dst, ns, st));
    }
    if (losses) {
        QAF_CUDA(cudaMemcpyAsync(losses, B->loss, ni * sizeof(double), cudaMemcpyDeviceToHost, st));
        QAF_CUDA(cudaStreamSynchronize(st));
    }
    return post_launch("qaf_adjoint_batch_forward");
}

template <typename real, int N>
qaf_status batch_backward(qaf_adjoint_batch* B, const void* const* gT, const double* glosses, void* const* g0,
                          void* galpha, cudaStream_t st) {
    using O = BatchOps<real>;
    constexpr int H = N / 2;
    // several columns per CTA: coalesced 16-32 byte segments of the T arrays (a batch has CTAs to spare)
    constexpr int W0 = sizeof(real) == 4 ? 4 : 2;
    constexpr int P = pow2_size(N);
    constexpr int W = W0 < H ? W0 : H, EC = fit_e(N, P / 16 > 4 ? P / 16 : 4);
    constexpr int COL_THREADS = NGA * W * (N / EC);
    constexpr size_t COL_SMEM = (size_t)NGA * N * (W > 1 ? W : 2) * sizeof(cplx<real>);
    constexpr int ER = fit_e(H, P / 32 < 2 ? 2 : (P / 32 > 16 ? 16 : P / 32));
    constexpr int ROW_THREADS = NGA * (H / ER);
    constexpr size_t ROW_SMEM = (size_t)NGA * H * sizeof(cplx<real>);
    static DeviceOnce attrs;   // kernel attributes, per device
    QAF_TRY(attrs.get(nullptr, [](int*) -> qaf_status {
        QAF_CUDA(cudaFuncSetAttribute(adj_colp_kernel<real, N, W, EC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)COL_SMEM));
        QAF_CUDA(cudaFuncSetAttribute(adj_row_kernel<real, N, ER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ROW_SMEM));
        return QAF_OK;
    }));
    qaf_ensemble* e = B->ens;
    EnsGroup<real>& g = O::group(B);
    const size_t ns = B->ns, cb = sizeof(cplx<real>), ni = (size_t)B->ninst;
    const qaf_params& p = e->p;
    AdjArgs<real> a;
    std::memset(&a, 0, sizeof(a));
    a.dkx = (real)(2 * M_PI / e->lx); a.dky = (real)(2 * M_PI / e->ly); a.dt = (real)p.dt; a.lambda = (real)p.lambda;
    a.ce = (real)(1.0 / (p.er * p.re));
    a.advect = p.advect_omega ? 1 : 0;
    set_mask(a, N, N, p.no_dealias);
    a.tw = g.w.tw; a.ex = g.w.ex; a.ey = g.w.ey;
    host_if_e0<real>(p.dt, p.re, p.rf, p.q_lin, a.e0);
    a.Tg = reinterpret_cast<cplx<real>*>(B->Tg); a.Tx = reinterpret_cast<cplx<real>*>(B->Tx);
    for (int f = 0; f < 3; ++f) {
        a.abar[f] = bfield<real>(B->abar, ns, B->ninst, f);
        a.sacc[f] = bfield<real>(B->sacc, ns, B->ninst, f);
        a.sbar[f] = bfield<real>(B->sbar, ns, B->ninst, f);
    }
    a.alpha_field = B->have_alpha ? reinterpret_cast<const real*>(B->alpha) : nullptr;
    a.alpha = (real)p.alpha;
    a.alpha_grad = reinterpret_cast<real*>(B->agrad);
    a.ninst = B->ninst;
    a.s_istride = ns;
    a.tg_istride = (size_t)NGA * N * H;
    a.tx_istride = (size_t)PF_COUNT * N * H;
    a.p_istride = (size_t)PF_COUNT * N * N;
    a.a_istride = B->have_alpha ? (size_t)N * N : 0;
    a.g_istride = (size_t)N * N;
    std::vector<real> lw(ni, (real)0);   // dL/dloss_k / window per instance
    bool any_loss = false;
    if (glosses && B->window > 0)
        for (size_t k = 0; k < ni; ++k) {
            lw[k] = (real)(glosses[k] / B->window);
            any_loss |= glosses[k] != 0.0;
        }
    QAF_CUDA(cudaMemcpyAsync(B->lossw, lw.data(), ni * sizeof(real), cudaMemcpyHostToDevice, st));
    a.loss_wv = reinterpret_cast<const real*>(B->lossw);
    for (int f = 0; f < 3; ++f) {
        if (gT[f]) QAF_CUDA(cudaMemcpyAsync(a.sbar[f], gT[f], ni * ns * cb, cudaMemcpyDeviceToDevice, st));
        else QAF_CUDA(cudaMemsetAsync(a.sbar[f], 0, ni * ns * cb, st));
    }
    QAF_CUDA(cudaMemsetAsync(B->agrad, 0, ni * N * N * sizeof(real), st));
    const int T = B->nsteps;
    auto in_window = [&](int n) { return B->window > 0 && any_loss && n >= T - B->window + 1; };
    auto col = [&]() { adj_colp_kernel<real, N, W, EC><<<(H / W + 1) * B->ninst, COL_THREADS, COL_SMEM, st>>>(a); };
    const size_t slot = ni * PF_COUNT * N * N;
    bool started = false;
    for (int seg = B->nseg - 1; seg >= 0; --seg) {
        const int t0 = seg * B->K, t1 = std::min(T, t0 + B->K);
        unsigned char* c = B->ckpt + (size_t)seg * 3 * ni * ns * cb;
        const cplx<real>* src[3] = {bfield<real>(c, ns, B->ninst, 0), bfield<real>(c, ns, B->ninst, 1),
                                    bfield<real>(c, ns, B->ninst, 2)};
        QAF_TRY(O::load(B, src, ns, st));
        // w after local step s (state t0 + s + 1) for the states in the loss window
        const int wfrom = std::max(0, T - B->window - t0);
        QAF_TRY(O::template advance<N>(B, t1 - t0, reinterpret_cast<real*>(B->phys), reinterpret_cast<cplx<real>*>(B->wlog),
                                       wfrom, false, 0, 0.0, st));
        auto w_at = [&](int n) -> const cplx<real>* {   // w of the state at time n, t0 <= n <= t1
            if (n == t0) return bfield<real>(c, ns, B->ninst, 0);
            return reinterpret_cast<const cplx<real>*>(B->wlog) + (size_t)(n - 1 - t0 - wfrom) * ni * ns;
        };
        for (int n = t1 - 1; n >= t0; --n) {
            if (!started) {
                a.stage = 0; a.emit = 1;
                a.wstate = in_window(T) ? w_at(T) : nullptr;
                col();
                started = true;
            }
            for (int s = 4; s >= 1; --s) {
                a.phys = reinterpret_cast<const real*>(B->phys) + ((size_t)(n - t0) * 4 + (s - 1)) * slot;
                adj_row_kernel<real, N, ER><<<N * B->ninst, ROW_THREADS, ROW_SMEM, st>>>(a);
                a.stage = s;
                a.emit = (s > 1 || n > 0) ? 1 : 0;
                a.wstate = (s == 1 && in_window(n)) ? w_at(n) : nullptr;
                col();
            }
        }
    }
    for (int f = 0; f < 3; ++f)
        if (g0[f]) QAF_CUDA(cudaMemcpyAsync(g0[f], a.sbar[f], ni * ns * cb, cudaMemcpyDeviceToDevice, st));
    if (galpha) QAF_CUDA(cudaMemcpyAsync(galpha, B->agrad, ni * N * N * sizeof(real), cudaMemcpyDeviceToDevice, st));
    return post_launch("qaf_adjoint_batch_backward");
}

template <class F>
qaf_status with_small_n(int N, F&& f) {
#ifdef QAF_ONLY_N
    if constexpr (QAF_ONLY_N <= 256) {
        if (N == QAF_ONLY_N) return f(std::integral_constant<int, QAF_ONLY_N>{});
    }
    return fail(QAF_ERR_UNSUPPORTED, "batched adjoint: no kernels for this grid size");
#endif
    switch (N) {
        case 16: return f(std::integral_constant<int, 16>{});
        case 32: return f(std::integral_constant<int, 32>{});
        case 64: return f(std::integral_constant<int, 64>{});
        case 128: return f(std::integral_constant<int, 128>{});
        case 256: return f(std::integral_constant<int, 256>{});
        case 48: return f(std::integral_constant<int, 48>{});
        case 96: return f(std::integral_constant<int, 96>{});
        case 192: return f(std::integral_constant<int, 192>{});
        default: return fail(QAF_ERR_UNSUPPORTED, "batched adjoint: grids up to 256 x 256");
    }
}

}  // namespace

extern "C" {

qaf_status qaf_adjoint_batch_create(int ninst, int n, double lx, double ly, qaf_dtype dtype, const qaf_params* p,
                                    int nsteps, int checkpoint_every, int loss_window, qaf_adjoint_batch** out) {
    if (!out || !p) return fail(QAF_ERR_INVALID, "null argument");
    *out = nullptr;
    if (ninst < 1) return fail(QAF_ERR_INVALID, "ninst must be >= 1");
    if (n > 256) return fail(QAF_ERR_UNSUPPORTED, "batched adjoint: grids up to 256 x 256");
    if (nsteps < 1 || checkpoint_every < 1) return fail(QAF_ERR_INVALID, "nsteps and checkpoint_every must be >= 1");
    if (loss_window < 0 || loss_window > nsteps) return fail(QAF_ERR_INVALID, "loss_window must be in [0, nsteps]");
    std::vector<int> sizes(ninst, n);
    std::vector<double> al(ninst, p->alpha), rf(ninst, p->rf);
    qaf_adjoint_batch* B = new qaf_adjoint_batch();
    qaf_status s = qaf_ensemble_create(ninst, sizes.data(), lx, ly, dtype, p, al.data(), rf.data(), &B->ens);
    if (s != QAF_OK) { delete B; return s; }
    B->ninst = ninst; B->n = n; B->nsteps = nsteps; B->K = std::min(checkpoint_every, nsteps);
    B->window = loss_window; B->nseg = (nsteps + B->K - 1) / B->K;
    B->ns = (size_t)(n / 2 + 1) * n; B->np = (size_t)n * n;
    const size_t rb = dtype == QAF_F64 ? 8 : 4, cb = 2 * rb, ni = (size_t)ninst;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
    const size_t o_ck = take((size_t)B->nseg * 3 * ni * B->ns * cb);
    const size_t o_wl = take((size_t)std::min(B->K, std::max(loss_window, 1)) * ni * B->ns * cb);
    const size_t o_ph = take((size_t)B->K * 4 * ni * PF_COUNT * B->np * rb);
    const size_t o_tg = take(ni * NGA * n * (n / 2) * cb);
    const size_t o_tx = take(ni * PF_COUNT * n * (n / 2) * cb);
    const size_t o_ab = take(3 * ni * B->ns * cb), o_sa = take(3 * ni * B->ns * cb), o_sb = take(3 * ni * B->ns * cb);
    const size_t o_ag = take(ni * B->np * rb), o_al = take(ni * B->np * rb), o_lw = take(ni * rb);
    const size_t o_ls = take(ni * sizeof(double));
    cudaError_t e = cudaMalloc((void**)&B->blk, off);
    if (e != cudaSuccess) {
        qaf_ensemble_destroy(B->ens);
        delete B;
        return fail(QAF_ERR_ALLOC, std::string("qaf_adjoint_batch_create: cudaMalloc of ") + std::to_string(off >> 20) +
                                       " MiB: " + cudaGetErrorString(e));
    }
    B->ckpt = B->blk + o_ck; B->wlog = B->blk + o_wl; B->phys = B->blk + o_ph; B->Tg = B->blk + o_tg;
    B->Tx = B->blk + o_tx; B->abar = B->blk + o_ab; B->sacc = B->blk + o_sa; B->sbar = B->blk + o_sb;
    B->agrad = B->blk + o_ag; B->alpha = B->blk + o_al; B->lossw = B->blk + o_lw;
    B->loss = reinterpret_cast<double*>(B->blk + o_ls);
    *out = B;
    return QAF_OK;
}

qaf_status qaf_adjoint_batch_destroy(qaf_adjoint_batch* B) {
    if (!B) return QAF_OK;
    if (B->blk) cudaFree(B->blk);
    qaf_ensemble_destroy(B->ens);
    delete B;
    return QAF_OK;
}

qaf_status qaf_adjoint_batch_forward(qaf_adjoint_batch* B, const void* w0, const void* r1_0, const void* r2_0,
                                     const void* alpha, void* wT, void* r1T, void* r2T, double* losses, void* stream) {
    if (!B) return fail(QAF_ERR_INVALID, "null batch");
    if (!w0 || !r1_0 || !r2_0) return fail(QAF_ERR_INVALID, "null initial state");
    const void* s0[3] = {w0, r1_0, r2_0};
    void* sT[3] = {wT, r1T, r2T};
    B->have_forward = false;
    QAF_TRY(with_small_n(B->n, [&](auto nn) -> qaf_status {
        constexpr int N = decltype(nn)::value;
        return B->ens->dtype == QAF_F64 ? batch_forward<double, N>(B, s0, alpha, sT, losses, (cudaStream_t)stream)
                                        : batch_forward<float, N>(B, s0, alpha, sT, losses, (cudaStream_t)stream);
    }));
    B->have_forward = true;
    return QAF_OK;
}

qaf_status qaf_adjoint_batch_backward(qaf_adjoint_batch* B, const void* gwT, const void* gr1T, const void* gr2T,
                                      const double* glosses, void* gw0, void* gr1_0, void* gr2_0, void* galpha,
                                      void* stream) {
    if (!B) return fail(QAF_ERR_INVALID, "null batch");
    if (!B->have_forward) return fail(QAF_ERR_INVALID, "qaf_adjoint_batch_backward needs a forward first");
    const void* gT[3] = {gwT, gr1T, gr2T};
    void* g0[3] = {gw0, gr1_0, gr2_0};
    return with_small_n(B->n, [&](auto nn) -> qaf_status {
        constexpr int N = decltype(nn)::value;
        return B->ens->dtype == QAF_F64 ? batch_backward<double, N>(B, gT, glosses, g0, galpha, (cudaStream_t)stream)
                                        : batch_backward<float, N>(B, gT, glosses, g0, galpha, (cudaStream_t)stream);
    });
}

}  // extern "C"
