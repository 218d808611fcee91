// qaf_internal.cuh — declarations shared by the library's translation units:
// error status helpers, per-device set-up, the launch configuration per
// (precision, size) and the per-size launchers. qaf_api.cu holds the C ABI;
// the launchers' definitions (qaf_launch.cuh) are instantiated in
// qaf_launch_*.cu.
#pragma once

#include "qaf.h"

#include "qaf_kernels.cuh"
#include "qaf_ops.cuh"
#include "qaf_variants.cuh"

#include <atomic>
#include <mutex>
#include <string>

namespace qaf {
namespace detail {

// records msg as the message of the last failing call on this thread and returns st
qaf_status fail(qaf_status st, const std::string& msg);

#define QAF_CUDA(call)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return fail(QAF_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

#define QAF_TRY(expr)                  \
    do {                               \
        qaf_status s_ = (expr);        \
        if (s_ != QAF_OK) return s_;   \
    } while (0)

inline bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// ---------------------------------------------------------------------------
// One-time set-up per device. Kernel attributes (cudaFuncSetAttribute) and
// occupancy apply to the device that is current when they are set, so every
// set-up step keeps one slot per device index, filled under one lock the first
// time a call runs on that device; later calls read it without the lock.
// ---------------------------------------------------------------------------
constexpr int kMaxDevices = 64;
extern std::mutex g_setup_mu;   // guards every per-device set-up

inline qaf_status current_device(int* dev) {
    QAF_CUDA(cudaGetDevice(dev));
    if (*dev < 0 || *dev >= kMaxDevices) return fail(QAF_ERR_UNSUPPORTED, "device index out of range");
    return QAF_OK;
}

struct DeviceOnce {
    std::atomic<int> v[kMaxDevices] = {};   // 0: not set up on that device
    // the value for the current device; init(int* value) runs once per device
    // (value >= 1 once set up)
    template <class F>
    qaf_status get(int* out, F&& init) {
        int dev = 0;
        QAF_TRY(current_device(&dev));
        int x = v[dev].load(std::memory_order_acquire);
        if (x == 0) {
            std::lock_guard<std::mutex> g(g_setup_mu);
            x = v[dev].load(std::memory_order_relaxed);
            if (x == 0) {
                QAF_TRY(init(&x));
                if (x < 1) x = 1;
                v[dev].store(x, std::memory_order_release);
            }
        }
        if (out) *out = x;
        return QAF_OK;
    }
    // the value set up for the current device, 0 if none
    int peek() const {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
        return v[dev].load(std::memory_order_acquire);
    }
};

// Launch-shape defaults (values per thread of the column / row FFTs, threads
// per row-kernel CTA); overridable at build time for tuning.
#ifndef QAF_COL_E
#define QAF_COL_E 8
#endif
#ifndef QAF_ROW_E
#define QAF_ROW_E 8
#endif
#ifndef QAF_ROW_THREADS
#define QAF_ROW_THREADS 256
#endif
#ifndef QAF_COL1024_MODE
#define QAF_COL1024_MODE 82
#endif
constexpr int kMinN = 16, kMaxN = 1024;
constexpr int gcd_c(int a, int b) { return b == 0 ? a : gcd_c(b, a % b); }
// the largest power of two <= min(x, cap)
constexpr int pow2_floor(int x, int cap) { return (x > cap ? cap : x) <= 1 ? 1 : 2 * pow2_floor((x > cap ? cap : x) / 2, cap); }
// grid sizes with kernels: powers of two in [16, 1024] and 3 * 2^k in [48, 768]
// (the reference's own drivers run 768 = 512 * 3 / 2, friction.cu:109)
inline bool size_supported(int n) {
    return (pow2(n) && n >= kMinN && n <= kMaxN) || (n % 3 == 0 && pow2(n / 3) && n >= 48 && n <= 768);
}

// ---------------------------------------------------------------------------
// launch configuration per (precision, N)
// ---------------------------------------------------------------------------
template <typename real, int N>
struct Cfg {
    static constexpr int H = N / 2;
    static constexpr bool F32 = sizeof(real) == 4;
    // CTAs per SM the register budget is sized for (FP64 kernels need > 128 registers)
    static constexpr int MINB = F32 ? 2 : 1;
    // values per thread of a length-N y-FFT (standalone transforms, adjoint)
    static constexpr int EC = fit_e(N, QAF_COL_E);
    // the step's column kernel (persistent): a tile of TW kx-columns per work
    // item, ECS values per thread, MINBC CTAs per SM for the register budget,
    // and the ColKernel mode: at 1024^2 FP32 the shared twiddle table, the
    // item code compiled once (the kernel runs one copy of it for both item
    // kinds and both fields of an item: 71.9 -> 67.2 us per launch, the
    // no_instruction stall gone from the top stalls), the
    // double-buffered swizzled exchange and the ky table in shared memory
    // with 4 values per thread in one 1024-thread CTA per SM (no spills at
    // 64 registers); the shared twiddle table (mode 1) for FP32 768^2, FP64
    // from 512^2 and every batch (ensemble) launch; otherwise register
    // twiddle bases (mode 0: for single small grids, whose launches are
    // latency-bound, the table's fill at kernel start measured slower)
    //
    // The small FP32 grids take the shapes that timed fastest on the B200
    // when every shape was timed on one box (single grid and an 85-instance
    // batch each): 64^2 four values per column thread (26-28% faster than
    // eight), 128^2 and 256^2 batches six column CTAs per SM, 128^2 and
    // 256^2 single grids two rows per row CTA (5-9%).
    static constexpr bool WIDE1024 = F32 && N == 1024;
    static constexpr int ECS = WIDE1024 || (F32 && N == 64) ? 4 : EC;
    // (+64 with the shared table: the item code compiled once, ColKernel::ONE_BODY;
    // measured per step on one box, batches of 85: 64^2 214 -> 177 us,
    // 128^2 645 -> 592 us, 256^2 2002 -> 1548 us with six CTAs per SM; a
    // single 64^2 grid 120 -> 111 us)
    static constexpr int COL_MODE = WIDE1024 ? QAF_COL1024_MODE
                                             : (((F32 && (N == 768 || N == 64)) || (!F32 && N >= 512)) ? 65 : 0);
    // batches of instances
    static constexpr int COL_MODE_B = WIDE1024 ? QAF_COL1024_MODE : 65;
    static constexpr int MINBC = WIDE1024 ? 1 : MINB;
    static constexpr int MINBC_B = (F32 && (N == 128 || N == 256)) ? 6 : MINBC;
    // batches launch their own kernel where its shape differs from the single grids'
    static constexpr bool SEP_B = COL_MODE_B != COL_MODE || MINBC_B != MINBC;
    // single square grids of 32^2, 128^2 and 256^2: the field-parallel column
    // pass (colfp_kernel, one CTA per kx-column running all of its transforms
    // at once). Measured per step on one box, in CUDA graphs: 32^2 116 us
    // against 136 us, 128^2 127 against 150 (the persistent kernel's best
    // shape), 256^2 140 against 155; at 64^2 the persistent kernel stays
    // faster (102-106 against 126)
    static constexpr bool COL_FP = N == 32 || N == 128 || N == 256;
    static constexpr int COL_THREADS = TW * (N / ECS);
    static constexpr size_t COL_SMEM = ColKernel<real, N, ECS, COL_MODE>::SMEM;
    static constexpr size_t COL_SMEM_B = ColKernel<real, N, ECS, COL_MODE_B>::SMEM;
    // row kernel: ER values per thread of a length-N x-FFT, ROWS rows per CTA
    static constexpr int ER = fit_e(N, QAF_ROW_E);
    static constexpr int TEAM_R = N / ER;
    static constexpr int ROWS_A = QAF_ROW_THREADS / TEAM_R > 0 ? QAF_ROW_THREADS / TEAM_R : 1;
    static constexpr int ROWS_B = N / 8 > 0 ? N / 8 : 1;
    // a power of two of at most 16, so that it divides the row count ny of any
    // supported grid (all multiples of 16), not only N
    static constexpr int ROWS = pow2_floor(gcd_c(N, ROWS_A < ROWS_B ? ROWS_A : ROWS_B), 16);
    static constexpr int ROW_THREADS = ROWS * TEAM_R;
    static constexpr size_t ROW_SMEM = RowKernel<real, N, ER, ROWS>::SMEM;
    static_assert(16 % ROWS == 0, "rows per CTA divide every row count");
    // square single grids (ninst == 1): two rows per CTA at 128^2 and 256^2 FP32
    static constexpr int ROWS_S = (F32 && (N == 128 || N == 256)) ? 2 : ROWS;
    static constexpr int ROW_THREADS_S = ROWS_S * TEAM_R;
    static constexpr size_t ROW_SMEM_S = RowKernel<real, N, ER, ROWS_S>::SMEM;
    static_assert(16 % ROWS_S == 0, "rows per CTA divide every row count");
    // standalone transforms: W kx-columns per CTA, half-length row FFTs
    static constexpr int W = 4 < H ? 4 : H;
    static constexpr int COLT_THREADS = W * (N / EC);
    static constexpr size_t COLT_SMEM = (size_t)W * N * sizeof(cplx<real>);
    static constexpr int ERT = fit_e(H, F32 ? 8 : 4);
    static constexpr int TEAM_T = H / ERT;
    static constexpr int ROWS_T = (TEAM_T >= 128) ? 1 : pow2_floor(gcd_c(N, 128 / TEAM_T), 16);
    static constexpr int ROWT_THREADS = ROWS_T * TEAM_T;
    static constexpr size_t ROWT_SMEM = (size_t)ROWS_T * H * sizeof(cplx<real>);
    static_assert(16 % ROWS_T == 0, "rows per CTA divide every row count");
};

// Launches of the kernels whose transform length is N: the row kernel and
// row transforms of a grid with nx = N, the column kernel and column
// transforms of a grid with ny = N (the other size is an argument). Defined
// in qaf_launch.cuh and instantiated for every supported (precision, N) in
// the qaf_launch_*.cu translation units, which compile in parallel.
template <typename real, int N>
struct Launch {
    using C = Cfg<real, N>;
    // resident column CTAs per device (the persistent grid size) of the
    // single-grid and the batch column kernels
    static DeviceOnce col_slots, col_slots_b;
    static qaf_status setup();
    // the column kernel of a grid with ny = N (a.nx / 2 / TW tiles)
    static void col(const StageArgs<real>& a, cudaStream_t st);
    // the row kernel of a grid with nx = N (a.ny / ROWS CTAs per instance)
    static void row(const StageArgs<real>& a, cudaStream_t st);
    // transforms: nx / 2 columns of length N; ny rows of length N
    static void col_ifft(const cplx<real>* spec, cplx<real>* T, const cplx<real>* tw_y, int nx, cudaStream_t st);
    static void col_fft(const cplx<real>* T, cplx<real>* spec, const cplx<real>* tw_y, int nx, cudaStream_t st);
    static void row_c2r(const cplx<real>* T, real* phys, const cplx<real>* tw, int ny, cudaStream_t st);
    static void row_r2c(const real* phys, cplx<real>* T, const cplx<real>* tw, int ny, cudaStream_t st);
    // BwdTrans / FwdTrans of an N x N grid
    static void bwd(const cplx<real>* spec, cplx<real>* T, real* phys, const cplx<real>* tw, cudaStream_t st);
    static void fwd(const real* phys, cplx<real>* T, cplx<real>* spec, const cplx<real>* tw, cudaStream_t st);
};

// the launch-shape variant the autotuner chose for (n, kind 0 column / 1 row,
// batched), or nullptr for the built-in shape; *slots its persistent grid size
StepVariant<float>* tuned_variant(int n, int kind, bool batched, int* slots);
// test hook of qaf_test_lose_copy: consumed by the next column launch
extern std::atomic<int> g_test_drop;        // slab + 1, 0: off
extern std::atomic<unsigned> g_test_polls;

}  // namespace detail
}  // namespace qaf
