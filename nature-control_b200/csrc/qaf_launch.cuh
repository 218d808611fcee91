// qaf_launch.cuh — definitions of the per-size launchers (qaf_internal.cuh),
// included by the qaf_launch_*.cu translation units that instantiate them.
#pragma once

#include "qaf_internal.cuh"

#include <type_traits>

namespace qaf {
namespace detail {

template <typename real, int N>
DeviceOnce Launch<real, N>::col_slots;
template <typename real, int N>
DeviceOnce Launch<real, N>::col_slots_b;

template <typename real, int N>
qaf_status Launch<real, N>::setup() {
    QAF_TRY(col_slots_b.get(nullptr, [](int* slots) -> qaf_status {
        QAF_CUDA(cudaFuncSetAttribute(col_kernel<real, N, C::ECS, C::MINBC_B, C::COL_MODE_B>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::COL_SMEM_B));
        int dev = 0, sms = 0, per_sm = 0;
        QAF_CUDA(cudaGetDevice(&dev));
        QAF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        QAF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, col_kernel<real, N, C::ECS, C::MINBC_B, C::COL_MODE_B>,
                                                               C::COL_THREADS, C::COL_SMEM_B));
        if (per_sm < 1) return fail(QAF_ERR_UNSUPPORTED, "column kernel does not fit on an SM");
        *slots = sms * per_sm;
        return QAF_OK;
    }));
    return col_slots.get(nullptr, [](int* slots) -> qaf_status {
        QAF_CUDA(cudaFuncSetAttribute(col_kernel<real, N, C::ECS, C::MINBC, C::COL_MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::COL_SMEM));
        QAF_CUDA(cudaFuncSetAttribute(row_kernel<real, N, C::ER, C::ROWS, C::MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::ROW_SMEM));
        QAF_CUDA(cudaFuncSetAttribute(row_kernel<real, N, C::ER, C::ROWS_S, C::MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)C::ROW_SMEM_S));
        // the same kernels for grids with nx != ny (sizes from the launch arguments)
        QAF_CUDA(cudaFuncSetAttribute(col_kernel<real, N, C::ECS, C::MINBC, C::COL_MODE, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::COL_SMEM));
        QAF_CUDA(cudaFuncSetAttribute(row_kernel<real, N, C::ER, C::ROWS, C::MINB, 0, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::ROW_SMEM));
        QAF_CUDA(cudaFuncSetAttribute(col_ifft_kernel<real, N, C::W, C::EC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::COLT_SMEM));
        if constexpr (C::COL_FP)
            QAF_CUDA(cudaFuncSetAttribute(colfp_kernel<real, N, C::EC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)ColFP<real, N, C::EC>::SMEM));
        QAF_CUDA(cudaFuncSetAttribute(col_fft_kernel<real, N, C::W, C::EC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::COLT_SMEM));
        int dev = 0, sms = 0, per_sm = 0;
        QAF_CUDA(cudaGetDevice(&dev));
        QAF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        QAF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, col_kernel<real, N, C::ECS, C::MINBC, C::COL_MODE>,
                                                               C::COL_THREADS, C::COL_SMEM));
        if (per_sm < 1) return fail(QAF_ERR_UNSUPPORTED, "column kernel does not fit on an SM");
        *slots = sms * per_sm;
        return QAF_OK;
    });
}

template <typename real, int N>
void Launch<real, N>::col(const StageArgs<real>& a0, cudaStream_t st) {
    StageArgs<real> hooked;
    const StageArgs<real>* ap = &a0;
    if (a0.mode == MODE_STAGE && g_test_drop.load(std::memory_order_relaxed) != 0) {
        if (const int d = g_test_drop.exchange(0)) {
            hooked = a0;
            hooked.drop_slab = d;
            hooked.wait_polls = g_test_polls.load();
            ap = &hooked;
        }
    }
    const StageArgs<real>& a = *ap;
    if constexpr (std::is_same<real, float>::value) {
        int slots = 0;
        if (a.nx == a.ny) {
            if (StepVariant<float>* v = tuned_variant(N, 0, a.ninst > 1, &slots)) {
                v->launch(a, slots, st);
                return;
            }
        }
    }
    // a single small square grid: the field-parallel column pass (a test
    // hook's launch, which withholds one of the persistent kernel's copies,
    // keeps the persistent kernel)
    if constexpr (C::COL_FP) {
        if (a.ninst == 1 && a.nx == N && a.drop_slab == 0) {
            colfp_kernel<real, N, C::EC><<<N / 2 + 3, ColFP<real, N, C::EC>::NTHREADS, ColFP<real, N, C::EC>::SMEM, st>>>(a);
            return;
        }
    }
    const long items = (long)(2 * (a.nx / 2 / TW) + 3) * a.ninst;
    if (a.ninst > 1 && C::SEP_B) {
        const int slots = col_slots_b.peek();
        const int grid = slots > 0 && items > slots ? slots : (int)items;
        col_kernel<real, N, C::ECS, C::MINBC_B, C::COL_MODE_B><<<grid, C::COL_THREADS, C::COL_SMEM_B, st>>>(a);
        return;
    }
    const int slots = col_slots.peek();   // set up by every operation before its launches
    const int grid = slots > 0 && items > slots ? slots : (int)items;
    if (a.nx == N)
        col_kernel<real, N, C::ECS, C::MINBC, C::COL_MODE><<<grid, C::COL_THREADS, C::COL_SMEM, st>>>(a);
    else
        col_kernel<real, N, C::ECS, C::MINBC, C::COL_MODE, false><<<grid, C::COL_THREADS, C::COL_SMEM, st>>>(a);
}

template <typename real, int N>
void Launch<real, N>::row(const StageArgs<real>& a, cudaStream_t st) {
    if constexpr (std::is_same<real, float>::value) {
        int slots = 0;
        if (a.nx == a.ny) {
            if (StepVariant<float>* v = tuned_variant(N, 1, a.ninst > 1, &slots)) {
                v->launch(a, slots, st);
                return;
            }
        }
    }
    if (a.ny == N && a.ninst == 1)
        row_kernel<real, N, C::ER, C::ROWS_S, C::MINB><<<a.ny / C::ROWS_S, C::ROW_THREADS_S, C::ROW_SMEM_S, st>>>(a);
    else if (a.ny == N)
        row_kernel<real, N, C::ER, C::ROWS, C::MINB><<<(a.ny / C::ROWS) * a.ninst, C::ROW_THREADS, C::ROW_SMEM, st>>>(a);
    else
        row_kernel<real, N, C::ER, C::ROWS, C::MINB, 0, false>
            <<<(a.ny / C::ROWS) * a.ninst, C::ROW_THREADS, C::ROW_SMEM, st>>>(a);
}

template <typename real, int N>
void Launch<real, N>::col_ifft(const cplx<real>* spec, cplx<real>* T, const cplx<real>* tw_y, int nx, cudaStream_t st) {
    col_ifft_kernel<real, N, C::W, C::EC><<<nx / 2 / C::W, C::COLT_THREADS, C::COLT_SMEM, st>>>(spec, T, tw_y, nx);
}

template <typename real, int N>
void Launch<real, N>::col_fft(const cplx<real>* T, cplx<real>* spec, const cplx<real>* tw_y, int nx, cudaStream_t st) {
    col_fft_kernel<real, N, C::W, C::EC><<<nx / 2 / C::W, C::COLT_THREADS, C::COLT_SMEM, st>>>(T, spec, tw_y, nx);
}

template <typename real, int N>
void Launch<real, N>::row_c2r(const cplx<real>* T, real* phys, const cplx<real>* tw, int ny, cudaStream_t st) {
    row_c2r_kernel<real, N, C::ERT, C::ROWS_T><<<ny / C::ROWS_T, C::ROWT_THREADS, C::ROWT_SMEM, st>>>(T, phys, tw);
}

template <typename real, int N>
void Launch<real, N>::row_r2c(const real* phys, cplx<real>* T, const cplx<real>* tw, int ny, cudaStream_t st) {
    row_r2c_kernel<real, N, C::ERT, C::ROWS_T><<<ny / C::ROWS_T, C::ROWT_THREADS, C::ROWT_SMEM, st>>>(phys, T, tw);
}

template <typename real, int N>
void Launch<real, N>::bwd(const cplx<real>* spec, cplx<real>* T, real* phys, const cplx<real>* tw, cudaStream_t st) {
    col_ifft(spec, T, tw, N, st);
    row_c2r(T, phys, tw, N, st);
}

template <typename real, int N>
void Launch<real, N>::fwd(const real* phys, cplx<real>* T, cplx<real>* spec, const cplx<real>* tw, cudaStream_t st) {
    row_r2c(phys, T, tw, N, st);
    col_fft(T, spec, tw, N, st);
}

}  // namespace detail
}  // namespace qaf
