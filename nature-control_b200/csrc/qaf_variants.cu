// qaf_variants.cu — FP32 launch variants of the fused step kernels for the
// autotuner (see qaf_variants.cuh): column kernel with 16 (or, at 64^2, 4)
// values per thread of the y-FFT instead of 8; row kernel with fewer rows per
// CTA (more CTAs for small grids) or 16 values per thread of the x-FFT.
#include "qaf_kernels.cuh"
#include "qaf_variants.cuh"

namespace qaf {
namespace {

template <int N, int EC>
struct ColV {
    static constexpr int THREADS = TW * (N / EC);
    static constexpr size_t SMEM = ColKernel<float, N, EC>::SMEM;
    static constexpr int ITEMS = ColKernel<float, N, EC>::NITEMS;
    static cudaError_t setup(int* slots) {
        cudaError_t e = cudaFuncSetAttribute(col_kernel<float, N, EC, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)SMEM);
        if (e != cudaSuccess) return e;
        int dev = 0, sms = 0, per_sm = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, col_kernel<float, N, EC, 2>, THREADS, SMEM)) !=
            cudaSuccess)
            return e;
        if (per_sm < 1) return cudaErrorInvalidConfiguration;
        *slots = sms * per_sm;
        return cudaSuccess;
    }
    static void launch(const StageArgs<float>& a, int slots, cudaStream_t st) {
        const long items = (long)ITEMS * a.ninst;
        const int grid = items < slots ? (int)items : slots;
        col_kernel<float, N, EC, 2><<<grid, THREADS, SMEM, st>>>(a);
    }
};

template <int N, int ER, int ROWS>
struct RowV {
    static constexpr int THREADS = ROWS * (N / ER);
    static constexpr size_t SMEM = RowKernel<float, N, ER, ROWS>::SMEM;
    static cudaError_t setup(int* slots) {
        *slots = 0;
        return cudaFuncSetAttribute(row_kernel<float, N, ER, ROWS, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)SMEM);
    }
    static void launch(const StageArgs<float>& a, int, cudaStream_t st) {
        row_kernel<float, N, ER, ROWS, 2><<<(N / ROWS) * a.ninst, THREADS, SMEM, st>>>(a);
    }
};

template <class V>
constexpr StepVariant<float> make(const char* name, int kind) {
    return StepVariant<float>{name, kind, &V::setup, &V::launch, 0};
}

StepVariant<float> v64[] = {make<ColV<64, 4>>("col:e4", 0), make<RowV<64, 8, 2>>("row:e8r2", 1),
                            make<RowV<64, 16, 4>>("row:e16r4", 1)};
StepVariant<float> v128[] = {make<ColV<128, 16>>("col:e16", 0), make<RowV<128, 8, 2>>("row:e8r2", 1),
                             make<RowV<128, 16, 8>>("row:e16r8", 1)};
StepVariant<float> v256[] = {make<ColV<256, 16>>("col:e16", 0), make<RowV<256, 8, 2>>("row:e8r2", 1),
                             make<RowV<256, 16, 8>>("row:e16r8", 1)};
StepVariant<float> v1024[] = {make<ColV<1024, 16>>("col:e16", 0), make<RowV<1024, 8, 1>>("row:e8r1", 1),
                              make<RowV<1024, 16, 4>>("row:e16r4", 1)};

}  // namespace

int step_variants_f32(int n, StepVariant<float>** out) {
    switch (n) {
        case 64: *out = v64; return 3;
        case 128: *out = v128; return 3;
        case 256: *out = v256; return 3;
        case 1024: *out = v1024; return 3;
        default: *out = nullptr; return 0;
    }
}

}  // namespace qaf
