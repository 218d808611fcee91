// qaf_variants.cu — FP32 launch variants of the fused step kernels for the
// autotuner (see qaf_variants.cuh): column kernel with 16 (or, at 64^2, 4 —
// the built-in shape there since it timed fastest) values per thread of the
// y-FFT instead of 8, or a tighter register budget
// (more resident CTAs); at 1024^2, where the built-in column kernel takes 4
// values per thread in one 1024-thread CTA per SM, the 8-value two-CTA
// shapes (twiddle bases in shared memory or in registers); row kernel with
// fewer rows per CTA (more CTAs for
// small grids), 16 values per thread of the x-FFT, or a tighter register budget
// (row:e8r1m7 at 1024^2: one row per CTA at 7 CTAs per SM, so the 1024 rows
// fit the 1036 slots of one wave; 72 registers with spills, within 1% of the
// built-in two-row shape in same-box A/B runs).
#include "qaf_kernels.cuh"
#include "qaf_variants.cuh"

namespace qaf {
namespace {

template <int N, int EC, int MINB = 2, int MODE = 0>
struct ColV {
    static constexpr int THREADS = TW * (N / EC);
    static constexpr size_t SMEM = ColKernel<float, N, EC, MODE>::SMEM;
    static cudaError_t setup(int* slots) {
        cudaError_t e = cudaFuncSetAttribute(col_kernel<float, N, EC, MINB, MODE>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
        if (e != cudaSuccess) return e;
        int dev = 0, sms = 0, per_sm = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, col_kernel<float, N, EC, MINB, MODE>, THREADS,
                                                               SMEM)) != cudaSuccess)
            return e;
        if (per_sm < 1) return cudaErrorInvalidConfiguration;
        *slots = sms * per_sm;
        return cudaSuccess;
    }
    static void launch(const StageArgs<float>& a, int slots, cudaStream_t st) {
        const long items = (long)(2 * (a.nx / 2 / TW) + 3) * a.ninst;
        const int grid = items < slots ? (int)items : slots;
        col_kernel<float, N, EC, MINB, MODE><<<grid, THREADS, SMEM, st>>>(a);
    }
};

template <int N, int ER, int ROWS, int MINB = 2, int MODE = 0>
struct RowV {
    static constexpr int THREADS = ROWS * (N / ER);
    static constexpr size_t SMEM = RowKernel<float, N, ER, ROWS, MODE>::SMEM;
    static cudaError_t setup(int* slots) {
        *slots = 0;
        return cudaFuncSetAttribute(row_kernel<float, N, ER, ROWS, MINB, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)SMEM);
    }
    static void launch(const StageArgs<float>& a, int, cudaStream_t st) {
        row_kernel<float, N, ER, ROWS, MINB, MODE><<<(a.ny / ROWS) * a.ninst, THREADS, SMEM, st>>>(a);
    }
};

template <class V>
constexpr StepVariant<float> make(const char* name, int kind) {
    return StepVariant<float>{name, kind, &V::setup, &V::launch};
}

// "m<k>": register budget for k resident CTAs per SM (occupancy for batched small grids)
StepVariant<float> v64[] = {make<ColV<64, 4>>("col:e4", 0), make<ColV<64, 8, 8>>("col:e8m8", 0),
                            make<RowV<64, 8, 2>>("row:e8r2", 1), make<RowV<64, 16, 4>>("row:e16r4", 1),
                            make<RowV<64, 8, 8, 4>>("row:e8r8m4", 1)};
StepVariant<float> v128[] = {make<ColV<128, 16>>("col:e16", 0), make<ColV<128, 8, 6>>("col:e8m6", 0),
                             make<RowV<128, 8, 2>>("row:e8r2", 1), make<RowV<128, 16, 8>>("row:e16r8", 1),
                             make<RowV<128, 8, 16, 3>>("row:e8r16m3", 1)};
StepVariant<float> v256[] = {make<ColV<256, 16>>("col:e16", 0), make<ColV<256, 8, 4>>("col:e8m4", 0),
                             make<ColV<256, 8, 6>>("col:e8m6", 0), make<RowV<256, 8, 2>>("row:e8r2", 1),
                             make<RowV<256, 16, 8>>("row:e16r8", 1), make<RowV<256, 8, 8, 3>>("row:e8r8m3", 1)};
StepVariant<float> v1024[] = {make<ColV<1024, 16>>("col:e16", 0), make<ColV<1024, 8, 2, 1>>("col:e8s", 0),
                              make<ColV<1024, 8>>("col:e8", 0), make<RowV<1024, 8, 1>>("row:e8r1", 1),
                              make<RowV<1024, 16, 4>>("row:e16r4", 1), make<RowV<1024, 8, 1, 7>>("row:e8r1m7", 1),
                              make<RowV<1024, 4, 4, 1>>("row:e4r4", 1), make<RowV<1024, 4, 4, 1, 1>>("row:e4r4s", 1),
                              make<RowV<1024, 4, 2, 2, 1>>("row:e4r2s", 1)};

}  // namespace

int step_variants_f32(int n, StepVariant<float>** out) {
    switch (n) {
        case 64: *out = v64; return (int)(sizeof(v64) / sizeof(v64[0]));
        case 128: *out = v128; return (int)(sizeof(v128) / sizeof(v128[0]));
        case 256: *out = v256; return (int)(sizeof(v256) / sizeof(v256[0]));
        case 1024: *out = v1024; return (int)(sizeof(v1024) / sizeof(v1024[0]));
        default: *out = nullptr; return 0;
    }
}

}  // namespace qaf
