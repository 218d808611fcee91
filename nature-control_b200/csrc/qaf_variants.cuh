// qaf_variants.cuh — alternative launch shapes of the fused step kernels,
// chosen at run time by the autotuner (qaf_autotune in include/qaf.h).
//
// The state, Y/G and edge layouts do not depend on these shapes (only on TW),
// so a variant can replace the built-in launch of a kernel between any two
// launches. Variants exist for FP32 at the sizes the ensemble and adjoint
// workloads use; they are compiled in their own translation unit
// (qaf_variants.cu) in parallel with the rest of the library.
#pragma once

#include <cuda_runtime.h>

#include "qaf_stage.cuh"

namespace qaf {

template <typename real>
struct StepVariant {
    const char* name;   // "col:e16", "row:e8r2", ...
    int kind;           // 0: column kernel, 1: row kernel
    // attributes and resident column CTAs for the current device (the caller
    // runs it once per device)
    cudaError_t (*setup)(int* slots);
    void (*launch)(const StageArgs<real>& a, int slots, cudaStream_t st);
};

// the variants for grid size n (FP32); *out points at a static table, returns its length (0: none)
int step_variants_f32(int n, StepVariant<float>** out);

}  // namespace qaf
