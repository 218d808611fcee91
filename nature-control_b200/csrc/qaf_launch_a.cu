// qaf_launch_a.cu — instantiates the per-size launchers (qaf_launch.cuh) for
// grid sizes 1024, 16 and 32 in FP32 and FP64; the four qaf_launch_*.cu files split
// the library's kernel instantiations so that they compile in parallel.
#include "qaf_launch.cuh"

namespace qaf {
namespace detail {

#if !defined(QAF_ONLY_N) || QAF_ONLY_N == 1024
template struct Launch<float, 1024>;
template struct Launch<double, 1024>;
#endif
#if !defined(QAF_ONLY_N) || QAF_ONLY_N == 16
template struct Launch<float, 16>;
template struct Launch<double, 16>;
#endif
#if !defined(QAF_ONLY_N) || QAF_ONLY_N == 32
template struct Launch<float, 32>;
template struct Launch<double, 32>;
#endif

}  // namespace detail
}  // namespace qaf
