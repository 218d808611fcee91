// qaf_launch_b.cu — instantiates the per-size launchers (qaf_launch.cuh) for
// grid sizes 768, 48 and 64 in FP32 and FP64; the four qaf_launch_*.cu files split
// the library's kernel instantiations so that they compile in parallel.
#include "qaf_launch.cuh"

namespace qaf {
namespace detail {

#if !defined(QAF_ONLY_N) || QAF_ONLY_N == 768
template struct Launch<float, 768>;
template struct Launch<double, 768>;
#endif
#if !defined(QAF_ONLY_N) || QAF_ONLY_N == 48
template struct Launch<float, 48>;
template struct Launch<double, 48>;
#endif
#if !defined(QAF_ONLY_N) || QAF_ONLY_N == 64
template struct Launch<float, 64>;
template struct Launch<double, 64>;
#endif

}  // namespace detail
}  // namespace qaf
