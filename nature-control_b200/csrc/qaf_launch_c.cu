// qaf_launch_c.cu — instantiates the per-size launchers (qaf_launch.cuh) for
// grid sizes 512, 96 and 128 in FP32 and FP64; the four qaf_launch_*.cu files split
// the library's kernel instantiations so that they compile in parallel.
#include "qaf_launch.cuh"

namespace qaf {
namespace detail {

#if !defined(QAF_ONLY_N) || QAF_ONLY_N == 512
template struct Launch<float, 512>;
template struct Launch<double, 512>;
#endif
#if !defined(QAF_ONLY_N) || QAF_ONLY_N == 96
template struct Launch<float, 96>;
template struct Launch<double, 96>;
#endif
#if !defined(QAF_ONLY_N) || QAF_ONLY_N == 128
template struct Launch<float, 128>;
template struct Launch<double, 128>;
#endif

}  // namespace detail
}  // namespace qaf
