// qaf_launch_d.cu — instantiates the per-size launchers (qaf_launch.cuh) for
// grid sizes 384, 192 and 256 in FP32 and FP64; the four qaf_launch_*.cu files split
// the library's kernel instantiations so that they compile in parallel.
#include "qaf_launch.cuh"

namespace qaf {
namespace detail {

#if !defined(QAF_ONLY_N) || QAF_ONLY_N == 384
template struct Launch<float, 384>;
template struct Launch<double, 384>;
#endif
#if !defined(QAF_ONLY_N) || QAF_ONLY_N == 192
template struct Launch<float, 192>;
template struct Launch<double, 192>;
#endif
#if !defined(QAF_ONLY_N) || QAF_ONLY_N == 256
template struct Launch<float, 256>;
template struct Launch<double, 256>;
#endif

}  // namespace detail
}  // namespace qaf
