// The characteristic-variable 2D acoustics kernel with MC on wave 1 and
// another limiter compiled in on wave 2 (order 2, transverse 2; FP64
// contracted and FP32), in its own translation unit so that the pairs compile
// in parallel.  Built with fused multiply-add contraction.
#include "char2d_runner.cuh"

namespace clawb200 {
template std::unique_ptr<Runner> char_pair_limited<4, 1>(bool, int);
template std::unique_ptr<Runner> char_pair_limited<4, 2>(bool, int);
template std::unique_ptr<Runner> char_pair_limited<4, 3>(bool, int);
}  // namespace clawb200
