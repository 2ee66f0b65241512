// The characteristic-variable 2D acoustics kernel with superbee compiled in
// on both waves at order 2 (FP64 contracted and FP32), in its own translation
// unit so that the limiters compile in parallel.  Built with fused
// multiply-add contraction.
#include "char2d_runner.cuh"

namespace clawb200 {
template std::unique_ptr<Runner> char_order2_limited<2>(bool, int, int);
}  // namespace clawb200
