// The 2D dimensionally split step in the reference's order of operations
// (--fmad=false): bit-identical to the oracle's dimsp2 / step2ds.  FP32 and
// fused FP64 go to the contracted build (split2d_fast.cu).
#include "split2d_runner.cuh"

namespace clawb200 {

std::unique_ptr<Runner> make_split_runner(const claw_config& cfg) {
    if (cfg.num_dim != 2 || cfg.dimensional_split <= 0) return nullptr;
    if (cfg.precision != CLAW_FP64) return make_fast_split_runner(cfg);
    return split_runner_for<double, 0>(cfg);
}

}  // namespace clawb200
