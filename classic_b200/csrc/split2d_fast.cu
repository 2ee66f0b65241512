// The 2D dimensionally split step with fused multiply-adds (CLAW_FP64_FMA) and
// in FP32 (CLAW_FP32; Courant numbers, dt and time stay FP64): the kernels of
// split2d.cu compiled with --fmad=true.
#include "split2d_runner.cuh"

namespace clawb200 {

std::unique_ptr<Runner> make_fast_split_runner(const claw_config& cfg) {
    if (cfg.num_dim != 2 || cfg.dimensional_split <= 0) return nullptr;
    if (auto r = make_char_split_runner(cfg)) return r;  // constant-coefficient acoustics
    if (cfg.precision == CLAW_FP32) return split_runner_for<float, 1>(cfg);
    if (cfg.precision == CLAW_FP64_FMA) return split_runner_for<double, 1>(cfg);
    return nullptr;
}

}  // namespace clawb200
