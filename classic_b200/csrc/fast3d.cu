// The 3D step with fused multiply-adds (CLAW_FP64_FMA) and in FP32
// (CLAW_FP32; Courant number, dt and time stay FP64): the same kernels as
// claw3d.cu compiled with --fmad=true.
#include "runner3d.cuh"

namespace clawb200 {

std::unique_ptr<Runner> make_fast_runner3d(const claw_config& cfg) {
    if (cfg.solver_id != CLAW_SOLVER_VC_ACOUSTICS_3D) return nullptr;
    if (cfg.dimensional_split > 0) {
        if (cfg.precision == CLAW_FP32)
            return std::unique_ptr<Runner>(new SplitRunner3D<VCAcoustics3D<float>, 1>());
        if (cfg.precision == CLAW_FP64_FMA)
            return std::unique_ptr<Runner>(new SplitRunner3D<VCAcoustics3D<double>, 1>());
        return nullptr;
    }
    if (cfg.precision == CLAW_FP32) return runner3d_for<float, 1>(cfg);
    if (cfg.precision == CLAW_FP64_FMA) return runner3d_for<double, 1>(cfg);
    return nullptr;
}

}  // namespace clawb200
