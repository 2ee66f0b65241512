// The 3D step in the reference's order of operations (--fmad=false):
// bit-identical to the CPU restatement of step3 / flux3 / claw3, and of
// dimsp3 / step3ds when dimensional splitting is on.  FP32 and fused FP64 go
// to the contracted build (fast3d.cu).
#include "runner3d.cuh"

namespace clawb200 {

std::unique_ptr<Runner> make_runner3d(const claw_config& cfg) {
    if (cfg.solver_id != CLAW_SOLVER_VC_ACOUSTICS_3D) return nullptr;
    if (cfg.precision != CLAW_FP64) return make_fast_runner3d(cfg);
    // src/3d/claw3ez.f:136: any splitting request runs dimsp3's Godunov splitting
    if (cfg.dimensional_split > 0)
        return std::unique_ptr<Runner>(new SplitRunner3D<VCAcoustics3D<double>, 0>());
    return runner3d_for<double, 0>(cfg);
}

}  // namespace clawb200
