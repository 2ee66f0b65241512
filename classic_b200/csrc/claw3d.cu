// The 3D step in the reference's order of operations (--fmad=false):
// bit-identical to the CPU restatement of step3 / flux3 / claw3.
#include "runner3d.cuh"

namespace clawb200 {

std::unique_ptr<Runner> make_runner3d(const claw_config& cfg) {
    if (cfg.solver_id != CLAW_SOLVER_VC_ACOUSTICS_3D) return nullptr;
    if (cfg.precision != CLAW_FP64) return make_fast_runner3d(cfg);
    return runner3d_for<double, 0>(cfg);
}

}  // namespace clawb200
