// The 2D unsplit step of the contracted build (CLAW_FP64_FMA) for the
// methods and solvers the characteristic-variable kernel does not serve:
// step2d.cuh's kernel with fused multiply-adds (this translation unit is
// compiled with --fmad=true), Newton reciprocals and square roots, and
// compare-and-select limiters (Method2D<..., FAST = 1>).  The Courant number
// is formed as in the reference-order build.
#include <cmath>
#include <memory>

#include "riemann.cuh"
#include "runner2d.cuh"

namespace clawb200 {

namespace {

bool mc_everywhere(const claw_config& cfg) {
    bool mc = cfg.order == 2 && cfg.transverse_waves == 2 && cfg.capa_index == 0 && !cfg.use_fwaves;
    for (int k = 0; k < cfg.num_waves; ++k) mc = mc && cfg.limiter[k] == 4;
    return mc;
}

template <class S>
std::unique_ptr<Runner> fast_runner(const claw_config& cfg, const S& s) {
    if (mc_everywhere(cfg)) return std::unique_ptr<Runner>(new Runner2D<S, MethodMC2DFast>(s));
    return std::unique_ptr<Runner>(new Runner2D<S, MethodGeneric2DFast>(s));
}

}  // namespace

std::unique_ptr<Runner> make_fast_runner2d(const claw_config& cfg) {
    if (cfg.num_dim != 2 || cfg.precision != CLAW_FP64_FMA || cfg.dimensional_split > 0) return nullptr;
    if (cfg.source_id != CLAW_SOURCE_NONE && cfg.source_split != 0) return nullptr;
    const int id = cfg.solver_id;
    if (id == CLAW_SOLVER_ACOUSTICS_2D) {
        const double rho = cfg.solver_params[0], bulk = cfg.solver_params[1];
        const double cc = std::sqrt(bulk / rho), zz = rho * cc, hz = 0.5 / zz;
        return fast_runner(cfg, Acoustics2D<double>{cc, zz, hz});
    }
    if (id == CLAW_SOLVER_EULER_ROE_2D) {
        const double gamma = cfg.solver_params[0];
        return fast_runner(cfg, EulerRoe2D<double, true>{gamma, gamma - 1.0});
    }
    if (id == CLAW_SOLVER_VC_ADVECTION_2D)
        return std::unique_ptr<Runner>(
            new Runner2D<VCAdvection2D<double>, MethodGeneric2DFast>(VCAdvection2D<double>{}));
    return nullptr;
}

}  // namespace clawb200
