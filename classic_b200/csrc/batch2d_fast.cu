// The batched 2D step of the contracted build (CLAW_FP64_FMA): the batch
// kernel of batch2d.cu compiled with --fmad=true, with Newton reciprocals and
// square roots in the Roe solver and compare-and-select limiters
// (Method2D<..., FAST = 1>, EulerRoe2D<double, true>).  Each instance's
// Courant number is formed as in the reference-order build.
#include <cmath>
#include <memory>

#include "batch2d_runner.cuh"
#include "riemann.cuh"

namespace clawb200 {

namespace {

template <class S>
std::unique_ptr<BatchRunner> fast_batch_runner(const claw_config& cfg, const S& s) {
    bool mc = cfg.order == 2 && cfg.transverse_waves == 2 && cfg.capa_index == 0 && !cfg.use_fwaves;
    for (int k = 0; k < cfg.num_waves; ++k) mc = mc && cfg.limiter[k] == 4;
    if (mc) return std::unique_ptr<BatchRunner>(new BatchRunnerT<S, MethodMC2DFast>(s));
    return std::unique_ptr<BatchRunner>(new BatchRunnerT<S, MethodGeneric2DFast>(s));
}

}  // namespace

std::unique_ptr<BatchRunner> make_fast_batch_runner(const claw_config& cfg) {
    if (cfg.solver_id == CLAW_SOLVER_EULER_ROE_2D) {
        const double gamma = cfg.solver_params[0];
        return fast_batch_runner(cfg, EulerRoe2D<double, true>{gamma, gamma - 1.0});
    }
    if (cfg.solver_id == CLAW_SOLVER_ACOUSTICS_2D) {
        const double rho = cfg.solver_params[0], bulk = cfg.solver_params[1];
        const double cc = std::sqrt(bulk / rho), zz = rho * cc, hz = 0.5 / zz;
        return fast_batch_runner(cfg, Acoustics2D<double>{cc, zz, hz});
    }
    return nullptr;
}

}  // namespace clawb200
