// Characteristic-variable 2D acoustics runner (char2d.cuh, char2d_runner.cuh).
// This translation unit is compiled with fused multiply-add contraction; it
// serves CLAW_FP64_FMA and CLAW_FP32.
#include "char2d_runner.cuh"

namespace clawb200 {

namespace {

// (order, transverse_waves): at order 2 one limiter on both waves is compiled
// in (MC here; minmod, superbee and van Leer in their own units), and at
// transverse 2 so is every pair of two different ones of these four (the
// fast2d_pairs_*.cu units); other settings -- none or Beam-Warming on a wave,
// a pair at transverse 0 or 1 -- read the limiters at run time (LIM = -1);
// order 1 uses none.
template <typename real, int BCM>
std::unique_ptr<Runner> pick_lim(int l1, int l2, int order, int trans) {
    const int lim = l1 == l2 ? l1 : -1;
    if (order == 2) {
        if (trans < 0 || trans > 2) return nullptr;
        if (lim == -1 && trans == 2) {
            auto r = char_pair_runner(l1, l2, sizeof(real) == 4, BCM);
            if (r) return r;
        }
        if (lim == 4) return char_order2<real, 4, BCM>(trans);
        if (lim >= 1 && lim <= 3) {
            constexpr bool f32 = sizeof(real) == 4;
            if (lim == 1) return char_order2_limited<1>(f32, BCM, trans);
            if (lim == 2) return char_order2_limited<2>(f32, BCM, trans);
            return char_order2_limited<3>(f32, BCM, trans);
        }
        return char_order2<real, -1, BCM>(trans);
    }
    if (order == 1 && trans == 1) return std::unique_ptr<Runner>(new CharRunner<real, -1, BCM, 1, 1>());
    if (order == 1 && trans == 0) return std::unique_ptr<Runner>(new CharRunner<real, -1, BCM, 1, 0>());
    return nullptr;
}

template <typename real>
std::unique_ptr<Runner> pick(const claw_config& cfg) {
    const bool px = cfg.bc_lower[0] == BC_PERIODIC || cfg.bc_upper[0] == BC_PERIODIC;
    bool extrap = true;
    for (int d = 0; d < 2; ++d) extrap = extrap && cfg.bc_lower[d] == BC_EXTRAP && cfg.bc_upper[d] == BC_EXTRAP;
    const int o = cfg.order, tr = cfg.transverse_waves;
    const int l1 = cfg.limiter[0], l2 = cfg.limiter[1];
    if (px) return pick_lim<real, CHAR_BC_PERX>(l1, l2, o, tr);
    if (extrap) return pick_lim<real, CHAR_BC_EXTRAP>(l1, l2, o, tr);
    return pick_lim<real, CHAR_BC_WALLS>(l1, l2, o, tr);
}

}  // namespace

std::unique_ptr<Runner> make_char_runner(const claw_config& cfg) {
    if (cfg.solver_id != CLAW_SOLVER_ACOUSTICS_2D || cfg.num_dim != 2) return nullptr;
    if (cfg.order < 1 || cfg.order > 2 || cfg.transverse_waves < 0 || cfg.transverse_waves > cfg.order ||
        cfg.capa_index != 0 || cfg.use_fwaves)
        return nullptr;
    if (cfg.num_waves != 2) return nullptr;
    if (cfg.precision == CLAW_FP32) return pick<float>(cfg);
    if (cfg.precision == CLAW_FP64_FMA) return pick<double>(cfg);
    return nullptr;
}

}  // namespace clawb200
