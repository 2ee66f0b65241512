// Characteristic-variable 2D acoustics runner (char2d.cuh).  This
// translation unit is compiled with fused multiply-add contraction; it
// serves CLAW_FP64_FMA and CLAW_FP32.
#include <algorithm>
#include <cstring>
#include <memory>

#include "char2d.cuh"
#include "host.h"

#ifndef CLAW_CHAR_MIN_ROWS
#define CLAW_CHAR_MIN_ROWS 8  // fewest rows of a work item (small grids: more items, more warps)
#endif

namespace clawb200 {

namespace {

template <typename real, int LIM, int BCM, int ORD, int TRN>
struct CharRunner : Runner {
    CharArgs<real> args;
    int grid = 1, smem = 0;

    int prepare(const claw_config& cfg, const Geometry& g) override {
        using R = CharRing<real>;
        std::memset(&args, 0, sizeof(args));
        const double rho = cfg.solver_params[0], bulk = cfg.solver_params[1];
        const double cc = std::sqrt(bulk / rho), zz = rho * cc;
        args.s = CharAcoustics2D<real>{(real)cc, (real)zz, (real)(0.5 / zz)};
        args.q[0] = static_cast<real*>(g.q[0]);
        args.q[1] = static_cast<real*>(g.q[1]);
        args.ld = g.ld;
        args.fstride = g.fstride;
        args.mx = g.mx;
        args.my = g.my;
        args.nstrips = (g.mx + STRIP2 - 1) / STRIP2;
        args.bc[0] = cfg.bc_lower[0];
        args.bc[1] = cfg.bc_upper[0];
        args.bc[2] = cfg.bc_lower[1];
        args.bc[3] = cfg.bc_upper[1];
        args.lim = cfg.limiter[0];
        args.lim2 = cfg.num_waves > 1 ? cfg.limiter[1] : cfg.limiter[0];
        args.dx = g.dx;
        args.dy = g.dy;
        args.ctl = g.ctl;
        for (int k = 0; k < 2; ++k) {
            const int rc = make_map3(&args.tmq[k], g.q[k], g.es, g.mx, g.my, 3, g.ld, g.fstride, R::W, 1, 3);
            if (rc) return rc;
        }
        smem = R::SMEM;
        CUDA_TRY(cudaFuncSetAttribute(step2_char_kernel<real, LIM, BCM, ORD, TRN>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        int dev = 0, nsm = 0, per_sm = 0;
        CUDA_TRY(cudaGetDevice(&dev));
        CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step2_char_kernel<real, LIM, BCM, ORD, TRN>,
                                                               32 * WARPS2D, smem));
        if (per_sm < 1) return fail(CLAW_E_CUDA, "characteristic kernel cannot be resident");
        const long long full = (long long)nsm * per_sm * WARPS2D;
        const int nw = row_blocks(full, args.nstrips, g.my, CLAW_CHAR_MIN_ROWS, &args.brows, &args.nblocks);
        grid = (nw + WARPS2D - 1) / WARPS2D;
        args.nwarps = nw;
        return 0;
    }

    cudaError_t launch(cudaStream_t s) override {
        step2_char_kernel<real, LIM, BCM, ORD, TRN><<<grid, 32 * WARPS2D, smem, s>>>(args);
        return cudaGetLastError();
    }
};

// (order, transverse_waves): MC at order 2 has its own instantiations; the
// other limiters read the limiter at run time (order 1 uses none).
template <typename real, int BCM>
std::unique_ptr<Runner> pick_lim(int lim, int order, int trans) {
    if (order == 2 && trans == 2) {
        if (lim == 4) return std::unique_ptr<Runner>(new CharRunner<real, 4, BCM, 2, 2>());
        return std::unique_ptr<Runner>(new CharRunner<real, -1, BCM, 2, 2>());
    }
    if (order == 2 && trans == 1) {
        if (lim == 4) return std::unique_ptr<Runner>(new CharRunner<real, 4, BCM, 2, 1>());
        return std::unique_ptr<Runner>(new CharRunner<real, -1, BCM, 2, 1>());
    }
    if (order == 2 && trans == 0) {
        if (lim == 4) return std::unique_ptr<Runner>(new CharRunner<real, 4, BCM, 2, 0>());
        return std::unique_ptr<Runner>(new CharRunner<real, -1, BCM, 2, 0>());
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
    // one limiter for both waves can be compiled in; two different ones are read at run time
    const int lim = cfg.limiter[0] == cfg.limiter[1] ? cfg.limiter[0] : -1;
    if (px) return pick_lim<real, CHAR_BC_PERX>(lim, o, tr);
    if (extrap) return pick_lim<real, CHAR_BC_EXTRAP>(lim, o, tr);
    return pick_lim<real, CHAR_BC_WALLS>(lim, o, tr);
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
