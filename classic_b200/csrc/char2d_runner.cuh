// Host side of the characteristic-variable 2D acoustics kernel (char2d.cuh):
// the runner that prepares its tensor maps and work split and launches it,
// and the factory for one limiter compiled in at order 2.  Included by the
// translation units that instantiate the kernel (all built with fused
// multiply-add contraction).
#pragma once
#include <algorithm>
#include <cstring>
#include <memory>

#include "char2d.cuh"
#include "host.h"

#ifndef CLAW_CHAR_MIN_ROWS
#define CLAW_CHAR_MIN_ROWS 8  // fewest rows of a work item (small grids: more items, more warps)
#endif

namespace clawb200 {

template <typename real, int LIM, int BCM, int ORD, int TRN, int LIM2 = LIM>
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
        CUDA_TRY(cudaFuncSetAttribute(step2_char_kernel<real, LIM, BCM, ORD, TRN, LIM2>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        int dev = 0, nsm = 0, per_sm = 0;
        CUDA_TRY(cudaGetDevice(&dev));
        CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step2_char_kernel<real, LIM, BCM, ORD, TRN, LIM2>,
                                                               32 * WARPS2D, smem));
        if (per_sm < 1) return fail(CLAW_E_CUDA, "characteristic kernel cannot be resident");
        const long long full = (long long)nsm * per_sm * WARPS2D;
        const int nw = row_blocks(full, args.nstrips, g.my, CLAW_CHAR_MIN_ROWS, &args.brows, &args.nblocks);
        grid = (nw + WARPS2D - 1) / WARPS2D;
        args.nwarps = nw;
        return 0;
    }

    cudaError_t launch(cudaStream_t s) override {
        return launch_step(step2_char_kernel<real, LIM, BCM, ORD, TRN, LIM2>, dim3(grid), dim3(32 * WARPS2D), smem, s,
                           args);
    }
};

// Order 2 with limiter LIM on both waves, for every transverse_waves setting
// (0, 1, 2) and boundary mode of the kernel; nullptr for other settings.
template <typename real, int LIM, int BCM>
std::unique_ptr<Runner> char_order2(int trans) {
    if (trans == 2) return std::unique_ptr<Runner>(new CharRunner<real, LIM, BCM, 2, 2>());
    if (trans == 1) return std::unique_ptr<Runner>(new CharRunner<real, LIM, BCM, 2, 1>());
    if (trans == 0) return std::unique_ptr<Runner>(new CharRunner<real, LIM, BCM, 2, 0>());
    return nullptr;
}

template <int LIM>
std::unique_ptr<Runner> char_order2_limited(bool fp32, int bcm, int trans) {
    if (fp32) {
        if (bcm == CHAR_BC_PERX) return char_order2<float, LIM, CHAR_BC_PERX>(trans);
        if (bcm == CHAR_BC_EXTRAP) return char_order2<float, LIM, CHAR_BC_EXTRAP>(trans);
        return char_order2<float, LIM, CHAR_BC_WALLS>(trans);
    }
    if (bcm == CHAR_BC_PERX) return char_order2<double, LIM, CHAR_BC_PERX>(trans);
    if (bcm == CHAR_BC_EXTRAP) return char_order2<double, LIM, CHAR_BC_EXTRAP>(trans);
    return char_order2<double, LIM, CHAR_BC_WALLS>(trans);
}

// minmod (1), superbee (2) and van Leer (3) each in a translation unit of its
// own (fast2d_minmod.cu, fast2d_superbee.cu, fast2d_vanleer.cu)
extern template std::unique_ptr<Runner> char_order2_limited<1>(bool, int, int);
extern template std::unique_ptr<Runner> char_order2_limited<2>(bool, int, int);
extern template std::unique_ptr<Runner> char_order2_limited<3>(bool, int, int);

// Order 2, transverse 2 with limiter L1 on wave 1 and L2 on wave 2 (L1 != L2,
// both of minmod 1, superbee 2, van Leer 3, MC 4), every boundary mode; the
// pairs with wave 1's limiter L1 are compiled in fast2d_pairs_<L1>.cu.
template <int L1, int L2>
std::unique_ptr<Runner> char_pair_limited(bool fp32, int bcm) {
    if (fp32) {
        if (bcm == CHAR_BC_PERX) return std::unique_ptr<Runner>(new CharRunner<float, L1, CHAR_BC_PERX, 2, 2, L2>());
        if (bcm == CHAR_BC_EXTRAP) return std::unique_ptr<Runner>(new CharRunner<float, L1, CHAR_BC_EXTRAP, 2, 2, L2>());
        return std::unique_ptr<Runner>(new CharRunner<float, L1, CHAR_BC_WALLS, 2, 2, L2>());
    }
    if (bcm == CHAR_BC_PERX) return std::unique_ptr<Runner>(new CharRunner<double, L1, CHAR_BC_PERX, 2, 2, L2>());
    if (bcm == CHAR_BC_EXTRAP) return std::unique_ptr<Runner>(new CharRunner<double, L1, CHAR_BC_EXTRAP, 2, 2, L2>());
    return std::unique_ptr<Runner>(new CharRunner<double, L1, CHAR_BC_WALLS, 2, 2, L2>());
}

#define CLAW_CHAR_PAIRS_OF(L1, A, B, C)                                                   \
    extern template std::unique_ptr<Runner> char_pair_limited<L1, A>(bool, int);          \
    extern template std::unique_ptr<Runner> char_pair_limited<L1, B>(bool, int);          \
    extern template std::unique_ptr<Runner> char_pair_limited<L1, C>(bool, int);
CLAW_CHAR_PAIRS_OF(1, 2, 3, 4)
CLAW_CHAR_PAIRS_OF(2, 1, 3, 4)
CLAW_CHAR_PAIRS_OF(3, 1, 2, 4)
CLAW_CHAR_PAIRS_OF(4, 1, 2, 3)
#undef CLAW_CHAR_PAIRS_OF

// The compiled runner for wave limiters l1 != l2 at order 2, transverse 2, or
// nullptr (another pair or setting: the limiters are read at run time).
inline std::unique_ptr<Runner> char_pair_runner(int l1, int l2, bool fp32, int bcm) {
    if (l1 < 1 || l1 > 4 || l2 < 1 || l2 > 4 || l1 == l2) return nullptr;
    switch (l1 * 10 + l2) {
        case 12: return char_pair_limited<1, 2>(fp32, bcm);
        case 13: return char_pair_limited<1, 3>(fp32, bcm);
        case 14: return char_pair_limited<1, 4>(fp32, bcm);
        case 21: return char_pair_limited<2, 1>(fp32, bcm);
        case 23: return char_pair_limited<2, 3>(fp32, bcm);
        case 24: return char_pair_limited<2, 4>(fp32, bcm);
        case 31: return char_pair_limited<3, 1>(fp32, bcm);
        case 32: return char_pair_limited<3, 2>(fp32, bcm);
        case 34: return char_pair_limited<3, 4>(fp32, bcm);
        case 41: return char_pair_limited<4, 1>(fp32, bcm);
        case 42: return char_pair_limited<4, 2>(fp32, bcm);
        case 43: return char_pair_limited<4, 3>(fp32, bcm);
    }
    return nullptr;
}

}  // namespace clawb200
