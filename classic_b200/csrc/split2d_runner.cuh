// Runner of the fused 2D dimensionally split step (step2ds.cuh), shared by the
// reference-order unit (split2d.cu, --fmad=false, BUILD 0) and the contracted
// unit (split2d_fast.cu, --fmad=true, BUILD 1): dimensional_split = 1
// (Godunov, method(3) = -1) and 2 (Strang, method(3) = -2), src/2d/claw2ez.f:126.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <type_traits>

#include "host.h"
#include "riemann.cuh"
#include "step2ds.cuh"

namespace clawb200 {

template <class S, class M, bool STRANG, bool SRC, int BUILD>
struct SplitRunner2D : Runner {
    using L = SplitLayout<S, STRANG>;
    Step2Args<S> args;
    int grid = 1, smem = 0;

    explicit SplitRunner2D(const S& s) { std::memset(&args, 0, sizeof(args)); args.solver = s; }

    int prepare(const claw_config& cfg, const Geometry& g) override {
        args.q[0] = static_cast<typename S::real*>(g.q[0]);
        args.q[1] = static_cast<typename S::real*>(g.q[1]);
        args.aux = static_cast<const typename S::real*>(g.aux);
        args.ld = g.ld;
        args.fstride = g.fstride;
        args.ald = g.ald;
        args.afstride = g.afstride;
        args.mx = g.mx;
        args.my = g.my;
        args.nstrips = (g.mx + L::STRIPW - 1) / L::STRIPW;
        args.bc[0] = cfg.bc_lower[0];
        args.bc[1] = cfg.bc_upper[0];
        args.bc[2] = cfg.bc_lower[1];
        args.bc[3] = cfg.bc_upper[1];
        for (int k = 0; k < 8; ++k) args.mthlim[k] = k < cfg.num_waves ? cfg.limiter[k] : 0;
        args.order = cfg.order;
        args.trans = -cfg.dimensional_split;
        args.fwave = cfg.use_fwaves;
        args.capa = cfg.capa_index;
        args.dx = g.dx;
        args.dy = g.dy;
        args.ctl = g.ctl;
        args.src_split = (SRC && cfg.source_id == CLAW_SOURCE_RADIAL) ? cfg.source_split : 0;
        args.src_nd1 = (double)(cfg.source_ndim - 1);
        args.src_bulk = cfg.solver_params[1];
        args.xlower = cfg.lower[0];
        for (int k = 0; k < 2; ++k) {
            int rc = make_map3(&args.tmq[k], g.q[k], g.es, g.mx, g.my, S::meqn, g.ld, g.fstride,
                               L::W, 1, S::meqn);
            if (rc) return rc;
        }
        if (S::maux > 0) {
            int rc = make_map3(&args.tmaux, g.aux, g.es, g.mx + 4, g.my + 4, S::maux, g.ald,
                               g.afstride, L::W, 1, S::maux);
            if (rc) return rc;
        }
        smem = L::SMEM;
        auto kern = split2_kernel<S, M, STRANG, SRC, BUILD>;
        CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        int dev = 0, nsm = 0, per_sm = 0;
        CUDA_TRY(cudaGetDevice(&dev));
        CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * WARPS2D, smem));
        if (per_sm < 1) return fail(CLAW_E_CUDA, "split step kernel cannot be resident on an SM");
        args.units = (long long)args.nstrips * g.my;
        const long long full = (long long)nsm * per_sm * WARPS2D;
        const int nw = row_blocks(full, args.nstrips, g.my, CLAW_STEP2_MIN_ROWS, &args.brows, &args.nblocks);
        grid = (nw + WARPS2D - 1) / WARPS2D;
        args.nwarps = nw;
        return 0;
    }

    cudaError_t launch(cudaStream_t s) override {
        return launch_step(split2_kernel<S, M, STRANG, SRC, BUILD>, dim3(grid), dim3(32 * WARPS2D), smem, s, args);
    }
};

template <class S, int BUILD>
std::unique_ptr<Runner> split_for(const claw_config& cfg, const S& s) {
    if constexpr (std::is_same<S, Acoustics2D<typename S::real>>::value) {
        if (cfg.source_id == CLAW_SOURCE_RADIAL && cfg.source_split != 0) {
            if (cfg.dimensional_split == 2)
                return std::unique_ptr<Runner>(new SplitRunner2D<S, MethodGeneric2D, true, true, BUILD>(s));
            return std::unique_ptr<Runner>(new SplitRunner2D<S, MethodGeneric2D, false, true, BUILD>(s));
        }
    }
    bool mc = cfg.order == 2 && cfg.capa_index == 0 && !cfg.use_fwaves;
    for (int k = 0; k < cfg.num_waves; ++k) mc = mc && cfg.limiter[k] == 4;
    // order 2, MC, no capacity, no f-waves: the specialised policy; the
    // transverse code is unused by the split kernels
    using MC = Method2D<2, -1, 4, 0, 0>;
    if (cfg.dimensional_split == 2) {
        if (mc) return std::unique_ptr<Runner>(new SplitRunner2D<S, MC, true, false, BUILD>(s));
        return std::unique_ptr<Runner>(new SplitRunner2D<S, MethodGeneric2D, true, false, BUILD>(s));
    }
    if (mc) return std::unique_ptr<Runner>(new SplitRunner2D<S, MC, false, false, BUILD>(s));
    return std::unique_ptr<Runner>(new SplitRunner2D<S, MethodGeneric2D, false, false, BUILD>(s));
}

template <typename real, int BUILD>
std::unique_ptr<Runner> split_runner_for(const claw_config& cfg) {
    switch (cfg.solver_id) {
        case CLAW_SOLVER_ACOUSTICS_2D: {
            const double rho = cfg.solver_params[0], bulk = cfg.solver_params[1];
            const double cc = std::sqrt(bulk / rho), zz = rho * cc, hz = 0.5 / zz;
            return split_for<Acoustics2D<real>, BUILD>(cfg, Acoustics2D<real>{(real)cc, (real)zz, (real)hz});
        }
        case CLAW_SOLVER_EULER_ROE_2D: {
            const double gamma = cfg.solver_params[0];
            return split_for<EulerRoe2D<real>, BUILD>(cfg, EulerRoe2D<real>{(real)gamma, (real)(gamma - 1.0)});
        }
        case CLAW_SOLVER_VC_ADVECTION_2D:
            return std::unique_ptr<Runner>(
                cfg.dimensional_split == 2
                    ? static_cast<Runner*>(new SplitRunner2D<VCAdvection2D<real>, MethodGeneric2D, true, false, BUILD>({}))
                    : static_cast<Runner*>(new SplitRunner2D<VCAdvection2D<real>, MethodGeneric2D, false, false, BUILD>({})));
        default:
            return nullptr;
    }
}

}  // namespace clawb200
