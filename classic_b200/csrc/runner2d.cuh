// The 2D unsplit step kernel (step2d.cuh) bound to one grid: TMA maps, launch
// shape and the launch.  Shared by the reference-order build (claw_b200.cu)
// and the contracted build (fma2d.cu), which instantiate it for distinct
// method policies so that their kernels stay distinct symbols.
#pragma once
#include <algorithm>
#include <cstring>

#include "host.h"
#include "step2d.cuh"

namespace clawb200 {

template <class S, class M, bool SRC = false>
struct Runner2D : Runner {
    Step2Args<S> args;
    int grid = 1, smem = 0;

    explicit Runner2D(const S& s) { std::memset(&args, 0, sizeof(args)); args.solver = s; }

    int prepare(const claw_config& cfg, const Geometry& g) override {
        using R = Ring2D<S>;
        args.q[0] = static_cast<typename S::real*>(g.q[0]);
        args.q[1] = static_cast<typename S::real*>(g.q[1]);
        args.aux = static_cast<const typename S::real*>(g.aux);
        args.ld = g.ld;
        args.fstride = g.fstride;
        args.ald = g.ald;
        args.afstride = g.afstride;
        args.mx = g.mx;
        args.my = g.my;
        args.nstrips = (g.mx + STRIP - 1) / STRIP;
        args.bc[0] = cfg.bc_lower[0];
        args.bc[1] = cfg.bc_upper[0];
        args.bc[2] = cfg.bc_lower[1];
        args.bc[3] = cfg.bc_upper[1];
        for (int k = 0; k < 8; ++k) args.mthlim[k] = k < cfg.num_waves ? cfg.limiter[k] : 0;
        args.order = cfg.order;
        args.trans = cfg.transverse_waves;
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
                               R::W, 1, S::meqn);
            if (rc) return rc;
        }
        if (S::maux > 0) {
            int rc = make_map3(&args.tmaux, g.aux, g.es, g.mx + 4, g.my + 4, S::maux, g.ald,
                               g.afstride, R::W, 1, S::maux);
            if (rc) return rc;
        }
        smem = R::SMEM;
        CUDA_TRY(cudaFuncSetAttribute(step2_kernel<S, M, SRC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem));
        int dev = 0, nsm = 0, per_sm = 0;
        CUDA_TRY(cudaGetDevice(&dev));
        CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step2_kernel<S, M, SRC>,
                                                               32 * WARPS2D, smem));
        if (per_sm < 1) return fail(CLAW_E_CUDA, "step2 kernel cannot be resident on an SM");
        args.units = (long long)args.nstrips * g.my;
        const long long full = (long long)nsm * per_sm * WARPS2D;
        const int nw = row_blocks(full, args.nstrips, g.my, CLAW_STEP2_MIN_ROWS, &args.brows, &args.nblocks);
        grid = (nw + WARPS2D - 1) / WARPS2D;
        args.nwarps = nw;
        return 0;
    }

    cudaError_t launch(cudaStream_t s) override {
        return launch_step(step2_kernel<S, M, SRC>, dim3(grid), dim3(32 * WARPS2D), smem, s, args);
    }
};

}  // namespace clawb200
