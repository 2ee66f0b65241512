// Runner of the characteristic-variable dimensionally split step
// (char2ds.cuh): 2D constant-coefficient acoustics, Godunov or Strang
// splitting, order 2, in the contracted FP64 and the FP32 builds.  Built with
// fused multiply-add contraction.  Other split settings (order 1, capacity,
// f-waves, source terms, other solvers) take the generic split kernel.
#include "char2d_runner.cuh"
#include "char2ds.cuh"

namespace clawb200 {

namespace {

template <typename real, int LIM, int BCM, bool STRANG>
struct CharSplitRunner : Runner {
    CharArgs<real> args;
    int grid = 1, smem = 0;

    int prepare(const claw_config& cfg, const Geometry& g) override {
        using R = CharRing<real>;
        constexpr int STRIPW = STRANG ? STRIP_STRANG : STRIP2;
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
        args.nstrips = (g.mx + STRIPW - 1) / STRIPW;
        args.bc[0] = cfg.bc_lower[0];
        args.bc[1] = cfg.bc_upper[0];
        args.bc[2] = cfg.bc_lower[1];
        args.bc[3] = cfg.bc_upper[1];
        args.lim = cfg.limiter[0];
        args.lim2 = cfg.limiter[1];
        args.dx = g.dx;
        args.dy = g.dy;
        args.ctl = g.ctl;
        for (int k = 0; k < 2; ++k) {
            const int rc = make_map3(&args.tmq[k], g.q[k], g.es, g.mx, g.my, 3, g.ld, g.fstride, R::W, 1, 3);
            if (rc) return rc;
        }
        smem = R::SMEM;
        auto kern = step2s_char_kernel<real, LIM, BCM, STRANG>;
        CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        int dev = 0, nsm = 0, per_sm = 0;
        CUDA_TRY(cudaGetDevice(&dev));
        CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * WARPS2D, smem));
        if (per_sm < 1) return fail(CLAW_E_CUDA, "split characteristic kernel cannot be resident");
        const long long full = (long long)nsm * per_sm * WARPS2D;
        const int nw = row_blocks(full, args.nstrips, g.my, CLAW_CHAR_MIN_ROWS, &args.brows, &args.nblocks);
        grid = (nw + WARPS2D - 1) / WARPS2D;
        args.nwarps = nw;
        return 0;
    }

    cudaError_t launch(cudaStream_t s) override {
        return launch_step(step2s_char_kernel<real, LIM, BCM, STRANG>, dim3(grid), dim3(32 * WARPS2D), smem, s,
                           args);
    }
};

// MC on both waves compiled in; any other limiters read at run time
template <typename real, int BCM, bool STRANG>
std::unique_ptr<Runner> pick_lim(int l1, int l2) {
    if (l1 == 4 && l2 == 4) return std::unique_ptr<Runner>(new CharSplitRunner<real, 4, BCM, STRANG>());
    return std::unique_ptr<Runner>(new CharSplitRunner<real, -1, BCM, STRANG>());
}

template <typename real, bool STRANG>
std::unique_ptr<Runner> pick(const claw_config& cfg) {
    const bool px = cfg.bc_lower[0] == BC_PERIODIC || cfg.bc_upper[0] == BC_PERIODIC;
    bool extrap = true;
    for (int d = 0; d < 2; ++d) extrap = extrap && cfg.bc_lower[d] == BC_EXTRAP && cfg.bc_upper[d] == BC_EXTRAP;
    const int l1 = cfg.limiter[0], l2 = cfg.limiter[1];
    if (px) return pick_lim<real, CHAR_BC_PERX, STRANG>(l1, l2);
    if (extrap) return pick_lim<real, CHAR_BC_EXTRAP, STRANG>(l1, l2);
    return pick_lim<real, CHAR_BC_WALLS, STRANG>(l1, l2);
}

}  // namespace

std::unique_ptr<Runner> make_char_split_runner(const claw_config& cfg) {
    if (cfg.solver_id != CLAW_SOLVER_ACOUSTICS_2D || cfg.num_dim != 2 || cfg.num_waves != 2) return nullptr;
    if (cfg.dimensional_split != 1 && cfg.dimensional_split != 2) return nullptr;
    if (cfg.order != 2 || cfg.capa_index != 0 || cfg.use_fwaves) return nullptr;
    if (cfg.source_id != CLAW_SOURCE_NONE && cfg.source_split != 0) return nullptr;
    const bool strang = cfg.dimensional_split == 2;
    if (cfg.precision == CLAW_FP32) return strang ? pick<float, true>(cfg) : pick<float, false>(cfg);
    if (cfg.precision == CLAW_FP64_FMA) return strang ? pick<double, true>(cfg) : pick<double, false>(cfg);
    return nullptr;
}

}  // namespace clawb200
