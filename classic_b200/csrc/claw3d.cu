// The 3D step in the reference's order of operations (--fmad=false):
// bit-identical to the CPU restatement of step3 / flux3 / claw3, and of
// dimsp3 / step3ds when dimensional splitting is on.
#include <algorithm>

#include "runner3d.cuh"
#include "step3ds.cuh"

namespace clawb200 {
namespace {

// Godunov-split 3D step (src/3d/dimsp3.f): x-, y- and z-sweep launches over a
// scratch array of the grid plus one ghost layer.
template <class S, int BUILD>
struct SplitRunner3D : Runner {
    using real = typename S::real;
    Split3Args<real> args;
    int grid[3] = {1, 1, 1};
    real* scratch = nullptr;

    ~SplitRunner3D() override {
        if (scratch) cudaFree(scratch);
    }

    int prepare(const claw_config& cfg, const Geometry& g) override {
        std::memset(&args, 0, sizeof(args));
        for (int k = 0; k < 2; ++k) {
            args.q[k] = static_cast<const real*>(g.q[k]);
            args.qw[k] = static_cast<real*>(g.q[k]);
        }
        args.aux = static_cast<const real*>(g.aux);
        args.qs[0] = 1;
        args.qs[1] = g.ld;
        args.qs[2] = g.ld * g.my;
        args.fstride = g.fstride;
        const long long px = g.mx + 2, py = g.my + 2, pz = g.mz + 2;
        args.ps[0] = 1;
        args.ps[1] = px;
        args.ps[2] = px * py;
        args.pfstride = px * py * pz;
        args.as[0] = 1;
        args.as[1] = g.ald;
        args.as[2] = g.ald * (g.my + 4);
        args.afstride = g.afstride;
        args.m[0] = g.mx;
        args.m[1] = g.my;
        args.m[2] = g.mz;
        for (int d = 0; d < 3; ++d) {
            args.bc[2 * d] = cfg.bc_lower[d];
            args.bc[2 * d + 1] = cfg.bc_upper[d];
        }
        args.mthlim[0] = cfg.limiter[0];
        args.mthlim[1] = cfg.limiter[1];
        args.order = cfg.order;
        args.d[0] = g.dx;
        args.d[1] = g.dy;
        args.d[2] = g.dz;
        args.xlower = cfg.lower[0];
        args.ylower = cfg.lower[1];
        args.nstripx = (g.mx + DS3_STRIPX - 1) / DS3_STRIPX;
        args.nstrip32 = (int)((px + 31) / 32);
        args.ctl = g.ctl;
        CUDA_TRY(cudaMalloc(&scratch, (size_t)args.pfstride * 4 * sizeof(real)));
        args.P = scratch;
        int dev = 0, nsm = 0;
        CUDA_TRY(cudaGetDevice(&dev));
        CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        const long long ux = (long long)args.nstripx * py * pz;
        const long long uy = (long long)args.nstrip32 * pz;
        const long long uz = (long long)args.nstrip32 * py;
        auto ctas = [&](long long units, long long cap) {
            return (int)std::max(1LL, std::min(cap, (units + DS3_WARPS - 1) / DS3_WARPS));
        };
        grid[0] = ctas(ux, (long long)nsm * 8);
        grid[1] = ctas(uy, 1LL << 30);
        grid[2] = ctas(uz, 1LL << 30);
        return 0;
    }

    cudaError_t launch(cudaStream_t s) override {
        split3_x_kernel<S, BUILD><<<grid[0], 32 * DS3_WARPS, 0, s>>>(args);
        split3_yz_kernel<S, 1, BUILD><<<grid[1], 32 * DS3_WARPS, 0, s>>>(args);
        split3_yz_kernel<S, 2, BUILD><<<grid[2], 32 * DS3_WARPS, 0, s>>>(args);
        return cudaGetLastError();
    }
    int launches_per_step() const override { return 3; }
};

}  // namespace

std::unique_ptr<Runner> make_runner3d(const claw_config& cfg) {
    if (cfg.solver_id != CLAW_SOLVER_VC_ACOUSTICS_3D) return nullptr;
    if (cfg.dimensional_split > 0) {
        // src/3d/claw3ez.f:136: any splitting request runs dimsp3's Godunov splitting
        if (cfg.precision == CLAW_FP32)
            return std::unique_ptr<Runner>(new SplitRunner3D<VCAcoustics3D<float>, 0>());
        return std::unique_ptr<Runner>(new SplitRunner3D<VCAcoustics3D<double>, 0>());
    }
    if (cfg.precision != CLAW_FP64) return make_fast_runner3d(cfg);
    return runner3d_for<double, 0>(cfg);
}

}  // namespace clawb200
