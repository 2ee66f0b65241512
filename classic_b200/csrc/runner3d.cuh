// Runner of the 3D step (one launch per sweep: x, y, z; the z-sweep's last
// CTA runs claw3's dt controller, src/3d/claw3.f:738-904), shared by the
// reference-order unit (claw3d.cu, --fmad=false, sweep3p_kernel) and the
// fused / FP32 unit (fast3d.cu, sweep3f_kernel).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>

#include "host.h"
#include "riemann.cuh"
#include "step3d.cuh"
#include "step3d_fast.cuh"
#include "step3ds.cuh"

namespace clawb200 {

template <class S, class M, int BUILD>
struct Runner3D : Runner {
    using real = typename S::real;
    Sweep3Args<real> args[3];
    int grid[3] = {1, 1, 1};
    static constexpr int SMEM = BUILD == 1 ? sweep3f_smem_bytes<real>() : sweep3_smem_bytes<real>();

    int prepare(const claw_config& cfg, const Geometry& g) override {
        Sweep3Args<real> b;
        std::memset(&b, 0, sizeof(b));
        b.q[0] = static_cast<real*>(g.q[0]);
        b.q[1] = static_cast<real*>(g.q[1]);
        b.aux = static_cast<const real*>(g.aux);
        b.qs[0] = 1;
        b.qs[1] = g.ld;
        b.qs[2] = g.ld * g.my;
        b.fstride = g.fstride;
        b.as[0] = 1;
        b.as[1] = g.ald;
        b.as[2] = g.ald * (g.my + 4);
        b.afstride = g.afstride;
        b.m[0] = g.mx;
        b.m[1] = g.my;
        b.m[2] = g.mz;
        for (int d = 0; d < 3; ++d) {
            b.bc[2 * d] = cfg.bc_lower[d];
            b.bc[2 * d + 1] = cfg.bc_upper[d];
        }
        b.mthlim[0] = cfg.limiter[0];
        b.mthlim[1] = cfg.limiter[1];
        b.order = cfg.order;
        b.m3 = cfg.transverse_waves / 10;
        b.m4 = cfg.transverse_waves - 10 * b.m3;
        b.d[0] = g.dx;
        b.d[1] = g.dy;
        b.d[2] = g.dz;
        b.xlower = cfg.lower[0];
        b.ylower = cfg.lower[1];
        b.ctl = g.ctl;
        const int m[3] = {g.mx, g.my, g.mz};
        for (int dir = 0; dir < 3; ++dir) {
            const int axa = dir == 0 ? 1 : 0, axb = dir == 2 ? 1 : 2;
            args[dir] = b;
            args[dir].tilesA = (m[axa] + T3A - 3) / (T3A - 2);
            args[dir].tilesB = (m[axb] + T3B - 3) / (T3B - 2);
            args[dir].nseg = (m[dir] + SEG3 - 1) / SEG3;
            const long long n = (long long)args[dir].tilesA * args[dir].tilesB * args[dir].nseg;
            if (n > 0x7fffffffLL) return fail(CLAW_E_UNSUPPORTED, "3D grid too large");
            grid[dir] = (int)n;
        }
        CUDA_TRY(cudaFuncSetAttribute(kernel<0, false>(), cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
        CUDA_TRY(cudaFuncSetAttribute(kernel<1, false>(), cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
        CUDA_TRY(cudaFuncSetAttribute(kernel<2, true>(), cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
        return 0;
    }

    // the sweep kernel of direction DIR for this unit
    template <int DIR, bool LAST>
    static auto kernel() {
        if constexpr (BUILD == 1) return &sweep3f_kernel<S, DIR, M, LAST>;
        else return &sweep3p_kernel<S, DIR, M, LAST, BUILD>;
    }

    cudaError_t launch(cudaStream_t s) override {
        cudaError_t e = launch_step(kernel<0, false>(), dim3(grid[0]), dim3(NT3P), SMEM, s, args[0]);
        if (e == cudaSuccess) e = launch_step(kernel<1, false>(), dim3(grid[1]), dim3(NT3P), SMEM, s, args[1]);
        if (e == cudaSuccess) e = launch_step(kernel<2, true>(), dim3(grid[2]), dim3(NT3P), SMEM, s, args[2]);
        return e;
    }
    int launches_per_step() const override { return 3; }
};


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
        // P: the four fields after the x-sweep; P2: p and v after the y-sweep
        CUDA_TRY(cudaMalloc(&scratch, (size_t)args.pfstride * 6 * sizeof(real)));
        args.P = scratch;
        args.P2 = scratch + (size_t)args.pfstride * 4;
        for (int d = 0; d < 3; ++d) args.nchunk[d] = (args.m[d] + DS3_CHUNK - 1) / DS3_CHUNK;
        int dev = 0, nsm = 0;
        CUDA_TRY(cudaGetDevice(&dev));
        CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        const long long ux = (long long)args.nstripx * py * pz;
        const long long uy = (long long)args.nstrip32 * pz * args.nchunk[1];
        const long long uz = (long long)args.nstrip32 * py * args.nchunk[2];
        auto ctas = [&](long long units, long long cap) {
            return (int)std::max(1LL, std::min(cap, (units + DS3_WARPS - 1) / DS3_WARPS));
        };
        grid[0] = ctas(ux, (long long)nsm * 8);
        grid[1] = ctas(uy, 1LL << 30);
        grid[2] = ctas(uz, 1LL << 30);
        return 0;
    }

    cudaError_t launch(cudaStream_t s) override {
        cudaError_t e = launch_step(split3_x_kernel<S, BUILD>, dim3(grid[0]), dim3(32 * DS3_WARPS), 0, s, args);
        if (e == cudaSuccess) e = launch_step(split3_yz_kernel<S, 1, BUILD>, dim3(grid[1]), dim3(32 * DS3_WARPS), 0, s, args);
        if (e == cudaSuccess) e = launch_step(split3_yz_kernel<S, 2, BUILD>, dim3(grid[2]), dim3(32 * DS3_WARPS), 0, s, args);
        if (e != cudaSuccess) return e;
        return cudaGetLastError();
    }
    int launches_per_step() const override { return 3; }
};

template <typename real, int BUILD>
std::unique_ptr<Runner> runner3d_for(const claw_config& cfg) {
    using S = VCAcoustics3D<real>;
    if (cfg.order == 2 && cfg.transverse_waves == 22 && cfg.limiter[0] == 4 && cfg.limiter[1] == 4)
        return std::unique_ptr<Runner>(new Runner3D<S, MethodMC3D, BUILD>());
    return std::unique_ptr<Runner>(new Runner3D<S, MethodGeneric3D, BUILD>());
}

}  // namespace clawb200
