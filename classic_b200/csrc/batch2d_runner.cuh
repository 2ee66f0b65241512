// The batched 2D step kernel (step2_batch_kernel in step2d.cuh) bound to the
// instances of one batch: per-instance arguments and TMA maps on the device,
// the launch shape and the launch.  Shared by the reference-order build
// (batch2d.cu) and the contracted build (batch2d_fast.cu), which instantiate
// it for distinct method policies so that their kernels stay distinct symbols.
#pragma once
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "host.h"
#include "step2d.cuh"

namespace clawb200 {

struct BatchRunner {
    virtual ~BatchRunner() {}
    virtual int prepare(const std::vector<Geometry>& g, const claw_config* cfgs, ClawCtl* ctls,
                        int* active, int* err) = 0;
    virtual cudaError_t launch(cudaStream_t s) = 0;
    // launch shape: tile height (rows per warp at least) and CTAs per SM
    virtual void set_shape(int min_rows, int ctas_per_sm) = 0;
    virtual int max_ctas_per_sm() const = 0;
    int min_rows = 48, ctas_per_sm = 0;
};

template <class S, class M>
struct BatchRunnerT : BatchRunner {
    S solver;
    Step2Batch<S> b;
    Step2Args<S>* inst_d = nullptr;
    int* units_d = nullptr;
    int grid = 1, smem = 0;

    explicit BatchRunnerT(const S& s) : solver(s) { std::memset(&b, 0, sizeof(b)); }
    ~BatchRunnerT() override {
        if (inst_d) cudaFree(inst_d);
        if (units_d) cudaFree(units_d);
    }

    int prepare(const std::vector<Geometry>& g, const claw_config* cfgs, ClawCtl* ctls, int* active,
                int* err) override {
        using R = Ring2D<S>;
        const int n = (int)g.size();
        std::vector<Step2Args<S>> inst(n);
        std::vector<int> units(n);
        for (int k = 0; k < n; ++k) {
            Step2Args<S>& a = inst[k];
            std::memset(&a, 0, sizeof(a));
            a.solver = solver;
            a.q[0] = static_cast<typename S::real*>(g[k].q[0]);
            a.q[1] = static_cast<typename S::real*>(g[k].q[1]);
            a.aux = static_cast<const typename S::real*>(g[k].aux);
            a.ld = g[k].ld;
            a.fstride = g[k].fstride;
            a.ald = g[k].ald;
            a.afstride = g[k].afstride;
            a.mx = g[k].mx;
            a.my = g[k].my;
            a.nstrips = (g[k].mx + STRIP - 1) / STRIP;
            const claw_config& cfg = cfgs[k];
            a.bc[0] = cfg.bc_lower[0];
            a.bc[1] = cfg.bc_upper[0];
            a.bc[2] = cfg.bc_lower[1];
            a.bc[3] = cfg.bc_upper[1];
            for (int w = 0; w < 8; ++w) a.mthlim[w] = w < cfg.num_waves ? cfg.limiter[w] : 0;
            a.order = cfg.order;
            a.trans = cfg.transverse_waves;
            a.fwave = cfg.use_fwaves;
            a.capa = cfg.capa_index;
            a.dx = g[k].dx;
            a.dy = g[k].dy;
            a.ctl = ctls + k;
            for (int c = 0; c < 2; ++c) {
                const int rc = make_map3(&a.tmq[c], g[k].q[c], g[k].es, g[k].mx, g[k].my, S::meqn,
                                         g[k].ld, g[k].fstride, R::W, 1, S::meqn);
                if (rc) return rc;
            }
            if (S::maux > 0) {
                const int rc = make_map3(&a.tmaux, g[k].aux, g[k].es, g[k].mx + 4, g[k].my + 4,
                                         S::maux, g[k].ald, g[k].afstride, R::W, 1, S::maux);
                if (rc) return rc;
            }
            const long long u = (long long)a.nstrips * a.my;
            if (u > 0x7fffffffLL) return fail(CLAW_E_UNSUPPORTED, "instance %d too large", k);
            units[k] = (int)u;
        }
        CUDA_TRY(cudaMalloc(&inst_d, sizeof(Step2Args<S>) * n));
        CUDA_TRY(cudaMemcpy(inst_d, inst.data(), sizeof(Step2Args<S>) * n, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMalloc(&units_d, sizeof(int) * n));
        CUDA_TRY(cudaMemcpy(units_d, units.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
        smem = R::SMEM;
        CUDA_TRY(cudaFuncSetAttribute(step2_batch_kernel<S, M>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        int dev = 0, nsm = 0, per_sm = 0;
        CUDA_TRY(cudaGetDevice(&dev));
        CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step2_batch_kernel<S, M>,
                                                               32 * WARPS2D, smem));
        if (per_sm < 1) return fail(CLAW_E_CUDA, "batch kernel cannot be resident on an SM");
        nsm_ = nsm;
        per_sm_ = per_sm;
        b.inst = inst_d;
        b.ctls = ctls;
        b.units = units_d;
        b.count = n;
        b.active = active;
        b.err = err;
        set_shape(48, per_sm);
        return 0;
    }

    void set_shape(int rows, int ctas) override {
        min_rows = std::max(1, rows);
        ctas_per_sm = std::max(1, std::min(ctas, per_sm_));
        grid = nsm_ * ctas_per_sm;
        b.nwarps = grid * WARPS2D;
        b.min_rows = min_rows;
    }
    int max_ctas_per_sm() const override { return per_sm_; }
    int nsm_ = 1, per_sm_ = 1;

    cudaError_t launch(cudaStream_t s) override {
        return launch_step(step2_batch_kernel<S, M>, dim3(grid), dim3(32 * WARPS2D), smem, s, b);
    }
};

// Contracted build of the batch (CLAW_FP64_FMA; batch2d_fast.cu); nullptr if
// cfg is not served.
std::unique_ptr<BatchRunner> make_fast_batch_runner(const claw_config& cfg);

}  // namespace clawb200
