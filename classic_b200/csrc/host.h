// Host-side pieces shared by the translation units of libclawb200.so:
// the geometry of one grid on the device, the kernel-runner interface, error
// reporting for claw_last_error() and TMA descriptor creation.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <memory>
#include <utility>

#include "../../include/claw_b200.h"
#include "common.cuh"

namespace clawb200 {

struct Geometry {
    int dim, mx, my, mz, meqn, maux, es;
    long long ld, fstride, ald, afstride;  // pitches in elements
    void* q[2];
    void* aux;
    void* aux_base;  // the aux claw_set_aux received, when a before-step routine rewrites aux
    ClawCtl* ctl;
    double dx, dy, dz;
};

// One compiled step kernel bound to one grid.
struct Runner {
    virtual ~Runner() {}
    virtual int prepare(const claw_config& cfg, const Geometry& g) = 0;
    virtual cudaError_t launch(cudaStream_t s) = 0;  // one time step
    virtual int launches_per_step() const { return 1; }
};

#ifndef CLAW_STEP2_MIN_ROWS
#define CLAW_STEP2_MIN_ROWS 16  // fewest rows of a work item of the generic and split 2D kernels
#endif

// Row-block-major work items of a 2D column-march kernel: as many row blocks
// as fill `full` resident warps with one item (strip x row block) each, every
// block at least min_rows high.  Returns the warps to launch.
inline int row_blocks(long long full, int nstrips, int my, int min_rows, int* brows, int* nblocks) {
    long long nb = full / nstrips;
    if (nb < 1) nb = 1;
    const long long cap = (my + min_rows - 1) / min_rows;
    if (nb > cap) nb = cap > 0 ? cap : 1;
    *brows = (int)((my + nb - 1) / nb);
    *nblocks = (my + *brows - 1) / *brows;
    const long long items = (long long)nstrips * *nblocks;
    return (int)(items < full ? items : full);
}

// Launch a step kernel; with CLAW_PDL, with programmatic stream serialization
// (the kernel calls grid_dependency_sync before it reads what the previous
// launch wrote).
template <typename... KArgs, typename... Args>
inline cudaError_t launch_step(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                               Args&&... args) {
#if CLAW_PDL
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
#else
    kernel<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
    return cudaGetLastError();
#endif
}

// Record an error message (claw_last_error) and return code.
int fail(int code, const char* fmt, ...);
void set_last_error(const char* msg);

// 3D tiled TMA map over an SoA array: dims (n0, n1, n2), pitches p1, p2 in
// elements, element size es (4 or 8), box (box0, box1, box2).
int make_map3(CUtensorMap* map, void* base, int es, long long n0, long long n1, long long n2,
              long long p1, long long p2, int box0, int box1, int box2);

// Characteristic-variable kernel for constant-coefficient 2D acoustics
// (char2d.cuh, built with fused multiply-add); nullptr if cfg is not served.
std::unique_ptr<Runner> make_char_runner(const claw_config& cfg);

// 2D unsplit step of the contracted build for the methods and solvers the
// characteristic kernel does not serve (fma2d.cu); nullptr if cfg is not served.
std::unique_ptr<Runner> make_fast_runner2d(const claw_config& cfg);

// 2D dimensionally split step (step2ds.cuh, one fused launch per step);
// nullptr if cfg is not served.
std::unique_ptr<Runner> make_split_runner(const claw_config& cfg);
// its fused-multiply-add / FP32 build (split2d_fast.cu)
std::unique_ptr<Runner> make_fast_split_runner(const claw_config& cfg);
// characteristic-variable split step for 2D constant-coefficient acoustics
// (split2d_char.cu), or nullptr
std::unique_ptr<Runner> make_char_split_runner(const claw_config& cfg);

// 3D step (step3d.cuh: one launch per sweep); nullptr if cfg is not served.
std::unique_ptr<Runner> make_runner3d(const claw_config& cfg);
// its fused-multiply-add / FP32 builds (fast3d.cu)
std::unique_ptr<Runner> make_fast_runner3d(const claw_config& cfg);

}  // namespace clawb200

#define CUDA_TRY(x)                                                                      \
    do {                                                                                 \
        cudaError_t e_ = (x);                                                            \
        if (e_ != cudaSuccess)                                                           \
            return ::clawb200::fail(CLAW_E_CUDA, "%s failed: %s", #x, cudaGetErrorString(e_)); \
    } while (0)
