// Host side of the C ABI declared in include/claw_b200.h: device memory,
// TMA descriptors, launch configuration, the CUDA-graph time loop and the
// claw2-style argument checks.  Kernels live in step*d.cuh.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>

#include "../../include/claw_b200.h"
#include "common.cuh"
#include "host.h"
#include "riemann.cuh"
#include "step1d.cuh"
#include "step2d.cuh"
#include "runner2d.cuh"

using namespace clawb200;

namespace clawb200 {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

void set_last_error(const char* msg) { g_err = msg; }

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult qr;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &qr) ==
                cudaSuccess &&
            qr == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

int make_map3(CUtensorMap* map, void* base, int es, long long n0, long long n1, long long n2,
              long long p1, long long p2, int box0, int box1, int box2) {
    auto fn = encode_fn();
    if (!fn) return fail(CLAW_E_CUDA, "cuTensorMapEncodeTiled is unavailable");
    const cuuint64_t dims[3] = {(cuuint64_t)n0, (cuuint64_t)n1, (cuuint64_t)n2};
    const cuuint64_t strides[2] = {(cuuint64_t)(p1 * es), (cuuint64_t)(p2 * es)};
    const cuuint32_t box[3] = {(cuuint32_t)box0, (cuuint32_t)box1, (cuuint32_t)box2};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = fn(map, es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                          3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(CLAW_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return 0;
}

}  // namespace clawb200

namespace {

long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

// ------------------------------------------------------------------ runners ---
template <class S>
struct Runner1D : Runner {
    Step1Args<S> args;
    int smem = 0;
    typename S::real* iface = nullptr;

    explicit Runner1D(const S& s) { std::memset(&args, 0, sizeof(args)); args.solver = s; }
    ~Runner1D() override {
        if (iface) cudaFree(iface);
    }

    int prepare(const claw_config& cfg, const Geometry& g) override {
        args.q[0] = static_cast<typename S::real*>(g.q[0]);
        args.q[1] = static_cast<typename S::real*>(g.q[1]);
        args.aux = static_cast<const typename S::real*>(g.aux);
        args.fstride = g.fstride;
        args.afstride = g.afstride;
        args.mx = g.mx;
        args.bc[0] = cfg.bc_lower[0];
        args.bc[1] = cfg.bc_upper[0];
        for (int k = 0; k < 8; ++k) args.mthlim[k] = k < cfg.num_waves ? cfg.limiter[k] : 0;
        args.order = cfg.order;
        args.fwave = cfg.use_fwaves;
        args.capa = cfg.capa_index;
        args.dx = g.dx;
        args.ctl = g.ctl;
        args.src_split = cfg.source_id == CLAW_SOURCE_RADIAL ? cfg.source_split : 0;
        args.src_nd1 = (double)(cfg.source_ndim - 1);
        args.src_bulk = cfg.solver_params[1];
        args.xlower = cfg.lower[0];
        int dev = 0, optin = 0;
        CUDA_TRY(cudaGetDevice(&dev));
        CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        long long bytes = step1_smem_bytes<S>(g.mx, true);
        if (bytes + 1024 > optin) {
            // the interface arrays move to an L2-resident global buffer
            bytes = step1_smem_bytes<S>(g.mx, false);
            if (bytes + 1024 > optin)
                return fail(CLAW_E_UNSUPPORTED, "1D grid of %d cells exceeds the single-CTA kernel", g.mx);
            CUDA_TRY(cudaMalloc(&iface, (size_t)step1_iface_doubles<S>(g.mx) * sizeof(typename S::real)));
        }
        args.iface = iface;
        smem = (int)bytes;
        CUDA_TRY(cudaFuncSetAttribute(step1_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem));
        return 0;
    }

    cudaError_t launch(cudaStream_t s) override {
        step1_kernel<S><<<1, STEP1_THREADS, smem, s>>>(args);
        return cudaGetLastError();
    }
};

// True when every wave uses the same limiter `lim`.
bool all_limiters(const claw_config& cfg, int lim) {
    for (int k = 0; k < cfg.num_waves; ++k)
        if (cfg.limiter[k] != lim) return false;
    return true;
}

// The hot method (order 2, transverse 2, MC on every wave, no capacity, no
// f-waves) runs a fully specialised kernel; every other method the generic one.
template <class S>
std::unique_ptr<Runner> runner2d(const claw_config& cfg, const S& s) {
    if constexpr (std::is_same<S, Acoustics2D<typename S::real>>::value) {
        // the radial source (src/2d/claw2.f:635-738 with 1drad/src1.f) fused into the step
        if (cfg.source_id == CLAW_SOURCE_RADIAL && cfg.source_split != 0)
            return std::unique_ptr<Runner>(new Runner2D<S, MethodGeneric2D, true>(s));
    }
    if (cfg.order == 2 && cfg.transverse_waves == 2 && all_limiters(cfg, 4) &&
        cfg.capa_index == 0 && !cfg.use_fwaves)
        return std::unique_ptr<Runner>(new Runner2D<S, MethodMC2D>(s));
    return std::unique_ptr<Runner>(new Runner2D<S, MethodGeneric2D>(s));
}

template <typename real>
std::unique_ptr<Runner> make_runner(const claw_config& cfg) {
    const int id = cfg.solver_id;
    if (cfg.num_dim == 3) return make_runner3d(cfg);
    if (cfg.dimensional_split > 0) return make_split_runner(cfg);
    const bool source = cfg.source_id != CLAW_SOURCE_NONE && cfg.source_split != 0;
    if (cfg.precision != CLAW_FP64 && !source) {
        // fused / FP32 arithmetic: constant-coefficient acoustics runs in
        // characteristic variables when the method allows it
        auto r = make_char_runner(cfg);
        if (r) return r;
        r = make_fast_runner2d(cfg);
        if (r) return r;
    }
    if (id == CLAW_SOLVER_ACOUSTICS_2D || id == CLAW_SOLVER_ACOUSTICS_1D) {
        const double rho = cfg.solver_params[0], bulk = cfg.solver_params[1];
        const double cc = std::sqrt(bulk / rho), zz = rho * cc, hz = 0.5 / zz;
        if (id == CLAW_SOLVER_ACOUSTICS_2D) {
            Acoustics2D<real> s{(real)cc, (real)zz, (real)hz};
            return runner2d(cfg, s);
        }
        Acoustics1D<real> s{(real)cc, (real)zz, (real)hz};
        return std::unique_ptr<Runner>(new Runner1D<Acoustics1D<real>>(s));
    }
    if (id == CLAW_SOLVER_EULER_ROE_2D) {
        const double gamma = cfg.solver_params[0];
        EulerRoe2D<real> s{(real)gamma, (real)(gamma - 1.0)};
        return runner2d(cfg, s);
    }
    if (id == CLAW_SOLVER_VC_ADVECTION_2D)
        return std::unique_ptr<Runner>(new Runner2D<VCAdvection2D<real>, MethodGeneric2D>(VCAdvection2D<real>{}));
    if (id == CLAW_SOLVER_VC_ACOUSTICS_1D)
        return std::unique_ptr<Runner>(new Runner1D<VCAcoustics1D<real>>(VCAcoustics1D<real>{}));
    if (id == CLAW_SOLVER_ADVECTION_1D)
        return std::unique_ptr<Runner>(
            new Runner1D<Advection1D<real>>(Advection1D<real>{(real)cfg.solver_params[0]}));
    if (id == CLAW_SOLVER_EULER_ROE_1D) {
        const double gamma = cfg.solver_params[0];
        return std::unique_ptr<Runner>(
            new Runner1D<EulerRoe1D<real>>(EulerRoe1D<real>{(real)gamma, (real)(gamma - 1.0)}));
    }
    return nullptr;
}

// ------------------------------------------------------- before-step hook ---
// b4step2 (src/2d/claw2.f:626-631) as a device routine launched ahead of each
// step kernel: CLAW_B4STEP_REVERSING writes the edge velocities (aux fields 1,
// 2) = the unscaled ones times cos(pi t / T) at the step's start time t, read
// from the control block, so the device-resident time loop needs no host
// round trip per step.
template <typename real>
__global__ void b4step_reversing_kernel(const ClawCtl* ctl, const real* __restrict__ base,
                                        real* __restrict__ aux, long long n, double period) {
    if (*(const volatile int*)&ctl->done) return;
    const double told = *(const volatile double*)&ctl->told;
    const double sc = cos(3.141592653589793 * told / period);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        aux[i] = (real)((double)base[i] * sc);
}

template <typename real>
struct B4StepRunner : Runner {
    std::unique_ptr<Runner> inner;
    const ClawCtl* ctl = nullptr;
    const real* base = nullptr;
    real* aux = nullptr;
    long long n = 0;
    double period = 1.0;
    int grid = 1;

    explicit B4StepRunner(std::unique_ptr<Runner> r) : inner(std::move(r)) {}

    int prepare(const claw_config& cfg, const Geometry& g) override {
        int rc = inner->prepare(cfg, g);
        if (rc) return rc;
        ctl = g.ctl;
        base = static_cast<const real*>(g.aux_base);
        aux = static_cast<real*>(g.aux);
        n = 2 * g.afstride;  // fields 1 and 2 are contiguous
        period = cfg.b4step_param;
        int dev = 0, nsm = 0;
        CUDA_TRY(cudaGetDevice(&dev));
        CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        grid = (int)std::min<long long>((n + 255) / 256, (long long)nsm * 8);
        return 0;
    }
    cudaError_t launch(cudaStream_t s) override {
        b4step_reversing_kernel<real><<<grid, 256, 0, s>>>(ctl, base, aux, n, period);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        return inner->launch(s);
    }
    int launches_per_step() const override { return inner->launches_per_step() + 1; }
};

// --------------------------------------------------------- conserved totals ---
// Sum over interior cells of capa * q_m (capa = 1 without a capacity
// function) in FP64 with Neumaier's compensated summation, whatever the
// storage precision.  Each block forms (sum, compensation) pairs over a fixed
// range of cells; one final block adds the block pairs in order, so the result
// does not depend on scheduling.
constexpr int TOT_THREADS = 256, TOT_BLOCKS_MAX = 1184;

__device__ __forceinline__ void neumaier_add(double& s, double& c, double x) {
    const double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
}

template <typename real>
__global__ void totals_partial_kernel(const real* __restrict__ q, const real* __restrict__ aux,
                                      int capa, long long ld, long long fstride, long long ald,
                                      long long afstride, int mx, int my, int mz, int dim,
                                      int meqn, double* __restrict__ part) {
    __shared__ double sh[2][TOT_THREADS / 32];
    const long long rows = (long long)my * mz;
    const long long ncell = rows * mx;
    const long long per = (ncell + gridDim.x - 1) / gridDim.x;
    const long long c0 = blockIdx.x * per, c1 = min(ncell, c0 + per);
    for (int m = 0; m < meqn; ++m) {
        double s = 0.0, c = 0.0;
        for (long long k = c0 + threadIdx.x; k < c1; k += blockDim.x) {
            const long long row = k / mx, i = k - row * mx;
            double v = (double)q[m * fstride + row * ld + i];
            if (capa > 0) {
                // aux has two ghost layers per axis: cell (i, j, l) at (i+2, j+2, l+2)
                const long long j = dim >= 2 ? row % my : 0, l = dim >= 3 ? row / my : 0;
                const long long ao = (capa - 1) * afstride + (i + 2) +
                                     (dim >= 2 ? (j + 2) * ald : 0) +
                                     (dim >= 3 ? (l + 2) * ald * (my + 4) : 0);
                v = (double)aux[ao] * v;
            }
            neumaier_add(s, c, v);
        }
        // fold the lanes' pairs (sum part exact by TwoSum, errors added)
        for (int off = 16; off > 0; off >>= 1) {
            const double s2 = __shfl_down_sync(0xffffffffu, s, off);
            const double c2 = __shfl_down_sync(0xffffffffu, c, off);
            const double t = s + s2;
            const double bp = t - s;
            const double e = (s - (t - bp)) + (s2 - bp);
            s = t;
            c = c + c2 + e;
        }
        const int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) { sh[0][w] = s; sh[1][w] = c; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double S = 0.0, C = 0.0;
            for (int k = 0; k < TOT_THREADS / 32; ++k) {
                neumaier_add(S, C, sh[0][k]);
                C += sh[1][k];
            }
            part[(blockIdx.x * meqn + m) * 2] = S;
            part[(blockIdx.x * meqn + m) * 2 + 1] = C;
        }
        __syncthreads();
    }
}

__global__ void totals_final_kernel(const double* __restrict__ part, int nblocks, int meqn,
                                    double* __restrict__ out) {
    const int m = threadIdx.x;
    if (m >= meqn) return;
    double S = 0.0, C = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        neumaier_add(S, C, part[(b * meqn + m) * 2]);
        C += part[(b * meqn + m) * 2 + 1];
    }
    out[m] = S + C;
}

struct SolverShape { int dim, meqn, mwaves, maux; };

bool solver_shape(int id, SolverShape* sh) {
    switch (id) {
        case CLAW_SOLVER_ACOUSTICS_2D: *sh = {2, 3, 2, 0}; return true;
        case CLAW_SOLVER_VC_ADVECTION_2D: *sh = {2, 1, 1, 3}; return true;
        case CLAW_SOLVER_EULER_ROE_2D: *sh = {2, 4, 3, 0}; return true;
        case CLAW_SOLVER_ACOUSTICS_1D: *sh = {1, 2, 2, 0}; return true;
        case CLAW_SOLVER_VC_ACOUSTICS_1D: *sh = {1, 2, 2, 2}; return true;
        case CLAW_SOLVER_ADVECTION_1D: *sh = {1, 1, 1, 0}; return true;
        case CLAW_SOLVER_EULER_ROE_1D: *sh = {1, 3, 3, 0}; return true;
        case CLAW_SOLVER_VC_ACOUSTICS_3D: *sh = {3, 4, 2, 2}; return true;
        default: return false;
    }
}

__global__ void widen_to_double(const float* src, double* dst, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}
__global__ void narrow_to_float(const double* src, float* dst, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}

}  // namespace

struct claw_handle {
    claw_config cfg;
    Geometry g;
    int cur = 0;
    cudaStream_t stream = nullptr;
    ClawCtl* ctl_h = nullptr;  // pinned mirror
    double* stage = nullptr;   // device staging (doubles) for FP32 conversion
    std::unique_ptr<Runner> runner;
    cudaGraphExec_t gexec = nullptr;
    int gsteps = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    long long launches = 0;
    int device = 0;
    double t_now = 0.0;  // time of the current q (time-dependent boundary conditions)
    double* totals_scratch = nullptr;  // block partials + result of claw_totals
    unsigned long long wait_ns = 0;    // device wait limit (0: the 2 s default)
    int skip_row = 0;                  // test hook: 1 + row whose copy is skipped

    // Frees everything the handle holds, so an error part-way through
    // claw_create (the handle lives in a unique_ptr there) leaks nothing.
    ~claw_handle() {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        if (gexec) cudaGraphExecDestroy(gexec);
        runner.reset();
        for (int k = 0; k < 2; ++k)
            if (g.q[k]) cudaFree(g.q[k]);
        if (g.aux) cudaFree(g.aux);
        if (g.aux_base) cudaFree(g.aux_base);
        if (totals_scratch) cudaFree(totals_scratch);
        if (g.ctl) cudaFree(g.ctl);
        if (stage) cudaFree(stage);
        if (ctl_h) cudaFreeHost(ctl_h);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

extern "C" {

const char* claw_last_error(void) { return g_err.c_str(); }

const char* claw_build_info(void) {
    return "clawb200 sm_100a; fp64 path built with --fmad=false (reference operation order)";
}

static int validate(const claw_config* c, SolverShape* sh) {
    if (!c) return fail(CLAW_E_INVALID, "null config");
    if (!solver_shape(c->solver_id, sh)) return fail(CLAW_E_UNSUPPORTED, "solver %d is not built", c->solver_id);
    if (c->num_dim != sh->dim) return fail(CLAW_E_INVALID, "num_dim %d does not match solver", c->num_dim);
    if (c->num_eqn != sh->meqn || c->num_waves != sh->mwaves || c->num_aux != sh->maux)
        return fail(CLAW_E_INVALID, "num_eqn/num_waves/num_aux (%d,%d,%d) do not match solver (%d,%d,%d)",
                    c->num_eqn, c->num_waves, c->num_aux, sh->meqn, sh->mwaves, sh->maux);
    if (c->num_ghost != 2) return fail(CLAW_E_INVALID, "num_ghost must be 2");
    for (int d = 0; d < c->num_dim; ++d) {
        if (c->num_cells[d] < 2) return fail(CLAW_E_INVALID, "num_cells[%d] must be >= 2", d);
        if (!(c->upper[d] > c->lower[d])) return fail(CLAW_E_INVALID, "upper[%d] <= lower[%d]", d, d);
        for (int side = 0; side < 2; ++side) {
            const int b = side ? c->bc_upper[d] : c->bc_lower[d];
            if (b == CLAW_BC_PISTON && d == 2 && side == 1 && c->solver_id == CLAW_SOLVER_VC_ACOUSTICS_3D)
                continue;
            if (b == 0 || b == CLAW_BC_PISTON)
                return fail(CLAW_E_UNSUPPORTED, "user boundary conditions are not built");
            if (b < 1 || b > 3) return fail(CLAW_E_INVALID, "bad boundary condition %d", b);
            if (b == 3 && c->num_eqn < d + 2)
                return fail(CLAW_E_INVALID, "wall BC needs a velocity component %d", d + 2);
        }
        if ((c->bc_lower[d] == 2) != (c->bc_upper[d] == 2))
            return fail(CLAW_E_INVALID, "periodic BCs must be set on both sides");
    }
    if (c->order < 1 || c->order > 2) return fail(CLAW_E_INVALID, "order must be 1 or 2");
    if (c->dimensional_split < 0 || c->dimensional_split > 2)
        return fail(CLAW_E_INVALID, "dimensional_split must be 0 (unsplit), 1 (Godunov) or 2 (Strang)");
    if (c->dimensional_split != 0 && c->num_dim == 1)
        return fail(CLAW_E_INVALID, "dimensional splitting needs 2 or 3 dimensions");
    if (c->source_split < 0 || c->source_split > 2)
        return fail(CLAW_E_INVALID, "source_split must be 0, 1 (Godunov) or 2 (Strang)");
    if (c->b4step_id != CLAW_B4STEP_NONE) {
        if (c->b4step_id != CLAW_B4STEP_REVERSING) return fail(CLAW_E_INVALID, "unknown b4step_id %d", c->b4step_id);
        if (c->solver_id != CLAW_SOLVER_VC_ADVECTION_2D)
            return fail(CLAW_E_UNSUPPORTED, "the reversing flow is built for the variable-velocity advection solver");
        if (!(c->b4step_param > 0.0)) return fail(CLAW_E_INVALID, "b4step_param (the period) must be > 0");
    }
    if (c->source_id != CLAW_SOURCE_NONE) {
        if (c->source_id != CLAW_SOURCE_RADIAL) return fail(CLAW_E_INVALID, "unknown source_id %d", c->source_id);
        if (c->solver_id != CLAW_SOLVER_ACOUSTICS_1D && c->solver_id != CLAW_SOLVER_ACOUSTICS_2D)
            return fail(CLAW_E_UNSUPPORTED, "the radial source is built for constant-coefficient acoustics");
        if (c->source_ndim < 1 || c->source_ndim > 3) return fail(CLAW_E_INVALID, "source_ndim must be 1..3");
        if (c->lower[0] < 0.0) return fail(CLAW_E_INVALID, "the radial source needs xlower >= 0 (x is the radius)");
    }
    if (c->capa_index < 0) return fail(CLAW_E_INVALID, "capa_index < 0");
    for (int k = 0; k < c->num_waves; ++k)
        if (c->limiter[k] < 0 || c->limiter[k] > 5) return fail(CLAW_E_INVALID, "invalid limiter %d", c->limiter[k]);
    if (c->precision < CLAW_FP64 || c->precision > CLAW_FP32) return fail(CLAW_E_INVALID, "bad precision");
    if (c->num_dim == 3) {
        if (c->capa_index != 0) return fail(CLAW_E_UNSUPPORTED, "3D capacity is not built");
        if (c->use_fwaves) return fail(CLAW_E_UNSUPPORTED, "3D f-waves are not built");
    }
    return 0;
}

int claw_create(const claw_config* cfg, claw_handle** out) {
    if (!out) return fail(CLAW_E_INVALID, "null out");
    *out = nullptr;
    SolverShape sh;
    int rc = validate(cfg, &sh);
    if (rc) return rc;
    std::unique_ptr<claw_handle> h(new claw_handle());
    h->cfg = *cfg;
    Geometry& g = h->g;
    std::memset(&g, 0, sizeof(g));
    g.dim = cfg->num_dim;
    g.mx = cfg->num_cells[0];
    g.my = g.dim >= 2 ? cfg->num_cells[1] : 1;
    g.mz = g.dim >= 3 ? cfg->num_cells[2] : 1;
    g.meqn = cfg->num_eqn;
    g.maux = cfg->num_aux;
    g.es = cfg->precision == CLAW_FP32 ? 4 : 8;
    // dx = (xupper - xlower)/float(mx), src/2d/claw2ez.f:191-192
    g.dx = (cfg->upper[0] - cfg->lower[0]) / (double)(float)g.mx;
    g.dy = g.dim >= 2 ? (cfg->upper[1] - cfg->lower[1]) / (double)(float)g.my : 1.0;
    g.dz = g.dim >= 3 ? (cfg->upper[2] - cfg->lower[2]) / (double)(float)g.mz : 1.0;
    g.ld = g.dim == 1 ? g.mx : round_up(g.mx, 32);
    g.fstride = g.ld * g.my * g.mz;
    const int ax = g.mx + 4;
    g.ald = g.dim == 1 ? ax : round_up(ax, 4);
    g.afstride = g.ald * (g.dim >= 2 ? g.my + 4 : 1) * (g.dim >= 3 ? g.mz + 4 : 1);
    CUDA_TRY(cudaGetDevice(&h->device));
    CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreate(&h->ev0));
    CUDA_TRY(cudaEventCreate(&h->ev1));
    const size_t qbytes = (size_t)g.fstride * g.meqn * g.es;
    for (int k = 0; k < 2; ++k) {
        CUDA_TRY(cudaMalloc(&g.q[k], qbytes));
        CUDA_TRY(cudaMemsetAsync(g.q[k], 0, qbytes, h->stream));
    }
    if (g.maux > 0) {
        const size_t abytes = (size_t)g.afstride * g.maux * g.es;
        CUDA_TRY(cudaMalloc(&g.aux, abytes));
        CUDA_TRY(cudaMemsetAsync(g.aux, 0, abytes, h->stream));
    }
    CUDA_TRY(cudaMalloc(&g.ctl, sizeof(ClawCtl)));
    CUDA_TRY(cudaMallocHost(&h->ctl_h, sizeof(ClawCtl)));
    std::memset(h->ctl_h, 0, sizeof(ClawCtl));
    h->ctl_h->done = 1;
    CUDA_TRY(cudaMemcpyAsync(g.ctl, h->ctl_h, sizeof(ClawCtl), cudaMemcpyHostToDevice, h->stream));
    if (g.es == 4) {
        const size_t n = std::max((size_t)g.fstride * g.meqn, (size_t)g.afstride * g.maux);
        CUDA_TRY(cudaMalloc(&h->stage, n * sizeof(double)));
    }
    h->runner = g.es == 8 ? make_runner<double>(*cfg) : make_runner<float>(*cfg);
    if (!h->runner) return fail(CLAW_E_UNSUPPORTED, "no kernel for solver %d", cfg->solver_id);
    if (cfg->b4step_id == CLAW_B4STEP_REVERSING) {
        CUDA_TRY(cudaMalloc(&g.aux_base, (size_t)g.afstride * g.maux * g.es));
        CUDA_TRY(cudaMemsetAsync(g.aux_base, 0, (size_t)g.afstride * g.maux * g.es, h->stream));
        if (g.es == 8) h->runner.reset(new B4StepRunner<double>(std::move(h->runner)));
        else h->runner.reset(new B4StepRunner<float>(std::move(h->runner)));
    }
    rc = h->runner->prepare(*cfg, g);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    *out = h.release();
    return 0;
}

int claw_destroy(claw_handle* h) {
    delete h;  // ~claw_handle frees the device state
    return 0;
}

// Copy a dense host field block [nfields][rows][width] to a pitched device array.
static int copy_fields(claw_handle* h, void* dev, long long pitch_el, long long fpitch_el,
                       const double* host, int nfields, long long width, long long rows,
                       bool to_device) {
    const Geometry& g = h->g;
    if (g.es == 8) {
        for (int m = 0; m < nfields; ++m) {
            char* d = static_cast<char*>(dev) + (size_t)m * fpitch_el * 8;
            const double* hp = host + (size_t)m * width * rows;
            if (to_device)
                CUDA_TRY(cudaMemcpy2DAsync(d, pitch_el * 8, hp, width * 8, width * 8, rows,
                                           cudaMemcpyHostToDevice, h->stream));
            else
                CUDA_TRY(cudaMemcpy2DAsync(const_cast<double*>(hp), width * 8, d, pitch_el * 8,
                                           width * 8, rows, cudaMemcpyDeviceToHost, h->stream));
        }
    } else {
        // FP32 storage: stage as doubles on the device, convert there.
        const long long n = (long long)nfields * fpitch_el;
        for (int m = 0; m < nfields; ++m) {
            double* sd = h->stage + (size_t)m * fpitch_el;
            const double* hp = host + (size_t)m * width * rows;
            if (to_device)
                CUDA_TRY(cudaMemcpy2DAsync(sd, pitch_el * 8, hp, width * 8, width * 8, rows,
                                           cudaMemcpyHostToDevice, h->stream));
        }
        if (to_device) {
            narrow_to_float<<<592, 256, 0, h->stream>>>(h->stage, static_cast<float*>(dev), n);
        } else {
            widen_to_double<<<592, 256, 0, h->stream>>>(static_cast<const float*>(dev), h->stage, n);
            for (int m = 0; m < nfields; ++m) {
                const double* sd = h->stage + (size_t)m * fpitch_el;
                double* hp = const_cast<double*>(host) + (size_t)m * width * rows;
                CUDA_TRY(cudaMemcpy2DAsync(hp, width * 8, sd, pitch_el * 8, width * 8, rows,
                                           cudaMemcpyDeviceToHost, h->stream));
            }
        }
        CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

int claw_set_q(claw_handle* h, const double* q) {
    if (!h || !q) return fail(CLAW_E_INVALID, "null argument");
    CUDA_TRY(cudaSetDevice(h->device));
    const Geometry& g = h->g;
    int rc = copy_fields(h, g.q[h->cur], g.ld, g.fstride, q, g.meqn, g.mx, (long long)g.my * g.mz, true);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

int claw_get_q(claw_handle* h, double* q) {
    if (!h || !q) return fail(CLAW_E_INVALID, "null argument");
    CUDA_TRY(cudaSetDevice(h->device));
    const Geometry& g = h->g;
    int rc = copy_fields(h, g.q[h->cur], g.ld, g.fstride, q, g.meqn, g.mx, (long long)g.my * g.mz, false);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

int claw_set_aux(claw_handle* h, const double* aux) {
    if (!h || !aux) return fail(CLAW_E_INVALID, "null argument");
    const Geometry& g = h->g;
    if (g.maux == 0) return 0;
    CUDA_TRY(cudaSetDevice(h->device));
    const long long rows = (long long)(g.dim >= 2 ? g.my + 4 : 1) * (g.dim >= 3 ? g.mz + 4 : 1);
    int rc = copy_fields(h, g.aux, g.ald, g.afstride, aux, g.maux, g.mx + 4, rows, true);
    if (rc) return rc;
    if (g.aux_base)  // the before-step routine scales from this copy
        CUDA_TRY(cudaMemcpyAsync(g.aux_base, g.aux, (size_t)g.afstride * g.maux * g.es,
                                 cudaMemcpyDeviceToDevice, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (h->cfg.capa_index > 0) {
        // the reference stops on a non-positive capacity (src/1d/step1.f90:67-70)
        const long long n = (long long)g.mx + 4;
        const double* cap = aux + (size_t)(h->cfg.capa_index - 1) * n * rows;
        for (long long i = 0; i < n * rows; ++i)
            if (!(cap[i] > 0.0)) return fail(CLAW_E_INVALID, "capacity must be positive");
    }
    return 0;
}

static int push_ctl(claw_handle* h) {
    CUDA_TRY(cudaMemcpyAsync(h->g.ctl, h->ctl_h, sizeof(ClawCtl), cudaMemcpyHostToDevice, h->stream));
    return 0;
}
static int pull_ctl(claw_handle* h) {
    CUDA_TRY(cudaMemcpyAsync(h->ctl_h, h->g.ctl, sizeof(ClawCtl), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

int claw_step(claw_handle* h, double dt, double* cfl) {
    if (!h) return fail(CLAW_E_INVALID, "null handle");
    CUDA_TRY(cudaSetDevice(h->device));
    ClawCtl* c = h->ctl_h;
    std::memset(c, 0, sizeof(ClawCtl));
    c->wait_ns = h->wait_ns;
    c->skip_row = h->skip_row;
    c->mode = CTL_SINGLE;
    c->dt = dt;
    c->cur = h->cur;
    c->maxn = 1;
    c->cfl_max = h->cfg.cfl_max;  // dimensional splitting stops at a sweep above it
    c->t = c->told = h->t_now;
    int rc = push_ctl(h);
    if (rc) return rc;
    CUDA_TRY(h->runner->launch(h->stream));
    h->launches += h->runner->launches_per_step();
    rc = pull_ctl(h);
    if (rc) return rc;
    h->cur = c->cur;  // unchanged when a device wait gave up (the step is not kept)
    if (cfl) *cfl = c->cfl_last;
    if (c->err & CTL_ERR_TMA_TIMEOUT) return fail(CLAW_E_DEVICE, "device wait timed out");
    h->t_now += dt;
    return 0;
}

static int ensure_graph(claw_handle* h, int steps) {
    if (h->gexec && h->gsteps == steps) return 0;
    if (h->gexec) {
        cudaGraphExecDestroy(h->gexec);
        h->gexec = nullptr;
    }
    cudaGraph_t graph;
    CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < steps; ++k) {
        cudaError_t e = h->runner->launch(h->stream);
        if (e != cudaSuccess) {
            cudaStreamEndCapture(h->stream, &graph);
            return fail(CLAW_E_CUDA, "launch during capture: %s", cudaGetErrorString(e));
        }
    }
    CUDA_TRY(cudaStreamEndCapture(h->stream, &graph));
    cudaError_t e = cudaGraphInstantiate(&h->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(CLAW_E_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    h->gsteps = steps;
    return 0;
}

int claw_advance(claw_handle* h, double tstart, double tend, double dt_initial, claw_stats* st) {
    if (!h) return fail(CLAW_E_INVALID, "null handle");
    CUDA_TRY(cudaSetDevice(h->device));
    const claw_config& cfg = h->cfg;
    ClawCtl* c = h->ctl_h;
    std::memset(c, 0, sizeof(ClawCtl));
    c->wait_ns = h->wait_ns;
    c->skip_row = h->skip_row;
    c->t = c->told = tstart;
    c->tstart = tstart;
    c->tend = tend;
    c->dt = dt_initial;
    c->dt_max = cfg.dt_max;
    c->cfl_max = cfg.cfl_max;
    c->cfl_desired = cfg.cfl_desired;
    c->dtmin = c->dtmax = dt_initial;
    c->mode = CTL_ADVANCE;
    c->dt_variable = cfg.dt_variable ? 1 : 0;
    c->cur = h->cur;
    int maxn = cfg.steps_max;
    int info = 0;
    // argument checks of claw2 (src/2d/claw2.f:508-543)
    if (!cfg.dt_variable) {
        if (tend < tstart) maxn = 1;
        else {
            maxn = (int)std::lround((tend - tstart) / dt_initial);
            if (std::fabs(maxn * dt_initial - (tend - tstart)) > 1e-5 * (tend - tstart)) info = 2;
        }
    }
    if (!info && cfg.dt_variable && cfg.cfl_desired > cfg.cfl_max) info = 3;
    if (!info && cfg.capa_index > cfg.num_aux) info = 5;
    // with dimensional splitting method(3) < 0 passes both checks
    const bool split = cfg.dimensional_split > 0;
    if (!info && !split && cfg.order < cfg.transverse_waves && cfg.num_dim == 2) info = 6;
    if (!info && !split && cfg.num_dim == 3) {
        // src/3d/chkmth.f: the unsplit transverse codes allowed per order
        const int t3 = cfg.transverse_waves;
        const bool ok = t3 == 0 || t3 == 10 || t3 == 11 ||
                        (cfg.order == 2 && (t3 == 20 || t3 == 21 || t3 == 22));
        if (!ok) info = 6;
    }
    c->maxn = maxn;
    c->done = (info != 0 || maxn == 0) ? 1 : 0;
    if (!c->done && c->told + c->dt > tend && tstart < tend) c->dt = tend - c->told;
    int rc = push_ctl(h);
    if (rc) return rc;
    const long long launches0 = h->launches;
    // graph chunk size: one host check per round, 8 steps per graph for large
    // grids; the graph is built before the timed region (one-time set-up)
    const long long cells = (long long)h->g.mx * h->g.my * h->g.mz;
    const int chunk = cells >= (1LL << 22) ? 8 : 32;
    if (!c->done && h->g.dim != 1) {
        rc = ensure_graph(h, chunk);
        if (rc) return rc;
    }
    CUDA_TRY(cudaEventRecord(h->ev0, h->stream));
    if (!c->done) {
        if (h->g.dim == 1) {
            // the 1D kernel runs the whole time loop inside one launch
            CUDA_TRY(h->runner->launch(h->stream));
            h->launches++;
            rc = pull_ctl(h);
            if (rc) return rc;
        } else {
            // Rounds: each launches the steps still needed as far as the host
            // can tell from the control block (the steps left to tend at the
            // current dt, or to steps_max), as graph chunks plus single
            // launches for the remainder, then reads the control block once.
            // A round that falls short (a rejected step, a smaller dt) is
            // followed by another; launches past `done` return at once.
            for (;;) {
                long long want = (long long)c->maxn - c->n;
                if (c->dt_variable && c->dt > 0.0) {
                    const double left = (c->tend - c->told) / c->dt;
                    if (left < (double)want) want = (long long)std::ceil(left - 1e-9);
                }
                want = std::max(1LL, std::min(want, 4096LL));
                long long k = 0;
                for (; k + chunk <= want; k += chunk)
                    CUDA_TRY(cudaGraphLaunch(h->gexec, h->stream));
                for (; k < want; ++k) CUDA_TRY(h->runner->launch(h->stream));
                h->launches += want * h->runner->launches_per_step();
                rc = pull_ctl(h);
                if (rc) return rc;
                if (c->done || c->err) break;
            }
        }
    }
    CUDA_TRY(cudaEventRecord(h->ev1, h->stream));
    CUDA_TRY(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->cur = c->cur;
    h->t_now = c->t;
    if (!info && cfg.dt_variable && c->t < tend && c->n == maxn) info = 11;
    if (!info && !cfg.dt_variable && c->cflmax_seen > cfg.cfl_max) info = 12;
    if (c->err & CTL_ERR_TMA_TIMEOUT) info = CLAW_E_DEVICE;
    else if (c->err & CTL_ERR_NAN_CFL) info = CLAW_E_NAN;
    if (st) {
        st->t_reached = c->t;
        st->dt_min = c->dtmin;
        st->dt_max_taken = c->dtmax;
        st->dt_next = c->dt;
        st->cfl_max_seen = c->cflmax_seen;
        st->cfl_last = c->cfl_last;
        st->steps_taken = c->n;
        st->steps_rejected = c->nrej;
        st->info = info;
        st->device_error = c->err;
        st->device_ms = ms;
        st->launches = h->launches - launches0;
    }
    if (info < 0) return fail(info, "device error flags 0x%x", c->err);
    return info;
}

int claw_advance_host(claw_handle* h, double* q, double tstart, double tend, double dt_initial,
                      claw_stats* st) {
    int rc = claw_set_q(h, q);
    if (rc) return rc;
    const int info = claw_advance(h, tstart, tend, dt_initial, st);
    if (info < 0) return info;
    rc = claw_get_q(h, q);
    if (rc) return rc;
    return info;
}

int claw_q_device(claw_handle* h, void** ptr, int* elem_bytes, long long* ld, long long* fp) {
    if (!h) return fail(CLAW_E_INVALID, "null handle");
    if (ptr) *ptr = h->g.q[h->cur];
    if (elem_bytes) *elem_bytes = h->g.es;
    if (ld) *ld = h->g.ld;
    if (fp) *fp = h->g.fstride;
    return 0;
}

long long claw_launch_count(claw_handle* h) { return h ? h->launches : 0; }

int claw_set_steps_max(claw_handle* h, int steps_max) {
    if (!h) return fail(CLAW_E_INVALID, "null handle");
    if (steps_max < 1) return fail(CLAW_E_INVALID, "steps_max must be >= 1");
    h->cfg.steps_max = steps_max;
    return 0;
}

int claw_debug_fault(claw_handle* h, long long wait_ns, int skip_row) {
    if (!h) return fail(CLAW_E_INVALID, "null handle");
    if (wait_ns < 0) return fail(CLAW_E_INVALID, "wait_ns must be >= 0");
    h->wait_ns = (unsigned long long)wait_ns;
    h->skip_row = skip_row < -2 ? 0 : skip_row + 1;
    return 0;
}

int claw_totals(claw_handle* h, double* totals) {
    if (!h || !totals) return fail(CLAW_E_INVALID, "null argument");
    CUDA_TRY(cudaSetDevice(h->device));
    const Geometry& g = h->g;
    const int meqn = g.meqn;
    if (!h->totals_scratch)
        CUDA_TRY(cudaMalloc(&h->totals_scratch, ((size_t)TOT_BLOCKS_MAX * meqn * 2 + meqn) * sizeof(double)));
    const long long ncell = (long long)g.mx * g.my * g.mz;
    const int nb = (int)std::max(1LL, std::min((long long)TOT_BLOCKS_MAX, (ncell + 4095) / 4096));
    double* part = h->totals_scratch;
    double* out = part + (size_t)TOT_BLOCKS_MAX * meqn * 2;
    const int capa = h->cfg.capa_index;
    if (g.es == 8)
        totals_partial_kernel<double><<<nb, TOT_THREADS, 0, h->stream>>>(
            static_cast<const double*>(g.q[h->cur]), static_cast<const double*>(g.aux), capa, g.ld,
            g.fstride, g.ald, g.afstride, g.mx, g.my, g.mz, g.dim, meqn, part);
    else
        totals_partial_kernel<float><<<nb, TOT_THREADS, 0, h->stream>>>(
            static_cast<const float*>(g.q[h->cur]), static_cast<const float*>(g.aux), capa, g.ld,
            g.fstride, g.ald, g.afstride, g.mx, g.my, g.mz, g.dim, meqn, part);
    CUDA_TRY(cudaGetLastError());
    totals_final_kernel<<<1, 32, 0, h->stream>>>(part, nb, meqn, out);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(totals, out, meqn * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

}  // extern "C"
