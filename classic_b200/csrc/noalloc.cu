// claw_step2d_noalloc: one 2D step on caller-owned device buffers without
// allocating any device memory.
//
// Who needs it: codes that own every byte of device memory through their own
// pool or arena (a host framework's caching allocator, a coupled model with
// a fixed memory budget, a memory-capped GPU partition) and callers that
// cannot accept cudaMalloc's implicit device-wide synchronisation inside a
// time loop.  The regular path (claw_create) allocates q, aux and a small
// control block with cudaMalloc; here the caller passes q_in, q_out and aux,
// and the step kernel's only scratch memory -- its control block (CFL
// accumulator, last-CTA counter, dt state) -- lives in the file-scope array
// below, which every GPU that loads the library holds until exit.
//
// The step kernel is the same one claw_step launches (step2d.cuh).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/claw_b200.h"
#include "common.cuh"
#include "riemann.cuh"
#include "step2d.cuh"

using namespace clawb200;

namespace clawb200 {
void set_last_error(const char* msg);  // message for claw_last_error()
}

namespace {

// Stated maximum of the scratch this entry point may use: 256 bytes.  One
// step needs exactly one control block, whatever the grid size.
constexpr size_t NOALLOC_SCRATCH_BYTES = 256;
static_assert(sizeof(ClawCtl) <= NOALLOC_SCRATCH_BYTES, "control block exceeds the scratch array");

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;

int nofail(int code, const char* msg) {
    clawb200::set_last_error(msg);
    return code;
}

// Device address of the scratch array on the current device.  The host-side
// name g_noalloc_scratch is only a stand-in; the kernel must be given this
// address.  It is looked up on every call (a lookup allocates nothing), so a
// context rebuilt after cudaDeviceReset is served from its own module.
int scratch_address(void** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        char buf[256];
        snprintf(buf, sizeof(buf), "cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        return nofail(CLAW_E_CUDA, buf);
    }
    *out = p;
    return 0;
}

// Per device and kernel instantiation: the dynamic shared-memory attribute
// has been set and the resident CTAs per SM are known.  A launch that fails
// (a context rebuilt after cudaDeviceReset has lost the attribute) clears the
// entry and is retried once after the set-up runs again.
template <class S, class M>
struct LaunchSetup {
    static int per_sm[MAX_DEVICES];
    static int nsm[MAX_DEVICES];
};
template <class S, class M>
int LaunchSetup<S, M>::per_sm[MAX_DEVICES] = {};
template <class S, class M>
int LaunchSetup<S, M>::nsm[MAX_DEVICES] = {};

PFN_cuTensorMapEncodeTiled_v12000 encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult qr;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &qr) ==
                cudaSuccess && qr == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

int map3(CUtensorMap* m, const void* base, long long n0, long long n1, long long n2,
         long long p1, long long p2, int box0, int box2) {
    auto fn = encode();
    if (!fn) return nofail(CLAW_E_CUDA, "cuTensorMapEncodeTiled is unavailable");
    const cuuint64_t dims[3] = {(cuuint64_t)n0, (cuuint64_t)n1, (cuuint64_t)n2};
    const cuuint64_t strides[2] = {(cuuint64_t)(p1 * 8), (cuuint64_t)(p2 * 8)};
    const cuuint32_t box[3] = {(cuuint32_t)box0, 1u, (cuuint32_t)box2};
    const cuuint32_t estr[3] = {1, 1, 1};
    if (fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void*>(base), dims, strides, box, estr,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return nofail(CLAW_E_INVALID, "cuTensorMapEncodeTiled rejected the buffers (pitch/alignment)");
    return 0;
}

template <class S, class M>
int launch_step(const claw_config* c, const S& solver, const double* q_in, double* q_out,
                long long q_ld, const double* aux, long long aux_ld, ClawCtl* ctl,
                cudaStream_t st) {
    using R = Ring2D<S>;
    Step2Args<S> a;
    std::memset(&a, 0, sizeof(a));
    a.solver = solver;
    const int mx = c->num_cells[0], my = c->num_cells[1];
    a.q[0] = const_cast<double*>(q_in);
    a.q[1] = q_out;
    a.aux = aux;
    a.ld = q_ld;
    a.fstride = q_ld * my;
    a.ald = aux_ld;
    a.afstride = aux_ld * (my + 4);
    a.mx = mx;
    a.my = my;
    a.nstrips = (mx + STRIP - 1) / STRIP;
    a.bc[0] = c->bc_lower[0];
    a.bc[1] = c->bc_upper[0];
    a.bc[2] = c->bc_lower[1];
    a.bc[3] = c->bc_upper[1];
    for (int k = 0; k < 8; ++k) a.mthlim[k] = k < c->num_waves ? c->limiter[k] : 0;
    a.order = c->order;
    a.trans = c->transverse_waves;
    a.fwave = c->use_fwaves;
    a.capa = c->capa_index;
    a.dx = (c->upper[0] - c->lower[0]) / (double)(float)mx;
    a.dy = (c->upper[1] - c->lower[1]) / (double)(float)my;
    a.ctl = ctl;
    int rc = map3(&a.tmq[0], q_in, mx, my, S::meqn, q_ld, a.fstride, R::W, S::meqn);
    if (rc) return rc;
    rc = map3(&a.tmq[1], q_out, mx, my, S::meqn, q_ld, a.fstride, R::W, S::meqn);
    if (rc) return rc;
    if (S::maux > 0) {
        rc = map3(&a.tmaux, aux, mx + 4, my + 4, S::maux, aux_ld, a.afstride, R::W, S::maux);
        if (rc) return rc;
    }
    const int smem = R::SMEM;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
        return nofail(CLAW_E_CUDA, "cudaGetDevice failed or device ordinal out of range");
    a.units = (long long)a.nstrips * my;
    for (int attempt = 0; attempt < 2; ++attempt) {
        int per_sm = 0, nsm = 0;
        {
            std::lock_guard<std::mutex> lock(g_mu);
            if (!LaunchSetup<S, M>::per_sm[dev]) {
                int n = 0, r = 0;
                if (cudaFuncSetAttribute(step2_kernel<S, M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         smem) != cudaSuccess)
                    return nofail(CLAW_E_CUDA, "cudaFuncSetAttribute failed");
                if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
                    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, step2_kernel<S, M>, 32 * WARPS2D,
                                                                  smem) != cudaSuccess || r < 1)
                    return nofail(CLAW_E_CUDA, "occupancy query failed");
                LaunchSetup<S, M>::nsm[dev] = n;
                LaunchSetup<S, M>::per_sm[dev] = r;
            }
            per_sm = LaunchSetup<S, M>::per_sm[dev];
            nsm = LaunchSetup<S, M>::nsm[dev];
        }
        const long long want = a.units / 48 > 0 ? a.units / 48 : 1;
        const long long full = (long long)nsm * per_sm * WARPS2D;
        const long long nw = want < full ? want : full;
        const int grid = (int)((nw + WARPS2D - 1) / WARPS2D);
        a.nwarps = (int)nw;
        step2_kernel<S, M><<<grid, 32 * WARPS2D, smem, st>>>(a);
        if (cudaGetLastError() == cudaSuccess) return 0;
        std::lock_guard<std::mutex> lock(g_mu);
        LaunchSetup<S, M>::per_sm[dev] = 0;
    }
    return nofail(CLAW_E_CUDA, "step kernel launch failed");
}

}  // namespace

extern "C" int claw_step2d_noalloc(const claw_config* cfg, const double* q_in, double* q_out,
                                   long long q_ld, const double* aux, long long aux_ld, double dt,
                                   double* cfl, void* stream) {
    if (!cfg || !q_in || !q_out || !cfl) return nofail(CLAW_E_INVALID, "null argument");
    if (cfg->num_dim != 2) return nofail(CLAW_E_INVALID, "claw_step2d_noalloc is 2D only");
    if (cfg->precision != CLAW_FP64) return nofail(CLAW_E_INVALID, "claw_step2d_noalloc is FP64 only");
    if (q_in == q_out) return nofail(CLAW_E_INVALID, "q_in and q_out must be distinct buffers");
    const int mx = cfg->num_cells[0], my = cfg->num_cells[1];
    if (mx < 2 || my < 2 || cfg->num_ghost != 2) return nofail(CLAW_E_INVALID, "bad grid");
    if (q_ld < mx || (q_ld * 8) % 16 != 0)
        return nofail(CLAW_E_INVALID, "q_ld must be >= mx and a multiple of 2 elements");
    if (((uintptr_t)q_in | (uintptr_t)q_out) % 16 != 0)
        return nofail(CLAW_E_INVALID, "q buffers must be 16-byte aligned");
    if (sizeof(ClawCtl) > NOALLOC_SCRATCH_BYTES)
        return nofail(CLAW_E_INVALID, "step needs more scratch than the 256-byte array holds");
    for (int d = 0; d < 2; ++d)
        if (cfg->bc_lower[d] < 1 || cfg->bc_lower[d] > 3 || cfg->bc_upper[d] < 1 || cfg->bc_upper[d] > 3)
            return nofail(CLAW_E_INVALID, "boundary conditions must be extrap, periodic or wall");
    if (cfg->order < 1 || cfg->order > 2 || cfg->dimensional_split != 0)
        return nofail(CLAW_E_INVALID, "unsupported method");
    // claw_step runs the before-step routine on a copy of the unscaled aux
    // that it allocates; without an allocation there is no such copy.
    if (cfg->b4step_id != CLAW_B4STEP_NONE)
        return nofail(CLAW_E_UNSUPPORTED, "claw_step2d_noalloc runs no before-step routine");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // Each call waits for the stream and uploads its control block from a
    // host variable, neither of which a captured graph could replay.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess)
        return nofail(CLAW_E_CUDA, "cudaStreamIsCapturing failed");
    if (cap != cudaStreamCaptureStatusNone)
        return nofail(CLAW_E_INVALID, "claw_step2d_noalloc must not be called during stream capture");
    void* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;

    // The array keeps the previous call's contents: reset the whole block.
    ClawCtl h;
    std::memset(&h, 0, sizeof(h));
    h.mode = CTL_SINGLE;
    h.dt = dt;
    h.cur = 0;
    h.maxn = 1;
    if (cudaMemcpyAsync(scratch, &h, sizeof(h), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return nofail(CLAW_E_CUDA, "control block upload failed");
    ClawCtl* ctl = static_cast<ClawCtl*>(scratch);

    const int id = cfg->solver_id;
    if (id == CLAW_SOLVER_ACOUSTICS_2D) {
        if (cfg->num_eqn != 3 || cfg->num_waves != 2 || cfg->num_aux != 0)
            return nofail(CLAW_E_INVALID, "acoustics_2d needs num_eqn 3, num_waves 2, num_aux 0");
        const double rho = cfg->solver_params[0], bulk = cfg->solver_params[1];
        const double cc = std::sqrt(bulk / rho), zz = rho * cc;
        const Acoustics2D<double> s{cc, zz, 0.5 / zz};
        bool mc = cfg->order == 2 && cfg->transverse_waves == 2 && cfg->capa_index == 0 && !cfg->use_fwaves;
        for (int k = 0; k < cfg->num_waves; ++k) mc = mc && cfg->limiter[k] == 4;
        rc = mc ? launch_step<Acoustics2D<double>, MethodMC2D>(cfg, s, q_in, q_out, q_ld, aux, aux_ld, ctl, st)
                : launch_step<Acoustics2D<double>, MethodGeneric2D>(cfg, s, q_in, q_out, q_ld, aux, aux_ld, ctl, st);
    } else if (id == CLAW_SOLVER_VC_ADVECTION_2D) {
        if (cfg->num_eqn != 1 || cfg->num_waves != 1 || cfg->num_aux != 3 || !aux)
            return nofail(CLAW_E_INVALID, "vc_advection_2d needs num_eqn 1, num_waves 1, 3 aux fields");
        if (aux_ld < mx + 4 || (aux_ld * 8) % 16 != 0 || (uintptr_t)aux % 16 != 0)
            return nofail(CLAW_E_INVALID, "aux_ld must be >= mx+4, a multiple of 2, aux 16-byte aligned");
        rc = launch_step<VCAdvection2D<double>, MethodGeneric2D>(cfg, VCAdvection2D<double>{}, q_in, q_out,
                                                                   q_ld, aux, aux_ld, ctl, st);
    } else {
        return nofail(CLAW_E_UNSUPPORTED, "claw_step2d_noalloc: solver not built for this entry point");
    }
    if (rc) return rc;
    if (cudaMemcpyAsync(&h, scratch, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return nofail(CLAW_E_CUDA, "step failed on the device");
    if (h.err & CTL_ERR_TMA_TIMEOUT) return nofail(CLAW_E_DEVICE, "device wait timed out");
    *cfl = h.cfl_last;
    // A NaN Courant number means a NaN in the new state (for instance a
    // capacity field that is not positive, which this path does not check).
    if (h.cfl_last != h.cfl_last) return nofail(CLAW_E_NAN, "Courant number is NaN");
    return 0;
}
