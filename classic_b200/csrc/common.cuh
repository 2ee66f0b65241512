// Shared device-side pieces of the wave-propagation kernels: the device
// control block (time/dt/CFL state of the claw2-style time loop), mbarrier and
// TMA helpers written directly in PTX for sm_100a, and the wave limiter.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace clawb200 {

// ----------------------------------------------------------- control block ---
// Device-resident state of one claw2-style advance (src/2d/claw2.f:494-784).
// Every step kernel reads dt / cur at entry; the last CTA to finish a step
// folds the CFL maximum and runs the accept/reject + next-dt logic here, so a
// whole time loop runs without a host round trip per step.
struct ClawCtl {
    double t, told, dt, tstart, tend;
    double dt_max, cfl_max, cfl_desired;
    double cflmax_seen, dtmin, dtmax, cfl_last;
    unsigned long long cfl_bits;   // atomicMax target (bit pattern of a double >= 0)
    unsigned int ctas_done;        // last-CTA counter, reset by the last CTA
    int cur;                       // index of the buffer holding the current q
    int n, maxn, nrej;             // accepted steps, step limit, rejected steps
    int done, info;
    int mode;                      // CTL_ADVANCE or CTL_SINGLE
    int dt_variable;
    int err;                       // device error flags (CTL_ERR_*)
    int skip_row;                  // test hook: 1 + the row whose copy strip 0 skips (0: none)
    unsigned long long cfl_sweep[2];  // dimensional splitting: Courant maxima of the
                                      // y-sweep and of Strang's last x-sweep
    unsigned long long wait_ns;    // limit of a device-side wait (0: the 2 s default)
};

constexpr unsigned long long WAIT_NS_DEFAULT = 2000000000ull;
__device__ __forceinline__ unsigned long long ctl_wait_ns(const ClawCtl* c) {
    const unsigned long long w = *(volatile const unsigned long long*)&c->wait_ns;
    return w ? w : WAIT_NS_DEFAULT;
}

enum { CTL_ADVANCE = 0, CTL_SINGLE = 1 };

// Boundary-condition codes (mthbc in claw.data).
enum { BC_USER = 0, BC_EXTRAP = 1, BC_PERIODIC = 2, BC_WALL = 3 };
enum { CTL_ERR_TMA_TIMEOUT = 1, CTL_ERR_NAN_CFL = 2 };

// Controller step: identical decisions to claw2's main loop.  Runs in exactly
// one thread after every CTA of the step has published its CFL maximum.
__device__ __forceinline__ void ctl_finish_step(ClawCtl* c) {
    const double cfl = __longlong_as_double((long long)atomicAdd(&c->cfl_bits, 0ull));
    c->cfl_bits = 0ull;
    c->ctas_done = 0u;
    c->cfl_last = cfl;
    if (c->err) {  // a device wait gave up: the step's output is incomplete
        c->done = 1;
        return;
    }
    if (c->mode == CTL_SINGLE) {
        c->cur ^= 1;
        return;
    }
    if (cfl != cfl) {  // NaN: stop instead of retrying forever
        c->err |= CTL_ERR_NAN_CFL;
        c->done = 1;
        return;
    }
    c->t = c->told + c->dt;
    if (cfl <= c->cfl_max) {
        c->cflmax_seen = fmax(cfl, c->cflmax_seen);
        c->cur ^= 1;
        if (c->dt_variable) {
            if (cfl == 0.0) c->dt = c->dt_max;
            else c->dt = fmin(c->dt_max, c->dt * c->cfl_desired / cfl);
            c->dtmin = fmin(c->dt, c->dtmin);
            c->dtmax = fmax(c->dt, c->dtmax);
        }
        c->n += 1;
        if (c->t >= c->tend || c->n >= c->maxn) {
            c->done = 1;
        } else {
            c->told = c->t;
            if (c->told + c->dt > c->tend && c->tstart < c->tend) c->dt = c->tend - c->told;
        }
    } else {
        c->t = c->told;
        c->nrej += 1;
        if (c->dt_variable) {
            c->dt = fmin(c->dt_max, c->dt * c->cfl_desired / cfl);
        } else {
            c->cflmax_seen = fmax(cfl, c->cflmax_seen);
            c->done = 1;
        }
    }
}

// Publish one CTA's CFL maximum and, in the last CTA, run the controller.
// Call with all threads of the CTA; red must hold >= blockDim/32 doubles.
__device__ __forceinline__ void cta_cfl_and_control(ClawCtl* ctl, double cfl, double* red) {
    for (int off = 16; off > 0; off >>= 1) cfl = fmax(cfl, __shfl_xor_sync(0xffffffffu, cfl, off));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) red[warp] = cfl;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
        if (!(m > 0.0)) m = (m != m) ? m : 0.0;  // canonical +0, keep NaN
        atomicMax(&ctl->cfl_bits, (unsigned long long)__double_as_longlong(m));
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->ctas_done, 1u);
        if (prev == gridDim.x - 1) {
            __threadfence();
            ctl_finish_step(ctl);
            __threadfence();
        }
    }
}

// ----------------------------------------------------------- PTX helpers ---
// Programmatic dependent launch: a step kernel launched with the programmatic
// stream-serialization attribute may be scheduled while the previous step's
// grid drains; it waits here, before its first read of the control block or
// q, for that grid to complete and its memory to be visible, then lets the
// next step's grid be scheduled in turn.  (Launched without the attribute,
// both instructions return at once.)  At 1024^2 the per-step time falls by
// 6-8 %: the launch and the CTAs' start-up overlap the previous grid's tail.
#ifndef CLAW_PDL
#define CLAW_PDL 1
#endif
__device__ __forceinline__ void grid_dependency_sync() {
#if CLAW_PDL
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait on an mbarrier phase: gives up after limit_ns of wall time
// (2 s unless the control block sets another limit) and reports failure
// instead of hanging the GPU.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  unsigned long long limit_ns = 2000000000ull) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 255u) == 0u && globaltimer_ns() - t0 > limit_ns) return false;
    }
}

// 3D tiled TMA load (no multicast): box -> shared memory, completion on bar.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            int w, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
        : "memory");
}

// ------------------------------------------------- contracted arithmetic ---
// Reciprocal and square root for the contracted (CLAW_FP64_FMA) kernels, by
// Newton-Raphson refinement of the hardware estimates (rcp.approx /
// rsqrt.approx, about 23 correct bits): each step doubles the correct bits,
// so two steps reach double precision to within about an ulp.  The
// reference-order kernels keep IEEE division and sqrt.
__device__ __forceinline__ double rcp_newton(double a) {
    // y <- y + y (1 - a y)
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
    double e = fma(-a, y, 1.0);
    y = fma(y, e, y);
    e = fma(-a, y, 1.0);
    y = fma(y, e, y);
    return y;
}
__device__ __forceinline__ float rcp_newton(float a) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(a));
    const float e = fmaf(-a, y, 1.0f);
    return fmaf(y, e, y);
}
// sqrt(a): y ~ 1/sqrt(a) refined by y <- y (3 - a y^2) / 2 twice, then the
// root s = a y corrected once by s <- s + y (a - s^2) / 2 (Newton on s^2 = a).
// a = 0 gives 0 and a < 0 NaN, as sqrt does.
__device__ __forceinline__ double sqrt_newton(double a) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
    double h = 0.5 * a;
    y = y * fma(-h * y, y, 1.5);
    y = y * fma(-h * y, y, 1.5);
    const double s = a * y;
    const double r = fma(0.5 * y, fma(-s, s, a), s);
    return a == 0.0 ? a : r;
}

// Arithmetic policy of a kernel build: IEEE division and square root in the
// reference-order build (bit-identical to the CPU restatement), Newton
// reciprocals and roots in the contracted build.
template <bool FAST>
struct Arith {
    template <typename real>
    __device__ __forceinline__ static real rcp(real a) { return real(1) / a; }
    template <typename real>
    __device__ __forceinline__ static real div(real a, real b) { return a / b; }
    template <typename real>
    __device__ __forceinline__ static real root(real a) { return sqrt(a); }
};
template <>
struct Arith<true> {
    template <typename real>
    __device__ __forceinline__ static real rcp(real a) { return rcp_newton(a); }
    template <typename real>
    __device__ __forceinline__ static real div(real a, real b) { return a * rcp_newton(b); }
    __device__ __forceinline__ static double root(double a) { return sqrt_newton(a); }
    __device__ __forceinline__ static float root(float a) { return sqrtf(a); }
};

// ------------------------------------------------------------- limiter ---
// Limiter function phi(r) of src/2d/inlinelimiter.f90:71-97
// (1 minmod, 2 superbee, 3 van Leer, 4 MC, 5 Beam-Warming).
template <typename real>
__device__ __forceinline__ real phi_limiter(int meth, real r) {
    const real zero = real(0), one = real(1), two = real(2);
    switch (meth) {
        case 1: return fmax(zero, fmin(one, r));
        case 2: return fmax(fmax(zero, fmin(one, two * r)), fmin(two, r));
        case 3: return (r + fabs(r)) / (one + fabs(r));
        case 4: {
            const real c = (one + r) * real(0.5);  // == (1+r)/2 exactly
            return fmax(zero, fmin(fmin(c, two), two * r));
        }
        case 5: return r;
        default: return one;
    }
}

// phi(r) of the contracted build: the same functions by compare-and-select
// (no fmin/fmax, whose NaN rules cost extra FP64 instructions) and a Newton
// reciprocal in van Leer's quotient.
template <typename real>
__device__ __forceinline__ real phi_limiter_fast(int meth, real r) {
    const real zero = real(0), one = real(1), two = real(2);
    auto mn = [](real a, real b) { return a < b ? a : b; };
    auto mx = [](real a, real b) { return a > b ? a : b; };
    switch (meth) {
        case 1: return mx(zero, mn(one, r));
        case 2: return mx(mx(zero, mn(one, two * r)), mn(two, r));
        case 3: {
            const real ar = fabs(r);
            return (r + ar) * rcp_newton(one + ar);
        }
        case 4: return mx(zero, mn(mn((one + r) * real(0.5), two), two * r));
        case 5: return r;
        default: return one;
    }
}

}  // namespace clawb200
