// 2D wave-propagation step for linear constant-coefficient acoustics in
// characteristic variables (the CLAW_FP64_FMA and CLAW_FP32 paths).
//
// Same algorithm as step2d.cuh (src/2d/step2.f90, flux2.f90,
// inlinelimiter.f90 with transverse_waves = 2, order 2), rewritten for a
// system whose eigenvectors do not vary in space:
//   * a jump dq splits into wave strengths a1, a2 on the fixed eigenvectors
//     (-Z,1,0), (Z,1,0) (normal velocity second), speeds -c, +c;
//   * the limiter ratio (w_i . w_j)/(w_i . w_i) of inlinelimiter.f90:53-68
//     is a_j / a_i exactly in real arithmetic, so only wave strengths cross
//     lanes;
//   * cqxx, fadd, amdq +/- cqxx and the transverse split of rpt2 collapse to
//     a few scalars per interface (the transverse split of a fluctuation
//     with pressure component A gives B-+ = (-+c/2 A, 0, c/(2Z) A)).
// The Courant number is formed exactly as in flux2 (dtdx*c, dtdy*c), so the
// dt sequence equals the reference's bit for bit; q differs from the
// reference-order FP64 path only by rounding (fused multiply-adds, a Newton
// reciprocal in the limiter ratio).
//
// Memory movement, boundary conditions, the TMA row ring and the device-side
// dt controller are those of step2d.cuh.
#pragma once
#include "common.cuh"
#include "step2d.cuh"

namespace clawb200 {

template <typename real>
struct CharAcoustics2D {
    real cc, zz, hz;  // c, Z, 1/(2Z)
};

__device__ __forceinline__ double rcp_newton(double a) {
    // reciprocal: hardware estimate (~23 bits) refined by two Newton-Raphson
    // steps y <- y + y(1 - a y), each doubling the correct bits
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

// phi(r) of inlinelimiter.f90:71-97 for a strength ratio r = num/den;
// den == 0 (no wave) gives a zero limited strength, as the reference skips it.
template <typename real, int LIM>
__device__ __forceinline__ real limited_strength(real a, real anb, int lim_rt) {
    const real inv = rcp_newton(a != real(0) ? a : real(1));
    const real r = anb * inv;
    const int lim = LIM >= 0 ? LIM : lim_rt;
    const real ph = lim == 0 ? real(1) : phi_limiter<real>(lim, r);
    return ph * a;
}

template <typename real>
struct CharArgs {
    CUtensorMap tmq[2];
    real* q[2];
    long long ld, fstride;
    int mx, my, nstrips;
    int bc[4];
    int lim;
    double dx, dy;
    long long units;
    int nwarps;
    ClawCtl* ctl;
    CharAcoustics2D<real> s;
};

template <typename real>
struct CharRing {
    static constexpr int W = BoxW<real>::value;
    static constexpr int QB = 3 * W * (int)sizeof(real);
    static constexpr int SLOT = ((QB + 127) / 128) * 128;
    static constexpr int WARP_BYTES = RING * SLOT;
    static constexpr int SMEM = WARPS2D * WARP_BYTES + WARPS2D * RING * 8 + 64;
};

template <typename real, int LIM>
__global__ void __launch_bounds__(32 * WARPS2D, sizeof(real) == 8 ? 5 : 6)
step2_char_kernel(const __grid_constant__ CharArgs<real> A) {
    using R = CharRing<real>;
    constexpr int W = R::W;
    constexpr unsigned FULL = 0xffffffffu;
    ClawCtl* ctl = A.ctl;
    __shared__ double red[WARPS2D];
    if (*(volatile int*)&ctl->done) return;
    const int cur = *(volatile int*)&ctl->cur;
    const double dtd = *(volatile double*)&ctl->dt;
    const double dtdx_d = dtd / A.dx, dtdy_d = dtd / A.dy;
    const real dtdx = (real)dtdx_d, dtdy = (real)dtdy_d;
    const real* __restrict__ qold = A.q[cur];
    real* __restrict__ qnew = A.q[cur ^ 1];
    const CUtensorMap* tmq = &A.tmq[cur];
    const real c = A.s.cc, Z = A.s.zz, h = A.s.hz;
    const real cZ = c * Z;
    // per-direction constants: kappa = c(1 - c dt/dx) (second-order
    // coefficient of flux2.f90:156-157), fadd = kappa/2 (...), transverse
    // gamma = dt/dx c/4 and delta = dt/dx c/(4Z) scaled by the other dt/d.
    const real kx = c * (real(1) - c * dtdx), ky = c * (real(1) - c * dtdy);
    const real fxp = real(0.5) * kx * Z, fxu = real(0.5) * kx;  // x: F = (fxp(a2-a1), fxu(a1+a2))
    const real fyp = real(0.5) * ky * Z, fyv = real(0.5) * ky;
    const real gx = dtdy * (dtdx * c * real(0.25)), dx4 = dtdy * (dtdx * c * real(0.25) / Z);
    const real gy = dtdx * (dtdy * c * real(0.25)), dy4 = dtdx * (dtdy * c * real(0.25) / Z);
    const real qpx = dtdx * cZ, qux = dtdx * c;  // Godunov: qadd from a1, a2 (x)
    const real qpy = dtdy * cZ, qvy = dtdy * c;

    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* ring = smem + warp * R::WARP_BYTES;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + WARPS2D * R::WARP_BYTES) + warp * RING;
    if (lane == 0) {
        for (int sl = 0; sl < RING; ++sl) mbar_init(&bars[sl], 1);
        fence_barrier_init();
    }
    __syncwarp();
    const int mx = A.mx, my = A.my;
    bool failed = false;
    uint32_t seq_base = 0;
    bool any_work = false;

    const long long gw = (long long)blockIdx.x * WARPS2D + warp;
    long long u0 = (gw < A.nwarps) ? gw * A.units / A.nwarps : 0;
    const long long u1 = (gw < A.nwarps) ? (gw + 1) * A.units / A.nwarps : 0;

    while (u0 < u1 && !failed) {
        any_work = true;
        const int strip = (int)(u0 / my);
        const int r0 = (int)(u0 % my);
        const int nr = (int)min((long long)(my - r0), u1 - u0);
        u0 += nr;
        const int b = strip * STRIP;
        const int col = b - 1 + lane;
        const int x0 = b - BoxW<real>::XQ;
        const int rfirst = r0 - 2, rlast = r0 + nr + 1;
        const int nrows = rlast - rfirst + 1;
        bool negm, negc;
        const int sm = bc_map(col - 1, mx, A.bc[0], A.bc[1], negm);
        const int sc = bc_map(col, mx, A.bc[0], A.bc[1], negc);
        const bool gm = (sm - x0) < 0 || (sm - x0) >= W;
        const bool gc = (sc - x0) < 0 || (sc - x0) >= W;
        const bool any_global = __any_sync(FULL, gm || gc);
        const int im = gm ? 0 : sm - x0, icc = gc ? 0 : sc - x0;

        auto seq_of = [&](int r) -> uint32_t { return seq_base + (uint32_t)(r - rfirst); };
        auto issue = [&](int r) {
            const uint32_t sq = seq_of(r);
            const int sl = (int)(sq & (RING - 1));
            bool nyneg;
            const int sr = bc_map(r, my, A.bc[2], A.bc[3], nyneg);
            mbar_arrive_expect_tx(&bars[sl], (uint32_t)R::QB);
            tma_load_3d(ring + sl * R::SLOT, tmq, x0, sr, 0, &bars[sl]);
        };
        if (lane == 0) {
            const int npre = nrows < RING ? nrows : RING;
            for (int k = 0; k < npre; ++k) issue(rfirst + k);
        }
        __syncwarp();
        auto wait_row = [&](int r) -> bool {
            const uint32_t sq = seq_of(r);
            return mbar_wait_bounded(&bars[sq & (RING - 1)], (sq >> RING_LOG) & 1u);
        };
        auto load_q = [&](int r, real* qm, real* qc) {
            const real* sq = reinterpret_cast<const real*>(ring + (int)(seq_of(r) & (RING - 1)) * R::SLOT);
            bool nyneg;
            const int sr = bc_map(r, my, A.bc[2], A.bc[3], nyneg);
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                real vm = sq[m * W + im];
                real vc = sq[m * W + icc];
                if (any_global) {
                    if (gm) vm = qold[m * A.fstride + (long long)sr * A.ld + sm];
                    if (gc) vc = qold[m * A.fstride + (long long)sr * A.ld + sc];
                }
                if (m == 1) { vm = negm ? -vm : vm; vc = negc ? -vc : vc; }
                if (m == 2 && nyneg) { vm = -vm; vc = -vc; }
                qm[m] = vm;
                qc[m] = vc;
            }
        };

        real qm_t[3], qc_t[3], qm_n[3], qc_n[3];
        real q2p[3] = {real(0), real(0), real(0)};  // x-part of (c, t) before row t+1
        real axp = real(0), axv = real(0);         // x-slice t-1 -> row t (p, v)
        real a1y = real(0), a2y = real(0);         // y-interface t strengths
        real a2y_lo = real(0);                     // a2 of y-interface t-1
        real A2y_lo = real(0), Fpy_lo = real(0), Fvy_lo = real(0);  // of y-interface t-1
        int last_issued = rfirst + (nrows < RING ? nrows : RING) - 1;
        int fail_row = rlast + 1;

        if (!wait_row(rfirst) || !wait_row(rfirst + 1)) { failed = true; fail_row = rfirst; }
        if (!failed) {
            load_q(rfirst, qm_t, qc_t);
            load_q(rfirst + 1, qm_n, qc_n);
            const real dp = qc_n[0] - qc_t[0], dv = qc_n[2] - qc_t[2];
            a1y = (Z * dv - dp) * h;
            a2y = (Z * dv + dp) * h;
#pragma unroll
            for (int m = 0; m < 3; ++m) { qm_t[m] = qm_n[m]; qc_t[m] = qc_n[m]; }
        }

        for (int t = r0 - 1; t <= r0 + nr && !failed; ++t) {
            if (!wait_row(t + 1)) { failed = true; fail_row = t + 1; break; }
            load_q(t + 1, qm_n, qc_n);

            // ---- x-slice t: interface at column col ----
            const real dpx = qc_t[0] - qm_t[0], dux = qc_t[1] - qm_t[1];
            const real a1 = (Z * dux - dpx) * h;
            const real a2 = (Z * dux + dpx) * h;
            const real a1r = __shfl_down_sync(FULL, a1, 1);  // interface col+1
            const real a2l = __shfl_up_sync(FULL, a2, 1);    // interface col-1
            const real al1 = limited_strength<real, LIM>(a1, a1r, A.lim);  // s<0: upwind is col+1
            const real al2 = limited_strength<real, LIM>(a2, a2l, A.lim);  // s>0: upwind is col-1
            const real Fp = fxp * (al2 - al1), Fu = fxu * (al1 + al2);
            const real A1 = fma(cZ, a1, real(2) * Fp);   // pressure of amdq + cqxx
            const real A2 = fma(cZ, a2, real(-2) * Fp);  // pressure of apdq - cqxx
            const real Fpr = __shfl_down_sync(FULL, Fp, 1);
            const real Fur = __shfl_down_sync(FULL, Fu, 1);
            const real A1r = __shfl_down_sync(FULL, A1, 1);
            const real S = A1r + A2;
            const real gS = gx * S, dS = dx4 * S;
            // x-part of cell (col, t): q + (row t-1's transfer) + qadd - dt/dx dF - dt/dy dG
            const real nq0 = (qc_t[0] + axp) - qpx * (a2 + a1r) - dtdx * (Fpr - Fp) + real(2) * gS;
            const real nq1 = qc_t[1] + qux * (a1r - a2) - dtdx * (Fur - Fu);
            const real nq2 = qc_t[2] + axv;
            // row t completes the x-part of (col, t-1)
            const real q3p = q2p[0] - gS, q3u = q2p[1], q3v = q2p[2] + dS;
            q2p[0] = nq0;
            q2p[1] = nq1;
            q2p[2] = nq2;
            axp = -gS;
            axv = -dS;

            // ---- y-interface t+1 raw; y-interface t limited; y-part of (col, t-1) ----
            const real dpy = qc_n[0] - qc_t[0], dvy = qc_n[2] - qc_t[2];
            const real a1n = (Z * dvy - dpy) * h;
            const real a2n = (Z * dvy + dpy) * h;
            const real bl1 = limited_strength<real, LIM>(a1y, a1n, A.lim);    // upwind t+1
            const real bl2 = limited_strength<real, LIM>(a2y, a2y_lo, A.lim); // upwind t-1
            const real Fpy = fyp * (bl2 - bl1), Fvy = fyv * (bl1 + bl2);
            const real A1y = fma(cZ, a1y, real(2) * Fpy);   // into cell t-1
            const real A2y = fma(cZ, a2y, real(-2) * Fpy);  // into cell t
            const real Sy = A1y + A2y_lo;
            const real hS = gy * Sy, kS = dy4 * Sy;
            const real hSl = __shfl_up_sync(FULL, hS, 1), kSl = __shfl_up_sync(FULL, kS, 1);
            const real hSr = __shfl_down_sync(FULL, hS, 1), kSr = __shfl_down_sync(FULL, kS, 1);
            const real o0 = q3p - qpy * (a2y_lo + a1y) - dtdy * (Fpy - Fpy_lo) + real(2) * hS - hSl - hSr;
            const real o1 = q3u - kSl + kSr;
            const real o2 = q3v + qvy * (a1y - a2y_lo) - dtdy * (Fvy - Fvy_lo);
            if ((t - 1 >= r0) && (lane >= 1) && (lane <= STRIP) && (col < mx)) {
                real* dst = qnew + (long long)(t - 1) * A.ld + col;
                dst[0] = o0;
                dst[A.fstride] = o1;
                dst[2 * A.fstride] = o2;
            }
            a2y_lo = a2y;
            A2y_lo = A2y;
            Fpy_lo = Fpy;
            Fvy_lo = Fvy;
            a1y = a1n;
            a2y = a2n;
#pragma unroll
            for (int m = 0; m < 3; ++m) { qm_t[m] = qm_n[m]; qc_t[m] = qc_n[m]; }

            __syncwarp();
            if (t - 1 + RING <= rlast) {
                if (lane == 0) issue(t - 1 + RING);
                last_issued = t - 1 + RING;
            }
            __syncwarp();
        }
        if (failed) {
            for (int r = fail_row + 1; r <= last_issued; ++r) (void)wait_row(r);
            if (lane == 0) atomicOr(&ctl->err, CTL_ERR_TMA_TIMEOUT);
        }
        seq_base += (uint32_t)nrows;
    }
    // Courant number as flux2 forms it (dt/dx * c over the x-interfaces,
    // dt/dy * c over the y-interfaces; constant speeds)
    double cfl = any_work ? fmax(dtdx_d * (double)c, dtdy_d * (double)c) : 0.0;
    if (!any_work) cfl = 0.0;
    cta_cfl_and_control(ctl, cfl, red);
}

}  // namespace clawb200
