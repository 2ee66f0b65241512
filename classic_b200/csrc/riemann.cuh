// Pointwise Riemann-solver plugins.
//
// These are compile-time device functors implementing the pointwise form of
// the reference's rpn2 / rpt2 contract (documented at src/2d/claw2.f:312-404;
// called per slice at src/2d/flux2.f90:110,204,220):
//
//   rpn(ixy, qL, qR, auxL, auxR, wave[MW][ME], s[MW], amdq[ME], apdq[ME])
//       normal Riemann problem at the interface between the cell on the left
//       (qL = q(i-1)) and on the right (qR = q(i)); ixy = 1 for an x-slice,
//       2 for a y-slice.
//   rpt(ixy, imp, qL, qR, aux1, aux2, aux3, asdq[ME], bmasdq[ME], bpasdq[ME])
//       transverse split of the fluctuation asdq (imp = 1: A^- dq, which
//       enters cell i-1; imp = 2: A^+ dq, entering cell i).  aux1/aux2/aux3 are
//       the aux vectors of that receiving cell and of its two transverse
//       neighbours (below/above for an x-slice, left/right for a y-slice),
//       the same cells the slice form passes as aux1/aux2/aux3(:, i-2+imp).
//
// A solver written to the reference's pointwise contract ports field for
// field.  The clawpack/riemann package is not vendored with the reference,
// so each solver here is written from the mathematics of its system; the
// CPU oracle restates the same arithmetic, operation for operation.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

#ifndef EULER_MINB
#define EULER_MINB 2
#endif

namespace clawb200 {

// ------------------------------------------------------------------------
// 2D linear acoustics, q = (p, u, v), constant rho and bulk modulus K.
// Waves: jump = a1*(-Z, 1, 0) + a2*(Z, 1, 0) in (p, u_normal, u_transverse),
// speeds -c and +c, with c = sqrt(K/rho), Z = rho*c, hz = 1/(2Z).
template <typename real_>
struct Acoustics2D {
    using real = real_;
    static constexpr int meqn = 3, mwaves = 2, maux = 0;
    real cc, zz, hz;

    // Structurally zero components (the kernels skip arithmetic on them; the
    // skipped terms are exact zeros, so results are value-identical):
    // waves and fluctuations of an ixy-slice carry no transverse velocity,
    // transverse splits carry no normal velocity.
    __host__ __device__ static constexpr bool wave_zero(int ixy, int m) { return m == (ixy == 1 ? 2 : 1); }
    __host__ __device__ static constexpr bool trans_zero(int ixy, int m) { return m == (ixy == 1 ? 1 : 2); }

    __device__ __forceinline__ void rpn(int ixy, const real* qL, const real* qR, const real*,
                                        const real*, real wave[mwaves][meqn], real s[mwaves],
                                        real amdq[meqn], real apdq[meqn]) const {
        const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
        const real dp = qR[0] - qL[0];
        const real du = qR[mu] - qL[mu];
        const real a1 = (zz * du - dp) * hz;
        const real a2 = (zz * du + dp) * hz;
        wave[0][0] = -(a1 * zz); wave[0][mu] = a1; wave[0][mv] = real(0);
        wave[1][0] = a2 * zz;    wave[1][mu] = a2; wave[1][mv] = real(0);
        s[0] = -cc;
        s[1] = cc;
        amdq[0] = cc * (a1 * zz); amdq[mu] = -(cc * a1); amdq[mv] = real(0);
        apdq[0] = cc * (a2 * zz); apdq[mu] = cc * a2;    apdq[mv] = real(0);
    }

    __device__ __forceinline__ void rpt(int ixy, int, const real*, const real*, const real*,
                                        const real*, const real*, const real* asdq,
                                        real bmasdq[meqn], real bpasdq[meqn]) const {
        const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
        const real b1 = (zz * asdq[mv] - asdq[0]) * hz;
        const real b2 = (zz * asdq[mv] + asdq[0]) * hz;
        bmasdq[0] = cc * (b1 * zz); bmasdq[mu] = real(0); bmasdq[mv] = -(cc * b1);
        bpasdq[0] = cc * (b2 * zz); bpasdq[mu] = real(0); bpasdq[mv] = cc * b2;
    }
};

// ------------------------------------------------------------------------
// 2D Euler equations, q = (rho, rho u, rho v, E), gamma-law gas.  Roe solver
// with three waves (u-a; the entropy and shear wave at u; u+a) and the
// Harten-Hyman entropy fix on transonic rarefactions in A^- dq (A^+ dq = the
// total flux difference minus A^- dq); the transverse split uses the
// eigenvectors of the transverse Jacobian at the same interface's Roe average.
// (LeVeque, Finite Volume Methods for Hyperbolic Problems, 15.3 and 18.8;
// Harten & Hyman, J. Comput. Phys. 50, 1983.)
// FAST (the contracted build): Newton reciprocals and square roots instead
// of IEEE division and sqrt (to about an ulp), compare-and-select instead of
// fmin/fmax.
template <typename real_, bool FAST = false>
struct EulerRoe2D {
    using real = real_;
    static constexpr int meqn = 4, mwaves = 3, maux = 0;
    static constexpr int min_blocks = EULER_MINB;  // registers for the Roe state
    real gamma, gamma1;
    using AR = Arith<FAST>;
    __device__ __forceinline__ static real min0(real x) {
        if constexpr (FAST) return x < real(0) ? x : real(0);
        else return fmin(x, real(0));
    }
    __device__ __forceinline__ static real max0(real x) {
        if constexpr (FAST) return x > real(0) ? x : real(0);
        else return fmax(x, real(0));
    }
    __host__ __device__ static constexpr bool wave_zero(int, int) { return false; }
    __host__ __device__ static constexpr bool trans_zero(int, int) { return false; }

    struct Roe { real u, v, enth, a, g1a2, euv, hu, ha; };  // ha = 1/(2a)

    // Interface context: the Roe average of (qL, qR) that rpn and both rpt
    // calls of one interface share (computed once; the same values).
    struct Ctx { real u, v, enth, a, g1a2, ha; };
    __device__ __forceinline__ Ctx context(int ixy, const real* qL, const real* qR) const {
        const int mu = ixy == 1 ? 1 : 2, mv = ixy == 1 ? 2 : 1;
        const Roe r = average(qL, qR, mu, mv);
        return Ctx{r.u, r.v, r.enth, r.a, r.g1a2, r.ha};
    }
    __device__ __forceinline__ static Roe expand(const Ctx& c) {
        Roe r;
        r.u = c.u; r.v = c.v; r.enth = c.enth; r.a = c.a; r.g1a2 = c.g1a2; r.ha = c.ha;
        const real u2v2 = r.u * r.u + r.v * r.v;
        r.euv = r.enth - u2v2;
        r.hu = real(0.5) * u2v2;
        return r;
    }

    // One reciprocal per square root and per sum (divisions are this solver's
    // costly operations); 1/rho = (1/sqrt(rho))^2.
    __device__ __forceinline__ Roe average(const real* qL, const real* qR, int mu, int mv) const {
        const real rhsqrtl = AR::root(qL[0]);
        const real rhsqrtr = AR::root(qR[0]);
        const real il = AR::rcp(rhsqrtl);
        const real ir = AR::rcp(rhsqrtr);
        const real pl = gamma1 * (qL[3] - real(0.5) * (qL[mu] * qL[mu] + qL[mv] * qL[mv]) * (il * il));
        const real pr = gamma1 * (qR[3] - real(0.5) * (qR[mu] * qR[mu] + qR[mv] * qR[mv]) * (ir * ir));
        const real i2 = AR::rcp(rhsqrtl + rhsqrtr);
        Roe r;
        r.u = (qL[mu] * il + qR[mu] * ir) * i2;
        r.v = (qL[mv] * il + qR[mv] * ir) * i2;
        r.enth = ((qL[3] + pl) * il + (qR[3] + pr) * ir) * i2;
        const real u2v2 = r.u * r.u + r.v * r.v;
        const real a2 = gamma1 * (r.enth - real(0.5) * u2v2);
        r.a = AR::root(a2);
        r.g1a2 = AR::div(gamma1, a2);
        r.ha = AR::div(real(0.5), r.a);
        r.euv = r.enth - u2v2;
        r.hu = real(0.5) * u2v2;
        return r;
    }

    // normal velocity and sound speed of a conserved state (one division)
    __device__ __forceinline__ void state(const real* q, int mu, int mv, real& un, real& c) const {
        const real ri = AR::rcp(q[0]);
        const real p = gamma1 * (q[3] - real(0.5) * (q[mu] * q[mu] + q[mv] * q[mv]) * ri);
        c = AR::root(gamma * p * ri);
        un = q[mu] * ri;
    }

    __device__ __forceinline__ void rpn(int ixy, const real* qL, const real* qR, const real*,
                                        const real*, real w[mwaves][meqn], real s[mwaves],
                                        real amdq[meqn], real apdq[meqn]) const {
        rpn_ctx(ixy, context(ixy, qL, qR), qL, qR, w, s, amdq, apdq);
    }

    __device__ __forceinline__ void rpn_ctx(int ixy, const Ctx& c, const real* qL, const real* qR,
                                            real w[mwaves][meqn], real s[mwaves], real amdq[meqn],
                                            real apdq[meqn]) const {
        const int mu = ixy == 1 ? 1 : 2, mv = ixy == 1 ? 2 : 1;
        const Roe r = expand(c);
        real d[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) d[m] = qR[m] - qL[m];
        const real a3 = r.g1a2 * (r.euv * d[0] + r.u * d[mu] + r.v * d[mv] - d[3]);
        const real a2 = d[mv] - r.v * d[0];
        const real a4 = (d[mu] + (r.a - r.u) * d[0] - r.a * a3) * r.ha;
        const real a1 = d[0] - a3 - a4;
        w[0][0] = a1; w[0][mu] = a1 * (r.u - r.a); w[0][mv] = a1 * r.v; w[0][3] = a1 * (r.enth - r.u * r.a);
        s[0] = r.u - r.a;
        w[1][0] = a3; w[1][mu] = a3 * r.u; w[1][mv] = a3 * r.v + a2; w[1][3] = a3 * r.hu + a2 * r.v;
        s[1] = r.u;
        w[2][0] = a4; w[2][mu] = a4 * (r.u + r.a); w[2][mv] = a4 * r.v; w[2][3] = a4 * (r.enth + r.u * r.a);
        s[2] = r.u + r.a;
#pragma unroll
        for (int m = 0; m < 4; ++m) amdq[m] = real(0);
        real ul, cl;
        state(qL, mu, mv, ul, cl);
        const real s0 = ul - cl;
        real q1[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) q1[m] = qL[m] + w[0][m];
        real u1, c1;
        state(q1, mu, mv, u1, c1);
        const real s1 = u1 - c1;
        if (!(s0 >= real(0) && s[0] > real(0))) {
            real sfract;
            if (s0 < real(0) && s1 > real(0)) sfract = AR::div(s0 * (s1 - s[0]), s1 - s0);
            else if (s[0] < real(0)) sfract = s[0];
            else sfract = real(0);
#pragma unroll
            for (int m = 0; m < 4; ++m) amdq[m] = sfract * w[0][m];
            if (s[1] < real(0)) {
#pragma unroll
                for (int m = 0; m < 4; ++m) amdq[m] = amdq[m] + s[1] * w[1][m];
                real ur, cr;
                state(qR, mu, mv, ur, cr);
                const real s3 = ur + cr;
                real q2[4];
#pragma unroll
                for (int m = 0; m < 4; ++m) q2[m] = qR[m] - w[2][m];
                real u2, c2;
                state(q2, mu, mv, u2, c2);
                const real s2 = u2 + c2;
                real sf3;
                if (s2 < real(0) && s3 > real(0)) sf3 = AR::div(s2 * (s3 - s[2]), s3 - s2);
                else if (s[2] < real(0)) sf3 = s[2];
                else sf3 = real(0);
#pragma unroll
                for (int m = 0; m < 4; ++m) amdq[m] = amdq[m] + sf3 * w[2][m];
            }
        }
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const real df = (s[0] * w[0][m] + s[1] * w[1][m]) + s[2] * w[2][m];
            apdq[m] = df - amdq[m];
        }
    }

    __device__ __forceinline__ void rpt(int ixy, int imp, const real* qL, const real* qR, const real*,
                                        const real*, const real*, const real* asdq,
                                        real bm[meqn], real bp[meqn]) const {
        rpt_ctx(ixy, imp, context(ixy, qL, qR), asdq, bm, bp);
    }

    __device__ __forceinline__ void rpt_ctx(int ixy, int, const Ctx& c, const real* asdq,
                                            real bm[meqn], real bp[meqn]) const {
        const int mu = ixy == 1 ? 1 : 2, mv = ixy == 1 ? 2 : 1;
        const Roe r = expand(c);
        const real a3 = r.g1a2 * (r.euv * asdq[0] + r.u * asdq[mu] + r.v * asdq[mv] - asdq[3]);
        const real a2 = asdq[mu] - r.u * asdq[0];
        const real a4 = (asdq[mv] + (r.a - r.v) * asdq[0] - r.a * a3) * r.ha;
        const real a1 = asdq[0] - a3 - a4;
        real w[3][4], sb[3];
        w[0][0] = a1; w[0][mu] = a1 * r.u; w[0][mv] = a1 * (r.v - r.a); w[0][3] = a1 * (r.enth - r.v * r.a);
        sb[0] = r.v - r.a;
        w[1][0] = a3; w[1][mu] = a3 * r.u + a2; w[1][mv] = a3 * r.v; w[1][3] = a3 * r.hu + a2 * r.u;
        sb[1] = r.v;
        w[2][0] = a4; w[2][mu] = a4 * r.u; w[2][mv] = a4 * (r.v + r.a); w[2][3] = a4 * (r.enth + r.v * r.a);
        sb[2] = r.v + r.a;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            bm[m] = (min0(sb[0]) * w[0][m] + min0(sb[1]) * w[1][m]) + min0(sb[2]) * w[2][m];
            bp[m] = (max0(sb[0]) * w[0][m] + max0(sb[1]) * w[1][m]) + max0(sb[2]) * w[2][m];
        }
    }
};

// ------------------------------------------------------------------------
// 2D advection with edge velocities (annulus example layout):
// aux = (u at the left edge of the cell, v at its bottom edge, capacity).
template <typename real_>
struct VCAdvection2D {
    using real = real_;
    static constexpr int meqn = 1, mwaves = 1, maux = 3;
    __host__ __device__ static constexpr bool wave_zero(int, int) { return false; }
    __host__ __device__ static constexpr bool trans_zero(int, int) { return false; }

    __device__ __forceinline__ void rpn(int ixy, const real* qL, const real* qR, const real*,
                                        const real* auxR, real wave[mwaves][meqn], real s[mwaves],
                                        real amdq[meqn], real apdq[meqn]) const {
        const real w = qR[0] - qL[0];
        const real si = auxR[ixy - 1];
        wave[0][0] = w;
        s[0] = si;
        amdq[0] = fmin(si, real(0)) * w;
        apdq[0] = fmax(si, real(0)) * w;
    }

    __device__ __forceinline__ void rpt(int ixy, int, const real*, const real*, const real*,
                                        const real* aux2, const real* aux3, const real* asdq,
                                        real bmasdq[meqn], real bpasdq[meqn]) const {
        const int it = 2 - ixy;  // transverse velocity component (0-based)
        bmasdq[0] = fmin(aux2[it], real(0)) * asdq[0];
        bpasdq[0] = fmax(aux3[it], real(0)) * asdq[0];
    }
};

}  // namespace clawb200

namespace clawb200 {

// ------------------------------------------------------------------------
// 1D linear acoustics, q = (p, u): the x-part of Acoustics2D.
template <typename real_>
struct Acoustics1D {
    using real = real_;
    static constexpr int meqn = 2, mwaves = 2, maux = 0;
    real cc, zz, hz;

    __device__ __forceinline__ void rp1(const real* qL, const real* qR, const real*, const real*,
                                        real wave[mwaves][meqn], real s[mwaves], real amdq[meqn],
                                        real apdq[meqn]) const {
        const real dp = qR[0] - qL[0];
        const real du = qR[1] - qL[1];
        const real a1 = (zz * du - dp) * hz;
        const real a2 = (zz * du + dp) * hz;
        wave[0][0] = -(a1 * zz); wave[0][1] = a1;
        wave[1][0] = a2 * zz;    wave[1][1] = a2;
        s[0] = -cc;
        s[1] = cc;
        amdq[0] = cc * (a1 * zz); amdq[1] = -(cc * a1);
        apdq[0] = cc * (a2 * zz); apdq[1] = cc * a2;
    }
};

// 1D advection q_t + u q_x = 0 with constant u (examples/advection_1d_example1,
// the rp1_advection plugin of clawpack/riemann, restated): one wave, the jump,
// with speed u; A-dq = min(u, 0) dq, A+dq = max(u, 0) dq.
template <typename real_>
struct Advection1D {
    using real = real_;
    static constexpr int meqn = 1, mwaves = 1, maux = 0;
    real u;

    __device__ __forceinline__ void rp1(const real* qL, const real* qR, const real*, const real*,
                                        real wave[mwaves][meqn], real s[mwaves], real amdq[meqn],
                                        real apdq[meqn]) const {
        const real d = qR[0] - qL[0];
        wave[0][0] = d;
        s[0] = u;
        amdq[0] = fmin(u, real(0)) * d;
        apdq[0] = fmax(u, real(0)) * d;
    }
};

// 1D Euler, q = (rho, rho u, E), gamma-law gas (examples/euler_1d_wcblast, the
// rp1_euler_with_efix plugin of clawpack/riemann): Roe averages, three waves
// (u-a, u, u+a), A-dq with the Harten-Hyman entropy fix in the 1- and 3-waves
// and A+dq = sum s w - A-dq; one reciprocal per square root and per sum, as
// in the 2D solver above.
template <typename real_>
struct EulerRoe1D {
    using real = real_;
    static constexpr int meqn = 3, mwaves = 3, maux = 0;
    real gamma, gamma1;

    // velocity and sound speed of a conserved state (one division)
    __device__ __forceinline__ void state(const real* q, real& u, real& c) const {
        const real ri = real(1) / q[0];
        const real p = gamma1 * (q[2] - real(0.5) * (q[1] * q[1]) * ri);
        c = sqrt(gamma * p * ri);
        u = q[1] * ri;
    }

    __device__ __forceinline__ void rp1(const real* qL, const real* qR, const real*, const real*,
                                        real w[mwaves][meqn], real s[mwaves], real amdq[meqn],
                                        real apdq[meqn]) const {
        const real rhsqrtl = sqrt(qL[0]);
        const real rhsqrtr = sqrt(qR[0]);
        const real il = real(1) / rhsqrtl;
        const real ir = real(1) / rhsqrtr;
        const real pl = gamma1 * (qL[2] - real(0.5) * (qL[1] * qL[1]) * (il * il));
        const real pr = gamma1 * (qR[2] - real(0.5) * (qR[1] * qR[1]) * (ir * ir));
        const real i2 = real(1) / (rhsqrtl + rhsqrtr);
        const real u = (qL[1] * il + qR[1] * ir) * i2;
        const real enth = ((qL[2] + pl) * il + (qR[2] + pr) * ir) * i2;
        const real u2 = u * u;
        const real a2 = gamma1 * (enth - real(0.5) * u2);
        const real a = sqrt(a2);
        const real g1a2 = gamma1 / a2;
        const real ha = real(0.5) / a;
        real d[3];
#pragma unroll
        for (int m = 0; m < 3; ++m) d[m] = qR[m] - qL[m];
        const real b2 = g1a2 * ((enth - u2) * d[0] + u * d[1] - d[2]);
        const real b3 = (d[1] + (a - u) * d[0] - a * b2) * ha;
        const real b1 = d[0] - b2 - b3;
        w[0][0] = b1; w[0][1] = b1 * (u - a); w[0][2] = b1 * (enth - u * a);
        s[0] = u - a;
        w[1][0] = b2; w[1][1] = b2 * u;       w[1][2] = b2 * (real(0.5) * u2);
        s[1] = u;
        w[2][0] = b3; w[2][1] = b3 * (u + a); w[2][2] = b3 * (enth + u * a);
        s[2] = u + a;
#pragma unroll
        for (int m = 0; m < 3; ++m) amdq[m] = real(0);
        real ul, cl;
        state(qL, ul, cl);
        const real s0 = ul - cl;
        real q1[3];
#pragma unroll
        for (int m = 0; m < 3; ++m) q1[m] = qL[m] + w[0][m];
        real u1, c1;
        state(q1, u1, c1);
        const real s1 = u1 - c1;
        if (!(s0 >= real(0) && s[0] > real(0))) {
            real sfract;
            if (s0 < real(0) && s1 > real(0)) sfract = s0 * (s1 - s[0]) / (s1 - s0);
            else if (s[0] < real(0)) sfract = s[0];
            else sfract = real(0);
#pragma unroll
            for (int m = 0; m < 3; ++m) amdq[m] = sfract * w[0][m];
            if (s[1] < real(0)) {
#pragma unroll
                for (int m = 0; m < 3; ++m) amdq[m] = amdq[m] + s[1] * w[1][m];
                real ur, cr;
                state(qR, ur, cr);
                const real s3 = ur + cr;
                real q2[3];
#pragma unroll
                for (int m = 0; m < 3; ++m) q2[m] = qR[m] - w[2][m];
                real u2s, c2;
                state(q2, u2s, c2);
                const real s2 = u2s + c2;
                real sf3;
                if (s2 < real(0) && s3 > real(0)) sf3 = s2 * (s3 - s[2]) / (s3 - s2);
                else if (s[2] < real(0)) sf3 = s[2];
                else sf3 = real(0);
#pragma unroll
                for (int m = 0; m < 3; ++m) amdq[m] = amdq[m] + sf3 * w[2][m];
            }
        }
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            const real df = (s[0] * w[0][m] + s[1] * w[1][m]) + s[2] * w[2][m];
            apdq[m] = df - amdq[m];
        }
    }
};

// 1D variable-coefficient acoustics, aux = (Z, c) per cell: the left-going
// wave lies on the eigenvector of the left cell, the right-going on the
// right cell's: jump = a1*(-Z_l, 1) + a2*(Z_r, 1), speeds -c_l, +c_r.
template <typename real_>
struct VCAcoustics1D {
    using real = real_;
    static constexpr int meqn = 2, mwaves = 2, maux = 2;

    __device__ __forceinline__ void rp1(const real* qL, const real* qR, const real* auxL,
                                        const real* auxR, real wave[mwaves][meqn], real s[mwaves],
                                        real amdq[meqn], real apdq[meqn]) const {
        const real zl = auxL[0], cl = auxL[1], zr = auxR[0], cr = auxR[1];
        const real dp = qR[0] - qL[0];
        const real du = qR[1] - qL[1];
        const real a1 = (zr * du - dp) / (zl + zr);
        const real a2 = (zl * du + dp) / (zl + zr);
        wave[0][0] = -(a1 * zl); wave[0][1] = a1;
        wave[1][0] = a2 * zr;    wave[1][1] = a2;
        s[0] = -cl;
        s[1] = cr;
        amdq[0] = cl * (a1 * zl); amdq[1] = -(cl * a1);
        apdq[0] = cr * (a2 * zr); apdq[1] = cr * a2;
    }
};


// Variable-coefficient 3D acoustics, q = (p, u, v, w), aux = (Z, c) per cell:
// the rpn3 / rpt3 / rptt3 plugins of examples/acoustics_3d_heterogeneous
// (clawpack/riemann rp{n,t,tt}3_vc_acoustics) in pointwise, compact form.
// Every fluctuation of this system has two non-zero components: the pressure
// and the velocity along the direction of its last split, so the solver
// works on (p, velocity) pairs and the step kernel places them.
template <typename real_>
struct VCAcoustics3D {
    using real = real_;
    static constexpr int meqn = 4, mwaves = 2, maux = 2;

    // Normal solve at one interface: jump (dp, dun) between cells with
    // impedance / sound speed (zl, cl) | (zr, cr).  w[k] = (p, un) of wave k.
    __device__ __forceinline__ static void rpn(real pL, real uL, real pR, real uR, real zl,
                                               real cl, real zr, real cr, real w[2][2],
                                               real s[2], real am[2], real ap[2]) {
        const real dp = pR - pL;
        const real du = uR - uL;
        const real a1 = (zr * du - dp) / (zl + zr);
        const real a2 = (zl * du + dp) / (zl + zr);
        w[0][0] = -(a1 * zl); w[0][1] = a1;
        w[1][0] = a2 * zr;    w[1][1] = a2;
        s[0] = -cl;
        s[1] = cr;
        am[0] = cl * (a1 * zl); am[1] = -(cl * a1);
        ap[0] = cr * (a2 * zr); ap[1] = cr * a2;
    }

    // Transverse split of a fluctuation whose pressure part is xp (its
    // velocity along the split direction is structurally zero) living in a
    // cell of impedance zm, between the neighbours below (zb, cb) and above
    // (za, ca): down = c_b (b1 Z_b, -b1), up = c_a (b2 Z_a, b2) with
    // b1 = -xp / (Z_b + Z_m), b2 = xp / (Z_m + Z_a).  rpt3 and rptt3 differ
    // only in which cells' coefficients they pass.
    struct Split { real dp, dt, up, ut; };
    __device__ __forceinline__ static Split split(real xp, real zb, real cb, real zm, real za,
                                                  real ca) {
        const real b1 = -xp / (zb + zm);
        const real b2 = xp / (zm + za);
        const real c1 = cb * b1, c2 = ca * b2;
        return Split{c1 * zb, -c1, c2 * za, c2};
    }
    // The same split given the face reciprocals rb = 1 / (Z_b + Z_m) and
    // ra = 1 / (Z_m + Z_a): multiplications only (the contracted and FP32
    // builds; the quotients round differently from the divisions above).
    __device__ __forceinline__ static Split split_r(real xp, real rb, real zb, real cb, real ra,
                                                    real za, real ca) {
        const real b1 = -(xp * rb);
        const real b2 = xp * ra;
        const real c1 = cb * b1, c2 = ca * b2;
        return Split{c1 * zb, -c1, c2 * za, c2};
    }
    // rpn with one reciprocal of the impedance sum instead of two divisions
    __device__ __forceinline__ static void rpn_r(real pL, real uL, real pR, real uR, real zl,
                                                 real cl, real zr, real cr, real w[2][2],
                                                 real s[2], real am[2], real ap[2]) {
        const real dp = pR - pL;
        const real du = uR - uL;
        const real r = real(1) / (zl + zr);
        const real a1 = (zr * du - dp) * r;
        const real a2 = (zl * du + dp) * r;
        w[0][0] = -(a1 * zl); w[0][1] = a1;
        w[1][0] = a2 * zr;    w[1][1] = a2;
        s[0] = -cl;
        s[1] = cr;
        am[0] = cl * (a1 * zl); am[1] = -(cl * a1);
        ap[0] = cr * (a2 * zr); ap[1] = cr * a2;
    }
};

}  // namespace clawb200
