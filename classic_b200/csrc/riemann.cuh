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
};

}  // namespace clawb200
