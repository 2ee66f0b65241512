// ============================================================================
// ORACLE — test infrastructure only.  CPU restatement of Clawpack Classic's
// wave-propagation step, used by tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py as the checker.  Nothing in
// the product (classic_b200/) links, imports or calls this file.
//
// It restates, loop for loop and in the same floating-point evaluation order,
// the reference Fortran routines (paths relative to clawpack/classic):
//   limiter  : src/2d/inlinelimiter.f90:25-105   (identical copies in 1d/, 3d/)
//   flux2    : src/2d/flux2.f90:5-235
//   step2    : src/2d/step2.f90:2-251
//   bc2      : src/2d/bc2.f:4-215
//   claw2    : src/2d/claw2.f:494-784            (dt / CFL control loop)
//   dimsp2   : src/2d/dimsp2.f, src/2d/step2ds.f90 (dimensional splitting)
//   step1    : src/1d/step1.f90:4-170
//   bc1      : src/1d/bc1.f
//   claw1    : src/1d/claw1.f:394-583
//   step3    : src/3d/step3.f90:3-873 (serial colour-block order)
//   flux3    : src/3d/flux3.f90:4-612
//   bc3      : src/3d/bc3.f (+ the piston BC of examples/acoustics_3d_heterogeneous/bc3.f)
//   claw3    : src/3d/claw3.f:738-928
//   dimsp3   : src/3d/dimsp3.f, src/3d/step3ds.f90 (dimensional splitting)
// Pins (tests/test_oracle_golden.py): the 3D regression sums are reproduced
// exactly, the 1D heterogeneous sums bit for bit, the 1D example to 1e-16.
// 2D Euler (Roe + Harten-Hyman entropy fix): parity unpinned -- the reference
// ships no 2D Euler solver, example or regression data; the restatement is
// checked by conservation and shock-tube properties (tests/test_oracle_euler.py).
// Arrays use the reference's Fortran layout: q(meqn, 1-mbc:mx+mbc, ...) with
// the equation index fastest.  Compile with -ffp-contract=off so every
// multiply and add rounds separately, as the GPU parity build does.
//
// The Riemann solvers live in the un-vendored clawpack/riemann package (the
// reference's regression data were recorded at riemann commit 48a46d3).  The
// solvers below are written from the mathematics of each system (eigen-
// decomposition of the acoustics and advection Jacobians) in the slice
// contract documented at src/2d/claw2.f:312-404 and src/1d/claw1.f; the
// exact arithmetic of each solver is fixed here and restated identically in
// the CUDA plugins, so oracle and GPU can be compared bit for bit.
// ============================================================================
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>
#include <algorithm>
#include <atomic>
#include <thread>

extern "C" {

// ---------------------------------------------------------------- solvers ---
// Solver ids (shared numbering with the product's C-ABI, include/claw_b200.h).
enum {
    ORC_ACOUSTICS_2D = 1,      // q = (p, u, v);  params: rho, bulk
    ORC_VC_ADVECTION_2D = 2,   // q = (q);  aux = (u at left edge, v at bottom edge, capa)
    ORC_EULER_ROE_2D = 3,      // q = (rho, rho u, rho v, E);  params: gamma
    ORC_ACOUSTICS_1D = 11,     // q = (p, u);  params: rho, bulk
    ORC_VC_ACOUSTICS_1D = 12,  // q = (p, u);  aux = (Z, c)
    ORC_ADVECTION_1D = 13,     // q = (q);  params: u
    ORC_EULER_ROE_1D = 14,     // q = (rho, rho u, E);  params: gamma
    ORC_VC_ACOUSTICS_3D = 21,  // q = (p, u, v, w);  aux = (Z, c)
};

// Problem parameters: the analogue of the reference's /cparam/ common block
// (non-reentrant, exactly like the reference).
static int g_solver = 0;
static double g_rho = 1.0, g_bulk = 1.0, g_cc = 1.0, g_zz = 1.0, g_hz = 0.5;
static double g_gamma = 1.4;
static double g_u = 1.0;  // 1D advection velocity

// Source term (the example's src1 / src2; 0 = the reference's default no-op).
// 1: examples/acoustics_2d_radial/1drad/src1.f:18-23, radial symmetry with x
// as the radius; bulk is the solver's (the shared /cparam/ block).
static int g_src = 0, g_src_ndim = 2;
static double g_src_xlower = 0.0;

int orc_set_source(int id, int ndim, double xlower) {
    g_src = id;
    g_src_ndim = ndim;
    g_src_xlower = xlower;
    return 0;
}

// Before-step routine (the example's b4step2; 0 = the reference's default
// no-op).  1: the edge velocities (aux fields 1, 2) of the variable-velocity
// advection solver scaled by cos(pi t / T), from an unscaled copy.
// Host threads of the timing variant (orc_set_threads); 1 runs the serial
// loops, which is the order every parity test compares against.
static int g_threads = 1;

int orc_set_threads(int n) {
    g_threads = n < 1 ? 1 : n;
    return g_threads;
}

static int g_b4 = 0;
static double g_b4_period = 1.0;

int orc_set_b4step(int id, double period) {
    g_b4 = id;
    g_b4_period = period;
    return 0;
}

// b4step2 at time t: aux_out = aux_base with the velocity fields scaled
// (aux in the reference layout aux(maux, cells)); a no-op copy for id 0.
int orc_b4step2(int maux, long long ncells, const double* aux_base, double* aux_out, double t) {
    const double sc = std::cos(3.141592653589793 * t / g_b4_period);
    for (long long k = 0; k < ncells; ++k)
        for (int ma = 0; ma < maux; ++ma) {
            const double v = aux_base[ma + (long long)maux * k];
            aux_out[ma + (long long)maux * k] = (g_b4 == 1 && ma < 2) ? v * sc : v;
        }
    return 0;
}

int orc_set_solver(int solver_id, const double* params, int nparams) {
    g_solver = solver_id;
    if (solver_id == ORC_ACOUSTICS_2D || solver_id == ORC_ACOUSTICS_1D) {
        if (nparams < 2) return -1;
        g_rho = params[0];
        g_bulk = params[1];
        g_cc = std::sqrt(g_bulk / g_rho);
        g_zz = g_rho * g_cc;
        g_hz = 0.5 / g_zz;
    } else if (solver_id == ORC_EULER_ROE_2D || solver_id == ORC_EULER_ROE_1D) {
        if (nparams < 1) return -1;
        g_gamma = params[0];
    } else if (solver_id == ORC_ADVECTION_1D) {
        if (nparams < 1) return -1;
        g_u = params[0];
    }
    return 0;
}

}  // extern "C"

namespace {

// Slice arrays (meqn, 1-mbc:maxm+mbc) -> flat index.
struct Slice {
    int n0, lo;  // leading dimension, lowest index
    inline int at(int m, int i) const { return (m - 1) + n0 * (i - lo); }
};

typedef void (*rpn2_t)(int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                       const double* ql, const double* qr, const double* auxl,
                       const double* auxr, double* wave, double* s, double* amdq,
                       double* apdq);
typedef void (*rpt2_t)(int ixy, int imp, int maxm, int meqn, int mwaves, int maux, int mbc,
                       int mx, const double* ql, const double* qr, const double* aux1,
                       const double* aux2, const double* aux3, const double* asdq,
                       double* bmasdq, double* bpasdq);

// ---- 2D constant-coefficient acoustics (p, u, v) ----------------------------
// Normal solve: jump dq = a1*(-Z,1,0) + a2*(Z,1,0) in (p, u_n, u_t) components,
// speeds -c, +c.  Transverse solve splits asdq on the transverse eigenvectors.
void rpn2_acoustics(int ixy, int maxm, int meqn, int mwaves, int, int mbc, int mx,
                    const double* ql, const double* qr, const double*, const double*,
                    double* wave, double* s, double* amdq, double* apdq) {
    const Slice q{meqn, 1 - mbc}, w{meqn * mwaves, 1 - mbc}, sv{mwaves, 1 - mbc};
    const int mu = (ixy == 1) ? 2 : 3, mv = (ixy == 1) ? 3 : 2;
    const double cc = g_cc, zz = g_zz, hz = g_hz;
    (void)maxm;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const double dp = ql[q.at(1, i)] - qr[q.at(1, i - 1)];
        const double du = ql[q.at(mu, i)] - qr[q.at(mu, i - 1)];
        const double a1 = (zz * du - dp) * hz;
        const double a2 = (zz * du + dp) * hz;
        double* w1 = &wave[w.at(1, i)];
        double* w2 = w1 + meqn;
        w1[0] = -(a1 * zz); w1[mu - 1] = a1; w1[mv - 1] = 0.0;
        w2[0] = a2 * zz;    w2[mu - 1] = a2; w2[mv - 1] = 0.0;
        s[sv.at(1, i)] = -cc;
        s[sv.at(2, i)] = cc;
        amdq[q.at(1, i)] = cc * (a1 * zz);
        amdq[q.at(mu, i)] = -(cc * a1);
        amdq[q.at(mv, i)] = 0.0;
        apdq[q.at(1, i)] = cc * (a2 * zz);
        apdq[q.at(mu, i)] = cc * a2;
        apdq[q.at(mv, i)] = 0.0;
    }
}

void rpt2_acoustics(int ixy, int, int, int meqn, int, int, int mbc, int mx, const double*,
                    const double*, const double*, const double*, const double*,
                    const double* asdq, double* bmasdq, double* bpasdq) {
    const Slice q{meqn, 1 - mbc};
    const int mu = (ixy == 1) ? 2 : 3, mv = (ixy == 1) ? 3 : 2;
    const double cc = g_cc, zz = g_zz, hz = g_hz;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const double b1 = (zz * asdq[q.at(mv, i)] - asdq[q.at(1, i)]) * hz;
        const double b2 = (zz * asdq[q.at(mv, i)] + asdq[q.at(1, i)]) * hz;
        bmasdq[q.at(1, i)] = cc * (b1 * zz);
        bmasdq[q.at(mu, i)] = 0.0;
        bmasdq[q.at(mv, i)] = -(cc * b1);
        bpasdq[q.at(1, i)] = cc * (b2 * zz);
        bpasdq[q.at(mu, i)] = 0.0;
        bpasdq[q.at(mv, i)] = cc * b2;
    }
}

// ---- 2D variable-coefficient advection with edge velocities ------------------
// aux(1,i) = normal velocity at the left edge of cell i, aux(2,i) at its bottom
// edge (the layout of the annulus example's setaux).  Upwinding by the sign of
// the edge velocity; the transverse split uses the transverse edge velocities
// of the cell that receives the fluctuation (cell i-1 for imp=1, i for imp=2).
void rpn2_vc_advection(int ixy, int, int meqn, int, int maux, int mbc, int mx,
                       const double* ql, const double* qr, const double* auxl,
                       const double*, double* wave, double* s, double* amdq, double* apdq) {
    const Slice q{meqn, 1 - mbc}, a{maux, 1 - mbc};
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const double w = ql[q.at(1, i)] - qr[q.at(1, i - 1)];
        const double si = auxl[a.at(ixy, i)];
        wave[q.at(1, i)] = w;
        s[i - (1 - mbc)] = si;
        amdq[q.at(1, i)] = std::fmin(si, 0.0) * w;
        apdq[q.at(1, i)] = std::fmax(si, 0.0) * w;
    }
}

void rpt2_vc_advection(int ixy, int imp, int, int meqn, int, int maux, int mbc, int mx,
                       const double*, const double*, const double*, const double* aux2,
                       const double* aux3, const double* asdq, double* bmasdq,
                       double* bpasdq) {
    const Slice q{meqn, 1 - mbc}, a{maux, 1 - mbc};
    const int it = 3 - ixy;  // transverse velocity index
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const int i1 = i - 2 + imp;
        const double vlo = aux2[a.at(it, i1)];
        const double vhi = aux3[a.at(it, i1)];
        bmasdq[q.at(1, i)] = std::fmin(vlo, 0.0) * asdq[q.at(1, i)];
        bpasdq[q.at(1, i)] = std::fmax(vhi, 0.0) * asdq[q.at(1, i)];
    }
}


// ---- 2D Euler equations, Roe solver with the Harten-Hyman entropy fix -------
// q = (rho, rho u, rho v, E), p = (gamma-1)(E - (rho u^2 + rho v^2)/2 / rho).
// Roe averages of u, v and the enthalpy H = (E + p)/rho between the left and
// right states; three waves: acoustic u-a, the entropy + shear wave u, and
// acoustic u+a (LeVeque, Finite Volume Methods for Hyperbolic Problems,
// sections 15.3 and 18.8).  The entropy fix splits a transonic rarefaction
// in the 1- or 3-wave by Harten and Hyman's linear interpolation of the
// characteristic speed across the wave (Harten & Hyman, J. Comput. Phys. 50,
// 1983).  This is the pointwise arithmetic, identical to the device functor.
struct RoeAvg {
    double u, v, enth, a, g1a2, euv, hu, ha;  // ha = 1/(2a)
};

inline RoeAvg roe_average(const double* qL, const double* qR, int mu, int mv) {
    // one reciprocal per square root and per sum (divisions are the costly
    // operations of this solver); 1/rho = (1/sqrt(rho))^2
    const double g1 = g_gamma - 1.0;
    const double rhsqrtl = std::sqrt(qL[0]);
    const double rhsqrtr = std::sqrt(qR[0]);
    const double il = 1.0 / rhsqrtl;
    const double ir = 1.0 / rhsqrtr;
    const double pl = g1 * (qL[3] - 0.5 * (qL[mu] * qL[mu] + qL[mv] * qL[mv]) * (il * il));
    const double pr = g1 * (qR[3] - 0.5 * (qR[mu] * qR[mu] + qR[mv] * qR[mv]) * (ir * ir));
    const double i2 = 1.0 / (rhsqrtl + rhsqrtr);
    RoeAvg r;
    r.u = (qL[mu] * il + qR[mu] * ir) * i2;
    r.v = (qL[mv] * il + qR[mv] * ir) * i2;
    r.enth = ((qL[3] + pl) * il + (qR[3] + pr) * ir) * i2;
    const double u2v2 = r.u * r.u + r.v * r.v;
    const double a2 = g1 * (r.enth - 0.5 * u2v2);
    r.a = std::sqrt(a2);
    r.g1a2 = g1 / a2;
    r.ha = 0.5 / r.a;
    r.euv = r.enth - u2v2;
    r.hu = 0.5 * u2v2;
    return r;
}

// sound speed and normal velocity of a conserved state (one division)
inline void euler_state(const double* q, int mu, int mv, double* un, double* c) {
    const double g1 = g_gamma - 1.0;
    const double ri = 1.0 / q[0];
    const double p = g1 * (q[3] - 0.5 * (q[mu] * q[mu] + q[mv] * q[mv]) * ri);
    *c = std::sqrt(g_gamma * p * ri);
    *un = q[mu] * ri;
}

// pointwise normal solve: qL = q(i-1), qR = q(i); mu/mv 0-based
void euler_rpn(const double* qL, const double* qR, int mu, int mv, double w[3][4],
               double s[3], double* amdq, double* apdq) {
    const RoeAvg r = roe_average(qL, qR, mu, mv);
    double d[4];
    for (int m = 0; m < 4; ++m) d[m] = qR[m] - qL[m];
    const double a3 = r.g1a2 * (r.euv * d[0] + r.u * d[mu] + r.v * d[mv] - d[3]);
    const double a2 = d[mv] - r.v * d[0];
    const double a4 = (d[mu] + (r.a - r.u) * d[0] - r.a * a3) * r.ha;
    const double a1 = d[0] - a3 - a4;
    w[0][0] = a1;
    w[0][mu] = a1 * (r.u - r.a);
    w[0][mv] = a1 * r.v;
    w[0][3] = a1 * (r.enth - r.u * r.a);
    s[0] = r.u - r.a;
    w[1][0] = a3;
    w[1][mu] = a3 * r.u;
    w[1][mv] = a3 * r.v + a2;
    w[1][3] = a3 * r.hu + a2 * r.v;
    s[1] = r.u;
    w[2][0] = a4;
    w[2][mu] = a4 * (r.u + r.a);
    w[2][mv] = a4 * r.v;
    w[2][3] = a4 * (r.enth + r.u * r.a);
    s[2] = r.u + r.a;
    // A^- dq with the entropy fix; A^+ dq = sum s w - A^- dq
    for (int m = 0; m < 4; ++m) amdq[m] = 0.0;
    double ul, cl;
    euler_state(qL, mu, mv, &ul, &cl);
    const double s0 = ul - cl;  // u - c left of the 1-wave
    double q1[4];
    for (int m = 0; m < 4; ++m) q1[m] = qL[m] + w[0][m];
    double u1, c1;
    euler_state(q1, mu, mv, &u1, &c1);
    const double s1 = u1 - c1;  // u - c right of the 1-wave
    if (!(s0 >= 0.0 && s[0] > 0.0)) {
        double sfract;
        if (s0 < 0.0 && s1 > 0.0) sfract = s0 * (s1 - s[0]) / (s1 - s0);
        else if (s[0] < 0.0) sfract = s[0];
        else sfract = 0.0;
        for (int m = 0; m < 4; ++m) amdq[m] = sfract * w[0][m];
        if (s[1] < 0.0) {
            for (int m = 0; m < 4; ++m) amdq[m] = amdq[m] + s[1] * w[1][m];
            double ur, cr;
            euler_state(qR, mu, mv, &ur, &cr);
            const double s3 = ur + cr;  // u + c right of the 3-wave
            double q2[4];
            for (int m = 0; m < 4; ++m) q2[m] = qR[m] - w[2][m];
            double u2, c2;
            euler_state(q2, mu, mv, &u2, &c2);
            const double s2 = u2 + c2;  // u + c left of the 3-wave
            double sf3;
            if (s2 < 0.0 && s3 > 0.0) sf3 = s2 * (s3 - s[2]) / (s3 - s2);
            else if (s[2] < 0.0) sf3 = s[2];
            else sf3 = 0.0;
            for (int m = 0; m < 4; ++m) amdq[m] = amdq[m] + sf3 * w[2][m];
        }
    }
    for (int m = 0; m < 4; ++m) {
        const double df = (s[0] * w[0][m] + s[1] * w[1][m]) + s[2] * w[2][m];
        apdq[m] = df - amdq[m];
    }
}

// pointwise transverse split of asdq on the eigenvectors of the transverse
// flux Jacobian at the Roe average of the interface's two states
void euler_rpt(const double* qL, const double* qR, int mu, int mv, const double* asdq,
               double* bm, double* bp) {
    const RoeAvg r = roe_average(qL, qR, mu, mv);
    const double a3 = r.g1a2 * (r.euv * asdq[0] + r.u * asdq[mu] + r.v * asdq[mv] - asdq[3]);
    const double a2 = asdq[mu] - r.u * asdq[0];
    const double a4 = (asdq[mv] + (r.a - r.v) * asdq[0] - r.a * a3) * r.ha;
    const double a1 = asdq[0] - a3 - a4;
    double w[3][4], sb[3];
    w[0][0] = a1; w[0][mu] = a1 * r.u; w[0][mv] = a1 * (r.v - r.a); w[0][3] = a1 * (r.enth - r.v * r.a);
    sb[0] = r.v - r.a;
    w[1][0] = a3; w[1][mu] = a3 * r.u + a2; w[1][mv] = a3 * r.v; w[1][3] = a3 * r.hu + a2 * r.u;
    sb[1] = r.v;
    w[2][0] = a4; w[2][mu] = a4 * r.u; w[2][mv] = a4 * (r.v + r.a); w[2][3] = a4 * (r.enth + r.v * r.a);
    sb[2] = r.v + r.a;
    for (int m = 0; m < 4; ++m) {
        bm[m] = (std::fmin(sb[0], 0.0) * w[0][m] + std::fmin(sb[1], 0.0) * w[1][m]) +
                std::fmin(sb[2], 0.0) * w[2][m];
        bp[m] = (std::fmax(sb[0], 0.0) * w[0][m] + std::fmax(sb[1], 0.0) * w[1][m]) +
                std::fmax(sb[2], 0.0) * w[2][m];
    }
}

void rpn2_euler_roe(int ixy, int, int meqn, int mwaves, int, int mbc, int mx, const double* ql,
                    const double* qr, const double*, const double*, double* wave, double* s,
                    double* amdq, double* apdq) {
    const Slice q{meqn, 1 - mbc}, w{meqn * mwaves, 1 - mbc}, sv{mwaves, 1 - mbc};
    const int mu = ixy == 1 ? 1 : 2, mv = ixy == 1 ? 2 : 1;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double wl[3][4], sl[3];
        euler_rpn(&qr[q.at(1, i - 1)], &ql[q.at(1, i)], mu, mv, wl, sl, &amdq[q.at(1, i)],
                  &apdq[q.at(1, i)]);
        for (int k = 0; k < 3; ++k) {
            for (int m = 0; m < 4; ++m) wave[w.at(1, i) + k * meqn + m] = wl[k][m];
            s[sv.at(k + 1, i)] = sl[k];
        }
    }
}

void rpt2_euler_roe(int ixy, int, int, int meqn, int, int, int mbc, int mx, const double* ql,
                    const double* qr, const double*, const double*, const double*,
                    const double* asdq, double* bmasdq, double* bpasdq) {
    const Slice q{meqn, 1 - mbc};
    const int mu = ixy == 1 ? 1 : 2, mv = ixy == 1 ? 2 : 1;
    for (int i = 2 - mbc; i <= mx + mbc; ++i)
        euler_rpt(&qr[q.at(1, i - 1)], &ql[q.at(1, i)], mu, mv, &asdq[q.at(1, i)],
                  &bmasdq[q.at(1, i)], &bpasdq[q.at(1, i)]);
}

// ---- 1D acoustics --------------------------------------------------------------
typedef void (*rp1_t)(int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                      const double* ql, const double* qr, const double* auxl,
                      const double* auxr, double* wave, double* s, double* amdq,
                      double* apdq);

void rp1_acoustics(int, int meqn, int mwaves, int, int mbc, int mx, const double* ql,
                   const double* qr, const double*, const double*, double* wave, double* s,
                   double* amdq, double* apdq) {
    const Slice q{meqn, 1 - mbc}, w{meqn * mwaves, 1 - mbc}, sv{mwaves, 1 - mbc};
    const double cc = g_cc, zz = g_zz, hz = g_hz;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const double dp = ql[q.at(1, i)] - qr[q.at(1, i - 1)];
        const double du = ql[q.at(2, i)] - qr[q.at(2, i - 1)];
        const double a1 = (zz * du - dp) * hz;
        const double a2 = (zz * du + dp) * hz;
        double* w1 = &wave[w.at(1, i)];
        double* w2 = w1 + meqn;
        w1[0] = -(a1 * zz); w1[1] = a1;
        w2[0] = a2 * zz;    w2[1] = a2;
        s[sv.at(1, i)] = -cc;
        s[sv.at(2, i)] = cc;
        amdq[q.at(1, i)] = cc * (a1 * zz);
        amdq[q.at(2, i)] = -(cc * a1);
        apdq[q.at(1, i)] = cc * (a2 * zz);
        apdq[q.at(2, i)] = cc * a2;
    }
}

// rp1_advection (clawpack/riemann, restated): wave = jump, s = u,
// A-dq = min(u, 0) wave, A+dq = max(u, 0) wave
void rp1_advection(int, int meqn, int mwaves, int, int mbc, int mx, const double* ql,
                   const double* qr, const double*, const double*, double* wave, double* s,
                   double* amdq, double* apdq) {
    const Slice q{meqn, 1 - mbc}, w{meqn * mwaves, 1 - mbc}, sv{mwaves, 1 - mbc};
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const double d = ql[q.at(1, i)] - qr[q.at(1, i - 1)];
        wave[w.at(1, i)] = d;
        s[sv.at(1, i)] = g_u;
        amdq[q.at(1, i)] = std::fmin(g_u, 0.0) * d;
        apdq[q.at(1, i)] = std::fmax(g_u, 0.0) * d;
    }
}

// 1D Euler Roe solver with the Harten-Hyman entropy fix (rp1_euler_with_efix
// of clawpack/riemann, restated from the mathematics; the same operations as
// the 2D solver above with the transverse velocity absent)
inline void euler1d_state(const double* q, double* u, double* c) {
    const double g1 = g_gamma - 1.0;
    const double ri = 1.0 / q[0];
    const double p = g1 * (q[2] - 0.5 * (q[1] * q[1]) * ri);
    *c = std::sqrt(g_gamma * p * ri);
    *u = q[1] * ri;
}

void euler1d_rp(const double* qL, const double* qR, double w[3][3], double s[3], double* amdq,
                double* apdq) {
    const double g1 = g_gamma - 1.0;
    const double rhsqrtl = std::sqrt(qL[0]);
    const double rhsqrtr = std::sqrt(qR[0]);
    const double il = 1.0 / rhsqrtl;
    const double ir = 1.0 / rhsqrtr;
    const double pl = g1 * (qL[2] - 0.5 * (qL[1] * qL[1]) * (il * il));
    const double pr = g1 * (qR[2] - 0.5 * (qR[1] * qR[1]) * (ir * ir));
    const double i2 = 1.0 / (rhsqrtl + rhsqrtr);
    const double u = (qL[1] * il + qR[1] * ir) * i2;
    const double enth = ((qL[2] + pl) * il + (qR[2] + pr) * ir) * i2;
    const double u2 = u * u;
    const double a2 = g1 * (enth - 0.5 * u2);
    const double a = std::sqrt(a2);
    const double g1a2 = g1 / a2;
    const double ha = 0.5 / a;
    double d[3];
    for (int m = 0; m < 3; ++m) d[m] = qR[m] - qL[m];
    const double b2 = g1a2 * ((enth - u2) * d[0] + u * d[1] - d[2]);
    const double b3 = (d[1] + (a - u) * d[0] - a * b2) * ha;
    const double b1 = d[0] - b2 - b3;
    w[0][0] = b1; w[0][1] = b1 * (u - a); w[0][2] = b1 * (enth - u * a);
    s[0] = u - a;
    w[1][0] = b2; w[1][1] = b2 * u;       w[1][2] = b2 * (0.5 * u2);
    s[1] = u;
    w[2][0] = b3; w[2][1] = b3 * (u + a); w[2][2] = b3 * (enth + u * a);
    s[2] = u + a;
    for (int m = 0; m < 3; ++m) amdq[m] = 0.0;
    double ul, cl;
    euler1d_state(qL, &ul, &cl);
    const double s0 = ul - cl;
    double q1[3];
    for (int m = 0; m < 3; ++m) q1[m] = qL[m] + w[0][m];
    double u1, c1;
    euler1d_state(q1, &u1, &c1);
    const double s1 = u1 - c1;
    if (!(s0 >= 0.0 && s[0] > 0.0)) {
        double sfract;
        if (s0 < 0.0 && s1 > 0.0) sfract = s0 * (s1 - s[0]) / (s1 - s0);
        else if (s[0] < 0.0) sfract = s[0];
        else sfract = 0.0;
        for (int m = 0; m < 3; ++m) amdq[m] = sfract * w[0][m];
        if (s[1] < 0.0) {
            for (int m = 0; m < 3; ++m) amdq[m] = amdq[m] + s[1] * w[1][m];
            double ur, cr;
            euler1d_state(qR, &ur, &cr);
            const double s3 = ur + cr;
            double q2[3];
            for (int m = 0; m < 3; ++m) q2[m] = qR[m] - w[2][m];
            double u2s, c2;
            euler1d_state(q2, &u2s, &c2);
            const double s2 = u2s + c2;
            double sf3;
            if (s2 < 0.0 && s3 > 0.0) sf3 = s2 * (s3 - s[2]) / (s3 - s2);
            else if (s[2] < 0.0) sf3 = s[2];
            else sf3 = 0.0;
            for (int m = 0; m < 3; ++m) amdq[m] = amdq[m] + sf3 * w[2][m];
        }
    }
    for (int m = 0; m < 3; ++m) {
        const double df = (s[0] * w[0][m] + s[1] * w[1][m]) + s[2] * w[2][m];
        apdq[m] = df - amdq[m];
    }
}

void rp1_euler_roe(int, int meqn, int mwaves, int, int mbc, int mx, const double* ql,
                   const double* qr, const double*, const double*, double* wave, double* s,
                   double* amdq, double* apdq) {
    const Slice q{meqn, 1 - mbc}, w{meqn * mwaves, 1 - mbc}, sv{mwaves, 1 - mbc};
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double wl[3][3], sl[3];
        euler1d_rp(&qr[q.at(1, i - 1)], &ql[q.at(1, i)], wl, sl, &amdq[q.at(1, i)], &apdq[q.at(1, i)]);
        for (int k = 0; k < 3; ++k) {
            for (int m = 0; m < 3; ++m) wave[w.at(1, i) + k * meqn + m] = wl[k][m];
            s[sv.at(k + 1, i)] = sl[k];
        }
    }
}

// Variable-coefficient acoustics, aux = (Z, c) per cell: left-going wave on
// the eigenvector of cell i-1, right-going on that of cell i.
void rp1_vc_acoustics(int, int meqn, int mwaves, int maux, int mbc, int mx,
                      const double* ql, const double* qr, const double* auxl,
                      const double* auxr, double* wave, double* s, double* amdq,
                      double* apdq) {
    const Slice q{meqn, 1 - mbc}, w{meqn * mwaves, 1 - mbc}, sv{mwaves, 1 - mbc},
        a{maux, 1 - mbc};
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const double zl = auxr[a.at(1, i - 1)], cl = auxr[a.at(2, i - 1)];
        const double zr = auxl[a.at(1, i)], cr = auxl[a.at(2, i)];
        const double dp = ql[q.at(1, i)] - qr[q.at(1, i - 1)];
        const double du = ql[q.at(2, i)] - qr[q.at(2, i - 1)];
        const double a1 = (zr * du - dp) / (zl + zr);
        const double a2 = (zl * du + dp) / (zl + zr);
        double* w1 = &wave[w.at(1, i)];
        double* w2 = w1 + meqn;
        w1[0] = -(a1 * zl); w1[1] = a1;
        w2[0] = a2 * zr;    w2[1] = a2;
        s[sv.at(1, i)] = -cl;
        s[sv.at(2, i)] = cr;
        amdq[q.at(1, i)] = cl * (a1 * zl);
        amdq[q.at(2, i)] = -(cl * a1);
        apdq[q.at(1, i)] = cr * (a2 * zr);
        apdq[q.at(2, i)] = cr * a2;
    }
}

// ---------------------------------------------------------------- limiter ---
// src/2d/inlinelimiter.f90:25-105.  Dot products use the unlimited waves:
// dotr is formed before the wave at i is scaled, and carried as dotl.
void limiter(int maxm, int meqn, int mwaves, int mbc, int mx, double* wave, const double* s,
             const int* mthlim) {
    (void)maxm;
    const Slice w{meqn * mwaves, 1 - mbc}, sv{mwaves, 1 - mbc};
    std::vector<double> dotr(mwaves, 0.0);
    for (int i = 0; i <= mx + 1; ++i) {
        for (int mw = 1; mw <= mwaves; ++mw) {
            if (mthlim[mw - 1] == 0) continue;
            double wnorm2 = 0.0;
            const double dotl = dotr[mw - 1];
            dotr[mw - 1] = 0.0;
            double* wi = &wave[w.at(1, i)] + (mw - 1) * meqn;
            const double* wn = &wave[w.at(1, i + 1)] + (mw - 1) * meqn;
            for (int m = 0; m < meqn; ++m) {
                wnorm2 = wnorm2 + wi[m] * wi[m];
                dotr[mw - 1] = dotr[mw - 1] + wi[m] * wn[m];
            }
            if (i == 0) continue;
            if (wnorm2 == 0.0) continue;
            double r;
            if (s[sv.at(mw, i)] > 0.0)
                r = dotl / wnorm2;
            else
                r = dotr[mw - 1] / wnorm2;
            double wlimiter;
            switch (mthlim[mw - 1]) {
                case 1: wlimiter = std::fmax(0.0, std::fmin(1.0, r)); break;
                case 2:
                    wlimiter = std::fmax(std::fmax(0.0, std::fmin(1.0, 2.0 * r)),
                                         std::fmin(2.0, r));
                    break;
                case 3: wlimiter = (r + std::fabs(r)) / (1.0 + std::fabs(r)); break;
                case 4: {
                    const double c = (1.0 + r) / 2.0;
                    wlimiter = std::fmax(0.0, std::fmin(std::fmin(c, 2.0), 2.0 * r));
                    break;
                }
                case 5: wlimiter = r; break;
                default: wlimiter = 1.0; break;  // rejected earlier by validation
            }
            for (int m = 0; m < meqn; ++m) wi[m] = wlimiter * wi[m];
        }
    }
}

// ------------------------------------------------------------------ flux2 ---
void flux2(int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
           const double* q1d, const double* dtdx1d, const double* aux1, const double* aux2,
           const double* aux3, const int* method, const int* mthlim, double* qadd,
           double* fadd, double* gadd, double* cfl1d, double* wave, double* s, double* amdq,
           double* apdq, double* cqxx, double* bmasdq, double* bpasdq, rpn2_t rpn2,
           rpt2_t rpt2, bool use_fwave) {
    const Slice q{meqn, 1 - mbc}, sv{mwaves, 1 - mbc}, w{meqn * mwaves, 1 - mbc};
    const Slice g{2 * meqn, 1 - mbc};
    auto D = [&](int i) { return dtdx1d[i - (1 - mbc)]; };
    auto G = [&](int m, int k, int i) -> double& { return gadd[(m - 1) + meqn * (k - 1) + g.n0 * (i - g.lo)]; };
    bool limit = false;
    for (int mw = 0; mw < mwaves; ++mw)
        if (mthlim[mw] > 0) limit = true;

    for (int i = 1 - mbc; i <= mx + mbc; ++i)
        for (int m = 1; m <= meqn; ++m) qadd[q.at(m, i)] = 0.0;

    rpn2(ixy, maxm, meqn, mwaves, maux, mbc, mx, q1d, q1d, aux2, aux2, wave, s, amdq, apdq);

    for (int i = 1; i <= mx + 1; ++i) {
        for (int m = 1; m <= meqn; ++m)
            qadd[q.at(m, i - 1)] = qadd[q.at(m, i - 1)] - D(i - 1) * amdq[q.at(m, i)];
        for (int m = 1; m <= meqn; ++m)
            qadd[q.at(m, i)] = qadd[q.at(m, i)] - D(i) * apdq[q.at(m, i)];
    }

    double c1 = 0.0;
    for (int i = 1; i <= mx + 1; ++i)
        for (int mw = 1; mw <= mwaves; ++mw) {
            const double sm = s[sv.at(mw, i)];
            c1 = std::fmax(std::fmax(c1, D(i) * sm), -D(i - 1) * sm);
        }
    *cfl1d = c1;

    if (method[1] != 1) {
        if (limit) limiter(maxm, meqn, mwaves, mbc, mx, wave, s, mthlim);
        for (int i = 2 - mbc; i <= mx + mbc; ++i) {
            const double dtdxave = 0.5 * (D(i - 1) + D(i));
            for (int m = 1; m <= meqn; ++m) cqxx[q.at(m, i)] = 0.0;
            for (int mw = 1; mw <= mwaves; ++mw) {
                const double sm = s[sv.at(mw, i)];
                const double coef = use_fwave
                                        ? std::copysign(1.0, sm) * (1.0 - std::fabs(sm) * dtdxave)
                                        : std::fabs(sm) * (1.0 - std::fabs(sm) * dtdxave);
                const double* wv = &wave[w.at(1, i)] + (mw - 1) * meqn;
                for (int m = 1; m <= meqn; ++m)
                    cqxx[q.at(m, i)] = cqxx[q.at(m, i)] + coef * wv[m - 1];
            }
            for (int m = 1; m <= meqn; ++m) fadd[q.at(m, i)] = 0.5 * cqxx[q.at(m, i)];
        }
    } else {
        // order 1: the reference leaves fadd unset (src/2d/flux2.f90:101-102,134);
        // the intended value is zero.
        for (int i = 1 - mbc; i <= mx + mbc; ++i)
            for (int m = 1; m <= meqn; ++m) fadd[q.at(m, i)] = 0.0;
    }

    if (method[2] <= 0) {
        // no transverse propagation: the reference leaves gadd unset
        // (src/2d/flux2.f90:104-105,186); the intended value is zero.
        for (int i = 1 - mbc; i <= mx + mbc; ++i)
            for (int k = 1; k <= 2; ++k)
                for (int m = 1; m <= meqn; ++m) G(m, k, i) = 0.0;
        return;
    }

    if (method[1] > 1 && method[2] == 2) {
        for (int i = 1; i <= mx + 1; ++i)
            for (int m = 1; m <= meqn; ++m) {
                amdq[q.at(m, i)] = amdq[q.at(m, i)] + cqxx[q.at(m, i)];
                apdq[q.at(m, i)] = apdq[q.at(m, i)] - cqxx[q.at(m, i)];
            }
    }

    rpt2(ixy, 1, maxm, meqn, mwaves, maux, mbc, mx, q1d, q1d, aux1, aux2, aux3, amdq, bmasdq,
         bpasdq);
    for (int i = 1; i <= mx + 1; ++i) {
        for (int m = 1; m <= meqn; ++m) G(m, 1, i - 1) = -(0.5 * D(i - 1) * bmasdq[q.at(m, i)]);
        for (int m = 1; m <= meqn; ++m) G(m, 2, i - 1) = -(0.5 * D(i - 1) * bpasdq[q.at(m, i)]);
    }
    rpt2(ixy, 2, maxm, meqn, mwaves, maux, mbc, mx, q1d, q1d, aux1, aux2, aux3, apdq, bmasdq,
         bpasdq);
    for (int i = 1; i <= mx + 1; ++i) {
        for (int m = 1; m <= meqn; ++m) G(m, 1, i) = G(m, 1, i) - 0.5 * D(i) * bmasdq[q.at(m, i)];
        for (int m = 1; m <= meqn; ++m) G(m, 2, i) = G(m, 2, i) - 0.5 * D(i) * bpasdq[q.at(m, i)];
    }
}

// src1.f:18-23 on the cells i = 1..mx+mbc of one slice (stride `st` doubles
// between cells, p at +0 and the radial velocity at +1)
void src_radial_slice(int mbc, int mx, double dx, double* q, int st, double dt) {
    for (int i = 1; i <= mx + mbc; ++i) {
        const double xcell = g_src_xlower + ((double)i - 0.5) * dx;
        double* c = q + (size_t)st * (i - (1 - mbc));
        c[0] = c[0] - dt * (double)(g_src_ndim - 1) * g_bulk / xcell * c[1];
    }
}

bool pick2(int solver, rpn2_t* rpn, rpt2_t* rpt) {
    switch (solver) {
        case ORC_ACOUSTICS_2D: *rpn = rpn2_acoustics; *rpt = rpt2_acoustics; return true;
        case ORC_VC_ADVECTION_2D: *rpn = rpn2_vc_advection; *rpt = rpt2_vc_advection; return true;
        case ORC_EULER_ROE_2D: *rpn = rpn2_euler_roe; *rpt = rpt2_euler_roe; return true;
        default: return false;
    }
}

}  // namespace

extern "C" {

// ------------------------------------------------------------------ step2 ---
// src/2d/step2.f90:2-251.  qold/qnew/aux in the reference layout with ghost
// cells; qnew must equal qold on entry.  Returns 0, or -1 for an unknown solver.
}  // extern "C"

// Run body(item, thread) for items 0..count-1 on g_threads host threads
// (std::thread; items handed out in order from an atomic counter), then join.
template <class F>
static void parallel_items(int count, int nthreads, F&& body) {
    std::atomic<int> next{0};
    auto worker = [&](int tid) {
        for (int k = next.fetch_add(1); k < count; k = next.fetch_add(1)) body(k, tid);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(worker, t);
    worker(0);
    for (auto& th : pool) th.join();
}

extern "C" {

int orc_step2(int meqn, int mwaves, int maux, int mbc, int mx, int my, const double* qold,
              double* qnew, const double* aux, double dx, double dy, double dt,
              const int* method, const int* mthlim, int use_fwave, double* cfl_out) {
    rpn2_t rpn2;
    rpt2_t rpt2;
    if (!pick2(g_solver, &rpn2, &rpt2)) return -1;
    const int maxm = std::max(mx, my);
    const int n = maxm + 2 * mbc;
    const int nx = mx + 2 * mbc;
    auto Q = [&](const double* a, int m, int i, int j) {
        return a[(m - 1) + meqn * ((i - (1 - mbc)) + nx * (j - (1 - mbc)))];
    };
    auto QN = [&](int m, int i, int j) -> double& {
        return qnew[(m - 1) + meqn * ((i - (1 - mbc)) + nx * (j - (1 - mbc)))];
    };
    auto A = [&](int ma, int i, int j) {
        return aux[(ma - 1) + maux * ((i - (1 - mbc)) + nx * (j - (1 - mbc)))];
    };
    // flux2's work arrays (one set per thread in the OpenMP timing build)
    struct Work {
        std::vector<double> qadd, fadd, gadd, q1d, dtdx1d, dtdy1d, aux1, aux2, aux3, wave, s, amdq,
            apdq, cqxx, bmasdq, bpasdq;
        Work(int meqn, int mwaves, int maux, int n)
            : qadd(meqn * n), fadd(meqn * n), gadd(2 * meqn * n), q1d(meqn * n), dtdx1d(n),
              dtdy1d(n), aux1(std::max(maux, 1) * n), aux2(std::max(maux, 1) * n),
              aux3(std::max(maux, 1) * n), wave(meqn * mwaves * n), s(mwaves * n), amdq(meqn * n),
              apdq(meqn * n), cqxx(meqn * n), bmasdq(meqn * n), bpasdq(meqn * n) {}
    };
    const Slice sl{meqn, 1 - mbc}, sa{maux, 1 - mbc};
    const int index_capa = method[5];
    const double dtdx = dt / dx, dtdy = dt / dy;
    auto init = [&](Work& w) {
        if (index_capa == 0)
            for (int i = 0; i < n; ++i) { w.dtdx1d[i] = dtdx; w.dtdy1d[i] = dtdy; }
    };

    // x-sweep of row j (src/2d/step2.f90:92-165)
    auto x_slice = [&](int j, Work& w, double& cfl) {
        auto GA = [&](int m, int k, int i) { return w.gadd[(m - 1) + meqn * (k - 1) + 2 * meqn * (i - (1 - mbc))]; };
        for (int i = 1 - mbc; i <= mx + mbc; ++i)
            for (int m = 1; m <= meqn; ++m) w.q1d[sl.at(m, i)] = Q(qold, m, i, j);
        if (index_capa > 0)
            for (int i = 1 - mbc; i <= mx + mbc; ++i) w.dtdx1d[i - (1 - mbc)] = dtdx / A(index_capa, i, j);
        if (maux > 0)
            for (int i = 1 - mbc; i <= mx + mbc; ++i)
                for (int ma = 1; ma <= maux; ++ma) {
                    w.aux1[sa.at(ma, i)] = A(ma, i, j - 1);
                    w.aux2[sa.at(ma, i)] = A(ma, i, j);
                    w.aux3[sa.at(ma, i)] = A(ma, i, j + 1);
                }
        double cfl1d;
        flux2(1, maxm, meqn, mwaves, maux, mbc, mx, w.q1d.data(), w.dtdx1d.data(), w.aux1.data(),
              w.aux2.data(), w.aux3.data(), method, mthlim, w.qadd.data(), w.fadd.data(),
              w.gadd.data(), &cfl1d, w.wave.data(), w.s.data(), w.amdq.data(), w.apdq.data(),
              w.cqxx.data(), w.bmasdq.data(), w.bpasdq.data(), rpn2, rpt2, use_fwave != 0);
        cfl = std::fmax(cfl, cfl1d);
        if (index_capa == 0) {
            for (int i = 1; i <= mx; ++i)
                for (int m = 1; m <= meqn; ++m) {
                    QN(m, i, j) = QN(m, i, j) + w.qadd[sl.at(m, i)] -
                                  dtdx * (w.fadd[sl.at(m, i + 1)] - w.fadd[sl.at(m, i)]) -
                                  dtdy * (GA(m, 2, i) - GA(m, 1, i));
                    QN(m, i, j - 1) = QN(m, i, j - 1) - dtdy * GA(m, 1, i);
                    QN(m, i, j + 1) = QN(m, i, j + 1) + dtdy * GA(m, 2, i);
                }
        } else {
            for (int i = 1; i <= mx; ++i)
                for (int m = 1; m <= meqn; ++m) {
                    QN(m, i, j) = QN(m, i, j) + w.qadd[sl.at(m, i)] -
                                  (dtdx * (w.fadd[sl.at(m, i + 1)] - w.fadd[sl.at(m, i)]) +
                                   dtdy * (GA(m, 2, i) - GA(m, 1, i))) /
                                      A(index_capa, i, j);
                    QN(m, i, j - 1) = QN(m, i, j - 1) - dtdy * GA(m, 1, i) / A(index_capa, i, j - 1);
                    QN(m, i, j + 1) = QN(m, i, j + 1) + dtdy * GA(m, 2, i) / A(index_capa, i, j + 1);
                }
        }
    };

    // y-sweep of column i (src/2d/step2.f90:173-248)
    auto y_slice = [&](int i, Work& w, double& cfl) {
        auto GA = [&](int m, int k, int i) { return w.gadd[(m - 1) + meqn * (k - 1) + 2 * meqn * (i - (1 - mbc))]; };
        for (int j = 1 - mbc; j <= my + mbc; ++j)
            for (int m = 1; m <= meqn; ++m) w.q1d[sl.at(m, j)] = Q(qold, m, i, j);
        if (index_capa > 0)
            for (int j = 1 - mbc; j <= my + mbc; ++j) w.dtdy1d[j - (1 - mbc)] = dtdy / A(index_capa, i, j);
        if (maux > 0)
            for (int j = 1 - mbc; j <= my + mbc; ++j)
                for (int ma = 1; ma <= maux; ++ma) {
                    w.aux1[sa.at(ma, j)] = A(ma, i - 1, j);
                    w.aux2[sa.at(ma, j)] = A(ma, i, j);
                    w.aux3[sa.at(ma, j)] = A(ma, i + 1, j);
                }
        double cfl1d;
        flux2(2, maxm, meqn, mwaves, maux, mbc, my, w.q1d.data(), w.dtdy1d.data(), w.aux1.data(),
              w.aux2.data(), w.aux3.data(), method, mthlim, w.qadd.data(), w.fadd.data(),
              w.gadd.data(), &cfl1d, w.wave.data(), w.s.data(), w.amdq.data(), w.apdq.data(),
              w.cqxx.data(), w.bmasdq.data(), w.bpasdq.data(), rpn2, rpt2, use_fwave != 0);
        cfl = std::fmax(cfl, cfl1d);
        if (index_capa == 0) {
            for (int j = 1; j <= my; ++j)
                for (int m = 1; m <= meqn; ++m) {
                    QN(m, i, j) = QN(m, i, j) +
                                  (w.qadd[sl.at(m, j)] -
                                   dtdy * (w.fadd[sl.at(m, j + 1)] - w.fadd[sl.at(m, j)]) -
                                   dtdx * (GA(m, 2, j) - GA(m, 1, j)));
                    QN(m, i - 1, j) = QN(m, i - 1, j) - dtdx * GA(m, 1, j);
                    QN(m, i + 1, j) = QN(m, i + 1, j) + dtdx * GA(m, 2, j);
                }
        } else {
            for (int j = 1; j <= my; ++j)
                for (int m = 1; m <= meqn; ++m) {
                    QN(m, i, j) = QN(m, i, j) + w.qadd[sl.at(m, j)] -
                                  (dtdy * (w.fadd[sl.at(m, j + 1)] - w.fadd[sl.at(m, j)]) +
                                   dtdx * (GA(m, 2, j) - GA(m, 1, j))) /
                                      A(index_capa, i, j);
                    QN(m, i - 1, j) = QN(m, i - 1, j) - dtdx * GA(m, 1, j) / A(index_capa, i - 1, j);
                    QN(m, i + 1, j) = QN(m, i + 1, j) + dtdx * GA(m, 2, j) / A(index_capa, i + 1, j);
                }
        }
    };

    double cfl = 0.0;
    if (g_threads > 1) {
        // Timing variant only: the reference's step2 is serial.  A slice
        // updates its own row and the two beside it, so slices three apart
        // never touch the same cell: each of three passes runs every third
        // slice in parallel (the scheme step3.f90 uses for its 3D slices).
        // Each cell then receives its contributions in another order than the
        // serial sweep's.
        const int nt = g_threads;
        std::vector<Work> ws;
        for (int t = 0; t < nt; ++t) { ws.emplace_back(meqn, mwaves, maux, n); init(ws.back()); }
        std::vector<double> cfls(nt, 0.0);
        for (int col = 0; col < 3; ++col)
            parallel_items((my + 2 - col + 2) / 3, nt, [&](int k, int t) { x_slice(col + 3 * k, ws[t], cfls[t]); });
        for (int col = 0; col < 3; ++col)
            parallel_items((mx + 2 - col + 2) / 3, nt, [&](int k, int t) { y_slice(col + 3 * k, ws[t], cfls[t]); });
        for (double c : cfls) cfl = std::fmax(cfl, c);
    } else {
        Work w(meqn, mwaves, maux, n);
        init(w);
        for (int j = 0; j <= my + 1; ++j) x_slice(j, w, cfl);
        for (int i = 0; i <= mx + 1; ++i) y_slice(i, w, cfl);
    }
    *cfl_out = cfl;
    return 0;
}

// ----------------------------------------------------------------- step2ds ---
// src/2d/step2ds.f90:1-275: one directional sweep of dimensional splitting.
// ids = 1: x-slices over every row j = 1-mbc..my+mbc (ghost rows included, so
// the following y-sweep sees x-updated ghost rows); ids = 2: y-slices over
// every column i = 1-mbc..mx+mbc.  Only the cells 1..mx (1..my) of each slice
// are updated; flux2 returns before its transverse part (method(3) < 0).
// qold supplies the slices and may alias qnew (each slice is gathered before
// its own update, and slices do not overlap).
int orc_step2ds(int meqn, int mwaves, int maux, int mbc, int mx, int my, const double* qold,
                double* qnew, const double* aux, double dx, double dy, double dt,
                const int* method, const int* mthlim, int ids, int use_fwave, double* cfl_out) {
    rpn2_t rpn2;
    rpt2_t rpt2;
    if (!pick2(g_solver, &rpn2, &rpt2)) return -1;
    const int maxm = std::max(mx, my);
    const int n = maxm + 2 * mbc;
    const int nx = mx + 2 * mbc;
    auto at = [&](int m, int i, int j) {
        return (size_t)(m - 1) + (size_t)meqn * ((i - (1 - mbc)) + (size_t)nx * (j - (1 - mbc)));
    };
    auto A = [&](int ma, int i, int j) {
        return aux[(ma - 1) + maux * ((i - (1 - mbc)) + nx * (j - (1 - mbc)))];
    };
    std::vector<double> qadd(meqn * n), fadd(meqn * n), gadd(2 * meqn * n), q1d(meqn * n);
    std::vector<double> dtdx1d(n), dtdy1d(n), aux1(std::max(maux, 1) * n),
        aux2(std::max(maux, 1) * n), aux3(std::max(maux, 1) * n);
    std::vector<double> wave(meqn * mwaves * n), s(mwaves * n), amdq(meqn * n), apdq(meqn * n),
        cqxx(meqn * n), bmasdq(meqn * n), bpasdq(meqn * n);
    const Slice sl{meqn, 1 - mbc}, sa{maux, 1 - mbc};
    const int index_capa = method[5];
    double cfl = 0.0;
    const double dtdx = dt / dx, dtdy = dt / dy;
    if (index_capa == 0)
        for (int i = 0; i < n; ++i) { dtdx1d[i] = dtdx; dtdy1d[i] = dtdy; }
    const int nslice = ids == 1 ? my : mx;   // slices across
    const int mlen = ids == 1 ? mx : my;     // cells along
    const double dtd = ids == 1 ? dtdx : dtdy;
    double* dtd1d = ids == 1 ? dtdx1d.data() : dtdy1d.data();
    for (int k = 1 - mbc; k <= nslice + mbc; ++k) {
        // (i, j) of cell l of slice k
        auto ij = [&](int l, int& i, int& j) {
            if (ids == 1) { i = l; j = k; } else { i = k; j = l; }
        };
        for (int l = 1 - mbc; l <= mlen + mbc; ++l) {
            int i, j;
            ij(l, i, j);
            for (int m = 1; m <= meqn; ++m) q1d[sl.at(m, l)] = qold[at(m, i, j)];
        }
        if (index_capa > 0)
            for (int l = 1 - mbc; l <= mlen + mbc; ++l) {
                int i, j;
                ij(l, i, j);
                dtd1d[l - (1 - mbc)] = dtd / A(index_capa, i, j);
            }
        if (maux > 0)
            for (int l = 1 - mbc; l <= mlen + mbc; ++l) {
                int i, j;
                ij(l, i, j);
                for (int ma = 1; ma <= maux; ++ma) aux2[sa.at(ma, l)] = A(ma, i, j);
            }
        double cfl1d;
        flux2(ids, maxm, meqn, mwaves, maux, mbc, mlen, q1d.data(), dtd1d, aux1.data(),
              aux2.data(), aux3.data(), method, mthlim, qadd.data(), fadd.data(), gadd.data(),
              &cfl1d, wave.data(), s.data(), amdq.data(), apdq.data(), cqxx.data(),
              bmasdq.data(), bpasdq.data(), rpn2, rpt2, use_fwave != 0);
        cfl = std::fmax(cfl, cfl1d);
        for (int l = 1; l <= mlen; ++l) {
            int i, j;
            ij(l, i, j);
            for (int m = 1; m <= meqn; ++m) {
                double& qn = qnew[at(m, i, j)];
                if (index_capa == 0)
                    qn = qn + qadd[sl.at(m, l)] - dtd * (fadd[sl.at(m, l + 1)] - fadd[sl.at(m, l)]);
                else
                    qn = qn + qadd[sl.at(m, l)] -
                         dtd * (fadd[sl.at(m, l + 1)] - fadd[sl.at(m, l)]) / A(index_capa, i, j);
            }
        }
    }
    *cfl_out = cfl;
    return 0;
}

// ------------------------------------------------------------------ dimsp2 ---
// src/2d/dimsp2.f:1-99: Godunov (method(3) = -1: x by dt, then y by dt) or
// Strang (method(3) = -2: x by dt/2, y by dt, x by dt/2) splitting.  A sweep
// whose Courant number exceeds cflv(1) ends the step with that number.
int orc_dimsp2(int meqn, int mwaves, int maux, int mbc, int mx, int my, const double* qold,
               double* qnew, const double* aux, double dx, double dy, double dt,
               const int* method, const int* mthlim, const double* cflv, int use_fwave,
               double* cfl_out) {
    const double dt2 = dt / 2.0;
    double cflx, cfly;
    int rc = orc_step2ds(meqn, mwaves, maux, mbc, mx, my, qold, qnew, aux, dx, dy,
                         method[2] == -2 ? dt2 : dt, method, mthlim, 1, use_fwave, &cflx);
    if (rc) return rc;
    if (cflx > cflv[0]) { *cfl_out = cflx; return 0; }
    rc = orc_step2ds(meqn, mwaves, maux, mbc, mx, my, qnew, qnew, aux, dx, dy, dt, method,
                     mthlim, 2, use_fwave, &cfly);
    if (rc) return rc;
    double cfl = std::fmax(cflx, cfly);
    if (method[2] == -2) {
        if (cfly > cflv[0]) { *cfl_out = cfly; return 0; }
        rc = orc_step2ds(meqn, mwaves, maux, mbc, mx, my, qnew, qnew, aux, dx, dy, dt2, method,
                         mthlim, 1, use_fwave, &cflx);
        if (rc) return rc;
        cfl = std::fmax(cfl, cflx);
    }
    *cfl_out = cfl;
    return 0;
}

// -------------------------------------------------------------------- bc2 ---
// src/2d/bc2.f:4-215.  mthbc: 1 extrap, 2 periodic, 3 wall; order L, R, B, T.
// Returns -1 for a user BC (mthbc=0), which the reference stops on.
int orc_bc2(int meqn, int mbc, int mx, int my, double* q, const int* mthbc) {
    const int nx = mx + 2 * mbc;
    auto Q = [&](int m, int i, int j) -> double& {
        return q[(m - 1) + meqn * ((i - (1 - mbc)) + nx * (j - (1 - mbc)))];
    };
    for (int k = 0; k < 4; ++k)
        if (mthbc[k] < 1 || mthbc[k] > 3) return -1;
    // left
    for (int j = 1 - mbc; j <= my + mbc; ++j)
        for (int ibc = 1; ibc <= mbc; ++ibc) {
            for (int m = 1; m <= meqn; ++m) {
                if (mthbc[0] == 1) Q(m, 1 - ibc, j) = Q(m, 1, j);
                else if (mthbc[0] == 2) Q(m, 1 - ibc, j) = Q(m, mx + 1 - ibc, j);
                else Q(m, 1 - ibc, j) = Q(m, ibc, j);
            }
            if (mthbc[0] == 3) Q(2, 1 - ibc, j) = -Q(2, ibc, j);
        }
    // right
    for (int j = 1 - mbc; j <= my + mbc; ++j)
        for (int ibc = 1; ibc <= mbc; ++ibc) {
            for (int m = 1; m <= meqn; ++m) {
                if (mthbc[1] == 1) Q(m, mx + ibc, j) = Q(m, mx, j);
                else if (mthbc[1] == 2) Q(m, mx + ibc, j) = Q(m, ibc, j);
                else Q(m, mx + ibc, j) = Q(m, mx + 1 - ibc, j);
            }
            if (mthbc[1] == 3) Q(2, mx + ibc, j) = -Q(2, mx + 1 - ibc, j);
        }
    // bottom
    for (int jbc = 1; jbc <= mbc; ++jbc)
        for (int i = 1 - mbc; i <= mx + mbc; ++i) {
            for (int m = 1; m <= meqn; ++m) {
                if (mthbc[2] == 1) Q(m, i, 1 - jbc) = Q(m, i, 1);
                else if (mthbc[2] == 2) Q(m, i, 1 - jbc) = Q(m, i, my + 1 - jbc);
                else Q(m, i, 1 - jbc) = Q(m, i, jbc);
            }
            if (mthbc[2] == 3) Q(3, i, 1 - jbc) = -Q(3, i, jbc);
        }
    // top
    for (int jbc = 1; jbc <= mbc; ++jbc)
        for (int i = 1 - mbc; i <= mx + mbc; ++i) {
            for (int m = 1; m <= meqn; ++m) {
                if (mthbc[3] == 1) Q(m, i, my + jbc) = Q(m, i, my);
                else if (mthbc[3] == 2) Q(m, i, my + jbc) = Q(m, i, jbc);
                else Q(m, i, my + jbc) = Q(m, i, my + 1 - jbc);
            }
            if (mthbc[3] == 3) Q(3, i, my + jbc) = -Q(3, i, my + 1 - jbc);
        }
    return 0;
}

// ------------------------------------------------------------------ claw2 ---
// src/2d/claw2.f:494-784: dt clamp to tend, bc2, copy, step2, accept/reject
// with retry, next dt = min(dt_max, dt*cfl_desired/cfl), info codes.
// dtv[5], cflv[4], nv[2], method[7] have the reference's meaning.
int orc_claw2(int meqn, int mwaves, int maux, int mbc, int mx, int my, double* q,
              const double* aux, double dx, double dy, double tstart, double* tend_io,
              double* dtv, double* cflv, int* nv, const int* method, const int* mthlim,
              const int* mthbc, int use_fwaves) {
    const double tend = *tend_io;
    int info = 0;
    double t = tstart;
    int maxn = nv[0];
    double dt = dtv[0];
    double cflmax = 0.0, dtmin = dt, dtmax = dt, cfl = 0.0;
    nv[1] = 0;
    const size_t nq = (size_t)meqn * (mx + 2 * mbc) * (my + 2 * mbc);
    std::vector<double> qwork(nq), qwork2(method[4] == 2 ? nq : 0);
    // b4step2 (src/2d/claw2.f:626-631) writes a working aux from the caller's
    const long long ncell = (long long)(mx + 2 * mbc) * (my + 2 * mbc);
    std::vector<double> auxw(g_b4 != 0 ? (size_t)maux * ncell : 0);
    const double* aux_step = g_b4 != 0 ? auxw.data() : aux;
    // the source routine over every row j = 1-mbc..my+mbc (0 = default no-op)
    auto src2 = [&](double* qq, double dts) {
        if (g_src != 1) return;
        for (int j = 0; j < my + 2 * mbc; ++j)
            src_radial_slice(mbc, mx, dx, qq + (size_t)meqn * (mx + 2 * mbc) * j, meqn, dts);
    };
    if (method[0] == 0) {
        if (tend < tstart) maxn = 1;
        else {
            maxn = (int)std::lround((tend - tstart) / dt);
            if (std::fabs(maxn * dt - (tend - tstart)) > 1e-5 * (tend - tstart)) {
                info = 2;
                goto done;
            }
        }
    }
    if (method[0] == 1 && cflv[1] > cflv[0]) { info = 3; goto done; }
    if (method[5] > method[6]) { info = 5; goto done; }
    if (method[1] < method[2]) { info = 6; goto done; }
    if (maxn == 0) goto done;
    for (int n = 1; n <= maxn; ++n) {
        const double told = t;
        if (told + dt > tend && tstart < tend) dt = tend - told;
        for (;;) {
            if (orc_bc2(meqn, mbc, mx, my, q, mthbc) != 0) { info = -2; goto done; }
            if (g_b4 != 0) orc_b4step2(maux, ncell, aux, auxw.data(), told);
            if (method[4] == 2) {
                // src/2d/claw2.f:635-647: keep q for a retry, then dt/2 of source
                std::memcpy(qwork2.data(), q, nq * sizeof(double));
                src2(q, dt / 2.0);
            }
            std::memcpy(qwork.data(), q, nq * sizeof(double));
            const int rc = method[2] >= 0
                               ? orc_step2(meqn, mwaves, maux, mbc, mx, my, qwork.data(), q,
                                           aux_step, dx, dy, dt, method, mthlim, use_fwaves, &cfl)
                               : orc_dimsp2(meqn, mwaves, maux, mbc, mx, my, qwork.data(), q,
                                            aux_step, dx, dy, dt, method, mthlim, cflv, use_fwaves,
                                            &cfl);
            if (rc != 0) {
                info = -1;
                goto done;
            }
            t = told + dt;
            if (cfl <= cflv[0]) {
                cflmax = std::fmax(cfl, cflmax);
                break;
            }
            t = told;
            std::memcpy(q, method[4] == 2 ? qwork2.data() : qwork.data(), nq * sizeof(double));
            if (method[0] == 1) {
                dt = std::fmin(dtv[1], dt * cflv[1] / cfl);
                continue;
            }
            cflmax = std::fmax(cfl, cflmax);
            goto done;
        }
        // src/2d/claw2.f:726-738: the source step after an accepted step
        if (method[4] == 2) src2(q, dt / 2.0);
        if (method[4] == 1) src2(q, dt);
        if (method[0] == 1) {
            if (cfl == 0.0) dt = dtv[1];
            else dt = std::fmin(dtv[1], dt * cflv[1] / cfl);
            dtmin = std::fmin(dt, dtmin);
            dtmax = std::fmax(dt, dtmax);
        }
        nv[1] = nv[1] + 1;
        if (t >= tend) break;
    }
done:
    if (method[0] == 1 && t < tend && nv[1] == maxn) info = 11;
    if (method[0] == 0 && cflmax > cflv[0]) info = 12;
    *tend_io = t;
    cflv[2] = cflmax;
    cflv[3] = cfl;
    dtv[2] = dtmin;
    dtv[3] = dtmax;
    dtv[4] = dt;
    return info;
}

// ================================================================ 3D path ===
// step3 (src/3d/step3.f90:3-873) in its serial execution order, flux3
// (src/3d/flux3.f90:4-612), bc3 (src/3d/bc3.f), claw3 (src/3d/claw3.f:738-928).
// Solver: variable-coefficient acoustics, q = (p, u, v, w), aux = (Z, c), with
// transverse (rpt3) and double-transverse (rptt3) splits written from the
// eigen-decomposition (the solver lives in the un-vendored clawpack/riemann).
// The 3D example links src/3d/limiter.f90 + philim.f90 instead of the inlined
// limiter; both form r = (w_i . w_upwind)/|w_i|^2 from unlimited waves with
// the same sums and the same phi(r), so `limiter` above serves here too.
}  // extern "C"

namespace {

// Normal velocity index (1-based) of a sweep, and of its y-like / z-like
// transverse directions: (x: y, z), (y: z, x), (z: x, y).
inline int vel_index(int dir) { return 1 + dir; }  // dir 1,2,3 -> 2,3,4
inline int trans_dir(int ixyz, int icoor) {       // icoor 2 = y-like, 3 = z-like
    return ((ixyz - 1 + (icoor - 1)) % 3) + 1;
}

struct Aux3 {  // aux slice arrays (maux, 1-mbc:maxm+mbc, 3)
    const double* a;
    int maux, n0lo, nlen;
    double at(int ma, int i, int l) const {  // l = 1..3
        return a[(ma - 1) + maux * ((i - n0lo) + nlen * (l - 1))];
    }
};

void rpn3_vc_acoustics(int ixyz, int meqn, int mbc, int mx, const double* q, const Aux3& a2,
                       double* wave, double* s, double* amdq, double* apdq) {
    const int mu = vel_index(ixyz);
    const Slice Q{meqn, 1 - mbc}, W{meqn * 2, 1 - mbc}, S{2, 1 - mbc};
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const double zl = a2.at(1, i - 1, 2), cl = a2.at(2, i - 1, 2);
        const double zr = a2.at(1, i, 2), cr = a2.at(2, i, 2);
        const double dp = q[Q.at(1, i)] - q[Q.at(1, i - 1)];
        const double du = q[Q.at(mu, i)] - q[Q.at(mu, i - 1)];
        const double a1 = (zr * du - dp) / (zl + zr);
        const double a2v = (zl * du + dp) / (zl + zr);
        double* w1 = &wave[W.at(1, i)];
        double* w2 = w1 + meqn;
        for (int m = 0; m < meqn; ++m) { w1[m] = 0.0; w2[m] = 0.0; amdq[Q.at(m + 1, i)] = 0.0; apdq[Q.at(m + 1, i)] = 0.0; }
        w1[0] = -(a1 * zl); w1[mu - 1] = a1;
        w2[0] = a2v * zr;   w2[mu - 1] = a2v;
        s[S.at(1, i)] = -cl;
        s[S.at(2, i)] = cr;
        amdq[Q.at(1, i)] = cl * (a1 * zl);
        amdq[Q.at(mu, i)] = -(cl * a1);
        apdq[Q.at(1, i)] = cr * (a2v * zr);
        apdq[Q.at(mu, i)] = cr * a2v;
    }
}

// Split a fluctuation living in cell (i1, mid) into the parts transmitted
// down (speed -c below) and up (speed +c above), given (Z, c) below, mid,
// above: b1 = (-asdq_p + Z_mid asdq_t)/(Z_below + Z_mid), down part
// c_below (b1 Z_below, -b1); b2 = (asdq_p + Z_mid asdq_t)/(Z_mid + Z_above),
// up part c_above (b2 Z_above, b2); the reflected remainder is dropped.
inline void vc_split(int meqn, int mt, const double* asdq, double zb, double cb, double zm,
                     double za, double ca, double* bm, double* bp) {
    const double b1 = (zm * asdq[mt - 1] - asdq[0]) / (zb + zm);
    const double b2 = (zm * asdq[mt - 1] + asdq[0]) / (zm + za);
    for (int m = 0; m < meqn; ++m) { bm[m] = 0.0; bp[m] = 0.0; }
    bm[0] = (cb * b1) * zb;
    bm[mt - 1] = -(cb * b1);
    bp[0] = (ca * b2) * za;
    bp[mt - 1] = ca * b2;
}

// rpt3(ixyz, icoor, imp): transverse split in the y-like (icoor 2) or z-like
// (icoor 3) direction of a fluctuation in cell i1 = i-2+imp (imp 0: the cell
// is irrelevant for constant coefficients; here aux is always present).
void rpt3_vc_acoustics(int ixyz, int icoor, int imp, int meqn, int mbc, int mx,
                       const Aux3& a1, const Aux3& a2, const Aux3& a3, const double* asdq,
                       double* bm, double* bp) {
    const int mt = vel_index(trans_dir(ixyz, icoor));
    const Slice Q{meqn, 1 - mbc};
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const int i1 = i - 2 + (imp == 0 ? 2 : imp);
        double zb, cb, zm, za, ca;
        if (icoor == 2) {
            zb = a1.at(1, i1, 2); cb = a1.at(2, i1, 2);
            zm = a2.at(1, i1, 2);
            za = a3.at(1, i1, 2); ca = a3.at(2, i1, 2);
        } else {
            zb = a2.at(1, i1, 1); cb = a2.at(2, i1, 1);
            zm = a2.at(1, i1, 2);
            za = a2.at(1, i1, 3); ca = a2.at(2, i1, 3);
        }
        vc_split(meqn, mt, &asdq[Q.at(1, i)], zb, cb, zm, za, ca, &bm[Q.at(1, i)], &bp[Q.at(1, i)]);
    }
}

// rptt3(ixyz, icoor, imp, impt): split, in direction icoor, a fluctuation
// already moved one cell in the other transverse direction (impt 1: down,
// 2: up), i.e. living at that neighbour of cell i1.
void rptt3_vc_acoustics(int ixyz, int icoor, int imp, int impt, int meqn, int mbc, int mx,
                        const Aux3& a1, const Aux3& a2, const Aux3& a3, const double* asdq,
                        double* bm, double* bp) {
    const int mt = vel_index(trans_dir(ixyz, icoor));
    const Slice Q{meqn, 1 - mbc};
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const int i1 = i - 2 + imp;
        double zb, cb, zm, za, ca;
        if (icoor == 2) {  // moved in z-like: level l = 1 (below) or 3 (above)
            const int l = impt == 1 ? 1 : 3;
            zb = a1.at(1, i1, l); cb = a1.at(2, i1, l);
            zm = a2.at(1, i1, l);
            za = a3.at(1, i1, l); ca = a3.at(2, i1, l);
        } else {  // moved in y-like: row aux1 (below) or aux3 (above)
            const Aux3& r = impt == 1 ? a1 : a3;
            zb = r.at(1, i1, 1); cb = r.at(2, i1, 1);
            zm = r.at(1, i1, 2);
            za = r.at(1, i1, 3); ca = r.at(2, i1, 3);
        }
        vc_split(meqn, mt, &asdq[Q.at(1, i)], zb, cb, zm, za, ca, &bm[Q.at(1, i)], &bp[Q.at(1, i)]);
    }
}

// flux3 for one slice; gadd/hadd laid out (m, k=1:2, l=-1:1, i).
void flux3(int ixyz, int meqn, int mwaves, int mbc, int mx, const double* q1d,
           const double* dtdx1d, double dtdy, double dtdz, const Aux3& a1, const Aux3& a2,
           const Aux3& a3, const int* method, const int* mthlim, double* qadd, double* fadd,
           double* gadd, double* hadd, double* cfl1d, bool use_fwave) {
    const int n = mx + 2 * mbc + 1;
    const Slice Q{meqn, 1 - mbc}, S{mwaves, 1 - mbc}, W{meqn * mwaves, 1 - mbc};
    auto D = [&](int i) { return dtdx1d[i - (1 - mbc)]; };
    auto G = [&](double* g, int m, int k, int l, int i) -> double& {
        return g[(m - 1) + meqn * ((k - 1) + 2 * ((l + 1) + 3 * (i - (1 - mbc))))];
    };
    std::vector<double> wave(meqn * mwaves * n), s(mwaves * n), amdq(meqn * n), apdq(meqn * n),
        cqxx(meqn * n, 0.0);
    std::vector<double> bmamdq(meqn * n), bmapdq(meqn * n), bpamdq(meqn * n), bpapdq(meqn * n),
        cmamdq(meqn * n), cmapdq(meqn * n), cpamdq(meqn * n), cpapdq(meqn * n),
        cmamdq2(meqn * n), cmapdq2(meqn * n), cpamdq2(meqn * n), cpapdq2(meqn * n),
        bmcqxxp(meqn * n), bpcqxxp(meqn * n), bmcqxxm(meqn * n), bpcqxxm(meqn * n),
        cmcqxxp(meqn * n), cpcqxxp(meqn * n), cmcqxxm(meqn * n), cpcqxxm(meqn * n),
        bmcmamdq(meqn * n), bmcmapdq(meqn * n), bpcmamdq(meqn * n), bpcmapdq(meqn * n),
        bmcpamdq(meqn * n), bmcpapdq(meqn * n), bpcpamdq(meqn * n), bpcpapdq(meqn * n);
    bool limit = false;
    for (int mw = 0; mw < mwaves; ++mw)
        if (mthlim[mw] > 0) limit = true;
    for (int i = 1 - mbc; i <= mx + mbc; ++i)
        for (int m = 1; m <= meqn; ++m) {
            qadd[Q.at(m, i)] = 0.0;
            fadd[Q.at(m, i)] = 0.0;
            for (int k = 1; k <= 2; ++k)
                for (int l = -1; l <= 1; ++l) { G(gadd, m, k, l, i) = 0.0; G(hadd, m, k, l, i) = 0.0; }
        }
    int m3, m4;
    if (method[2] < 0) { m3 = -1; m4 = 0; }
    else { m3 = method[2] / 10; m4 = method[2] - 10 * m3; }

    rpn3_vc_acoustics(ixyz, meqn, mbc, mx, q1d, a2, wave.data(), s.data(), amdq.data(), apdq.data());
    // forall: the first statement for every i, then the second
    for (int i = 1; i <= mx + 1; ++i)
        for (int m = 1; m <= meqn; ++m) qadd[Q.at(m, i)] = qadd[Q.at(m, i)] - D(i) * apdq[Q.at(m, i)];
    for (int i = 1; i <= mx + 1; ++i)
        for (int m = 1; m <= meqn; ++m)
            qadd[Q.at(m, i - 1)] = qadd[Q.at(m, i - 1)] - D(i - 1) * amdq[Q.at(m, i)];
    double c1 = 0.0;
    for (int i = 1; i <= mx + 1; ++i)
        for (int mw = 1; mw <= mwaves; ++mw) {
            const double sm = s[S.at(mw, i)];
            c1 = std::fmax(std::fmax(c1, D(i) * sm), -D(i - 1) * sm);
        }
    *cfl1d = c1;
    if (method[1] != 1) {
        if (limit) limiter(mx, meqn, mwaves, mbc, mx, wave.data(), s.data(), mthlim);
        for (int i = 2 - mbc; i <= mx + mbc; ++i) {
            const double dtdxave = 0.5 * (D(i - 1) + D(i));
            for (int m = 1; m <= meqn; ++m) cqxx[Q.at(m, i)] = 0.0;
            for (int mw = 1; mw <= mwaves; ++mw) {
                const double sm = s[S.at(mw, i)];
                const double coef = use_fwave ? 0.5 * std::copysign(1.0, sm) * (1.0 - std::fabs(sm) * dtdxave)
                                              : 0.5 * std::fabs(sm) * (1.0 - std::fabs(sm) * dtdxave);
                const double* wv = &wave[W.at(1, i)] + (mw - 1) * meqn;
                for (int m = 1; m <= meqn; ++m) cqxx[Q.at(m, i)] = cqxx[Q.at(m, i)] + coef * wv[m - 1];
            }
            for (int m = 1; m <= meqn; ++m) fadd[Q.at(m, i)] = fadd[Q.at(m, i)] + cqxx[Q.at(m, i)];
        }
    }
    if (m3 <= 0) return;
    rpt3_vc_acoustics(ixyz, 2, 1, meqn, mbc, mx, a1, a2, a3, amdq.data(), bmamdq.data(), bpamdq.data());
    rpt3_vc_acoustics(ixyz, 2, 2, meqn, mbc, mx, a1, a2, a3, apdq.data(), bmapdq.data(), bpapdq.data());
    rpt3_vc_acoustics(ixyz, 3, 1, meqn, mbc, mx, a1, a2, a3, amdq.data(), cmamdq.data(), cpamdq.data());
    rpt3_vc_acoustics(ixyz, 3, 2, meqn, mbc, mx, a1, a2, a3, apdq.data(), cmapdq.data(), cpapdq.data());
    if (m3 == 2) {
        // maux > 0: split cqxx with imp = 1 and 2 in each transverse direction.
        // (src/3d/flux3.f90:331 passes an undefined scalar as aux3 for the
        // z-like imp=1 split; the z-like split reads only aux2, so aux3 is
        // passed here.)
        rpt3_vc_acoustics(ixyz, 2, 1, meqn, mbc, mx, a1, a2, a3, cqxx.data(), bmcqxxm.data(), bpcqxxm.data());
        rpt3_vc_acoustics(ixyz, 2, 2, meqn, mbc, mx, a1, a2, a3, cqxx.data(), bmcqxxp.data(), bpcqxxp.data());
        rpt3_vc_acoustics(ixyz, 3, 1, meqn, mbc, mx, a1, a2, a3, cqxx.data(), cmcqxxm.data(), cpcqxxm.data());
        rpt3_vc_acoustics(ixyz, 3, 2, meqn, mbc, mx, a1, a2, a3, cqxx.data(), cmcqxxp.data(), cpcqxxp.data());
    }
    for (int i = 0; i <= mx + 2; ++i)
        for (int m = 1; m <= meqn; ++m) {
            const int x = Q.at(m, i);
            if (m4 == 1) {
                cpapdq2[x] = cpapdq[x]; cpamdq2[x] = cpamdq[x];
                cmapdq2[x] = cmapdq[x]; cmamdq2[x] = cmamdq[x];
            } else if (m4 == 2) {
                cpapdq2[x] = cpapdq[x] - 3.0 * cpcqxxp[x];
                cpamdq2[x] = cpamdq[x] + 3.0 * cpcqxxm[x];
                cmapdq2[x] = cmapdq[x] - 3.0 * cmcqxxp[x];
                cmamdq2[x] = cmamdq[x] + 3.0 * cmcqxxm[x];
            }
        }
    if (m4 > 0) {
        rptt3_vc_acoustics(ixyz, 2, 2, 2, meqn, mbc, mx, a1, a2, a3, cpapdq2.data(), bmcpapdq.data(), bpcpapdq.data());
        rptt3_vc_acoustics(ixyz, 2, 1, 2, meqn, mbc, mx, a1, a2, a3, cpamdq2.data(), bmcpamdq.data(), bpcpamdq.data());
        rptt3_vc_acoustics(ixyz, 2, 2, 1, meqn, mbc, mx, a1, a2, a3, cmapdq2.data(), bmcmapdq.data(), bpcmapdq.data());
        rptt3_vc_acoustics(ixyz, 2, 1, 1, meqn, mbc, mx, a1, a2, a3, cmamdq2.data(), bmcmamdq.data(), bpcmamdq.data());
    }
    const double sixth = 1.0 / 6.0;
    auto trans_updates = [&](double* g, double dtt, const std::vector<double>& mam,
                             const std::vector<double>& pam, const std::vector<double>& map,
                             const std::vector<double>& pap, const std::vector<double>& pmcqm,
                             const std::vector<double>& ppcqm, const std::vector<double>& pmcqp,
                             const std::vector<double>& ppcqp) {
        for (int i = 1; i <= mx + 1; ++i)
            for (int m = 1; m <= meqn; ++m) {
                const int x = Q.at(m, i);
                G(g, m, 1, 0, i - 1) = G(g, m, 1, 0, i - 1) - 0.5 * D(i - 1) * mam[x];
                G(g, m, 2, 0, i - 1) = G(g, m, 2, 0, i - 1) - 0.5 * D(i - 1) * pam[x];
                G(g, m, 1, 0, i) = G(g, m, 1, 0, i) - 0.5 * D(i) * map[x];
                G(g, m, 2, 0, i) = G(g, m, 2, 0, i) - 0.5 * D(i) * pap[x];
                if (m4 > 0) {
                    G(g, m, 2, 0, i) = G(g, m, 2, 0, i) + sixth * D(i) * dtt * (bpcpapdq[x] - bpcmapdq[x]);
                    G(g, m, 1, 0, i) = G(g, m, 1, 0, i) + sixth * D(i) * dtt * (bmcpapdq[x] - bmcmapdq[x]);
                    G(g, m, 2, 1, i) = G(g, m, 2, 1, i) - sixth * D(i) * dtt * bpcpapdq[x];
                    G(g, m, 1, 1, i) = G(g, m, 1, 1, i) - sixth * D(i) * dtt * bmcpapdq[x];
                    G(g, m, 2, -1, i) = G(g, m, 2, -1, i) + sixth * D(i) * dtt * bpcmapdq[x];
                    G(g, m, 1, -1, i) = G(g, m, 1, -1, i) + sixth * D(i) * dtt * bmcmapdq[x];
                    G(g, m, 2, 0, i - 1) = G(g, m, 2, 0, i - 1) + sixth * D(i - 1) * dtt * (bpcpamdq[x] - bpcmamdq[x]);
                    G(g, m, 1, 0, i - 1) = G(g, m, 1, 0, i - 1) + sixth * D(i - 1) * dtt * (bmcpamdq[x] - bmcmamdq[x]);
                    G(g, m, 2, 1, i - 1) = G(g, m, 2, 1, i - 1) - sixth * D(i - 1) * dtt * bpcpamdq[x];
                    G(g, m, 1, 1, i - 1) = G(g, m, 1, 1, i - 1) - sixth * D(i - 1) * dtt * bmcpamdq[x];
                    G(g, m, 2, -1, i - 1) = G(g, m, 2, -1, i - 1) + sixth * D(i - 1) * dtt * bpcmamdq[x];
                    G(g, m, 1, -1, i - 1) = G(g, m, 1, -1, i - 1) + sixth * D(i - 1) * dtt * bmcmamdq[x];
                }
                if (m3 < 2) continue;
                G(g, m, 2, 0, i) = G(g, m, 2, 0, i) + D(i) * ppcqp[x];
                G(g, m, 1, 0, i) = G(g, m, 1, 0, i) + D(i) * pmcqp[x];
                G(g, m, 2, 0, i - 1) = G(g, m, 2, 0, i - 1) - D(i - 1) * ppcqm[x];
                G(g, m, 1, 0, i - 1) = G(g, m, 1, 0, i - 1) - D(i - 1) * pmcqm[x];
            }
    };
    // G fluxes (y-like), src/3d/flux3.f90:381-447
    trans_updates(gadd, dtdz, bmamdq, bpamdq, bmapdq, bpapdq, bmcqxxm, bpcqxxm, bmcqxxp, bpcqxxp);
    if (m4 == 2)
        for (int i = 0; i <= mx + 2; ++i)
            for (int m = 1; m <= meqn; ++m) {
                const int x = Q.at(m, i);
                bpapdq[x] = bpapdq[x] - 3.0 * bpcqxxp[x];
                bpamdq[x] = bpamdq[x] + 3.0 * bpcqxxm[x];
                bmapdq[x] = bmapdq[x] - 3.0 * bmcqxxp[x];
                bmamdq[x] = bmamdq[x] + 3.0 * bmcqxxm[x];
            }
    if (m4 > 0) {
        rptt3_vc_acoustics(ixyz, 3, 2, 2, meqn, mbc, mx, a1, a2, a3, bpapdq.data(), bmcpapdq.data(), bpcpapdq.data());
        rptt3_vc_acoustics(ixyz, 3, 1, 2, meqn, mbc, mx, a1, a2, a3, bpamdq.data(), bmcpamdq.data(), bpcpamdq.data());
        rptt3_vc_acoustics(ixyz, 3, 2, 1, meqn, mbc, mx, a1, a2, a3, bmapdq.data(), bmcmapdq.data(), bpcmapdq.data());
        rptt3_vc_acoustics(ixyz, 3, 1, 1, meqn, mbc, mx, a1, a2, a3, bmamdq.data(), bmcmamdq.data(), bpcmamdq.data());
    }
    // H fluxes (z-like), src/3d/flux3.f90:513-609
    trans_updates(hadd, dtdy, cmamdq, cpamdq, cmapdq, cpapdq, cmcqxxm, cpcqxxm, cmcqxxp, cpcqxxp);
}

}  // namespace

extern "C" {

// bc3 (src/3d/bc3.f): x, then y, then z, each over all other indices
// including ghosts; mthbc 1 extrap, 2 periodic, 3 wall (negate q(2|3|4)).
// bc code 10 at z-upper is the piston wall of
// examples/acoustics_3d_heterogeneous/bc3.f:596-606 (reflect, then
// q(4) = 2 s - q(4) with s = -exp(-500 r^2) exp(-500 t^2) for t < 0.1).
int orc_bc3(int meqn, int mbc, int mx, int my, int mz, double* q, const int* mthbc, double t,
            double xlower, double ylower, double dx, double dy) {
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    auto Q = [&](int m, int i, int j, int k) -> double& {
        return q[(m - 1) + meqn * ((i - (1 - mbc)) + nx * ((j - (1 - mbc)) + ny * (k - (1 - mbc))))];
    };
    const int n[3] = {mx, my, mz};
    for (int d = 0; d < 3; ++d)
        for (int side = 0; side < 2; ++side) {
            const int code = mthbc[2 * d + side];
            if (!(code >= 1 && code <= 3) && !(code == 10 && d == 2 && side == 1)) return -1;
        }
    for (int d = 0; d < 3; ++d) {
        for (int side = 0; side < 2; ++side) {
            const int code = mthbc[2 * d + side];
            for (int g = 1; g <= mbc; ++g) {
                const int dst = side == 0 ? 1 - g : n[d] + g;
                int src;
                if (code == 1) src = side == 0 ? 1 : n[d];
                else if (code == 2) src = side == 0 ? n[d] + 1 - g : g;
                else src = side == 0 ? g : n[d] + 1 - g;  // wall / piston: reflect
                for (int k = 1 - mbc; k <= mz + mbc; ++k)
                    for (int j = 1 - mbc; j <= my + mbc; ++j)
                        for (int i = 1 - mbc; i <= mx + mbc; ++i) {
                            int I[3] = {i, j, k};
                            if (I[d] != dst) continue;
                            int S[3] = {i, j, k};
                            S[d] = src;
                            for (int m = 1; m <= meqn; ++m) Q(m, i, j, k) = Q(m, S[0], S[1], S[2]);
                            if (code == 3) Q(2 + d, i, j, k) = -Q(2 + d, S[0], S[1], S[2]);
                            if (code == 10) {
                                double sp = 0.0;
                                if (t < 0.1) {
                                    const double xi = xlower + (i - 0.5) * dx;
                                    const double yj = ylower + (j - 0.5) * dy;
                                    const double r2 = (xi * xi + yj * yj);
                                    sp = -std::exp(-500.0 * r2) * std::exp(-(500.0 * (t * t)));
                                    if (std::fabs(sp) < 1e-6) sp = 0.0;
                                }
                                Q(4, i, j, k) = 2.0 * sp - Q(4, S[0], S[1], S[2]);
                            }
                        }
            }
        }
    }
    return 0;
}

// step3: x-, y-, z-sweeps, each over 2x2 blocks of slices in the colour
// order of the reference's OpenMP loops (koffset, joffset / ioffset), which
// fixes every cell's order of accumulation.
int orc_step3(int meqn, int mwaves, int maux, int mbc, int mx, int my, int mz, const double* qold,
              double* qnew, const double* aux, double dx, double dy, double dz, double dt,
              const int* method, const int* mthlim, int use_fwave, double* cfl_out) {
    if (g_solver != ORC_VC_ACOUSTICS_3D || maux < 2) return -1;
    if (method[5] != 0) return -3;  // capacity not restated for 3D
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    const int maxm = std::max(mx, std::max(my, mz));
    const int n1 = maxm + 2 * mbc;
    auto QO = [&](int m, int i, int j, int k) {
        return qold[(m - 1) + meqn * ((i - (1 - mbc)) + nx * ((j - (1 - mbc)) + ny * (k - (1 - mbc))))];
    };
    auto QN = [&](int m, int i, int j, int k) -> double& {
        return qnew[(m - 1) + meqn * ((i - (1 - mbc)) + nx * ((j - (1 - mbc)) + ny * (k - (1 - mbc))))];
    };
    auto AX = [&](int ma, int i, int j, int k) {
        return aux[(ma - 1) + maux * ((i - (1 - mbc)) + nx * ((j - (1 - mbc)) + ny * (k - (1 - mbc))))];
    };
    // flux3's work arrays (one set per thread in the OpenMP timing build)
    struct Work3 {
        std::vector<double> q1d, dtd1d, qadd, fadd, gadd, hadd, x1, x2, x3;
        Work3(int meqn, int maux, int n1)
            : q1d(meqn * n1), dtd1d(n1), qadd(meqn * n1), fadd(meqn * n1), gadd(meqn * 6 * n1),
              hadd(meqn * 6 * n1), x1(maux * n1 * 3), x2(maux * n1 * 3), x3(maux * n1 * 3) {}
    };
    const Slice Q{meqn, 1 - mbc};
    const double dtdx = dt / dx, dtdy = dt / dy, dtdz = dt / dz;
    double cfl = 0.0;
    const int dims[3] = {mx, my, mz};
    const double dtd[3] = {dtdx, dtdy, dtdz};
    auto Gv = [&](const std::vector<double>& g, int m, int k, int l, int i) {
        return g[(m - 1) + meqn * ((k - 1) + 2 * ((l + 1) + 3 * (i - (1 - mbc))))];
    };
    for (int ixyz = 1; ixyz <= 3; ++ixyz) {
        // directions: n = normal, e1 = y-like, e2 = z-like
        const int dn = ixyz - 1, d1 = trans_dir(ixyz, 2) - 1, d2 = trans_dir(ixyz, 3) - 1;
        const int len = dims[dn];
        // colour, block and slice loops run over the two slice indices in
        // the order of step3.f90: x: (k, j), y: (k, i), z: (j, i), i.e. the
        // higher-numbered axis outermost
        const int outer = std::max(d1, d2);  // slowest slice index
        const int inner = std::min(d1, d2);
        const int nblk_o = (dims[outer] + 2 + 1) / 2, nblk_i = (dims[inner] + 2 + 1) / 2;
        auto slice = [&](int so, int si, Work3& w, double& cfl) {
            std::vector<double>& q1d = w.q1d;
            std::vector<double>& qadd = w.qadd;
            std::vector<double>& fadd = w.fadd;
            std::vector<double>& gadd = w.gadd;
            std::vector<double>& hadd = w.hadd;
            int P[3];
            P[outer] = so;
            P[inner] = si;
            auto cell = [&](int a, int de1, int de2, int* c) {
                c[dn] = a;
                c[d1] = P[d1] + de1;
                c[d2] = P[d2] + de2;
            };
            for (int i = 0; i < n1; ++i) w.dtd1d[i] = dtd[dn];
            for (int a = 1 - mbc; a <= len + mbc; ++a) {
                int c[3];
                cell(a, 0, 0, c);
                for (int m = 1; m <= meqn; ++m) q1d[Q.at(m, a)] = QO(m, c[0], c[1], c[2]);
            }
            // aux1/aux2/aux3 = e1 offset -1/0/+1; third index = e2 offset -1..1
            for (int a = 1 - mbc; a <= len + mbc; ++a)
                for (int l = -1; l <= 1; ++l)
                    for (int ma = 1; ma <= maux; ++ma) {
                        const int o = (ma - 1) + maux * ((a - (1 - mbc)) + n1 * (l + 1));
                        int c[3];
                        cell(a, -1, l, c); w.x1[o] = AX(ma, c[0], c[1], c[2]);
                        cell(a, 0, l, c); w.x2[o] = AX(ma, c[0], c[1], c[2]);
                        cell(a, 1, l, c); w.x3[o] = AX(ma, c[0], c[1], c[2]);
                    }
            const Aux3 A1{w.x1.data(), maux, 1 - mbc, n1}, A2{w.x2.data(), maux, 1 - mbc, n1},
                A3{w.x3.data(), maux, 1 - mbc, n1};
            double cfl1d;
            flux3(ixyz, meqn, mwaves, mbc, len, q1d.data(), w.dtd1d.data(), dtd[d1],
                  dtd[d2], A1, A2, A3, method, mthlim, qadd.data(), fadd.data(),
                  gadd.data(), hadd.data(), &cfl1d, use_fwave != 0);
            cfl = std::fmax(cfl, cfl1d);
            const double te1 = dtd[d1], te2 = dtd[d2], tn = dtd[dn];
            for (int a = 1; a <= len; ++a)
                for (int de2 = -1; de2 <= 1; ++de2)
                    for (int de1 = -1; de1 <= 1; ++de1)
                        for (int m = 1; m <= meqn; ++m) {
                            int c[3];
                            cell(a, de1, de2, c);
                            double& v = QN(m, c[0], c[1], c[2]);
                            if (de1 == 0 && de2 == 0) {
                                v = v + qadd[Q.at(m, a)] -
                                    tn * (fadd[Q.at(m, a + 1)] - fadd[Q.at(m, a)]) -
                                    te1 * (Gv(gadd, m, 2, 0, a) - Gv(gadd, m, 1, 0, a)) -
                                    te2 * (Gv(hadd, m, 2, 0, a) - Gv(hadd, m, 1, 0, a));
                                continue;
                            }
                            // e1 (G) term, then e2 (H) term
                            if (de1 == -1) v = v - te1 * Gv(gadd, m, 1, de2, a);
                            else if (de1 == 0) v = v - te1 * (Gv(gadd, m, 2, de2, a) - Gv(gadd, m, 1, de2, a));
                            else v = v + te1 * Gv(gadd, m, 2, de2, a);
                            if (de2 == -1) v = v - te2 * Gv(hadd, m, 1, de1, a);
                            else if (de2 == 0) v = v - te2 * (Gv(hadd, m, 2, de1, a) - Gv(hadd, m, 1, de1, a));
                            else v = v + te2 * Gv(hadd, m, 2, de1, a);
                        }
        };
        auto block = [&](int ob, int ib, Work3& w, double& cfl) {
            for (int so = ob * 2; so <= std::min(ob * 2 + 1, dims[outer] + 1); ++so)
                for (int si = ib * 2; si <= std::min(ib * 2 + 1, dims[inner] + 1); ++si)
                    slice(so, si, w, cfl);
        };
        if (g_threads > 1) {
            // Timing variant: blocks of one colour are at least three slices
            // apart, so they run in parallel as step3.f90:132-186 runs them;
            // each cell still receives its contributions in the serial order.
            const int nt = g_threads;
            std::vector<Work3> ws;
            for (int t = 0; t < nt; ++t) ws.emplace_back(meqn, maux, n1);
            std::vector<double> cfls(nt, 0.0);
            for (int oo = 0; oo <= 1; ++oo)
                for (int io = 0; io <= 1; ++io) {
                    const int no = (nblk_o - oo + 1) / 2, ni = (nblk_i - io + 1) / 2;
                    parallel_items(no * ni, nt, [&](int k, int t) {
                        block(oo + 2 * (k / ni), io + 2 * (k % ni), ws[t], cfls[t]);
                    });
                }
            for (double c : cfls) cfl = std::fmax(cfl, c);
        } else {
            Work3 w(meqn, maux, n1);
            for (int oo = 0; oo <= 1; ++oo)
                for (int io = 0; io <= 1; ++io)
                    for (int ob = oo; ob <= nblk_o - 1; ob += 2)
                        for (int ib = io; ib <= nblk_i - 1; ib += 2) block(ob, ib, w, cfl);
        }
    }
    *cfl_out = cfl;
    return 0;
}

// ----------------------------------------------------------------- step3ds ---
// src/3d/step3ds.f90:3-408: one directional sweep of dimensional splitting
// (idir 1 = x, 2 = y, 3 = z).  The slices cover one ghost layer across
// (x-sweeps: j = 0..my+1, k = 0..mz+1, and likewise for y and z); each slice
// updates its cells 1..len with qadd and fadd only (flux3 returns before the
// transverse part when method(3) < 0).  qold may alias qnew.
int orc_step3ds(int meqn, int mwaves, int maux, int mbc, int mx, int my, int mz,
                const double* qold, double* qnew, const double* aux, double dx, double dy,
                double dz, double dt, const int* method, const int* mthlim, int idir,
                int use_fwave, double* cfl_out) {
    if (g_solver != ORC_VC_ACOUSTICS_3D || maux < 2) return -1;
    if (method[5] != 0) return -3;  // capacity not restated for 3D
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    const int maxm = std::max(mx, std::max(my, mz));
    const int n1 = maxm + 2 * mbc;
    auto idx = [&](int i, int j, int k) {
        return (size_t)(i - (1 - mbc)) + (size_t)nx * ((j - (1 - mbc)) + (size_t)ny * (k - (1 - mbc)));
    };
    std::vector<double> q1d(meqn * n1), dtd1d(n1), qadd(meqn * n1), fadd(meqn * n1),
        gadd(meqn * 6 * n1), hadd(meqn * 6 * n1), x2(maux * n1 * 3), xdummy(maux * n1 * 3, 0.0);
    const Slice Q{meqn, 1 - mbc};
    const int dims[3] = {mx, my, mz};
    const double dtd[3] = {dt / dx, dt / dy, dt / dz};
    const int dn = idir - 1, d1 = trans_dir(idir, 2) - 1, d2 = trans_dir(idir, 3) - 1;
    const int len = dims[dn];
    const double tn = dtd[dn];
    for (int i = 0; i < n1; ++i) dtd1d[i] = tn;
    const int outer = std::max(d1, d2), inner = std::min(d1, d2);
    double cfl = 0.0;
    for (int so = 0; so <= dims[outer] + 1; ++so)
        for (int si = 0; si <= dims[inner] + 1; ++si) {
            int P[3];
            P[outer] = so;
            P[inner] = si;
            auto cell = [&](int a, int de2, int* c) {
                c[dn] = a;
                c[d1] = P[d1];
                c[d2] = P[d2] + de2;
            };
            for (int a = 1 - mbc; a <= len + mbc; ++a) {
                int c[3];
                cell(a, 0, c);
                for (int m = 1; m <= meqn; ++m) q1d[Q.at(m, a)] = qold[(m - 1) + meqn * idx(c[0], c[1], c[2])];
            }
            // only aux2 is gathered (its e2 offsets -1..1); flux3 reads its middle
            for (int a = 1 - mbc; a <= len + mbc; ++a)
                for (int l = -1; l <= 1; ++l)
                    for (int ma = 1; ma <= maux; ++ma) {
                        int c[3];
                        cell(a, l, c);
                        x2[(ma - 1) + maux * ((a - (1 - mbc)) + n1 * (l + 1))] =
                            aux[(ma - 1) + maux * idx(c[0], c[1], c[2])];
                    }
            const Aux3 A2{x2.data(), maux, 1 - mbc, n1}, AD{xdummy.data(), maux, 1 - mbc, n1};
            double cfl1d;
            flux3(idir, meqn, mwaves, mbc, len, q1d.data(), dtd1d.data(), dtd[d1], dtd[d2], AD,
                  A2, AD, method, mthlim, qadd.data(), fadd.data(), gadd.data(), hadd.data(),
                  &cfl1d, use_fwave != 0);
            cfl = std::fmax(cfl, cfl1d);
            for (int a = 1; a <= len; ++a) {
                int c[3];
                cell(a, 0, c);
                for (int m = 1; m <= meqn; ++m) {
                    double& v = qnew[(m - 1) + meqn * idx(c[0], c[1], c[2])];
                    v = v + qadd[Q.at(m, a)] - tn * (fadd[Q.at(m, a + 1)] - fadd[Q.at(m, a)]);
                }
            }
        }
    *cfl_out = cfl;
    return 0;
}

// ------------------------------------------------------------------ dimsp3 ---
// src/3d/dimsp3.f:1-87: Godunov splitting only (x, y, z by dt each); a sweep
// whose Courant number exceeds cflv(1) ends the step with that number.
int orc_dimsp3(int meqn, int mwaves, int maux, int mbc, int mx, int my, int mz,
               const double* qold, double* qnew, const double* aux, double dx, double dy,
               double dz, double dt, const int* method, const int* mthlim, const double* cflv,
               int use_fwave, double* cfl_out) {
    double c[3];
    for (int d = 1; d <= 3; ++d) {
        const int rc = orc_step3ds(meqn, mwaves, maux, mbc, mx, my, mz, d == 1 ? qold : qnew, qnew,
                                   aux, dx, dy, dz, dt, method, mthlim, d, use_fwave, &c[d - 1]);
        if (rc) return rc;
        if (d < 3 && c[d - 1] > cflv[0]) { *cfl_out = c[d - 1]; return 0; }
    }
    *cfl_out = std::fmax(std::fmax(c[0], c[1]), c[2]);
    return 0;
}

// claw3 (src/3d/claw3.f:738-928): the control flow of claw2 around bc3/step3.
int orc_claw3(int meqn, int mwaves, int maux, int mbc, int mx, int my, int mz, double* q,
              const double* aux, double xlower, double ylower, double dx, double dy, double dz,
              double tstart, double* tend_io, double* dtv, double* cflv, int* nv,
              const int* method, const int* mthlim, const int* mthbc, int use_fwaves) {
    const double tend = *tend_io;
    int info = 0;
    double t = tstart;
    int maxn = nv[0];
    double dt = dtv[0];
    double cflmax = 0.0, dtmin = dt, dtmax = dt, cfl = 0.0;
    nv[1] = 0;
    const size_t nq = (size_t)meqn * (mx + 2 * mbc) * (my + 2 * mbc) * (mz + 2 * mbc);
    std::vector<double> qwork(nq);
    if (method[0] == 0) {
        if (tend < tstart) maxn = 1;
        else {
            maxn = (int)std::lround((tend - tstart) / dt);
            if (std::fabs(maxn * dt - (tend - tstart)) > 1e-5 * (tend - tstart)) { info = 2; goto done; }
        }
    }
    if (method[0] == 1 && cflv[1] > cflv[0]) { info = 3; goto done; }
    if (maxn == 0) goto done;
    for (int n = 1; n <= maxn; ++n) {
        const double told = t;
        if (told + dt > tend && tstart < tend) dt = tend - told;
        for (;;) {
            if (orc_bc3(meqn, mbc, mx, my, mz, q, mthbc, told, xlower, ylower, dx, dy) != 0) { info = -2; goto done; }
            std::memcpy(qwork.data(), q, nq * sizeof(double));
            const int rc = method[2] >= 0
                               ? orc_step3(meqn, mwaves, maux, mbc, mx, my, mz, qwork.data(), q,
                                           aux, dx, dy, dz, dt, method, mthlim, use_fwaves, &cfl)
                               : orc_dimsp3(meqn, mwaves, maux, mbc, mx, my, mz, qwork.data(), q,
                                            aux, dx, dy, dz, dt, method, mthlim, cflv, use_fwaves,
                                            &cfl);
            if (rc != 0) { info = rc; goto done; }
            t = told + dt;
            if (cfl <= cflv[0]) { cflmax = std::fmax(cfl, cflmax); break; }
            t = told;
            std::memcpy(q, qwork.data(), nq * sizeof(double));
            if (method[0] == 1) { dt = std::fmin(dtv[1], dt * cflv[1] / cfl); continue; }
            cflmax = std::fmax(cfl, cflmax);
            goto done;
        }
        if (method[0] == 1) {
            if (cfl == 0.0) dt = dtv[1];
            else dt = std::fmin(dtv[1], dt * cflv[1] / cfl);
            dtmin = std::fmin(dt, dtmin);
            dtmax = std::fmax(dt, dtmax);
        }
        nv[1] = nv[1] + 1;
        if (t >= tend) break;
    }
done:
    if (method[0] == 1 && t < tend && nv[1] == maxn) info = 11;
    if (method[0] == 0 && cflmax > cflv[0]) info = 12;
    *tend_io = t;
    cflv[2] = cflmax;
    cflv[3] = cfl;
    dtv[2] = dtmin;
    dtv[3] = dtmax;
    dtv[4] = dt;
    return info;
}

// ================================================================ 1D path ===
// -------------------------------------------------------------------- bc1 ---
int orc_bc1(int meqn, int mbc, int mx, double* q, const int* mthbc) {
    auto Q = [&](int m, int i) -> double& { return q[(m - 1) + meqn * (i - (1 - mbc))]; };
    if (mthbc[0] < 1 || mthbc[0] > 3 || mthbc[1] < 1 || mthbc[1] > 3) return -1;
    for (int ibc = 1; ibc <= mbc; ++ibc) {
        for (int m = 1; m <= meqn; ++m) {
            if (mthbc[0] == 1) Q(m, 1 - ibc) = Q(m, 1);
            else if (mthbc[0] == 2) Q(m, 1 - ibc) = Q(m, mx + 1 - ibc);
            else Q(m, 1 - ibc) = Q(m, ibc);
        }
        if (mthbc[0] == 3) Q(2, 1 - ibc) = -Q(2, ibc);
    }
    for (int ibc = 1; ibc <= mbc; ++ibc) {
        for (int m = 1; m <= meqn; ++m) {
            if (mthbc[1] == 1) Q(m, mx + ibc) = Q(m, mx);
            else if (mthbc[1] == 2) Q(m, mx + ibc) = Q(m, ibc);
            else Q(m, mx + ibc) = Q(m, mx + 1 - ibc);
        }
        if (mthbc[1] == 3) Q(2, mx + ibc) = -Q(2, mx + 1 - ibc);
    }
    return 0;
}

// ------------------------------------------------------------------ step1 ---
// src/1d/step1.f90:4-170 — in-place Godunov update, then the limited
// second-order correction flux f (with the 0.5 folded into each term).
int orc_step1(int meqn, int mwaves, int mbc, int maux, int mx, double* q, const double* aux,
              double dx, double dt, const int* method, const int* mthlim, int use_fwave,
              double* cfl_out) {
    rp1_t rp1;
    if (g_solver == ORC_ACOUSTICS_1D) rp1 = rp1_acoustics;
    else if (g_solver == ORC_VC_ACOUSTICS_1D) rp1 = rp1_vc_acoustics;
    else if (g_solver == ORC_ADVECTION_1D) rp1 = rp1_advection;
    else if (g_solver == ORC_EULER_ROE_1D) rp1 = rp1_euler_roe;
    else return -1;
    const int n = mx + 2 * mbc;
    const Slice sl{meqn, 1 - mbc}, sv{mwaves, 1 - mbc}, w{meqn * mwaves, 1 - mbc};
    std::vector<double> f(meqn * (n + 1), 0.0), wave(meqn * mwaves * n), s(mwaves * n),
        amdq(meqn * n), apdq(meqn * n), dtdx(n);
    bool limit = false;
    for (int mw = 0; mw < mwaves; ++mw)
        if (mthlim[mw] > 0) limit = true;
    const int index_capa = method[5];
    auto D = [&](int i) { return dtdx[i - (1 - mbc)]; };
    for (int i = 1 - mbc; i <= mx + mbc; ++i) {
        if (index_capa > 0) {
            const double capa = aux[(index_capa - 1) + maux * (i - (1 - mbc))];
            if (capa <= 0.0) return -3;
            dtdx[i - (1 - mbc)] = dt / (dx * capa);
        } else {
            dtdx[i - (1 - mbc)] = dt / dx;
        }
    }
    rp1(mx, meqn, mwaves, maux, mbc, mx, q, q, aux, aux, wave.data(), s.data(), amdq.data(),
        apdq.data());
    for (int i = 1; i <= mx + 1; ++i) {
        for (int m = 1; m <= meqn; ++m)
            q[sl.at(m, i - 1)] = q[sl.at(m, i - 1)] - D(i - 1) * amdq[sl.at(m, i)];
        for (int m = 1; m <= meqn; ++m)
            q[sl.at(m, i)] = q[sl.at(m, i)] - D(i) * apdq[sl.at(m, i)];
    }
    double cfl = 0.0;
    for (int i = 1; i <= mx + 1; ++i)
        for (int mw = 1; mw <= mwaves; ++mw) {
            const double sm = s[sv.at(mw, i)];
            cfl = std::fmax(std::fmax(cfl, D(i) * sm), -D(i - 1) * sm);
        }
    *cfl_out = cfl;
    if (method[1] == 1) return 0;
    if (limit) limiter(mx, meqn, mwaves, mbc, mx, wave.data(), s.data(), mthlim);
    for (int i = 1; i <= mx + 1; ++i) {
        for (int m = 1; m <= meqn; ++m) f[sl.at(m, i)] = 0.0;
        const double dtdxave = 0.5 * (D(i - 1) + D(i));
        for (int mw = 1; mw <= mwaves; ++mw) {
            const double sm = s[sv.at(mw, i)];
            const double coef = use_fwave
                                    ? 0.5 * std::copysign(1.0, sm) * (1.0 - std::fabs(sm) * dtdxave)
                                    : 0.5 * std::fabs(sm) * (1.0 - std::fabs(sm) * dtdxave);
            const double* wv = &wave[w.at(1, i)] + (mw - 1) * meqn;
            for (int m = 1; m <= meqn; ++m) f[sl.at(m, i)] = f[sl.at(m, i)] + coef * wv[m - 1];
        }
    }
    // f(:, mx+2) is never set by the reference (it only feeds ghost cell
    // mx+1); it is zero here.
    for (int i = 1; i <= mx + 1; ++i)
        for (int m = 1; m <= meqn; ++m)
            q[sl.at(m, i)] = q[sl.at(m, i)] - D(i) * (f[sl.at(m, i + 1)] - f[sl.at(m, i)]);
    return 0;
}

// ------------------------------------------------------------------ claw1 ---
// src/1d/claw1.f:394-583.  Unlike claw2, the next dt is chosen before the
// Courant-number check (src/1d/claw1.f:520-529 vs 533-554).
int orc_claw1(int meqn, int mwaves, int maux, int mbc, int mx, double* q, const double* aux,
              double dx, double tstart, double* tend_io, double* dtv, double* cflv, int* nv,
              const int* method, const int* mthlim, const int* mthbc, int use_fwaves) {
    const double tend = *tend_io;
    int info = 0;
    double t = tstart;
    int maxn = nv[0];
    double dt = dtv[0];
    double cflmax = 0.0, dtmin = dt, dtmax = dt, cfl = 0.0;
    nv[1] = 0;
    const size_t nq = (size_t)meqn * (mx + 2 * mbc);
    std::vector<double> qwork(nq);
    if (method[0] == 0) {
        if (tend < tstart) maxn = 1;
        else {
            maxn = (int)std::lround((tend - tstart) / dt);
            if (std::fabs(maxn * dt - (tend - tstart)) > 1e-5 * (tend - tstart)) {
                info = 2;
                goto done;
            }
        }
    }
    if (method[0] == 1 && cflv[1] > cflv[0]) { info = 3; goto done; }
    if (maxn == 0) goto done;
    for (int n = 1; n <= maxn; ++n) {
        const double told = t;
        if (told + dt > tend && tstart < tend) dt = tend - told;
        if (method[0] == 1) std::memcpy(qwork.data(), q, nq * sizeof(double));
        for (;;) {
            t = told + dt;
            if (orc_bc1(meqn, mbc, mx, q, mthbc) != 0) { info = -2; goto done; }
            // src/1d/claw1.f:486-509: the source steps sit around step1, before
            // the Courant check (a rejected step restores q saved before bc1)
            if (method[4] == 2 && g_src == 1) src_radial_slice(mbc, mx, dx, q, meqn, dt / 2.0);
            const int rc = orc_step1(meqn, mwaves, mbc, maux, mx, q, aux, dx, dt, method, mthlim,
                                     use_fwaves, &cfl);
            if (rc != 0) { info = rc == -3 ? -3 : -1; goto done; }
            if (method[4] == 2 && g_src == 1) src_radial_slice(mbc, mx, dx, q, meqn, dt / 2.0);
            if (method[4] == 1 && g_src == 1) src_radial_slice(mbc, mx, dx, q, meqn, dt);
            if (method[0] == 1) {
                if (cfl > 0.0) {
                    dt = std::fmin(dtv[1], dt * cflv[1] / cfl);
                    dtmin = std::fmin(dt, dtmin);
                    dtmax = std::fmax(dt, dtmax);
                } else {
                    dt = dtv[1];
                }
            }
            if (cfl <= cflv[0]) {
                cflmax = std::fmax(cfl, cflmax);
                break;
            }
            t = told;
            std::memcpy(q, qwork.data(), nq * sizeof(double));
            if (method[0] == 1) continue;
            cflmax = std::fmax(cfl, cflmax);
            goto done;
        }
        nv[1] = nv[1] + 1;
        if (t >= tend) break;
    }
done:
    if (method[0] == 1 && t < tend && nv[1] == maxn) info = 11;
    if (method[0] == 0 && cflmax > cflv[0]) info = 12;
    *tend_io = t;
    cflv[2] = cflmax;
    cflv[3] = cfl;
    dtv[2] = dtmin;
    dtv[3] = dtmax;
    dtv[4] = dt;
    return info;
}

}  // extern "C"
