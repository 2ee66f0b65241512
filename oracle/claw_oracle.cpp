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
//   step1    : src/1d/step1.f90:4-170
//   bc1      : src/1d/bc1.f
//   claw1    : src/1d/claw1.f:394-583
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

extern "C" {

// ---------------------------------------------------------------- solvers ---
// Solver ids (shared numbering with the product's C-ABI, include/claw_b200.h).
enum {
    ORC_ACOUSTICS_2D = 1,      // q = (p, u, v);  params: rho, bulk
    ORC_VC_ADVECTION_2D = 2,   // q = (q);  aux = (u at left edge, v at bottom edge, capa)
    ORC_EULER_ROE_2D = 3,      // q = (rho, rho u, rho v, E);  params: gamma
    ORC_ACOUSTICS_1D = 11,     // q = (p, u);  params: rho, bulk
    ORC_VC_ACOUSTICS_1D = 12,  // q = (p, u);  aux = (Z, c)
    ORC_VC_ACOUSTICS_3D = 21,  // q = (p, u, v, w);  aux = (Z, c)
};

// Problem parameters: the analogue of the reference's /cparam/ common block
// (non-reentrant, exactly like the reference).
static int g_solver = 0;
static double g_rho = 1.0, g_bulk = 1.0, g_cc = 1.0, g_zz = 1.0, g_hz = 0.5;
static double g_gamma = 1.4;

int orc_set_solver(int solver_id, const double* params, int nparams) {
    g_solver = solver_id;
    if (solver_id == ORC_ACOUSTICS_2D || solver_id == ORC_ACOUSTICS_1D) {
        if (nparams < 2) return -1;
        g_rho = params[0];
        g_bulk = params[1];
        g_cc = std::sqrt(g_bulk / g_rho);
        g_zz = g_rho * g_cc;
        g_hz = 0.5 / g_zz;
    } else if (solver_id == ORC_EULER_ROE_2D) {
        if (nparams < 1) return -1;
        g_gamma = params[0];
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

bool pick2(int solver, rpn2_t* rpn, rpt2_t* rpt) {
    switch (solver) {
        case ORC_ACOUSTICS_2D: *rpn = rpn2_acoustics; *rpt = rpt2_acoustics; return true;
        case ORC_VC_ADVECTION_2D: *rpn = rpn2_vc_advection; *rpt = rpt2_vc_advection; return true;
        default: return false;
    }
}

}  // namespace

// Euler / 3D solvers and step3 live in claw_oracle_ext.cpp.
namespace orc_ext {
bool pick2_ext(int solver, rpn2_t* rpn, rpt2_t* rpt);
}

extern "C" {

// ------------------------------------------------------------------ step2 ---
// src/2d/step2.f90:2-251.  qold/qnew/aux in the reference layout with ghost
// cells; qnew must equal qold on entry.  Returns 0, or -1 for an unknown solver.
int orc_step2(int meqn, int mwaves, int maux, int mbc, int mx, int my, const double* qold,
              double* qnew, const double* aux, double dx, double dy, double dt,
              const int* method, const int* mthlim, int use_fwave, double* cfl_out) {
    rpn2_t rpn2;
    rpt2_t rpt2;
    if (!pick2(g_solver, &rpn2, &rpt2) && !orc_ext::pick2_ext(g_solver, &rpn2, &rpt2)) return -1;
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
    std::vector<double> qadd(meqn * n), fadd(meqn * n), gadd(2 * meqn * n), q1d(meqn * n);
    std::vector<double> dtdx1d(n), dtdy1d(n), aux1(std::max(maux, 1) * n),
        aux2(std::max(maux, 1) * n), aux3(std::max(maux, 1) * n);
    std::vector<double> wave(meqn * mwaves * n), s(mwaves * n), amdq(meqn * n), apdq(meqn * n),
        cqxx(meqn * n), bmasdq(meqn * n), bpasdq(meqn * n);
    const Slice sl{meqn, 1 - mbc}, sa{maux, 1 - mbc};
    auto GA = [&](int m, int k, int i) { return gadd[(m - 1) + meqn * (k - 1) + 2 * meqn * (i - (1 - mbc))]; };
    const int index_capa = method[5];
    double cfl = 0.0;
    const double dtdx = dt / dx, dtdy = dt / dy;
    if (index_capa == 0)
        for (int i = 0; i < n; ++i) { dtdx1d[i] = dtdx; dtdy1d[i] = dtdy; }

    // x-sweeps (src/2d/step2.f90:92-165)
    for (int j = 0; j <= my + 1; ++j) {
        for (int i = 1 - mbc; i <= mx + mbc; ++i)
            for (int m = 1; m <= meqn; ++m) q1d[sl.at(m, i)] = Q(qold, m, i, j);
        if (index_capa > 0)
            for (int i = 1 - mbc; i <= mx + mbc; ++i) dtdx1d[i - (1 - mbc)] = dtdx / A(index_capa, i, j);
        if (maux > 0)
            for (int i = 1 - mbc; i <= mx + mbc; ++i)
                for (int ma = 1; ma <= maux; ++ma) {
                    aux1[sa.at(ma, i)] = A(ma, i, j - 1);
                    aux2[sa.at(ma, i)] = A(ma, i, j);
                    aux3[sa.at(ma, i)] = A(ma, i, j + 1);
                }
        double cfl1d;
        flux2(1, maxm, meqn, mwaves, maux, mbc, mx, q1d.data(), dtdx1d.data(), aux1.data(),
              aux2.data(), aux3.data(), method, mthlim, qadd.data(), fadd.data(), gadd.data(),
              &cfl1d, wave.data(), s.data(), amdq.data(), apdq.data(), cqxx.data(),
              bmasdq.data(), bpasdq.data(), rpn2, rpt2, use_fwave != 0);
        cfl = std::fmax(cfl, cfl1d);
        if (index_capa == 0) {
            for (int i = 1; i <= mx; ++i)
                for (int m = 1; m <= meqn; ++m) {
                    QN(m, i, j) = QN(m, i, j) + qadd[sl.at(m, i)] -
                                  dtdx * (fadd[sl.at(m, i + 1)] - fadd[sl.at(m, i)]) -
                                  dtdy * (GA(m, 2, i) - GA(m, 1, i));
                    QN(m, i, j - 1) = QN(m, i, j - 1) - dtdy * GA(m, 1, i);
                    QN(m, i, j + 1) = QN(m, i, j + 1) + dtdy * GA(m, 2, i);
                }
        } else {
            for (int i = 1; i <= mx; ++i)
                for (int m = 1; m <= meqn; ++m) {
                    QN(m, i, j) = QN(m, i, j) + qadd[sl.at(m, i)] -
                                  (dtdx * (fadd[sl.at(m, i + 1)] - fadd[sl.at(m, i)]) +
                                   dtdy * (GA(m, 2, i) - GA(m, 1, i))) /
                                      A(index_capa, i, j);
                    QN(m, i, j - 1) = QN(m, i, j - 1) - dtdy * GA(m, 1, i) / A(index_capa, i, j - 1);
                    QN(m, i, j + 1) = QN(m, i, j + 1) + dtdy * GA(m, 2, i) / A(index_capa, i, j + 1);
                }
        }
    }

    // y-sweeps (src/2d/step2.f90:173-248)
    for (int i = 0; i <= mx + 1; ++i) {
        for (int j = 1 - mbc; j <= my + mbc; ++j)
            for (int m = 1; m <= meqn; ++m) q1d[sl.at(m, j)] = Q(qold, m, i, j);
        if (index_capa > 0)
            for (int j = 1 - mbc; j <= my + mbc; ++j) dtdy1d[j - (1 - mbc)] = dtdy / A(index_capa, i, j);
        if (maux > 0)
            for (int j = 1 - mbc; j <= my + mbc; ++j)
                for (int ma = 1; ma <= maux; ++ma) {
                    aux1[sa.at(ma, j)] = A(ma, i - 1, j);
                    aux2[sa.at(ma, j)] = A(ma, i, j);
                    aux3[sa.at(ma, j)] = A(ma, i + 1, j);
                }
        double cfl1d;
        flux2(2, maxm, meqn, mwaves, maux, mbc, my, q1d.data(), dtdy1d.data(), aux1.data(),
              aux2.data(), aux3.data(), method, mthlim, qadd.data(), fadd.data(), gadd.data(),
              &cfl1d, wave.data(), s.data(), amdq.data(), apdq.data(), cqxx.data(),
              bmasdq.data(), bpasdq.data(), rpn2, rpt2, use_fwave != 0);
        cfl = std::fmax(cfl, cfl1d);
        if (index_capa == 0) {
            for (int j = 1; j <= my; ++j)
                for (int m = 1; m <= meqn; ++m) {
                    QN(m, i, j) = QN(m, i, j) +
                                  (qadd[sl.at(m, j)] -
                                   dtdy * (fadd[sl.at(m, j + 1)] - fadd[sl.at(m, j)]) -
                                   dtdx * (GA(m, 2, j) - GA(m, 1, j)));
                    QN(m, i - 1, j) = QN(m, i - 1, j) - dtdx * GA(m, 1, j);
                    QN(m, i + 1, j) = QN(m, i + 1, j) + dtdx * GA(m, 2, j);
                }
        } else {
            for (int j = 1; j <= my; ++j)
                for (int m = 1; m <= meqn; ++m) {
                    QN(m, i, j) = QN(m, i, j) + qadd[sl.at(m, j)] -
                                  (dtdy * (fadd[sl.at(m, j + 1)] - fadd[sl.at(m, j)]) +
                                   dtdx * (GA(m, 2, j) - GA(m, 1, j))) /
                                      A(index_capa, i, j);
                    QN(m, i - 1, j) = QN(m, i - 1, j) - dtdx * GA(m, 1, j) / A(index_capa, i - 1, j);
                    QN(m, i + 1, j) = QN(m, i + 1, j) + dtdx * GA(m, 2, j) / A(index_capa, i + 1, j);
                }
        }
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
    if (method[5] > method[6]) { info = 5; goto done; }
    if (method[1] < method[2]) { info = 6; goto done; }
    if (maxn == 0) goto done;
    for (int n = 1; n <= maxn; ++n) {
        const double told = t;
        if (told + dt > tend && tstart < tend) dt = tend - told;
        for (;;) {
            if (orc_bc2(meqn, mbc, mx, my, q, mthbc) != 0) { info = -2; goto done; }
            std::memcpy(qwork.data(), q, nq * sizeof(double));
            if (orc_step2(meqn, mwaves, maux, mbc, mx, my, qwork.data(), q, aux, dx, dy, dt,
                          method, mthlim, use_fwaves, &cfl) != 0) {
                info = -1;
                goto done;
            }
            t = told + dt;
            if (cfl <= cflv[0]) {
                cflmax = std::fmax(cfl, cflmax);
                break;
            }
            t = told;
            std::memcpy(q, qwork.data(), nq * sizeof(double));
            if (method[0] == 1) {
                dt = std::fmin(dtv[1], dt * cflv[1] / cfl);
                continue;
            }
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
            const int rc = orc_step1(meqn, mwaves, mbc, maux, mx, q, aux, dx, dt, method, mthlim,
                                     use_fwaves, &cfl);
            if (rc != 0) { info = rc == -3 ? -3 : -1; goto done; }
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
