// Fused 2D dimensionally split step (dimsp2 + step2ds + flux2 without the
// transverse part + bc2 + the CFL reductions + claw2's dt controller) for
// sm_100a.
//
// Reference: src/2d/dimsp2.f:1-99, src/2d/step2ds.f90:1-275,
// src/2d/flux2.f90:5-186, src/2d/inlinelimiter.f90:25-105, src/2d/bc2.f:4-215,
// src/2d/claw2.f:659-680.
//
// The reference sweeps the whole grid three (Strang) or two (Godunov) times,
// each sweep reading and writing every cell.  Here one warp marches up the
// rows of a strip of columns and applies all sweeps to a row as it passes, so
// q is read once from HBM and written once per step:
//   stage A  x-slice of row t (dt, or dt/2 for Strang) -> xA(t), on every row
//            the reference x-sweeps, ghost rows included;
//   stage B  y-interface between xA(t-1) and xA(t); row t-2 gets its y-update
//            (limited waves of the interfaces t-3|t-2 .. t-1|t) -> yB(t-2);
//   stage C  (Strang only) x-slice of yB(t-2) with dt/2 -> the new q.
// Lane l holds column c = b - H + l (b = first output column of the strip):
// stage A is exact on lanes 2..29, so Godunov outputs lanes 2..29 (H = 2,
// 28 columns per strip) and Strang, whose stage C needs stage B on two more
// columns either side, lanes 4..27 (H = 4, 24 columns).
//
// Ghost cells follow step2ds exactly: ghost columns are not x-updated (their
// stage A value is the bc2 value), ghost rows are x-updated, the y-sweep runs
// on ghost columns as well (their Courant numbers count, and Strang's last
// x-sweep reads them), and Strang's last sweep sees the ghost columns of the
// first, as src/2d/dimsp2.f:88-90 notes.  The Courant numbers of the sweeps
// are reduced separately, so the step reports what dimsp2 reports when a
// sweep exceeds cfl_max and the step is abandoned.
//
// Each cell's increments are added in step2ds's order with the same
// operations, so the result is bit-identical to the reference order of
// operations (built with --fmad=false).
#pragma once
#include "step2d.cuh"

namespace clawb200 {

template <class S, bool STRANG>
struct SplitLayout {
    using real = typename S::real;
    static constexpr int H = STRANG ? 4 : 2;        // halo lanes left of the strip
    static constexpr int STRIPW = 32 - 2 * H;        // output columns per warp
    static constexpr int XOFF = STRANG ? 8 : 4;      // ring box starts XOFF columns left of b
    static constexpr int W = STRANG ? 40 : 36;       // ring box width (columns)
    static constexpr int QI = XOFF - H;              // ring index of lane 0's column
    static constexpr int QB = S::meqn * W * (int)sizeof(real);
    static constexpr int QBP = ((QB + 127) / 128) * 128;
    static constexpr int AB = S::maux * W * (int)sizeof(real);
    static constexpr int SLOT = ((QBP + AB + 127) / 128) * 128;
    static constexpr int WARP_BYTES = RING * SLOT;
    static constexpr int SMEM = WARPS2D * WARP_BYTES + WARPS2D * RING * 8 + 64;
    // b is a multiple of STRIPW, so b - XOFF keeps a TMA box start on a
    // 16-byte boundary for 4- and 8-byte elements
    static_assert(STRIPW % 4 == 0 && XOFF % 4 == 0, "box start must stay 16-byte aligned");
};

template <class S>
struct SplitConsts {
    typename S::real dtdx_a, dtdy, dtdx_c;  // stage A (dt or dt/2), stage B (dt), stage C (dt/2)
    double dtdx_a_d, dtdy_d, dtdx_c_d;
    const typename S::real* qold;
    typename S::real* qnew;
    const CUtensorMap* tmq;
    int src;                       // source split of this launch (0 in claw_step)
    double src_pre, src_post;      // source time steps before / after the step
};

// One x-slice step on the row the warp holds (lane l: own column c, values qc
// with the boundary conditions applied; ac its aux).  All 32 lanes call it.
// Returns in xq the updated value where lanes l-2..l+2 hold real data and
// `update` is set, else qc.  The Courant number of interface c-1|c is folded
// into cfl when cfl_ok (src/2d/flux2.f90:97-181 without the transverse part;
// update src/2d/step2ds.f90:201-214).
template <class S, class M>
__device__ __forceinline__ void split_xslice(const Step2Args<S>& A, const typename S::real* qc,
                                             const typename S::real* ac, typename S::real dtdx,
                                             double dtdx_d, bool update, bool cfl_ok,
                                             typename S::real* xq, double& cfl) {
    using real = typename S::real;
    constexpr int ME = S::meqn, MW = S::mwaves, MA = S::maux;
    constexpr int MAX = MA > 0 ? MA : 1;
    constexpr unsigned FULL = 0xffffffffu;
    const int order = M::order >= 0 ? M::order : A.order;
    const bool capa = M::capa >= 0 ? (M::capa != 0) : (A.capa > 0);
    const bool fwave = M::fwave >= 0 ? (M::fwave != 0) : (A.fwave != 0);
    const int ic = capa ? A.capa - 1 : 0;
    bool limit = M::lim > 0;
    if (M::lim < 0)
        limit = (A.mthlim[0] | A.mthlim[1] | A.mthlim[2] | A.mthlim[3] | A.mthlim[4] |
                 A.mthlim[5] | A.mthlim[6] | A.mthlim[7]) != 0;

    real qm[ME], am[MAX];
#pragma unroll
    for (int m = 0; m < ME; ++m) qm[m] = __shfl_up_sync(FULL, qc[m], 1);
#pragma unroll
    for (int k = 0; k < MAX; ++k) am[k] = MA > 0 ? __shfl_up_sync(FULL, ac[k], 1) : real(0);

    real w[MW][ME], s[MW], amdq[ME], apdq[ME];
    {
        const auto cx = iface_ctx(A.solver, 1, qm, qc);
        if constexpr (solver_ctx<S>::value) A.solver.rpn_ctx(1, cx, qm, qc, w, s, amdq, apdq);
        else A.solver.rpn(1, qm, qc, am, ac, w, s, amdq, apdq);
    }
    const real dtm = capa ? dtdx / am[ic] : dtdx;  // dtdx1d(i-1)
    const real dtc = capa ? dtdx / ac[ic] : dtdx;  // dtdx1d(i)
    if (cfl_ok) {
        const double dm = capa ? dtdx_d / (double)am[ic] : dtdx_d;
        const double dc = capa ? dtdx_d / (double)ac[ic] : dtdx_d;
#pragma unroll
        for (int mw = 0; mw < MW; ++mw) cfl = fmax(fmax(cfl, dc * (double)s[mw]), -dm * (double)s[mw]);
    }
    real send1[ME], qadd[ME], F[ME];
#pragma unroll
    for (int m = 0; m < ME; ++m) {
        const bool z = S::wave_zero(1, m);
        send1[m] = z ? real(0) : dtm * amdq[m];
        qadd[m] = z ? real(0) : -(dtc * apdq[m]);
        F[m] = real(0);
    }
    if (order != 1) {
        if (limit) {
            real dotr[MW], wn2[MW];
#pragma unroll
            for (int mw = 0; mw < MW; ++mw) {
                real dr = real(0), nn = real(0);
                bool first = true;
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    if (S::wave_zero(1, m)) continue;
                    const real wr = __shfl_down_sync(FULL, w[mw][m], 1);
                    if (first) {
                        nn = w[mw][m] * w[mw][m];
                        dr = w[mw][m] * wr;
                        first = false;
                    } else {
                        nn = nn + w[mw][m] * w[mw][m];
                        dr = dr + w[mw][m] * wr;
                    }
                }
                dotr[mw] = dr;
                wn2[mw] = nn;
            }
#pragma unroll
            for (int mw = 0; mw < MW; ++mw) {
                const int ml = M::lim >= 0 ? M::lim : A.mthlim[mw];
                const real dl = __shfl_up_sync(FULL, dotr[mw], 1);
                if (ml == 0) continue;
                const real r = (s[mw] > real(0) ? dl : dotr[mw]) / wn2[mw];
                const real ph = wn2[mw] != real(0) ? phi_limiter<real>(ml, r) : real(1);
#pragma unroll
                for (int m = 0; m < ME; ++m)
                    if (!S::wave_zero(1, m)) w[mw][m] = ph * w[mw][m];
            }
        }
        const real ave = real(0.5) * (dtm + dtc);
        real cq[ME];
#pragma unroll
        for (int m = 0; m < ME; ++m) cq[m] = real(0);
#pragma unroll
        for (int mw = 0; mw < MW; ++mw) {
            const real as = fabs(s[mw]);
            const real coef = fwave ? copysign(real(1), s[mw]) * (real(1) - as * ave)
                                    : as * (real(1) - as * ave);
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                if (S::wave_zero(1, m)) continue;
                cq[m] = mw == 0 ? coef * w[mw][m] : cq[m] + coef * w[mw][m];
            }
        }
#pragma unroll
        for (int m = 0; m < ME; ++m) F[m] = real(0.5) * cq[m];
    }
#pragma unroll
    for (int m = 0; m < ME; ++m) {
        const real r1 = __shfl_down_sync(FULL, send1[m], 1);
        const real r2 = __shfl_down_sync(FULL, F[m], 1);
        real v = qc[m];
        if (update && !S::wave_zero(1, m)) {
            const real qa = qadd[m] - r1;
            const real dF = r2 - F[m];
            v = capa ? (v + qa) - dtdx * dF / ac[ic] : (v + qa) - dtdx * dF;
        }
        xq[m] = v;
    }
}

template <class S, class M, bool STRANG, bool SRC>
__device__ __forceinline__ void split2_rows(const Step2Args<S>& A, const SplitConsts<S>& K,
                                            const int strip, const int r0, const int nr,
                                            unsigned char* ring, uint64_t* bars,
                                            uint32_t& seq_base, double* cfl, bool& failed) {
    using real = typename S::real;
    using L = SplitLayout<S, STRANG>;
    constexpr int ME = S::meqn, MW = S::mwaves, MA = S::maux;
    constexpr int MAX = MA > 0 ? MA : 1;
    constexpr int W = L::W;
    constexpr unsigned FULL = 0xffffffffu;
    ClawCtl* ctl = A.ctl;
    const real* __restrict__ qold = K.qold;
    real* __restrict__ qnew = K.qnew;
    const CUtensorMap* tmq = K.tmq;

    const int order = M::order >= 0 ? M::order : A.order;
    const bool capa = M::capa >= 0 ? (M::capa != 0) : (A.capa > 0);
    const bool fwave = M::fwave >= 0 ? (M::fwave != 0) : (A.fwave != 0);
    const int ic = capa ? A.capa - 1 : 0;
    bool limit = M::lim > 0;
    if (M::lim < 0)
        limit = (A.mthlim[0] | A.mthlim[1] | A.mthlim[2] | A.mthlim[3] | A.mthlim[4] |
                 A.mthlim[5] | A.mthlim[6] | A.mthlim[7]) != 0;
    const int lane = threadIdx.x & 31;
    const int mx = A.mx, my = A.my;

    const int b = strip * L::STRIPW;
    const int c = b - L::H + lane;
    const int x0 = b - L::XOFF;
    const int rfirst = r0 - 2, rlast = r0 + nr + 1;
    const int nrows = rlast - rfirst + 1;

    bool negc;
    const int sc = bc_map(c, mx, A.bc[0], A.bc[1], negc);
    const bool gc = (sc - x0) < 0 || (sc - x0) >= W;
    const bool any_global = __any_sync(FULL, gc);
    const int icc = gc ? 0 : sc - x0;
    const bool interior_col = c >= 0 && c < mx;
    const bool ghost_col = (c >= -2 && c < 0) || (c >= mx && c <= mx + 1);
    // stage A is exact on lanes 2..29; ghost columns keep their bc2 values
    const bool a_exact = lane >= 2 && lane <= 29;
    const bool x_upd = interior_col && a_exact;
    // x-interface c-1|c counts for c = 0..mx (src/2d/flux2.f90:124-132)
    const bool cx_ok = c >= 0 && c <= mx && lane >= 1;
    // stage B input is right on ghost columns and on lanes 2..29
    const bool cy_ok = (ghost_col || (interior_col && a_exact));
    // stage C: exact on lanes 4..27; interface c-1|c needs stage B on c-1, c
    const bool cc_ok = c >= 0 && c <= mx && lane >= 3 && lane <= 29;
    const bool out_lane = lane >= L::H && lane < L::H + L::STRIPW && c < mx;

    auto seq_of = [&](int r) -> uint32_t { return seq_base + (uint32_t)(r - rfirst); };
    auto issue = [&](int r) {
        const uint32_t sq = seq_of(r);
        const int sl = (int)(sq & (RING - 1));
        unsigned char* dst = ring + sl * L::SLOT;
        bool nyneg;
        const int sr = bc_map(r, my, A.bc[2], A.bc[3], nyneg);
        mbar_arrive_expect_tx(&bars[sl], (uint32_t)(L::QB + L::AB));
        tma_load_3d(dst, tmq, x0, sr, 0, &bars[sl]);
        if constexpr (MA > 0) tma_load_3d(dst + L::QBP, &A.tmaux, x0, r + 2, 0, &bars[sl]);
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
    auto slot_ptr = [&](int r) -> const unsigned char* {
        return ring + (int)(seq_of(r) & (RING - 1)) * L::SLOT;
    };
    // q(c, r) with the x and y boundary conditions applied, and aux(c, r)
    auto load_row = [&](int r, real* qv, real* av) {
        const real* sq = reinterpret_cast<const real*>(slot_ptr(r));
        bool nyneg;
        const int sr = bc_map(r, my, A.bc[2], A.bc[3], nyneg);
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            real v = sq[m * W + icc];
            if (any_global && gc) v = qold[m * A.fstride + (long long)sr * A.ld + sc];
            if (m == 1 && negc) v = -v;
            if (m == 2 && nyneg) v = -v;
            qv[m] = v;
        }
        if constexpr (SRC) {
            if (K.src == 2) src_radial_cell(A, qv, c, K.src_pre);  // Strang: before the step
        }
        if constexpr (MA > 0) {
            const real* sa = reinterpret_cast<const real*>(slot_ptr(r) + L::QBP);
#pragma unroll
            for (int k = 0; k < MA; ++k) av[k] = sa[k * W + L::QI + 2 + lane];
        } else {
            av[0] = real(0);
        }
    };
    // stage A on row r: x-update on ghost rows too (step2ds sweeps every row)
    auto stage_a = [&](int r, real* xa, real* av) {
        real qv[ME];
        load_row(r, qv, av);
        split_xslice<S, M>(A, qv, av, K.dtdx_a, K.dtdx_a_d, x_upd, cx_ok, xa, cfl[0]);
    };

    // ---- march state ----
    real xa_p[ME], xa_t[ME];            // xA(t-2), xA(t-1)
    real aux_p[MAX], aux_t[MAX];        // aux of those rows
    real wy[MW][ME], sy[MW], amy[ME], apy[ME], dotl_y[MW];  // y-interface t-2|t-1
    real P1[ME], Fy_prev[ME];           // from interface t-3|t-2
#pragma unroll
    for (int m = 0; m < ME; ++m) P1[m] = Fy_prev[m] = real(0);
#pragma unroll
    for (int mw = 0; mw < MW; ++mw) dotl_y[mw] = real(0);

    int last_issued = rfirst + (nrows < RING ? nrows : RING) - 1;
    int fail_row = rlast + 1;

    auto yrpn = [&](const real* lo, const real* hi, const real* alo, const real* ahi,
                    real (*wv)[ME], real* sv, real* am, real* ap) {
        const auto cy = iface_ctx(A.solver, 2, lo, hi);
        if constexpr (solver_ctx<S>::value) A.solver.rpn_ctx(2, cy, lo, hi, wv, sv, am, ap);
        else A.solver.rpn(2, lo, hi, alo, ahi, wv, sv, am, ap);
    };
    auto ycfl = [&](int t, const real* sv, const real* alo, const real* ahi) {
        // y-interface t-1|t counts for t = 0..my
        if (cy_ok && t >= 0 && t <= my) {
            const double d0 = capa ? K.dtdy_d / (double)alo[ic] : K.dtdy_d;
            const double d1 = capa ? K.dtdy_d / (double)ahi[ic] : K.dtdy_d;
#pragma unroll
            for (int mw = 0; mw < MW; ++mw)
                cfl[1] = fmax(fmax(cfl[1], d1 * (double)sv[mw]), -d0 * (double)sv[mw]);
        }
    };
    // Strang stage C on a row whose y-sweep is done (all lanes call)
    auto stage_c = [&](int r, const real* yb, const real* av, bool write) {
        real out[ME];
        split_xslice<S, M>(A, yb, av, K.dtdx_c, K.dtdx_c_d, interior_col && lane >= 4 && lane <= 27,
                           cc_ok, out, cfl[2]);
        if constexpr (SRC) {
            if (write && K.src != 0) src_radial_cell(A, out, c, K.src == 2 ? K.src_pre : K.src_post);
        }
        if (write && out_lane) {
            real* __restrict__ dst = qnew + (long long)r * A.ld + c;
#pragma unroll
            for (int m = 0; m < ME; ++m) dst[m * A.fstride] = out[m];
        }
    };

    // ---- prologue: rows r0-2, r0-1 and the y-interface between them ----
    if (!wait_row(rfirst)) { failed = true; fail_row = rfirst; }
    if (!failed && !wait_row(rfirst + 1)) { failed = true; fail_row = rfirst + 1; }
    if (__any_sync(FULL, failed)) failed = true;
    if (!failed) {
        stage_a(rfirst, xa_p, aux_p);
        stage_a(rfirst + 1, xa_t, aux_t);
        yrpn(xa_p, xa_t, aux_p, aux_t, wy, sy, amy, apy);
        ycfl(rfirst + 1, sy, aux_p, aux_t);
    }

    for (int t = rfirst + 2; t <= rlast && !failed; ++t) {
        if (!wait_row(t)) { failed = true; fail_row = t; }
        if (__any_sync(FULL, failed)) { failed = true; break; }
        real xa_n[ME], aux_n[MAX];
        stage_a(t, xa_n, aux_n);

        // y-interface t-1|t raw
        real wn[MW][ME], sn[MW], amn[ME], apn[ME];
        yrpn(xa_t, xa_n, aux_t, aux_n, wn, sn, amn, apn);
        ycfl(t, sn, aux_t, aux_n);

        // limit y-interface t-2|t-1
        const real dty_p = capa ? K.dtdy / aux_p[ic] : K.dtdy;  // dtdy1d(t-2)
        const real dty_t = capa ? K.dtdy / aux_t[ic] : K.dtdy;  // dtdy1d(t-1)
        real Fy[ME], dotr_y[MW];
#pragma unroll
        for (int m = 0; m < ME; ++m) Fy[m] = real(0);
#pragma unroll
        for (int mw = 0; mw < MW; ++mw) {
            real dr = real(0);
            bool first = true;
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                if (S::wave_zero(2, m)) continue;
                dr = first ? wy[mw][m] * wn[mw][m] : dr + wy[mw][m] * wn[mw][m];
                first = false;
            }
            dotr_y[mw] = dr;
        }
        if (order != 1) {
            if (limit) {
#pragma unroll
                for (int mw = 0; mw < MW; ++mw) {
                    const int ml = M::lim >= 0 ? M::lim : A.mthlim[mw];
                    if (ml == 0) continue;
                    real nn = real(0);
                    bool first = true;
#pragma unroll
                    for (int m = 0; m < ME; ++m) {
                        if (S::wave_zero(2, m)) continue;
                        nn = first ? wy[mw][m] * wy[mw][m] : nn + wy[mw][m] * wy[mw][m];
                        first = false;
                    }
                    const real r = (sy[mw] > real(0) ? dotl_y[mw] : dotr_y[mw]) / nn;
                    const real ph = nn != real(0) ? phi_limiter<real>(ml, r) : real(1);
#pragma unroll
                    for (int m = 0; m < ME; ++m)
                        if (!S::wave_zero(2, m)) wy[mw][m] = ph * wy[mw][m];
                }
            }
            const real ave = real(0.5) * (dty_p + dty_t);
            real cqy[ME];
#pragma unroll
            for (int m = 0; m < ME; ++m) cqy[m] = real(0);
#pragma unroll
            for (int mw = 0; mw < MW; ++mw) {
                const real as = fabs(sy[mw]);
                const real coef = fwave ? copysign(real(1), sy[mw]) * (real(1) - as * ave)
                                        : as * (real(1) - as * ave);
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    if (S::wave_zero(2, m)) continue;
                    cqy[m] = mw == 0 ? coef * wy[mw][m] : cqy[m] + coef * wy[mw][m];
                }
            }
#pragma unroll
            for (int m = 0; m < ME; ++m) Fy[m] = real(0.5) * cqy[m];
        }

        // y-update of row t-2 (src/2d/step2ds.f90:250-266)
        const int ro = t - 2;
        real yb[ME];
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            real v = xa_p[m];
            if (ro >= 0 && ro < my && !S::wave_zero(2, m)) {
                const real qa = P1[m] - dty_p * amy[m];
                const real dF = Fy[m] - Fy_prev[m];
                v = capa ? (v + qa) - K.dtdy * dF / aux_p[ic] : (v + qa) - K.dtdy * dF;
            }
            yb[m] = v;
        }
        if constexpr (STRANG) {
            // rows r0-2, r0-1 of an interior chunk lack their lower limiter
            // neighbours; ghost rows (not y-updated) are exact
            if (ro >= r0 || ro < 0) stage_c(ro, yb, aux_p, ro >= r0);
        } else {
            if constexpr (SRC) {
                if (K.src != 0) src_radial_cell(A, yb, c, K.src == 2 ? K.src_pre : K.src_post);
            }
            if (ro >= r0 && out_lane) {
                real* __restrict__ dst = qnew + (long long)ro * A.ld + c;
#pragma unroll
                for (int m = 0; m < ME; ++m) dst[m * A.fstride] = yb[m];
            }
        }

        // roll the window
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            P1[m] = S::wave_zero(2, m) ? real(0) : -(dty_t * apy[m]);
            Fy_prev[m] = Fy[m];
            amy[m] = amn[m];
            apy[m] = apn[m];
            xa_p[m] = xa_t[m];
            xa_t[m] = xa_n[m];
        }
#pragma unroll
        for (int k = 0; k < MAX; ++k) { aux_p[k] = aux_t[k]; aux_t[k] = aux_n[k]; }
#pragma unroll
        for (int mw = 0; mw < MW; ++mw) {
            dotl_y[mw] = dotr_y[mw];
            sy[mw] = sn[mw];
#pragma unroll
            for (int m = 0; m < ME; ++m) wy[mw][m] = wn[mw][m];
        }
        // release row t-2 and prefetch row t-2+RING into its slot
        __syncwarp();
        if (t - 2 + RING <= rlast) {
            if (lane == 0) issue(t - 2 + RING);
            last_issued = t - 2 + RING;
        }
        __syncwarp();
    }
    if constexpr (STRANG) {
        // ghost rows my, my+1: stage C on xA (Courant number only)
        if (!failed && rlast == my + 1) {
            stage_c(my, xa_p, aux_p, false);
            stage_c(my + 1, xa_t, aux_t, false);
        }
    }
    if (failed) {
        for (int r = fail_row + 1; r <= last_issued; ++r) (void)wait_row(r);
        if (lane == 0) atomicOr(&ctl->err, CTL_ERR_TMA_TIMEOUT);
    }
    seq_base += (uint32_t)nrows;
}

// Fold the per-sweep Courant maxima of every CTA; the last CTA combines them
// as dimsp2 does and runs the controller.
__device__ __forceinline__ void cta_split_cfl_and_control(ClawCtl* ctl, const double* c3, int nsw,
                                                          double* red) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = (int)(blockDim.x >> 5);
    for (int k = 0; k < nsw; ++k) {
        double v = c3[k];
        for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
        if (lane == 0) red[k * nw + warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < nsw; ++k) {
            double m = 0.0;
            for (int w = 0; w < nw; ++w) m = fmax(m, red[k * nw + w]);
            if (!(m > 0.0)) m = (m != m) ? m : 0.0;
            unsigned long long* slot = k == 0 ? &ctl->cfl_bits : &ctl->cfl_sweep[k - 1];
            atomicMax(slot, (unsigned long long)__double_as_longlong(m));
        }
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->ctas_done, 1u);
        if (prev == gridDim.x - 1) {
            __threadfence();
            const double ca = __longlong_as_double((long long)atomicAdd(&ctl->cfl_bits, 0ull));
            const double cb = __longlong_as_double((long long)atomicAdd(&ctl->cfl_sweep[0], 0ull));
            const double cc = nsw > 2
                                  ? __longlong_as_double((long long)atomicAdd(&ctl->cfl_sweep[1], 0ull))
                                  : 0.0;
            ctl->cfl_sweep[0] = 0ull;
            ctl->cfl_sweep[1] = 0ull;
            // src/2d/dimsp2.f:65-96
            // a NaN in any sweep stays NaN (the controller stops on it)
            auto nmax = [](double a, double b2) { return a != a ? a : (b2 != b2 ? b2 : fmax(a, b2)); };
            double cfl;
            if (ca > ctl->cfl_max) cfl = ca;
            else if (nsw > 2 && cb > ctl->cfl_max) cfl = cb;
            else {
                cfl = nmax(ca, cb);
                if (nsw > 2) cfl = nmax(cfl, cc);
            }
            ctl->cfl_bits = (unsigned long long)__double_as_longlong(cfl);
            ctl_finish_step(ctl);
            __threadfence();
        }
    }
}

// BUILD tells apart the instantiations of the reference-order unit (0) and the
// contracted unit (1), which must not share a symbol.
template <class S, class M, bool STRANG, bool SRC, int BUILD>
__global__ void __launch_bounds__(32 * WARPS2D, step2_minb<S>::value)
split2_kernel(const __grid_constant__ Step2Args<S> A) {
    using L = SplitLayout<S, STRANG>;
    using real = typename S::real;
    ClawCtl* ctl = A.ctl;
    __shared__ double red[3 * WARPS2D];
    grid_dependency_sync();
    if (*(volatile int*)&ctl->done) return;
    const int cur = *(volatile int*)&ctl->cur;
    const double dtd = *(volatile double*)&ctl->dt;

    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* ring = smem + warp * L::WARP_BYTES;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + WARPS2D * L::WARP_BYTES) + warp * RING;
    if (lane == 0) {
        for (int sl = 0; sl < RING; ++sl) mbar_init(&bars[sl], 1);
        fence_barrier_init();
    }
    __syncwarp();

    SplitConsts<S> K;
    const double dta = STRANG ? dtd / 2.0 : dtd;  // src/2d/dimsp2.f:52-62
    K.dtdx_a_d = dta / A.dx;
    K.dtdy_d = dtd / A.dy;
    K.dtdx_c_d = (dtd / 2.0) / A.dx;
    K.dtdx_a = (real)K.dtdx_a_d;
    K.dtdy = (real)K.dtdy_d;
    K.dtdx_c = (real)K.dtdx_c_d;
    K.qold = A.q[cur];
    K.qnew = A.q[cur ^ 1];
    K.tmq = &A.tmq[cur];
    // claw2 wraps the source steps around the split step; claw_step runs it alone
    K.src = (SRC && ctl->mode == CTL_ADVANCE) ? A.src_split : 0;
    K.src_pre = dtd / 2.0;
    K.src_post = dtd;

    const int my = A.my;
    double cfl[3] = {0.0, 0.0, 0.0};
    bool failed = false;
    uint32_t seq_base = 0;
    const long long gw = (long long)blockIdx.x * WARPS2D + warp;
    long long u0 = (gw < A.nwarps) ? gw * A.units / A.nwarps : 0;
    const long long u1 = (gw < A.nwarps) ? (gw + 1) * A.units / A.nwarps : 0;
    if (A.brows > 0) {  // row-block-major work items (Step2Args)
        const int items = A.nstrips * A.nblocks;
        for (int item = (int)gw; gw < A.nwarps && item < items && !failed; item += A.nwarps) {
            const int strip = item % A.nstrips, r0 = (item / A.nstrips) * A.brows;
            split2_rows<S, M, STRANG, SRC>(A, K, strip, r0, min(A.brows, my - r0), ring, bars,
                                           seq_base, cfl, failed);
        }
    }
    while (A.brows == 0 && u0 < u1 && !failed) {
        const int strip = (int)(u0 / my);
        const int r0 = (int)(u0 % my);
        const int nr = (int)min((long long)(my - r0), u1 - u0);
        u0 += nr;
        split2_rows<S, M, STRANG, SRC>(A, K, strip, r0, nr, ring, bars, seq_base, cfl, failed);
    }
    cta_split_cfl_and_control(ctl, cfl, STRANG ? 3 : 2, red);
}

}  // namespace clawb200
