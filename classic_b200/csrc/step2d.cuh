// Fused 2D unsplit wave-propagation step (step2 + flux2 + limiter + bc2 +
// CFL reduction + claw2 dt controller) for sm_100a.
//
// Reference: src/2d/step2.f90:2-251, src/2d/flux2.f90:5-235,
// src/2d/inlinelimiter.f90:25-105, src/2d/bc2.f:4-215, src/2d/claw2.f:596-760.
//
// Design ("column march").  Each warp owns a strip of STRIP = 28 output
// columns and marches up a range of rows.  Lane l holds column
// c = b - 1 + l (b = first output column), so lanes 1..28 produce output and
// lanes 0, 29..31 supply the halo.  Per row t the warp
//   * solves the x-interfaces of row t (one per lane; the limiter's neighbour
//     waves and the flux corrections of the right interface arrive by warp
//     shuffle), and
//   * solves the y-interface between rows t and t+1 of its own column, keeping
//     the last y-interface in registers so the y-limiter needs no exchange.
// Each cell's increments are applied in exactly the order step2 applies them:
// x-slice j-1, x-slice j, x-slice j+1, then y-slice i-1, i, i+1, so the
// result is bit-identical to the reference order of operations.
//
// Memory: q is SoA, interior cells only (ghost cells are synthesised from the
// boundary conditions, bc2's corner rule included); aux is SoA with two ghost
// layers.  Rows stream into a per-warp shared-memory ring by TMA
// (cp.async.bulk.tensor, one box of 34(36) x 1 x meqn per row, ghost rows
// loaded from their mapped source row), completion on an mbarrier per slot,
// prefetching RING-3 rows ahead.  q is read once from HBM and written once.
//
// Specialisation: the method (order, transverse_waves, limiter, capacity,
// f-waves) is a compile-time policy for the configurations that matter, so
// a row of the march is straight-line code; Method2D<-1,...> reads every
// choice at run time and covers all other configurations.  Solver traits
// (wave_zero / trans_zero) remove arithmetic on structurally zero
// components; the skipped terms are exact zeros, so results are unchanged.
#pragma once
#include <type_traits>

#include "common.cuh"

namespace clawb200 {

constexpr int STRIP = 28;      // output columns per warp
constexpr int RING = 8;        // rows in flight per warp (power of two)
constexpr int RING_LOG = 3;
constexpr int WARPS2D = 4;     // warps per CTA
static_assert((1 << RING_LOG) == RING, "RING must be 2^RING_LOG");

// A TMA box must start at an x coordinate whose byte offset is a multiple of
// 16: q boxes start XQ columns left of the strip (b is a multiple of 28, so
// b - 2 is even and b - 4 a multiple of 4), aux boxes at padded column b.
template <typename real>
struct BoxW { static constexpr int value = 34; static constexpr int XQ = 2; };
template <>
struct BoxW<float> { static constexpr int value = 36; static constexpr int XQ = 4; };
static_assert(STRIP % 4 == 0, "strip width must keep b a multiple of 4");

// Method policy: -1 = read from the kernel arguments at run time.  FAST = 1
// is the contracted build (CLAW_FP64_FMA): Newton reciprocals instead of IEEE
// divisions in the limiter ratio and the capacity scalings, compare-and-select
// instead of fmin/fmax; the Courant number is formed as in the reference-order
// build, so the dt sequence is the same.
template <int ORDER, int TRANS, int LIM, int CAPA, int FWAVE, int FAST = 0>
struct Method2D {
    static constexpr int order = ORDER, trans = TRANS, lim = LIM, capa = CAPA, fwave = FWAVE;
    static constexpr bool fast = FAST != 0;
};
using MethodGeneric2D = Method2D<-1, -1, -1, -1, -1>;
using MethodMC2D = Method2D<2, 2, 4, 0, 0>;  // order 2, transverse 2, MC, no capa
using MethodGeneric2DFast = Method2D<-1, -1, -1, -1, -1, 1>;
using MethodMC2DFast = Method2D<2, 2, 4, 0, 0, 1>;

template <class S>
struct Step2Args {
    CUtensorMap tmq[2];  // q buffers: dims (mx, my, meqn)
    CUtensorMap tmaux;   // aux: dims (mx+4, my+4, maux)
    typename S::real* q[2];
    const typename S::real* aux;
    long long ld, fstride;    // q row pitch / field pitch (elements)
    long long ald, afstride;  // aux row pitch / field pitch (elements)
    int mx, my, nstrips;
    int bc[4];                // x-lower, x-upper, y-lower, y-upper
    int mthlim[8];
    int order, trans, fwave, capa;  // method(2), method(3), use_fwaves, capa index (1-based, 0 none)
    double dx, dy;
    long long units;          // nstrips * my
    int nwarps;               // warps sharing the units
    // Row-block-major work items (brows > 0): item = block * nstrips + strip,
    // block b covering rows [b brows, (b+1) brows); warp w takes items w,
    // w + nwarps, ...  The warps at work on one row block hold adjacent
    // strips, so they stream neighbouring DRAM pages.  brows = 0: warp w
    // takes units [w units / nwarps, (w+1) units / nwarps) in strip-major
    // order.
    int brows, nblocks;
    // source term (src/2d/claw2.f:635-738): 0 none, 1 Godunov, 2 Strang; the
    // radial term of examples/acoustics_2d_radial/1drad/src1.f on every row
    int src_split;
    double src_nd1, src_bulk, xlower;  // ndim - 1, bulk, xlower
    ClawCtl* ctl;
    S solver;
};

// The radial source at 0-based column c (src1.f:18-23 covers the cells
// i = c+1 >= 1 of a row, right ghosts included): p -= dts (ndim-1) bulk / x u.
// q[0] is the pressure and q[1] the radial velocity.
template <class S>
__device__ __forceinline__ void src_radial_cell(const Step2Args<S>& A, typename S::real* q, int c,
                                                double dts) {
    if (c < 0) return;
    const double xcell = A.xlower + ((double)(c + 1) - 0.5) * A.dx;
    const double coef = dts * A.src_nd1 * A.src_bulk / xcell;
    q[0] = q[0] - (typename S::real)(coef * (double)q[1]);
}

// Map a (possibly ghost) index to its source interior index under the BC of
// that side.  Returns the source index; sets neg when a wall reflects it.
__device__ __forceinline__ int bc_map(int x, int n, int blo, int bhi, bool& neg) {
    neg = false;
    if (x < 0) {
        if (x < -2) x = -2;  // beyond the two ghost layers: only halo lanes past the edge
        if (blo == BC_PERIODIC) return x + n;
        if (blo == BC_WALL) { neg = true; return -1 - x; }
        return 0;
    }
    if (x >= n) {
        if (x > n + 1) x = n + 1;
        if (bhi == BC_PERIODIC) return x - n;
        if (bhi == BC_WALL) { neg = true; return 2 * n - 1 - x; }
        return n - 1;
    }
    return x;
}

template <class S>
struct Ring2D {
    using real = typename S::real;
    static constexpr int W = BoxW<real>::value;
    static constexpr int QB = S::meqn * W * (int)sizeof(real);
    static constexpr int QBP = ((QB + 127) / 128) * 128;  // aux box starts 128-byte aligned
    static constexpr int AB = S::maux * W * (int)sizeof(real);
    static constexpr int SLOT = ((QBP + AB + 127) / 128) * 128;
    static constexpr int WARP_BYTES = RING * SLOT;
    static constexpr int SMEM = WARPS2D * WARP_BYTES + WARPS2D * RING * 8 + 64;
};

#ifndef CLAW_STEP2_MINB
#define CLAW_STEP2_MINB 4  // 128 registers: 16 warps per SM hide the FP64 latency
#endif

// One chunk of the march: output rows [r0, r0+nr) of strip `strip`, step dt
// from buffer `cur`.  Per warp; ring/bars/seq_base are the warp's TMA ring.
// Folds the chunk's Courant numbers into cfl; on a device-wait time-out sets
// `failed` and the grid's error flag after draining its copies.
// Optional solver hook: an interface context (S::Ctx, S::context) shared by
// the normal solve and both transverse splits of one interface.  Solvers
// without it are called through the plain rpn / rpt contract.
template <class S, class = void>
struct solver_ctx {
    struct type {};
    static constexpr bool value = false;
};
template <class S>
struct solver_ctx<S, std::void_t<typename S::Ctx>> {
    using type = typename S::Ctx;
    static constexpr bool value = true;
};

template <class S>
__device__ __forceinline__ typename solver_ctx<S>::type iface_ctx(const S& s, int ixy,
                                                                  const typename S::real* qL,
                                                                  const typename S::real* qR) {
    if constexpr (solver_ctx<S>::value) return s.context(ixy, qL, qR);
    else return typename solver_ctx<S>::type{};
}

template <class S>
struct StepConsts {
    typename S::real dtdx, dtdy;   // dt/dx, dt/dy in the update's precision
    double dtdx_d, dtdy_d;         // the same in FP64 for the Courant number
    const typename S::real* qold;
    typename S::real* qnew;
    const CUtensorMap* tmq;        // TMA map of qold
    int src;                       // source split of this launch (0 in claw_step / batches)
    double src_pre, src_post;      // source time steps before / after the step
};

template <class S>
__device__ __forceinline__ StepConsts<S> step_consts(const Step2Args<S>& A, int cur, double dtd) {
    using real = typename S::real;
    StepConsts<S> k;
    k.dtdx = (real)(dtd / A.dx);
    k.dtdy = (real)(dtd / A.dy);
    k.dtdx_d = dtd / A.dx;
    k.dtdy_d = dtd / A.dy;
    k.qold = A.q[cur];
    k.qnew = A.q[cur ^ 1];
    k.tmq = &A.tmq[cur];
    k.src = 0;
    k.src_pre = dtd / 2.0;
    k.src_post = dtd;
    return k;
}

template <class S, class M, bool SRC = false>
__device__ __forceinline__ void step2_rows(const Step2Args<S>& A, const StepConsts<S>& K,
                                           const int strip, const int r0, const int nr,
                                           unsigned char* ring, uint64_t* bars,
                                           uint32_t& seq_base, double& cfl, bool& failed) {
    using real = typename S::real;
    constexpr int ME = S::meqn, MW = S::mwaves, MA = S::maux;
    constexpr int MAX = MA > 0 ? MA : 1;
    using R = Ring2D<S>;
    constexpr int W = R::W;
    constexpr unsigned FULL = 0xffffffffu;
    ClawCtl* ctl = A.ctl;
    const real dtdx = K.dtdx, dtdy = K.dtdy;
    const double dtdx_d = K.dtdx_d, dtdy_d = K.dtdy_d;
    const real* __restrict__ qold = K.qold;
    real* __restrict__ qnew = K.qnew;
    const CUtensorMap* tmq = K.tmq;

    // method: compile-time where the policy fixes it
    const int order = M::order >= 0 ? M::order : A.order;
    const int trans = M::trans >= 0 ? M::trans : A.trans;
    const bool capa = M::capa >= 0 ? (M::capa != 0) : (A.capa > 0);
    const bool fwave = M::fwave >= 0 ? (M::fwave != 0) : (A.fwave != 0);
    const int ic = capa ? A.capa - 1 : 0;
    bool limit = M::lim > 0;
    if (M::lim < 0)
        limit = (A.mthlim[0] | A.mthlim[1] | A.mthlim[2] | A.mthlim[3] | A.mthlim[4] |
                 A.mthlim[5] | A.mthlim[6] | A.mthlim[7]) != 0;
    auto lim_of = [&](int mw) -> int { return M::lim >= 0 ? M::lim : A.mthlim[mw]; };
    using AR = Arith<M::fast>;
    // max of two Courant numbers (the same value as fmax for non-NaN operands)
    auto dmax = [](double a, double b) -> double {
        if constexpr (M::fast) return b > a ? b : a;
        else return fmax(a, b);
    };
    auto phi = [](int ml, real r) -> real {
        if constexpr (M::fast) return phi_limiter_fast<real>(ml, r);
        else return phi_limiter<real>(ml, r);
    };
    const int lane = threadIdx.x & 31;
    const int mx = A.mx, my = A.my;

    const int b = strip * STRIP;
    const int c = b - 1 + lane;
    const int x0 = b - BoxW<real>::XQ;  // first q column held in the ring
    const int rfirst = r0 - 2, rlast = r0 + nr + 1;  // rows streamed
    const int nrows = rlast - rfirst + 1;

    // Column sources of q(c-1) and q(c) under the x boundary conditions.
    bool negm, negc;
    const int sm = bc_map(c - 1, mx, A.bc[0], A.bc[1], negm);
    const int sc = bc_map(c, mx, A.bc[0], A.bc[1], negc);
    const bool gm = (sm - x0) < 0 || (sm - x0) >= W;
    const bool gc = (sc - x0) < 0 || (sc - x0) >= W;
    const bool any_global = __any_sync(FULL, gm || gc);
    const int im = gm ? 0 : sm - x0, icc = gc ? 0 : sc - x0;
    // x-interface c counts toward the CFL for columns 0..mx, y-interface
    // of column c for columns -1..mx (src/2d/flux2.f90:124-132 over the
    // slices of src/2d/step2.f90:92,173)
    const bool cx_ok = c >= 0 && c <= mx;
    const bool cy_ok = c >= -1 && c <= mx;

    // wait limit; test hook: strip 0 skips the copy of one row (its wait then
    // runs out, nothing faults)
    const unsigned long long wait_ns = ctl_wait_ns(ctl);
    const int skip1 = strip == 0 ? *(volatile const int*)&ctl->skip_row : 0;
    auto seq_of = [&](int r) -> uint32_t { return seq_base + (uint32_t)(r - rfirst); };
    auto issue = [&](int r) {
        if (skip1 != 0 && r == skip1 - 1) return;
        const uint32_t sq = seq_of(r);
        const int sl = (int)(sq & (RING - 1));
        unsigned char* dst = ring + sl * R::SLOT;
        bool nyneg;
        const int sr = bc_map(r, my, A.bc[2], A.bc[3], nyneg);
        mbar_arrive_expect_tx(&bars[sl], (uint32_t)(R::QB + R::AB));
        tma_load_3d(dst, tmq, x0, sr, 0, &bars[sl]);
        if constexpr (MA > 0) tma_load_3d(dst + R::QBP, &A.tmaux, b, r + 2, 0, &bars[sl]);
    };
    if (lane == 0) {
        const int npre = nrows < RING ? nrows : RING;
        for (int k = 0; k < npre; ++k) issue(rfirst + k);
    }
    __syncwarp();

    auto wait_row = [&](int r) -> bool {
        const uint32_t sq = seq_of(r);
        return mbar_wait_bounded(&bars[sq & (RING - 1)], (sq >> RING_LOG) & 1u, wait_ns);
    };
    auto slot_ptr = [&](int r) -> const unsigned char* {
        return ring + (int)(seq_of(r) & (RING - 1)) * R::SLOT;
    };
    // q(c-1, r), q(c, r) with the x and y boundary conditions applied.
    auto load_q = [&](int r, real* qm, real* qc) {
        const real* sq = reinterpret_cast<const real*>(slot_ptr(r));
        bool nyneg;
        const int sr = bc_map(r, my, A.bc[2], A.bc[3], nyneg);
#pragma unroll
        for (int m = 0; m < ME; ++m) {
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
        if constexpr (SRC) {
            if (K.src == 2) {  // Strang: dt/2 of source on the data the step reads
                src_radial_cell(A, qm, c - 1, K.src_pre);
                src_radial_cell(A, qc, c, K.src_pre);
            }
        }
    };
    // aux of column (c + dc) at row r (ring already resident).
    auto aux_at = [&](int r, int dc, real* a) {
        if constexpr (MA > 0) {
            const real* sa = reinterpret_cast<const real*>(slot_ptr(r) + R::QBP);
#pragma unroll
            for (int k = 0; k < MA; ++k) a[k] = sa[k * W + lane + 1 + dc];
        }
    };

    // ---- march state ----
    real qm_t[ME], qc_t[ME];        // row t
    real qm_n[ME], qc_n[ME];        // row t+1
    real qc_p[ME];                  // q(c, t-1)
    real Ax_prev[ME], q2_prev[ME];  // x-slice increments carried to row t
    // y-interface t (between rows t-1 and t): raw waves and fluctuations
    real wy[MW][ME], sy[MW], amy[ME], apy[ME], dotl_y[MW];
    // contributions of y-interface t-1 to cell (c, t-1)
    real P1[ME], P3[ME], P4[ME], Fy_prev[ME];
    typename solver_ctx<S>::type cy{};  // context of y-interface t
#pragma unroll
    for (int m = 0; m < ME; ++m) {
        Ax_prev[m] = q2_prev[m] = real(0);
        P1[m] = P3[m] = P4[m] = Fy_prev[m] = real(0);
    }
#pragma unroll
    for (int mw = 0; mw < MW; ++mw) dotl_y[mw] = real(0);

    int last_issued = rfirst + (nrows < RING ? nrows : RING) - 1;
    int fail_row = rlast + 1;

    // ---- prologue: rows r0-2, r0-1 and the y-interface between them ----
    if (!wait_row(rfirst)) { failed = true; fail_row = rfirst; }
    if (!failed && !wait_row(rfirst + 1)) { failed = true; fail_row = rfirst + 1; }
    if (!failed) {
        load_q(rfirst, qm_t, qc_t);
        load_q(rfirst + 1, qm_n, qc_n);
        real a_c[MAX], a_cn[MAX];
        aux_at(rfirst, 0, a_c);
        aux_at(rfirst + 1, 0, a_cn);
        cy = iface_ctx(A.solver, 2, qc_t, qc_n);
        if constexpr (solver_ctx<S>::value) A.solver.rpn_ctx(2, cy, qc_t, qc_n, wy, sy, amy, apy);
        else A.solver.rpn(2, qc_t, qc_n, a_c, a_cn, wy, sy, amy, apy);
        if (cy_ok && rfirst + 1 >= 0) {
            const double dt0 = capa ? dtdy_d / (double)a_c[ic] : dtdy_d;
            const double dt1 = capa ? dtdy_d / (double)a_cn[ic] : dtdy_d;
            double em = 0.0;
#pragma unroll
            for (int mw = 0; mw < MW; ++mw)
                em = dmax(em, dmax(dt1 * (double)sy[mw], -dt0 * (double)sy[mw]));
            cfl = dmax(cfl, em);
        }
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            qc_p[m] = qc_t[m];
            qm_t[m] = qm_n[m];
            qc_t[m] = qc_n[m];
        }
    }

    for (int t = r0 - 1; t <= r0 + nr && !failed; ++t) {
        // ---------------- read row t+1 ----------------
        if (!wait_row(t + 1)) { failed = true; fail_row = t + 1; break; }
        load_q(t + 1, qm_n, qc_n);
        real a_m[MAX], a_c[MAX], a_cn[MAX], a_p[MAX], a_cp[MAX], a_mp[MAX], a_pp[MAX], a_mn[MAX];
        aux_at(t, -1, a_m);       // (c-1, t)
        aux_at(t, 0, a_c);        // (c,   t)
        aux_at(t, 1, a_p);        // (c+1, t)
        aux_at(t + 1, 0, a_cn);   // (c,   t+1)
        aux_at(t + 1, -1, a_mn);  // (c-1, t+1)
        aux_at(t - 1, 0, a_cp);   // (c,   t-1)
        aux_at(t - 1, -1, a_mp);  // (c-1, t-1)
        aux_at(t - 1, 1, a_pp);   // (c+1, t-1)

        // ======== x-slice t: interface c (between columns c-1, c) ========
        real q3[ME];
        {
            real w[MW][ME], s[MW], amdq[ME], apdq[ME];
            const auto cx = iface_ctx(A.solver, 1, qm_t, qc_t);
            if constexpr (solver_ctx<S>::value) A.solver.rpn_ctx(1, cx, qm_t, qc_t, w, s, amdq, apdq);
            else A.solver.rpn(1, qm_t, qc_t, a_m, a_c, w, s, amdq, apdq);
            const real dtm = capa ? AR::div(dtdx, a_m[ic]) : dtdx;  // dtdx1d(i-1)
            const real dtc = capa ? AR::div(dtdx, a_c[ic]) : dtdx;  // dtdx1d(i)
            {
                const double dm = capa ? dtdx_d / (double)a_m[ic] : dtdx_d;
                const double dc = capa ? dtdx_d / (double)a_c[ic] : dtdx_d;
                double em = 0.0;
#pragma unroll
                for (int mw = 0; mw < MW; ++mw)
                    em = dmax(em, dmax(dc * (double)s[mw], -dm * (double)s[mw]));
                cfl = (cx_ok && t >= -1 && t <= my) ? dmax(cfl, em) : cfl;
            }
            real send1[ME], qadd[ME], F[ME], cq[ME];
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                const bool z = S::wave_zero(1, m);
                send1[m] = z ? real(0) : dtm * amdq[m];   // qadd of cell c-1 from this interface
                qadd[m] = z ? real(0) : -(dtc * apdq[m]);  // qadd of cell c, first term
                F[m] = real(0);
                cq[m] = real(0);
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
                        const int ml = lim_of(mw);
                        if (ml == 0) continue;
                        const real dl = __shfl_up_sync(FULL, dotr[mw], 1);
                        const real r = AR::div(s[mw] > real(0) ? dl : dotr[mw], wn2[mw]);
                        const real ph = wn2[mw] != real(0) ? phi(ml, r) : real(1);
#pragma unroll
                        for (int m = 0; m < ME; ++m)
                            if (!S::wave_zero(1, m)) w[mw][m] = ph * w[mw][m];
                    }
                }
                const real ave = real(0.5) * (dtm + dtc);
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
            real s3[ME], s4[ME], g1b[ME], g2b[ME];
#pragma unroll
            for (int m = 0; m < ME; ++m) s3[m] = s4[m] = g1b[m] = g2b[m] = real(0);
            if (trans > 0) {
                if (order != 1 && trans == 2) {
#pragma unroll
                    for (int m = 0; m < ME; ++m) {
                        if (S::wave_zero(1, m)) continue;
                        amdq[m] = amdq[m] + cq[m];
                        apdq[m] = apdq[m] - cq[m];
                    }
                }
                real bm[ME], bp[ME];
                if constexpr (solver_ctx<S>::value) A.solver.rpt_ctx(1, 1, cx, amdq, bm, bp);
                else A.solver.rpt(1, 1, qm_t, qc_t, a_mp, a_m, a_mn, amdq, bm, bp);
                const real hm = real(0.5) * dtm, hc = real(0.5) * dtc;
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    if (S::trans_zero(1, m)) continue;
                    s3[m] = -(hm * bm[m]);  // gadd(:,1,i-1) from this interface
                    s4[m] = -(hm * bp[m]);  // gadd(:,2,i-1)
                }
                if constexpr (solver_ctx<S>::value) A.solver.rpt_ctx(1, 2, cx, apdq, bm, bp);
                else A.solver.rpt(1, 2, qm_t, qc_t, a_cp, a_c, a_cn, apdq, bm, bp);
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    if (S::trans_zero(1, m)) continue;
                    g1b[m] = hc * bm[m];
                    g2b[m] = hc * bp[m];
                }
            }
            // interface c+1 (lane+1) finishes cell c
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                const bool wz = S::wave_zero(1, m), tz = S::trans_zero(1, m) || trans <= 0;
                real qa = real(0), dF = real(0), G1 = real(0), G2 = real(0);
                if (!wz) {
                    const real r1 = __shfl_down_sync(FULL, send1[m], 1);
                    const real r2 = __shfl_down_sync(FULL, F[m], 1);
                    qa = qadd[m] - r1;
                    dF = r2 - F[m];
                }
                if (!tz) {
                    const real r3 = __shfl_down_sync(FULL, s3[m], 1);
                    const real r4 = __shfl_down_sync(FULL, s4[m], 1);
                    G1 = r3 - g1b[m];
                    G2 = r4 - g2b[m];
                }
                real q2, Ax = real(0), Bx = real(0);
                if (!capa) {
                    q2 = qc_t[m];
                    if (!tz) q2 = q2 + Ax_prev[m];
                    if (!wz) q2 = (q2 + qa) - dtdx * dF;
                    if (!tz) {
                        q2 = q2 - dtdy * (G2 - G1);
                        Ax = dtdy * G2;
                        Bx = dtdy * G1;
                    }
                } else {
                    q2 = ((qc_t[m] + Ax_prev[m]) + qa) - AR::div(dtdx * dF + dtdy * (G2 - G1), a_c[ic]);
                    Ax = AR::div(dtdy * G2, a_cn[ic]);
                    Bx = AR::div(dtdy * G1, a_cp[ic]);
                }
                q3[m] = (!tz || capa) ? q2_prev[m] - Bx : q2_prev[m];  // x-part of (c, t-1)
                q2_prev[m] = q2;
                Ax_prev[m] = Ax;
            }
        }

        // ======== y-interface t+1 raw; y-interface t limited; y-part of (c, t-1) ========
        real wn[MW][ME], sn[MW], amn[ME], apn[ME];
        const auto cyn = iface_ctx(A.solver, 2, qc_t, qc_n);
        if constexpr (solver_ctx<S>::value) A.solver.rpn_ctx(2, cyn, qc_t, qc_n, wn, sn, amn, apn);
        else A.solver.rpn(2, qc_t, qc_n, a_c, a_cn, wn, sn, amn, apn);
        {
            const double dt0 = capa ? dtdy_d / (double)a_c[ic] : dtdy_d;
            const double dt1 = capa ? dtdy_d / (double)a_cn[ic] : dtdy_d;
            double em = 0.0;
#pragma unroll
            for (int mw = 0; mw < MW; ++mw)
                em = dmax(em, dmax(dt1 * (double)sn[mw], -dt0 * (double)sn[mw]));
            cfl = (cy_ok && t + 1 <= my) ? dmax(cfl, em) : cfl;
        }
        const real dty_p = capa ? AR::div(dtdy, a_cp[ic]) : dtdy;  // dtdy1d(t-1)
        const real dty_t = capa ? AR::div(dtdy, a_c[ic]) : dtdy;   // dtdy1d(t)
        real cqy[ME], Fy[ME], dotr_y[MW];
#pragma unroll
        for (int m = 0; m < ME; ++m) { cqy[m] = real(0); Fy[m] = real(0); }
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
                    const int ml = lim_of(mw);
                    if (ml == 0) continue;
                    real nn = real(0);
                    bool first = true;
#pragma unroll
                    for (int m = 0; m < ME; ++m) {
                        if (S::wave_zero(2, m)) continue;
                        nn = first ? wy[mw][m] * wy[mw][m] : nn + wy[mw][m] * wy[mw][m];
                        first = false;
                    }
                    const real r = AR::div(sy[mw] > real(0) ? dotl_y[mw] : dotr_y[mw], nn);
                    const real ph = nn != real(0) ? phi(ml, r) : real(1);
#pragma unroll
                    for (int m = 0; m < ME; ++m)
                        if (!S::wave_zero(2, m)) wy[mw][m] = ph * wy[mw][m];
                }
            }
            const real ave = real(0.5) * (dty_p + dty_t);
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
        real amo[ME], apo[ME];
#pragma unroll
        for (int m = 0; m < ME; ++m) { amo[m] = amy[m]; apo[m] = apy[m]; }
        real bma[ME], bpa[ME], bmb[ME], bpb[ME];
#pragma unroll
        for (int m = 0; m < ME; ++m) bma[m] = bpa[m] = bmb[m] = bpb[m] = real(0);
        if (trans > 0) {
            if (order != 1 && trans == 2) {
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    if (S::wave_zero(2, m)) continue;
                    amy[m] = amy[m] + cqy[m];
                    apy[m] = apy[m] - cqy[m];
                }
            }
            if constexpr (solver_ctx<S>::value) {
                A.solver.rpt_ctx(2, 1, cy, amy, bma, bpa);
                A.solver.rpt_ctx(2, 2, cy, apy, bmb, bpb);
            } else {
                A.solver.rpt(2, 1, qc_p, qc_t, a_mp, a_cp, a_pp, amy, bma, bpa);
                A.solver.rpt(2, 2, qc_p, qc_t, a_m, a_c, a_p, apy, bmb, bpb);
            }
        }
        const real hp = real(0.5) * dty_p, ht = real(0.5) * dty_t;
        const bool out = (t - 1 >= r0) && (lane >= 1) && (lane <= STRIP) && (c < mx);
        real* __restrict__ dst = qnew + (long long)(t - 1) * A.ld + c;
        real qo[ME];
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            const bool wz = S::wave_zero(2, m), tz = S::trans_zero(2, m) || trans <= 0;
            const real qa = wz ? real(0) : P1[m] - dty_p * amo[m];
            const real dF = wz ? real(0) : Fy[m] - Fy_prev[m];
            const real G1 = tz ? real(0) : -(hp * bma[m]) - P3[m];
            const real G2 = tz ? real(0) : -(hp * bpa[m]) - P4[m];
            real q6;
            if (!capa) {
                real q5 = q3[m];
                if (!tz) q5 = q5 + __shfl_up_sync(FULL, dtdx * G2, 1);  // from column c-1
                if (!wz && !tz) q5 = q5 + ((qa - dtdy * dF) - dtdx * (G2 - G1));
                else if (!wz) q5 = q5 + (qa - dtdy * dF);
                else if (!tz) q5 = q5 + (-(dtdx * (G2 - G1)));
                q6 = tz ? q5 : q5 - __shfl_down_sync(FULL, dtdx * G1, 1);  // from column c+1
            } else {
                const real Al = __shfl_up_sync(FULL, AR::div(dtdx * G2, a_pp[ic]), 1);
                const real Br = __shfl_down_sync(FULL, AR::div(dtdx * G1, a_mp[ic]), 1);
                const real q4 = q3[m] + Al;
                const real q5 = (q4 + qa) - AR::div(dtdy * dF + dtdx * (G2 - G1), a_cp[ic]);
                q6 = q5 - Br;
            }
            qo[m] = q6;
        }
        if constexpr (SRC) {
            if (K.src != 0) src_radial_cell(A, qo, c, K.src == 2 ? K.src_pre : K.src_post);
        }
        if (out) {
#pragma unroll
            for (int m = 0; m < ME; ++m) dst[m * A.fstride] = qo[m];
        }
        // contributions of y-interface t to cell (c, t); roll the window
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            P1[m] = S::wave_zero(2, m) ? real(0) : -(dty_t * apo[m]);
            P3[m] = S::trans_zero(2, m) ? real(0) : ht * bmb[m];
            P4[m] = S::trans_zero(2, m) ? real(0) : ht * bpb[m];
            Fy_prev[m] = Fy[m];
            amy[m] = amn[m];
            apy[m] = apn[m];
            qc_p[m] = qc_t[m];
            qm_t[m] = qm_n[m];
            qc_t[m] = qc_n[m];
        }
        cy = cyn;
#pragma unroll
        for (int mw = 0; mw < MW; ++mw) {
            dotl_y[mw] = dotr_y[mw];
            sy[mw] = sn[mw];
#pragma unroll
            for (int m = 0; m < ME; ++m) wy[mw][m] = wn[mw][m];
        }
        // release row t-1 and prefetch row t-1+RING into its slot
        __syncwarp();
        if (t - 1 + RING <= rlast) {
            if (lane == 0) issue(t - 1 + RING);
            last_issued = t - 1 + RING;
        }
        __syncwarp();
    }
    if (failed) {
        // drain: wait (bounded) for the rows still in flight before leaving
        for (int r = fail_row + 1; r <= last_issued; ++r) (void)wait_row(r);
        if (lane == 0) atomicOr(&ctl->err, CTL_ERR_TMA_TIMEOUT);
    }
    seq_base += (uint32_t)nrows;
}

// Resident CTAs per SM the step kernel is compiled for: CLAW_STEP2_MINB unless
// the solver asks for fewer (more registers per thread), via S::min_blocks.
template <class S, class = void>
struct step2_minb { static constexpr int value = CLAW_STEP2_MINB; };
template <class S>
struct step2_minb<S, std::void_t<decltype(S::min_blocks)>> { static constexpr int value = S::min_blocks; };

template <class S, class M, bool SRC = false>
__global__ void __launch_bounds__(32 * WARPS2D, step2_minb<S>::value)
step2_kernel(const __grid_constant__ Step2Args<S> A) {
    ClawCtl* ctl = A.ctl;
    __shared__ double red[WARPS2D];
    grid_dependency_sync();
    if (*(volatile int*)&ctl->done) return;
    const int cur = *(volatile int*)&ctl->cur;
    const double dtd = *(volatile double*)&ctl->dt;
    using R = Ring2D<S>;

    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* ring = smem + warp * R::WARP_BYTES;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + WARPS2D * R::WARP_BYTES) + warp * RING;
    if (lane == 0) {
        for (int sl = 0; sl < RING; ++sl) mbar_init(&bars[sl], 1);
        fence_barrier_init();
    }
    __syncwarp();

    const int my = A.my;
    double cfl = 0.0;
    bool failed = false;
    uint32_t seq_base = 0;

    const long long gw = (long long)blockIdx.x * WARPS2D + warp;
    long long u0 = (gw < A.nwarps) ? gw * A.units / A.nwarps : 0;
    const long long u1 = (gw < A.nwarps) ? (gw + 1) * A.units / A.nwarps : 0;
    StepConsts<S> K = step_consts(A, cur, dtd);
    // claw2 wraps the source steps around step2; a single step (claw_step) is step2 alone
    if (SRC && ctl->mode == CTL_ADVANCE) K.src = A.src_split;

    if (A.brows > 0) {
        const int items = A.nstrips * A.nblocks;
        for (int item = (int)gw; gw < A.nwarps && item < items && !failed; item += A.nwarps) {
            const int strip = item % A.nstrips, r0 = (item / A.nstrips) * A.brows;
            step2_rows<S, M, SRC>(A, K, strip, r0, min(A.brows, my - r0), ring, bars, seq_base,
                                  cfl, failed);
        }
    }
    while (A.brows == 0 && u0 < u1 && !failed) {
        const int strip = (int)(u0 / my);
        const int r0 = (int)(u0 % my);
        const int nr = (int)min((long long)(my - r0), u1 - u0);
        u0 += nr;
        step2_rows<S, M, SRC>(A, K, strip, r0, nr, ring, bars, seq_base, cfl, failed);
    }

    cta_cfl_and_control(ctl, cfl, red);
}

}  // namespace clawb200

namespace clawb200 {

// ------------------------------------------------------------- batch step ---
// Many independent grids (instances) of one solver and method, of uneven
// sizes, advance one step each per launch.  Each instance keeps its own
// claw2-style control block (its own dt from its own Courant number).  A
// persistent launch splits the rows of all instances that are not done
// evenly over its warps; the warp that completes an instance's last row runs
// that instance's controller.
constexpr int BATCH_MAX = 1024;

template <class S>
struct Step2Batch {
    const Step2Args<S>* inst;  // [count] per-instance arguments (TMA maps included)
    ClawCtl* ctls;             // [count] control blocks (inst[k].ctl == ctls + k)
    const int* units;          // [count] strips * my
    int count;
    int nwarps;                // warps of the launch
    int min_rows;              // tile height: fewest rows a sharing warp takes
    int* active;               // instances still advancing (polled by the host)
    int* err;                  // device error flags of the batch
};

template <class S, class M>
__global__ void __launch_bounds__(32 * WARPS2D, step2_minb<S>::value)
step2_batch_kernel(const __grid_constant__ Step2Batch<S> B) {
    using R = Ring2D<S>;
    constexpr unsigned FULL = 0xffffffffu;
    __shared__ int pre[BATCH_MAX + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    grid_dependency_sync();
    // units of the active instances, then their prefix sums
    for (int k = threadIdx.x; k < B.count; k += blockDim.x)
        pre[k + 1] = *(volatile int*)&B.ctls[k].done ? 0 : B.units[k];
    __syncthreads();
    if (warp == 0) {
        int run = 0;
        for (int base = 0; base < B.count; base += 32) {
            const int k = base + lane;
            int x = k < B.count ? pre[k + 1] : 0;
            for (int off = 1; off < 32; off <<= 1) {
                const int y = __shfl_up_sync(FULL, x, off);
                if (lane >= off) x += y;
            }
            if (k < B.count) pre[k + 1] = run + x;
            run += __shfl_sync(FULL, x, 31);
        }
        if (lane == 0) pre[0] = 0;
    }
    __syncthreads();
    const long long total = pre[B.count];
    if (total == 0) return;
    // every sharing warp gets >= min_rows rows of a strip (tile height, tuned)
    const long long nw = min((long long)B.nwarps, max(1LL, total / B.min_rows));
    const long long gw = (long long)blockIdx.x * WARPS2D + warp;
    if (gw >= nw) return;

    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* ring = smem + warp * R::WARP_BYTES;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + WARPS2D * R::WARP_BYTES) + warp * RING;
    if (lane == 0) {
        for (int sl = 0; sl < RING; ++sl) mbar_init(&bars[sl], 1);
        fence_barrier_init();
    }
    __syncwarp();

    long long u0 = gw * total / nw;
    const long long u1 = (gw + 1) * total / nw;
    uint32_t seq_base = 0;
    bool failed = false;
    int k = 0;
    {   // instance holding u0: the last k with pre[k] <= u0
        int lo = 0, hi = B.count - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (pre[mid] <= u0) lo = mid; else hi = mid - 1;
        }
        k = lo;
    }
    while (u0 < u1 && !failed) {
        while (pre[k + 1] <= u0) ++k;
        const Step2Args<S>& A = B.inst[k];
        ClawCtl* ctl = B.ctls + k;
        const int cur = *(volatile int*)&ctl->cur;
        const double dtd = *(volatile double*)&ctl->dt;
        const StepConsts<S> K = step_consts(A, cur, dtd);
        const long long off = u0 - pre[k];
        const int my = A.my;
        const int strip = (int)(off / my), r0 = (int)(off % my);
        const int nr = (int)min((long long)(my - r0), u1 - u0);
        u0 += nr;
        double cfl = 0.0;
        step2_rows<S, M>(A, K, strip, r0, nr, ring, bars, seq_base, cfl, failed);
        for (int o = 16; o > 0; o >>= 1) cfl = fmax(cfl, __shfl_xor_sync(FULL, cfl, o));
        if (lane == 0) {
            if (failed) atomicOr(B.err, CTL_ERR_TMA_TIMEOUT);
            double m = cfl;
            if (!(m > 0.0)) m = (m != m) ? m : 0.0;  // canonical +0, keep NaN
            atomicMax(&ctl->cfl_bits, (unsigned long long)__double_as_longlong(m));
            __threadfence();
            const unsigned prev = atomicAdd(&ctl->ctas_done, (unsigned)nr);
            if (prev + (unsigned)nr == (unsigned)B.units[k]) {
                __threadfence();
                ctl_finish_step(ctl);
                if (ctl->done) atomicSub(B.active, 1);
                __threadfence();
            }
        }
        __syncwarp();
    }
}

}  // namespace clawb200
