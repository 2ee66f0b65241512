// Dimensionally split 2D step (dimsp2 + step2ds, Godunov and Strang) for
// linear constant-coefficient acoustics in characteristic variables: the
// CLAW_FP64_FMA and CLAW_FP32 path of claw2's method(3) = -1 / -2.
//
// Reference: src/2d/dimsp2.f:1-99, src/2d/step2ds.f90:1-275 with
// src/2d/flux2.f90:97-181 (no transverse part), src/2d/bc2.f, and
// src/2d/claw2.f:659-680.
//
// The sweeps are those of the generic fused split kernel (step2ds.cuh) --
// one warp marches up the rows of a strip and applies every sweep to a row as
// it passes, so q is read once and written once per step:
//   stage A  x-sweep of row t (dt, Strang dt/2) on every row the reference
//            x-sweeps, ghost rows included; ghost columns keep their bc2
//            value;
//   stage B  y-sweep: the interface between the x-swept rows t and t+1 is
//            formed, the one below limited, and row t-1 gets its y-update;
//   stage C  (Strang) x-sweep of that y-swept row with dt/2, from its lane
//            neighbours' stage B values.
// -- written in characteristic variables as step2_char_kernel writes the
// unsplit step: a jump splits into strengths on the fixed eigenvectors
// (-Z,1,0), (Z,1,0) along x and (-Z,0,1), (Z,0,1) along y, the limiter is the
// closed form phi(n/a)·a, and fadd reduces to two scalars per interface.
// Two columns per lane: stage A is exact on lanes 1..30, so Godunov writes the
// 60 columns of lanes 1..30 (the unsplit kernel's strip and ring box) and
// Strang, whose stage C needs stage B on both neighbours, the 56 of lanes
// 2..29 (box from 6 / 8 columns left of the strip, 16-byte aligned).
//
// The Courant number of each sweep is (dt_sweep/dx) c as step2ds forms it
// over every interface (the speeds are constant), and dimsp2's choice among
// the sweeps' is cta_split_cfl_and_control's, so the dt sequence equals the
// reference-order split path's bit for bit.
#pragma once
#include "char2d.cuh"
#include "step2ds.cuh"

namespace clawb200 {

// Coefficients of one x-sweep.  The sweep carries the wave strengths
// unscaled (2Z a1 = Z du - dp, 2Z a2 = Z du + dp) and the correction fluxes as
// the bare limited sums d = b2 - b1 (pressure) and s = b1 + b2 (velocity):
// every limiter is positively homogeneous of degree one and each flux enters
// only its own difference, so 1/(2Z) and kappa/2 sit in these coefficients
// (Z / (2Z) = 1/2).
template <typename real>
struct CharSplitConsts {
    real qpxh, quxh;  // dt/dx cZ and dt/dx c, over 2Z
    real kpx, kux;    // dt/dx kappa Z/2 and dt/dx kappa/2, over 2Z
};

template <typename real>
__device__ __forceinline__ CharSplitConsts<real> char_xsweep_consts(double dtdx_d, const CharAcoustics2D<real>& S) {
    CharSplitConsts<real> k;
    const real dtdx = (real)dtdx_d, c = S.cc, h = S.hz;
    const real kx = c * (real(1) - c * dtdx);
    k.qpxh = real(0.5) * (dtdx * c);
    k.quxh = dtdx * c * h;
    k.kpx = real(0.25) * (dtdx * kx);
    k.kux = real(0.5) * (dtdx * kx * h);
    return k;
}

// One x-sweep of a row, two columns per lane: (p0, u0), (p1, u1) at columns
// c0, c1 and (pM, uM) at c0-1; returns the swept p and u of c0 and c1 (exact
// where lanes l-1 and l+1 hold real data).  flux2 without the transverse part
// (flux2.f90:110-181) and step2ds's update (step2ds.f90:201-214).
template <typename real, int LIM>
__device__ __forceinline__ void char_xsweep(real pM, real uM, real p0, real u0, real p1, real u1,
                                            const CharSplitConsts<real>& K, const CharAcoustics2D<real>& S,
                                            int lim, int lim2, real& xp0, real& xu0, real& xp1, real& xu1) {
    constexpr unsigned FULL = 0xffffffffu;
    const real Z = S.zz;
    const real a1_0 = Z * (u0 - uM) - (p0 - pM);
    const real a2_0 = Z * (u0 - uM) + (p0 - pM);
    const real a1_1 = Z * (u1 - u0) - (p1 - p0);
    const real a2_1 = Z * (u1 - u0) + (p1 - p0);
    const real a1_R = __shfl_down_sync(FULL, a1_0, 1);  // interface c1+1 (lane+1's I0)
    const real a2_L = __shfl_up_sync(FULL, a2_1, 1);    // interface c0-1 (lane-1's I1)
    const real l1_0 = limited_strength<real, LIM>(a1_0, a1_1, lim);
    const real l2_0 = limited_strength<real, LIM>(a2_0, a2_L, lim2);
    const real l1_1 = limited_strength<real, LIM>(a1_1, a1_R, lim);
    const real l2_1 = limited_strength<real, LIM>(a2_1, a2_0, lim2);
    const real d0 = l2_0 - l1_0, s0 = l1_0 + l2_0;
    const real d1 = l2_1 - l1_1, s1 = l1_1 + l2_1;
    const real dR = __shfl_down_sync(FULL, d0, 1), sR = __shfl_down_sync(FULL, s0, 1);
    xp0 = (p0 - K.qpxh * (a2_0 + a1_1)) - K.kpx * (d1 - d0);
    xu0 = (u0 + K.quxh * (a1_1 - a2_0)) - K.kux * (s1 - s0);
    xp1 = (p1 - K.qpxh * (a2_1 + a1_R)) - K.kpx * (dR - d1);
    xu1 = (u1 + K.quxh * (a1_R - a2_1)) - K.kux * (sR - s1);
}

constexpr int STRIP_STRANG = 56;  // output columns of a Strang strip (lanes 2..29)

template <typename real, int LIM, int BCM, bool STRANG>
__global__ void __launch_bounds__(32 * WARPS2D, sizeof(real) == 8 ? CLAW_CHAR_MINB : CLAW_CHAR_MINB_F32)
step2s_char_kernel(const __grid_constant__ CharArgs<real> A) {
    constexpr bool PX = BCM == CHAR_BC_PERX;
    constexpr bool WALLS = BCM != CHAR_BC_EXTRAP;
    using R = CharRing<real>;
    using P2 = typename Pair<real>::type;
    constexpr int W = R::W;
    constexpr unsigned FULL = 0xffffffffu;
    constexpr int STRIPW = STRANG ? STRIP_STRANG : STRIP2;
    // the ring box starts XQS columns left of the strip; lane 0's first column is b - LEFT
    constexpr int XQS = STRANG ? (sizeof(real) == 8 ? 6 : 8) : R::XQ;
    constexpr int LEFT = STRANG ? 4 : 2;
    ClawCtl* ctl = A.ctl;
    __shared__ double red[3 * WARPS2D];
    grid_dependency_sync();
    if (*(volatile int*)&ctl->done) return;
    const int cur = *(volatile int*)&ctl->cur;
    const double dtd = *(volatile double*)&ctl->dt;
    // the sweeps' lengths as dimsp2 takes them (src/2d/dimsp2.f:52-62)
    const double dta = STRANG ? dtd / 2.0 : dtd;
    const double dtdx_a_d = dta / A.dx, dtdy_d = dtd / A.dy, dtdx_c_d = (dtd / 2.0) / A.dx;
    const CharSplitConsts<real> KA = char_xsweep_consts<real>(dtdx_a_d, A.s);
    const CharSplitConsts<real> KC = char_xsweep_consts<real>(dtdx_c_d, A.s);
    const real c = A.s.cc, Z = A.s.zz, h = A.s.hz;
    const real dtdy = (real)dtdy_d;
    const real ky = c * (real(1) - c * dtdy);
    // the y-sweep's coefficients, scaled as the x-sweep's (char_xsweep_consts)
    const real qpyh = real(0.5) * (dtdy * c), qvyh = dtdy * c * h;
    const real kpy = real(0.25) * (dtdy * ky), kvy = real(0.5) * (dtdy * ky * h);
    const real* __restrict__ qold = A.q[cur];
    real* __restrict__ qnew = A.q[cur ^ 1];
    const CUtensorMap* tmq = &A.tmq[cur];

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
    const unsigned long long wait_ns = ctl_wait_ns(ctl);
    bool failed = false;
    uint32_t seq_base = 0;
    bool any_work = false;
    const int gw = blockIdx.x * WARPS2D + warp;
    const int items = A.nstrips * A.nblocks;

    for (int item = gw; gw < A.nwarps && item < items && !failed; item += A.nwarps) {
        any_work = true;
        const int strip = item % A.nstrips;
        const int r0 = (item / A.nstrips) * A.brows;
        const int nr = min(A.brows, my - r0);
        const int b = strip * STRIPW;
        const int c0 = b - LEFT + 2 * lane, c1 = c0 + 1;  // this lane's two columns
        const int x0 = b - XQS;
        const int rfirst = r0 - 2, rlast = r0 + nr + 1;
        const int nrows = rlast - rfirst + 1;
        const int skip1 = strip == 0 ? *(volatile const int*)&ctl->skip_row : 0;  // test hook

        auto seq_of = [&](int r) -> uint32_t { return seq_base + (uint32_t)(r - rfirst); };
        auto issue = [&](int r) {
            if (skip1 != 0 && r == skip1 - 1) return;
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
            return mbar_wait_bounded(&bars[sq & (RING - 1)], (sq >> RING_LOG) & 1u, wait_ns);
        };
        auto row_ptr = [&](int r) -> const real* {
            return reinterpret_cast<const real*>(ring + (int)(seq_of(r) & (RING - 1)) * R::SLOT);
        };
        // Godunov writes lanes 1..30, Strang (stage C) lanes 2..29
        const bool out_lane = STRANG ? (lane >= 2 && lane <= 29) : (lane >= 1 && lane <= 30);
        // ghost columns are not x-swept (step2ds.f90: the x-sweep updates 1..mx)
        const bool xin0 = c0 >= 0 && c0 < mx, xin1 = c1 >= 0 && c1 < mx;

        auto march = [&](auto int_tag) {
            constexpr bool INT = decltype(int_tag)::value;
            auto colsrc = [&](int col) -> ColSrc {
                ColSrc cs;
                cs.src = bc_map(col, mx, A.bc[0], A.bc[1], cs.neg);
                cs.glob = (cs.src - x0) < 0 || (cs.src - x0) >= W;
                cs.idx = cs.glob ? 0 : cs.src - x0;
                return cs;
            };
            const ColSrc sM = colsrc(c0 - 1), s0 = colsrc(c0), s1 = colsrc(c1);
            const bool any_global = !INT && PX && __any_sync(FULL, sM.glob || s0.glob || s1.glob);
            const bool out0 = out_lane && (INT || c0 < mx), out1 = out_lane && (INT || c1 < mx);
            const int ib = c0 - x0;  // ring index of c0 in an interior strip
            auto fetch = [&](const real* sq, int sr, bool nyneg, const ColSrc& cs, int m) -> real {
                real v = sq[m * W + cs.idx];
                if constexpr (PX && !INT) {
                    if (any_global && cs.glob) v = qold[m * A.fstride + (long long)sr * A.ld + cs.src];
                }
                if constexpr (WALLS) {
                    if (!INT && m == 1 && cs.neg) v = -v;
                    if (m == 2 && nyneg) v = -v;
                }
                return v;
            };
            auto fetch2 = [&](const real* sq, int sr, bool nyneg, int m, real& v0, real& v1) {
                if constexpr (INT) {
                    const P2 v = *reinterpret_cast<const P2*>(sq + m * W + ib);
                    v0 = v.x;
                    v1 = v.y;
                    if constexpr (WALLS) {
                        if (m == 2 && nyneg) { v0 = -v0; v1 = -v1; }
                    }
                } else {
                    v0 = fetch(sq, sr, nyneg, s0, m);
                    v1 = fetch(sq, sr, nyneg, s1, m);
                }
            };
            auto fetchM = [&](const real* sq, int sr, bool nyneg, int m) -> real {
                if constexpr (INT) return sq[m * W + ib - 1];
                else return fetch(sq, sr, nyneg, sM, m);
            };
            // stage A of row r: x-swept (p, u) of c0, c1; v untouched by an x-sweep
            auto stage_a = [&](int r, real xa[2][3]) {
                bool ng = false;
                int sr = 0;
                if constexpr (WALLS || PX) sr = bc_map(r, my, A.bc[2], A.bc[3], ng);
                const real* sq = row_ptr(r);
                real p[2], u[2], v[2];
                fetch2(sq, sr, ng, 0, p[0], p[1]);
                fetch2(sq, sr, ng, 1, u[0], u[1]);
                fetch2(sq, sr, ng, 2, v[0], v[1]);
                const real pM = fetchM(sq, sr, ng, 0), uM = fetchM(sq, sr, ng, 1);
                real xp0, xu0, xp1, xu1;
                char_xsweep<real, LIM>(pM, uM, p[0], u[0], p[1], u[1], KA, A.s, A.lim, A.lim2, xp0, xu0, xp1,
                                       xu1);
                xa[0][0] = (INT || xin0) ? xp0 : p[0];
                xa[0][1] = (INT || xin0) ? xu0 : u[0];
                xa[0][2] = v[0];
                xa[1][0] = (INT || xin1) ? xp1 : p[1];
                xa[1][1] = (INT || xin1) ? xu1 : u[1];
                xa[1][2] = v[1];
            };

            // carried per column k: x-swept rows t-1 (xb) and t (xc); y-interface
            // t (between them) and t-1 (below)
            real xb[2][3], xc[2][3];
            real a1y[2], a2y[2];
            real a2y_lo[2] = {}, dy_lo[2] = {}, sy_lo[2] = {};
            int last_issued = rfirst + (nrows < RING ? nrows : RING) - 1;
            int fail_row = rlast + 1;

            if (!wait_row(rfirst) || !wait_row(rfirst + 1)) { failed = true; fail_row = rfirst; }
            if (!failed) {
                stage_a(rfirst, xb);
                stage_a(rfirst + 1, xc);
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const real dp = xc[k][0] - xb[k][0], dv = xc[k][2] - xb[k][2];
                    a1y[k] = Z * dv - dp;
                    a2y[k] = Z * dv + dp;
                }
            }

            for (int t = r0 - 1; t <= r0 + nr && !failed; ++t) {
                if (!wait_row(t + 1)) { failed = true; fail_row = t + 1; break; }
                real xn[2][3];
                stage_a(t + 1, xn);
                // ---- stage B: interface t+1 raw, interface t limited, row t-1 updated
                real o[2][3], dyk[2], syk[2], a1n[2], a2n[2];
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const real dp = xn[k][0] - xc[k][0], dv = xn[k][2] - xc[k][2];
                    a1n[k] = Z * dv - dp;
                    a2n[k] = Z * dv + dp;
                    const real b1 = limited_strength<real, LIM>(a1y[k], a1n[k], A.lim);      // upwind t+1
                    const real b2 = limited_strength<real, LIM>(a2y[k], a2y_lo[k], A.lim2);  // upwind t-1
                    dyk[k] = b2 - b1;
                    syk[k] = b1 + b2;
                    o[k][0] = (xb[k][0] - qpyh * (a2y_lo[k] + a1y[k])) - kpy * (dyk[k] - dy_lo[k]);
                    o[k][1] = xb[k][1];
                    o[k][2] = (xb[k][2] + qvyh * (a1y[k] - a2y_lo[k])) - kvy * (syk[k] - sy_lo[k]);
                }
                if constexpr (STRANG) {
                    // ---- stage C: the y-swept row t-1 x-swept with dt/2; column
                    // c0-1 is lane l-1's c1 (ghost columns keep the y-swept value)
                    const real pM = __shfl_up_sync(FULL, o[1][0], 1), uM = __shfl_up_sync(FULL, o[1][1], 1);
                    real xp0, xu0, xp1, xu1;
                    char_xsweep<real, LIM>(pM, uM, o[0][0], o[0][1], o[1][0], o[1][1], KC, A.s, A.lim, A.lim2,
                                           xp0, xu0, xp1, xu1);
                    if (INT || xin0) { o[0][0] = xp0; o[0][1] = xu0; }
                    if (INT || xin1) { o[1][0] = xp1; o[1][1] = xu1; }
                }
                if (t - 1 >= r0) {
                    real* dst = qnew + (long long)(t - 1) * A.ld + c0;
                    if constexpr (INT) {
                        if (out_lane) {
                            *reinterpret_cast<P2*>(dst) = P2{o[0][0], o[1][0]};
                            *reinterpret_cast<P2*>(dst + A.fstride) = P2{o[0][1], o[1][1]};
                            *reinterpret_cast<P2*>(dst + 2 * A.fstride) = P2{o[0][2], o[1][2]};
                        }
                    } else {
                        if (out0) { dst[0] = o[0][0]; dst[A.fstride] = o[0][1]; dst[2 * A.fstride] = o[0][2]; }
                        if (out1) { dst[1] = o[1][0]; dst[A.fstride + 1] = o[1][1]; dst[2 * A.fstride + 1] = o[1][2]; }
                    }
                }
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    a2y_lo[k] = a2y[k];
                    dy_lo[k] = dyk[k];
                    sy_lo[k] = syk[k];
                    a1y[k] = a1n[k];
                    a2y[k] = a2n[k];
#pragma unroll
                    for (int m = 0; m < 3; ++m) {
                        xb[k][m] = xc[k][m];
                        xc[k][m] = xn[k][m];
                    }
                }
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
        };
        // interior strip: the warp's columns and lane 0's left neighbour inside the grid
        const bool interior = c0 - 2 * lane - 1 >= 0 && b - LEFT + 63 <= mx - 1;
        if (interior) march(std::true_type{});
        else march(std::false_type{});
        seq_base += (uint32_t)nrows;
    }
    // the sweeps' Courant numbers as step2ds forms them over every interface
    // (dt_sweep/dx c; the speeds are constant), combined as dimsp2 combines them
    const double cd = (double)c;
    const double c3[3] = {any_work ? dtdx_a_d * cd : 0.0, any_work ? dtdy_d * cd : 0.0,
                          any_work ? dtdx_c_d * cd : 0.0};
    cta_split_cfl_and_control(ctl, c3, STRANG ? 3 : 2, red);
}

}  // namespace clawb200
