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

// x with the sign of s flipped in (x * sign(s)), and copysign, by bit operations.
__device__ __forceinline__ double sign_times(double x, double s) {
    return __longlong_as_double(__double_as_longlong(x) ^
                                (__double_as_longlong(s) & (long long)0x8000000000000000ull));
}
__device__ __forceinline__ float sign_times(float x, float s) {
    return __int_as_float(__float_as_int(x) ^ (__float_as_int(s) & (int)0x80000000u));
}

// MC in FP64 by compare-and-select on magnitudes.  When a and n share a
// sign, phi a = sign(a) 2 min(|a|, |n|, (|a|+|n|)/4); otherwise 0.  Same value
// as the min/max form below (every candidate is formed by the same
// operations), but no fmin/fmax: their NaN rules cost extra instructions in
// FP64, and the select picks one of two registers.
__device__ __forceinline__ double mc_strength(double a, double n) {
    const double mn = fabs(a) < fabs(n) ? a : n;  // |mn| = min(|a|, |n|)
    const double q = 0.25 * (fabs(a) + fabs(n));
    const double r = q < fabs(mn) ? q : mn;       // |r| = the smaller of the two
    const int ah = __double2hiint(a), nh = __double2hiint(n);
    // +-2 with the sign of a when the signs agree, else +0 (n = +-0 gives r = 0)
    const int s2 = (ah ^ nh) >= 0 ? ((ah & (int)0x80000000u) | 0x40000000) : 0;
    return fabs(r) * __hiloint2double(s2, 0);
}

// min / max by compare-and-select in FP64 (the same values as fmin / fmax for
// non-NaN operands, fewer instructions); the native ones in FP32
template <typename real>
__device__ __forceinline__ real mn2(real x, real y) {
    if constexpr (sizeof(real) == 8) return x < y ? x : y;
    else return fminf(x, y);
}
template <typename real>
__device__ __forceinline__ real mx2(real x, real y) {
    if constexpr (sizeof(real) == 8) return x > y ? x : y;
    else return fmaxf(x, y);
}

// phi(r) * a of inlinelimiter.f90:71-97 (philim.f90 of src/2d) for the
// strength ratio r = n / a (n = upwind neighbour's strength), written with
// A = |a| and N = n sign(a), so that r = N / A (multiply phi's arguments by
// a, reversing min/max when a < 0):
//   minmod    sign(a) max(0, min(A, N))
//   superbee  sign(a) max(0, min(A, 2N), min(2A, N))
//   van Leer  sign(a) 2AN / (A + N) for N > 0, else 0   (one reciprocal)
//   MC        sign(a) max(0, min(2A, 2N, (A + N) / 2))
//   Beam-Warming  n
// a == 0 gives 0, as the reference skips a zero wave.
// LIM >= 0 fixes the limiter at compile time; LIM = -1 reads it at run time
// (a warp-uniform branch).
template <typename real, int LIM>
__device__ __forceinline__ real limited_strength(real a, real n, int lim_rt) {
    const int lim = LIM >= 0 ? LIM : lim_rt;
    if constexpr (sizeof(real) == 8) {
        if (lim == 4) return mc_strength(a, n);
    }
    if (lim == 0) return a;
    if (lim == 5) return a != real(0) ? n : real(0);
    const real A = fabs(a), N = sign_times(n, a);
    real m;
    if (lim == 1) {
        m = mn2(A, N);
    } else if (lim == 2) {
        m = mx2(mn2(A, real(2) * N), mn2(real(2) * A, N));
    } else if (lim == 3) {
        const real pos = N > real(0) ? N : real(0);
        m = real(2) * A * pos * rcp_newton(A + (N > real(0) ? N : real(1)));
    } else {
        m = real(2) * mn2(mn2(A, N), real(0.25) * (A + N));
    }
    return sign_times(mx2(real(0), m), a);
}

template <typename real>
struct CharArgs {
    CUtensorMap tmq[2];
    real* q[2];
    long long ld, fstride;
    int mx, my, nstrips;
    int bc[4];
    int lim, lim2;  // limiters of wave 1 (speed -c) and wave 2 (speed +c), mthlim(1:2)
    double dx, dy;
    // Work items: row block b (brows rows) of strip s, item = b * nstrips + s,
    // so the warps at work on one row block hold adjacent strips and stream
    // neighbouring DRAM pages.  Warp w takes items w, w + nwarps, ...
    int brows, nblocks;
    int nwarps;
    ClawCtl* ctl;
    CharAcoustics2D<real> s;
};

// Two columns per lane: a warp covers 64 columns and writes STRIP2 = 60.
constexpr int STRIP2 = 60;
static_assert(STRIP2 % 4 == 0, "strip start must stay a multiple of 4 for TMA");

template <typename real>
struct CharRing {
    // columns b-4 .. b+61 (b-4 keeps the box start 16-byte aligned)
    static constexpr int XQ = 4;
    static constexpr int W = sizeof(real) == 8 ? 66 : 68;
    static constexpr int QB = 3 * W * (int)sizeof(real);
    static constexpr int SLOT = ((QB + 127) / 128) * 128;
    static constexpr int WARP_BYTES = RING * SLOT;
    static constexpr int SMEM = WARPS2D * WARP_BYTES + WARPS2D * RING * 8 + 64;
};

// One column's q source in the ring (or, for a periodic ghost outside the
// box, in global memory) and its wall sign flip.
struct ColSrc {
    int idx;   // ring index
    int src;   // interior column (global fallback)
    bool neg;  // wall: negate the normal velocity
    bool glob; // periodic ghost outside the ring box
};

#ifndef CLAW_CHAR_MINB
#define CLAW_CHAR_MINB 3  // FP64: 168 registers, 12 warps per SM, no spills (fastest measured)
#endif
#ifndef CLAW_CHAR_MINB_F32
// FP32: 121 registers, 16 warps per SM, no spills; 10 % faster than 3 CTAs,
// and faster than 5 (93 registers: 115 against 119 us per 4096^2 step) or 6
// (spills: 138 us), whose more and shorter row blocks add halo rows
#define CLAW_CHAR_MINB_F32 4
#endif
#ifndef CLAW_CHAR_UNROLL
#define CLAW_CHAR_UNROLL 2
#endif

// Boundary-condition classes compiled separately:
//   CHAR_BC_EXTRAP  extrapolation on every side (no sign flips)
//   CHAR_BC_WALLS   any mix without periodic x (wall sign flips applied)
//   CHAR_BC_PERX    periodic x: halo lanes of the edge strips may need a
//                   column from the far side of the grid that is not in the
//                   ring box, read from global memory
enum { CHAR_BC_EXTRAP = 0, CHAR_BC_WALLS = 1, CHAR_BC_PERX = 2 };

// Two adjacent values of one field (columns c0, c0+1) as one shared-memory
// load; the pair starts on a 16-byte (FP64) / 8-byte (FP32) boundary.
template <typename real> struct Pair;
template <> struct Pair<double> { using type = double2; };
template <> struct Pair<float> { using type = float2; };

// ORD = method(2) (1: first order, no correction fluxes), TRN = method(3)
// (0: no transverse propagation; 1: the fluctuations alone are split; 2: with
// the correction fluxes incorporated, flux2.f90:186-195).  LIM is wave 1's
// limiter (mthlim(1)), LIM2 wave 2's (mthlim(2)); -1 reads it at run time.
template <typename real, int LIM, int BCM, int ORD = 2, int TRN = 2, int LIM2 = LIM>
__global__ void __launch_bounds__(32 * WARPS2D, sizeof(real) == 8 ? CLAW_CHAR_MINB : CLAW_CHAR_MINB_F32)
step2_char_kernel(const __grid_constant__ CharArgs<real> A) {
    static_assert((ORD == 1 || ORD == 2) && TRN >= 0 && TRN <= ORD, "transverse_waves <= order");
    constexpr bool PX = BCM == CHAR_BC_PERX;
    constexpr bool WALLS = BCM != CHAR_BC_EXTRAP;
    constexpr int kUnroll = CLAW_CHAR_UNROLL;
    using R = CharRing<real>;
    using P2 = typename Pair<real>::type;
    constexpr int W = R::W;
    constexpr unsigned FULL = 0xffffffffu;
    ClawCtl* ctl = A.ctl;
    __shared__ double red[WARPS2D];
    grid_dependency_sync();
    if (*(volatile int*)&ctl->done) return;
    const int cur = *(volatile int*)&ctl->cur;
    const double dtd = *(volatile double*)&ctl->dt;
    const double dtdx_d = dtd / A.dx, dtdy_d = dtd / A.dy;
    const real dtdx = (real)dtdx_d, dtdy = (real)dtdy_d;
    const real* __restrict__ qold = A.q[cur];
    real* __restrict__ qnew = A.q[cur ^ 1];
    const CUtensorMap* tmq = &A.tmq[cur];
    const real c = A.s.cc, Z = A.s.zz, h = A.s.hz;
    // kappa = c(1 - c dt/dx): second-order coefficient (flux2.f90:156-157);
    // fadd = kappa/2 (Z(b2-b1), b1+b2); transverse gamma = (dt/dx) c/4,
    // delta = (dt/dx) c/(4Z), each scaled by the other direction's dt/d.
    const real kx = c * (real(1) - c * dtdx), ky = c * (real(1) - c * dtdy);
    const real gx = dtdy * (dtdx * c * real(0.25)), dx4 = dtdy * (dtdx * c * real(0.25) / Z);
    const real gy = dtdx * (dtdy * c * real(0.25)), dy4 = dtdx * (dtdy * c * real(0.25) / Z);
    const real gx2 = real(2) * gx, gy2 = real(2) * gy;
    // The march carries the strengths unscaled, 2Z a1 = Z du - dp and
    // 2Z a2 = Z du + dp; the pressure correction flux doubled, Fp' = 2 Fp;
    // and for the velocity correction flux, which enters only its own
    // difference, the bare sum s = b1 + b2.  Every limiter is positively
    // homogeneous of degree one and every use of a strength or a flux is
    // linear, so the factors 1/(2Z), 2 and kappa/2 sit in these coefficients
    // instead of costing a multiply per interface (Z / (2Z) = 1/2).
    const real fxp2 = real(0.5) * kx, fyp2 = real(0.5) * ky;        // Fp' per (b2 - b1)
    const real kux = real(0.5) * (dtdx * kx * h), kvy = real(0.5) * (dtdy * ky * h);  // dt/d Fu per s
    const real qpxh = real(0.5) * (dtdx * c), quxh = dtdx * c * h;  // dt/dx cZ, dt/dx c over 2Z
    const real qpyh = real(0.5) * (dtdy * c), qvyh = dtdy * c * h;
    const real cZh = real(0.5) * c;                                  // cZ over 2Z
    const real dtdx2 = real(0.5) * dtdx, dtdy2 = real(0.5) * dtdy;  // dt/d on Fp' differences

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
        const int b = strip * STRIP2;
        const int c0 = b - 2 + 2 * lane, c1 = c0 + 1;  // this lane's two columns
        const int x0 = b - R::XQ;
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
        const bool out_lane = lane >= 1 && lane <= 30;

        // The march over the rows of one work item.  INT: every column of the
        // strip (b-3 .. b+61) is interior, so a lane's columns sit at ring
        // index 2+2*lane (+1) with no x boundary condition: pairs of values
        // load and store as one vector access.  Otherwise the columns go
        // through the boundary maps (edge strips).
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
            const int ib = 2 + 2 * lane;  // ring index of c0 in an interior strip
            // field m of column cs at row r (boundary conditions applied)
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
            // fields m of columns c0, c1 at row r
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

            // carried per column k = 0, 1
            real q2p[2][3] = {};            // x-part of (c_k, t) awaiting row t+1's transfer
            [[maybe_unused]] real sxp[2] = {};  // x-slice t-1's transverse sum S, whose split reaches row t
            real a1y[2] = {}, a2y[2] = {};  // y-interface t strengths
            real a2y_lo[2] = {}, Fpy_lo[2] = {}, Svy_lo[2] = {};  // y-interface t-1
            real pc[2] = {}, vc[2] = {};    // p, v of row t (row t+1 of the previous trip)
            int last_issued = rfirst + (nrows < RING ? nrows : RING) - 1;
            int fail_row = rlast + 1;

            if (!wait_row(rfirst) || !wait_row(rfirst + 1)) { failed = true; fail_row = rfirst; }
            if (!failed) {
                bool ng0, ng1;
                const int sr0 = bc_map(rfirst, my, A.bc[2], A.bc[3], ng0);
                const int sr1 = bc_map(rfirst + 1, my, A.bc[2], A.bc[3], ng1);
                const real* q0p = row_ptr(rfirst);
                const real* q1p = row_ptr(rfirst + 1);
                real p0[2], v0[2];
                fetch2(q0p, sr0, ng0, 0, p0[0], p0[1]);
                fetch2(q0p, sr0, ng0, 2, v0[0], v0[1]);
                fetch2(q1p, sr1, ng1, 0, pc[0], pc[1]);
                fetch2(q1p, sr1, ng1, 2, vc[0], vc[1]);
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const real dp = pc[k] - p0[k];
                    const real dv = vc[k] - v0[k];
                    a1y[k] = Z * dv - dp;
                    a2y[k] = Z * dv + dp;
                }
            }

            // two rows per trip: the carried state rotates by renaming, not copies
#pragma unroll kUnroll
            for (int t = r0 - 1; t <= r0 + nr && !failed; ++t) {
                if (!wait_row(t + 1)) { failed = true; fail_row = t + 1; break; }
                bool ngt = false, ngn = false;
                int srt = 0, srn = 0;
                if constexpr (WALLS || PX) {
                    srt = bc_map(t, my, A.bc[2], A.bc[3], ngt);
                    srn = bc_map(t + 1, my, A.bc[2], A.bc[3], ngn);
                }
                const real* qt = row_ptr(t);
                const real* qn = row_ptr(t + 1);
                // row t: p, u at columns c0-1, c0, c1 (p carried); v carried.
                // row t+1: p, v.
                const real pM = fetchM(qt, srt, ngt, 0), uM = fetchM(qt, srt, ngt, 1);
                real p[2] = {pc[0], pc[1]}, v[2] = {vc[0], vc[1]}, u[2], pn[2], vn[2];
                fetch2(qt, srt, ngt, 1, u[0], u[1]);
                fetch2(qn, srn, ngn, 0, pn[0], pn[1]);
                fetch2(qn, srn, ngn, 2, vn[0], vn[1]);

                // ---- x-slice t: interfaces I0 = (c0-1 | c0) and I1 = (c0 | c1) ----
                const real a1_0 = Z * (u[0] - uM) - (p[0] - pM);
                const real a2_0 = Z * (u[0] - uM) + (p[0] - pM);
                const real a1_1 = Z * (u[1] - u[0]) - (p[1] - p[0]);
                const real a2_1 = Z * (u[1] - u[0]) + (p[1] - p[0]);
                const real a1_R = __shfl_down_sync(FULL, a1_0, 1);  // interface c1+1 (lane+1's I0)
                const real a2_L = __shfl_up_sync(FULL, a2_1, 1);    // interface c0-1 (lane-1's I1)
                // wave 1 (speed -c) looks right, wave 2 (speed +c) looks left
                [[maybe_unused]] real Fp0 = real(0), Su0 = real(0), Fp1 = real(0), Su1 = real(0);
                if constexpr (ORD == 2) {
                    const real l1_0 = limited_strength<real, LIM>(a1_0, a1_1, A.lim);
                    const real l2_0 = limited_strength<real, LIM2>(a2_0, a2_L, A.lim2);
                    const real l1_1 = limited_strength<real, LIM>(a1_1, a1_R, A.lim);
                    const real l2_1 = limited_strength<real, LIM2>(a2_1, a2_0, A.lim2);
                    Fp0 = fxp2 * (l2_0 - l1_0);
                    Su0 = l1_0 + l2_0;
                    Fp1 = fxp2 * (l2_1 - l1_1);
                    Su1 = l1_1 + l2_1;
                }
                [[maybe_unused]] real FpR = real(0), SuR = real(0);
                if constexpr (ORD == 2) {
                    FpR = __shfl_down_sync(FULL, Fp0, 1);
                    SuR = __shfl_down_sync(FULL, Su0, 1);
                }
                // cell c0: interfaces I0 (left) and I1 (right); cell c1: I1 and lane+1's I0.
                // X = the strengths entering the cell (apdq of its left interface,
                // amdq of its right one), D = the difference of its Fp'.
                real q3[2][3];
                {
                    const real X0 = a2_0 + a1_1, X1 = a2_1 + a1_R;
                    [[maybe_unused]] real D0 = real(0), D1 = real(0);
                    if constexpr (ORD == 2) {
                        D0 = Fp1 - Fp0;
                        D1 = FpR - Fp1;
                    }
                    real pt0 = p[0], pt1 = p[1], vt0 = v[0], vt1 = v[1];
                    if constexpr (TRN > 0) {  // row t's share of the split of slice t-1
                        pt0 = fma(-gx, sxp[0], pt0);
                        pt1 = fma(-gx, sxp[1], pt1);
                        vt0 = fma(-dx4, sxp[0], vt0);
                        vt1 = fma(-dx4, sxp[1], vt1);
                    }
                    real n00 = pt0 - qpxh * X0;
                    real n01 = u[0] + quxh * (a1_1 - a2_0);
                    const real n02 = vt0;
                    real n10 = pt1 - qpxh * X1;
                    real n11 = u[1] + quxh * (a1_R - a2_1);
                    const real n12 = vt1;
                    if constexpr (ORD == 2) {
                        n00 = n00 - dtdx2 * D0;
                        n01 = n01 - kux * (Su1 - Su0);
                        n10 = n10 - dtdx2 * D1;
                        n11 = n11 - kux * (SuR - Su1);
                    }
                    if constexpr (TRN > 0) {
                        // pressure part of the cell's amdq(right) + apdq(left), the
                        // fluctuations rpt2 splits (with + cqxx and - cqxx at
                        // transverse 2): cZ/(2Z) X (+ D)
                        const real S0 = TRN == 2 ? fma(cZh, X0, D0) : cZh * X0;
                        const real S1 = TRN == 2 ? fma(cZh, X1, D1) : cZh * X1;
                        // split into rows t-1 (gamma, delta), t (-2 gamma) and t+1 (carried)
                        n00 = fma(gx2, S0, n00);
                        n10 = fma(gx2, S1, n10);
                        q3[0][0] = fma(-gx, S0, q2p[0][0]); q3[0][1] = q2p[0][1]; q3[0][2] = fma(dx4, S0, q2p[0][2]);
                        q3[1][0] = fma(-gx, S1, q2p[1][0]); q3[1][1] = q2p[1][1]; q3[1][2] = fma(dx4, S1, q2p[1][2]);
                        sxp[0] = S0;
                        sxp[1] = S1;
                    } else {
#pragma unroll
                        for (int k = 0; k < 2; ++k)
                            for (int m = 0; m < 3; ++m) q3[k][m] = q2p[k][m];
                    }
                    q2p[0][0] = n00; q2p[0][1] = n01; q2p[0][2] = n02;
                    q2p[1][0] = n10; q2p[1][1] = n11; q2p[1][2] = n12;
                }

                // ---- y: interface t+1 raw, interface t limited, y-part of (c_k, t-1) ----
                real Sy[2], o[2][3], Fpy[2], Svy[2], a1n[2], a2n[2];
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const real dp = pn[k] - p[k], dv = vn[k] - v[k];
                    a1n[k] = Z * dv - dp;
                    a2n[k] = Z * dv + dp;
                    Fpy[k] = real(0);
                    Svy[k] = real(0);
                    if constexpr (ORD == 2) {
                        const real b1 = limited_strength<real, LIM>(a1y[k], a1n[k], A.lim);    // upwind t+1
                        const real b2 = limited_strength<real, LIM2>(a2y[k], a2y_lo[k], A.lim2); // upwind t-1
                        Fpy[k] = fyp2 * (b2 - b1);
                        Svy[k] = b1 + b2;
                    }
                    // cell t-1: amdq of interface t and apdq of interface t-1 enter it
                    const real Y = a2y_lo[k] + a1y[k];
                    [[maybe_unused]] real Dy = real(0);
                    if constexpr (ORD == 2) Dy = Fpy[k] - Fpy_lo[k];
                    o[k][0] = q3[k][0] - qpyh * Y;
                    o[k][1] = q3[k][1];
                    o[k][2] = q3[k][2] + qvyh * (a1y[k] - a2y_lo[k]);
                    if constexpr (ORD == 2) {
                        o[k][0] = o[k][0] - dtdy2 * Dy;
                        o[k][2] = o[k][2] - kvy * (Svy[k] - Svy_lo[k]);
                    }
                    Sy[k] = real(0);
                    if constexpr (TRN > 0) {
                        Sy[k] = TRN == 2 ? fma(cZh, Y, Dy) : cZh * Y;
                        o[k][0] = fma(gy2, Sy[k], o[k][0]);
                    }
                }
                if constexpr (TRN > 0) {
                    // transverse transfers: column c0 from c0-1 (lane-1's c1) and c1;
                    // column c1 from c0 and c1+1 (lane+1's c0): -gamma S into p,
                    // -+delta S into u
                    const real SL = __shfl_up_sync(FULL, Sy[1], 1), SR = __shfl_down_sync(FULL, Sy[0], 1);
                    o[0][0] = fma(-gy, SL + Sy[1], o[0][0]);
                    o[0][1] = fma(dy4, Sy[1] - SL, o[0][1]);
                    o[1][0] = fma(-gy, Sy[0] + SR, o[1][0]);
                    o[1][1] = fma(dy4, SR - Sy[0], o[1][1]);
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
                    Fpy_lo[k] = Fpy[k];
                    Svy_lo[k] = Svy[k];
                    a1y[k] = a1n[k];
                    a2y[k] = a2n[k];
                    pc[k] = pn[k];
                    vc[k] = vn[k];
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
        // interior strip: columns b-3 .. b+61 inside the grid
        const bool interior = b - 3 >= 0 && b + 61 <= mx - 1;
        if (interior) march(std::true_type{});
        else march(std::false_type{});
        seq_base += (uint32_t)nrows;
    }
    // Courant number as flux2 forms it (dt/dx * c over x-interfaces, dt/dy * c
    // over y-interfaces; the speeds are constant)
    const double cfl = any_work ? fmax(dtdx_d * (double)c, dtdy_d * (double)c) : 0.0;
    cta_cfl_and_control(ctl, cfl, red);
}

}  // namespace clawb200
