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
#pragma once
#include "common.cuh"

namespace clawb200 {

constexpr int STRIP = 28;      // output columns per warp
constexpr int RING = 12;       // rows in flight per warp
constexpr int WARPS2D = 4;     // warps per CTA

template <typename real>
struct BoxW { static constexpr int value = 34; };
template <>
struct BoxW<float> { static constexpr int value = 36; };

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
    ClawCtl* ctl;
    S solver;
};

// Map a (possibly ghost) index to its source interior index under the BC of
// that side.  Returns the source index; sets neg when a wall reflects it.
__device__ __forceinline__ int bc_map(int x, int n, int blo, int bhi, bool& neg) {
    neg = false;
    if (x < 0) {
        if (x < -2) x = -2;  // beyond the two ghost layers: only garbage lanes
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

template <class S>
__global__ void __launch_bounds__(32 * WARPS2D)
step2_kernel(const __grid_constant__ Step2Args<S> A) {
    using real = typename S::real;
    constexpr int ME = S::meqn, MW = S::mwaves, MA = S::maux;
    constexpr int MAX = MA > 0 ? MA : 1;
    using R = Ring2D<S>;
    constexpr int W = R::W;

    ClawCtl* ctl = A.ctl;
    __shared__ double red[WARPS2D];
    if (*(volatile int*)&ctl->done) return;
    const int cur = *(volatile int*)&ctl->cur;
    const double dtd = *(volatile double*)&ctl->dt;
    const real dtdx = (real)(dtd / A.dx), dtdy = (real)(dtd / A.dy);
    const double dtdx_d = dtd / A.dx, dtdy_d = dtd / A.dy;
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
    const bool limit = (A.mthlim[0] | A.mthlim[1] | A.mthlim[2] | A.mthlim[3] | A.mthlim[4] |
                        A.mthlim[5] | A.mthlim[6] | A.mthlim[7]) != 0;
    const bool capa = A.capa > 0;
    const int ic = A.capa - 1;
    double cfl = 0.0;
    bool failed = false;
    uint32_t seq_base = 0;

    const long long gw = (long long)blockIdx.x * WARPS2D + warp;
    long long u0 = (gw < A.nwarps) ? gw * A.units / A.nwarps : 0;
    const long long u1 = (gw < A.nwarps) ? (gw + 1) * A.units / A.nwarps : 0;

    while (u0 < u1 && !failed) {
        const int strip = (int)(u0 / my);
        const int r0 = (int)(u0 % my);
        const int nr = (int)min((long long)(my - r0), u1 - u0);
        u0 += nr;
        const int b = strip * STRIP;
        const int c = b - 1 + lane;
        const int x0 = b - 2;  // first column held in the ring
        const int rfirst = r0 - 2, rlast = r0 + nr + 1;  // rows streamed
        const int nrows = rlast - rfirst + 1;

        // Column sources of q(c-1) and q(c) under the x boundary conditions.
        bool negm, negc;
        const int sm = bc_map(c - 1, mx, A.bc[0], A.bc[1], negm);
        const int sc = bc_map(c, mx, A.bc[0], A.bc[1], negc);
        const bool gm = (sm - x0) < 0 || (sm - x0) >= W;
        const bool gc = (sc - x0) < 0 || (sc - x0) >= W;
        const int im = gm ? 0 : sm - x0, icc = gc ? 0 : sc - x0;

        auto slot_of = [&](int r) -> int { return (int)((seq_base + (uint32_t)(r - rfirst)) % RING); };
        auto parity_of = [&](int r) -> uint32_t {
            return ((seq_base + (uint32_t)(r - rfirst)) / RING) & 1u;
        };
        auto issue = [&](int r) {
            const int sl = slot_of(r);
            unsigned char* dst = ring + sl * R::SLOT;
            bool nyneg;
            const int sr = bc_map(r, my, A.bc[2], A.bc[3], nyneg);
            mbar_arrive_expect_tx(&bars[sl], (uint32_t)(R::QB + R::AB));
            tma_load_3d(dst, tmq, x0, sr, 0, &bars[sl]);
            if constexpr (MA > 0) tma_load_3d(dst + R::QBP, &A.tmaux, x0 + 2, r + 2, 0, &bars[sl]);
        };
        if (lane == 0) {
            const int npre = nrows < RING ? nrows : RING;
            for (int k = 0; k < npre; ++k) issue(rfirst + k);
        }
        __syncwarp();

        // Wait for row r and load q(c-1, r), q(c, r).
        auto wait_row = [&](int r) -> bool {
            return mbar_wait_bounded(&bars[slot_of(r)], parity_of(r));
        };
        auto load_q = [&](int r, real* qm, real* qc) {
            const real* sq = reinterpret_cast<const real*>(ring + slot_of(r) * R::SLOT);
            bool nyneg;
            const int sr = bc_map(r, my, A.bc[2], A.bc[3], nyneg);
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                real vm = gm ? qold[m * A.fstride + (long long)sr * A.ld + sm] : sq[m * W + im];
                real vc = gc ? qold[m * A.fstride + (long long)sr * A.ld + sc] : sq[m * W + icc];
                if (m == 1) { if (negm) vm = -vm; if (negc) vc = -vc; }
                if (m == 2 && nyneg) { vm = -vm; vc = -vc; }
                qm[m] = vm;
                qc[m] = vc;
            }
        };
        // aux of column (c + dc) at row r (ring already resident).
        auto aux_at = [&](int r, int dc, real* a) {
            if constexpr (MA > 0) {
                const real* sa = reinterpret_cast<const real*>(ring + slot_of(r) * R::SLOT + R::QBP);
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
#pragma unroll
        for (int m = 0; m < ME; ++m) {
            Ax_prev[m] = q2_prev[m] = qc_p[m] = real(0);
            P1[m] = P3[m] = P4[m] = Fy_prev[m] = real(0);
            amy[m] = apy[m] = real(0);
        }
#pragma unroll
        for (int mw = 0; mw < MW; ++mw) {
            dotl_y[mw] = real(0);
            sy[mw] = real(0);
#pragma unroll
            for (int m = 0; m < ME; ++m) wy[mw][m] = real(0);
        }

        int last_issued = rfirst + (nrows < RING ? nrows : RING) - 1;
        int fail_row = rlast + 1;
        if (!wait_row(rfirst)) { failed = true; fail_row = rfirst; }
        if (!failed) load_q(rfirst, qm_t, qc_t);

        for (int t = rfirst; t <= r0 + nr && !failed; ++t) {
            // ---------------- read row t+1 ----------------
            if (!wait_row(t + 1)) { failed = true; fail_row = t + 1; break; }
            load_q(t + 1, qm_n, qc_n);
            real a_m[MAX], a_c[MAX], a_cn[MAX];  // aux at (c-1,t), (c,t), (c,t+1)
            aux_at(t, -1, a_m);
            aux_at(t, 0, a_c);
            aux_at(t + 1, 0, a_cn);
            // raw y-interface t+1 (rows t, t+1) and its CFL
            real wn[MW][ME], sn[MW], amn[ME], apn[ME];
            A.solver.rpn(2, qc_t, qc_n, a_c, a_cn, wn, sn, amn, apn);
            if (c >= -1 && c <= mx && t + 1 >= 0 && t + 1 <= my) {
                const double dt0 = capa ? dtdy_d / (double)a_c[ic] : dtdy_d;
                const double dt1 = capa ? dtdy_d / (double)a_cn[ic] : dtdy_d;
#pragma unroll
                for (int mw = 0; mw < MW; ++mw)
                    cfl = fmax(fmax(cfl, dt1 * (double)sn[mw]), -dt0 * (double)sn[mw]);
            }

            if (t >= r0 - 1) {
                // rows t-1 .. t+1 are resident from here on
                real a_p[MAX], a_cp[MAX], a_mp[MAX], a_pp[MAX], a_mn[MAX];
                aux_at(t, 1, a_p);        // (c+1, t)
                aux_at(t - 1, 0, a_cp);   // (c,   t-1)
                aux_at(t - 1, -1, a_mp);  // (c-1, t-1)
                aux_at(t - 1, 1, a_pp);   // (c+1, t-1)
                aux_at(t + 1, -1, a_mn);  // (c-1, t+1)

                // ======== x-slice t: interface c (between columns c-1, c) ========
                real q3[ME];
                {
                    real w[MW][ME], s[MW], amdq[ME], apdq[ME];
                    A.solver.rpn(1, qm_t, qc_t, a_m, a_c, w, s, amdq, apdq);
                    const real dtm = capa ? dtdx / a_m[ic] : dtdx;  // dtdx1d(i-1)
                    const real dtc = capa ? dtdx / a_c[ic] : dtdx;  // dtdx1d(i)
                    if (c >= 0 && c <= mx && t >= -1 && t <= my) {
                        const double dm = capa ? dtdx_d / (double)a_m[ic] : dtdx_d;
                        const double dc = capa ? dtdx_d / (double)a_c[ic] : dtdx_d;
#pragma unroll
                        for (int mw = 0; mw < MW; ++mw)
                            cfl = fmax(fmax(cfl, dc * (double)s[mw]), -dm * (double)s[mw]);
                    }
                    real send1[ME], qadd[ME], F[ME], cq[ME];
#pragma unroll
                    for (int m = 0; m < ME; ++m) {
                        send1[m] = dtm * amdq[m];           // qadd of cell c-1 from this interface
                        qadd[m] = real(0) - dtc * apdq[m];  // qadd of cell c, first term
                        F[m] = real(0);
                        cq[m] = real(0);
                    }
                    if (A.order != 1) {
                        if (limit) {
                            real dotr[MW], wn2[MW];
#pragma unroll
                            for (int mw = 0; mw < MW; ++mw) {
                                real dr = real(0), nn = real(0);
#pragma unroll
                                for (int m = 0; m < ME; ++m) {
                                    const real wr = __shfl_down_sync(0xffffffffu, w[mw][m], 1);
                                    nn = nn + w[mw][m] * w[mw][m];
                                    dr = dr + w[mw][m] * wr;
                                }
                                dotr[mw] = dr;
                                wn2[mw] = nn;
                            }
#pragma unroll
                            for (int mw = 0; mw < MW; ++mw) {
                                const real dl = __shfl_up_sync(0xffffffffu, dotr[mw], 1);
                                const int ml = A.mthlim[mw];
                                if (ml != 0 && wn2[mw] != real(0)) {
                                    const real r = (s[mw] > real(0) ? dl : dotr[mw]) / wn2[mw];
                                    const real ph = phi_limiter<real>(ml, r);
#pragma unroll
                                    for (int m = 0; m < ME; ++m) w[mw][m] = ph * w[mw][m];
                                }
                            }
                        }
                        const real ave = real(0.5) * (dtm + dtc);
#pragma unroll
                        for (int mw = 0; mw < MW; ++mw) {
                            const real as = fabs(s[mw]);
                            const real coef = A.fwave ? copysign(real(1), s[mw]) * (real(1) - as * ave)
                                                      : as * (real(1) - as * ave);
#pragma unroll
                            for (int m = 0; m < ME; ++m) cq[m] = cq[m] + coef * w[mw][m];
                        }
#pragma unroll
                        for (int m = 0; m < ME; ++m) F[m] = real(0.5) * cq[m];
                    }
                    real s3[ME], s4[ME], g1b[ME], g2b[ME];
                    if (A.trans > 0) {
                        if (A.order != 1 && A.trans == 2) {
#pragma unroll
                            for (int m = 0; m < ME; ++m) {
                                amdq[m] = amdq[m] + cq[m];
                                apdq[m] = apdq[m] - cq[m];
                            }
                        }
                        real bm[ME], bp[ME];
                        A.solver.rpt(1, 1, qm_t, qc_t, a_mp, a_m, a_mn, amdq, bm, bp);
                        const real hm = real(0.5) * dtm, hc = real(0.5) * dtc;
#pragma unroll
                        for (int m = 0; m < ME; ++m) {
                            s3[m] = -(hm * bm[m]);  // gadd(:,1,i-1) from this interface
                            s4[m] = -(hm * bp[m]);  // gadd(:,2,i-1)
                        }
                        A.solver.rpt(1, 2, qm_t, qc_t, a_cp, a_c, a_cn, apdq, bm, bp);
#pragma unroll
                        for (int m = 0; m < ME; ++m) {
                            g1b[m] = hc * bm[m];
                            g2b[m] = hc * bp[m];
                        }
                    } else {
#pragma unroll
                        for (int m = 0; m < ME; ++m) s3[m] = s4[m] = g1b[m] = g2b[m] = real(0);
                    }
                    // interface c+1 (lane+1) finishes cell c
#pragma unroll
                    for (int m = 0; m < ME; ++m) {
                        const real r1 = __shfl_down_sync(0xffffffffu, send1[m], 1);
                        const real r2 = __shfl_down_sync(0xffffffffu, F[m], 1);
                        const real r3 = __shfl_down_sync(0xffffffffu, s3[m], 1);
                        const real r4 = __shfl_down_sync(0xffffffffu, s4[m], 1);
                        const real qa = qadd[m] - r1;
                        const real G1 = r3 - g1b[m];
                        const real G2 = r4 - g2b[m];
                        const real dF = r2 - F[m];
                        real q2, Ax, Bx;
                        if (!capa) {
                            q2 = (((qc_t[m] + Ax_prev[m]) + qa) - dtdx * dF) - dtdy * (G2 - G1);
                            Ax = dtdy * G2;
                            Bx = dtdy * G1;
                        } else {
                            q2 = ((qc_t[m] + Ax_prev[m]) + qa) -
                                 (dtdx * dF + dtdy * (G2 - G1)) / a_c[ic];
                            Ax = dtdy * G2 / a_cn[ic];
                            Bx = dtdy * G1 / a_cp[ic];
                        }
                        q3[m] = q2_prev[m] - Bx;  // x-part of cell (c, t-1) complete
                        q2_prev[m] = q2;
                        Ax_prev[m] = Ax;
                    }
                }

                // ======== y-interface t (rows t-1, t) limited; y-part of cell (c, t-1) ========
                const real dty_p = capa ? dtdy / a_cp[ic] : dtdy;  // dtdy1d(t-1)
                const real dty_t = capa ? dtdy / a_c[ic] : dtdy;   // dtdy1d(t)
                real cqy[ME], Fy[ME], dotr_y[MW];
#pragma unroll
                for (int m = 0; m < ME; ++m) { cqy[m] = real(0); Fy[m] = real(0); }
#pragma unroll
                for (int mw = 0; mw < MW; ++mw) {
                    real dr = real(0);
#pragma unroll
                    for (int m = 0; m < ME; ++m) dr = dr + wy[mw][m] * wn[mw][m];
                    dotr_y[mw] = dr;
                }
                if (A.order != 1) {
                    if (limit) {
#pragma unroll
                        for (int mw = 0; mw < MW; ++mw) {
                            real nn = real(0);
#pragma unroll
                            for (int m = 0; m < ME; ++m) nn = nn + wy[mw][m] * wy[mw][m];
                            const int ml = A.mthlim[mw];
                            if (ml != 0 && nn != real(0)) {
                                const real r = (sy[mw] > real(0) ? dotl_y[mw] : dotr_y[mw]) / nn;
                                const real ph = phi_limiter<real>(ml, r);
#pragma unroll
                                for (int m = 0; m < ME; ++m) wy[mw][m] = ph * wy[mw][m];
                            }
                        }
                    }
                    const real ave = real(0.5) * (dty_p + dty_t);
#pragma unroll
                    for (int mw = 0; mw < MW; ++mw) {
                        const real as = fabs(sy[mw]);
                        const real coef = A.fwave ? copysign(real(1), sy[mw]) * (real(1) - as * ave)
                                                  : as * (real(1) - as * ave);
#pragma unroll
                        for (int m = 0; m < ME; ++m) cqy[m] = cqy[m] + coef * wy[mw][m];
                    }
#pragma unroll
                    for (int m = 0; m < ME; ++m) Fy[m] = real(0.5) * cqy[m];
                }
                real amo[ME], apo[ME];
#pragma unroll
                for (int m = 0; m < ME; ++m) { amo[m] = amy[m]; apo[m] = apy[m]; }
                real bma[ME], bpa[ME], bmb[ME], bpb[ME];
                if (A.trans > 0) {
                    if (A.order != 1 && A.trans == 2) {
#pragma unroll
                        for (int m = 0; m < ME; ++m) {
                            amy[m] = amy[m] + cqy[m];
                            apy[m] = apy[m] - cqy[m];
                        }
                    }
                    A.solver.rpt(2, 1, qc_p, qc_t, a_mp, a_cp, a_pp, amy, bma, bpa);
                    A.solver.rpt(2, 2, qc_p, qc_t, a_m, a_c, a_p, apy, bmb, bpb);
                } else {
#pragma unroll
                    for (int m = 0; m < ME; ++m) bma[m] = bpa[m] = bmb[m] = bpb[m] = real(0);
                }
                const real hp = real(0.5) * dty_p, ht = real(0.5) * dty_t;
                const bool out = (t - 1 >= r0) && (lane >= 1) && (lane <= STRIP) && (c < mx);
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    const real qa = P1[m] - dty_p * amo[m];
                    const real G1 = -(hp * bma[m]) - P3[m];
                    const real G2 = -(hp * bpa[m]) - P4[m];
                    const real dF = Fy[m] - Fy_prev[m];
                    real Ay, By, q5pre;
                    if (!capa) {
                        Ay = dtdx * G2;
                        By = dtdx * G1;
                    } else {
                        Ay = dtdx * G2 / a_pp[ic];
                        By = dtdx * G1 / a_mp[ic];
                    }
                    const real Al = __shfl_up_sync(0xffffffffu, Ay, 1);    // from column c-1
                    const real Br = __shfl_down_sync(0xffffffffu, By, 1);  // from column c+1
                    const real q4 = q3[m] + Al;
                    if (!capa) q5pre = q4 + ((qa - dtdy * dF) - dtdx * (G2 - G1));
                    else q5pre = (q4 + qa) - (dtdy * dF + dtdx * (G2 - G1)) / a_cp[ic];
                    const real q6 = q5pre - Br;
                    if (out) qnew[m * A.fstride + (long long)(t - 1) * A.ld + c] = q6;
                }
                // contributions of y-interface t to cell (c, t)
#pragma unroll
                for (int m = 0; m < ME; ++m) {
                    P1[m] = real(0) - dty_t * apo[m];
                    P3[m] = ht * bmb[m];
                    P4[m] = ht * bpb[m];
                    Fy_prev[m] = Fy[m];
                }
#pragma unroll
                for (int mw = 0; mw < MW; ++mw) dotl_y[mw] = dotr_y[mw];
            }
            // roll the y-interface window and the rows: t-1 <- t, t <- t+1
#pragma unroll
            for (int m = 0; m < ME; ++m) {
                amy[m] = amn[m];
                apy[m] = apn[m];
                qc_p[m] = qc_t[m];
                qm_t[m] = qm_n[m];
                qc_t[m] = qc_n[m];
            }
#pragma unroll
            for (int mw = 0; mw < MW; ++mw) {
                sy[mw] = sn[mw];
#pragma unroll
                for (int m = 0; m < ME; ++m) wy[mw][m] = wn[mw][m];
            }
            // release row t-1 and prefetch row t-1+RING into its slot
            __syncwarp();
            if (t - 1 >= rfirst && t - 1 + RING <= rlast) {
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

    cta_cfl_and_control(ctl, cfl, red);
}

}  // namespace clawb200
