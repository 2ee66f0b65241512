// 3D unsplit step, contracted FP64 and FP32 builds (src/3d/step3.f90 with
// src/3d/flux3.f90, transverse codes of flux3.f90:189-197), for sm_100a.
//
// The tiling, the march and the per-value arithmetic are those of the
// reference-order kernel in step3d.cuh, with three changes that the exact
// build cannot take:
//   * the pair of threads that shares a slice is the same lane of two
//     neighbouring warps, so each warp's role h is a compile-time constant and
//     every shared-memory index folds to an immediate offset; the four
//     combinations each role needs from the other's splits
//     (flux3.f90:363-376 and :488-495) cross through shared memory under a
//     64-thread named barrier of the warp pair, the centre terms with the
//     CTA barrier of the position;
//   * the aux ring holds the face reciprocals 1 / (Z + Z_next) along the
//     tile's two axes, so the 16 transverse splits of a slice position
//     multiply instead of dividing (rounding differs from the divisions);
//   * Z, c and the next position's q values are copied by cp.async issued at
//     the top of a position and awaited just before its CTA barrier, so their
//     latency overlaps the position's arithmetic, and the reciprocals of a
//     ring position are formed from the landed Z one position later;
//   * a cell adds its nine neighbour terms in a fixed order instead of
//     step3's 2x2-block colour order.
// The Courant number is the same FP64 product as the exact build's, so the
// dt sequence is identical.
#pragma once
#include "step3d.cuh"

namespace clawb200 {

constexpr int XCH3 = 10;  // exchange planes of NT3 values: L [h][2], R [h][2], centre [h]
constexpr int NPL3F = 4;  // aux planes: Z, c, 1/(Z+Z_e1), 1/(Z+Z_e2)

// Shared memory is sized to the carveout steps (100, 132, 164, 196, 228 KB):
// what the carveout leaves is L1, which serves the x-sweep's strided loads.
// buffers of neighbour terms: two (by position parity) in FP32 (106 KB, the
// 132 KB step); one in FP64, with a second CTA barrier per position (149 KB,
// the 164 KB step, instead of the 228 KB step)
template <typename real>
__host__ __device__ constexpr int term3_bufs() {
    return sizeof(real) == 4 ? 2 : 1;
}

constexpr int VST3 = 8;  // staged values of the cells each role updates: [position & 1][role][2]

template <typename real>
__host__ __device__ constexpr int sweep3f_smem_bytes() {
    return (RING3 * NPL3F * NS3 + term3_bufs<real>() * NTERM3 * NT3 +
            (XCH3 + QST3 + VST3) * NT3) *
               (int)sizeof(real) +
           16 * (int)sizeof(double);
}

__device__ __forceinline__ void pair_sync(int id) {
    asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory");
}

// The march of one tile of slices for the threads of role H; returns the
// thread's Courant number.
template <class S, int DIR, class M, int H>
__device__ __forceinline__ double sweep3f_march(const Sweep3Args<typename S::real>& a,
                                               unsigned char* smem_raw) {
    using real = typename S::real;
    using Split = typename S::Split;
    constexpr int AXN = DIR, AXA = DIR == 0 ? 1 : 0, AXB = DIR == 2 ? 1 : 2;
    constexpr bool E1A = DIR != 1;
    constexpr int CN = 1 + AXN, CE1 = 1 + (E1A ? AXA : AXB), CE2 = 1 + (E1A ? AXB : AXA);
    constexpr int NPL = NPL3F;
    constexpr int NTB = term3_bufs<real>();
    // shared-memory steps of this role's own split direction and the other
    constexpr int E1S = E1A ? 1 : S3A, E2S = E1A ? S3A : 1;
    constexpr int OWNS = H ? E2S : E1S, OTHS = H ? E1S : E2S;
    constexpr int CA = H ? CE1 : 0, CB = H ? CE2 : CN;  // components this role updates

    real* saux = reinterpret_cast<real*>(smem_raw);  // [RING3][NPL][NS3]
    real* sterm = saux + RING3 * NPL * NS3;          // [NTB][NTERM3][NT3]
    real* sxch = sterm + NTB * NTERM3 * NT3;         // [XCH3][NT3]
    real* sq = sxch + XCH3 * NT3;                    // [QST3][NT3]
    real* sv = sq + QST3 * NT3;                      // [VST3][NT3]

    ClawCtl* ctl = a.ctl;
    const int cur = ctl->cur;
    const real* __restrict__ qold = a.q[cur];
    real* __restrict__ qnew = a.q[cur ^ 1];
    const real* __restrict__ aux = a.aux;
    const double dt = ctl->dt;
    const double tbc = ctl->told;
    const double tn_d = dt / a.d[AXN];
    const real tn = (real)tn_d;
    const real te1 = (real)(dt / a.d[E1A ? AXA : AXB]);
    const real te2 = (real)(dt / a.d[E1A ? AXB : AXA]);
    const real H5 = real(0.5) * tn;
    const real S6g = (real(1.0) / real(6.0)) * tn * te2;
    const real S6h = (real(1.0) / real(6.0)) * tn * te1;
    const real dtdxave = real(0.5) * (tn + tn);
    const real t_own = H ? te2 : te1;
    const real S6own = H ? S6h : S6g;

    const int m3 = M::m3 >= 0 ? M::m3 : a.m3;
    const int m4 = M::m4 >= 0 ? M::m4 : a.m4;
    const int order = M::m3 >= 0 ? 2 : a.order;

    const int mN = a.m[AXN], mA = a.m[AXA], mB = a.m[AXB];
    const int bid = blockIdx.x;
    const int seg = bid % a.nseg, tile = bid / a.nseg;
    const int A0 = 1 + (tile % a.tilesA) * (T3A - 2);
    const int B0 = 1 + (tile / a.tilesA) * (T3B - 2);
    const int p0 = 1 + seg * SEG3;
    const int p1 = min(p0 + SEG3, mN + 1);
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int sl = (warp >> 1) * 32 + (tid & 31);  // slice within the tile
    const int pair_id = 1 + (warp >> 1);           // named barrier of the warp pair
    const int ta = sl % T3A, tb = sl / T3A;
    const int A = A0 - 1 + ta, B = B0 - 1 + tb;
    const bool active = A <= mA + 1 && B <= mB + 1;
    const bool apply = active && ta >= 1 && ta <= T3A - 2 && tb >= 1 && tb <= T3B - 2 &&
                       A <= mA && B <= mB;

    bool flipA, flipB;
    const int Am = bc3_src(min(max(A, -1), mA + 2), mA, a.bc[2 * AXA], a.bc[2 * AXA + 1], flipA);
    const int Bm = bc3_src(min(max(B, -1), mB + 2), mB, a.bc[2 * AXB], a.bc[2 * AXB + 1], flipB);
    const long long qoffAB = (long long)(Am - 1) * a.qs[AXA] + (long long)(Bm - 1) * a.qs[AXB];
    const bool pistonB = AXB == 2 && B > mB && a.bc[5] == BC_PISTON;

    auto load_pn = [&](int pos, real& qp, real& qn) {
        bool fN;
        const int pm = bc3_src(pos, mN, a.bc[2 * AXN], a.bc[2 * AXN + 1], fN);
        const long long off = qoffAB + (long long)(pm - 1) * a.qs[AXN];
        qp = qold[off];
        qn = qold[off + CN * a.fstride];
        if (fN) qn = -qn;
        if (CN == 3) {
            const bool pist = (AXN == 2 && pos > mN && a.bc[5] == BC_PISTON) || pistonB;
            if (pist) {
                const int ci = AXN == 0 ? pos : A;
                const int cj = AXN == 1 ? pos : (AXA == 1 ? A : B);
                qn = (real)(2.0 * piston_speed(a, ci, cj, tbc)) - qn;
            }
        }
    };
    // Z and c of ring position pos, copied asynchronously
    auto load_aux = [&](int pos) {
        real* dst = saux + (pos & (RING3 - 1)) * NPL * NS3;
        const long long pofs = (long long)(pos + 1) * a.as[AXN];
        for (int e = tid; e < NS3; e += NT3P) {
            const int sa = e % S3A, sb = e / S3A;
            const int Ai = min(A0 - 2 + sa, mA + 2), Bi = min(B0 - 2 + sb, mB + 2);
            const long long o = pofs + (long long)(Ai + 1) * a.as[AXA] + (long long)(Bi + 1) * a.as[AXB];
            cp_async_el(dst + e, aux + o);
            cp_async_el(dst + NS3 + e, aux + o + a.afstride);
        }
    };
    // 1 / (Z + Z_next) along A and B of ring position pos, from its landed Z.
    // The next tile element is the next cell, or the same clamped cell past
    // the grid's last ghost; the tile's last row and column are never read.
    auto make_rcp = [&](int pos) {
        real* dst = saux + (pos & (RING3 - 1)) * NPL * NS3;
        for (int e = tid; e < NS3; e += NT3P) {
            const int sa = e % S3A, sb = e / S3A;
            if (sa == S3A - 1 || sb == S3B - 1) continue;
            const real z = dst[e];
            const real rA = real(1) / (z + dst[e + 1]);
            const real rB = real(1) / (z + dst[e + S3A]);
            dst[(E1A ? 2 : 3) * NS3 + e] = rA;
            dst[(E1A ? 3 : 2) * NS3 + e] = rB;
        }
    };
    // q of this slice at position pos: role 0 stages p, role 1 the normal
    // velocity; boundary conditions are applied when the pair takes them
    auto issue_q = [&](int pos) {
        if (!active) return;
        bool fN;
        const int pm = bc3_src(pos, mN, a.bc[2 * AXN], a.bc[2 * AXN + 1], fN);
        const long long off = qoffAB + (long long)(pm - 1) * a.qs[AXN] + (H ? CN * a.fstride : 0);
        cp_async_el(sq + ((pos & 1) * 2 + H) * NT3 + sl, qold + off);
    };
    auto take_q = [&](int pos, real& qp, real& qn) {
        qp = sq[((pos & 1) * 2) * NT3 + sl];
        qn = sq[((pos & 1) * 2 + 1) * NT3 + sl];
        bool fN;
        (void)bc3_src(pos, mN, a.bc[2 * AXN], a.bc[2 * AXN + 1], fN);
        if (fN) qn = -qn;
        if (CN == 3) {
            const bool pist = (AXN == 2 && pos > mN && a.bc[5] == BC_PISTON) || pistonB;
            if (pist) {
                const int ci = AXN == 0 ? pos : A;
                const int cj = AXN == 1 ? pos : (AXA == 1 ? A : B);
                qn = (real)(2.0 * piston_speed(a, ci, cj, tbc)) - qn;
            }
        }
    };
    const int sown = (tb + 1) * S3A + (ta + 1);
    auto plane = [&](int pos, int k) -> const real* {
        return saux + (pos & (RING3 - 1)) * NPL * NS3 + k * NS3 + sown;
    };
    // split in the own direction of a fluctuation at the cell `w` across
    auto split_own = [&](real xp, int pos, int w) -> Split {
        const real* Zp = plane(pos, 0);
        const real* Cp = plane(pos, 1);
        const real* Rp = plane(pos, 2 + H);  // 1 / (Z + Z_next) along the own direction
        return S::split_r(xp, Rp[-OWNS + w * OTHS], Zp[-OWNS + w * OTHS], Cp[-OWNS + w * OTHS],
                          Rp[w * OTHS], Zp[OWNS + w * OTHS], Cp[OWNS + w * OTHS]);
    };

    double cfl = 0.0;
    auto solve = [&](int i, real pL, real uL, real pR, real uR, real w[2][2], real am[2], real ap[2]) {
        real s[2];
        const real zl = *plane(i - 1, 0), cl = *plane(i - 1, 1);
        const real zr = *plane(i, 0), cr = *plane(i, 1);
        S::rpn_r(pL, uL, pR, uR, zl, cl, zr, cr, w, s, am, ap);
        if (i >= 1 && i <= mN + 1) {
            for (int k = 0; k < 2; ++k) {  // Courant number in FP64 (FP32 builds too)
                const double c = tn_d * (double)s[k];
                cfl = fmax(fmax(cfl, c), -c);
            }
        }
    };

    load_aux(p0 - 2);
    load_aux(p0 - 1);
    load_aux(p0);
    load_aux(p0 + 1);
    issue_q(p0 + 1);
    cp_async_wait_all();
    __syncthreads();
    make_rcp(p0 - 1);
    make_rcp(p0);
    __syncthreads();

    real wA[2][2], wB[2][2];
    real amB[2], apB[2];
    real qLp = 0, qLn = 0;
    real F0[2] = {0, 0};
    real Qs[2] = {0, 0};
    real O[2][3][2];  // own side's gadd or hadd (side, level, comp) of cell p
    for (int s_ = 0; s_ < 2; ++s_)
        for (int l = 0; l < 3; ++l)
            for (int c = 0; c < 2; ++c) O[s_][l][c] = 0;
    if (active) {
        real q0p, q0n, q1p, q1n;
        load_pn(p0 - 2, q0p, q0n);
        load_pn(p0 - 1, q1p, q1n);
        load_pn(p0, qLp, qLn);
        real am_[2], ap_[2];
        solve(p0 - 1, q0p, q0n, q1p, q1n, wA, am_, ap_);
        solve(p0, q1p, q1n, qLp, qLn, wB, amB, apB);
    }
    __syncthreads();

    const bool xch = m3 > 0 && m4 > 0;  // the pair exchanges split combinations
    // exchange planes: [side L/R][role][value] of NT3 slices each
    auto xplane = [&](int side, int role, int v) -> real* {
        return sxch + ((side * 2 + role) * 2 + v) * NT3 + sl;
    };

    for (int p = p0 - 1; p < p1; ++p) {
        const bool emit = p >= p0;
        // position p+3: its ring slot and staged q were last read before the
        // previous position's barrier
        if (p + 3 <= p1 + 1) {
            load_aux(p + 3);
            issue_q(p + 3);
        }
        // the reciprocals of position p+2 (its Z landed before the last barrier)
        if (p + 2 <= p1 + 1) make_rcp(p + 2);
        const real* vsrc = DIR == 0 ? qold : qnew;
        real vA = 0, vB = 0;
        // the cell values of position p+1, staged for the next position (only
        // this thread writes that cell, at that position)
        if (apply && p + 1 >= p0 && p + 1 < p1) {
            const long long off = qoffAB + (long long)p * a.qs[AXN];
            real* dv = sv + (((p + 1) & 1) * 2 + H) * 2 * NT3 + sl;
            cp_async_el(dv, vsrc + off + CA * a.fstride);
            cp_async_el(dv + NT3, vsrc + off + CB * a.fstride);
        }
        real F1[2] = {0, 0};
        real Qp[2] = {0, 0};
        real wC[2][2] = {}, amC[2] = {}, apC[2] = {}, qRp = 0, qRn = 0;
        real cterm = 0, own_c = 0;  // centre terms: sent to the partner / kept
        real cq[2] = {0, 0};
        Split qm = {0, 0, 0, 0};
        const int L = p, R = p + 1;
        if (active) {
            take_q(p + 2, qRp, qRn);
            solve(p + 2, qLp, qLn, qRp, qRn, wC, amC, apC);
            real wl[2][2];
            const real sB[2] = {-*plane(p, 1), *plane(p + 1, 1)};
            for (int k = 0; k < 2; ++k) {
                wl[k][0] = wB[k][0];
                wl[k][1] = wB[k][1];
                const int lim = M::lim >= 0 ? M::lim : a.mthlim[k];
                if (order == 2 && lim > 0) {
                    const real wn2 = wB[k][0] * wB[k][0] + wB[k][1] * wB[k][1];
                    if (wn2 != real(0)) {
                        const real dl = wA[k][0] * wB[k][0] + wA[k][1] * wB[k][1];
                        const real dr = wB[k][0] * wC[k][0] + wB[k][1] * wC[k][1];
                        const real r = (sB[k] > real(0) ? dl : dr) / wn2;
                        const real phi = phi_limiter<real>(lim, r);
                        wl[k][0] = phi * wB[k][0];
                        wl[k][1] = phi * wB[k][1];
                    }
                }
            }
            if (order == 2) {
                for (int k = 0; k < 2; ++k) {
                    const real as_ = fabs(sB[k]);
                    const real coef = (real(0.5) * as_) * (real(1) - as_ * dtdxave);
                    cq[0] = cq[0] + coef * wl[k][0];
                    cq[1] = cq[1] + coef * wl[k][1];
                }
            }
            F1[0] = cq[0];
            F1[1] = cq[1];
            Qp[0] = Qs[0] - tn * amB[0];
            Qp[1] = Qs[1] - tn * amB[1];
            Qs[0] = real(0) - tn * apB[0];
            Qs[1] = real(0) - tn * apB[1];

            // ---- cell p: the amdq side of interface p+1 completes gadd/hadd
            if (m3 > 0) {
                const Split ma = split_own(amB[0], L, 0);
                if (m3 == 2) qm = split_own(cq[0], L, 0);
                O[0][1][0] = O[0][1][0] - H5 * ma.dp;
                O[0][1][1] = O[0][1][1] - H5 * ma.dt;
                O[1][1][0] = O[1][1][0] - H5 * ma.up;
                O[1][1][1] = O[1][1][1] - H5 * ma.ut;
                if (m4 > 0) {
                    // the combinations the partner splits (flux3.f90:363-376, 488-495)
                    real x1 = ma.up, x3 = ma.dp;
                    if (m4 == 2) {
                        x1 = ma.up + real(3) * qm.up;
                        x3 = ma.dp + real(3) * qm.dp;
                    }
                    *xplane(0, H, 0) = x1;
                    *xplane(0, H, 1) = x3;
                }
            }
        }
        if (xch) {
            pair_sync(pair_id);
            if (active) {
                const real y1 = *xplane(0, 1 - H, 0), y3 = *xplane(0, 1 - H, 1);
                const Split tpm = split_own(y1, L, 1), tmm = split_own(y3, L, -1);
                O[1][1][0] = O[1][1][0] + S6own * (tpm.up - tmm.up);
                O[1][1][1] = O[1][1][1] + S6own * (tpm.ut - tmm.ut);
                O[0][1][0] = O[0][1][0] + S6own * (tpm.dp - tmm.dp);
                O[0][1][1] = O[0][1][1] + S6own * (tpm.dt - tmm.dt);
                O[1][2][0] = O[1][2][0] - S6own * tpm.up;
                O[1][2][1] = O[1][2][1] - S6own * tpm.ut;
                O[0][2][0] = O[0][2][0] - S6own * tpm.dp;
                O[0][2][1] = O[0][2][1] - S6own * tpm.dt;
                O[1][0][0] = O[1][0][0] + S6own * tmm.up;
                O[1][0][1] = O[1][0][1] + S6own * tmm.ut;
                O[0][0][0] = O[0][0][0] + S6own * tmm.dp;
                O[0][0][1] = O[0][0][1] + S6own * tmm.dt;
            }
        }
        Split qp = {0, 0, 0, 0};
        if (active) {
            if (m3 == 2) {
                O[1][1][0] = O[1][1][0] - tn * qm.up;
                O[1][1][1] = O[1][1][1] - tn * qm.ut;
                O[0][1][0] = O[0][1][0] - tn * qm.dp;
                O[0][1][1] = O[0][1][1] - tn * qm.dt;
            }
            if (emit) {
                // terms for the eight neighbours: own offset o (the side), other w (the level)
                real* out = sterm + (NTB == 2 ? (p & 1) : 0) * NTERM3 * NT3 + sl;
#pragma unroll
                for (int w = -1; w <= 1; ++w)
#pragma unroll
                    for (int o = -1; o <= 1; ++o) {
                        if (o == 0 && w == 0) continue;
                        const int de1 = H ? w : o, de2 = H ? o : w;
                        const int idx9 = (de2 + 1) * 3 + (de1 + 1);
                        const int nb = idx9 < 4 ? idx9 : idx9 - 1;
#pragma unroll
                        for (int c = 0; c < 2; ++c) {
                            const real tv = o < 0 ? -(t_own * O[0][w + 1][c])
                                          : o == 0 ? -(t_own * (O[1][w + 1][c] - O[0][w + 1][c]))
                                                   : t_own * O[1][w + 1][c];
                            out[(nb * 4 + 2 * H + c) * NT3] = tv;
                        }
                    }
                // centre: h = 0 keeps te1*dG_p and sends te1*dG_e1; h = 1
                // keeps te2*dH_e2 and sends te2*dH_p
                const real dp_ = t_own * (O[1][1][0] - O[0][1][0]);
                const real dv_ = t_own * (O[1][1][1] - O[0][1][1]);
                cterm = H ? dp_ : dv_;
                own_c = H ? dv_ : dp_;
            }
            // ---- cell p+1: the apdq side of interface p+1 starts gadd/hadd
            for (int s_ = 0; s_ < 2; ++s_)
                for (int l = 0; l < 3; ++l)
                    for (int c = 0; c < 2; ++c) O[s_][l][c] = 0;
            if (m3 > 0) {
                const Split mp = split_own(apB[0], R, 0);
                if (m3 == 2) qp = split_own(cq[0], R, 0);
                O[0][1][0] = O[0][1][0] - H5 * mp.dp;
                O[0][1][1] = O[0][1][1] - H5 * mp.dt;
                O[1][1][0] = O[1][1][0] - H5 * mp.up;
                O[1][1][1] = O[1][1][1] - H5 * mp.ut;
                if (m4 > 0) {
                    real x0 = mp.up, x2 = mp.dp;
                    if (m4 == 2) {
                        x0 = mp.up - real(3) * qp.up;
                        x2 = mp.dp - real(3) * qp.dp;
                    }
                    *xplane(1, H, 0) = x0;
                    *xplane(1, H, 1) = x2;
                }
            }
        }
        if (xch) {
            pair_sync(pair_id);
            if (active) {
                const real y0 = *xplane(1, 1 - H, 0), y2 = *xplane(1, 1 - H, 1);
                const Split tpp = split_own(y0, R, 1), tmp = split_own(y2, R, -1);
                O[1][1][0] = O[1][1][0] + S6own * (tpp.up - tmp.up);
                O[1][1][1] = O[1][1][1] + S6own * (tpp.ut - tmp.ut);
                O[0][1][0] = O[0][1][0] + S6own * (tpp.dp - tmp.dp);
                O[0][1][1] = O[0][1][1] + S6own * (tpp.dt - tmp.dt);
                O[1][2][0] = O[1][2][0] - S6own * tpp.up;
                O[1][2][1] = O[1][2][1] - S6own * tpp.ut;
                O[0][2][0] = O[0][2][0] - S6own * tpp.dp;
                O[0][2][1] = O[0][2][1] - S6own * tpp.dt;
                O[1][0][0] = O[1][0][0] + S6own * tmp.up;
                O[1][0][1] = O[1][0][1] + S6own * tmp.ut;
                O[0][0][0] = O[0][0][0] + S6own * tmp.dp;
                O[0][0][1] = O[0][0][1] + S6own * tmp.dt;
            }
        }
        if (active && m3 == 2) {
            O[1][1][0] = O[1][1][0] + tn * qp.up;
            O[1][1][1] = O[1][1][1] + tn * qp.ut;
            O[0][1][0] = O[0][1][0] + tn * qp.dp;
            O[0][1][1] = O[0][1][1] + tn * qp.dt;
        }
        // centre term for the partner, double-buffered by the position's parity
        // centre term for the partner.  Its last value was read in the
        // partner's previous gather, which precedes the partner's arrival at
        // this position's pair barriers (one is added where the method has
        // no split exchange).
        if (!xch) pair_sync(pair_id);
        sxch[(8 + H) * NT3 + sl] = cterm;
        cp_async_wait_all();
        __syncthreads();
        if (emit && apply) {
            const real crecv = sxch[(8 + 1 - H) * NT3 + sl];
            {
                const real* vv = sv + ((p & 1) * 2 + H) * 2 * NT3 + sl;
                vA = vv[0];
                vB = vv[NT3];
            }
            const real* in = sterm + (NTB == 2 ? (p & 1) : 0) * NTERM3 * NT3 + sl;
            auto add_term = [&](int code) {
                if (code == 4) {
                    if (H == 0) {
                        vA = vA + Qp[0] - tn * (F1[0] - F0[0]) - own_c - crecv;
                        vB = vB + Qp[1] - tn * (F1[1] - F0[1]);
                    } else {
                        vA = vA - crecv;
                        vB = vB - own_c;
                    }
                } else {
                    const int da = code % 3 - 1, db = code / 3 - 1;
                    const int u = E1A ? -da : -db, w = E1A ? -db : -da;
                    const int idx9 = (w + 1) * 3 + (u + 1);
                    const int nb = idx9 < 4 ? idx9 : idx9 - 1;
                    const int so = db * T3A + da;
                    if (H == 0) {
                        vA = vA + in[(nb * 4 + 0) * NT3 + so] + in[(nb * 4 + 2) * NT3 + so];
                    } else {
                        vA = vA + in[(nb * 4 + 1) * NT3 + so];
                        vB = vB + in[(nb * 4 + 3) * NT3 + so];
                    }
                }
            };
#pragma unroll
            for (int k = 0; k < 9; ++k) add_term(k);
            const long long off = qoffAB + (long long)(p - 1) * a.qs[AXN];
            qnew[off + CA * a.fstride] = vA;
            qnew[off + CB * a.fstride] = vB;
        }
        if (active) {
            for (int k = 0; k < 2; ++k)
                for (int c = 0; c < 2; ++c) { wA[k][c] = wB[k][c]; wB[k][c] = wC[k][c]; }
            amB[0] = amC[0]; amB[1] = amC[1];
            apB[0] = apC[0]; apB[1] = apC[1];
            qLp = qRp; qLn = qRn;
            F0[0] = F1[0]; F0[1] = F1[1];
        }
        // one term buffer: every gather of p ends before a publish of p+1
        if constexpr (NTB == 1) __syncthreads();
    }
    return cfl;
}

template <class S, int DIR, class M, bool LAST>
__global__ void __launch_bounds__(NT3P, CLAW_SWEEP3_MINB) sweep3f_kernel(const Sweep3Args<typename S::real> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using real = typename S::real;
    double* red = reinterpret_cast<double*>(reinterpret_cast<real*>(smem_raw) +
                                            RING3 * NPL3F * NS3 + term3_bufs<real>() * NTERM3 * NT3 +
                                            (XCH3 + QST3 + VST3) * NT3);
    ClawCtl* ctl = a.ctl;
    grid_dependency_sync();
    if (ctl->done) return;
    // warps 2k (role 0) and 2k+1 (role 1) share 32 slices
    const double cfl = ((threadIdx.x >> 5) & 1) ? sweep3f_march<S, DIR, M, 1>(a, smem_raw)
                                                : sweep3f_march<S, DIR, M, 0>(a, smem_raw);
    if (LAST) {
        cta_cfl_and_control(ctl, cfl, red);
    } else {
        double c = cfl;
        for (int off = 16; off > 0; off >>= 1) c = fmax(c, __shfl_xor_sync(0xffffffffu, c, off));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = 0.0;
            for (int w = 0; w < NT3P / 32; ++w) m = fmax(m, red[w]);
            if (!(m > 0.0)) m = (m != m) ? m : 0.0;
            atomicMax(&ctl->cfl_bits, (unsigned long long)__double_as_longlong(m));
        }
    }
}

}  // namespace clawb200
