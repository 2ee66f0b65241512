// 3D unsplit wave-propagation step (src/3d/step3.f90:3-873 with
// src/3d/flux3.f90:4-612) for sm_100a.
//
// One kernel per sweep direction.  A CTA owns a T3A x T3B tile of slices of
// that sweep (the outer ring of the tile is a one-slice halo) and marches the
// tile along the slice direction, one cell position per iteration; each thread
// carries one slice's Riemann state (normal solve at interface p+2, limiter
// and second-order correction at p+1, the transverse and double-transverse
// splits of p+1, and the gadd/hadd partial sums of cells p and p+1).
//
// A cell receives contributions from the nine slices around it.  step3 adds
// them in the order of its 2x2-block colouring (colour of the slow slice
// index, colour of the fast one, then slow, then fast index), which fixes the
// rounding of every cell.  Here each slice publishes the terms it adds to its
// eight neighbours in shared memory and every cell adds its nine terms in
// that same order, so the x-, y- and z-sweeps reproduce the serial loop nest
// bit for bit; the three sweeps run as three launches in step3's order.
//
// q is stored for interior cells only; ghost values come from the boundary
// conditions of bc3 (x pass, then y, then z, so corners compose the maps).
#pragma once
#include "common.cuh"
#include "riemann.cuh"

namespace clawb200 {

#ifndef CLAW_T3B
#define CLAW_T3B 16
#endif
#ifndef CLAW_SWEEP3_MINB
#define CLAW_SWEEP3_MINB 1  // resident CTAs per SM the sweep kernels are compiled for
#endif
constexpr int T3A = 16, T3B = CLAW_T3B, NT3 = T3A * T3B;   // thread tile, incl. the halo ring
constexpr int S3A = T3A + 2, S3B = T3B + 2, NS3 = S3A * S3B;  // aux tile, one more ring
constexpr int SEG3 = 64;                              // cell positions per CTA march
constexpr int RING3 = 4;                              // aux positions held in shared memory
constexpr int NTERM3 = 32;                            // published terms per slice and position
constexpr int BC_PISTON = 10;                         // user BC of acoustics_3d_heterogeneous

template <typename real>
struct Sweep3Args {
    real* q[2];
    const real* aux;
    long long qs[3];     // q strides in elements along x, y, z (1, ld, ld*my)
    long long fstride;   // q field pitch
    long long as[3];     // aux strides (1, ald, ald*(my+4))
    long long afstride;  // aux field pitch
    int m[3];            // mx, my, mz
    int bc[6];           // [2*axis + side]: mthbc
    int mthlim[2];
    int order, m3, m4;
    double d[3];         // dx, dy, dz
    double xlower, ylower;
    int tilesA, tilesB, nseg;
    ClawCtl* ctl;
};

constexpr int QST3 = 4;  // staged q planes of NT3 values: [position & 1][p, normal velocity]

// aux ring, two neighbour-term buffers, staged q: 160 KB in FP64, inside the
// 164 KB shared-memory carveout (the rest of the SM's 256 KB is L1)
template <typename real>
__host__ __device__ constexpr int sweep3_smem_bytes() {
    return (RING3 * 2 * NS3 + 2 * NTERM3 * NT3 + QST3 * NT3) * (int)sizeof(real) +
           16 * (int)sizeof(double);
}

// one element global -> shared, asynchronously (cp.async, 4 or 8 bytes)
template <typename real>
__device__ __forceinline__ void cp_async_el(real* dst, const real* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src),
                 "n"((int)sizeof(real))
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Source index of (possibly ghost) cell idx along an axis of n cells, and
// whether a solid wall negates the normal velocity (src/3d/bc3.f).
__device__ __forceinline__ int bc3_src(int idx, int n, int lo, int hi, bool& flip) {
    flip = false;
    if (idx < 1) {
        if (lo == BC_PERIODIC) return idx + n;
        if (lo == BC_EXTRAP) return 1;
        flip = (lo == BC_WALL);
        return 1 - idx;
    }
    if (idx > n) {
        if (hi == BC_PERIODIC) return idx - n;
        if (hi == BC_EXTRAP) return n;
        flip = (hi == BC_WALL);
        return 2 * n + 1 - idx;  // wall and piston reflect
    }
    return idx;
}

// Piston velocity of examples/acoustics_3d_heterogeneous/bc3.f:296-309 at the
// ghost column (i, j) and time t: s = -exp(-500 r^2) exp(-500 t^2) for t < 0.1,
// flushed to 0 below 1e-6 in magnitude.
__device__ __forceinline__ double piston_speed(const Sweep3Args<double>& a, int i, int j, double t) {
    if (!(t < 0.1)) return 0.0;
    const double xi = a.xlower + ((double)i - 0.5) * a.d[0];
    const double yj = a.ylower + ((double)j - 0.5) * a.d[1];
    const double r2 = xi * xi + yj * yj;
    double s = -(exp(-(500.0 * r2)) * exp(-(500.0 * (t * t))));
    if (fabs(s) < 1e-6) s = 0.0;
    return s;
}
__device__ __forceinline__ double piston_speed(const Sweep3Args<float>& a, int i, int j, double t) {
    Sweep3Args<double> b;
    b.xlower = a.xlower; b.ylower = a.ylower; b.d[0] = a.d[0]; b.d[1] = a.d[1];
    return piston_speed(b, i, j, t);
}

// flux3's method split (src/3d/flux3.f90:189-197) as compile-time values when
// known (-1: read from the arguments).
template <int M3, int M4, int LIM>
struct Method3D {
    static constexpr int m3 = M3, m4 = M4, lim = LIM;
};
using MethodGeneric3D = Method3D<-1, -1, -1>;
using MethodMC3D = Method3D<2, 2, 4>;  // transverse_waves 22, MC on both waves

// ------------------------------------------------------------ pair variant ---
// Each slice's work is split over a thread pair: both
// threads solve the normal problem, limit and form cqxx (a few dozen
// operations, duplicated); thread h = 0 then owns flux3's y-like side (the
// rpt3 splits in e1, the rptt3 splits of the z-like parts in e1, gadd) and
// h = 1 the z-like side (splits in e2, hadd).  The four combinations each
// side needs from the other's splits (flux3.f90:363-376 and :488-495) cross
// by one shuffle, as do the two centre terms.  Half the registers per thread
// give twice the resident warps of a thread per slice (which needs 255
// registers).  Operation order per value is flux3's, so results are
// bit-identical to the serial reference order in FP64 without contraction.
constexpr int NT3P = 2 * NT3;

// BUILD tells apart the instantiations of the reference-order unit (0,
// --fmad=false) and the contracted unit (1, --fmad=true): the same template
// arguments in both would be one symbol with two different bodies.
template <class S, int DIR, class M, bool LAST, int BUILD>
__global__ void __launch_bounds__(NT3P, CLAW_SWEEP3_MINB) sweep3p_kernel(const Sweep3Args<typename S::real> a) {
    using real = typename S::real;
    using Split = typename S::Split;
    constexpr int AXN = DIR, AXA = DIR == 0 ? 1 : 0, AXB = DIR == 2 ? 1 : 2;
    constexpr bool E1A = DIR != 1;
    constexpr int CN = 1 + AXN, CE1 = 1 + (E1A ? AXA : AXB), CE2 = 1 + (E1A ? AXB : AXA);
    constexpr unsigned FULL = 0xffffffffu;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    real* saux = reinterpret_cast<real*>(smem_raw);  // [RING3][2][NS3]
    real* sterm = saux + RING3 * 2 * NS3;            // [2][NTERM3][NT3]
    real* sq = sterm + 2 * NTERM3 * NT3;             // [QST3][NT3]
    double* red = reinterpret_cast<double*>(sq + QST3 * NT3);

    ClawCtl* ctl = a.ctl;
    grid_dependency_sync();
    if (ctl->done) return;
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
    const int h = tid & 1;           // 0: y-like side (gadd), 1: z-like side (hadd)
    const int sl = tid >> 1;         // slice within the tile
    const int ta = sl % T3A, tb = sl / T3A;
    const int A = A0 - 1 + ta, B = B0 - 1 + tb;
    const bool active = A <= mA + 1 && B <= mB + 1;
    const bool apply = active && ta >= 1 && ta <= T3A - 2 && tb >= 1 && tb <= T3B - 2 &&
                       A <= mA && B <= mB;
    const unsigned amask = __ballot_sync(FULL, active);  // pairs are active together

    unsigned long long perm = 0;
    {
        int code[9], key[9];
        for (int k = 0; k < 9; ++k) {
            const int da = k % 3 - 1, db = k / 3 - 1;
            const int sA = A + da, sB = B + db;
            code[k] = k;
            key[k] = (((sB >> 1) & 1) << 5) | (((sA >> 1) & 1) << 4) | ((db + 1) << 2) | (da + 1);
        }
        for (int i = 1; i < 9; ++i)
            for (int j = i; j > 0 && key[j - 1] > key[j]; --j) {
                int t = key[j]; key[j] = key[j - 1]; key[j - 1] = t;
                t = code[j]; code[j] = code[j - 1]; code[j - 1] = t;
            }
        for (int k = 0; k < 9; ++k) perm |= (unsigned long long)code[k] << (4 * k);
    }

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
    // Z and c of ring position pos, copied asynchronously: issued at the top
    // of a position, awaited just before its CTA barrier
    auto load_aux = [&](int pos) {
        real* dst = saux + (pos & (RING3 - 1)) * 2 * NS3;
        const long long pofs = (long long)(pos + 1) * a.as[AXN];
        for (int e = tid; e < NS3; e += NT3P) {
            const int sa = e % S3A, sb = e / S3A;
            const int Ai = min(A0 - 2 + sa, mA + 2), Bi = min(B0 - 2 + sb, mB + 2);
            const long long o = pofs + (long long)(Ai + 1) * a.as[AXA] + (long long)(Bi + 1) * a.as[AXB];
            cp_async_el(dst + e, aux + o);
            cp_async_el(dst + NS3 + e, aux + o + a.afstride);
        }
    };
    // q of this slice at position pos, staged the same way: h = 0 copies p,
    // h = 1 the normal velocity; boundary conditions apply when the pair takes them
    auto issue_q = [&](int pos) {
        if (!active) return;
        bool fN;
        const int pm = bc3_src(pos, mN, a.bc[2 * AXN], a.bc[2 * AXN + 1], fN);
        const long long off = qoffAB + (long long)(pm - 1) * a.qs[AXN] + (h ? CN * a.fstride : 0);
        cp_async_el(sq + ((pos & 1) * 2 + h) * NT3 + sl, qold + off);
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
    // shared-memory steps of this thread's own split direction and the other
    const int sown = (tb + 1) * S3A + (ta + 1);
    const int e1s = E1A ? 1 : S3A, e2s = E1A ? S3A : 1;
    const int ownS = h ? e2s : e1s, othS = h ? e1s : e2s;
    auto Zo = [&](int pos, int o, int w) -> real {
        return saux[(pos & (RING3 - 1)) * 2 * NS3 + sown + o * ownS + w * othS];
    };
    auto Co = [&](int pos, int o, int w) -> real {
        return saux[(pos & (RING3 - 1)) * 2 * NS3 + NS3 + sown + o * ownS + w * othS];
    };
    // split in the own direction of a fluctuation at the cell `w` across
    auto split_own = [&](real xp, int pos, int w) -> Split {
        return S::split(xp, Zo(pos, -1, w), Co(pos, -1, w), Zo(pos, 0, w), Zo(pos, 1, w), Co(pos, 1, w));
    };
    const real t_own = h ? te2 : te1;
    const real S6own = h ? S6h : S6g;

    double cfl = 0.0;
    auto solve = [&](int i, real pL, real uL, real pR, real uR, real w[2][2], real am[2], real ap[2]) {
        real s[2];
        S::rpn(pL, uL, pR, uR, Zo(i - 1, 0, 0), Co(i - 1, 0, 0), Zo(i, 0, 0), Co(i, 0, 0), w, s, am, ap);
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

    for (int p = p0 - 1; p < p1; ++p) {
        const bool emit = p >= p0;
        // position p+3: its ring slot and staged q were last read before the
        // previous position's barrier
        if (p + 3 <= p1 + 1) {
            load_aux(p + 3);
            issue_q(p + 3);
        }
        const int cA = h ? CE1 : 0, cB = h ? CE2 : CN;  // components this thread updates
        real vA = 0, vB = 0;
        if (emit && apply) {
            const long long off = qoffAB + (long long)(p - 1) * a.qs[AXN];
            const real* src = DIR == 0 ? qold : qnew;
            vA = src[off + cA * a.fstride];
            vB = src[off + cB * a.fstride];
        }
        real F1[2] = {0, 0};
        real Qp[2] = {0, 0};
        real wC[2][2], amC[2], apC[2], qRp = 0, qRn = 0;
        real cterm = 0, own_c = 0;  // centre terms: sent to the partner / kept
        if (active) {
            take_q(p + 2, qRp, qRn);
            solve(p + 2, qLp, qLn, qRp, qRn, wC, amC, apC);
            real wl[2][2];
            const real sB[2] = {-Co(p, 0, 0), Co(p + 1, 0, 0)};
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
            real cq[2] = {0, 0};
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

            const int L = p, R = p + 1;
            // ---- cell p: the amdq side of interface p+1 completes gadd/hadd
            if (m3 > 0) {
                const Split ma = split_own(amB[0], L, 0);
                Split qm = {0, 0, 0, 0};
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
                    const real y1 = __shfl_xor_sync(amask, x1, 1);
                    const real y3 = __shfl_xor_sync(amask, x3, 1);
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
                if (m3 == 2) {
                    O[1][1][0] = O[1][1][0] - tn * qm.up;
                    O[1][1][1] = O[1][1][1] - tn * qm.ut;
                    O[0][1][0] = O[0][1][0] - tn * qm.dp;
                    O[0][1][1] = O[0][1][1] - tn * qm.dt;
                }
            }
            if (emit) {
                // terms for the eight neighbours: own offset o (the side), other w (the level)
                real* out = sterm + (p & 1) * NTERM3 * NT3 + sl;
                for (int w = -1; w <= 1; ++w)
                    for (int o = -1; o <= 1; ++o) {
                        if (o == 0 && w == 0) continue;
                        const int de1 = h ? w : o, de2 = h ? o : w;
                        const int idx9 = (de2 + 1) * 3 + (de1 + 1);
                        const int nb = idx9 < 4 ? idx9 : idx9 - 1;
                        for (int c = 0; c < 2; ++c) {
                            const real tv = o < 0 ? -(t_own * O[0][w + 1][c])
                                          : o == 0 ? -(t_own * (O[1][w + 1][c] - O[0][w + 1][c]))
                                                   : t_own * O[1][w + 1][c];
                            out[(nb * 4 + 2 * h + c) * NT3] = tv;
                        }
                    }
                // centre: h = 0 keeps te1*dG_p and sends te1*dG_e1; h = 1
                // keeps te2*dH_e2 and sends te2*dH_p
                const real dp_ = t_own * (O[1][1][0] - O[0][1][0]);
                const real dv_ = t_own * (O[1][1][1] - O[0][1][1]);
                cterm = h ? dp_ : dv_;
                own_c = h ? dv_ : dp_;
            }
            // ---- cell p+1: the apdq side of interface p+1 starts gadd/hadd
            for (int s_ = 0; s_ < 2; ++s_)
                for (int l = 0; l < 3; ++l)
                    for (int c = 0; c < 2; ++c) O[s_][l][c] = 0;
            if (m3 > 0) {
                const Split mp = split_own(apB[0], R, 0);
                Split qp = {0, 0, 0, 0};
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
                    const real y0 = __shfl_xor_sync(amask, x0, 1);
                    const real y2 = __shfl_xor_sync(amask, x2, 1);
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
                if (m3 == 2) {
                    O[1][1][0] = O[1][1][0] + tn * qp.up;
                    O[1][1][1] = O[1][1][1] + tn * qp.ut;
                    O[0][1][0] = O[0][1][0] + tn * qp.dp;
                    O[0][1][1] = O[0][1][1] + tn * qp.dt;
                }
            }
        }
        const real crecv = __shfl_xor_sync(FULL, cterm, 1);
        cp_async_wait_all();
        __syncthreads();
        if (emit && apply) {
            const real* in = sterm + (p & 1) * NTERM3 * NT3;
            for (int k = 0; k < 9; ++k) {
                const int code = (int)((perm >> (4 * k)) & 15ull);
                if (code == 4) {
                    if (h == 0) {
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
                    const int src = sl + db * T3A + da;
                    if (h == 0) {
                        vA = vA + in[(nb * 4 + 0) * NT3 + src] + in[(nb * 4 + 2) * NT3 + src];
                    } else {
                        vA = vA + in[(nb * 4 + 1) * NT3 + src];
                        vB = vB + in[(nb * 4 + 3) * NT3 + src];
                    }
                }
            }
            const long long off = qoffAB + (long long)(p - 1) * a.qs[AXN];
            qnew[off + cA * a.fstride] = vA;
            qnew[off + cB * a.fstride] = vB;
        }
        if (active) {
            for (int k = 0; k < 2; ++k)
                for (int c = 0; c < 2; ++c) { wA[k][c] = wB[k][c]; wB[k][c] = wC[k][c]; }
            amB[0] = amC[0]; amB[1] = amC[1];
            apB[0] = apC[0]; apB[1] = apC[1];
            qLp = qRp; qLn = qRn;
            F0[0] = F1[0]; F0[1] = F1[1];
        }
    }

    if (LAST) {
        cta_cfl_and_control(ctl, cfl, red);
    } else {
        for (int off = 16; off > 0; off >>= 1) cfl = fmax(cfl, __shfl_xor_sync(FULL, cfl, off));
        if ((tid & 31) == 0) red[tid >> 5] = cfl;
        __syncthreads();
        if (tid == 0) {
            double m = 0.0;
            for (int w = 0; w < NT3P / 32; ++w) m = fmax(m, red[w]);
            if (!(m > 0.0)) m = (m != m) ? m : 0.0;
            atomicMax(&ctl->cfl_bits, (unsigned long long)__double_as_longlong(m));
        }
    }
}

}  // namespace clawb200
