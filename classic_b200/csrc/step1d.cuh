// 1D wave-propagation path: the whole claw1 time loop in ONE persistent CTA.
//
// Reference: src/1d/step1.f90:4-170 (in-place Godunov update, limiter,
// correction flux f), src/1d/bc1.f, src/1d/claw1.f:450-583 (time loop; the
// next dt is chosen before the Courant check, unlike claw2).
//
// 1D grids in this code family are small (hundreds to ~2000 cells), so the
// B200 shape is one CTA holding the grid, its ghost cells, the saved copy for
// rejected steps and all interface quantities in shared memory; each time
// step is four barrier-separated phases and the dt controller runs in thread
// 0.  One launch replaces ~10^3 step launches and host round trips.
#pragma once
#include "common.cuh"

namespace clawb200 {

constexpr int STEP1_THREADS = 512;

template <class S>
struct Step1Args {
    typename S::real* q[2];
    const typename S::real* aux;  // [maux][mx+4]
    long long fstride, afstride;
    int mx;
    int bc[2];
    int mthlim[8];
    int order, fwave, capa;
    double dx;
    // source term (src/1d/claw1.f:486-509): src_split 0 none, 1 Godunov, 2
    // Strang; the radial term of examples/acoustics_2d_radial/1drad/src1.f
    int src_split;
    double src_nd1, src_bulk, xlower;  // ndim - 1, bulk, xlower
    // per-interface waves, speeds and fluctuations: in shared memory when
    // null, else this global buffer of step1_iface_doubles(mx) reals (grids
    // whose interface arrays do not fit the CTA's shared memory; the buffer
    // stays in L2, and __syncthreads orders the CTA's global accesses too)
    typename S::real* iface;
    ClawCtl* ctl;
    S solver;
};

// src1.f:18-23 on cells 0..mx+1 (i = 1..mx+2): p -= dt (ndim-1) bulk / x_i u.
// Thread tid owns the cells k = tid mod blockDim, as the update phases do.
template <class S>
__device__ __forceinline__ void step1_source(const Step1Args<S>& A, typename S::real* qs, int n,
                                             double dts) {
    using real = typename S::real;
    for (int k = threadIdx.x; k < A.mx + 2; k += blockDim.x) {
        const double xcell = A.xlower + ((double)(k + 1) - 0.5) * A.dx;
        const double coef = dts * A.src_nd1 * A.src_bulk / xcell;
        qs[k + 2] = qs[k + 2] - (real)(coef * (double)qs[n + k + 2]);
    }
}

// per-interface wave/s/amdq/apdq (f reuses amdq)
template <class S>
__host__ __device__ constexpr long long step1_iface_doubles(int mx) {
    return (long long)(S::mwaves * S::meqn + S::mwaves + 2 * S::meqn) * (mx + 4);
}

template <class S>
__host__ __device__ constexpr long long step1_smem_doubles(int mx, bool iface_in_smem) {
    // q, aux, dtdx (+ the interface arrays), reduction; the copy kept for a
    // rejected step lives in the output buffer
    return (long long)(S::meqn + S::maux + 1) * (mx + 4) + (iface_in_smem ? step1_iface_doubles<S>(mx) : 0) +
           32;
}

template <class S>
long long step1_smem_bytes(int mx, bool iface_in_smem) {
    return step1_smem_doubles<S>(mx, iface_in_smem) * (long long)sizeof(typename S::real) + 64 * 8;
}

template <class S>
__global__ void __launch_bounds__(STEP1_THREADS, 1) step1_kernel(const __grid_constant__ Step1Args<S> A) {
    using real = typename S::real;
    constexpr int ME = S::meqn, MW = S::mwaves, MA = S::maux;
    constexpr int MAX = MA > 0 ? MA : 1;
    ClawCtl* ctl = A.ctl;
    const int mx = A.mx, n = mx + 4;  // cell k (0-based) lives at k+2
    const int ne = mx + 4;            // interface e in [-1, mx+1] lives at e+1
    extern __shared__ __align__(16) unsigned char smem_raw[];
    real* qs = reinterpret_cast<real*>(smem_raw);
    real* as = qs + ME * n;
    real* dtdx = as + MA * n;
    real* wv = A.iface ? A.iface : dtdx + n;  // [MW][ME][ne]
    real* sv = wv + MW * ME * ne;   // [MW][ne]
    real* amd = sv + MW * ne;       // [ME][ne]
    real* apd = amd + ME * ne;
    real* fl = amd;                 // [ME][ne], once the Godunov update has used amdq
    __shared__ double red[STEP1_THREADS / 32];
    __shared__ double sh_dt, sh_cfl;
    __shared__ int sh_state;  // 0 continue, 1 retry, 2 stop

    const int tid = threadIdx.x;
    const int cur = ctl->cur;
    real* __restrict__ qsave = A.q[cur ^ 1];  // interior copy for a rejected step
    // a single step (claw_step) is step1 alone: accepted whatever its Courant
    // number, without the source steps that claw1 wraps around it
    const bool single = ctl->mode == CTL_SINGLE;
    const int src_split = single ? 0 : A.src_split;
    const real* qin = A.q[cur];
    for (int i = tid; i < ME * mx; i += blockDim.x) {
        const int m = i / mx, k = i % mx;
        qs[m * n + k + 2] = qin[m * A.fstride + k];
    }
    for (int i = tid; i < MA * n; i += blockDim.x) as[i] = A.aux[(i / n) * A.afstride + (i % n)];
    double t = ctl->t, dt = ctl->dt;
    const double tstart = ctl->tstart, tend = ctl->tend;
    const double dxd = A.dx;
    bool limit = false;
    for (int k = 0; k < MW; ++k) limit |= A.mthlim[k] != 0;
    __syncthreads();

    double cflmax = 0.0, dtmin = ctl->dtmin, dtmaxs = ctl->dtmax, cfl = 0.0;
    int nacc = 0, nrej = 0;
    bool stop = false;
    const int maxn = ctl->maxn;
    for (int step = 0; step < maxn && !stop; ++step) {
        const double told = t;
        if (told + dt > tend && tstart < tend) dt = tend - told;
        for (int i = tid; i < ME * mx; i += blockDim.x)
            qsave[(i / mx) * A.fstride + i % mx] = qs[(i / mx) * n + i % mx + 2];
        __syncthreads();
        for (;;) {
            t = told + dt;
            // ---- bc1 (src/1d/bc1.f): ghosts -1,-2 and mx,mx+1; wall negates q(2)
            if (tid < 4 * ME) {
                const int side = tid / (2 * ME), r = tid % (2 * ME), ibc = 1 + r / ME, m = r % ME;
                const int bcode = A.bc[side];
                int dst, src;
                if (side == 0) {
                    dst = -ibc;
                    src = bcode == BC_PERIODIC ? mx - ibc : (bcode == BC_WALL ? ibc - 1 : 0);
                } else {
                    dst = mx - 1 + ibc;
                    src = bcode == BC_PERIODIC ? ibc - 1 : (bcode == BC_WALL ? mx - ibc : mx - 1);
                }
                real v = qs[m * n + src + 2];
                if (bcode == BC_WALL && m == 1) v = -v;
                qs[m * n + dst + 2] = v;
            }
            for (int k = tid; k < n; k += blockDim.x) {
                if (A.capa > 0) dtdx[k] = (real)(dt / (dxd * (double)as[(A.capa - 1) * n + k]));
                else dtdx[k] = (real)(dt / dxd);
            }
            __syncthreads();
            if (src_split == 2) {  // Strang: dt/2 of source before the step
                step1_source(A, qs, n, dt / 2.0);
                __syncthreads();
            }
            // ---- rp1 at interfaces e = -1 .. mx+1 (src/1d/step1.f90:82) + CFL
            double c_loc = 0.0;
            for (int e = tid - 1; e <= mx + 1; e += blockDim.x) {
                real qL[ME], qR[ME], aL[MAX], aR[MAX];
                for (int m = 0; m < ME; ++m) { qL[m] = qs[m * n + e + 1]; qR[m] = qs[m * n + e + 2]; }
                for (int k = 0; k < MA; ++k) { aL[k] = as[k * n + e + 1]; aR[k] = as[k * n + e + 2]; }
                real w[MW][ME], s[MW], am[ME], ap[ME];
                A.solver.rp1(qL, qR, aL, aR, w, s, am, ap);
                for (int mw = 0; mw < MW; ++mw) {
                    for (int m = 0; m < ME; ++m) wv[(mw * ME + m) * ne + e + 1] = w[mw][m];
                    sv[mw * ne + e + 1] = s[mw];
                }
                for (int m = 0; m < ME; ++m) { amd[m * ne + e + 1] = am[m]; apd[m * ne + e + 1] = ap[m]; }
                if (e >= 0 && e <= mx) {
                    const double dR = (double)dtdx[e + 2], dL = (double)dtdx[e + 1];
                    for (int mw = 0; mw < MW; ++mw)
                        c_loc = fmax(fmax(c_loc, dR * (double)s[mw]), -dL * (double)s[mw]);
                }
            }
            __syncthreads();
            // ---- Godunov update of cells 0..mx-1 (in place) and the limited
            //      correction flux f at interfaces 0..mx
            for (int k = tid; k < mx; k += blockDim.x) {
                const real d = dtdx[k + 2];
                for (int m = 0; m < ME; ++m)
                    qs[m * n + k + 2] = (qs[m * n + k + 2] - d * apd[m * ne + k + 1]) - d * amd[m * ne + k + 2];
            }
            if (A.order != 1) {
                __syncthreads();  // f overwrites amdq
                for (int e = tid; e <= mx; e += blockDim.x) {
                    real w[MW][ME];
                    for (int mw = 0; mw < MW; ++mw)
                        for (int m = 0; m < ME; ++m) w[mw][m] = wv[(mw * ME + m) * ne + e + 1];
                    if (limit) {
                        for (int mw = 0; mw < MW; ++mw) {
                            const int ml = A.mthlim[mw];
                            if (ml == 0) continue;
                            real nn = real(0), dl = real(0), dr = real(0);
                            for (int m = 0; m < ME; ++m) {
                                const real wl = wv[(mw * ME + m) * ne + e];
                                const real wr = wv[(mw * ME + m) * ne + e + 2];
                                nn = nn + w[mw][m] * w[mw][m];
                                dr = dr + w[mw][m] * wr;
                                dl = dl + wl * w[mw][m];
                            }
                            if (nn == real(0)) continue;
                            const real r = (sv[mw * ne + e + 1] > real(0) ? dl : dr) / nn;
                            const real ph = phi_limiter<real>(ml, r);
                            for (int m = 0; m < ME; ++m) w[mw][m] = ph * w[mw][m];
                        }
                    }
                    const real ave = real(0.5) * (dtdx[e + 1] + dtdx[e + 2]);
                    real f[ME];
                    for (int m = 0; m < ME; ++m) f[m] = real(0);
                    for (int mw = 0; mw < MW; ++mw) {
                        const real sm = sv[mw * ne + e + 1], as_ = fabs(sm);
                        const real coef = A.fwave ? real(0.5) * copysign(real(1), sm) * (real(1) - as_ * ave)
                                                  : real(0.5) * as_ * (real(1) - as_ * ave);
                        for (int m = 0; m < ME; ++m) f[m] = f[m] + coef * w[mw][m];
                    }
                    for (int m = 0; m < ME; ++m) fl[m * ne + e + 1] = f[m];
                }
            }
            // CFL reduction
            for (int off = 16; off > 0; off >>= 1) c_loc = fmax(c_loc, __shfl_xor_sync(0xffffffffu, c_loc, off));
            if ((tid & 31) == 0) red[tid >> 5] = c_loc;
            __syncthreads();
            if (A.order != 1) {
                for (int k = tid; k < mx; k += blockDim.x) {
                    const real d = dtdx[k + 2];
                    for (int m = 0; m < ME; ++m)
                        qs[m * n + k + 2] = qs[m * n + k + 2] - d * (fl[m * ne + k + 2] - fl[m * ne + k + 1]);
                }
            }
            // source after the step, before the Courant check (claw1.f:499-509)
            if (src_split == 2) step1_source(A, qs, n, dt / 2.0);
            if (src_split == 1) step1_source(A, qs, n, dt);
            if (tid == 0) {
                double cm = 0.0;
                for (int w = 0; w < STEP1_THREADS / 32; ++w) cm = fmax(cm, red[w]);
                sh_cfl = cm;
                // claw1: choose the next dt first (src/1d/claw1.f:520-529) ...
                double dtn = dt;
                if (ctl->dt_variable) {
                    if (cm > 0.0) {
                        dtn = fmin(ctl->dt_max, dt * ctl->cfl_desired / cm);
                        dtmin = fmin(dtn, dtmin);
                        dtmaxs = fmax(dtn, dtmaxs);
                    } else {
                        dtn = ctl->dt_max;
                    }
                }
                sh_dt = dtn;
                // ... then check the Courant number (src/1d/claw1.f:533-554)
                if (cm != cm) sh_state = single ? 0 : 3;
                else if (single || cm <= ctl->cfl_max) sh_state = 0;
                else sh_state = ctl->dt_variable ? 1 : 2;
            }
            __syncthreads();
            cfl = sh_cfl;
            dt = sh_dt;
            const int st = sh_state;
            if (st == 0) {
                cflmax = fmax(cfl, cflmax);
                break;
            }
            t = told;
            for (int i = tid; i < ME * mx; i += blockDim.x)
                qs[(i / mx) * n + i % mx + 2] = qsave[(i / mx) * A.fstride + i % mx];
            __syncthreads();
            if (st == 1) { ++nrej; continue; }
            if (st == 3) { if (tid == 0) ctl->err |= CTL_ERR_NAN_CFL; stop = true; break; }
            cflmax = fmax(cfl, cflmax);
            stop = true;
            break;
        }
        if (stop) break;
        ++nacc;
        if (t >= tend) break;
        __syncthreads();
    }
    __syncthreads();
    real* qout = A.q[cur ^ 1];
    for (int i = tid; i < ME * mx; i += blockDim.x) {
        const int m = i / mx, k = i % mx;
        qout[m * A.fstride + k] = qs[m * n + k + 2];
    }
    if (tid == 0) {
        ctl->t = t;
        ctl->dt = dt;
        ctl->cflmax_seen = cflmax;
        ctl->cfl_last = cfl;
        ctl->dtmin = dtmin;
        ctl->dtmax = dtmaxs;
        ctl->n = nacc;
        ctl->nrej = nrej;
        ctl->cur = cur ^ 1;
        ctl->done = 1;
    }
}

}  // namespace clawb200
