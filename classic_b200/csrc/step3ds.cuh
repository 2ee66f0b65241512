// 3D dimensionally split step (dimsp3 + step3ds + flux3 with method(3) < 0)
// for sm_100a: Godunov splitting, one launch per sweep direction.
//
// Reference: src/3d/dimsp3.f:1-87, src/3d/step3ds.f90:3-408,
// src/3d/flux3.f90:171-277 (normal solve, limiter, second-order correction;
// flux3 returns before its transverse part when method(3) < 0), src/3d/bc3.f.
//
// The x-sweep updates the slices j = 0..my+1, k = 0..mz+1 (one ghost layer
// across), the y-sweep i = 0..mx+1, k = 0..mz+1 and the z-sweep i = 0..mx+1,
// j = 0..my+1; every other ghost cell keeps its bc3 value for the whole step.
// The intermediate state lives in scratch arrays over cells 0..m+1 of each
// axis:
//   X  reads q (interior cells, ghost values from the boundary maps) and
//      writes P: x-updated for i = 1..mx, bc3 values for i = 0, mx+1;
//   Y  reads P and writes the y-updated p and v of cells j = 1..my to P2;
//   Z  reads P / P2 (bc3 values beyond them) and writes the new q's interior.
// Lanes of a warp hold consecutive x positions: X exchanges neighbours by
// shuffle, Y and Z march chunks of 32 cells along y or z with every lane on
// its own slice, so all global accesses are coalesced and no warp reads what
// another writes.  Each sweep's Courant maximum is kept apart and the
// z-sweep's last CTA combines them as dimsp3 does.
//
// Arithmetic per value is flux3's / step3ds's, so the FP64 result is
// bit-identical to the reference order of operations (built with
// --fmad=false).
#pragma once
#include "common.cuh"
#include "riemann.cuh"
#include "step3d.cuh"

namespace clawb200 {

constexpr int DS3_WARPS = 8;      // warps per CTA of the split sweeps
constexpr int DS3_STRIPX = 28;    // x-sweep output columns per warp (lanes 2..29)
constexpr int DS3_CHUNK = 32;     // y- and z-sweep cells per warp march

template <typename real>
struct Split3Args {
    const real* q[2];    // interior cells (the handle's two buffers)
    real* qw[2];
    real* P;             // scratch: cells 0..m+1 of every axis (after the x-sweep)
    real* P2;            // p and v after the y-sweep (cells 1..my of each column)
    const real* aux;     // (Z, c), two ghost layers
    long long qs[3], fstride;
    long long ps[3], pfstride;
    long long as[3], afstride;
    int m[3];
    int bc[6];
    int mthlim[2];
    int order;
    double d[3];
    double xlower, ylower;
    int nstripx, nstrip32;
    int nchunk[3];       // march chunks along y and z
    ClawCtl* ctl;
};

template <typename real>
__device__ __forceinline__ double ds3_piston(const Split3Args<real>& a, int i, int j, double t) {
    Sweep3Args<double> b;
    b.xlower = a.xlower;
    b.ylower = a.ylower;
    b.d[0] = a.d[0];
    b.d[1] = a.d[1];
    return piston_speed(b, i, j, t);
}

// q at the 1-based cell (i, j, k) as bc3 leaves it before the step: each axis
// maps to its source cell (and a wall negates that axis' velocity); the piston
// wall at z-upper sets w = 2 s(i, j, t) - w of the mirror cell.
template <typename real>
__device__ __forceinline__ void ds3_raw(const Split3Args<real>& a, const real* __restrict__ q,
                                        int i, int j, int k, double tbc, real* v) {
    bool fx, fy, fz;
    const int si = bc3_src(min(max(i, -1), a.m[0] + 2), a.m[0], a.bc[0], a.bc[1], fx);
    const int sj = bc3_src(min(max(j, -1), a.m[1] + 2), a.m[1], a.bc[2], a.bc[3], fy);
    const int sk = bc3_src(min(max(k, -1), a.m[2] + 2), a.m[2], a.bc[4], a.bc[5], fz);
    const long long o = (long long)(si - 1) * a.qs[0] + (long long)(sj - 1) * a.qs[1] +
                        (long long)(sk - 1) * a.qs[2];
#pragma unroll
    for (int m = 0; m < 4; ++m) v[m] = q[o + m * a.fstride];
    if (fx) v[1] = -v[1];
    if (fy) v[2] = -v[2];
    if (fz) v[3] = -v[3];
    if (k > a.m[2] && a.bc[5] == BC_PISTON) v[3] = (real)(2.0 * ds3_piston(a, i, j, tbc)) - v[3];
}

template <typename real>
__device__ __forceinline__ long long ds3_aux_off(const Split3Args<real>& a, int i, int j, int k) {
    i = min(max(i, -1), a.m[0] + 2);
    j = min(max(j, -1), a.m[1] + 2);
    k = min(max(k, -1), a.m[2] + 2);
    return (long long)(i + 1) * a.as[0] + (long long)(j + 1) * a.as[1] + (long long)(k + 1) * a.as[2];
}

template <typename real>
__device__ __forceinline__ long long ds3_p_off(const Split3Args<real>& a, int i, int j, int k) {
    return (long long)i * a.ps[0] + (long long)j * a.ps[1] + (long long)k * a.ps[2];
}

// Publish one CTA's maximum of a sweep's Courant numbers into `slot`.
__device__ __forceinline__ void ds3_publish(double cfl, unsigned long long* slot, double* red) {
    for (int off = 16; off > 0; off >>= 1) cfl = fmax(cfl, __shfl_xor_sync(0xffffffffu, cfl, off));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cfl;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
        if (!(m > 0.0)) m = (m != m) ? m : 0.0;
        atomicMax(slot, (unsigned long long)__double_as_longlong(m));
    }
}

// The limited second-order flux of one interface (flux3.f90:227-275):
// w = waves (p, normal velocity), s = speeds, dl / dr = dot products with the
// neighbouring interfaces' unlimited waves.
template <typename real>
__device__ __forceinline__ void ds3_flux(const Split3Args<real>& a, const real (*w)[2],
                                         const real* s, real dl_0, real dl_1, real dr_0,
                                         real dr_1, real dtdxave, real* F) {
    const real dl[2] = {dl_0, dl_1}, dr[2] = {dr_0, dr_1};
    real cq[2] = {real(0), real(0)};
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        real w0 = w[k][0], w1 = w[k][1];
        const int lim = a.mthlim[k];
        if (lim > 0) {
            const real wn2 = w[k][0] * w[k][0] + w[k][1] * w[k][1];
            if (wn2 != real(0)) {
                const real r = (s[k] > real(0) ? dl[k] : dr[k]) / wn2;
                const real phi = phi_limiter<real>(lim, r);
                w0 = phi * w[k][0];
                w1 = phi * w[k][1];
            }
        }
        const real as_ = fabs(s[k]);
        const real coef = (real(0.5) * as_) * (real(1) - as_ * dtdxave);
        cq[0] = cq[0] + coef * w0;
        cq[1] = cq[1] + coef * w1;
    }
    F[0] = cq[0];
    F[1] = cq[1];
}

// ---------------------------------------------------------------- x-sweep ---
template <class S, int BUILD>
__global__ void __launch_bounds__(32 * DS3_WARPS) split3_x_kernel(const Split3Args<typename S::real> a) {
    using real = typename S::real;
    constexpr unsigned FULL = 0xffffffffu;
    __shared__ double red[DS3_WARPS];
    ClawCtl* ctl = a.ctl;
    grid_dependency_sync();
    if (*(volatile int*)&ctl->done) return;
    const int cur = *(volatile int*)&ctl->cur;
    const double dt = *(volatile double*)&ctl->dt;
    const double tbc = *(volatile double*)&ctl->told;
    const real* __restrict__ q = a.q[cur];
    real* __restrict__ P = a.P;
    const double tn_d = dt / a.d[0];
    const real tn = (real)tn_d;
    const real dtdxave = real(0.5) * (tn + tn);
    const int mx = a.m[0], my = a.m[1], mz = a.m[2];
    const int lane = threadIdx.x & 31;
    const long long units = (long long)a.nstripx * (my + 2) * (mz + 2);
    const long long nwarps = (long long)gridDim.x * DS3_WARPS;
    double cfl = 0.0;
    for (long long u = (long long)blockIdx.x * DS3_WARPS + (threadIdx.x >> 5); u < units; u += nwarps) {
        const int sx = (int)(u % a.nstripx);
        const long long jk = u / a.nstripx;
        const int j = (int)(jk % (my + 2)), k = (int)(jk / (my + 2));
        const int b = 1 + sx * DS3_STRIPX;
        const int i = b - 2 + lane;
        real v[4];
        ds3_raw(a, q, i, j, k, tbc, v);
        const long long ao = ds3_aux_off(a, i, j, k);
        const real Z = a.aux[ao], C = a.aux[ao + a.afstride];
        // interface i-1|i on lane l
        const real pm = __shfl_up_sync(FULL, v[0], 1), um = __shfl_up_sync(FULL, v[1], 1);
        const real zm = __shfl_up_sync(FULL, Z, 1), cm = __shfl_up_sync(FULL, C, 1);
        real w[2][2], s[2], am[2], ap[2];
        S::rpn(pm, um, v[0], v[1], zm, cm, Z, C, w, s, am, ap);
        if (lane >= 1 && i >= 1 && i <= mx + 1) {
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {
                const double c = tn_d * (double)s[kk];
                cfl = fmax(fmax(cfl, c), -c);
            }
        }
        real F[2] = {real(0), real(0)};
        if (a.order == 2) {
            real wl[2][2], wr[2][2];
#pragma unroll
            for (int kk = 0; kk < 2; ++kk)
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    wl[kk][c] = __shfl_up_sync(FULL, w[kk][c], 1);
                    wr[kk][c] = __shfl_down_sync(FULL, w[kk][c], 1);
                }
            ds3_flux(a, w, s, wl[0][0] * w[0][0] + wl[0][1] * w[0][1],
                     wl[1][0] * w[1][0] + wl[1][1] * w[1][1], w[0][0] * wr[0][0] + w[0][1] * wr[0][1],
                     w[1][0] * wr[1][0] + w[1][1] * wr[1][1], dtdxave, F);
        }
        const real amr0 = __shfl_down_sync(FULL, am[0], 1), amr1 = __shfl_down_sync(FULL, am[1], 1);
        const real Fr0 = __shfl_down_sync(FULL, F[0], 1), Fr1 = __shfl_down_sync(FULL, F[1], 1);
        const bool upd = lane >= 2 && lane <= 29 && i >= 1 && i <= mx;
        if (upd) {
            const real qa0 = (real(0) - tn * ap[0]) - tn * amr0;
            const real qa1 = (real(0) - tn * ap[1]) - tn * amr1;
            v[0] = (v[0] + qa0) - tn * (Fr0 - F[0]);
            v[1] = (v[1] + qa1) - tn * (Fr1 - F[1]);
        }
        if (upd || i == 0 || i == mx + 1) {
            real* dst = P + ds3_p_off(a, i, j, k);
#pragma unroll
            for (int m = 0; m < 4; ++m) dst[m * a.pfstride] = v[m];
        }
    }
    ds3_publish(cfl, &ctl->cfl_bits, red);
}

// --------------------------------------------------------- y- and z-sweep ---
// AX = 1: columns (i, k), march along j, write p and v of cells 1..my to P2.
// AX = 2: columns (i, j), march along k, write the new q's interior; the last
// CTA combines the three sweeps' Courant numbers and runs claw3's controller.
// A warp marches DS3_CHUNK cells of 32 columns (two cells of halo either side
// are re-solved), so no warp reads what another writes.
template <class S, int AX, int BUILD>
__global__ void __launch_bounds__(32 * DS3_WARPS, 2) split3_yz_kernel(const Split3Args<typename S::real> a) {
    using real = typename S::real;
    __shared__ double red[DS3_WARPS];
    ClawCtl* ctl = a.ctl;
    grid_dependency_sync();
    if (*(volatile int*)&ctl->done) return;
    const int cur = *(volatile int*)&ctl->cur;
    const double dt = *(volatile double*)&ctl->dt;
    const double tbc = *(volatile double*)&ctl->told;
    const real* __restrict__ q = a.q[cur];
    real* __restrict__ qn = a.qw[cur ^ 1];
    const real* __restrict__ P = a.P;
    real* __restrict__ P2 = a.P2;
    const double tn_d = dt / a.d[AX];
    const real tn = (real)tn_d;
    const real dtdxave = real(0.5) * (tn + tn);
    const int mx = a.m[0], my = a.m[1], mz = a.m[2];
    const int mA = a.m[AX];                 // along the march
    const int mO = AX == 1 ? mz : my;       // the other transverse axis
    const int lane = threadIdx.x & 31;
    const int nch = a.nchunk[AX];
    const long long units = (long long)a.nstrip32 * (mO + 2) * nch;
    const long long nwarps = (long long)gridDim.x * DS3_WARPS;
    constexpr int CN = 1 + AX;              // normal velocity component
    double cfl = 0.0;

    for (long long u = (long long)blockIdx.x * DS3_WARPS + (threadIdx.x >> 5); u < units; u += nwarps) {
        const int sx = (int)(u % a.nstrip32);
        const long long rest = u / a.nstrip32;
        const int ch = (int)(rest % nch);
        const int o = (int)(rest / nch);
        const int c_lo = 1 + ch * DS3_CHUNK, c_hi = min(mA, c_lo + DS3_CHUNK - 1);
        const int i = sx * 32 + lane;       // 0..mx+1 valid
        const bool live = i <= mx + 1;
        const int ic = min(i, mx + 1);
        auto cell = [&](int t, int& ci, int& cj, int& ck) {
            ci = ic;
            cj = AX == 1 ? t : o;
            ck = AX == 1 ? o : t;
        };
        // (p, normal velocity) and (Z, c) at march position t
        auto load = [&](int t, real* v, real* zc) {
            int ci, cj, ck;
            cell(t, ci, cj, ck);
            if (t >= 0 && t <= mA + 1) {
                const long long po = ds3_p_off(a, ci, cj, ck);
                if (AX == 2 && cj >= 1 && cj <= my) {
                    v[0] = P2[po];                     // y-updated p
                    v[1] = P[po + CN * a.pfstride];    // w, untouched by the y-sweep
                } else {
                    v[0] = P[po];
                    v[1] = P[po + CN * a.pfstride];
                }
            } else {
                real r[4];
                ds3_raw(a, q, ci, cj, ck, tbc, r);
                v[0] = r[0];
                v[1] = r[CN];
            }
            const long long ao = ds3_aux_off(a, ci, cj, ck);
            zc[0] = a.aux[ao];
            zc[1] = a.aux[ao + a.afstride];
        };

        real vp[2], vt[2], zp[2], zt[2];    // cells t-2, t-1
        real w[2][2], s[2], am[2], ap[2];   // interface t-2|t-1
        real dl0 = 0, dl1 = 0, P1[2] = {0, 0}, Fp[2] = {0, 0};
        load(c_lo - 2, vp, zp);
        load(c_lo - 1, vt, zt);
        S::rpn(vp[0], vp[1], vt[0], vt[1], zp[0], zp[1], zt[0], zt[1], w, s, am, ap);
        real vn[2], zn[2];
        load(c_lo, vn, zn);
        for (int t = c_lo; t <= c_hi + 2; ++t) {
            // prefetch t+1 while working on t
            real vf[2] = {0, 0}, zf[2] = {0, 0};
            if (t + 1 <= c_hi + 2) load(t + 1, vf, zf);
            real wn[2][2], sn[2], amn[2], apn[2];
            S::rpn(vt[0], vt[1], vn[0], vn[1], zt[0], zt[1], zn[0], zn[1], wn, sn, amn, apn);
            if (live && t >= 1 && t <= mA + 1) {  // interface t-1|t, t = 1..m+1
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) {
                    const double c = tn_d * (double)sn[kk];
                    cfl = fmax(fmax(cfl, c), -c);
                }
            }
            const real dr0 = w[0][0] * wn[0][0] + w[0][1] * wn[0][1];
            const real dr1 = w[1][0] * wn[1][0] + w[1][1] * wn[1][1];
            real F[2] = {real(0), real(0)};
            if (a.order == 2) ds3_flux(a, w, s, dl0, dl1, dr0, dr1, dtdxave, F);
            // cell c = t-2: step3ds.f90:220-226 / 304-310 / 388-394
            const int c = t - 2;
            if (live && c >= c_lo && c <= c_hi) {
                const real qa0 = P1[0] - tn * am[0];
                const real qa1 = P1[1] - tn * am[1];
                const real np0 = (vp[0] + qa0) - tn * (F[0] - Fp[0]);
                const real np1 = (vp[1] + qa1) - tn * (F[1] - Fp[1]);
                int ci, cj, ck;
                cell(c, ci, cj, ck);
                const long long po = ds3_p_off(a, ci, cj, ck);
                if (AX == 1) {
                    P2[po] = np0;
                    P2[po + a.pfstride] = np1;
                } else if (ci >= 1 && ci <= mx && cj >= 1 && cj <= my) {
                    const long long qo = (long long)(ci - 1) * a.qs[0] + (long long)(cj - 1) * a.qs[1] +
                                         (long long)(ck - 1) * a.qs[2];
                    qn[qo] = np0;
                    qn[qo + a.fstride] = P[po + a.pfstride];
                    qn[qo + 2 * a.fstride] = P2[po + a.pfstride];
                    qn[qo + 3 * a.fstride] = np1;
                }
            }
            // roll: interface t-1|t becomes current
            P1[0] = real(0) - tn * ap[0];
            P1[1] = real(0) - tn * ap[1];
            Fp[0] = F[0];
            Fp[1] = F[1];
            dl0 = dr0;
            dl1 = dr1;
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {
                s[kk] = sn[kk];
                am[kk] = amn[kk];
                ap[kk] = apn[kk];
                w[kk][0] = wn[kk][0];
                w[kk][1] = wn[kk][1];
                vp[kk] = vt[kk];
                vt[kk] = vn[kk];
                vn[kk] = vf[kk];
                zp[kk] = zt[kk];
                zt[kk] = zn[kk];
                zn[kk] = zf[kk];
            }
        }
    }

    if (AX == 1) {
        ds3_publish(cfl, &ctl->cfl_sweep[0], red);
        return;
    }
    ds3_publish(cfl, &ctl->cfl_sweep[1], red);
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->ctas_done, 1u);
        if (prev == gridDim.x - 1) {
            __threadfence();
            const double cx = __longlong_as_double((long long)atomicAdd(&ctl->cfl_bits, 0ull));
            const double cy = __longlong_as_double((long long)atomicAdd(&ctl->cfl_sweep[0], 0ull));
            const double cz = __longlong_as_double((long long)atomicAdd(&ctl->cfl_sweep[1], 0ull));
            ctl->cfl_sweep[0] = 0ull;
            ctl->cfl_sweep[1] = 0ull;
            // src/3d/dimsp3.f:55-84; a NaN in any sweep stays NaN
            auto nmax = [](double x, double y) { return x != x ? x : (y != y ? y : fmax(x, y)); };
            double c;
            if (cx > ctl->cfl_max) c = cx;
            else if (cy > ctl->cfl_max) c = cy;
            else c = nmax(nmax(cx, cy), cz);
            ctl->cfl_bits = (unsigned long long)__double_as_longlong(c);
            ctl_finish_step(ctl);
            __threadfence();
        }
    }
}

}  // namespace clawb200
