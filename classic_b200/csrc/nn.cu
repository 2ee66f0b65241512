// Convolutional coarse-grid corrector: the network's kernels (C ABI, raw
// device pointers, declared in include/claw_nn.h).
//
// The corrector is a stack of 3x3 "same" convolutions over NHWC BF16
// activations with FP32 accumulation on the tensor cores, GELU between
// layers.  The forward convolution (and the data gradient, the same
// convolution with flipped and transposed weights) runs on the 5th-generation
// tensor cores: tcgen05.mma of shared-memory operands into a TMEM
// accumulator, read back with tcgen05.ld for the epilogue.  Training runs on
// the device with the kernels below: the forward convolution (optionally
// saving the FP32 pre-activation), the data gradient, the weight/bias
// gradient (a pixel-reduction GEMM per tile with mma.sync, plus a reduction
// over tiles), GELU's derivative, the MSE loss gradient and Adam.  Glue kernels move between the solver's FP64 SoA q and
// the network: block averages of a fine grid, input features, residual
// targets, and the corrector's application with a per-tile conservative
// projection and a positivity fallback to the plain step.
#include <algorithm>
#include <atomic>

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include "../../include/claw_nn.h"
#include "common.cuh"

// Device-side error flags of the network kernels (bit 0: a tensor-core
// accumulator wait gave up); read and cleared by nn_device_error().
__device__ int g_nn_err;

namespace {

constexpr int TILE = 16;              // output tile edge (pixels)
constexpr int HALO = TILE + 2;        // input tile edge with the 3x3 halo
constexpr int NPIX = TILE * TILE;     // 256 output pixels per CTA
constexpr int NTHREADS = 256;         // 8 warps

__device__ __forceinline__ void mma_bf16(float d[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) {
    return *reinterpret_cast<const uint32_t*>(p);
}
__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// GELU in its tanh form (Hendrycks and Gimpel, "Gaussian Error Linear Units",
// 2016): GELU(z) = z/2 (1 + tanh(u)), u = sqrt(2/pi) (z + 0.044715 z^3), with
// the hardware tanh (tanh.approx.f32, relative error about 2^-11).  It is
// within 5e-4 of z Phi(z), below the resolution of the BF16 activations, and
// costs about 7 instructions per value where the erf form costs several
// times that: the convolution's epilogue applies it to every output.
// Derivative: (1 + t)/2 + z/2 (1 - t^2) du/dz, du/dz = sqrt(2/pi) (1 + 3 0.044715 z^2).
__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float GELU_K0 = 0.79788456080286536f;  // sqrt(2/pi)
constexpr float GELU_K1 = 0.044715f;
__device__ __forceinline__ float gelu(float z) {
    const float t = tanh_hw(GELU_K0 * fmaf(GELU_K1 * z, z * z, z));
    const float hz = 0.5f * z;
    return fmaf(hz, t, hz);
}
__device__ __forceinline__ float gelu_grad(float z) {
    const float t = tanh_hw(GELU_K0 * fmaf(GELU_K1 * z, z * z, z));
    const float du = GELU_K0 * fmaf(3.0f * GELU_K1 * z, z, 1.0f);
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * du;
}

// Load a HALO x HALO x CP input tile (zero outside the image) into shared
// memory with a row pitch of CP + 8 elements (conflict-free fragment loads).
template <int CP>
__device__ __forceinline__ void load_halo(__nv_bfloat16* xs, const __nv_bfloat16* x, int n, int h,
                                          int w, int y0, int x0) {
    constexpr int CH = CP / 8;  // 16-byte chunks per pixel
    for (int e = threadIdx.x; e < HALO * HALO * CH; e += NTHREADS) {
        const int pix = e / CH, ck = e % CH;
        const int gy = y0 + pix / HALO - 1, gx = x0 + pix % HALO - 1;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (gy >= 0 && gy < h && gx >= 0 && gx < w)
            v = *reinterpret_cast<const uint4*>(x + (((long long)n * h + gy) * w + gx) * CP + ck * 8);
        *reinterpret_cast<uint4*>(xs + pix * (CP + 8) + ck * 8) = v;
    }
}

// ------------------------------------------------- forward conv, tcgen05 ---
// The convolution as an implicit GEMM on the 5th-generation tensor cores.
// A tile is 16 rows x 8 columns of output: M = 128 pixels, N = COUT, K = 9
// taps x CIN.  The halo tile (18 x 10 pixels) and the weights sit in shared
// memory in the UMMA no-swizzle K-major layout (core matrices of 8 rows x 16
// bytes: 8 pixels or 8 output channels, 8 input channels), so each tap's
// operand A is the halo tile itself with the start address moved by the
// tap's offset: 8-row groups (tile rows) are HW*16 bytes apart, 8-channel
// chunks one halo plane apart.  One thread issues the 9 x CIN/16
// tcgen05.mma (M128 N=COUT K16, BF16 -> FP32) into a TMEM accumulator and
// commits them to an mbarrier; each warp of the tile's group then reads its
// 32 pixels (TMEM lanes) with tcgen05.ld and applies bias, GELU and the
// stores.  These are the shared pieces; the kernel is conv3x3_fwd_tcp below.
namespace tc {
constexpr int TW = 8, TH = 16, HW = TW + 2, HH = TH + 2, NPX = HW * HH;
constexpr int NTH = 128;

__host__ __device__ constexpr uint32_t idesc_bf16_f32(int m, int n) {
    // c_format F32 (bits 4-5), a/b format BF16 (bits 7-9, 10-12), both K-major,
    // N >> 3 (bits 17-22), M >> 4 (bits 24-28)
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
// shared-memory matrix descriptor: no swizzle, lbo = bytes between core
// matrices adjacent in K, sbo = bytes between 8-row groups; version 1
__device__ __forceinline__ uint64_t desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                    uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(clawb200::smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void alloc(uint32_t* slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(clawb200::smem_u32(slot)), "r"(cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
// 32 lanes x 16 columns of 32-bit values (this warp's lane quarter)
__device__ __forceinline__ void ld16(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

}  // namespace tc

// ------------------------------------- forward conv, tcgen05, persistent ---
// The implicit GEMM in a persistent CTA that keeps the weights in shared
// memory and pipelines its tiles.  The driver keeps one CTA of a TMEM-allocating kernel
// per SM, so the CTA runs NPIPE independent pipelines, one per group of four
// warps, each with three halo stages in shared memory and two TMEM
// accumulators of its own.  In a pipeline, while the tensor core runs tile
// i's 9 x CIN/16 MMAs into one accumulator, the group runs tile i-1's
// epilogue (tcgen05.ld, bias, GELU, stores) from the other, then starts the
// copy of tile i+2's halo into the third stage: TMA boxes issued by the
// pipeline's first thread, completing on the stage's mbarrier, which that
// thread alone waits on before it issues the tile's MMAs.  A stage is
// refilled only after the MMAs that read it have committed (the epilogue's
// mbarrier wait); an accumulator is reused only after every thread's
// tcgen05.ld of it has completed: each thread arrives on the accumulator's
// mbarrier after its loads (behind a tcgen05 fence) and the issuing thread
// alone waits on it, so the group's warps never stop for one another.
// Every wait is bounded.
namespace tcp {
constexpr int NST = 3;    // halo stages per pipeline
constexpr int NPIPE = 4;  // pipelines (groups of 4 warps) per CTA
constexpr int NTH = NPIPE * tc::NTH;
__device__ __forceinline__ void arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(clawb200::smem_u32(bar)) : "memory");
}
// one 8-channel plane of a halo tile, padded so that every TMA destination
// starts on a 128-byte boundary
constexpr int PLANE = ((tc::NPX * 16 + 127) / 128) * 128;
template <int CIN>
__host__ __device__ constexpr int stage_bytes() { return (CIN / 8) * PLANE; }
template <int CIN, int COUT>
__host__ __device__ constexpr int smem_bytes() {
    // + 128: the base is rounded up to a 128-byte boundary in the kernel
    return 128 + NPIPE * NST * stage_bytes<CIN>() + 9 * (CIN / 8) * COUT * 16 + COUT * 4;
}
}  // namespace tcp

template <int CIN, int COUT, int ACT, bool OUTF32, bool SAVEZ>
__global__ void __launch_bounds__(tcp::NTH, 1) conv3x3_fwd_tcp(const __nv_bfloat16* __restrict__ x,
                                                            const __nv_bfloat16* __restrict__ wt,
                                                            const float* __restrict__ bias, void* out,
                                                            float* __restrict__ zsave, int n, int h,
                                                            int w, const __grid_constant__ CUtensorMap tmx) {
    using namespace tc;
    static_assert(CIN % 16 == 0 && (COUT == 16 || COUT == 32), "UMMA M128: N in {16, 32}, K in steps of 16");
    constexpr int KC = CIN / 8;
    constexpr int APLANE = tcp::PLANE;
    constexpr int ASTAGE = tcp::stage_bytes<CIN>();
    constexpr int BPLANE = COUT * 16;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // TMA writes the halo planes: start them on a 128-byte boundary
    unsigned char* smem = smem_raw + ((128u - (clawb200::smem_u32(smem_raw) & 127u)) & 127u);
    __shared__ uint64_t bar[tcp::NPIPE][2];           // a tile's MMAs committed (per accumulator)
    __shared__ uint64_t full[tcp::NPIPE][tcp::NST];   // a stage's halo landed (TMA bytes)
    __shared__ uint64_t freed[tcp::NPIPE][2];         // every thread has read an accumulator
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = warp >> 2;               // pipeline of this thread
    const int gt = tid & (tc::NTH - 1);    // thread within the pipeline
    const int gw = warp & 3;               // warp within the pipeline = its TMEM lane quarter
    unsigned char* As = smem + g * tcp::NST * ASTAGE;        // this pipeline's [NST][KC][NPX][8 ch]
    unsigned char* Bs = smem + tcp::NPIPE * tcp::NST * ASTAGE;  // [9][KC][COUT][8 ch]
    float* bs = reinterpret_cast<float*>(Bs + 9 * KC * BPLANE);
    const int tiles_x = w / TW, tiles_img = tiles_x * (h / TH);
    const int ntiles = tiles_img * n;

    if (warp == 0) alloc(&tslot, 64 * tcp::NPIPE);
    if (gt == 0) {
        clawb200::mbar_init(&bar[g][0], 1);
        clawb200::mbar_init(&bar[g][1], 1);
        for (int st = 0; st < tcp::NST; ++st) clawb200::mbar_init(&full[g][st], 1);
        clawb200::mbar_init(&freed[g][0], tc::NTH);
        clawb200::mbar_init(&freed[g][1], tc::NTH);
        clawb200::fence_barrier_init();
    }
    // Launched with programmatic dependent launch, this CTA may start while the
    // previous launch drains: it waits here, before its first read of x, the
    // weights or the bias and its first write, for that launch to complete.
    clawb200::grid_dependency_sync();
    // halo tile of tile t into stage st of this pipeline: KC boxes of 8
    // channels x 10 x 18 pixels (NHWC), issued by the pipeline's first
    // thread; the box starts one pixel up and left of the tile and the copy
    // fills with zeros outside the image
    auto load_tile = [&](int t, int st) {
        if (t >= ntiles || gt != 0) return;
        const int img = t / tiles_img, r = t % tiles_img;
        const int y0 = (r / tiles_x) * TH, x0 = (r % tiles_x) * TW;
        unsigned char* A = As + st * ASTAGE;
        clawb200::mbar_arrive_expect_tx(&full[g][st], (uint32_t)(KC * NPX * 16));
#pragma unroll
        for (int kc = 0; kc < KC; ++kc)
            clawb200::tma_load_4d(A + kc * APLANE, &tmx, kc * 8, x0 - 1, y0 - 1, img, &full[g][st]);
    };
    bool ok = true;
    // epilogue of tile t, the j-th of this pipeline (accumulator j & 1)
    auto epilogue = [&](int t, int j) {
        const int b = j & 1;
        const bool done = clawb200::mbar_wait_bounded(&bar[g][b], (uint32_t)((j >> 1) & 1));
        if (!done) {  // never expected: record it, give the MMAs a second bound, skip the stores
            if (lane == 0) atomicOr(&g_nn_err, 1);
            (void)clawb200::mbar_wait_bounded(&bar[g][b], (uint32_t)((j >> 1) & 1));
            ok = false;
        }
        fence_after();
        const int img = t / tiles_img, r = t % tiles_img;
        const int y0 = (r / tiles_x) * TH, x0 = (r % tiles_x) * TW;
        const int m = gw * 32 + lane;
        const long long pix = ((long long)img * h + y0 + m / TW) * w + x0 + m % TW;
        const uint32_t trow = tslot + ((uint32_t)(gw * 32) << 16) + (uint32_t)(g * 64 + b * 32);
        // every column of the accumulator in flight at once, one wait
        uint32_t rr[COUT];
#pragma unroll
        for (int c0 = 0; c0 < COUT; c0 += 16) ld16(trow + c0, rr + c0);
        wait_ld();
        fence_before();
        tcp::arrive(&freed[g][b]);  // this thread is done with accumulator b
        if (!ok) return;
#pragma unroll
        for (int c0 = 0; c0 < COUT; c0 += 16) {
            float z[16], yv[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                z[q] = __uint_as_float(rr[c0 + q]) + bs[c0 + q];
                yv[q] = ACT ? gelu(z[q]) : z[q];
            }
            if (SAVEZ) {
#pragma unroll
                for (int q = 0; q < 16; q += 4)
                    *reinterpret_cast<float4*>(zsave + pix * COUT + c0 + q) =
                        make_float4(z[q], z[q + 1], z[q + 2], z[q + 3]);
            }
            if (OUTF32) {
#pragma unroll
                for (int q = 0; q < 16; q += 4)
                    *reinterpret_cast<float4*>(static_cast<float*>(out) + pix * COUT + c0 + q) =
                        make_float4(yv[q], yv[q + 1], yv[q + 2], yv[q + 3]);
            } else {
                uint32_t pk[8];
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    pk[q] = pack2(__float2bfloat16_rn(yv[2 * q]), __float2bfloat16_rn(yv[2 * q + 1]));
                uint4* dst = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(out) + pix * COUT + c0);
                dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            }
        }
    };

    const int first = blockIdx.x * tcp::NPIPE + g, stride = gridDim.x * tcp::NPIPE;
    // the first two halo copies fly while the weights are staged
    load_tile(first, 0);
    load_tile(first + stride, 1);
    for (int e = tid; e < COUT * 9 * KC; e += tcp::NTH) {  // wt[co][tap][ci] -> [tap][kc][co]
        const int co = e / (9 * KC), r = e % (9 * KC), tap = r / KC, kc = r % KC;
        *reinterpret_cast<uint4*>(Bs + (tap * KC + kc) * BPLANE + co * 16) =
            *reinterpret_cast<const uint4*>(wt + ((long long)co * 9 + tap) * CIN + kc * 8);
    }
    for (int e = tid; e < COUT; e += tcp::NTH) bs[e] = bias[e];
    clawb200::fence_proxy_async_smem();  // the tensor core reads the weights these threads wrote
    fence_before();
    __syncthreads();  // barriers initialised, weights in place, TMEM allocated
    fence_after();
    const uint32_t tacc = tslot + (uint32_t)(g * 64);
    constexpr uint32_t idesc = idesc_bf16_f32(128, COUT);
    const uint32_t b0 = clawb200::smem_u32(Bs);
    int i = 0;
    for (int t = first; t < ntiles; t += stride, ++i) {
        if (gt == 0) {
            // accumulator i & 1 is free: every thread's tcgen05.ld of tile i-2 is done
            if (i >= 2) {
                const uint32_t par = (uint32_t)(((i - 2) >> 1) & 1);
                if (!clawb200::mbar_wait_bounded(&freed[g][i & 1], par)) {
                    atomicOr(&g_nn_err, 1);
                    (void)clawb200::mbar_wait_bounded(&freed[g][i & 1], par);
                }
                fence_after();
            }
            // tile i's halo has landed (only the MMAs read it)
            const int st = i % tcp::NST;
            if (!clawb200::mbar_wait_bounded(&full[g][st], (uint32_t)((i / tcp::NST) & 1))) {
                atomicOr(&g_nn_err, 1);  // never expected: record it, give the copy a second bound
                (void)clawb200::mbar_wait_bounded(&full[g][st], (uint32_t)((i / tcp::NST) & 1));
            }
            const uint32_t a0 = clawb200::smem_u32(As + st * ASTAGE);
            const uint32_t acc_addr = tacc + (uint32_t)((i & 1) * 32);
            uint32_t acc = 0;
#pragma unroll
            for (int tap = 0; tap < 9; ++tap) {
                const int ky = tap / 3, kx = tap % 3;
#pragma unroll
                for (int kk = 0; kk < CIN / 16; ++kk) {
                    const uint64_t da = desc(a0 + (ky * HW + kx) * 16 + 2 * kk * APLANE, APLANE, HW * 16);
                    const uint64_t db = desc(b0 + (tap * KC + 2 * kk) * BPLANE, BPLANE, 128);
                    mma(acc_addr, da, db, idesc, acc);
                    acc = 1;
                }
            }
            commit(&bar[g][i & 1]);
        }
        if (i > 0) epilogue(t - stride, i - 1);
        // the stage tile i-1's MMAs read: they have committed (the epilogue waited)
        load_tile(t + 2 * stride, (i + 2) % tcp::NST);
        fence_before();
    }
    if (i > 0) epilogue(first + (i - 1) * stride, i - 1);
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        dealloc(tslot, 64 * tcp::NPIPE);
    }
}


// ------------------------------------------------------- weight gradient ---
// partial[blk][co][tap*CIN + ci] = sum over the tile's pixels p of
//   dz[p, co] * x[p + off(tap), ci];  pdb[blk][co] = sum_p dz[p, co].
// GEMM M = COUT (dz transposed in shared memory), N = 9*CIN (im2col of the
// halo tile), K = the tile's 256 pixels.
template <int CIN, int COUT>
__global__ void __launch_bounds__(NTHREADS) conv3x3_wgrad(const __nv_bfloat16* __restrict__ x,
                                                           const __nv_bfloat16* __restrict__ dz,
                                                           float* __restrict__ partial,
                                                           float* __restrict__ pdb, int h, int w) {
    constexpr int XP = CIN + 8, DP = NPIX + 8;
    constexpr int MT = COUT / 16, NT = 9 * CIN / 8, TILES = MT * NT, TPW = (TILES + 7) / 8;
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* xs = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* dzt = xs + HALO * HALO * XP;  // [COUT][NPIX + 8]
    const int n = blockIdx.z, y0 = blockIdx.y * TILE, x0 = blockIdx.x * TILE;
    const long long blk = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    load_halo<CIN>(xs, x, n, h, w, y0, x0);
    for (int e = threadIdx.x; e < NPIX * COUT; e += NTHREADS) {
        const int p = e / COUT, co = e % COUT;
        const long long pix = ((long long)n * h + y0 + p / TILE) * w + x0 + p % TILE;
        dzt[co * DP + p] = dz[pix * COUT + co];
    }
    __syncthreads();
    if (threadIdx.x < COUT) {
        float s = 0.f;
        for (int p = 0; p < NPIX; ++p) s += __bfloat162float(dzt[threadIdx.x * DP + p]);
        pdb[blk * COUT + threadIdx.x] = s;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    float acc[TPW][4];
#pragma unroll
    for (int i = 0; i < TPW; ++i)
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[i][k] = 0.f;
#pragma unroll 1
    for (int k0 = 0; k0 < NPIX; k0 += 16) {
        // pixels k0+2t, k0+2t+1 (b0) and k0+2t+8, +9 (b1): all in tile row k0/16
        const int prow = k0 / TILE;
#pragma unroll
        for (int i = 0; i < TPW; ++i) {
            const int tile = warp + 8 * i;
            if (tile >= TILES) break;
            const int mt = tile / NT, nt = tile % NT;
            const int co = mt * 16 + g;
            const __nv_bfloat16* ap = dzt + co * DP + k0 + 2 * t;
            const uint32_t a[4] = {ld32(ap), ld32(ap + 8 * DP), ld32(ap + 8), ld32(ap + 8 * DP + 8)};
            const int tap = (nt * 8) / CIN, ci = (nt * 8) % CIN + g;
            const int ky = tap / 3, kx = tap % 3;
            const __nv_bfloat16* xr = xs + ((prow + ky) * HALO + kx) * XP + ci;
            const int c0 = 2 * t;  // tile column of the first pixel of b0
            uint32_t b[2];
            b[0] = pack2(xr[(c0)*XP], xr[(c0 + 1) * XP]);
            b[1] = pack2(xr[(c0 + 8) * XP], xr[(c0 + 9) * XP]);
            mma_bf16(acc[i], a, b);
        }
    }
    float* out = partial + blk * (long long)(COUT * 9 * CIN);
#pragma unroll
    for (int i = 0; i < TPW; ++i) {
        const int tile = warp + 8 * i;
        if (tile >= TILES) break;
        const int mt = tile / NT, nt = tile % NT;
        const int col = nt * 8 + 2 * t;
        const int r0 = mt * 16 + g, r1 = r0 + 8;
        out[r0 * 9 * CIN + col] = acc[i][0];
        out[r0 * 9 * CIN + col + 1] = acc[i][1];
        out[r1 * 9 * CIN + col] = acc[i][2];
        out[r1 * 9 * CIN + col + 1] = acc[i][3];
    }
}

template <int CIN, int COUT>
constexpr int wgrad_smem() {
    return HALO * HALO * (CIN + 8) * 2 + COUT * (NPIX + 8) * 2;
}

// sum over tiles: dst[j] = sum_b src[b][j]
__global__ void reduce_tiles(const float* __restrict__ src, float* __restrict__ dst, long long nblk,
                             int len) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < len; j += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (long long b = 0; b < nblk; ++b) s += src[b * len + j];
        dst[j] = s;
    }
}

// Wt[ci][tap][co] = W[co][8 - tap][ci]: the data gradient's weights
__global__ void flip_weights(const __nv_bfloat16* __restrict__ w, __nv_bfloat16* __restrict__ wt,
                             int cout, int cin) {
    const int n = cout * 9 * cin;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int ci = e / (9 * cout), rest = e % (9 * cout), tap = rest / cout, co = rest % cout;
        wt[e] = w[((long long)co * 9 + (8 - tap)) * cin + ci];
    }
}

__global__ void gelu_backward(const __nv_bfloat16* __restrict__ dy, const float* __restrict__ z,
                              __nv_bfloat16* __restrict__ dz, long long n) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x)
        dz[e] = __float2bfloat16_rn(__bfloat162float(dy[e]) * gelu_grad(z[e]));
}

// MSE over the first nc of cp channels: dy = 2 (pred - target) / count,
// loss accumulated in FP64 (one atomic per block)
__global__ void mse_grad(const float* __restrict__ pred, const float* __restrict__ target,
                         __nv_bfloat16* __restrict__ dy, double* __restrict__ loss, long long npix,
                         int cp, int nc, float inv_count, float delta) {
    __shared__ double red[NTHREADS / 32];
    double acc = 0.0;
    const long long n = npix * cp;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const long long p = e / cp;
        const int c = (int)(e % cp);
        float g = 0.f;
        const float tg = c < nc ? target[p * nc + c] : 0.f;
        if (c < nc && tg == tg) {  // a NaN target masks the pixel out
            const float d = pred[e] - tg;
            if (delta > 0.f && fabsf(d) > delta) {  // Huber: linear beyond delta
                acc += 2.0 * (double)delta * (double)fabsf(d) - (double)delta * (double)delta;
                g = 2.f * copysignf(delta, d) * inv_count;
            } else {
                acc += (double)d * (double)d;
                g = 2.f * d * inv_count;
            }
        }
        dy[e] = __float2bfloat16_rn(g);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < NTHREADS / 32; ++k) s += red[k];
        atomicAdd(loss, s);
    }
}

__global__ void adam_step(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, __nv_bfloat16* __restrict__ w16, long long n,
                          float lr, float b1, float b2, float eps, float c1, float c2) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const float ge = g[e];
        const float me = b1 * m[e] + (1.f - b1) * ge;
        const float ve = b2 * v[e] + (1.f - b2) * ge * ge;
        m[e] = me;
        v[e] = ve;
        const float wn = w[e] - lr * (me / c1) / (sqrtf(ve / c2) + eps);
        w[e] = wn;
        if (w16) w16[e] = __float2bfloat16_rn(wn);
    }
}

// ---------------------------------------------------------- solver glue ---
// coarse[m][j][i] = mean of the r x r fine block (FP64 SoA, row pitches ldf/ldc)
__global__ void block_average(const double* __restrict__ fine, long long ldf, long long fsf,
                              double* __restrict__ coarse, long long ldc, long long fsc, int mxc,
                              int myc, int r, int meqn) {
    const long long n = (long long)meqn * mxc * myc;
    const double inv = 1.0 / (double)(r * r);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(e / ((long long)mxc * myc));
        const long long rest = e % ((long long)mxc * myc);
        const int j = (int)(rest / mxc), i = (int)(rest % mxc);
        double s = 0.0;
        for (int b = 0; b < r; ++b)
            for (int a = 0; a < r; ++a)
                s += fine[m * fsf + (long long)(j * r + b) * ldf + (i * r + a)];
        coarse[m * fsc + (long long)j * ldc + i] = s * inv;
    }
}

// features x[p][c] (BF16, 16 channels): c < 4 the normalised state
// (q - mu_c) / s_c, 4 <= c < 8 the plain step's increment (qs - q) / d_c,
// the rest zero.
__global__ void features(const double* __restrict__ q, const double* __restrict__ qs, long long ld,
                         long long fs, int mx, int my, int img, const float* __restrict__ norm,
                         __nv_bfloat16* __restrict__ x) {
    const long long n = (long long)mx * my;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(p / mx), i = (int)(p % mx);
        __nv_bfloat16 v[8];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const double a = q[c * fs + (long long)j * ld + i], b = qs[c * fs + (long long)j * ld + i];
            v[c] = __float2bfloat16_rn((float)((a - (double)norm[c]) * (double)norm[4 + c]));
            v[4 + c] = __float2bfloat16_rn((float)((b - a) * (double)norm[8 + c]));
        }
        uint4* dst = reinterpret_cast<uint4*>(x + ((long long)img * n + p) * 16);
        dst[0] = make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
        dst[1] = make_uint4(0, 0, 0, 0);
    }
}

// target[p][c] = (qf - qs) * norm[12 + c]: the residual the corrector learns
__global__ void residual_target(const double* __restrict__ qf, const double* __restrict__ qs,
                                long long ld, long long fs, int mx, int my, int img,
                                const float* __restrict__ norm, float* __restrict__ target) {
    const long long n = (long long)mx * my;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(p / mx), i = (int)(p % mx);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const long long o = c * fs + (long long)j * ld + i;
            target[((long long)img * n + p) * 4 + c] = (float)((qf[o] - qs[o]) * (double)norm[12 + c]);
        }
    }
}

// Apply the corrector to one grid, one CTA per 16x16 tile: the residual of
// each field (r[p][c] / norm[12+c]) minus its tile mean (so the tile's
// conserved totals are unchanged), added to the plain step qs; a tile whose
// corrected density or pressure is not positive, or whose totals moved by
// more than tol relative, keeps the plain step.  flags[tile] = 1 if
// corrected, 0 if it fell back.
__global__ void __launch_bounds__(NTHREADS) apply_correction(double* __restrict__ qs, long long ld,
                                                             long long fs, int mx, int my,
                                                             const float* __restrict__ r, int rcp,
                                                             const float* __restrict__ norm,
                                                             double gamma, double tol,
                                                             int* __restrict__ flags) {
    __shared__ double red[4][NTHREADS / 32];
    __shared__ double mean[4], tot[4], scale[4];
    __shared__ int bad;
    const int tx = threadIdx.x % TILE, ty = threadIdx.x / TILE;
    const int i = blockIdx.x * TILE + tx, j = blockIdx.y * TILE + ty;
    const bool in = i < mx && j < my;
    const long long p = (long long)j * mx + i;
    double d[4], q0[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        d[c] = in ? (double)r[p * rcp + c] / (double)norm[12 + c] : 0.0;
        q0[c] = in ? qs[c * fs + (long long)j * ld + i] : 0.0;
    }
    const int cnt = min(TILE, mx - blockIdx.x * TILE) * min(TILE, my - blockIdx.y * TILE);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto block_sum = [&](double v[4], double out[4]) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            double s = v[c];
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) red[c][warp] = s;
        }
        __syncthreads();
        if (threadIdx.x < 4) {
            double s = 0.0;
            for (int k = 0; k < NTHREADS / 32; ++k) s += red[threadIdx.x][k];
            out[threadIdx.x] = s;
        }
        __syncthreads();
    };
    block_sum(d, mean);
    double qn[4], aq[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const double dc = in ? d[c] - mean[c] / (double)cnt : 0.0;
        qn[c] = q0[c] + dc;
        aq[c] = in ? fabs(q0[c]) : 0.0;
    }
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    if (in) {
        const double ke = 0.5 * (qn[1] * qn[1] + qn[2] * qn[2]) / qn[0];
        const double pr = (gamma - 1.0) * (qn[3] - ke);
        if (!(qn[0] > 0.0) || !(pr > 0.0)) atomicOr(&bad, 1);
    }
    // conserved totals of the tile before and after
    double diff[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) diff[c] = in ? qn[c] - q0[c] : 0.0;
    block_sum(diff, tot);
    block_sum(aq, scale);
    if (threadIdx.x == 0) {
        for (int c = 0; c < 4; ++c)
            if (fabs(tot[c]) > tol * (scale[c] > 0.0 ? scale[c] : 1.0)) bad = 1;
    }
    __syncthreads();
    if (in && !bad)
        for (int c = 0; c < 4; ++c) qs[c * fs + (long long)j * ld + i] = qn[c];
    if (threadIdx.x == 0) flags[blockIdx.y * gridDim.x + blockIdx.x] = bad ? 0 : 1;
}

int grid_for(long long n) {
    long long b = (n + 255) / 256;
    return (int)(b < 592 ? (b > 0 ? b : 1) : 592);
}

// Tensor map of an NHWC BF16 activation tensor for the forward kernel's
// halo boxes: dims (C, W, H, N), box (8 channels, 10, 18, 1), zero fill
// outside the tensor.
PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult qr;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &qr) == cudaSuccess &&
            qr == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

int halo_map(CUtensorMap* map, const void* x, int n, int h, int w, int c) {
    auto fn = encode_tiled();
    if (!fn || (reinterpret_cast<uintptr_t>(x) & 15u)) return NN_E_CUDA;
    const cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)n};
    const cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)w * c * 2, (cuuint64_t)h * w * c * 2};
    const cuuint32_t box[4] = {8, (cuuint32_t)tc::HW, (cuuint32_t)tc::HH, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(x), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : NN_E_CUDA;
}

template <int CIN, int COUT, int ACT, bool OUTF32, bool SAVEZ>
int launch_fwd(const void* x, const void* w, const float* b, void* y, float* z, int n, int h,
               int wd, cudaStream_t s) {
    constexpr int SM = tcp::smem_bytes<CIN, COUT>();
    auto k = conv3x3_fwd_tcp<CIN, COUT, ACT, OUTF32, SAVEZ>;
    // One persistent CTA per SM (the driver's limit for a TMEM-allocating
    // kernel).  The function attributes and the resident CTA count are set up
    // once per device and instantiation (0 = not yet); a launch that fails
    // with a cached set-up (a new context after cudaDeviceReset has lost the
    // attributes) sets it up again and retries once.
    constexpr int MAXDEV = 64;
    static std::atomic<long long> resident[MAXDEV];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAXDEV) return NN_E_CUDA;
    auto setup = [&]() -> long long {
        int nsm = 0, per_sm = 0;
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, SM) != cudaSuccess ||
            cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared) != cudaSuccess ||
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, tcp::NTH, SM) != cudaSuccess || per_sm < 1)
            return 0;
        const long long cap = (long long)nsm * per_sm;
        resident[dev].store(cap, std::memory_order_release);
        return cap;
    };
    CUtensorMap map;
    if (halo_map(&map, x, n, h, wd, CIN) != 0) return NN_E_CUDA;
    const __nv_bfloat16* xb = static_cast<const __nv_bfloat16*>(x);
    const __nv_bfloat16* wb = static_cast<const __nv_bfloat16*>(w);
    const long long ntiles = (long long)n * (h / tc::TH) * (wd / tc::TW);
    const long long groups = (ntiles + tcp::NPIPE - 1) / tcp::NPIPE;
    long long cap = resident[dev].load(std::memory_order_acquire);
    const bool cached = cap != 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
        if (cap == 0 && (cap = setup()) == 0) return NN_E_CUDA;
        const int grid = (int)std::min<long long>(groups, cap);
        cudaError_t e;
#if CLAW_PDL
        // programmatic dependent launch: the CTAs' set-up overlaps the previous
        // launch's tail (the kernel waits before touching its operands)
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(tcp::NTH);
        cfg.dynamicSmemBytes = SM;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelEx(&cfg, k, xb, wb, b, y, z, n, h, wd, map);
#else
        k<<<grid, tcp::NTH, SM, s>>>(xb, wb, b, y, z, n, h, wd, map);
        e = cudaGetLastError();
#endif
        if (e == cudaSuccess) return 0;
        if (!cached || attempt == 1) return NN_E_CUDA;
        cap = 0;  // the cached set-up may be stale: redo it once
    }
    return NN_E_CUDA;
}

template <int CIN, int COUT>
int launch_wgrad(const void* x, const void* dz, float* partial, float* pdb, int n, int h, int wd,
                 cudaStream_t s) {
    constexpr int SM = wgrad_smem<CIN, COUT>();
    auto k = conv3x3_wgrad<CIN, COUT>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, SM) != cudaSuccess)
        return NN_E_CUDA;
    k<<<dim3(wd / TILE, h / TILE, n), NTHREADS, SM, s>>>(static_cast<const __nv_bfloat16*>(x),
                                                          static_cast<const __nv_bfloat16*>(dz),
                                                          partial, pdb, h, wd);
    return cudaGetLastError() == cudaSuccess ? 0 : NN_E_CUDA;
}

bool shape_ok(int n, int h, int w) { return n > 0 && h > 0 && w > 0 && h % TILE == 0 && w % TILE == 0; }

}  // namespace

extern "C" {

int nn_conv3x3_forward(const void* x, const void* w, const float* b, void* y, float* z, int n,
                       int h, int wd, int cin, int cout, int act, int out_f32, void* stream) {
    if (!x || !w || !b || !y || !shape_ok(n, h, wd)) return NN_E_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool save = z != nullptr;
    if (cin == 16 && cout == 32 && act == 1 && !out_f32)
        return save ? launch_fwd<16, 32, 1, false, true>(x, w, b, y, z, n, h, wd, s)
                    : launch_fwd<16, 32, 1, false, false>(x, w, b, y, z, n, h, wd, s);
    if (cin == 32 && cout == 32 && act == 1 && !out_f32)
        return save ? launch_fwd<32, 32, 1, false, true>(x, w, b, y, z, n, h, wd, s)
                    : launch_fwd<32, 32, 1, false, false>(x, w, b, y, z, n, h, wd, s);
    if (cin == 32 && cout == 16 && act == 0 && out_f32 && !save)
        return launch_fwd<32, 16, 0, true, false>(x, w, b, y, z, n, h, wd, s);
    // data gradients: no activation, BF16 out
    if (cin == 32 && cout == 32 && act == 0 && !out_f32 && !save)
        return launch_fwd<32, 32, 0, false, false>(x, w, b, y, z, n, h, wd, s);
    if (cin == 16 && cout == 32 && act == 0 && !out_f32 && !save)
        return launch_fwd<16, 32, 0, false, false>(x, w, b, y, z, n, h, wd, s);
    return NN_E_UNSUPPORTED;
}

int nn_conv3x3_wgrad(const void* x, const void* dz, float* partial, float* pdb, float* dw,
                     float* db, int n, int h, int wd, int cin, int cout, void* stream) {
    if (!x || !dz || !partial || !pdb || !dw || !db || !shape_ok(n, h, wd)) return NN_E_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc;
    if (cin == 16 && cout == 32) rc = launch_wgrad<16, 32>(x, dz, partial, pdb, n, h, wd, s);
    else if (cin == 32 && cout == 32) rc = launch_wgrad<32, 32>(x, dz, partial, pdb, n, h, wd, s);
    else if (cin == 32 && cout == 16) rc = launch_wgrad<32, 16>(x, dz, partial, pdb, n, h, wd, s);
    else return NN_E_UNSUPPORTED;
    if (rc) return rc;
    const long long nblk = (long long)n * (h / TILE) * (wd / TILE);
    const int len = cout * 9 * cin;
    reduce_tiles<<<(len + 255) / 256, 256, 0, s>>>(partial, dw, nblk, len);
    reduce_tiles<<<1, 256, 0, s>>>(pdb, db, nblk, cout);
    return cudaGetLastError() == cudaSuccess ? 0 : NN_E_CUDA;
}

int nn_device_error(int clear) {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_nn_err, sizeof(int)) != cudaSuccess) return NN_E_CUDA;
    if (clear) {
        const int zero = 0;
        if (cudaMemcpyToSymbol(g_nn_err, &zero, sizeof(int)) != cudaSuccess) return NN_E_CUDA;
    }
    return v;
}

int nn_flip_weights(const void* w, void* wt, int cout, int cin, void* stream) {
    if (!w || !wt || cout <= 0 || cin <= 0) return NN_E_INVALID;
    const int n = cout * 9 * cin;
    flip_weights<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(w), static_cast<__nv_bfloat16*>(wt), cout, cin);
    return cudaGetLastError() == cudaSuccess ? 0 : NN_E_CUDA;
}

int nn_gelu_backward(const void* dy, const float* z, void* dz, long long n, void* stream) {
    if (!dy || !z || !dz || n < 0) return NN_E_INVALID;
    gelu_backward<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(dy), z, static_cast<__nv_bfloat16*>(dz), n);
    return cudaGetLastError() == cudaSuccess ? 0 : NN_E_CUDA;
}

int nn_mse_grad(const float* pred, const float* target, void* dy, double* loss, long long npix,
                int cp, int nc, float delta, void* stream) {
    if (!pred || !target || !dy || !loss || npix <= 0 || nc > cp || delta < 0.f) return NN_E_INVALID;
    const float inv = 1.0f / (float)(npix * nc);
    mse_grad<<<grid_for(npix * cp), NTHREADS, 0, static_cast<cudaStream_t>(stream)>>>(
        pred, target, static_cast<__nv_bfloat16*>(dy), loss, npix, cp, nc, inv, delta);
    return cudaGetLastError() == cudaSuccess ? 0 : NN_E_CUDA;
}

int nn_adam(float* w, const float* g, float* m, float* v, void* w16, long long n, float lr,
            float b1, float b2, float eps, int step, void* stream) {
    if (!w || !g || !m || !v || n < 0 || step < 1) return NN_E_INVALID;
    float c1 = 1.f, c2 = 1.f;
    for (int k = 0; k < step && k < 100000; ++k) { c1 *= b1; c2 *= b2; }
    adam_step<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        w, g, m, v, static_cast<__nv_bfloat16*>(w16), n, lr, b1, b2, eps, 1.f - c1, 1.f - c2);
    return cudaGetLastError() == cudaSuccess ? 0 : NN_E_CUDA;
}

int nn_block_average(const double* fine, long long ldf, long long fsf, double* coarse, long long ldc,
                     long long fsc, int mxc, int myc, int r, int meqn, void* stream) {
    if (!fine || !coarse || r < 1 || mxc < 1 || myc < 1) return NN_E_INVALID;
    block_average<<<grid_for((long long)meqn * mxc * myc), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        fine, ldf, fsf, coarse, ldc, fsc, mxc, myc, r, meqn);
    return cudaGetLastError() == cudaSuccess ? 0 : NN_E_CUDA;
}

int nn_features(const double* q, const double* qs, long long ld, long long fs, int mx, int my,
                int img, const float* norm, void* x, void* stream) {
    if (!q || !qs || !norm || !x) return NN_E_INVALID;
    features<<<grid_for((long long)mx * my), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        q, qs, ld, fs, mx, my, img, norm, static_cast<__nv_bfloat16*>(x));
    return cudaGetLastError() == cudaSuccess ? 0 : NN_E_CUDA;
}

int nn_residual_target(const double* qf, const double* qs, long long ld, long long fs, int mx,
                       int my, int img, const float* norm, float* target, void* stream) {
    if (!qf || !qs || !norm || !target) return NN_E_INVALID;
    residual_target<<<grid_for((long long)mx * my), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        qf, qs, ld, fs, mx, my, img, norm, target);
    return cudaGetLastError() == cudaSuccess ? 0 : NN_E_CUDA;
}

int nn_apply_correction(double* qs, long long ld, long long fs, int mx, int my, const float* r,
                        int rcp, const float* norm, double gamma, double tol, int* flags,
                        void* stream) {
    if (!qs || !r || !norm || !flags || rcp < 4) return NN_E_INVALID;
    const dim3 grid((mx + TILE - 1) / TILE, (my + TILE - 1) / TILE);
    apply_correction<<<grid, NTHREADS, 0, static_cast<cudaStream_t>(stream)>>>(
        qs, ld, fs, mx, my, r, rcp, norm, gamma, tol, flags);
    return cudaGetLastError() == cudaSuccess ? 0 : NN_E_CUDA;
}

}  // extern "C"
