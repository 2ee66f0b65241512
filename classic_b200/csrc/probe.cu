// FP64 fused multiply-add throughput of the device: the second ceiling (beside
// HBM bandwidth) of the FP64 step kernels, which issue about 90 FP64
// operations per cell-update.  No counterpart in the reference.
#include <cuda_runtime.h>

#include <cstdio>

#include "../../include/claw_b200.h"
#include "common.cuh"

namespace clawb200 {
int fail(int code, const char* fmt, ...);
}

namespace {

constexpr int CHAINS = 8;  // independent FMA chains per thread hide the pipe latency

__global__ void __launch_bounds__(256) fp64_fma_probe(double* out, int iters, double a, double b) {
    double x[CHAINS];
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) x[k] = 1e-3 * (threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < CHAINS; ++k) x[k] = fma(x[k], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) s += x[k];
    out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void newton_check_kernel(const double* x, int n, double* r, double* q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        r[i] = clawb200::rcp_newton(x[i]);
        q[i] = clawb200::sqrt_newton(x[i]);
    }
}

}  // namespace

extern "C" int claw_check_newton(const double* x, int n, double* rcp, double* root) {
    if (!x || !rcp || !root || n < 1) return clawb200::fail(CLAW_E_INVALID, "bad arguments");
    double* d = nullptr;
    const size_t bytes = sizeof(double) * (size_t)n;
    if (cudaMalloc(&d, 3 * bytes) != cudaSuccess) return clawb200::fail(CLAW_E_CUDA, "cudaMalloc failed");
    int rc = 0;
    if (cudaMemcpy(d, x, bytes, cudaMemcpyHostToDevice) != cudaSuccess) rc = CLAW_E_CUDA;
    if (!rc) {
        newton_check_kernel<<<(n + 255) / 256, 256>>>(d, n, d + n, d + 2 * (size_t)n);
        if (cudaGetLastError() != cudaSuccess || cudaMemcpy(rcp, d + n, bytes, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(root, d + 2 * (size_t)n, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = CLAW_E_CUDA;
    }
    cudaFree(d);
    return rc ? clawb200::fail(rc, "claw_check_newton failed") : 0;
}

extern "C" int claw_probe_fp64(double* tflops, double* ms_best) {
    if (!tflops) return clawb200::fail(CLAW_E_INVALID, "null argument");
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return clawb200::fail(CLAW_E_CUDA, "device query failed");
    const int threads = 256, blocks = nsm * 8, iters = 1 << 14;
    double* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * (size_t)threads * blocks) != cudaSuccess)
        return clawb200::fail(CLAW_E_CUDA, "cudaMalloc failed");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int rc = 0;
    for (int rep = 0; rep < 6 && !rc; ++rep) {  // the first launch warms up
        cudaEventRecord(e0);
        fp64_fma_probe<<<blocks, threads>>>(out, iters, 0.9999999, 1e-7);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess) rc = clawb200::fail(CLAW_E_CUDA, "probe failed");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (rc) return rc;
    const double flops = 2.0 * CHAINS * (double)iters * threads * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    if (ms_best) *ms_best = best;
    return 0;
}
