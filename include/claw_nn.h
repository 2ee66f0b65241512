/*
 * claw_nn.h — C ABI of the learned coarse-grid corrector's device kernels
 * (classic_b200/csrc/nn.cu, part of libclawb200.so).  No counterpart in the
 * reference: the corrector is this library's addition on top of the 2D Euler
 * step (include/claw_b200.h).
 *
 * Tensors are device pointers.  Activations are NHWC BF16 [n][h][w][c] with
 * h, w multiples of 16 and c padded (16 or 32); weights are BF16
 * [cout][9][cin] with tap = 3*ky + kx for the offset (ky-1, kx-1); biases,
 * pre-activations, gradients and optimiser state are FP32.  "Same" 3x3
 * convolutions with zero padding; products on the tensor cores with FP32
 * accumulation.  stream is a cudaStream_t (NULL = default stream); every
 * call is asynchronous on it.
 */
#ifndef CLAW_NN_H
#define CLAW_NN_H

#ifdef __cplusplus
extern "C" {
#endif

enum nn_error { NN_E_INVALID = -1, NN_E_CUDA = -2, NN_E_UNSUPPORTED = -3 };

/* y = act(conv3x3(x, w) + b); act 0 = identity, 1 = GELU.  z (optional) keeps
 * the FP32 pre-activation for the backward pass.  (cin, cout, act, out_f32):
 * (16,32,1,0) (32,32,1,0) (32,16,0,1), and the data-gradient shapes
 * (32,32,0,0) (16,32,0,0).  Runs as tcgen05.mma (M128 x N=cout x K16 BF16
 * products, FP32 accumulator in tensor memory) on 16 x 8 pixel tiles. */
int nn_conv3x3_forward(const void* x, const void* w, const float* b, void* y, float* z, int n,
                       int h, int wd, int cin, int cout, int act, int out_f32, void* stream);
/* dw[cout][9][cin] = sum_p dz[p][co] x[p + off][ci], db[co] = sum_p dz[p][co];
 * partial / pdb: scratch of n*(h/16)*(wd/16) blocks x (cout*9*cin) / cout floats. */
int nn_conv3x3_wgrad(const void* x, const void* dz, float* partial, float* pdb, float* dw,
                     float* db, int n, int h, int wd, int cin, int cout, void* stream);
/* Device-side error flags of these kernels (bit 0: a wait on the tensor-core
 * accumulator gave up, and that launch left its output unwritten); clear != 0
 * resets them.  Synchronises with the device. */
int nn_device_error(int clear);
/* wt[ci][tap][co] = w[co][8-tap][ci]: the data gradient dx = conv3x3(dz, wt). */
int nn_flip_weights(const void* w, void* wt, int cout, int cin, void* stream);
/* dz = dy * GELU'(z), n elements. */
int nn_gelu_backward(const void* dy, const float* z, void* dz, long long n, void* stream);
/* Mean squared error (delta = 0) or Huber loss (quadratic within delta,
 * linear beyond) over the first nc of cp channels of pred [npix][cp] against
 * target [npix][nc]: dy = d(loss)/d(pred) (BF16 [npix][cp]); the summed loss
 * is added to *loss (FP64, device).  A NaN target value masks
 * that entry out (no loss, zero gradient); count is npix * nc. */
int nn_mse_grad(const float* pred, const float* target, void* dy, double* loss, long long npix,
                int cp, int nc, float delta, void* stream);
/* One Adam step on FP32 weights (step >= 1); w16 (optional) receives the BF16 copy. */
int nn_adam(float* w, const float* g, float* m, float* v, void* w16, long long n, float lr,
            float b1, float b2, float eps, int step, void* stream);

/* Solver glue on FP64 SoA fields [meqn][my][ld] (field pitch fs):
 * coarse = r x r block average of fine. */
int nn_block_average(const double* fine, long long ldf, long long fsf, double* coarse, long long ldc,
                     long long fsc, int mxc, int myc, int r, int meqn, void* stream);
/* x[img][p][16]: (q - norm[c]) * norm[4+c] for c < 4, (qs - q) * norm[8+c]
 * for the next 4, zeros after; q before and qs after the plain step. */
int nn_features(const double* q, const double* qs, long long ld, long long fs, int mx, int my,
                int img, const float* norm, void* x, void* stream);
/* target[img][p][4] = (qf - qs) * norm[12+c]: qf the block-averaged fine
 * solution, qs the plain coarse step. */
int nn_residual_target(const double* qf, const double* qs, long long ld, long long fs, int mx,
                       int my, int img, const float* norm, float* target, void* stream);
/* qs += r / norm[12+c] per 16x16 tile, minus the tile mean of the residual
 * (conserved totals unchanged); a tile whose corrected density or pressure is
 * not positive, or whose totals move by more than tol relative, keeps the
 * plain step.  flags[tile] = 1 corrected / 0 plain. */
int nn_apply_correction(double* qs, long long ld, long long fs, int mx, int my, const float* r,
                        int rcp, const float* norm, double gamma, double tol, int* flags,
                        void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CLAW_NN_H */
