/* C ABI of the warm-start network kernels in liblippmannschwinger.so (no reference
 * counterpart: the reference has no learned component). A spectral-convolution network
 * maps the Lame fields of a microstructure to the six strain fields of its unit load
 * cases; these kernels are its forward and backward building blocks. All pointers are
 * device pointers; every call is asynchronous on `stream` (a cudaStream_t as void*).
 *
 * Layouts (C order): real activations [batch][channels][nv] float; spectra
 * [batch][channels][nx][ny][nz/2+1] complex64 (interleaved re, im); pointwise weights
 * [cout][cin] bf16 with bias [cout] float; spectral weights [modes][cin][cout][2] bf16,
 * mode m = (ix * my + iy) * mz + iz, kx = ix for ix < mx/2 else nx - mx + ix (likewise
 * ky), kz = iz. Gradient buffers are float and accumulate (the caller zeroes them), except
 * the spectral weight gradient, which is overwritten.
 * Return value 0 on success, negative on a bad argument (lsn_last_error()). */
#ifndef SPECTRAL_NET_B200_H
#define SPECTRAL_NET_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* y = act(W x + bias + add); pre (optional) receives the pre-activation.
 * act: 0 identity, 1 GELU (erf form). Channel pairs (cin, cout): (2,32), (32,32),
 * (32,36), (2,4), (4,4), (4,6). add and bias may be NULL. The pairs with cin = 32 run on
 * the tensor cores when nv is a multiple of 16 (x rounded to bf16 for the products, FP32
 * accumulation); the others, and any nv, on FP32 FMA kernels. */
int lsn_pointwise_forward(int batch, int cin, int cout, long long nv, const float *x,
                          const void *w_bf16, const float *bias, const float *add, float *pre,
                          float *y, int act, void *stream);

/* Backward of lsn_pointwise_forward for the output gradient dy: dpre = dy * act'(pre)
 * (written when dpre != NULL; it is also the gradient of `add`), dx = W^T dpre (when
 * dx != NULL), dw += dpre x^T summed over voxels and batch, db += sum of dpre. */
int lsn_pointwise_backward(int batch, int cin, int cout, long long nv, const float *x,
                           const void *w_bf16, const float *pre, const float *dy, int act,
                           float *dx, float *dpre, float *dw, float *db, void *stream);

/* Per-mode channel mixing on the retained modes: yh[b][o][k] = sum_i xh[b][i][k] W[k][i][o]
 * for the modes k of `modes` (mx, my even); the other entries of yh are not written.
 * n = grid (nx, ny, nz); batch <= 16; cin, cout <= 32. */
int lsn_spectral_forward(int batch, int cin, int cout, const int n[3], const int modes[3],
                         const void *xh, const void *w_bf16, void *yh, void *stream);

/* Backward: dxh[b][i][k] = sum_o dyh[b][o][k] conj(W[k][i][o]) at the retained modes
 * (dxh optional; other entries not written); dw[k][i][o] = sum_b conj(xh[b][i][k])
 * dyh[b][o][k] as float [modes][cin][cout][2], overwritten. */
int lsn_spectral_backward(int batch, int cin, int cout, const int n[3], const int modes[3],
                          const void *xh, const void *w_bf16, const void *dyh, void *dxh,
                          float *dw, void *stream);

/* Truncated transforms between `fields` real fields f [fields][nx][ny][nz] float and their
 * retained modes X [fields][mx][my][mz] complex64 (the dense mode layout above, i.e.
 * lsn_spectral_forward/backward with n = (mx, my, 2 (mz - 1))):
 *   forward:  X[m] = scale w(kz) sum_v f[v] exp(-2 pi i k.v / n)
 *   inverse:  f[v] = scale Re sum_m w(kz) X[m] exp(+2 pi i k.v / n)
 * with w(kz) = w_int for 0 < kz < nz/2, else 1. forward(1, 1) is numpy's rfftn at the
 * retained modes, inverse(1/(nx ny nz), 2) numpy's irfftn of the zero-padded half spectrum;
 * as real-linear maps forward(1, 1) and inverse(1, 1) are each other's transposes, and so
 * are inverse(s, w) and forward(s, w), which gives the backward passes. work: device
 * complex64 [fields][nx][my][mz]. fields <= 65535, ny nz <= 16384. */
int lsn_truncated_forward(int fields, const int n[3], const int modes[3], const float *f,
                          void *work, void *out, float scale, float w_int, void *stream);
int lsn_truncated_inverse(int fields, const int n[3], const int modes[3], const void *x,
                          void *work, float *f, float scale, float w_int, void *stream);

/* Adam step `step` (>= 1, bias-corrected) on n float parameters. */
int lsn_adam(long long n, float *param, const float *grad, float *m, float *v, float lr,
             float beta1, float beta2, float eps, int step, void *stream);

const char *lsn_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* SPECTRAL_NET_B200_H */
