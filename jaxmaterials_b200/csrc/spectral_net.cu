// Kernels of the spectral-convolution network that predicts warm-start strain fields
// (forward and backward): pointwise channel mixing with bias, optional residual input and
// GELU; per-mode complex channel mixing on the retained Fourier modes; Adam.
//
// Weights are BF16, activations and accumulation FP32. Layouts (C order):
//   real activations  [batch][channels][nv]
//   spectra           [batch][channels][nx][ny][nz/2+1] complex64 (R2C layout)
//   pointwise weight  [cout][cin] BF16, bias [cout] FP32
//   spectral weight   [modes][cin][cout][2] BF16 (re, im); mode m = (ix * my + iy) * mz + iz
//                     with kx = ix for ix < mx/2 and nx - mx + ix otherwise (likewise y),
//                     kz = iz.
// Every reduction over voxels is a per-block partial sum added atomically into the FP32
// gradient buffers, which the caller zeroes.
#include <cuda_bf16.h>

#include <cmath>
#include <cstdio>
#include <string>

#include "../../include/spectral_net.h"

namespace {

thread_local std::string g_err;

int fail(int code, const char* msg) {
  g_err = msg;
  return code;
}

__device__ __forceinline__ float bf(const __nv_bfloat16* w, int i) { return __bfloat162float(w[i]); }

// GELU (erf form) and its derivative.
__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}

constexpr int kPwThreads = 128;

template <int CIN, int COUT>
__global__ void __launch_bounds__(kPwThreads) pw_forward(long long nv, const float* __restrict__ x,
                                                         const __nv_bfloat16* __restrict__ w,
                                                         const float* __restrict__ bias,
                                                         const float* __restrict__ add,
                                                         float* __restrict__ pre,
                                                         float* __restrict__ y, int act) {
  __shared__ float ws[COUT * CIN];
  __shared__ float bs[COUT];
  for (int i = threadIdx.x; i < COUT * CIN; i += blockDim.x) ws[i] = bf(w, i);
  for (int i = threadIdx.x; i < COUT; i += blockDim.x) bs[i] = bias ? bias[i] : 0.f;
  __syncthreads();
  const int b = blockIdx.y;
  const float* xb = x + (size_t)b * CIN * nv;
  const size_t ob = (size_t)b * COUT * nv;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nv;
       v += (long long)gridDim.x * blockDim.x) {
    float xi[CIN];
#pragma unroll
    for (int i = 0; i < CIN; ++i) xi[i] = xb[(size_t)i * nv + v];
#pragma unroll 4
    for (int o = 0; o < COUT; ++o) {
      float a = bs[o];
#pragma unroll
      for (int i = 0; i < CIN; ++i) a = fmaf(ws[o * CIN + i], xi[i], a);
      const size_t k = ob + (size_t)o * nv + v;
      if (add) a += add[k];
      if (pre) pre[k] = a;
      y[k] = act ? gelu(a) : a;
    }
  }
}

// One tile = kPwThreads voxels, one per thread. dpre = dy * act'(pre) and x of the tile
// are staged in shared memory ([voxel][channel], channel fastest) so that each thread
// accumulates its (o, i) weight-gradient pairs over the tile.
template <int CIN, int COUT>
__global__ void __launch_bounds__(kPwThreads) pw_backward(
    long long nv, int batch, const float* __restrict__ x, const __nv_bfloat16* __restrict__ w,
    const float* __restrict__ pre, const float* __restrict__ dy, int act, float* __restrict__ dx,
    float* __restrict__ dpre_out, float* __restrict__ dw, float* __restrict__ db) {
  constexpr int NP = (COUT * CIN + kPwThreads - 1) / kPwThreads;  // pairs per thread
  __shared__ float ws[COUT * CIN];
  __shared__ float sd[kPwThreads][COUT + 1];
  __shared__ float sx[kPwThreads][CIN + 1];
  for (int i = threadIdx.x; i < COUT * CIN; i += blockDim.x) ws[i] = bf(w, i);
  float acc[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) acc[k] = 0.f;
  float bacc = 0.f;
  const long long tiles_per_inst = (nv + kPwThreads - 1) / kPwThreads;
  const long long tiles = tiles_per_inst * batch;
  for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int b = (int)(t / tiles_per_inst);
    const long long v = (t - (long long)b * tiles_per_inst) * kPwThreads + threadIdx.x;
    const bool in = v < nv;
    __syncthreads();  // the previous tile's shared data is no longer read
    float d[COUT];
#pragma unroll
    for (int o = 0; o < COUT; ++o) {
      float g = 0.f;
      if (in) {
        const size_t k = ((size_t)b * COUT + o) * nv + v;
        g = dy[k];
        if (act) g *= gelu_grad(pre[k]);
        if (dpre_out) dpre_out[k] = g;
      }
      d[o] = g;
      sd[threadIdx.x][o] = g;
    }
#pragma unroll
    for (int i = 0; i < CIN; ++i) sx[threadIdx.x][i] = in ? x[((size_t)b * CIN + i) * nv + v] : 0.f;
    if (dx && in) {
#pragma unroll 4
      for (int i = 0; i < CIN; ++i) {
        float a = 0.f;
#pragma unroll
        for (int o = 0; o < COUT; ++o) a = fmaf(ws[o * CIN + i], d[o], a);
        dx[((size_t)b * CIN + i) * nv + v] = a;
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const int p = threadIdx.x + k * kPwThreads;
      if (p < COUT * CIN) {
        const int o = p / CIN, i = p - o * CIN;
        float a = acc[k];
        for (int u = 0; u < kPwThreads; ++u) a = fmaf(sd[u][o], sx[u][i], a);
        acc[k] = a;
      }
    }
    if (threadIdx.x < COUT)
      for (int u = 0; u < kPwThreads; ++u) bacc += sd[u][threadIdx.x];
  }
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    const int p = threadIdx.x + k * kPwThreads;
    if (p < COUT * CIN) atomicAdd(dw + p, acc[k]);
  }
  if (db && threadIdx.x < COUT) atomicAdd(db + threadIdx.x, bacc);
}

struct ModeMap {
  int nx, ny, nzh, mx, my, mz;
  __device__ __forceinline__ size_t offset(int m) const {
    const int iz = m % mz, r = m / mz, iy = r % my, ix = r / my;
    const int kx = ix < mx / 2 ? ix : nx - mx + ix;
    const int ky = iy < my / 2 ? iy : ny - my + iy;
    return ((size_t)kx * ny + ky) * nzh + iz;
  }
};

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__device__ __forceinline__ float2 cjmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

constexpr int kMaxSpecBatch = 16;
constexpr int kMaxSpecChannels = 32;

// Block per retained mode: Y[b][o] = sum_i X[b][i] W[i][o].
__global__ void spec_forward(int batch, int cin, int cout, ModeMap mm, size_t plane,
                             const float2* __restrict__ xh, const __nv_bfloat16* __restrict__ w,
                             float2* __restrict__ yh) {
  extern __shared__ float2 sm[];
  float2* xs = sm;                         // [batch][cin]
  float2* wsm = sm + batch * cin;          // [cin][cout]
  const int m = blockIdx.x;
  const size_t off = mm.offset(m);
  for (int i = threadIdx.x; i < batch * cin; i += blockDim.x)
    xs[i] = xh[(size_t)i * plane + off];   // (b, c) row-major = b * cin + c
  const __nv_bfloat16* wm = w + (size_t)m * cin * cout * 2;
  for (int i = threadIdx.x; i < cin * cout; i += blockDim.x)
    wsm[i] = make_float2(bf(wm, 2 * i), bf(wm, 2 * i + 1));
  __syncthreads();
  for (int j = threadIdx.x; j < batch * cout; j += blockDim.x) {
    const int b = j / cout, o = j - b * cout;
    float2 a = make_float2(0.f, 0.f);
    for (int i = 0; i < cin; ++i) {
      const float2 p = cmulf(xs[b * cin + i], wsm[i * cout + o]);
      a.x += p.x;
      a.y += p.y;
    }
    yh[((size_t)b * cout + o) * plane + off] = a;
  }
}

// Block per retained mode: dX[b][i] = sum_o dY[b][o] conj(W[i][o]);
// dW[i][o] = sum_b conj(X[b][i]) dY[b][o] (FP32, [modes][cin][cout][2], overwritten).
__global__ void spec_backward(int batch, int cin, int cout, ModeMap mm, size_t plane,
                              const float2* __restrict__ xh, const __nv_bfloat16* __restrict__ w,
                              const float2* __restrict__ dyh, float2* __restrict__ dxh,
                              float2* __restrict__ dw) {
  extern __shared__ float2 sm[];
  float2* xs = sm;                        // [batch][cin]
  float2* ds = xs + batch * cin;          // [batch][cout]
  float2* wsm = ds + batch * cout;        // [cin][cout]
  const int m = blockIdx.x;
  const size_t off = mm.offset(m);
  for (int i = threadIdx.x; i < batch * cin; i += blockDim.x) xs[i] = xh[(size_t)i * plane + off];
  for (int i = threadIdx.x; i < batch * cout; i += blockDim.x) ds[i] = dyh[(size_t)i * plane + off];
  const __nv_bfloat16* wm = w + (size_t)m * cin * cout * 2;
  for (int i = threadIdx.x; i < cin * cout; i += blockDim.x)
    wsm[i] = make_float2(bf(wm, 2 * i), bf(wm, 2 * i + 1));
  __syncthreads();
  if (dxh)
    for (int j = threadIdx.x; j < batch * cin; j += blockDim.x) {
      const int b = j / cin, i = j - b * cin;
      float2 a = make_float2(0.f, 0.f);
      for (int o = 0; o < cout; ++o) {
        const float2 p = cjmulf(wsm[i * cout + o], ds[b * cout + o]);
        a.x += p.x;
        a.y += p.y;
      }
      dxh[((size_t)b * cin + i) * plane + off] = a;
    }
  float2* dwm = dw + (size_t)m * cin * cout;
  for (int j = threadIdx.x; j < cin * cout; j += blockDim.x) {
    const int i = j / cout, o = j - i * cout;
    float2 a = make_float2(0.f, 0.f);
    for (int b = 0; b < batch; ++b) {
      const float2 p = cjmulf(xs[b * cin + i], ds[b * cout + o]);
      a.x += p.x;
      a.y += p.y;
    }
    dwm[j] = a;
  }
}

__global__ void adam_kernel(long long n, float* __restrict__ p, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

int grid_for(long long work, int threads) {
  long long g = (work + threads - 1) / threads;
  return (int)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

template <int CIN, int COUT>
void pw_fwd_launch(int batch, long long nv, const float* x, const void* w, const float* bias,
                   const float* add, float* pre, float* y, int act, cudaStream_t s) {
  dim3 grid(grid_for(nv, kPwThreads), batch);
  pw_forward<CIN, COUT><<<grid, kPwThreads, 0, s>>>(nv, x, (const __nv_bfloat16*)w, bias, add,
                                                    pre, y, act);
}

template <int CIN, int COUT>
void pw_bwd_launch(int batch, long long nv, const float* x, const void* w, const float* pre,
                   const float* dy, int act, float* dx, float* dpre, float* dw, float* db,
                   cudaStream_t s) {
  const long long tiles = (nv + kPwThreads - 1) / kPwThreads * batch;
  const int grid = (int)(tiles < 148 * 8 ? tiles : 148 * 8);
  pw_backward<CIN, COUT><<<grid, kPwThreads, 0, s>>>(nv, batch, x, (const __nv_bfloat16*)w, pre,
                                                     dy, act, dx, dpre, dw, db);
}

// (cin, cout) pairs the network uses
#define LSN_PAIRS(X) X(2, 32) X(32, 32) X(32, 36) X(2, 4) X(4, 4) X(4, 6)

int spec_check(int batch, int cin, int cout, const int n[3], const int modes[3]) {
  if (batch < 1 || batch > kMaxSpecBatch || cin < 1 || cin > kMaxSpecChannels || cout < 1 ||
      cout > kMaxSpecChannels)
    return fail(-1, "spectral layer: batch or channels out of range");
  if (modes[0] < 1 || modes[1] < 1 || modes[2] < 1 || modes[0] > n[0] || modes[1] > n[1] ||
      modes[2] > n[2] / 2 + 1 || (modes[0] % 2) || (modes[1] % 2))
    return fail(-1, "spectral layer: retained modes do not fit the grid (mx, my even)");
  return 0;
}

}  // namespace

extern "C" {

const char* lsn_last_error(void) { return g_err.c_str(); }

int lsn_pointwise_forward(int batch, int cin, int cout, long long nv, const float* x,
                          const void* w, const float* bias, const float* add, float* pre,
                          float* y, int act, void* stream) {
  if (batch < 1 || nv < 1 || !x || !w || !y) return fail(-1, "lsn_pointwise_forward: bad argument");
  if (batch > 65535) return fail(-1, "lsn_pointwise_forward: batch above 65535");
  cudaStream_t s = (cudaStream_t)stream;
#define X(a, b) \
  if (cin == a && cout == b) { pw_fwd_launch<a, b>(batch, nv, x, w, bias, add, pre, y, act, s); return 0; }
  LSN_PAIRS(X)
#undef X
  return fail(-1, "lsn_pointwise_forward: unsupported channel pair");
}

int lsn_pointwise_backward(int batch, int cin, int cout, long long nv, const float* x,
                           const void* w, const float* pre, const float* dy, int act, float* dx,
                           float* dpre, float* dw, float* db, void* stream) {
  if (batch < 1 || nv < 1 || !x || !w || !dy || !dw || (act && !pre))
    return fail(-1, "lsn_pointwise_backward: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
#define X(a, b) \
  if (cin == a && cout == b) { pw_bwd_launch<a, b>(batch, nv, x, w, pre, dy, act, dx, dpre, dw, db, s); return 0; }
  LSN_PAIRS(X)
#undef X
  return fail(-1, "lsn_pointwise_backward: unsupported channel pair");
}

int lsn_spectral_forward(int batch, int cin, int cout, const int n[3], const int modes[3],
                         const void* xh, const void* w, void* yh, void* stream) {
  if (!n || !modes || !xh || !w || !yh) return fail(-1, "lsn_spectral_forward: null argument");
  if (int rc = spec_check(batch, cin, cout, n, modes)) return rc;
  const ModeMap mm{n[0], n[1], n[2] / 2 + 1, modes[0], modes[1], modes[2]};
  const size_t plane = (size_t)n[0] * n[1] * (n[2] / 2 + 1);
  const size_t smem = sizeof(float2) * (size_t)(batch * cin + cin * cout);
  const int nm = modes[0] * modes[1] * modes[2];
  spec_forward<<<nm, 256, smem, (cudaStream_t)stream>>>(batch, cin, cout, mm, plane,
                                                         (const float2*)xh,
                                                         (const __nv_bfloat16*)w, (float2*)yh);
  return 0;
}

int lsn_spectral_backward(int batch, int cin, int cout, const int n[3], const int modes[3],
                          const void* xh, const void* w, const void* dyh, void* dxh, float* dw,
                          void* stream) {
  if (!n || !modes || !xh || !w || !dyh || !dw) return fail(-1, "lsn_spectral_backward: null argument");
  if (int rc = spec_check(batch, cin, cout, n, modes)) return rc;
  const ModeMap mm{n[0], n[1], n[2] / 2 + 1, modes[0], modes[1], modes[2]};
  const size_t plane = (size_t)n[0] * n[1] * (n[2] / 2 + 1);
  const size_t smem = sizeof(float2) * (size_t)(batch * cin + batch * cout + cin * cout);
  const int nm = modes[0] * modes[1] * modes[2];
  spec_backward<<<nm, 256, smem, (cudaStream_t)stream>>>(
      batch, cin, cout, mm, plane, (const float2*)xh, (const __nv_bfloat16*)w,
      (const float2*)dyh, (float2*)dxh, (float2*)dw);
  return 0;
}

int lsn_adam(long long n, float* param, const float* grad, float* m, float* v, float lr,
             float beta1, float beta2, float eps, int step, void* stream) {
  if (n < 0 || !param || !grad || !m || !v || step < 1) return fail(-1, "lsn_adam: bad argument");
  if (n == 0) return 0;
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  adam_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, param, grad, m, v, lr, beta1,
                                                                  beta2, eps, c1, c2);
  return 0;
}

}  // extern "C"
