// Kernels of the spectral-convolution network that predicts warm-start strain fields
// (forward and backward): pointwise channel mixing with bias, optional residual input and
// GELU; per-mode complex channel mixing on the retained Fourier modes; Adam.
//
// Weights are BF16, accumulation FP32; activations FP32, rounded to BF16 where a layer runs
// on the tensor cores (a multiple of 16 input channels: mma.sync m16n8k16, see
// pw_forward_tc / pw_backward_tc). Layouts (C order):
//   real activations  [batch][channels][nv]
//   spectra           [batch][channels][nx][ny][nz/2+1] complex64 (R2C layout)
//   pointwise weight  [cout][cin] BF16, bias [cout] FP32
//   spectral weight   [modes][cin][cout][2] BF16 (re, im); mode m = (ix * my + iy) * mz + iz
//                     with kx = ix for ix < mx/2 and nx - mx + ix otherwise (likewise y),
//                     kz = iz.
// Every reduction over voxels is a per-block partial sum added atomically into the FP32
// gradient buffers, which the caller zeroes.
#include <cuda_bf16.h>

#include <algorithm>
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

// ---- tensor-core pointwise layers (cin a multiple of 16; cout padded to 8 or 16)
//
// One warp owns a tile of 16 voxels of one sample; a voxel tile times the weight matrix is
// a chain of mma.sync m16n8k16 BF16 products with FP32 accumulation (the weights are
// BF16; the activations enter as BF16, rounded once when they are loaded). Fragments are
// loaded straight from the [batch][channel][nv] layout: for a fixed channel the eight
// lanes of a group read eight consecutive voxels (32-byte segments), so no shared-memory
// staging is needed; the weight fragments stay in registers for the whole kernel.
// Backward: per 16-voxel tile, dpre = dy * act'(pre) is formed once in the layout of the
// weight-gradient product (rows = output channels, k = voxels); movmatrix transposes its
// 8x8 blocks into the layout of the input-gradient product (rows = voxels, k = output
// channels). dW and db are accumulated in registers over the warp's tiles, summed over
// the block in shared memory and added atomically into the caller's zeroed buffers.
__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const unsigned*>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], unsigned a0, unsigned a1, unsigned a2,
                                         unsigned a3, unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
      "{%8, %9}, {%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Transpose of an 8x8 block of 16-bit values held one row pair per lane (fragment layout).
__device__ __forceinline__ unsigned movmatrix_t(unsigned a) {
  unsigned r;
  asm volatile("movmatrix.sync.aligned.m8n8.trans.b16 %0, %1;" : "=r"(r) : "r"(a));
  return r;
}

constexpr int kTcWarps = 4;

template <int CIN, int COUT>
__global__ void __launch_bounds__(32 * kTcWarps) pw_forward_tc(long long nv, int batch,
                                                               const float* __restrict__ x,
                                                               const __nv_bfloat16* __restrict__ w,
                                                               const float* __restrict__ bias,
                                                               const float* __restrict__ add,
                                                               float* __restrict__ pre,
                                                               float* __restrict__ y, int act) {
  static_assert(CIN % 16 == 0, "k steps of 16 input channels");
  constexpr int KS = CIN / 16, NT = (COUT + 7) / 8;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  unsigned wb[KS][NT][2];
  float bs[NT][2];
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    const int o = nt * 8 + g;
#pragma unroll
    for (int s = 0; s < KS; ++s) {
      const int k0 = s * 16 + 2 * t;
      if (o < COUT) {
        wb[s][nt][0] = pack_bf16(bf(w, o * CIN + k0), bf(w, o * CIN + k0 + 1));
        wb[s][nt][1] = pack_bf16(bf(w, o * CIN + k0 + 8), bf(w, o * CIN + k0 + 9));
      } else {
        wb[s][nt][0] = wb[s][nt][1] = 0u;
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int oc = nt * 8 + 2 * t + h;
      bs[nt][h] = (bias && oc < COUT) ? bias[oc] : 0.f;
    }
  }
  const long long tpi = nv / 16, tiles = tpi * batch;
  for (long long tile = (long long)blockIdx.x * kTcWarps + warp; tile < tiles;
       tile += (long long)gridDim.x * kTcWarps) {
    const int b = (int)(tile / tpi);
    const long long v0 = (tile - (long long)b * tpi) * 16;
    const float* xb = x + (size_t)b * CIN * nv + v0;
    unsigned a[KS][4];
#pragma unroll
    for (int s = 0; s < KS; ++s) {
      const float* c0 = xb + (size_t)(s * 16 + 2 * t) * nv;
      a[s][0] = pack_bf16(c0[g], c0[nv + g]);
      a[s][1] = pack_bf16(c0[g + 8], c0[nv + g + 8]);
      a[s][2] = pack_bf16(c0[8 * nv + g], c0[9 * nv + g]);
      a[s][3] = pack_bf16(c0[8 * nv + g + 8], c0[9 * nv + g + 8]);
    }
    const size_t ob = (size_t)b * COUT * nv + v0;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      float d[4] = {bs[nt][0], bs[nt][1], bs[nt][0], bs[nt][1]};
#pragma unroll
      for (int s = 0; s < KS; ++s) mma_bf16(d, a[s][0], a[s][1], a[s][2], a[s][3], wb[s][nt][0], wb[s][nt][1]);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int o = nt * 8 + 2 * t + (e & 1);
        if (o >= COUT) continue;
        const size_t k = ob + (size_t)o * nv + g + (e >> 1) * 8;
        float val = d[e];
        if (add) val += add[k];
        if (pre) pre[k] = val;
        y[k] = act ? gelu(val) : val;
      }
    }
  }
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(32 * kTcWarps) pw_backward_tc(
    long long nv, int batch, const float* __restrict__ x, const __nv_bfloat16* __restrict__ w,
    const float* __restrict__ pre, const float* __restrict__ dy, int act, float* __restrict__ dx,
    float* __restrict__ dpre_out, float* __restrict__ dw, float* __restrict__ db) {
  static_assert(CIN % 16 == 0, "k steps of 16 input channels");
  constexpr int MT = (COUT + 15) / 16;  // 16-row tiles of output channels (dW rows, dx k steps)
  constexpr int NT = CIN / 8;           // 8-column tiles of input channels
  __shared__ float red[COUT * CIN + COUT];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  for (int i = threadIdx.x; i < COUT * CIN + COUT; i += blockDim.x) red[i] = 0.f;
  // dx = W^T dpre: B[k = o][n = i] = W[o][i]
  unsigned wf[MT][NT][2];
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const int i = nt * 8 + g, o0 = mt * 16 + 2 * t;
      auto W = [&](int o) { return o < COUT ? bf(w, o * CIN + i) : 0.f; };
      wf[mt][nt][0] = pack_bf16(W(o0), W(o0 + 1));
      wf[mt][nt][1] = pack_bf16(W(o0 + 8), W(o0 + 9));
    }
  float acc[MT][NT][4];
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[mt][nt][e] = 0.f;
  float bacc[MT][2] = {};
  const long long tpi = nv / 16, tiles = tpi * batch;
  for (long long tile = (long long)blockIdx.x * kTcWarps + warp; tile < tiles;
       tile += (long long)gridDim.x * kTcWarps) {
    const int b = (int)(tile / tpi);
    const long long v0 = (tile - (long long)b * tpi) * 16;
    // dpre in the dW layout: rows o = mt*16 + g (+8), k = voxels 2t, 2t+1 (+8)
    unsigned pa[MT][4];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int o = mt * 16 + g + 8 * r;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float2 d2 = make_float2(0.f, 0.f);
          if (o < COUT) {
            const size_t k = ((size_t)b * COUT + o) * nv + v0 + 2 * t + 8 * h;
            d2 = *reinterpret_cast<const float2*>(dy + k);
            if (act) {
              const float2 p2 = *reinterpret_cast<const float2*>(pre + k);
              d2.x *= gelu_grad(p2.x);
              d2.y *= gelu_grad(p2.y);
            }
            if (dpre_out) *reinterpret_cast<float2*>(dpre_out + k) = d2;
          }
          bacc[mt][r] += d2.x + d2.y;
          pa[mt][r + 2 * h] = pack_bf16(d2.x, d2.y);
        }
      }
    }
    // dW += dpre x^T: B[k = v][n = i] = x[i][v]
    const float* xb = x + (size_t)b * CIN * nv + v0;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const float* xi = xb + (size_t)(nt * 8 + g) * nv;
      const float2 p0 = *reinterpret_cast<const float2*>(xi + 2 * t);
      const float2 p1 = *reinterpret_cast<const float2*>(xi + 2 * t + 8);
      const unsigned b0 = pack_bf16(p0.x, p0.y), b1 = pack_bf16(p1.x, p1.y);
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) mma_bf16(acc[mt][nt], pa[mt][0], pa[mt][1], pa[mt][2], pa[mt][3], b0, b1);
    }
    if (!dx) continue;
    // dx = dpre^T W in the layout rows = voxels, k = o: the 8x8 blocks of pa transposed
    float dd[NT][4];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) dd[nt][e] = 0.f;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
      const unsigned q0 = movmatrix_t(pa[mt][0]), q1 = movmatrix_t(pa[mt][2]);
      const unsigned q2 = movmatrix_t(pa[mt][1]), q3 = movmatrix_t(pa[mt][3]);
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) mma_bf16(dd[nt], q0, q1, q2, q3, wf[mt][nt][0], wf[mt][nt][1]);
    }
    float* dxb = dx + (size_t)b * CIN * nv + v0;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) dxb[(size_t)(nt * 8 + 2 * t + (e & 1)) * nv + g + (e >> 1) * 8] = dd[nt][e];
  }
  __syncthreads();  // (red zeroed)
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int o = mt * 16 + g + (e >> 1) * 8, i = nt * 8 + 2 * t + (e & 1);
        if (o < COUT) atomicAdd(&red[o * CIN + i], acc[mt][nt][e]);
      }
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int o = mt * 16 + g + 8 * r;
      if (o < COUT) atomicAdd(&red[COUT * CIN + o], bacc[mt][r]);
    }
  __syncthreads();
  for (int i = threadIdx.x; i < COUT * CIN; i += blockDim.x) atomicAdd(dw + i, red[i]);
  if (db)
    for (int i = threadIdx.x; i < COUT; i += blockDim.x) atomicAdd(db + i, red[COUT * CIN + i]);
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

// Layers with a multiple of 16 input channels over whole 16-voxel tiles run on the tensor
// cores (activations rounded to BF16 as they enter the products); the others on the FP32
// FMA kernels.
template <int CIN>
bool use_tc(long long nv) { return CIN % 16 == 0 && nv % 16 == 0; }

template <int CIN, int COUT>
void pw_fwd_launch(int batch, long long nv, const float* x, const void* w, const float* bias,
                   const float* add, float* pre, float* y, int act, cudaStream_t s) {
  if constexpr (CIN % 16 == 0) {
    if (use_tc<CIN>(nv)) {
      const long long blocks = (nv / 16 * batch + kTcWarps - 1) / kTcWarps;
      const int grid = (int)(blocks < 148 * 8 ? blocks : 148 * 8);
      pw_forward_tc<CIN, COUT><<<grid, 32 * kTcWarps, 0, s>>>(nv, batch, x, (const __nv_bfloat16*)w,
                                                              bias, add, pre, y, act);
      return;
    }
  }
  dim3 grid(grid_for(nv, kPwThreads), batch);
  pw_forward<CIN, COUT><<<grid, kPwThreads, 0, s>>>(nv, x, (const __nv_bfloat16*)w, bias, add,
                                                    pre, y, act);
}

template <int CIN, int COUT>
void pw_bwd_launch(int batch, long long nv, const float* x, const void* w, const float* pre,
                   const float* dy, int act, float* dx, float* dpre, float* dw, float* db,
                   cudaStream_t s) {
  if constexpr (CIN % 16 == 0) {
    if (use_tc<CIN>(nv)) {
      const long long blocks = (nv / 16 * batch + kTcWarps - 1) / kTcWarps;
      const int grid = (int)(blocks < 148 * 4 ? blocks : 148 * 4);
      pw_backward_tc<CIN, COUT><<<grid, 32 * kTcWarps, 0, s>>>(nv, batch, x, (const __nv_bfloat16*)w, pre,
                                                               dy, act, dx, dpre, dw, db);
      return;
    }
  }
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

// ---- truncated transforms between the real fields and the retained modes
//
// The spectral layers only read and write the retained modes kx(ix) (ix < mx: the lowest
// |kx|, mx even), ky(iy) likewise, kz = iz < mz, so instead of full 3-D FFTs the network
// transforms with direct sums over those modes, dense [bc][mx][my][mz] complex:
//   fwd:  X[m] = scale w(iz) sum_{x,y,z} f[x][y][z] exp(-2 pi i (kx x/nx + ky y/ny + iz z/nz))
//   inv:  f[x][y][z] = scale Re sum_m w(iz) Y[m] exp(+2 pi i (...))
// with w(iz) = w_int for 0 < iz < nz/2 and 1 for iz = 0 and the z Nyquist index. fwd with
// (1, 1) is numpy's rfftn restricted to the retained modes; inv with (1/N, 2) is numpy's
// irfftn of the zero-padded half spectrum (for iz = 0 and the Nyquist index the sine of
// the z phase vanishes at every voxel, so the imaginary parts irfftn drops contribute
// nothing); and, as real-linear maps, the transpose of fwd(1, 1) is inv(1, 1) and the
// transpose of inv(s, w) is fwd(s, w): the backward passes use the same two kernels.
// Each transform is two kernels: the (y, z) part per x-plane in shared memory (a block per
// field walks every kTrPlaneBlocks-th x-plane, its twiddle tables built once), and the x
// part per retained (ky, kz) column.
constexpr int kTrThreads = 256;
constexpr size_t kTrMaxPlane = 64 * 1024;  // bytes of one x-plane of floats (ny nz <= 16384)
constexpr int kTrMaxModes = 64;            // mx, my, mz (the twiddle rows in shared memory)
constexpr int kTrPlaneBlocks = 8;          // blocks per field of the (y, z) parts (x-planes looped)

__device__ __forceinline__ int kmode(int i, int m, int n) { return i < m / 2 ? i : n - m + i; }

__device__ __forceinline__ float zweight(int iz, int nz, float w_int) {
  return (iz == 0 || 2 * iz == nz) ? 1.f : w_int;
}

// Per-block twiddle tables in shared memory: base[j] = (cos, sin)(2 pi j / n) for j < n, and
// the rows tab[i][j] = base[(k(i) j) mod n] that a stage reads, laid out so that the lanes
// of a warp read one entry (broadcast) or consecutive entries.
__device__ __forceinline__ void base_table(float2* base, int n) {
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    float sn, cs;
    sincospif(2.f * (float)j / (float)n, &sn, &cs);
    base[j] = make_float2(cs, sn);
  }
}

// Tensor-core stage of the inverse (y, z) part: real products on mma.sync m16n8k8 TF32 with the
// three-term split a b = a_hi b_hi + a_hi b_lo + a_lo b_hi (hi = a rounded to TF32,
// lo = the rest rounded to TF32), which keeps the FP32 accuracy of the direct sums.
__device__ __forceinline__ void split_tf32(float x, unsigned& hi, unsigned& lo) {
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
  const float r = x - __uint_as_float(hi);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
      "{%8, %9}, {%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// D[m][n] = sum_k A[m][k] B[k][n] over one 16 x 8 output tile at (m0, n0) (A row-major with
// row stride lda, B row-major [k][n] with row stride ldb, K a multiple of 8); the warp's
// fragment of D is returned in d (rows m0 + g, m0 + g + 8; columns n0 + 2t, n0 + 2t + 1).
__device__ __forceinline__ void tile_product_tf32(const float* A, int lda, const float* B, int ldb, int K,
                                                  int m0, int n0, float (&d)[4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  d[0] = d[1] = d[2] = d[3] = 0.f;
  for (int k0 = 0; k0 < K; k0 += 8) {
    unsigned ah[4], al[4], bh0, bl0, bh1, bl1;
    split_tf32(A[(m0 + g) * lda + k0 + t], ah[0], al[0]);
    split_tf32(A[(m0 + g + 8) * lda + k0 + t], ah[1], al[1]);
    split_tf32(A[(m0 + g) * lda + k0 + t + 4], ah[2], al[2]);
    split_tf32(A[(m0 + g + 8) * lda + k0 + t + 4], ah[3], al[3]);
    split_tf32(B[(k0 + t) * ldb + n0 + g], bh0, bl0);
    split_tf32(B[(k0 + t + 4) * ldb + n0 + g], bh1, bl1);
    mma_tf32(d, al, bh0, bh1);
    mma_tf32(d, ah, bl0, bl1);
    mma_tf32(d, ah, bh0, bh1);
  }
}

// Row stride (floats) of a shared-memory matrix with n columns read as B fragments (lanes
// (t, g) at rows t, columns g): rows four or eight banks apart, so the 32 lanes are distinct.
__host__ __device__ __forceinline__ int frag_ld(int n) { return n % 16 == 8 ? n : n + 8; }
__host__ __device__ __forceinline__ int pad8(int n) { return (n + 7) / 8 * 8; }

// fwd, (y, z) part: P[bc][x][iy][iz] = sum_{y,z} f[bc][x][y][z] e^{-i(ky y + iz z)}.
// Stage 1: thread (y, group) accumulates the iz of its group over z (plane rows padded by
// one float so that the lanes, consecutive y, hit distinct banks; the twiddle row of an iz
// is the same for the whole warp). Stage 2: thread (iy, iz) over y.
__global__ void __launch_bounds__(kTrThreads) trunc_fwd_yz(int nx, int ny, int nz, int my, int mz,
                                                           const float* __restrict__ f,
                                                           float2* __restrict__ p) {
  extern __shared__ __align__(16) unsigned char trraw[];
  const int ld = nz + 1;
  float2* tz = reinterpret_cast<float2*>(trraw);  // [mz][nz]
  float2* ty = tz + mz * nz;                      // [my][ny]
  float2* zt = ty + my * ny;                      // [ny][mz]
  float2* base = zt + ny * mz;                    // [max(ny, nz)]
  float* plane = reinterpret_cast<float*>(base + (ny > nz ? ny : nz));  // [ny][nz + 1]
  const size_t bc = blockIdx.y;
  base_table(base, nz);
  __syncthreads();
  for (int i = threadIdx.x; i < mz * nz; i += blockDim.x) {
    const int iz = i / nz, z = i - iz * nz;
    tz[i] = base[(int)((long long)iz * z % nz)];
  }
  __syncthreads();
  base_table(base, ny);
  __syncthreads();
  for (int i = threadIdx.x; i < my * ny; i += blockDim.x) {
    const int iy = i / ny, y = i - iy * ny;
    ty[i] = base[(int)((long long)kmode(iy, my, ny) * y % ny)];
  }
  // the block's x-planes (the tables above are built once per block)
  for (int x = blockIdx.x; x < nx; x += gridDim.x) {
  __syncthreads();  // (tables built; the previous plane's stage 2 done)
  const float* src = f + (bc * nx + x) * (size_t)ny * nz;
  for (int i = threadIdx.x; i < ny * nz; i += blockDim.x) plane[(i / nz) * ld + i % nz] = src[i];
  __syncthreads();
  // stage 1
  const int groups = ny >= (int)blockDim.x ? 1 : (int)blockDim.x / ny;
  for (int o = threadIdx.x; o < ny * groups; o += blockDim.x) {
    const int y = o % ny, grp = o / ny;
    for (int iz0 = grp; iz0 < mz; iz0 += 4 * groups) {
      float re[4] = {0.f, 0.f, 0.f, 0.f}, im[4] = {0.f, 0.f, 0.f, 0.f};
      for (int z = 0; z < nz; ++z) {
        const float v = plane[y * ld + z];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int iz = iz0 + u * groups;
          if (iz < mz) {
            const float2 t = tz[iz * nz + z];
            re[u] = fmaf(v, t.x, re[u]);
            im[u] = fmaf(-v, t.y, im[u]);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int iz = iz0 + u * groups;
        if (iz < mz) zt[y * mz + iz] = make_float2(re[u], im[u]);
      }
    }
  }
  __syncthreads();
  // stage 2
  float2* dst = p + (bc * nx + x) * (size_t)my * mz;
  for (int o = threadIdx.x; o < my * mz; o += blockDim.x) {
    const int iy = o / mz, iz = o - iy * mz;
    float re = 0.f, im = 0.f;
    for (int y = 0; y < ny; ++y) {
      const float2 a = zt[y * mz + iz], t = ty[iy * ny + y];  // a conj(t)
      re = fmaf(a.x, t.x, fmaf(a.y, t.y, re));
      im = fmaf(a.y, t.x, fmaf(-a.x, t.y, im));
    }
    dst[o] = make_float2(re, im);
  }
  }
}

// x parts: one block per (field, 256 consecutive outputs) with the x twiddles in shared
// memory. fwd: X[bc][ix][iy][iz] = scale w(iz) sum_x P[bc][x][iy][iz] e^{-i kx x};
// inv: Q[bc][x][iy][iz] = scale w(iz) sum_ix Y[bc][ix][iy][iz] e^{+i kx x}.
__global__ void __launch_bounds__(256) trunc_fwd_x(long long total, int nx, int nz, int mx, int my, int mz,
                                                   float scale, float w_int, const float2* __restrict__ p,
                                                   float2* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char trraw[];
  float2* base = reinterpret_cast<float2*>(trraw);  // [nx]
  base_table(base, nx);
  __syncthreads();
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (id >= total) return;
  const int cols = my * mz;
  const long long bc = id / ((long long)mx * cols);
  const int r = (int)(id - bc * mx * cols), ix = r / cols, col = r - ix * cols, iz = col % mz;
  const int kx = kmode(ix, mx, nx);
  const float2* src = p + bc * nx * (size_t)cols + col;
  float re = 0.f, im = 0.f;
  int j = 0;
  for (int x = 0; x < nx; ++x) {
    const float2 t = base[j], a = src[(size_t)x * cols];
    re = fmaf(a.x, t.x, fmaf(a.y, t.y, re));
    im = fmaf(a.y, t.x, fmaf(-a.x, t.y, im));
    j += kx;
    if (j >= nx) j -= nx;
  }
  const float sw = scale * zweight(iz, nz, w_int);
  out[id] = make_float2(re * sw, im * sw);
}

__global__ void __launch_bounds__(256) trunc_inv_x(long long total, int nx, int nz, int mx, int my, int mz,
                                                   float scale, float w_int, const float2* __restrict__ y,
                                                   float2* __restrict__ q) {
  extern __shared__ __align__(16) unsigned char trraw[];
  float2* base = reinterpret_cast<float2*>(trraw);  // [nx]
  base_table(base, nx);
  __syncthreads();
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (id >= total) return;
  const int cols = my * mz;
  const long long bc = id / ((long long)nx * cols);
  const int r = (int)(id - bc * nx * cols), x = r / cols, col = r - x * cols, iz = col % mz;
  const float2* src = y + bc * mx * (size_t)cols + col;
  float re = 0.f, im = 0.f;
  for (int ix = 0; ix < mx; ++ix) {
    const float2 t = base[(int)((long long)kmode(ix, mx, nx) * x % nx)], a = src[(size_t)ix * cols];
    re = fmaf(a.x, t.x, fmaf(-a.y, t.y, re));
    im = fmaf(a.y, t.x, fmaf(a.x, t.y, im));
  }
  const float sw = scale * zweight(iz, nz, w_int);
  q[id] = make_float2(re * sw, im * sw);
}

// inv, (y, z) part: f[bc][x][y][z] = Re sum_{iy,iz} Q[bc][x][iy][iz] e^{+i(ky y + iz z)}.
// Stage 1: thread (y, iz) over iy. Stage 2: thread (y, z), z fastest, over iz (the row of
// stage 1 is the same for the warp's lanes, the twiddles of an iz consecutive).
__global__ void __launch_bounds__(kTrThreads) trunc_inv_yz(int nx, int ny, int nz, int my, int mz, int tc,
                                                           const float2* __restrict__ q,
                                                           float* __restrict__ f) {
  extern __shared__ __align__(16) unsigned char trraw[];
  // tc: stage 2 on the tensor cores (ny % 16 == 0, nz % 8 == 0) as the product of rt
  // [ny][2 mz] (re, im interleaved, zero-padded to a multiple of 8 columns) with bi
  // [2 mz][nz] (rows cos, -sin of 2 pi iz z / nz)
  const int kp = pad8(2 * mz), mzr = tc ? kp / 2 + 2 : mz;  // rt row: mzr complex values
  const int ldb = frag_ld(nz);
  float2* tz = reinterpret_cast<float2*>(trraw);  // [mz][nz]
  float2* ty = tz + mz * nz;                      // [my][ny]
  float2* qs = ty + my * ny;                      // [my][mz]
  float2* rt = qs + my * mz;                      // [ny][mzr]
  float2* base = rt + ny * mzr;                   // [max(ny, nz)]
  float* bi = reinterpret_cast<float*>(base + (ny > nz ? ny : nz));  // [kp][ldb] (tc)
  const size_t bc = blockIdx.y;
  base_table(base, nz);
  __syncthreads();
  for (int i = threadIdx.x; i < mz * nz; i += blockDim.x) {
    const int iz = i / nz, z = i - iz * nz;
    tz[i] = base[(int)((long long)iz * z % nz)];
  }
  if (tc) {
    for (int i = threadIdx.x; i < kp * ldb; i += blockDim.x) {
      const int k = i / ldb, z = i - k * ldb, iz = k >> 1;
      float v = 0.f;
      if (k < 2 * mz && z < nz) {
        const float2 w = base[(int)((long long)iz * z % nz)];
        v = (k & 1) ? -w.y : w.x;
      }
      bi[i] = v;
    }
    // the padding columns of rt stay zero
    for (int i = threadIdx.x; i < ny * mzr; i += blockDim.x) rt[i] = make_float2(0.f, 0.f);
  }
  __syncthreads();
  base_table(base, ny);
  __syncthreads();
  for (int i = threadIdx.x; i < my * ny; i += blockDim.x) {
    const int iy = i / ny, y = i - iy * ny;
    ty[i] = base[(int)((long long)kmode(iy, my, ny) * y % ny)];
  }
  // the block's x-planes (the tables above are built once per block)
  for (int x = blockIdx.x; x < nx; x += gridDim.x) {
  __syncthreads();  // (tables built; the previous plane's stage 2 done)
  const float2* src = q + (bc * nx + x) * (size_t)my * mz;
  for (int i = threadIdx.x; i < my * mz; i += blockDim.x) qs[i] = src[i];
  __syncthreads();
  for (int o = threadIdx.x; o < ny * mz; o += blockDim.x) {
    const int y = o / mz, iz = o - y * mz;
    float re = 0.f, im = 0.f;
    for (int iy = 0; iy < my; ++iy) {
      const float2 a = qs[iy * mz + iz], t = ty[iy * ny + y];
      re = fmaf(a.x, t.x, fmaf(-a.y, t.y, re));
      im = fmaf(a.y, t.x, fmaf(a.x, t.y, im));
    }
    rt[y * mzr + iz] = make_float2(re, im);
  }
  __syncthreads();
  float* dst = f + (bc * nx + x) * (size_t)ny * nz;
  if (tc) {
    const int nt = nz / 8, tiles = ny / 16 * nt;
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int tile = threadIdx.x >> 5; tile < tiles; tile += blockDim.x >> 5) {
      const int m0 = tile / nt * 16, n0 = tile % nt * 8;
      float d[4];
      tile_product_tf32(reinterpret_cast<const float*>(rt), 2 * mzr, bi, ldb, kp, m0, n0, d);
      *reinterpret_cast<float2*>(dst + (size_t)(m0 + g) * nz + n0 + 2 * t) = make_float2(d[0], d[1]);
      *reinterpret_cast<float2*>(dst + (size_t)(m0 + g + 8) * nz + n0 + 2 * t) = make_float2(d[2], d[3]);
    }
    continue;
  }
  for (int o = threadIdx.x; o < ny * nz; o += blockDim.x) {
    const int y = o / nz, z = o - y * nz;
    float v = 0.f;
    for (int iz = 0; iz < mz; ++iz) {
      const float2 a = rt[y * mzr + iz], t = tz[iz * nz + z];  // Re(a t)
      v = fmaf(a.x, t.x, fmaf(-a.y, t.y, v));
    }
    dst[o] = v;
  }
  }
}

// The (y, z) parts use the tensor-core stages when the plane tiles into 16 x 8 fragments.
int tc_planes(int ny, int nz) { return ny % 16 == 0 && nz % 8 == 0 ? 1 : 0; }

int trunc_check(long long bc, const int n[3], const int modes[3]) {
  if (bc < 1 || bc > 65535) return fail(-1, "truncated transform: fields outside [1, 65535]");
  if (n[0] < 1 || n[1] < 1 || n[2] < 1 || (size_t)n[1] * n[2] * 4 > kTrMaxPlane)
    return fail(-1, "truncated transform: grid outside the supported sizes (ny nz <= 16384)");
  if (modes[0] < 2 || modes[1] < 2 || modes[2] < 1 || modes[0] > n[0] || modes[1] > n[1] ||
      modes[2] > n[2] / 2 + 1 || (modes[0] % 2) || (modes[1] % 2) || modes[0] > kTrMaxModes ||
      modes[1] > kTrMaxModes || modes[2] > kTrMaxModes)
    return fail(-1, "truncated transform: retained modes do not fit the grid (mx, my even, <= 64)");
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

int lsn_truncated_forward(int fields, const int n[3], const int modes[3], const float* f, void* work,
                          void* out, float scale, float w_int, void* stream) {
  if (!n || !modes || !f || !work || !out) return fail(-1, "lsn_truncated_forward: null argument");
  if (int rc = trunc_check(fields, n, modes)) return rc;
  const int nx = n[0], ny = n[1], nz = n[2], mx = modes[0], my = modes[1], mz = modes[2];
  const size_t smem = sizeof(float2) * ((size_t)mz * nz + (size_t)my * ny + (size_t)ny * mz + (ny > nz ? ny : nz)) +
                      sizeof(float) * (size_t)ny * (nz + 1);
  static bool big = false;
  if (!big) {
    cudaFuncSetAttribute(trunc_fwd_yz, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    cudaFuncSetAttribute(trunc_inv_yz, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    big = true;
  }
  cudaStream_t s = (cudaStream_t)stream;
  trunc_fwd_yz<<<dim3(std::min(nx, kTrPlaneBlocks), fields), kTrThreads, smem, s>>>(nx, ny, nz, my, mz, f,
                                                                                   (float2*)work);
  const long long total = (long long)fields * mx * my * mz;
  trunc_fwd_x<<<(unsigned)((total + 255) / 256), 256, sizeof(float2) * nx, s>>>(
      total, nx, nz, mx, my, mz, scale, w_int, (const float2*)work, (float2*)out);
  return 0;
}

int lsn_truncated_inverse(int fields, const int n[3], const int modes[3], const void* y, void* work,
                          float* f, float scale, float w_int, void* stream) {
  if (!n || !modes || !y || !work || !f) return fail(-1, "lsn_truncated_inverse: null argument");
  if (int rc = trunc_check(fields, n, modes)) return rc;
  const int nx = n[0], ny = n[1], nz = n[2], mx = modes[0], my = modes[1], mz = modes[2];
  const int tc = tc_planes(ny, nz);
  const int mzr = tc ? pad8(2 * mz) / 2 + 2 : mz;
  const size_t smem = sizeof(float2) * ((size_t)mz * nz + (size_t)my * ny + (size_t)my * mz + (size_t)ny * mzr +
                                        (ny > nz ? ny : nz)) +
                      (tc ? sizeof(float) * (size_t)pad8(2 * mz) * frag_ld(nz) : 0);
  static bool big = false;
  if (!big) {
    cudaFuncSetAttribute(trunc_fwd_yz, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    cudaFuncSetAttribute(trunc_inv_yz, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    big = true;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const long long total = (long long)fields * nx * my * mz;
  trunc_inv_x<<<(unsigned)((total + 255) / 256), 256, sizeof(float2) * nx, s>>>(
      total, nx, nz, mx, my, mz, scale, w_int, (const float2*)y, (float2*)work);
  trunc_inv_yz<<<dim3(std::min(nx, kTrPlaneBlocks), fields), kTrThreads, smem, s>>>(nx, ny, nz, my, mz, tc,
                                                                                   (const float2*)work, f);
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
