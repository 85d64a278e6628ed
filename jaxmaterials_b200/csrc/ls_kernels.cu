// Kernels of the Moulinec-Suquet Lippmann-Schwinger iteration.
//
// One iteration of the reference loop (cuda/src/lippmann_schwinger.cu:192-216:
// stress -> R2C -> criterion -> Gamma^0 -> C2R -> update) is regrouped into passes
// that each stream the fields once:
//
//   xpass    forward x-DFT, FP64 equilibrium-residual partials and the zero mode,
//            r_hat = -Gamma^0 sigma_hat in registers, inverse x-DFT      (per ky, kz tile)
//   finalize criterion e, stop decision, iteration count               (one block / instance)
//   ypass    inverse y-DFT                                              (per x, kz tile)
//   zpass    z-C2R, eps += r / N, sigma = lambda tr(eps) I + 2 mu eps, z-R2C (per z line)
//   ypass    forward y-DFT
//
// The stop decision lives on the device: every kernel of an instance returns at once
// after `done` is set, so the host can enqueue many iterations without reading back.
#include <cfloat>
#include <cmath>

#include "fft_smem.cuh"
#include "ls_kernels.cuh"

namespace lsb {

// ----------------------------------------------------------------------------- z pass
// Lines l = x * ny + y; pair p of components (2p, 2p+1) shares one complex line
// z = a + i b (two real transforms for the price of one complex transform).
template <int VPT>
__global__ void __launch_bounds__(kMaxThreads) zpass_kernel(GridDesc g, int mode, int L,
                                                     const float* __restrict__ lambda,
                                                     const float* __restrict__ mu,
                                                     float* __restrict__ eps,
                                                     float2* __restrict__ spec,
                                                     const float* __restrict__ eps_bar,
                                                     const float* __restrict__ eps0,
                                                     const InstanceState* __restrict__ st,
                                                     SolveParams sp) {
  extern __shared__ float2 zbuf[];
  const int b = blockIdx.y;
  if (mode == 1 && st[b].done) return;
  const int nz = g.nz, nzh = g.nzh;
  const long long nlines = (long long)g.nx * g.ny;
  const long long l0 = (long long)blockIdx.x * L;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int ldz = nz;
  float* eb = eps + (size_t)b * 6 * g.nv;
  float2* sb = spec + (size_t)b * 6 * g.nm;

  if (mode == 1) {
    // Build conj(Z) with Z[k] = A[k] + i B[k] on the full line (Hermitian extension);
    // DC and (even nz) Nyquist terms are taken as real, as a C2R transform does.
    const int work = 3 * L * nzh;
    for (int idx = tid; idx < work; idx += nt) {
      int p = idx / (L * nzh);
      int rem = idx - p * L * nzh;
      int l = rem / nzh, k = rem - l * nzh;
      long long line = l0 + l;
      if (line >= nlines) continue;
      float2 A = sb[((size_t)(2 * p) * nlines + line) * nzh + k];
      float2 B = sb[((size_t)(2 * p + 1) * nlines + line) * nzh + k];
      const bool selfconj = (k == 0) || (2 * k == nz);
      if (selfconj) { A.y = 0.f; B.y = 0.f; }
      float2* Z = zbuf + (size_t)(p * L + l) * ldz;
      Z[k] = make_float2(A.x - B.y, -(A.y + B.x));
      if (!selfconj) Z[nz - k] = make_float2(A.x + B.y, A.y - B.x);
    }
    __syncthreads();
    fft_lines<VPT, false>(zbuf, 3 * L, 1, ldz, g.pz);
  }

  // Pointwise stage: update the strain, evaluate the stress, pack pairs for the R2C.
  {
    const int work = L * nz;
    const float inv_nv = sp.inv_nv;
    for (int idx = tid; idx < work; idx += nt) {
      int l = idx / nz, n = idx - l * nz;
      long long line = l0 + l;
      if (line >= nlines) continue;
      size_t v = (size_t)line * nz + n;
      float e[6];
      if (mode == 1) {
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          float2 w = zbuf[(size_t)(p * L + l) * ldz + n];
          // z = conj(w): r_{2p} = Re z = w.x, r_{2p+1} = Im z = -w.y
          e[2 * p] = eb[(size_t)(2 * p) * g.nv + v] + w.x * inv_nv;
          e[2 * p + 1] = eb[(size_t)(2 * p + 1) * g.nv + v] - w.y * inv_nv;
        }
      } else if (eps0 != nullptr) {
#pragma unroll
        for (int c = 0; c < 6; ++c) e[c] = eps0[((size_t)b * 6 + c) * g.nv + v];
      } else {
#pragma unroll
        for (int c = 0; c < 6; ++c) e[c] = eps_bar[b * 6 + c];
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) eb[(size_t)c * g.nv + v] = e[c];
      const float lam = lambda[v], tmu = 2.f * mu[v];
      const float ltr = lam * (e[0] + e[1] + e[2]);
      float s[6];
#pragma unroll
      for (int c = 0; c < 3; ++c) s[c] = tmu * e[c] + ltr;
#pragma unroll
      for (int c = 3; c < 6; ++c) s[c] = tmu * e[c];
#pragma unroll
      for (int p = 0; p < 3; ++p)
        zbuf[(size_t)(p * L + l) * ldz + n] = make_float2(s[2 * p], s[2 * p + 1]);
    }
  }
  __syncthreads();
  fft_lines<VPT, false>(zbuf, 3 * L, 1, ldz, g.pz);

  // Unpack the two real spectra: A = (Z[k] + conj Z[-k]) / 2, B = (Z[k] - conj Z[-k]) / 2i.
  {
    const int work = 3 * L * nzh;
    for (int idx = tid; idx < work; idx += nt) {
      int p = idx / (L * nzh);
      int rem = idx - p * L * nzh;
      int l = rem / nzh, k = rem - l * nzh;
      long long line = l0 + l;
      if (line >= nlines) continue;
      const float2* Z = zbuf + (size_t)(p * L + l) * ldz;
      float2 zk = Z[k];
      float2 zm = Z[k == 0 ? 0 : nz - k];
      float2 A = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
      float2 B = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
      sb[((size_t)(2 * p) * nlines + line) * nzh + k] = A;
      sb[((size_t)(2 * p + 1) * nlines + line) * nzh + k] = B;
    }
  }
}

// ----------------------------------------------------------------------------- y pass
// Block = (kz tile, x, instance * 6 + component); smem holds ny rows of T columns.
template <int VPT>
__global__ void __launch_bounds__(kMaxThreads) ypass_kernel(GridDesc g, int inverse, int T,
                                                     float2* __restrict__ spec,
                                                     const InstanceState* __restrict__ st) {
  extern __shared__ float2 ybuf[];
  const int bc = blockIdx.z;
  const int b = bc / 6;
  if (st[b].done) return;
  const int x = blockIdx.y;
  const int kz0 = blockIdx.x * T;
  const int ny = g.ny, nzh = g.nzh;
  const int tid = threadIdx.x, nt = blockDim.x;
  float2* base = spec + ((size_t)bc * g.nx + x) * (size_t)ny * nzh;
  const int work = ny * T;
  for (int idx = tid; idx < work; idx += nt) {
    int y = idx / T, t = idx - y * T;
    int kz = kz0 + t;
    float2 v = make_float2(0.f, 0.f);
    if (kz < nzh) v = base[(size_t)y * nzh + kz];
    if (inverse) v.y = -v.y;
    ybuf[idx] = v;
  }
  __syncthreads();
  fft_lines<VPT, true>(ybuf, T, T, 1, g.py);
  for (int idx = tid; idx < work; idx += nt) {
    int y = idx / T, t = idx - y * T;
    int kz = kz0 + t;
    float2 v = ybuf[idx];
    if (inverse) v.y = -v.y;
    if (kz < nzh) base[(size_t)y * nzh + kz] = v;
  }
}

// ----------------------------------------------------------------------------- x pass
// Block = (kz tile, ky, instance). Row kx of smem holds the 6*T values
// (component c, column t) at c*T + t.
template <int VPT>
__global__ void __launch_bounds__(kMaxThreads) xpass_kernel(GridDesc g, int T,
                                                     float2* __restrict__ spec,
                                                     const Medium* __restrict__ med,
                                                     InstanceState* __restrict__ st,
                                                     double* __restrict__ partials) {
  extern __shared__ float2 xbuf[];
  __shared__ double red[32];
  const int b = blockIdx.z;
  if (st[b].done) return;
  const int ky = blockIdx.y;
  const int kz0 = blockIdx.x * T;
  const int nx = g.nx, ny = g.ny, nzh = g.nzh;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int W = 6 * T;  // values per row
  float2* sb = spec + (size_t)b * 6 * g.nm;
  const size_t cstride = (size_t)g.nm;               // component stride
  const size_t xstride = (size_t)ny * nzh;           // x stride

  const int work = nx * W;
  for (int idx = tid; idx < work; idx += nt) {
    int kx = idx / W, q = idx - kx * W;
    int c = q / T, t = q - c * T;
    int kz = kz0 + t;
    float2 v = make_float2(0.f, 0.f);
    if (kz < nzh) v = sb[c * cstride + kx * xstride + (size_t)ky * nzh + kz];
    xbuf[idx] = v;
  }
  __syncthreads();
  fft_lines<VPT, true>(xbuf, W, W, 1, g.px);

  // Residual partials, zero mode and Gamma^0 (written conjugated for the inverse DFT).
  const float c_a = med->c_a, c_b = med->c_b;
  const double sxs = 2.0 * g.nx / g.Lx, sys = 2.0 * g.ny / g.Ly, szs = 2.0 * g.nz / g.Lz;
  double acc = 0.0;
  const int modes = nx * T;
  for (int idx = tid; idx < modes; idx += nt) {
    int kx = idx / T, t = idx - kx * T;
    int kz = kz0 + t;
    if (kz >= nzh) continue;
    float2* row = xbuf + (size_t)kx * W + t;
    float2 s[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) s[c] = row[c * T];
    // modified wave vector tilde(xi) in FP64 (fourier.py:9-58 order of products)
    const double x0 = sxs * g.sx[kx] * g.cy[ky] * g.cz[kz];
    const double x1 = sys * g.cx[kx] * g.sy[ky] * g.cz[kz];
    const double x2 = szs * g.cx[kx] * g.cy[ky] * g.sz[kz];
    // divergence xi . sigma_hat in FP32, weighted |.|^2 in FP64
    {
      const float f0 = (float)x0, f1 = (float)x1, f2 = (float)x2;
      float2 d0 = make_float2(f0 * s[0].x + f1 * s[3].x + f2 * s[4].x, f0 * s[0].y + f1 * s[3].y + f2 * s[4].y);
      float2 d1 = make_float2(f0 * s[3].x + f1 * s[1].x + f2 * s[5].x, f0 * s[3].y + f1 * s[1].y + f2 * s[5].y);
      float2 d2 = make_float2(f0 * s[4].x + f1 * s[5].x + f2 * s[2].x, f0 * s[4].y + f1 * s[5].y + f2 * s[2].y);
      double m2 = (double)d0.x * d0.x + (double)d0.y * d0.y + (double)d1.x * d1.x +
                  (double)d1.y * d1.y + (double)d2.x * d2.x + (double)d2.y * d2.y;
      const double w = (kz == 0 || 2 * kz == g.nz) ? 1.0 : 2.0;
      acc += w * m2;
    }
    if (kx == 0 && ky == 0 && kz == 0) {
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        st[b].sig0[2 * c] = s[c].x;
        st[b].sig0[2 * c + 1] = s[c].y;
      }
    }
    // normalised wave vector (fourier.py:61-85): FP64 with the 1e-12 guard, then FP32
    double nrm = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
    if (nrm < 1.0e-12) nrm = 1.0;
    const float z0 = (float)(x0 / nrm), z1 = (float)(x1 / nrm), z2 = (float)(x2 / nrm);
    // r_hat = C_A A(xi) sigma_hat + C_B (xi xi : sigma_hat) xi xi   (fourier.cu:268-327)
    const float z00 = z0 * z0, z11 = z1 * z1, z22 = z2 * z2;
    const float z01 = z0 * z1, z02 = z0 * z2, z12 = z1 * z2;
    float2 r[6];
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      float t0 = part ? s[0].y : s[0].x, t1 = part ? s[1].y : s[1].x, t2 = part ? s[2].y : s[2].x;
      float t3 = part ? s[3].y : s[3].x, t4 = part ? s[4].y : s[4].x, t5 = part ? s[5].y : s[5].x;
      float rho = z00 * t0 + z11 * t1 + z22 * t2 + 2.f * (z01 * t3 + z02 * t4 + z12 * t5);
      float a0 = z0 * (z0 * t0 + z2 * t4 + z1 * t3);
      float a1 = z1 * (z1 * t1 + z2 * t5 + z0 * t3);
      float a2 = z2 * (z2 * t2 + z1 * t5 + z0 * t4);
      float a3 = 0.5f * (z01 * (t0 + t1) + (z00 + z11) * t3 + z2 * (z0 * t5 + z1 * t4));
      float a4 = 0.5f * (z02 * (t0 + t2) + (z00 + z22) * t4 + z1 * (z0 * t5 + z2 * t3));
      float a5 = 0.5f * (z12 * (t1 + t2) + (z11 + z22) * t5 + z0 * (z1 * t4 + z2 * t3));
      float o0 = c_a * a0 + c_b * rho * z00;
      float o1 = c_a * a1 + c_b * rho * z11;
      float o2 = c_a * a2 + c_b * rho * z22;
      float o3 = c_a * a3 + c_b * rho * z01;
      float o4 = c_a * a4 + c_b * rho * z02;
      float o5 = c_a * a5 + c_b * rho * z12;
      if (part == 0) {
        r[0].x = o0; r[1].x = o1; r[2].x = o2; r[3].x = o3; r[4].x = o4; r[5].x = o5;
      } else {
        r[0].y = -o0; r[1].y = -o1; r[2].y = -o2; r[3].y = -o3; r[4].y = -o4; r[5].y = -o5;
      }
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) row[c * T] = r[c];
  }
  __syncthreads();
  fft_lines<VPT, true>(xbuf, W, W, 1, g.px);
  for (int idx = tid; idx < work; idx += nt) {
    int kx = idx / W, q = idx - kx * W;
    int c = q / T, t = q - c * T;
    int kz = kz0 + t;
    if (kz < nzh) {
      float2 v = xbuf[idx];
      sb[c * cstride + kx * xstride + (size_t)ky * nzh + kz] = make_float2(v.x, -v.y);
    }
  }

  // Deterministic block reduction of the residual partial.
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((tid & 31) == 0) red[tid >> 5] = acc;
  __syncthreads();
  if (tid < 32) {
    double v = (tid < (nt + 31) / 32) ? red[tid] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (tid == 0) {
      const int nblk = gridDim.x * gridDim.y;
      partials[(size_t)b * nblk + blockIdx.y * gridDim.x + blockIdx.x] = v;
    }
  }
}

// ----------------------------------------------------------------------------- finalize
// Criterion (lippmann_schwinger.py:118-143 / lippmann_schwinger.cu:95-109) and the stop
// rule (lippmann_schwinger.cu:201-206; lippmann_schwinger.py:196-206).
__global__ void finalize_kernel(int nblk, InstanceState* __restrict__ st,
                                const double* __restrict__ partials, double* __restrict__ history,
                                int history_len, SolveParams sp) {
  __shared__ double red[32];
  const int b = blockIdx.x;
  InstanceState& s = st[b];
  if (s.done) return;
  const int tid = threadIdx.x, nt = blockDim.x;
  double acc = 0.0;
  for (int i = tid; i < nblk; i += nt) acc += partials[(size_t)b * nblk + i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((tid & 31) == 0) red[tid >> 5] = acc;
  __syncthreads();
  if (tid == 0) {
    double num2 = 0.0;
    for (int w = 0; w < (nt + 31) / 32; ++w) num2 += red[w];
    double den2 = 0.0;
    for (int c = 0; c < 6; ++c) {
      double m2 = s.sig0[2 * c] * s.sig0[2 * c] + s.sig0[2 * c + 1] * s.sig0[2 * c + 1];
      den2 += (c < 3 ? 1.0 : 2.0) * m2;
    }
    double e = (num2 == 0.0) ? 0.0 : sqrt(num2) / sqrt(den2);
    if (s.evals == 0) s.e0 = e;
    if (history != nullptr && s.evals < history_len) history[(size_t)b * history_len + s.evals] = e;
    s.evals += 1;
    s.e = e;
    const double thr = fmax((double)sp.rtol * s.e0, (double)sp.atol);
    const bool conv = sp.rule == 0 ? (e < thr) : (e <= thr);
    if (!isfinite(e)) {
      s.done = 1;
      s.status = kNonFinite;
    } else if (conv) {
      s.done = 1;
      s.status = kConverged;
    } else if (s.iter >= sp.maxiter) {
      s.done = 1;
      s.status = kMaxIter;
    } else {
      s.iter += 1;
    }
  }
}

__global__ void reset_state_kernel(int batch, InstanceState* st) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < batch) {
    InstanceState z = {};
    st[b] = z;
  }
}

// ----------------------------------------------------------------------------- medium
__global__ void minmax_partial_kernel(long long nv, const float* __restrict__ lambda,
                                      const float* __restrict__ mu, float* __restrict__ scratch) {
  __shared__ float sh[4][32];
  float lmin = FLT_MAX, lmax = -FLT_MAX, mmin = FLT_MAX, mmax = -FLT_MAX;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
       i += (long long)gridDim.x * blockDim.x) {
    float l = lambda[i], m = mu[i];
    lmin = fminf(lmin, l); lmax = fmaxf(lmax, l);
    mmin = fminf(mmin, m); mmax = fmaxf(mmax, m);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lmin = fminf(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
    lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    mmin = fminf(mmin, __shfl_xor_sync(0xffffffffu, mmin, o));
    mmax = fmaxf(mmax, __shfl_xor_sync(0xffffffffu, mmax, o));
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { sh[0][w] = lmin; sh[1][w] = lmax; sh[2][w] = mmin; sh[3][w] = mmax; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (blockDim.x + 31) / 32; ++i) {
      lmin = fminf(lmin, sh[0][i]); lmax = fmaxf(lmax, sh[1][i]);
      mmin = fminf(mmin, sh[2][i]); mmax = fmaxf(mmax, sh[3][i]);
    }
    scratch[4 * blockIdx.x + 0] = lmin;
    scratch[4 * blockIdx.x + 1] = lmax;
    scratch[4 * blockIdx.x + 2] = mmin;
    scratch[4 * blockIdx.x + 3] = mmax;
  }
}

__global__ void minmax_final_kernel(int nblk, const float* __restrict__ scratch, Medium* med) {
  if (threadIdx.x != 0) return;
  float lmin = FLT_MAX, lmax = -FLT_MAX, mmin = FLT_MAX, mmax = -FLT_MAX;
  for (int i = 0; i < nblk; ++i) {
    lmin = fminf(lmin, scratch[4 * i + 0]); lmax = fmaxf(lmax, scratch[4 * i + 1]);
    mmin = fminf(mmin, scratch[4 * i + 2]); mmax = fmaxf(mmax, scratch[4 * i + 3]);
  }
  Medium m;
  m.lmin = lmin; m.lmax = lmax; m.mmin = mmin; m.mmax = mmax;
  // lambda0 = 1/2 (min + max) in FP32 (lippmann_schwinger.py:171-172)
  m.lambda0 = 0.5f * (lmin + lmax);
  m.mu0 = 0.5f * (mmin + mmax);
  const double l0 = m.lambda0, m0 = m.mu0;
  m.c_a = (float)(-1.0 / m0);
  m.c_b = (float)((l0 + m0) / (m0 * (l0 + 2.0 * m0)));
  *med = m;
}

// ----------------------------------------------------------------------------- stress
__global__ void stress_kernel(long long nv, int batch, const float* __restrict__ lambda,
                              const float* __restrict__ mu, const float* __restrict__ eps,
                              float* __restrict__ sigma, double* __restrict__ scratch) {
  __shared__ double sh[6][32];
  const int b = blockIdx.y;
  const float* eb = eps + (size_t)b * 6 * nv;
  float* sg = sigma ? sigma + (size_t)b * 6 * nv : nullptr;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
       i += (long long)gridDim.x * blockDim.x) {
    float e[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) e[c] = eb[(size_t)c * nv + i];
    const float lam = lambda[i], tmu = 2.f * mu[i];
    const float ltr = lam * (e[0] + e[1] + e[2]);
    float s[6];
#pragma unroll
    for (int c = 0; c < 3; ++c) s[c] = tmu * e[c] + ltr;
#pragma unroll
    for (int c = 3; c < 6; ++c) s[c] = tmu * e[c];
    if (sg) {
#pragma unroll
      for (int c = 0; c < 6; ++c) sg[(size_t)c * nv + i] = s[c];
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[c] += s[c];
  }
  if (scratch == nullptr) return;
#pragma unroll
  for (int c = 0; c < 6; ++c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int c = 0; c < 6; ++c) sh[c][w] = acc[c];
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double v = 0.0;
    for (int i = 0; i < (blockDim.x + 31) / 32; ++i) v += sh[threadIdx.x][i];
    scratch[((size_t)b * 6 + threadIdx.x) * gridDim.x + blockIdx.x] = v;
  }
}

__global__ void mean_final_kernel(int nblk, long long nv, const double* __restrict__ scratch,
                                  double* __restrict__ mean) {
  const int bc = blockIdx.x;  // instance * 6 + component
  if (threadIdx.x != 0) return;
  double v = 0.0;
  for (int i = 0; i < nblk; ++i) v += scratch[(size_t)bc * nblk + i];
  mean[bc] = v / (double)nv;
}

// ----------------------------------------------------------------------------- host side
static int pick_pow2_leq(int v) {
  int p = 1;
  while (p * 2 <= v) p *= 2;
  return p;
}

LaunchShape plan_launch(const GridDesc& g) {
  LaunchShape s;
  const long long kElems = kPassElems;
  // z pass: 3 complex lines of nz per (x, y) line
  s.lines_per_block = (int)std::max<long long>(1, kElems / (3LL * g.nz));
  s.lines_per_block = std::min<long long>(s.lines_per_block, (long long)g.nx * g.ny);
  s.z_threads = threads_for(g.pz, 3LL * s.lines_per_block * g.nz, kVPT);
  while (s.z_threads > kMaxThreads && s.lines_per_block > 1) {
    s.lines_per_block -= 1;
    s.z_threads = threads_for(g.pz, 3LL * s.lines_per_block * g.nz, kVPT);
  }
  s.z_blocks = (int)(((long long)g.nx * g.ny + s.lines_per_block - 1) / s.lines_per_block);
  s.z_smem = (size_t)3 * s.lines_per_block * g.nz * sizeof(float2);
  // y pass
  s.ty = std::max(1, std::min(16, (int)(kElems / g.ny)));
  s.ty = std::min(s.ty, g.nzh);
  s.y_tiles = (g.nzh + s.ty - 1) / s.ty;
  s.y_threads = threads_for(g.py, (long long)g.ny * s.ty, kVPT);
  while (s.y_threads > kMaxThreads && s.ty > 1) {
    s.ty -= 1;
    s.y_threads = threads_for(g.py, (long long)g.ny * s.ty, kVPT);
  }
  s.y_tiles = (g.nzh + s.ty - 1) / s.ty;
  s.y_smem = (size_t)g.ny * s.ty * sizeof(float2);
  // x pass
  s.tx = std::max(1, std::min(16, pick_pow2_leq((int)std::max<long long>(1, kElems / (6LL * g.nx)))));
  s.tx = std::min(s.tx, g.nzh);
  s.x_tiles = (g.nzh + s.tx - 1) / s.tx;
  s.x_threads = threads_for(g.px, 6LL * g.nx * s.tx, kVPT);
  while (s.x_threads > kMaxThreads && s.tx > 1) {
    s.tx /= 2;
    s.x_threads = threads_for(g.px, 6LL * g.nx * s.tx, kVPT);
  }
  s.x_tiles = (g.nzh + s.tx - 1) / s.tx;
  s.x_smem = (size_t)6 * g.nx * s.tx * sizeof(float2);
  s.x_blocks_per_instance = s.x_tiles * g.ny;
  return s;
}

// Every pass is planned with at most kPassElems complex values of dynamic shared memory,
// so one fixed opt-in serves all solvers alive in the process.
cudaError_t configure_kernels(const LaunchShape& s) {
  const int bytes = (int)(kPassElems * sizeof(float2));
  if (s.z_smem > (size_t)bytes || s.y_smem > (size_t)bytes || s.x_smem > (size_t)bytes)
    return cudaErrorInvalidValue;
  cudaError_t e;
  e = cudaFuncSetAttribute(zpass_kernel<kVPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(ypass_kernel<kVPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(xpass_kernel<kVPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  return e;
}

void launch_zpass(const GridDesc& g, const LaunchShape& s, int mode, int batch, const float* lambda,
                  const float* mu, float* eps, float2* spec, const float* eps_bar,
                  const float* eps0, const InstanceState* st, const SolveParams& sp,
                  cudaStream_t stream) {
  dim3 grid(s.z_blocks, batch);
  zpass_kernel<kVPT><<<grid, s.z_threads, s.z_smem, stream>>>(
      g, mode, s.lines_per_block, lambda, mu, eps, spec, eps_bar, eps0, st, sp);
}

void launch_ypass(const GridDesc& g, const LaunchShape& s, bool inverse, int batch, float2* spec,
                  const InstanceState* st, cudaStream_t stream) {
  dim3 grid(s.y_tiles, g.nx, 6 * batch);
  ypass_kernel<kVPT><<<grid, s.y_threads, s.y_smem, stream>>>(g, inverse ? 1 : 0, s.ty, spec, st);
}

void launch_xpass(const GridDesc& g, const LaunchShape& s, int batch, float2* spec, const Medium* med,
                  InstanceState* st, double* partials, cudaStream_t stream) {
  dim3 grid(s.x_tiles, g.ny, batch);
  xpass_kernel<kVPT><<<grid, s.x_threads, s.x_smem, stream>>>(g, s.tx, spec, med, st, partials);
}

void launch_finalize(const GridDesc& g, const LaunchShape& s, int batch, InstanceState* st,
                     const double* partials, double* history, int history_len,
                     const SolveParams& sp, cudaStream_t stream) {
  (void)g;
  finalize_kernel<<<batch, 256, 0, stream>>>(s.x_blocks_per_instance, st, partials, history,
                                              history_len, sp);
}

void launch_reset_state(int batch, InstanceState* st, cudaStream_t stream) {
  reset_state_kernel<<<(batch + 127) / 128, 128, 0, stream>>>(batch, st);
}

void launch_medium(long long nv, const float* lambda, const float* mu, float* scratch, Medium* med,
                   cudaStream_t stream) {
  int nblk = (int)std::min<long long>(1024, (nv + 255) / 256);
  if (nblk < 1) nblk = 1;
  minmax_partial_kernel<<<nblk, 256, 0, stream>>>(nv, lambda, mu, scratch);
  minmax_final_kernel<<<1, 32, 0, stream>>>(nblk, scratch, med);
}

void launch_stress(const GridDesc& g, int batch, const float* lambda, const float* mu,
                   const float* eps, float* sigma, double* scratch, double* mean,
                   cudaStream_t stream) {
  int nblk = (int)std::min<long long>(1024, (g.nv + 255) / 256);
  if (nblk < 1) nblk = 1;
  dim3 grid(nblk, batch);
  stress_kernel<<<grid, 256, 0, stream>>>(g.nv, batch, lambda, mu, eps, sigma,
                                          mean ? scratch : nullptr);
  if (mean) mean_final_kernel<<<6 * batch, 32, 0, stream>>>(nblk, g.nv, scratch, mean);
}

}  // namespace lsb
