// Damage extension of the solver (src/jaxmaterials/solver/lippmann_schwinger.py:36-100,
// 330-547): the pointwise degraded stress and tensile energy as library calls, and the
// phase-field solve, a scalar FFT fixed point on the solver's grid.
//
// Phase field (lippmann_schwinger.py:457-547): with A = 1/lc^2 + 2H/(gc lc), B = 2H/(gc lc)
// and A0 = (min A + max A)/2, iterate d = F^-1[F[chi] / (A0 + |xi~|^2)],
// chi = B - (A - A0) d until ||chi_new - chi|| <= tolerance ||chi_new||. One iteration is
// five passes over a complex work field W [x][y][z] (full spectrum): z transform of chi,
// y transform, x transform + division + inverse x transform, inverse y, inverse z fused
// with the update of d and chi and the FP64 partial norms; a one-block kernel then forms
// the residual and the stop decision on the device. Every kernel returns at once when the
// solve has stopped, so the host enqueues iterations in chunks and reads the state between
// chunks. Inverse transforms use the forward kernels on conjugated data.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/lippmann_schwinger.h"
#include "damage.cuh"
#include "fft_smem.cuh"
#include "ls_kernels.cuh"
#include "ls_solver_impl.cuh"

using namespace lsb;
using namespace lsb::detail;

namespace {

// ------------------------------------------------------------------ pointwise laws
template <typename T>
__global__ void damaged_stress_kernel(long long nv, const T* __restrict__ eps,
                                      const T* __restrict__ lambda, const T* __restrict__ mu,
                                      const T* __restrict__ dmg, T k, T* __restrict__ sigma) {
  const int b = blockIdx.y;
  const T* e_b = eps + (size_t)b * 6 * nv;
  T* s_b = sigma + (size_t)b * 6 * nv;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
       i += (long long)gridDim.x * blockDim.x) {
    T e[6], s[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) e[c] = e_b[(size_t)c * nv + i];
    T g = (T)1;  // no damage field: sigma+ + sigma-
    if (dmg) {
      const T om = (T)1 - dmg[i];
      g = om * om + k;
    }
    damaged_stress<T>(e, lambda[i], mu[i], g, s);
#pragma unroll
    for (int c = 0; c < 6; ++c) s_b[(size_t)c * nv + i] = s[c];
  }
}

template <typename T>
__global__ void strain_energy_kernel(long long nv, const T* __restrict__ eps,
                                     const T* __restrict__ lambda, const T* __restrict__ mu,
                                     T* __restrict__ psi, T* __restrict__ hist) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
       i += (long long)gridDim.x * blockDim.x) {
    T e[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) e[c] = eps[(size_t)c * nv + i];
    const T p = tensile_energy<T>(e, lambda[i], mu[i]);
    if (psi) psi[i] = p;
    if (hist) hist[i] = hist[i] > p ? hist[i] : p;  // H = max(H, psi)
  }
}

// ------------------------------------------------------------------ phase field
// complex values per thread in the phase-field transforms and values per block (small
// enough to keep the butterfly registers of a thread in registers in FP64)
constexpr int kPfVPT = 4;
constexpr int kPfTile = 1024;

struct PFState {
  double a0;      // reference coefficient A0
  double resid;   // last residual
  int iter;       // iterations done
  int done;       // stopped (converged, maxiter, or nothing to do)
};

struct PFCoef {
  double inv_lc2;  // 1 / lc^2
  double gclc;     // gc lc
};

template <typename T>
__device__ __forceinline__ T coef_a(T h, const PFCoef& c) {
  return (T)c.inv_lc2 + ((T)2 * h) / (T)c.gclc;
}
template <typename T>
__device__ __forceinline__ T coef_b(T h, const PFCoef& c) {
  return ((T)2 * h) / (T)c.gclc;
}

template <typename T>
__global__ void __launch_bounds__(256) pf_minmax_kernel(long long nv, const T* __restrict__ h,
                                                        double* __restrict__ part) {
  __shared__ double smin[256], smax[256];
  double lo = INFINITY, hi = -INFINITY;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = (double)h[i];
    lo = v < lo ? v : lo;
    hi = v > hi ? v : hi;
  }
  smin[threadIdx.x] = lo;
  smax[threadIdx.x] = hi;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + s]);
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = smin[0];
    part[2 * blockIdx.x + 1] = smax[0];
  }
}

// A0 = (A(min H) + A(max H)) / 2 in the field precision (A is monotone in H), and the
// initial state (one update at least, as the reference's loop starts at residual 1).
// One block of 256 threads: thread t folds partials t, t + 256, ... in order, then a fixed
// tree combines the threads (deterministic for a given partial count).
template <bool MINMAX>
__device__ __forceinline__ void fold_pairs(int nblk, const double* __restrict__ part, double& a,
                                           double& b) {
  __shared__ double sa[256], sb[256];
  double x = MINMAX ? INFINITY : 0.0, y = MINMAX ? -INFINITY : 0.0;
  for (int k = threadIdx.x; k < nblk; k += blockDim.x) {
    if (MINMAX) {
      x = fmin(x, part[2 * k]);
      y = fmax(y, part[2 * k + 1]);
    } else {
      x += part[2 * k];
      y += part[2 * k + 1];
    }
  }
  sa[threadIdx.x] = x;
  sb[threadIdx.x] = y;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      if (MINMAX) {
        sa[threadIdx.x] = fmin(sa[threadIdx.x], sa[threadIdx.x + s]);
        sb[threadIdx.x] = fmax(sb[threadIdx.x], sb[threadIdx.x + s]);
      } else {
        sa[threadIdx.x] += sa[threadIdx.x + s];
        sb[threadIdx.x] += sb[threadIdx.x + s];
      }
    }
    __syncthreads();
  }
  a = sa[0];
  b = sb[0];
}

template <typename T>
__global__ void __launch_bounds__(256) pf_setup_kernel(int nblk, const double* __restrict__ part, PFCoef c,
                                                       double tolerance, int maxiter,
                                                       PFState* __restrict__ st) {
  double lo, hi;
  fold_pairs<true>(nblk, part, lo, hi);
  if (threadIdx.x != 0) return;
  const T amin = coef_a<T>((T)lo, c), amax = coef_a<T>((T)hi, c);
  st->a0 = (double)((T)0.5 * (amin + amax));
  st->resid = 1.0;
  st->iter = 0;
  st->done = (1.0 > tolerance && maxiter > 0) ? 0 : 1;
}

// chi = B - (A - A0) d (initial polarisation).
template <typename T>
__global__ void pf_chi_kernel(long long nv, const T* __restrict__ h, const T* __restrict__ d,
                              PFCoef c, const PFState* __restrict__ st, T* __restrict__ chi) {
  const T a0 = (T)st->a0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
       i += (long long)gridDim.x * blockDim.x)
    chi[i] = coef_b<T>(h[i], c) - (coef_a<T>(h[i], c) - a0) * d[i];
}

// z transform of chi (real) into W, L lines per block.
template <typename T>
__global__ void __launch_bounds__(kMaxThreads) pf_zfwd_kernel(GridDesc g, int L, const T* __restrict__ chi,
                                                               cplx<T>* __restrict__ w,
                                                               const PFState* __restrict__ st) {
  using C = cplx<T>;
  if (st->done) return;
  extern __shared__ __align__(16) unsigned char raw[];
  C* buf = reinterpret_cast<C*>(raw);
  const long long nlines = (long long)g.nx * g.ny, l0 = (long long)blockIdx.x * L;
  const int nz = g.nz;
  for (int idx = threadIdx.x; idx < L * nz; idx += blockDim.x) {
    const int l = idx / nz, k = idx - l * nz;
    buf[idx] = mk<C>(l0 + l < nlines ? chi[(l0 + l) * nz + k] : (T)0, (T)0);
  }
  __syncthreads();
  fft_lines<kPfVPT, false>(buf, L, 1, nz, g.pz, twiddles<T>(g.pz));
  for (int idx = threadIdx.x; idx < L * nz; idx += blockDim.x) {
    const int l = idx / nz;
    if (l0 + l < nlines) w[l0 * nz + idx] = buf[idx];
  }
}

// y transform (inverse: conjugated in and out) of T consecutive z columns of one x.
template <typename T>
__global__ void __launch_bounds__(kMaxThreads) pf_y_kernel(GridDesc g, int TT, int inverse,
                                                            cplx<T>* __restrict__ w,
                                                            const PFState* __restrict__ st) {
  using C = cplx<T>;
  if (st->done) return;
  extern __shared__ __align__(16) unsigned char raw[];
  C* buf = reinterpret_cast<C*>(raw);  // [y][t]
  const int x = blockIdx.y, z0 = blockIdx.x * TT, ny = g.ny, nz = g.nz;
  for (int idx = threadIdx.x; idx < ny * TT; idx += blockDim.x) {
    const int y = idx / TT, t = idx - y * TT;
    C v = mk<C>((T)0, (T)0);
    if (z0 + t < nz) v = w[((size_t)x * ny + y) * nz + z0 + t];
    if (inverse) v.y = -v.y;
    buf[idx] = v;
  }
  __syncthreads();
  fft_lines<kPfVPT, true>(buf, TT, TT, 1, g.py, twiddles<T>(g.py));
  for (int idx = threadIdx.x; idx < ny * TT; idx += blockDim.x) {
    const int y = idx / TT, t = idx - y * TT;
    if (z0 + t < nz) {
      C v = buf[idx];
      if (inverse) v.y = -v.y;
      w[((size_t)x * ny + y) * nz + z0 + t] = v;
    }
  }
}

// x transform, division by A0 + |xi~|^2, inverse x transform, for T consecutive z
// columns of one y. |xi~|^2 from the FP64 sin/cos tables (lippmann_schwinger.py:490-493,
// fourier.py:9-58); the z tables hold kz <= nz/2, and |xi~|^2 is even in kz.
template <typename T>
__global__ void __launch_bounds__(kMaxThreads) pf_x_kernel(GridDesc g, int TT, cplx<T>* __restrict__ w,
                                                            const PFState* __restrict__ st) {
  using C = cplx<T>;
  if (st->done) return;
  extern __shared__ __align__(16) unsigned char raw[];
  C* buf = reinterpret_cast<C*>(raw);  // [x][t]
  const int ky = blockIdx.y, z0 = blockIdx.x * TT, nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t xs = (size_t)ny * nz;
  for (int idx = threadIdx.x; idx < nx * TT; idx += blockDim.x) {
    const int x = idx / TT, t = idx - x * TT;
    buf[idx] = z0 + t < nz ? w[x * xs + (size_t)ky * nz + z0 + t] : mk<C>((T)0, (T)0);
  }
  __syncthreads();
  fft_lines<kPfVPT, true>(buf, TT, TT, 1, g.px, twiddles<T>(g.px));
  const T a0 = (T)st->a0;
  for (int idx = threadIdx.x; idx < nx * TT; idx += blockDim.x) {
    const int kx = idx / TT, t = idx - kx * TT;
    const int kz = min(z0 + t, nz - 1);
    const int kzh = kz <= nz / 2 ? kz : nz - kz;
    const double x0 = (2.0 * g.nx / g.Lx) * g.sx[kx] * g.cy[ky] * g.cz[kzh];
    const double x1 = (2.0 * g.ny / g.Ly) * g.cx[kx] * g.sy[ky] * g.cz[kzh];
    const double x2 = (2.0 * g.nz / g.Lz) * g.cx[kx] * g.cy[ky] * g.sz[kzh];
    const T f0 = (T)x0, f1 = (T)x1, f2 = (T)x2;
    const T div = a0 + (f0 * f0 + f1 * f1 + f2 * f2);
    C v = buf[idx];
    v.x /= div;
    v.y = -v.y / div;  // conjugate for the inverse transform
    buf[idx] = v;
  }
  __syncthreads();
  fft_lines<kPfVPT, true>(buf, TT, TT, 1, g.px, twiddles<T>(g.px));
  for (int idx = threadIdx.x; idx < nx * TT; idx += blockDim.x) {
    const int x = idx / TT, t = idx - x * TT;
    if (z0 + t < nz) {
      C v = buf[idx];
      v.y = -v.y;
      w[x * xs + (size_t)ky * nz + z0 + t] = v;
    }
  }
}

// Inverse z transform of W, d = Re / N, chi = B - (A - A0) d, and the block's FP64 sums
// of (chi_new - chi)^2 and chi_new^2.
template <typename T>
__global__ void __launch_bounds__(kMaxThreads) pf_zinv_kernel(GridDesc g, int L, const cplx<T>* __restrict__ w,
                                                               const T* __restrict__ h, PFCoef c,
                                                               T* __restrict__ d, T* __restrict__ chi,
                                                               double* __restrict__ part,
                                                               const PFState* __restrict__ st) {
  using C = cplx<T>;
  if (st->done) return;
  extern __shared__ __align__(16) unsigned char raw[];
  C* buf = reinterpret_cast<C*>(raw);
  __shared__ double red[2][kMaxThreads / 32];
  const long long nlines = (long long)g.nx * g.ny, l0 = (long long)blockIdx.x * L;
  const int nz = g.nz;
  for (int idx = threadIdx.x; idx < L * nz; idx += blockDim.x) {
    const int l = idx / nz;
    C v = l0 + l < nlines ? w[l0 * nz + idx] : mk<C>((T)0, (T)0);
    v.y = -v.y;
    buf[idx] = v;
  }
  __syncthreads();
  fft_lines<kPfVPT, false>(buf, L, 1, nz, g.pz, twiddles<T>(g.pz));
  const T inv_n = (T)(1.0 / (double)g.nv);
  const T a0 = (T)st->a0;
  double s_diff = 0.0, s_new = 0.0;
  for (int idx = threadIdx.x; idx < L * nz; idx += blockDim.x) {
    const int l = idx / nz;
    if (l0 + l >= nlines) continue;
    const size_t i = (size_t)(l0 * nz + idx);
    const T dn = buf[idx].x * inv_n;
    const T hv = h[i];
    const T cn = coef_b<T>(hv, c) - (coef_a<T>(hv, c) - a0) * dn;
    const double df = (double)cn - (double)chi[i];
    s_diff += df * df;
    s_new += (double)cn * (double)cn;
    d[i] = dn;
    chi[i] = cn;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s_diff += __shfl_xor_sync(0xffffffffu, s_diff, o);
    s_new += __shfl_xor_sync(0xffffffffu, s_new, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = s_diff;
    red[1][threadIdx.x >> 5] = s_new;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int k = 0; k < (int)(blockDim.x + 31) / 32; ++k) {
      a += red[0][k];
      b += red[1][k];
    }
    part[2 * blockIdx.x] = a;
    part[2 * blockIdx.x + 1] = b;
  }
}

// residual = ||chi_new - chi|| / ||chi_new|| (0 when ||chi_new|| <= 1e-12), stop decision
// (lippmann_schwinger.py:503-520).
__global__ void __launch_bounds__(256) pf_finalize_kernel(int nblk, const double* __restrict__ part,
                                                          double tolerance, int maxiter,
                                                          PFState* __restrict__ st) {
  if (st->done) return;
  double a, b;
  fold_pairs<false>(nblk, part, a, b);
  if (threadIdx.x != 0) return;
  const double nb = sqrt(b);
  st->resid = nb > 1e-12 ? sqrt(a) / nb : 0.0;
  st->iter += 1;
  if (!(st->resid > tolerance && st->iter < maxiter)) st->done = 1;
}

template <typename T>
int phase_field(lsb_solver* s, const T* d_h, T* d_d, double gc, double lc, double tolerance,
                int maxiter, int* iters, double* residual) {
  using C = cplx<T>;
  const GridDesc& g = s->g;
  cudaStream_t st = s->stream;
  const long long nv = g.nv;
  const long long nlines = (long long)g.nx * g.ny;
  // lines per block for the z passes and columns per block for the y and x passes: about
  // kPfTile complex values per block
  const int Lz = (int)std::max<long long>(1, std::min<long long>(nlines, kPfTile / g.nz));
  const int Ty = std::max(1, std::min(g.nz, kPfTile / g.ny));
  const int Tx = std::max(1, std::min(g.nz, kPfTile / g.nx));
  const int tz = threads_for(g.pz, (long long)Lz * g.nz, kPfVPT);
  const int ty = threads_for(g.py, (long long)Ty * g.ny, kPfVPT);
  const int tx = threads_for(g.px, (long long)Tx * g.nx, kPfVPT);
  if (tz > kMaxThreads || ty > kMaxThreads || tx > kMaxThreads)
    return fail(-1, "phase field: FFT blocks above %d threads", kMaxThreads);
  const int zblocks = (int)((nlines + Lz - 1) / Lz);
  const int mmblk = (int)std::min<long long>(1024, (nv + 255) / 256);
  const int pblk = std::max(zblocks, mmblk);
  // work buffers kept by the solver across calls (sized for FP64, so either precision fits)
  if (!s->d_pf_w) {
    cudaError_t ae = cudaMalloc(&s->d_pf_w, sizeof(double2) * nv);
    if (ae == cudaSuccess) ae = cudaMalloc(&s->d_pf_chi, sizeof(double) * nv);
    if (ae == cudaSuccess) ae = cudaMalloc(&s->d_pf_part, sizeof(double) * 2 * pblk);
    if (ae == cudaSuccess) ae = cudaMalloc(&s->d_pf_state, sizeof(PFState));
    if (ae == cudaSuccess) ae = cudaMallocHost(&s->h_pf_state, sizeof(PFState));
    if (ae != cudaSuccess) {
      void** bufs[] = {&s->d_pf_w, &s->d_pf_chi, &s->d_pf_part, &s->d_pf_state};
      for (void** b : bufs) {
        if (*b) cudaFree(*b);
        *b = nullptr;
      }
      if (s->h_pf_state) cudaFreeHost(s->h_pf_state);
      s->h_pf_state = nullptr;
      return fail(-3, "phase field: allocation: %s", cudaGetErrorString(ae));
    }
  }
  C* w = static_cast<C*>(s->d_pf_w);
  T* chi = static_cast<T*>(s->d_pf_chi);
  double* part = static_cast<double*>(s->d_pf_part);
  PFState* dst = static_cast<PFState*>(s->d_pf_state);
  PFState* hst = static_cast<PFState*>(s->h_pf_state);
  cudaError_t e = cudaSuccess;
  const PFCoef c{1.0 / (lc * lc), gc * lc};
  const size_t smz = sizeof(C) * Lz * g.nz, smy = sizeof(C) * Ty * g.ny, smx = sizeof(C) * Tx * g.nx;
  pf_minmax_kernel<T><<<mmblk, 256, 0, st>>>(nv, d_h, part);
  pf_setup_kernel<T><<<1, 256, 0, st>>>(mmblk, part, c, tolerance, maxiter, dst);
  pf_chi_kernel<T><<<mmblk, 256, 0, st>>>(nv, d_h, d_d, c, dst, chi);
  s->launches += 3;
  const dim3 gy((g.nz + Ty - 1) / Ty, g.nx), gx((g.nz + Tx - 1) / Tx, g.ny);
  int done_iters = 0;
  for (int chunk = 1;; chunk = std::min(chunk * 2, 64)) {
    for (int k = 0; k < chunk; ++k) {
      pf_zfwd_kernel<T><<<zblocks, tz, smz, st>>>(g, Lz, chi, w, dst);
      pf_y_kernel<T><<<gy, ty, smy, st>>>(g, Ty, 0, w, dst);
      pf_x_kernel<T><<<gx, tx, smx, st>>>(g, Tx, w, dst);
      pf_y_kernel<T><<<gy, ty, smy, st>>>(g, Ty, 1, w, dst);
      pf_zinv_kernel<T><<<zblocks, tz, smz, st>>>(g, Lz, w, d_h, c, d_d, chi, part, dst);
      pf_finalize_kernel<<<1, 256, 0, st>>>(zblocks, part, tolerance, maxiter, dst);
    }
    s->launches += 6LL * chunk;
    e = cudaMemcpyAsync(hst, dst, sizeof(PFState), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) break;
    done_iters = hst->iter;
    if (hst->done) break;
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (iters) *iters = done_iters;
  if (residual) *residual = e == cudaSuccess ? hst->resid : NAN;
  if (e != cudaSuccess) return fail(-2, "phase field: %s", cudaGetErrorString(e));
  return 0;
}

int launch_grid(long long nv) { return (int)std::max<long long>(1, std::min<long long>(2048, (nv + 255) / 256)); }

}  // namespace

extern "C" {

int lsb_damage_stress(long long nv, int batch, const void* d_eps, const void* d_lambda,
                      const void* d_mu, const void* d_damage, double k, void* d_sigma,
                      int elem_size, void* stream) {
  if (nv < 0 || batch < 0) return fail(-1, "nv and batch must be >= 0");
  if (nv == 0 || batch == 0) return 0;
  if (!d_eps || !d_lambda || !d_mu || !d_sigma) return fail(-1, "null argument");
  if (batch > 65535) return fail(-1, "batch above 65535");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const dim3 grid(launch_grid(nv), batch);
  if (elem_size == 4)
    damaged_stress_kernel<float><<<grid, 256, 0, st>>>(
        nv, static_cast<const float*>(d_eps), static_cast<const float*>(d_lambda),
        static_cast<const float*>(d_mu), static_cast<const float*>(d_damage), (float)k,
        static_cast<float*>(d_sigma));
  else if (elem_size == 8)
    damaged_stress_kernel<double><<<grid, 256, 0, st>>>(
        nv, static_cast<const double*>(d_eps), static_cast<const double*>(d_lambda),
        static_cast<const double*>(d_mu), static_cast<const double*>(d_damage), k,
        static_cast<double*>(d_sigma));
  else
    return fail(-1, "elem_size must be 4 or 8");
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : fail(-2, "damage stress: %s", cudaGetErrorString(e));
}

int lsb_strain_energy(long long nv, const void* d_eps, const void* d_lambda, const void* d_mu,
                      void* d_psi, void* d_history, int elem_size, void* stream) {
  if (nv < 0) return fail(-1, "nv must be >= 0");
  if (nv == 0) return 0;
  if (!d_eps || !d_lambda || !d_mu || (!d_psi && !d_history)) return fail(-1, "null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (elem_size == 4)
    strain_energy_kernel<float><<<launch_grid(nv), 256, 0, st>>>(
        nv, static_cast<const float*>(d_eps), static_cast<const float*>(d_lambda),
        static_cast<const float*>(d_mu), static_cast<float*>(d_psi), static_cast<float*>(d_history));
  else if (elem_size == 8)
    strain_energy_kernel<double><<<launch_grid(nv), 256, 0, st>>>(
        nv, static_cast<const double*>(d_eps), static_cast<const double*>(d_lambda),
        static_cast<const double*>(d_mu), static_cast<double*>(d_psi),
        static_cast<double*>(d_history));
  else
    return fail(-1, "elem_size must be 4 or 8");
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : fail(-2, "strain energy: %s", cudaGetErrorString(e));
}

int lsb_phase_field_solve(lsb_solver* solver, const void* d_history, void* d_damage, double gc,
                          double lc, double tolerance, int maxiter, int elem_size, int* iters,
                          double* residual) {
  if (!solver) return fail(-1, "null solver");
  if (!d_history || !d_damage) return fail(-1, "null argument");
  if (!(gc > 0.0) || !(lc > 0.0)) return fail(-1, "gc and lc must be positive");
  if (maxiter < 0) return fail(-1, "maxiter must be >= 0");
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != solver->device) return fail(-1, "solver was created on device %d, current is %d", solver->device, cur);
  if (elem_size == 4)
    return phase_field<float>(solver, static_cast<const float*>(d_history), static_cast<float*>(d_damage),
                              gc, lc, tolerance, maxiter, iters, residual);
  if (elem_size == 8)
    return phase_field<double>(solver, static_cast<const double*>(d_history),
                               static_cast<double*>(d_damage), gc, lc, tolerance, maxiter, iters,
                               residual);
  return fail(-1, "elem_size must be 4 or 8");
}

}  // extern "C"
