// Kernels of the Moulinec-Suquet Lippmann-Schwinger iteration.
//
// One iteration of the reference loop (cuda/src/lippmann_schwinger.cu:192-216:
// stress -> R2C -> criterion -> Gamma^0 -> C2R -> update) is regrouped into passes
// that each stream the fields once:
//
//   xpass    forward x-DFT, FP64 equilibrium-residual partials and the zero mode,
//            r_hat = -Gamma^0 sigma_hat in registers, inverse x-DFT      (per ky, kz tile)
//   finalize criterion e, stop / stall decision, iteration count       (one block / instance)
//   ypass    inverse y-DFT                                              (per x, kz tile)
//   zpass    z-C2R, eps += r / N, sigma = lambda tr(eps) I + 2 mu eps, z-R2C (per z line)
//   ypass    forward y-DFT
//
// Every pass exists for FP32 fields (T = float) and FP64 fields (T = double). An
// instance is processed by the passes of its current phase (0: FP32, 1: FP64) until it
// is done, so the host can enqueue many iterations without reading anything back.
#include <cfloat>
#include <cmath>

#include "aniso.cuh"
#include "damage.cuh"
#include "fft_smem.cuh"
#include "ls_kernels.cuh"

namespace lsb {

template <typename T>
__device__ __forceinline__ bool active(const InstanceState& s) {
  return !s.done && s.phase == (sizeof(T) == 8 ? 1 : 0);
}

// ----------------------------------------------------------------------------- z pass
// Lines l = x * ny + y; pair p of components (2p, 2p+1) shares one complex line
// z = a + i b (two real transforms for the price of one complex transform).
// mode 0: eps = eps_bar (or eps0); mode 1: eps += r / N with r from the spectrum;
// mode 2: keep eps (continuation of an instance in another precision, or the iterate
//         written by anderson_combine_kernel); eps is not rewritten;
// mode 3: Anderson residual: r from the spectrum into the rings, g = eps + r (no stress,
//         no forward transform; anderson_gram_kernel then forms the Gram row).
template <typename T>
__device__ __forceinline__ void anderson_slots(const InstanceState& s, int depth, int& slot, int& filled) {
  const int j = s.iter - 1 - s.aa_base;
  slot = j % (depth + 1);
  filled = j + 1 < depth + 1 ? j + 1 : depth + 1;
}

// Block-wide FP64 sums of v[0..n) (n <= kMaxDepth + 1) written to out[0..n).
__device__ __forceinline__ void block_sum_slots(double* v, int n, double (*red)[32], double* out) {
  const int tid = threadIdx.x;
  for (int s = 0; s < n; ++s) {
    double a = v[s];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if ((tid & 31) == 0) red[s][tid >> 5] = a;
  }
  __syncthreads();
  if (tid < n) {
    double a = 0.0;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) a += red[tid][w];
    out[tid] = a;
  }
}

template <typename T, int VPT>
__global__ void __launch_bounds__(kMaxThreads) zpass_kernel(GridDesc g, int mode, int L,
                                                     const T* __restrict__ lambda,
                                                     const T* __restrict__ mu,
                                                     T* __restrict__ eps,
                                                     cplx<T>* __restrict__ spec,
                                                     const double* __restrict__ eps_bar,
                                                     const T* __restrict__ eps0,
                                                     InstanceState* __restrict__ st,
                                                     const Medium* __restrict__ med,
                                                     AndersonArgs<T> aa) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char zraw[];
  C* zbuf = reinterpret_cast<C*>(zraw);
  const int b = blockIdx.y;
  if (!active<T>(st[b])) return;
  const int nz = g.nz, nzh = g.nzh;
  const long long nlines = (long long)g.nx * g.ny;
  const long long l0 = (long long)blockIdx.x * L;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int ldz = nz;
  T* eb = eps + (size_t)b * 6 * g.nv;
  C* sb = spec + (size_t)b * 6 * g.nm;
  const Plan1D& pz = g.pz;
  const C* tw = twiddles<T>(pz);
  lambda += (size_t)(b / g.lame_group) * g.nv;
  mu += (size_t)(b / g.lame_group) * g.nv;
  med += b / g.lame_group;
  const T* dmg = damage_field<T>(g);
  if (dmg) dmg += (size_t)(b / g.lame_group) * g.nv;
  const T* cf = stiffness_field<T>(g);
  if (cf) cf += (size_t)(b / g.lame_group) * 21 * g.nv;

  if (mode == 1 || mode == 3) {
    // Build conj(Z) with Z[k] = A[k] + i B[k] on the full line (Hermitian extension);
    // DC and (even nz) Nyquist terms are taken as real, as a C2R transform does.
    const int work = 3 * L * nzh;
    for (int idx = tid; idx < work; idx += nt) {
      int p = idx / (L * nzh);
      int rem = idx - p * L * nzh;
      int l = rem / nzh, k = rem - l * nzh;
      long long line = l0 + l;
      if (line >= nlines) continue;
      C A = sb[((size_t)(2 * p) * nlines + line) * nzh + k];
      C B = sb[((size_t)(2 * p + 1) * nlines + line) * nzh + k];
      const bool selfconj = (k == 0) || (2 * k == nz);
      if (selfconj) { A.y = 0; B.y = 0; }
      C* Z = zbuf + (size_t)(p * L + l) * ldz;
      Z[k] = mk<C>(A.x - B.y, -(A.y + B.x));
      if (!selfconj) Z[nz - k] = mk<C>(A.x + B.y, A.y - B.x);
    }
    __syncthreads();
    fft_lines<VPT, false>(zbuf, 3 * L, 1, ldz, pz, tw);
  }

  if (mode == 3) {
    // Anderson residual: rings, then done.
    int slot, filled;
    anderson_slots<T>(st[b], aa.depth, slot, filled);
    const int M1 = aa.depth + 1;
    const size_t ring = (size_t)6 * g.nv;   // one slot
    typename ResRing<T>::type* rb = aa.r + (size_t)b * M1 * ring;
    T* gb = aa.g + (size_t)b * M1 * ring;
    const T inv_nv = (T)(1.0 / (double)g.nv);
    float rscale = 1.f;  // FP16 residual ring: the slot's power-of-two scale
    if constexpr (sizeof(T) == 4) {
      const int k = ring_exponent(st[b].ring_max, eps_bar + 6 * b);
      rscale = ldexpf(1.f, k);
      if (blockIdx.x == 0 && tid == 0) st[b].ring_exp[slot] = k;
    }
    for (int idx = tid; idx < L * nz; idx += nt) {
      int l = idx / nz, n = idx - l * nz;
      long long line = l0 + l;
      if (line >= nlines) continue;
      size_t v = (size_t)line * nz + n;
      T r[6];
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        C w = zbuf[(size_t)(p * L + l) * ldz + n];
        r[2 * p] = w.x * inv_nv;
        r[2 * p + 1] = -w.y * inv_nv;
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        const size_t o = (size_t)c * g.nv + v;
        if constexpr (sizeof(T) == 4)
          rb[slot * ring + o] = ring_store(r[c], rscale);
        else
          rb[slot * ring + o] = r[c];
        gb[slot * ring + o] = eb[o] + r[c];
      }
    }
    return;
  }

  // Shift of the forward transform: the current mean-stress estimate (see InstanceState).
  T shift[6];
  if (mode != 0) {
#pragma unroll
    for (int c = 0; c < 6; ++c) shift[c] = (T)st[b].shift[c];
  } else {
    // <sigma(eps_bar)> = <lambda> tr(eps_bar) I + 2 <mu> eps_bar
    const double* e = eps_bar + 6 * b;
    const double tr = e[0] + e[1] + e[2];
    double sh[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) sh[c] = (c < 3 ? med->lmean * tr : 0.0) + 2.0 * med->mmean * e[c];
    if (cf) {  // anisotropic: C^0 eps_bar
      const double* c0 = g.c0 + (size_t)(b / g.lame_group) * 21;
      aniso_stress<double>([&](int k) { return c0[k]; }, e, sh);
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) shift[c] = (T)sh[c];
    if (blockIdx.x == 0 && tid == 0) {
#pragma unroll
      for (int c = 0; c < 6; ++c) st[b].shift[c] = (double)shift[c];
    }
  }

  // Pointwise stage: update the strain, evaluate the stress, pack pairs for the R2C.
  {
    const int work = L * nz;
    const T inv_nv = (T)(1.0 / (double)g.nv);
    for (int idx = tid; idx < work; idx += nt) {
      int l = idx / nz, n = idx - l * nz;
      long long line = l0 + l;
      if (line >= nlines) continue;
      size_t v = (size_t)line * nz + n;
      T e[6];
      if (mode == 1) {
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          C w = zbuf[(size_t)(p * L + l) * ldz + n];
          // z = conj(w): r_{2p} = Re z = w.x, r_{2p+1} = Im z = -w.y
          e[2 * p] = eb[(size_t)(2 * p) * g.nv + v] + w.x * inv_nv;
          e[2 * p + 1] = eb[(size_t)(2 * p + 1) * g.nv + v] - w.y * inv_nv;
        }
      } else if (mode == 2) {
#pragma unroll
        for (int c = 0; c < 6; ++c) e[c] = eb[(size_t)c * g.nv + v];
      } else if (eps0 != nullptr) {
#pragma unroll
        for (int c = 0; c < 6; ++c) e[c] = eps0[((size_t)b * 6 + c) * g.nv + v];
      } else {
#pragma unroll
        for (int c = 0; c < 6; ++c) e[c] = (T)eps_bar[b * 6 + c];
      }
      if (mode != 2) {
#pragma unroll
        for (int c = 0; c < 6; ++c) eb[(size_t)c * g.nv + v] = e[c];
      }
      T s[6];
      if (cf) {
        aniso_stress<T>([&](int k) { return cf[(size_t)k * g.nv + v]; }, e, s);
      } else if (dmg) {
        const T om = (T)1 - dmg[v];
        damaged_stress<T>(e, lambda[v], mu[v], om * om + (T)g.dmg_k, s);
      } else {
        const T lam = lambda[v], tmu = (T)2 * mu[v];
        const T ltr = lam * (e[0] + e[1] + e[2]);
#pragma unroll
        for (int c = 0; c < 3; ++c) s[c] = tmu * e[c] + ltr;
#pragma unroll
        for (int c = 3; c < 6; ++c) s[c] = tmu * e[c];
      }
#pragma unroll
      for (int p = 0; p < 3; ++p)
        zbuf[(size_t)(p * L + l) * ldz + n] =
            mk<C>(s[2 * p] - shift[2 * p], s[2 * p + 1] - shift[2 * p + 1]);
    }
  }
  __syncthreads();
  fft_lines<VPT, false>(zbuf, 3 * L, 1, ldz, pz, tw);

  // Unpack the two real spectra: A = (Z[k] + conj Z[-k]) / 2, B = (Z[k] - conj Z[-k]) / 2i.
  {
    const int work = 3 * L * nzh;
    const T h = (T)0.5;
    for (int idx = tid; idx < work; idx += nt) {
      int p = idx / (L * nzh);
      int rem = idx - p * L * nzh;
      int l = rem / nzh, k = rem - l * nzh;
      long long line = l0 + l;
      if (line >= nlines) continue;
      const C* Z = zbuf + (size_t)(p * L + l) * ldz;
      C zk = Z[k];
      C zm = Z[k == 0 ? 0 : nz - k];
      sb[((size_t)(2 * p) * nlines + line) * nzh + k] = mk<C>(h * (zk.x + zm.x), h * (zk.y - zm.y));
      sb[((size_t)(2 * p + 1) * nlines + line) * nzh + k] = mk<C>(h * (zk.y + zm.y), -h * (zk.x - zm.x));
    }
  }
}

// ----------------------------------------------------------------------------- y pass
// Block = (kz tile, x, instance * 6 + component); smem holds ny rows of TT columns.
template <typename T, int VPT>
__global__ void __launch_bounds__(kMaxThreads) ypass_kernel(GridDesc g, int inverse, int TT,
                                                     cplx<T>* __restrict__ spec,
                                                     const InstanceState* __restrict__ st) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char yraw[];
  C* ybuf = reinterpret_cast<C*>(yraw);
  const int bc = blockIdx.z;
  const int b = bc / 6;
  if (!active<T>(st[b])) return;
  const int x = blockIdx.y;
  const int kz0 = blockIdx.x * TT;
  const int ny = g.ny, nzh = g.nzh;
  const int tid = threadIdx.x, nt = blockDim.x;
  C* base = spec + ((size_t)bc * g.nx + x) * (size_t)ny * nzh;
  const int work = ny * TT;
  for (int idx = tid; idx < work; idx += nt) {
    int y = idx / TT, t = idx - y * TT;
    int kz = kz0 + t;
    C v = mk<C>(0, 0);
    if (kz < nzh) v = base[(size_t)y * nzh + kz];
    if (inverse) v.y = -v.y;
    ybuf[idx] = v;
  }
  __syncthreads();
  fft_lines<VPT, true>(ybuf, TT, TT, 1, g.py, twiddles<T>(g.py));
  for (int idx = tid; idx < work; idx += nt) {
    int y = idx / TT, t = idx - y * TT;
    int kz = kz0 + t;
    C v = ybuf[idx];
    if (inverse) v.y = -v.y;
    if (kz < nzh) base[(size_t)y * nzh + kz] = v;
  }
}

// ----------------------------------------------------------------------------- x pass
// Block = (kz tile, ky, instance). Row kx of smem holds the 6*TT values
// (component c, column t) at c*TT + t.
template <typename T, int VPT>
__global__ void __launch_bounds__(kMaxThreads) xpass_kernel(GridDesc g, int TT,
                                                     cplx<T>* __restrict__ spec,
                                                     const Medium* __restrict__ med,
                                                     InstanceState* __restrict__ st,
                                                     double* __restrict__ partials) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char xraw[];
  C* xbuf = reinterpret_cast<C*>(xraw);
  __shared__ double red[32];
  const int b = blockIdx.z;
  if (!active<T>(st[b])) return;
  const int ky = blockIdx.y;
  const int kz0 = blockIdx.x * TT;
  const int nx = g.nx, ny = g.ny, nzh = g.nzh;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int W = 6 * TT;  // values per row
  C* sb = spec + (size_t)b * 6 * g.nm;
  const size_t cstride = (size_t)g.nm;               // component stride
  const size_t xstride = (size_t)ny * nzh;           // x stride
  const C* tw = twiddles<T>(g.px);

  const int work = nx * W;
  for (int idx = tid; idx < work; idx += nt) {
    int kx = idx / W, q = idx - kx * W;
    int c = q / TT, t = q - c * TT;
    int kz = kz0 + t;
    C v = mk<C>(0, 0);
    if (kz < nzh) v = sb[c * cstride + kx * xstride + (size_t)ky * nzh + kz];
    xbuf[idx] = v;
  }
  __syncthreads();
  fft_lines<VPT, true>(xbuf, W, W, 1, g.px, tw);

  // Residual partials, zero mode and Gamma^0 (written conjugated for the inverse DFT).
  const Medium& mb = med[b / g.lame_group];
  const T c_a = medium_ca<T>(mb), c_b = medium_cb<T>(mb);
  const double sxs = 2.0 * g.nx / g.Lx, sys = 2.0 * g.ny / g.Ly, szs = 2.0 * g.nz / g.Lz;
  double acc = 0.0;
  const int modes = nx * TT;
  for (int idx = tid; idx < modes; idx += nt) {
    int kx = idx / TT, t = idx - kx * TT;
    int kz = kz0 + t;
    if (kz >= nzh) continue;
    C* row = xbuf + (size_t)kx * W + t;
    C s[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) s[c] = row[c * TT];
    // modified wave vector tilde(xi) in FP64 (fourier.py:9-58 order of products)
    const double x0 = sxs * g.sx[kx] * g.cy[ky] * g.cz[kz];
    const double x1 = sys * g.cx[kx] * g.sy[ky] * g.cz[kz];
    const double x2 = szs * g.cx[kx] * g.cy[ky] * g.sz[kz];
    // divergence xi . sigma_hat in the field precision, weighted |.|^2 in FP64
    {
      const T f0 = (T)x0, f1 = (T)x1, f2 = (T)x2;
      C d0 = mk<C>(f0 * s[0].x + f1 * s[3].x + f2 * s[4].x, f0 * s[0].y + f1 * s[3].y + f2 * s[4].y);
      C d1 = mk<C>(f0 * s[3].x + f1 * s[1].x + f2 * s[5].x, f0 * s[3].y + f1 * s[1].y + f2 * s[5].y);
      C d2 = mk<C>(f0 * s[4].x + f1 * s[5].x + f2 * s[2].x, f0 * s[4].y + f1 * s[5].y + f2 * s[2].y);
      double m2 = (double)d0.x * d0.x + (double)d0.y * d0.y + (double)d1.x * d1.x +
                  (double)d1.y * d1.y + (double)d2.x * d2.x + (double)d2.y * d2.y;
      const double w = (kz == 0 || 2 * kz == g.nz) ? 1.0 : 2.0;
      acc += w * m2;
    }
    if (kx == 0 && ky == 0 && kz == 0) {
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        st[b].sig0[2 * c] = (double)s[c].x + (double)g.nv * st[b].shift[c];
        st[b].sig0[2 * c + 1] = (double)s[c].y;
      }
    }
    // normalised wave vector (fourier.py:61-85): FP64 with the 1e-12 guard
    double nrm = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
    const bool guarded = nrm < 1.0e-12;
    if (guarded) nrm = 1.0;
    if (g.c0) {
      // anisotropic reference stiffness: r = -Gamma^0 tau through the inverse acoustic
      // matrix (aniso.cuh); modes without a direction (the zero mode, the guarded ones)
      // get r = 0, the limit of the isotropic closed form there
      const double zd[3] = {x0 / nrm, x1 / nrm, x2 / nrm};
      double nd[6];
      const bool ok = !guarded && aniso_inverse_acoustic(g.c0 + (size_t)(b / g.lame_group) * 21, zd, nd);
      T o[2][6];
      if (ok) {
        const T zt[3] = {(T)zd[0], (T)zd[1], (T)zd[2]};
        T nt[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) nt[k] = (T)nd[k];
#pragma unroll
        for (int part = 0; part < 2; ++part) {
          T tv[6];
#pragma unroll
          for (int c = 0; c < 6; ++c) tv[c] = part ? s[c].y : s[c].x;
          aniso_gamma<T>(nt, zt, tv, o[part]);
        }
      } else {
#pragma unroll
        for (int c = 0; c < 6; ++c) o[0][c] = o[1][c] = (T)0;
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) row[c * TT] = mk<C>(o[0][c], -o[1][c]);
      continue;
    }
    const T z0 = (T)(x0 / nrm), z1 = (T)(x1 / nrm), z2 = (T)(x2 / nrm);
    // r_hat = C_A A(xi) sigma_hat + C_B (xi xi : sigma_hat) xi xi   (fourier.cu:268-327)
    const T z00 = z0 * z0, z11 = z1 * z1, z22 = z2 * z2;
    const T z01 = z0 * z1, z02 = z0 * z2, z12 = z1 * z2;
    T o[2][6];
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      T t0 = part ? s[0].y : s[0].x, t1 = part ? s[1].y : s[1].x, t2 = part ? s[2].y : s[2].x;
      T t3 = part ? s[3].y : s[3].x, t4 = part ? s[4].y : s[4].x, t5 = part ? s[5].y : s[5].x;
      T rho = z00 * t0 + z11 * t1 + z22 * t2 + (T)2 * (z01 * t3 + z02 * t4 + z12 * t5);
      T a0 = z0 * (z0 * t0 + z2 * t4 + z1 * t3);
      T a1 = z1 * (z1 * t1 + z2 * t5 + z0 * t3);
      T a2 = z2 * (z2 * t2 + z1 * t5 + z0 * t4);
      T a3 = (T)0.5 * (z01 * (t0 + t1) + (z00 + z11) * t3 + z2 * (z0 * t5 + z1 * t4));
      T a4 = (T)0.5 * (z02 * (t0 + t2) + (z00 + z22) * t4 + z1 * (z0 * t5 + z2 * t3));
      T a5 = (T)0.5 * (z12 * (t1 + t2) + (z11 + z22) * t5 + z0 * (z1 * t4 + z2 * t3));
      o[part][0] = c_a * a0 + c_b * rho * z00;
      o[part][1] = c_a * a1 + c_b * rho * z11;
      o[part][2] = c_a * a2 + c_b * rho * z22;
      o[part][3] = c_a * a3 + c_b * rho * z01;
      o[part][4] = c_a * a4 + c_b * rho * z02;
      o[part][5] = c_a * a5 + c_b * rho * z12;
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) row[c * TT] = mk<C>(o[0][c], -o[1][c]);
  }
  __syncthreads();
  fft_lines<VPT, true>(xbuf, W, W, 1, g.px, tw);
  for (int idx = tid; idx < work; idx += nt) {
    int kx = idx / W, q = idx - kx * W;
    int c = q / TT, t = q - c * TT;
    int kz = kz0 + t;
    if (kz < nzh) {
      C v = xbuf[idx];
      sb[c * cstride + kx * xstride + (size_t)ky * nzh + kz] = mk<C>(v.x, -v.y);
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
// Criterion (lippmann_schwinger.py:118-143 / lippmann_schwinger.cu:95-109), the stop
// rule (lippmann_schwinger.cu:201-206; lippmann_schwinger.py:196-206) and, for mixed
// precision, the switch to FP64 fields once FP32 round-off stalls the criterion near
// the tolerance.
__global__ void finalize_kernel(int nblk, int phase, InstanceState* __restrict__ st,
                                const double* __restrict__ partials, double* __restrict__ history,
                                int history_len, SolveParams sp) {
  __shared__ double red[32];
  const int b = blockIdx.x;
  InstanceState& s = st[b];
  if (s.done || s.phase != phase) return;
  const int tid = threadIdx.x, nt = blockDim.x;
  double acc = 0.0;
  for (int i = tid; i < nblk; i += nt) acc += partials[(size_t)b * nblk + i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((tid & 31) == 0) red[tid >> 5] = acc;
  __syncthreads();
  if (tid != 0) return;
  double num2 = 0.0;
  for (int w = 0; w < (nt + 31) / 32; ++w) num2 += red[w];
  double den2 = 0.0;
  for (int c = 0; c < 6; ++c) {
    double m2 = s.sig0[2 * c] * s.sig0[2 * c] + s.sig0[2 * c + 1] * s.sig0[2 * c + 1];
    den2 += (c < 3 ? 1.0 : 2.0) * m2;
  }
  const double e = (num2 == 0.0) ? 0.0 : sqrt(num2) / sqrt(den2);
  if (s.evals == 0) {
    s.e0 = e;
    s.best_e = e;
    s.best_eval = 0;
  }
  if (history != nullptr && s.evals < history_len) history[(size_t)b * history_len + s.evals] = e;
  s.evals += 1;
  s.e = e;
  const double thr = fmax(sp.rtol * (s.e0_ref > 0.0 ? s.e0_ref : s.e0), sp.atol);
  const bool conv = sp.rule == 0 ? (e < thr) : (e <= thr);
  // the next forward transform is shifted by the current mean stress
  const double inv_nv = 1.0 / (double)sp.nv;
  for (int c = 0; c < 6; ++c) s.shift[c] = s.sig0[2 * c] * inv_nv;
  if (!isfinite(e)) {
    s.done = 1;
    s.status = kNonFinite;
    return;
  }
  if (conv) {
    s.done = 1;
    s.status = kConverged;
    return;
  }
  if (s.iter >= sp.maxiter) {
    s.done = 1;
    s.status = kMaxIter;
    return;
  }
  if (e < sp.stall_improve * s.best_e) s.best_eval = s.evals;
  if (e < s.best_e) s.best_e = e;
  const bool stalled = phase == 0 && sp.precision != kPrecFP64 && sp.stall_window > 0 &&
                       s.best_e < sp.stall_near * thr &&
                       s.evals - s.best_eval >= sp.stall_window;
  if (stalled) {
    if (sp.precision == kPrecMixed) {
      // continue from this iterate with FP64 fields; no FP32 update for this evaluation
      s.phase = 1;
      s.switched = 1;
      s.switch_iter = s.iter;
      s.best_eval = s.evals;
    } else {
      s.done = 1;
      s.status = kStalled;
    }
    return;
  }
  s.iter += 1;
}

// Ring access of VW consecutive elements: float4 for VW = 4 (FP32 rings whose slot length
// 6 nv is a multiple of 4, so that every slot starts 16-byte aligned), scalars otherwise.
// Wide loads keep four times the bytes in flight per load, which the streaming kernels
// below need at their register-limited occupancy.
template <typename T, int VW>
struct RingVec { using type = T; };
template <>
struct RingVec<float, 4> { using type = float4; };
template <typename T>
__device__ __forceinline__ T lane_of(const T& v, int) { return v; }
__device__ __forceinline__ float lane_of(const float4& v, int k) {
  return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}

// Gram-row partials of the newest residual r_j (slot j of the ring) for every instance in
// `phase`: partials[b][blk][q] = sum over block blk's ring elements (component c, voxel) of
// w_c r_j r_q, with Voigt weights w = (1,1,1,2,2,2), accumulated in FP64
// (lippmann_schwinger.py:217-231); partials[b][blk][M1] = the block's max |r_j|.
// FP32 phase: the ring holds FP16 values r_q 2^k_q; eight neighbouring weighted products are
// summed in FP32, the sum added in FP64 (the kernel is bound by its FP64 issue rate
// otherwise), and the block's sums are scaled back by 2^-(k_j + k_q) (exact). The rounding
// of the stored residuals is independent from element to element, so it averages out of
// the sums: relative to the FP32 ring the Gram entries change by about 2^-11 / sqrt(n).
// A streaming kernel of its own, walking the 6 nv elements of a slot as the combine does, VW
// elements per load (16 bytes of FP16 for VW = 8), every slot of an element requested
// before the first product (M1 = depth + 1 slots, a template constant).
__device__ __forceinline__ void unpack8(const uint4& u, float* f) {
  const unsigned w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float2 t = __half22float2(*reinterpret_cast<const __half2*>(&w[k]));
    f[2 * k] = t.x;
    f[2 * k + 1] = t.y;
  }
}

template <typename T, int M1, int VW>
__global__ void __launch_bounds__(256, M1 <= 6 ? 4 : 3) anderson_gram_kernel(long long nv, int phase,
                                                            const InstanceState* __restrict__ st,
                                                            const typename ResRing<T>::type* __restrict__ r,
                                                            double* __restrict__ partials) {
  using R = typename ResRing<T>::type;
  __shared__ double red[kMaxDepth + 1][32];
  __shared__ float redm[32];
  const int b = blockIdx.y;
  const InstanceState& s = st[b];
  if (s.done || s.phase != phase) return;
  int slot, filled;
  anderson_slots<T>(s, M1 - 1, slot, filled);
  const long long n6 = 6 * nv, nvec = n6 / VW, n3 = 3 * nv;
  const R* rb = r + (size_t)b * M1 * n6;
  double dots[M1];
#pragma unroll
  for (int q = 0; q < M1; ++q) dots[q] = 0.0;
  float amax = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvec;
       i += (long long)gridDim.x * blockDim.x) {
    if constexpr (sizeof(T) == 4 && VW == 8) {
      uint4 rq[M1];
#pragma unroll
      for (int q = 0; q < M1; ++q)
        if (q < filled) rq[q] = reinterpret_cast<const uint4*>(rb + (size_t)q * n6)[i];
      uint4 xu = rq[0];
#pragma unroll
      for (int q = 1; q < M1; ++q) xu = q == slot ? rq[q] : xu;
      float wx[8];
      unpack8(xu, wx);
      const long long e0 = i * 8;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        amax = fmaxf(amax, fabsf(wx[k]));
        if (e0 + k >= n3) wx[k] *= 2.f;
      }
#pragma unroll
      for (int q = 0; q < M1; ++q)
        if (q < filled) {
          float f[8];
          unpack8(rq[q], f);
          float sum = 0.f;
#pragma unroll
          for (int k = 0; k < 8; ++k) sum = fmaf(wx[k], f[k], sum);
          dots[q] += (double)sum;
        }
    } else if constexpr (sizeof(T) == 4) {
      float rq[M1];
#pragma unroll
      for (int q = 0; q < M1; ++q)
        if (q < filled) rq[q] = __half2float(rb[(size_t)q * n6 + i]);
      float x = rq[0];
#pragma unroll
      for (int q = 1; q < M1; ++q) x = q == slot ? rq[q] : x;
      amax = fmaxf(amax, fabsf(x));
      const float wx = (i < n3 ? 1.f : 2.f) * x;
#pragma unroll
      for (int q = 0; q < M1; ++q)
        if (q < filled) dots[q] += (double)(wx * rq[q]);
    } else {
      T rq[M1];
#pragma unroll
      for (int q = 0; q < M1; ++q)
        if (q < filled) rq[q] = rb[(size_t)q * n6 + i];
      T x = rq[0];
#pragma unroll
      for (int q = 1; q < M1; ++q) x = q == slot ? rq[q] : x;
      const double wx = (i < n3 ? 1.0 : 2.0) * (double)x;
#pragma unroll
      for (int q = 0; q < M1; ++q)
        if (q < filled) dots[q] += wx * (double)rq[q];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  if ((threadIdx.x & 31) == 0) redm[threadIdx.x >> 5] = amax;
  double pad[kMaxDepth + 1];
#pragma unroll
  for (int q = 0; q <= kMaxDepth; ++q) pad[q] = q < M1 ? dots[q < M1 ? q : 0] : 0.0;
  double out[kMaxDepth + 1];
  block_sum_slots(pad, filled, red, out);  // (its barrier also orders redm)
  double* pb = partials + ((size_t)b * gridDim.x + blockIdx.x) * (M1 + 1);
  const int t = threadIdx.x;
  if (t < filled) {
    double v = out[t];
    if constexpr (sizeof(T) == 4) v = ldexp(v, -(s.ring_exp[slot] + s.ring_exp[t]));
    pb[t] = v;
  }
  if (t == 0) {
    float m = 0.f;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) m = fmaxf(m, redm[w]);
    pb[M1] = sizeof(T) == 4 ? ldexp((double)m, -s.ring_exp[slot]) : 0.0;
  }
}

// Anderson combine for every instance in `phase`: eps = sum_s alpha_s g_s over the filled
// slots (lippmann_schwinger.py:228-231), accumulated in the field precision in slot order,
// VW elements per load.
template <typename T, int M1, int VW>
__global__ void __launch_bounds__(256) anderson_combine_kernel(long long n6, int phase,
                                                               const InstanceState* __restrict__ st,
                                                               const T* __restrict__ g,
                                                               const double* __restrict__ alpha,
                                                               const T* __restrict__ inject,
                                                               T* __restrict__ eps) {
  using V = typename RingVec<T, VW>::type;
  const int b = blockIdx.y;
  const InstanceState& s = st[b];
  if (s.done || s.phase != phase) return;
  int slot, filled;
  anderson_slots<T>(s, M1 - 1, slot, filled);
  const T* gb = g + (size_t)b * M1 * n6;
  const double* al = alpha + (size_t)b * M1;
  T a[M1];
#pragma unroll
  for (int q = 0; q < M1; ++q) a[q] = q < filled ? (T)al[q] : (T)0;
  T* eb = eps + (size_t)b * n6;
  const long long nvec = n6 / VW;
  if (inject && s.iter == 1 && s.aa_base == 0) {
    // first update with a warm start in the history: the next iterate is the given field,
    // whose residual then enters the ring beside the cold start's
    const T* ib = inject + (size_t)b * n6;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n6;
         i += (long long)gridDim.x * blockDim.x)
      eb[i] = ib[i];
    return;
  }
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvec;
       i += (long long)gridDim.x * blockDim.x) {
    V gv[M1];
#pragma unroll
    for (int q = 0; q < M1; ++q)
      if (q < filled) gv[q] = reinterpret_cast<const V*>(gb + (size_t)q * n6)[i];
    if constexpr (VW == 4 && sizeof(T) == 4) {
      float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int q = 0; q < M1; ++q)
        if (q < filled) {
          e.x += a[q] * gv[q].x;
          e.y += a[q] * gv[q].y;
          e.z += a[q] * gv[q].z;
          e.w += a[q] * gv[q].w;
        }
      reinterpret_cast<float4*>(eb)[i] = e;
    } else {
      T e = 0;
#pragma unroll
      for (int q = 0; q < M1; ++q)
        if (q < filled) e += a[q] * gv[q];
      eb[i] = e;
    }
  }
}


// Anderson mixing coefficients (lippmann_schwinger.py:219-228): the new Gram row
// <r_j, r_s>_w replaces row and column `slot` of A (the reference's roll of A is a
// relabelling of the ring), A v = 1 is solved over the filled slots in FP64 by Gaussian
// elimination with partial pivoting, alpha = v / sum(v). A singular or non-finite solve
// falls back to the plain update alpha = e_slot.
// The Gram row's block partials (nzblk rows of M1 values and the block's max |r_j|) are
// summed by the whole block, each thread over a few rows with independent loads, then
// across warps; the max of the newest residual goes to the instance state, for the scale of
// the next FP16 slot. A is staged in shared memory. The elimination runs on one thread over an M1 x M1 system held in
// registers (compile-time M1): rows and columns past `filled` are an identity block with a
// zero right-hand side, which leaves the filled block's arithmetic, pivots and solution
// as they are and gives v = 0 on the padding.
constexpr int kSolveThreads = 256;
template <int M1>
__global__ void __launch_bounds__(kSolveThreads) anderson_solve_kernel(
    int nzblk, int phase, InstanceState* __restrict__ st,
    const double* __restrict__ partials, double* __restrict__ amat, double* __restrict__ alpha) {
  __shared__ double red[kSolveThreads / 32][M1 + 1];
  __shared__ double sA[M1 * M1];
  const int b = blockIdx.x;
  InstanceState& s = st[b];
  if (s.done || s.phase != phase) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int slot, filled;
  anderson_slots<double>(s, M1 - 1, slot, filled);
  double* A = amat + (size_t)b * M1 * M1;
  if (tid < M1 * M1) sA[tid] = A[tid];
  double a[M1];
#pragma unroll
  for (int q = 0; q < M1; ++q) a[q] = 0.0;
  double mx = 0.0;
  const double* pb = partials + (size_t)b * nzblk * (M1 + 1);
#pragma unroll 4
  for (int i = tid; i < nzblk; i += kSolveThreads) {
#pragma unroll
    for (int q = 0; q < M1; ++q)
      if (q < filled) a[q] += pb[(size_t)i * (M1 + 1) + q];
    mx = fmax(mx, pb[(size_t)i * (M1 + 1) + M1]);
  }
#pragma unroll
  for (int q = 0; q < M1; ++q) {
    if (q >= filled) break;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a[q] += __shfl_xor_sync(0xffffffffu, a[q], o);
    if (lane == 0) red[warp][q] = a[q];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0) red[warp][M1] = mx;
  __syncthreads();
  if (tid == M1) {
    double m = 0.0;
    for (int w = 0; w < kSolveThreads / 32; ++w) m = fmax(m, red[w][M1]);
    // (a residual whose stored values all underflowed FP16 at this slot's scale reports
    // the underflow threshold instead of 0, so that the next slot's scale rises by 2^34
    // rather than falling back to the first slot's guess)
    if (phase == 0) s.ring_max = m > 0.0 ? (float)m : ldexpf(1.f, -25 - s.ring_exp[slot]);
  }
  if (tid < filled) {
    double t = 0.0;
    for (int w = 0; w < kSolveThreads / 32; ++w) t += red[w][tid];
    sA[slot * M1 + tid] = t;
    sA[tid * M1 + slot] = t;
    A[slot * M1 + tid] = t;
    A[tid * M1 + slot] = t;
  }
  __syncthreads();
  if (tid != 0) return;
  double m[M1][M1 + 1];
#pragma unroll
  for (int i = 0; i < M1; ++i) {
#pragma unroll
    for (int j = 0; j < M1; ++j)
      m[i][j] = (i < filled && j < filled) ? sA[i * M1 + j] : (i == j ? 1.0 : 0.0);
    m[i][M1] = i < filled ? 1.0 : 0.0;
  }
  // (constant trip counts with guards, so that every index is a compile-time constant and
  // m stays in registers)
  bool ok = true;
#pragma unroll
  for (int c = 0; c < M1; ++c) {
    int piv = c;
    double pv = fabs(m[c][c]);
#pragma unroll
    for (int i = 0; i < M1; ++i)
      if (i > c) {
        const double av = fabs(m[i][c]);
        if (av > pv) { pv = av; piv = i; }
      }
    // (a zero pivot ends the solve; the remaining columns' arithmetic is discarded)
    if (!(pv > 0.0)) ok = false;
#pragma unroll
    for (int i = 0; i < M1; ++i)
      if (i > c) {
        const bool sw = piv == i;
#pragma unroll
        for (int j = 0; j <= M1; ++j)
          if (j >= c) {
            const double x = m[c][j], y = m[i][j];
            m[c][j] = sw ? y : x;
            m[i][j] = sw ? x : y;
          }
      }
#pragma unroll
    for (int i = 0; i < M1; ++i)
      if (i > c) {
        const double f = m[i][c] / m[c][c];
#pragma unroll
        for (int j = 0; j <= M1; ++j)
          if (j >= c) m[i][j] -= f * m[c][j];
      }
  }
  double v[M1];
  double sum = 0.0;
  if (ok) {
#pragma unroll
    for (int i = M1 - 1; i >= 0; --i) {
      double t = m[i][M1];
#pragma unroll
      for (int j = 0; j < M1; ++j)
        if (j > i) t -= m[i][j] * v[j];
      v[i] = t / m[i][i];
      sum += v[i];
    }
    ok = isfinite(sum) && sum != 0.0;
  }
  double* al = alpha + (size_t)b * M1;
#pragma unroll
  for (int q = 0; q < M1; ++q) al[q] = ok ? (q < filled ? v[q] / sum : 0.0) : (q == slot ? 1.0 : 0.0);
}

__global__ void reset_state_kernel(int batch, int phase, const double* e0_ref, InstanceState* st) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < batch) {
    InstanceState z = {};
    z.phase = phase;
    z.e0_ref = e0_ref ? e0_ref[b] : 0.0;
    st[b] = z;
  }
}

// ----------------------------------------------------------------------------- medium
// Structure blockIdx.y of [structure][nv] fields; partials to scratch[structure][block][6].
template <typename TL>
__global__ void minmax_partial_kernel(long long nv, const TL* __restrict__ lambda,
                                      const TL* __restrict__ mu, double* __restrict__ scratch) {
  __shared__ double sh[6][32];
  lambda += (size_t)blockIdx.y * nv;
  mu += (size_t)blockIdx.y * nv;
  scratch += (size_t)blockIdx.y * gridDim.x * 6;
  double lmin = DBL_MAX, lmax = -DBL_MAX, mmin = DBL_MAX, mmax = -DBL_MAX;
  double lsum = 0.0, msum = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
       i += (long long)gridDim.x * blockDim.x) {
    double l = lambda[i], m = mu[i];
    lmin = fmin(lmin, l); lmax = fmax(lmax, l);
    mmin = fmin(mmin, m); mmax = fmax(mmax, m);
    lsum += l;
    msum += m;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lmin = fmin(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
    lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    mmin = fmin(mmin, __shfl_xor_sync(0xffffffffu, mmin, o));
    mmax = fmax(mmax, __shfl_xor_sync(0xffffffffu, mmax, o));
    lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    msum += __shfl_xor_sync(0xffffffffu, msum, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    sh[0][w] = lmin; sh[1][w] = lmax; sh[2][w] = mmin; sh[3][w] = mmax;
    sh[4][w] = lsum; sh[5][w] = msum;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (blockDim.x + 31) / 32; ++i) {
      lmin = fmin(lmin, sh[0][i]); lmax = fmax(lmax, sh[1][i]);
      mmin = fmin(mmin, sh[2][i]); mmax = fmax(mmax, sh[3][i]);
      lsum += sh[4][i];
      msum += sh[5][i];
    }
    double* o = scratch + 6 * blockIdx.x;
    o[0] = lmin; o[1] = lmax; o[2] = mmin; o[3] = mmax; o[4] = lsum; o[5] = msum;
  }
}

// One warp per structure: Medium med[structure] from its nblk partials (lane-strided
// partial sums, then a fixed xor tree: deterministic).
__global__ void minmax_final_kernel(int nblk, long long nv, int fp64_fields,
                                    const double* __restrict__ scratch, Medium* med) {
  const int lane = threadIdx.x;
  scratch += (size_t)blockIdx.x * nblk * 6;
  med += blockIdx.x;
  double lmin = DBL_MAX, lmax = -DBL_MAX, mmin = DBL_MAX, mmax = -DBL_MAX;
  double lsum = 0.0, msum = 0.0;
  for (int i = lane; i < nblk; i += 32) {
    const double* o = scratch + 6 * i;
    lmin = fmin(lmin, o[0]); lmax = fmax(lmax, o[1]);
    mmin = fmin(mmin, o[2]); mmax = fmax(mmax, o[3]);
    lsum += o[4];
    msum += o[5];
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    lmin = fmin(lmin, __shfl_xor_sync(0xffffffffu, lmin, off));
    lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, off));
    mmin = fmin(mmin, __shfl_xor_sync(0xffffffffu, mmin, off));
    mmax = fmax(mmax, __shfl_xor_sync(0xffffffffu, mmax, off));
    lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
    msum += __shfl_xor_sync(0xffffffffu, msum, off);
  }
  if (lane != 0) return;
  Medium m;
  m.lmin = lmin; m.lmax = lmax; m.mmin = mmin; m.mmax = mmax;
  m.lmean = lsum / (double)nv;
  m.mmean = msum / (double)nv;
  // lambda0 = 1/2 (min + max) in the field precision (lippmann_schwinger.py:171-172)
  m.lambda0 = 0.5f * ((float)lmin + (float)lmax);
  m.mu0 = 0.5f * ((float)mmin + (float)mmax);
  m.c_a = (float)(-1.0 / (double)m.mu0);
  m.c_b = (float)(((double)m.lambda0 + m.mu0) / ((double)m.mu0 * ((double)m.lambda0 + 2.0 * m.mu0)));
  if (fp64_fields) {
    m.lambda0_64 = 0.5 * (lmin + lmax);
    m.mu0_64 = 0.5 * (mmin + mmax);
  } else {
    m.lambda0_64 = m.lambda0;
    m.mu0_64 = m.mu0;
  }
  m.c_a64 = -1.0 / m.mu0_64;
  m.c_b64 = (m.lambda0_64 + m.mu0_64) / (m.mu0_64 * (m.lambda0_64 + 2.0 * m.mu0_64));
  *med = m;
}

// ----------------------------------------------------------------------------- conversions
// out[b] = in[b] for every instance b with phase == 1 (and, if only_running, not done).
template <typename Tin, typename Tout>
__global__ void convert_fields_kernel(long long n_per_instance, int only_running,
                                      const InstanceState* __restrict__ st,
                                      const Tin* __restrict__ in, Tout* __restrict__ out) {
  const int b = blockIdx.y;
  if (st[b].phase != 1 || (only_running && st[b].done)) return;
  const Tin* ib = in + (size_t)b * n_per_instance;
  Tout* ob = out + (size_t)b * n_per_instance;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_per_instance;
       i += (long long)gridDim.x * blockDim.x)
    ob[i] = (Tout)ib[i];
}

template <typename Tin, typename Tout>
__global__ void convert_plain_kernel(long long n, const Tin* __restrict__ in, Tout* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = (Tout)in[i];
}

// ----------------------------------------------------------------------------- stress
// sigma = C : eps for every instance of the given phase; sigma is written in TS.
template <typename T, typename TS>
__global__ void stress_kernel(long long nv, int phase, int lame_group, const InstanceState* __restrict__ st,
                              const T* __restrict__ lambda, const T* __restrict__ mu,
                              const T* __restrict__ eps, TS* __restrict__ sigma,
                              double* __restrict__ scratch, const T* __restrict__ dmg, T dmg_k,
                              const T* __restrict__ cf) {
  __shared__ double sh[6][32];
  const int b = blockIdx.y;
  if (st[b].phase != phase) return;
  lambda += (size_t)(b / lame_group) * nv;
  mu += (size_t)(b / lame_group) * nv;
  if (dmg) dmg += (size_t)(b / lame_group) * nv;
  if (cf) cf += (size_t)(b / lame_group) * 21 * nv;
  const T* eb = eps + (size_t)b * 6 * nv;
  TS* sg = sigma ? sigma + (size_t)b * 6 * nv : nullptr;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
       i += (long long)gridDim.x * blockDim.x) {
    T e[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) e[c] = eb[(size_t)c * nv + i];
    T s[6];
    if (cf) {
      aniso_stress<T>([&](int k) { return cf[(size_t)k * nv + i]; }, e, s);
    } else if (dmg) {
      const T om = (T)1 - dmg[i];
      damaged_stress<T>(e, lambda[i], mu[i], om * om + dmg_k, s);
    } else {
      const T lam = lambda[i], tmu = (T)2 * mu[i];
      const T ltr = lam * (e[0] + e[1] + e[2]);
#pragma unroll
      for (int c = 0; c < 3; ++c) s[c] = tmu * e[c] + ltr;
#pragma unroll
      for (int c = 3; c < 6; ++c) s[c] = tmu * e[c];
    }
    if (sg) {
#pragma unroll
      for (int c = 0; c < 6; ++c) sg[(size_t)c * nv + i] = (TS)s[c];
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[c] += (double)s[c];
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

__global__ void mean_final_kernel(int nblk, long long nv, int phase,
                                  const InstanceState* __restrict__ st,
                                  const double* __restrict__ scratch, double* __restrict__ mean) {
  const int bc = blockIdx.x;  // instance * 6 + component
  if (threadIdx.x != 0 || st[bc / 6].phase != phase) return;
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

LaunchShape plan_launch(const GridDesc& g, int elem_bytes) {
  LaunchShape s;
  const long long kElems = kPassBytes / elem_bytes;
  // z pass: 3 complex lines of nz per (x, y) line
  s.lines_per_block = (int)std::max<long long>(1, kElems / (3LL * g.nz));
  s.lines_per_block = (int)std::min<long long>(s.lines_per_block, (long long)g.nx * g.ny);
  s.z_threads = threads_for(g.pz, 3LL * s.lines_per_block * g.nz, kVPT);
  while (s.z_threads > kMaxThreads && s.lines_per_block > 1) {
    s.lines_per_block -= 1;
    s.z_threads = threads_for(g.pz, 3LL * s.lines_per_block * g.nz, kVPT);
  }
  s.z_blocks = (int)(((long long)g.nx * g.ny + s.lines_per_block - 1) / s.lines_per_block);
  s.z_smem = (size_t)3 * s.lines_per_block * g.nz * elem_bytes;
  // y pass
  s.ty = std::max(1, std::min(16, (int)(kElems / g.ny)));
  s.ty = std::min(s.ty, g.nzh);
  s.y_threads = threads_for(g.py, (long long)g.ny * s.ty, kVPT);
  while (s.y_threads > kMaxThreads && s.ty > 1) {
    s.ty -= 1;
    s.y_threads = threads_for(g.py, (long long)g.ny * s.ty, kVPT);
  }
  s.y_tiles = (g.nzh + s.ty - 1) / s.ty;
  s.y_smem = (size_t)g.ny * s.ty * elem_bytes;
  // x pass
  s.tx = std::max(1, std::min(16, pick_pow2_leq((int)std::max<long long>(1, kElems / (6LL * g.nx)))));
  s.tx = std::min(s.tx, g.nzh);
  s.x_threads = threads_for(g.px, 6LL * g.nx * s.tx, kVPT);
  while (s.x_threads > kMaxThreads && s.tx > 1) {
    s.tx /= 2;
    s.x_threads = threads_for(g.px, 6LL * g.nx * s.tx, kVPT);
  }
  s.x_tiles = (g.nzh + s.tx - 1) / s.tx;
  s.x_smem = (size_t)6 * g.nx * s.tx * elem_bytes;
  s.x_blocks_per_instance = s.x_tiles * g.ny;
  return s;
}

// Every pass is planned with at most kPassBytes of dynamic shared memory, so one fixed
// opt-in serves all solvers alive in the process.
template <typename T>
static cudaError_t configure_for() {
  const int bytes = (int)kPassBytes;
  cudaError_t e;
  e = cudaFuncSetAttribute(zpass_kernel<T, kVPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(ypass_kernel<T, kVPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(xpass_kernel<T, kVPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

cudaError_t configure_kernels() {
  cudaError_t e = configure_for<float>();
  if (e != cudaSuccess) return e;
  return configure_for<double>();
}

template <typename T>
void launch_zpass(const GridDesc& g, const LaunchShape& s, int mode, int batch, const T* lambda,
                  const T* mu, T* eps, cplx<T>* spec, const double* eps_bar, const T* eps0,
                  InstanceState* st, const Medium* med, const AndersonArgs<T>& aa,
                  cudaStream_t stream) {
  dim3 grid(s.z_blocks, batch);
  zpass_kernel<T, kVPT><<<grid, s.z_threads, s.z_smem, stream>>>(
      g, mode, s.lines_per_block, lambda, mu, eps, spec, eps_bar, eps0, st, med, aa);
}

void launch_anderson_solve(int nzblk, int depth, int phase, int batch, InstanceState* st,
                           const double* partials, double* amat, double* alpha, cudaStream_t stream) {
  switch (depth + 1) {
#define LSB_SOLVE(M)                                                                          \
    case M:                                                                                   \
      anderson_solve_kernel<M><<<batch, kSolveThreads, 0, stream>>>(nzblk, phase, st, partials, \
                                                                    amat, alpha);              \
      break;
    LSB_SOLVE(2) LSB_SOLVE(3) LSB_SOLVE(4) LSB_SOLVE(5) LSB_SOLVE(6) LSB_SOLVE(7) LSB_SOLVE(8) LSB_SOLVE(9)
#undef LSB_SOLVE
    default: break;
  }
}

template <typename T>
void launch_anderson_gram(long long nv, int nblk, int depth, int phase, int batch,
                          const InstanceState* st, const typename ResRing<T>::type* r,
                          double* partials, cudaStream_t stream) {
  const dim3 grid(nblk, batch);
  const bool vec = sizeof(T) == 4 && (6 * nv) % 8 == 0;
  switch (depth + 1) {
#define LSB_GRAM(M)                                                                              \
    case M:                                                                                      \
      if constexpr (sizeof(T) == 4) {                                                            \
        if (vec) {                                                                               \
          anderson_gram_kernel<T, M, 8><<<grid, 256, 0, stream>>>(nv, phase, st, r, partials); \
          break;                                                                                 \
        }                                                                                        \
      }                                                                                          \
      anderson_gram_kernel<T, M, 1><<<grid, 256, 0, stream>>>(nv, phase, st, r, partials);     \
      break;
    LSB_GRAM(2) LSB_GRAM(3) LSB_GRAM(4) LSB_GRAM(5) LSB_GRAM(6) LSB_GRAM(7) LSB_GRAM(8) LSB_GRAM(9)
#undef LSB_GRAM
    default: break;
  }
}

template <typename T>
void launch_anderson_combine(long long nv, int depth, int phase, int batch, const InstanceState* st,
                             const T* g, const double* alpha, T* eps, cudaStream_t stream,
                             const T* inject) {
  const long long n6 = 6 * nv;
  const dim3 grid((unsigned)std::min<long long>(2048, (n6 + 255) / 256), batch);
  const bool vec = sizeof(T) == 4 && n6 % 4 == 0;
  switch (depth + 1) {
#define LSB_COMB(M)                                                                                        \
    case M:                                                                                                \
      if constexpr (sizeof(T) == 4) {                                                                      \
        if (vec) {                                                                                         \
          anderson_combine_kernel<T, M, 4><<<grid, 256, 0, stream>>>(n6, phase, st, g, alpha, inject, eps); \
          break;                                                                                           \
        }                                                                                                  \
      }                                                                                                    \
      anderson_combine_kernel<T, M, 1><<<grid, 256, 0, stream>>>(n6, phase, st, g, alpha, inject, eps);     \
      break;
    LSB_COMB(2) LSB_COMB(3) LSB_COMB(4) LSB_COMB(5) LSB_COMB(6) LSB_COMB(7) LSB_COMB(8) LSB_COMB(9)
#undef LSB_COMB
    default: break;
  }
}

template <typename T>
void launch_ypass(const GridDesc& g, const LaunchShape& s, bool inverse, int batch, cplx<T>* spec,
                  const InstanceState* st, cudaStream_t stream) {
  dim3 grid(s.y_tiles, g.nx, 6 * batch);
  ypass_kernel<T, kVPT><<<grid, s.y_threads, s.y_smem, stream>>>(g, inverse ? 1 : 0, s.ty, spec, st);
}

template <typename T>
void launch_xpass(const GridDesc& g, const LaunchShape& s, int batch, cplx<T>* spec, const Medium* med,
                  InstanceState* st, double* partials, cudaStream_t stream) {
  dim3 grid(s.x_tiles, g.ny, batch);
  xpass_kernel<T, kVPT><<<grid, s.x_threads, s.x_smem, stream>>>(g, s.tx, spec, med, st, partials);
}

void launch_finalize(const LaunchShape& s, int phase, int batch, InstanceState* st,
                     const double* partials, double* history, int history_len,
                     const SolveParams& sp, cudaStream_t stream) {
  finalize_kernel<<<batch, 256, 0, stream>>>(s.x_blocks_per_instance, phase, st, partials, history,
                                              history_len, sp);
}

void launch_reset_state(int batch, int phase, InstanceState* st, cudaStream_t stream,
                        const double* e0_ref) {
  reset_state_kernel<<<(batch + 127) / 128, 128, 0, stream>>>(batch, phase, e0_ref, st);
}

template <typename TL>
void launch_medium(long long nv, int nstruct, const TL* lambda, const TL* mu, double* scratch,
                   Medium* med, cudaStream_t stream) {
  int nblk = (int)std::min<long long>(std::max(1, 1024 / nstruct), (nv + 255) / 256);
  if (nblk < 1) nblk = 1;
  minmax_partial_kernel<TL><<<dim3(nblk, nstruct), 256, 0, stream>>>(nv, lambda, mu, scratch);
  minmax_final_kernel<<<nstruct, 32, 0, stream>>>(nblk, nv, sizeof(TL) == 8 ? 1 : 0, scratch, med);
}

template <typename Tin, typename Tout>
void launch_convert_fields(long long n_per_instance, int batch, int only_running,
                           const InstanceState* st, const Tin* in, Tout* out, cudaStream_t stream) {
  int nblk = (int)std::min<long long>(2048, (n_per_instance + 255) / 256);
  dim3 grid(std::max(nblk, 1), batch);
  convert_fields_kernel<Tin, Tout><<<grid, 256, 0, stream>>>(n_per_instance, only_running, st, in, out);
}

template <typename Tin, typename Tout>
void launch_convert(long long n, const Tin* in, Tout* out, cudaStream_t stream) {
  int nblk = (int)std::min<long long>(2048, (n + 255) / 256);
  convert_plain_kernel<Tin, Tout><<<std::max(nblk, 1), 256, 0, stream>>>(n, in, out);
}

template <typename T, typename TS>
void launch_stress(const GridDesc& g, int phase, int batch, const InstanceState* st,
                   const T* lambda, const T* mu, const T* eps, TS* sigma, double* scratch,
                   double* mean, cudaStream_t stream) {
  int nblk = (int)std::min<long long>(1024, (g.nv + 255) / 256);
  if (nblk < 1) nblk = 1;
  dim3 grid(nblk, batch);
  stress_kernel<T, TS><<<grid, 256, 0, stream>>>(g.nv, phase, g.lame_group, st, lambda, mu, eps, sigma,
                                                  mean ? scratch : nullptr, damage_field<T>(g),
                                                  (T)g.dmg_k, stiffness_field<T>(g));
  if (mean) mean_final_kernel<<<6 * batch, 32, 0, stream>>>(nblk, g.nv, phase, st, scratch, mean);
}

// explicit instantiations
#define LSB_INST(T)                                                                             \
  template void launch_zpass<T>(const GridDesc&, const LaunchShape&, int, int, const T*,        \
                                const T*, T*, cplx<T>*, const double*, const T*, InstanceState*, \
                                const Medium*, const AndersonArgs<T>&, cudaStream_t);           \
  template void launch_ypass<T>(const GridDesc&, const LaunchShape&, bool, int, cplx<T>*,       \
                                const InstanceState*, cudaStream_t);                            \
  template void launch_xpass<T>(const GridDesc&, const LaunchShape&, int, cplx<T>*,             \
                                const Medium*, InstanceState*, double*, cudaStream_t);          \
  template void launch_medium<T>(long long, int, const T*, const T*, double*, Medium*, cudaStream_t); \
  template void launch_anderson_gram<T>(long long, int, int, int, int, const InstanceState*,    \
                                        const typename ResRing<T>::type*, double*, cudaStream_t); \
  template void launch_anderson_combine<T>(long long, int, int, int, const InstanceState*,      \
                                           const T*, const double*, T*, cudaStream_t, const T*);
LSB_INST(float)
LSB_INST(double)
#undef LSB_INST
template void launch_convert_fields<float, double>(long long, int, int, const InstanceState*,
                                                   const float*, double*, cudaStream_t);
template void launch_convert_fields<double, float>(long long, int, int, const InstanceState*,
                                                   const double*, float*, cudaStream_t);
template void launch_convert<float, double>(long long, const float*, double*, cudaStream_t);
template void launch_convert<double, float>(long long, const double*, float*, cudaStream_t);
template void launch_stress<float, float>(const GridDesc&, int, int, const InstanceState*, const float*,
                                          const float*, const float*, float*, double*, double*,
                                          cudaStream_t);
template void launch_stress<double, float>(const GridDesc&, int, int, const InstanceState*,
                                           const double*, const double*, const double*, float*,
                                           double*, double*, cudaStream_t);
template void launch_stress<double, double>(const GridDesc&, int, int, const InstanceState*,
                                            const double*, const double*, const double*, double*,
                                            double*, double*, cudaStream_t);

}  // namespace lsb
