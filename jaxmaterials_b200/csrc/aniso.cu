// Anisotropic stiffness for the solver (lsb_set_anisotropic): the stress law and Gamma^0 of
// the derivation in doc/linear_elasticity.tex:372-402 (aniso.cuh), applied by the generic
// passes; the reference stiffness C^0 defaults to the mid-range of every entry over the
// structure, (min + max) / 2, as lambda0 and mu0 are for the isotropic law
// (lippmann_schwinger.py:171-172).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "../../include/lippmann_schwinger.h"
#include "ls_kernels.cuh"
#include "ls_solver_impl.cuh"

using namespace lsb;
using namespace lsb::detail;

namespace {

constexpr int kC0Blocks = 64;  // partial blocks per (structure, entry)

// part[((s * 21 + k) * kC0Blocks + blk) * 2 + {0, 1}] = min, max of entry k of structure s
// over the block's voxels.
template <typename T>
__global__ void __launch_bounds__(256) c0_partial_kernel(long long nv, const T* __restrict__ cf,
                                                         double* __restrict__ part) {
  __shared__ double smin[256], smax[256];
  const int k = blockIdx.y, s = blockIdx.z;
  const T* f = cf + ((size_t)s * 21 + k) * nv;
  double lo = INFINITY, hi = -INFINITY;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = (double)f[i];
    lo = fmin(lo, v);
    hi = fmax(hi, v);
  }
  smin[threadIdx.x] = lo;
  smax[threadIdx.x] = hi;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + w]);
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const size_t o = (((size_t)s * 21 + k) * kC0Blocks + blockIdx.x) * 2;
    part[o] = smin[0];
    part[o + 1] = smax[0];
  }
}

// c0[s * 21 + k] = (min + max) / 2; one thread per (structure, entry).
__global__ void c0_final_kernel(int n, const double* __restrict__ part, double* __restrict__ c0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double lo = INFINITY, hi = -INFINITY;
  for (int b = 0; b < kC0Blocks; ++b) {
    lo = fmin(lo, part[((size_t)i * kC0Blocks + b) * 2]);
    hi = fmax(hi, part[((size_t)i * kC0Blocks + b) * 2 + 1]);
  }
  c0[i] = 0.5 * (lo + hi);
}

}  // namespace

namespace lsb {
namespace detail {

int prepare_aniso(lsb_solver* s, int nstruct) {
  GridDesc& g = s->g;
  g.cf32 = nullptr;
  g.cf64 = nullptr;
  g.c0 = nullptr;
  if (!s->aniso_user) return 0;
  if (s->dmg_user) return fail(-1, "the damage law and an anisotropic stiffness cannot be combined");
  cudaStream_t st = s->stream;
  const long long n = (long long)nstruct * 21 * g.nv;
  const size_t bytes = (size_t)n * (s->aniso_elem == 4 ? sizeof(double) : sizeof(float));
  cudaError_t e = cudaSuccess;
  if (bytes > s->cf_conv_bytes) {
    if (s->d_cf_conv) cudaFree(s->d_cf_conv);
    s->d_cf_conv = nullptr;
    s->cf_conv_bytes = 0;
    e = cudaMalloc(&s->d_cf_conv, bytes);
    if (e != cudaSuccess) return fail(-3, "anisotropic stiffness: cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    s->cf_conv_bytes = bytes;
  }
  if (!s->d_c0) {
    e = cudaMalloc(&s->d_c0, sizeof(double) * 21 * s->batch_cap);
    if (e == cudaSuccess)
      e = cudaMalloc(&s->d_c0_part, sizeof(double) * 2 * kC0Blocks * 21 * s->batch_cap);
    if (e != cudaSuccess) return fail(-3, "anisotropic stiffness: %s", cudaGetErrorString(e));
  }
  if (s->aniso_elem == 4) {
    g.cf32 = static_cast<const float*>(s->aniso_user);
    g.cf64 = static_cast<const double*>(s->d_cf_conv);
    launch_convert<float, double>(n, g.cf32, static_cast<double*>(s->d_cf_conv), st);
  } else {
    g.cf64 = static_cast<const double*>(s->aniso_user);
    g.cf32 = static_cast<const float*>(s->d_cf_conv);
    launch_convert<double, float>(n, g.cf64, static_cast<float*>(s->d_cf_conv), st);
  }
  ++s->launches;
  if (s->aniso_c0_given) {
    for (int i = 0; i < nstruct; ++i) {
      e = cudaMemcpyAsync(s->d_c0 + 21 * i, s->aniso_c0, sizeof(double) * 21, cudaMemcpyHostToDevice, st);
      if (e != cudaSuccess) break;
    }
  } else {
    const dim3 grid(kC0Blocks, 21, nstruct);
    if (s->aniso_elem == 4)
      c0_partial_kernel<float><<<grid, 256, 0, st>>>(g.nv, g.cf32, s->d_c0_part);
    else
      c0_partial_kernel<double><<<grid, 256, 0, st>>>(g.nv, g.cf64, s->d_c0_part);
    c0_final_kernel<<<(21 * nstruct + 127) / 128, 128, 0, st>>>(21 * nstruct, s->d_c0_part, s->d_c0);
    s->launches += 2;
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return fail(-2, "anisotropic stiffness: %s", cudaGetErrorString(e));
  g.c0 = s->d_c0;
  return 0;
}

}  // namespace detail
}  // namespace lsb

extern "C" int lsb_set_anisotropic(lsb_solver* solver, const void* d_stiffness, int elem_size,
                                   const double* c0) {
  if (!solver) return fail(-1, "null solver");
  if (d_stiffness && elem_size != 4 && elem_size != 8) return fail(-1, "elem_size must be 4 or 8");
  if (c0)
    for (int k = 0; k < 21; ++k)
      if (!std::isfinite(c0[k])) return fail(-1, "c0[%d] is not finite", k);
  solver->aniso_user = d_stiffness;
  solver->aniso_elem = d_stiffness ? elem_size : 4;
  solver->aniso_c0_given = c0 != nullptr;
  if (c0) std::memcpy(solver->aniso_c0, c0, sizeof(double) * 21);
  if (!d_stiffness) {
    solver->g.cf32 = nullptr;
    solver->g.cf64 = nullptr;
    solver->g.c0 = nullptr;
  }
  return 0;
}
