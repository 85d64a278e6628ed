// Gradient of a loss of the effective stiffness with respect to the Lame fields.
//
// Row k of the effective stiffness M (lsb_c_eff, src/jaxmaterials/data/data.py:178-186) is
// the mean stress <sigma^k> for the unit macroscopic strain e_k (tensor shear). With the
// Voigt weights w = (1,1,1,2,2,2), B_kl = M_kl w_l = <eps^k : C : eps^l> is the energy
// form of the six converged strain fields eps^k (the fluctuation of eps^l is orthogonal
// to the divergence-free sigma^k). The Lippmann-Schwinger operator is self-adjoint in
// this inner product, so the adjoint solutions of the six load cases are the forward
// solutions themselves and, at equilibrium,
//     dB_kl / dlambda(x) = tr eps^k(x) tr eps^l(x) / N,
//     dB_kl / dmu(x)     = 2 eps^k(x) : eps^l(x) / N.
// For a loss L(M): dL/dlambda(x) = sum_kl G_kl / w_l * tr eps^k tr eps^l / N with
// G = dL/dM, and likewise for mu.
#include "../../include/lippmann_schwinger.h"
#include "ls_solver_impl.cuh"

namespace lsb {
namespace {

struct Weights {
  double v[36];  // G_kl / w_l, row-major
};

template <typename T>
__global__ void ceff_gradient_kernel(long long nv, const T* __restrict__ eps, Weights gw,
                                     T* __restrict__ dlambda, T* __restrict__ dmu) {
  __shared__ double sg[36];
  if (threadIdx.x < 36) sg[threadIdx.x] = gw.v[threadIdx.x];
  __syncthreads();
  const double inv_n = 1.0 / (double)nv;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
       i += (long long)gridDim.x * blockDim.x) {
    T e[6][6];
#pragma unroll
    for (int k = 0; k < 6; ++k)
#pragma unroll
      for (int a = 0; a < 6; ++a) e[k][a] = eps[((size_t)k * 6 + a) * nv + i];
    double tr[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) tr[k] = (double)e[k][0] + e[k][1] + e[k][2];
    double gl = 0.0, gm = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
#pragma unroll
      for (int l = 0; l < 6; ++l) {
        const double g = sg[k * 6 + l];
        double d = 0.0;
#pragma unroll
        for (int a = 0; a < 6; ++a) d += (a < 3 ? 1.0 : 2.0) * (double)e[k][a] * (double)e[l][a];
        gl += g * tr[k] * tr[l];
        gm += g * 2.0 * d;
      }
    }
    dlambda[i] = (T)(gl * inv_n);
    dmu[i] = (T)(gm * inv_n);
  }
}

template <typename T>
int gradient_impl(const int voxels[3], const T* d_eps, const double* dl_dc, T* d_dlambda, T* d_dmu,
                  void* stream) {
  if (!voxels || !d_eps || !dl_dc || !d_dlambda || !d_dmu) return detail::fail(-1, "null argument");
  long long nv = 1;
  for (int d = 0; d < 3; ++d) {
    if (voxels[d] < 1) return detail::fail(-1, "voxels[%d] must be >= 1", d);
    nv *= voxels[d];
  }
  Weights gw;  // G_kl / w_l
  for (int k = 0; k < 6; ++k)
    for (int l = 0; l < 6; ++l) gw.v[k * 6 + l] = dl_dc[k * 6 + l] / (l < 3 ? 1.0 : 2.0);
  cudaStream_t st = (cudaStream_t)stream;
  int nblk = (int)std::min<long long>(148 * 8, (nv + 255) / 256);
  ceff_gradient_kernel<T><<<std::max(nblk, 1), 256, 0, st>>>(nv, d_eps, gw, d_dlambda, d_dmu);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return detail::fail(-2, "gradient kernel: %s", cudaGetErrorString(e));
  return 0;
}

}  // namespace
}  // namespace lsb

extern "C" {

int lsb_ceff_gradient(const int voxels[3], const float* d_eps, const double* dl_dc, float* d_dlambda,
                      float* d_dmu, void* stream) {
  return lsb::gradient_impl<float>(voxels, d_eps, dl_dc, d_dlambda, d_dmu, stream);
}

int lsb_ceff_gradient_f64(const int voxels[3], const double* d_eps, const double* dl_dc,
                          double* d_dlambda, double* d_dmu, void* stream) {
  return lsb::gradient_impl<double>(voxels, d_eps, dl_dc, d_dlambda, d_dmu, stream);
}

}  // extern "C"
