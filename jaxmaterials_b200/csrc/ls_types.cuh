// Shared host/device types of the Lippmann-Schwinger solver library.
//
// Layouts (all row-major, last index fastest):
//   real fields      eps, sigma, r       [batch][6][nx][ny][nz]            float
//   Lame fields      lambda, mu          [nx][ny][nz]                      float
//   spectrum         S                   [batch][6][nx][ny][nzh], nzh = nz/2+1   float2
// The spectrum layout is that of a cuFFT R2C transform of batch 6 over z-fastest
// fields (cuda/src/lippmann_schwinger.cu:117-120 in the reference). Voigt order is
// (xx, yy, zz, xy, xz, yz) with tensor shear entries.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace lsb {

constexpr int kMaxStages = 20;   // radix stages of one 1-D transform
constexpr int kMaxDim = 1024;    // largest supported extent along any axis
constexpr int kMaxThreads = 384;  // largest block of the FFT passes (6144 values / 16 per thread)

// Mixed-radix Stockham plan for complex transforms of length n.
// tw[k] = exp(-2 pi i k / n), k in [0, n), computed in FP64 on the host.
struct Plan1D {
  int n;
  int nst;
  int radix[kMaxStages];
  const float2* tw;
};

struct GridDesc {
  int nx, ny, nz, nzh;
  long long nv;   // voxels
  long long nm;   // half-spectrum modes
  double Lx, Ly, Lz;
  Plan1D px, py, pz;
  // per-axis FP64 tables: s_d[k] = sin(pi k / n_d), c_d[k] = cos(pi k / n_d)
  const double* sx;
  const double* cx;
  const double* sy;
  const double* cy;
  const double* sz;
  const double* cz;
};

// Reference medium, derived on the device from min/max of the Lame fields.
struct Medium {
  float lambda0, mu0;
  float c_a;   // -1/mu0
  float c_b;   // (lambda0+mu0) / (mu0 (lambda0 + 2 mu0))
  float lmin, lmax, mmin, mmax;
};

enum Status : int {
  kRunning = 0,
  kConverged = 1,
  kMaxIter = 2,
  kNonFinite = 3,
};

// Per-instance iteration state, owned by the device.
struct InstanceState {
  int iter;      // updates performed
  int done;      // nonzero once the instance has stopped
  int status;    // Status
  int evals;     // criterion evaluations performed
  double e0;     // criterion at the first iterate
  double e;      // last criterion value
  double sig0[12];  // zero mode of sigma_hat (6 complex) at the last evaluation
};

struct SolveParams {
  float rtol, atol;
  int maxiter;
  int rule;       // 0: stop when e <  max(rtol e0, atol)  (C ABI rule)
                  // 1: stop when e <= max(rtol e0, atol)  (jax-signature rule)
  float inv_nv;   // 1 / voxels
};

}  // namespace lsb
