// Shared host/device types of the Lippmann-Schwinger solver library.
//
// Layouts (all row-major, last index fastest):
//   real fields      eps, sigma, r       [batch][6][nx][ny][nz]            float or double
//   Lame fields      lambda, mu          [nx][ny][nz]                      float or double
//   spectrum         S                   [batch][6][nx][ny][nzh], nzh = nz/2+1   float2 or double2
// The spectrum layout is that of a cuFFT R2C transform of batch 6 over z-fastest
// fields (cuda/src/lippmann_schwinger.cu:117-120 in the reference). Voigt order is
// (xx, yy, zz, xy, xz, yz) with tensor shear entries.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace lsb {

constexpr int kMaxStages = 20;    // radix stages of one 1-D transform
constexpr int kMaxDim = 1024;     // largest supported extent along any axis
constexpr int kMaxThreads = 384;  // largest block of the FFT passes

template <typename T>
struct Complex;
template <>
struct Complex<float> {
  using type = float2;
};
template <>
struct Complex<double> {
  using type = double2;
};
template <typename T>
using cplx = typename Complex<T>::type;

// Mixed-radix Stockham plan for complex transforms of length n.
// tw[k] = exp(-2 pi i k / n), k in [0, n), computed in FP64 on the host and stored in
// both precisions.
struct Plan1D {
  int n;
  int nst;
  int radix[kMaxStages];
  const float2* tw;
  const double2* tw64;
};

template <typename T>
__host__ __device__ inline const cplx<T>* twiddles(const Plan1D& p);
template <>
__host__ __device__ inline const float2* twiddles<float>(const Plan1D& p) { return p.tw; }
template <>
__host__ __device__ inline const double2* twiddles<double>(const Plan1D& p) { return p.tw64; }

struct GridDesc {
  int nx, ny, nz, nzh;
  long long nv;   // voxels
  long long nm;   // half-spectrum modes
  double Lx, Ly, Lz;
  Plan1D px, py, pz;
  // Consecutive instances that share one (lambda, mu) field and one reference medium:
  // instance b uses field b / lame_group ([structure][nv] arrays) and medium[b / lame_group].
  int lame_group;
  // per-axis FP64 tables: s_d[k] = sin(pi k / n_d), c_d[k] = cos(pi k / n_d)
  const double* sx;
  const double* cx;
  const double* sy;
  const double* cy;
  const double* sz;
  const double* cz;
  // Damage field of the damage extension (null: the linear law): instance b reads structure
  // b / lame_group ([structure][nv]); dmg_k is the stiffness left at full damage. The FP32
  // and FP64 passes read the copy of their precision.
  const float* dmg32 = nullptr;
  const double* dmg64 = nullptr;
  double dmg_k = 0.0;
  // Anisotropic stiffness (null: the isotropic lambda, mu law): C [structure][21][nv] in the
  // numbering of aniso.cuh, per precision, and the reference stiffness C^0 [structure][21].
  const float* cf32 = nullptr;
  const double* cf64 = nullptr;
  const double* c0 = nullptr;
};

template <typename T>
__host__ __device__ inline const T* stiffness_field(const GridDesc& g);
template <>
__host__ __device__ inline const float* stiffness_field<float>(const GridDesc& g) { return g.cf32; }
template <>
__host__ __device__ inline const double* stiffness_field<double>(const GridDesc& g) { return g.cf64; }

template <typename T>
__host__ __device__ inline const T* damage_field(const GridDesc& g);
template <>
__host__ __device__ inline const float* damage_field<float>(const GridDesc& g) { return g.dmg32; }
template <>
__host__ __device__ inline const double* damage_field<double>(const GridDesc& g) { return g.dmg64; }

// Reference medium, derived on the device from min/max of the Lame fields
// (lambda0 = (min + max) / 2, evaluated in the precision of the iteration).
struct Medium {
  double lmin, lmax, mmin, mmax;
  double lmean, mmean;    // FP64 means of the Lame fields
  float lambda0, mu0;     // FP32 iteration
  float c_a, c_b;         // -1/mu0 and (lambda0+mu0) / (mu0 (lambda0 + 2 mu0))
  double lambda0_64, mu0_64, c_a64, c_b64;  // FP64 iteration
};

template <typename T>
__device__ inline T medium_ca(const Medium& m);
template <>
__device__ inline float medium_ca<float>(const Medium& m) { return m.c_a; }
template <>
__device__ inline double medium_ca<double>(const Medium& m) { return m.c_a64; }
template <typename T>
__device__ inline T medium_cb(const Medium& m);
template <>
__device__ inline float medium_cb<float>(const Medium& m) { return m.c_b; }
template <>
__device__ inline double medium_cb<double>(const Medium& m) { return m.c_b64; }

enum Status : int {
  kRunning = 0,
  kConverged = 1,
  kMaxIter = 2,
  kNonFinite = 3,
  kStalled = 4,   // FP32 round-off floor reached above the tolerance (FP32-only mode)
  kTimeout = 5,   // a bounded wait for asynchronous copies ran out (the solve was abandoned)
};

// Per-instance iteration state, owned by the device.
struct InstanceState {
  int iter;       // updates performed
  int done;       // nonzero once the instance has stopped
  int status;     // Status
  int evals;      // criterion evaluations performed
  int phase;      // 0: FP32 fields, 1: FP64 fields
  int best_eval;  // evaluation at which best_e last improved significantly
  int switched;   // 1 once the instance moved from FP32 to FP64
  int aa_base;    // iteration count when the Anderson history (re)started
  int copies_lost;  // a block gave up waiting for its asynchronous copies twice (kTimeout)
  int switch_iter;  // updates done in FP32 before the switch to FP64 fields (switched = 1)
  double e0;      // criterion at the first iterate
  double e0_ref;  // > 0: the stop threshold is rtol * e0_ref instead of rtol * e0
  double e;       // last criterion value
  double best_e;  // smallest criterion value seen in the current phase
  double sig0[12];  // zero mode of sigma_hat (6 complex) at the last evaluation
  // Per-component constant subtracted from sigma before the forward transform. Keeping
  // the near-mean out of the transform keeps the round-off of the lines that carry the
  // zero frequency at the level of the stress fluctuation; the zero mode is restored in
  // FP64 (sig0), and Gamma^0 and xi vanish there, so nothing else depends on it.
  double shift[6];
  // FP32 phase, Anderson residual ring in FP16: slot q holds r_q * 2^ring_exp[q]; ring_max
  // is max |r| of the newest residual (from the Gram row), from which the next slot's
  // exponent is chosen.
  float ring_max;
  int ring_exp[9];
};

enum Precision : int { kPrecFP32 = 0, kPrecMixed = 1, kPrecFP64 = 2 };

constexpr int kMaxDepth = 8;  // largest Anderson depth m (ring of m+1 slots)
static_assert(sizeof(InstanceState::ring_exp) / sizeof(int) == kMaxDepth + 1, "one exponent per slot");

// Element type of the residual ring: the residuals enter only the Gram row (the mixing
// coefficients), never the iterate, so the FP32 phase stores them in FP16, scaled per slot
// by a power of two; the FP64 phase keeps doubles.
template <typename T>
struct ResRing { using type = T; };
template <>
struct ResRing<float> { using type = __half; };

// Anderson acceleration state of one batch (lippmann_schwinger.py:217-231). For update j
// of an instance (j = iter - 1 - aa_base), slot j mod (m+1) of the rings receives
// r_j = -Gamma^0 sigma_j (real space, normalised) and g_j = eps_j + r_j; the next
// iterate is eps = sum_s alpha_s g_s over the filled slots.
template <typename T>
struct AndersonArgs {
  int depth;                        // m (0: plain iteration)
  T* g;                             // [batch][m+1][6][nv]
  typename ResRing<T>::type* r;     // [batch][m+1][6][nv]
  double* partials;                 // [batch][z blocks][m+1] Gram-row partials
  const double* alpha;              // [batch][m+1] mixing coefficients of the current update
};

// Scale exponent of the FP16 residual slot written by the current update: the newest
// residual's max |r| (or, for the first slot of a history, 8 max |eps_bar|) is mapped below
// 2^10, so a residual may grow 64-fold between updates before FP16's 65504 is reached, and
// elements down to 2^-24 of that max keep full FP16 precision.
__host__ __device__ __forceinline__ int ring_exponent(float ring_max, const double* eps_bar6) {
  float m = ring_max;
  if (!(m > 0.f) || !(m < 3.0e38f)) {
    double e = 0.0;
    for (int c = 0; c < 6; ++c) e = fmax(e, fabs(eps_bar6[c]));
    m = (float)(8.0 * (e > 0.0 && e < 1e30 ? e : 1.0));
  }
  int ex;
  frexpf(m, &ex);  // m < 2^ex
  int k = 10 - ex;
  return k < -60 ? -60 : (k > 60 ? 60 : k);
}

// r * 2^k rounded to FP16, saturated at +-65504 (k in [-60, 60]); a NaN stays NaN, so that
// the Gram solve sees it and falls back to the plain update.
__device__ __forceinline__ __half ring_store(float r, float scale) {
  const float t = r * scale;
  return __float2half_rn(t != t ? t : fminf(fmaxf(t, -65504.f), 65504.f));
}

struct SolveParams {
  double rtol, atol;
  int maxiter;
  int rule;         // 0: stop when e <  max(rtol e0, atol); 1: stop when e <= ...
  long long nv;     // voxels
  int precision;    // Precision
  int stall_window;       // evaluations without a significant improvement => stalled
  double stall_improve;   // significant improvement: e < stall_improve * best_e
  double stall_near;      // stall is only declared while best_e < stall_near * threshold
};

}  // namespace lsb
