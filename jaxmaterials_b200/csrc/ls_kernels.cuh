// Kernel launchers of the Lippmann-Schwinger solver (implemented in ls_kernels.cu).
#pragma once

#include <algorithm>

#include "ls_types.cuh"

namespace lsb {

constexpr int kVPT = 16;                 // complex values per thread in the shared-memory FFTs
constexpr long long kPassBytes = 49152;  // dynamic shared memory of one FFT block

struct LaunchShape {
  int lines_per_block = 1;  // z pass
  int z_threads = 32;
  int z_blocks = 1;
  int ty = 1, y_threads = 32, y_tiles = 1;    // y pass: columns per block
  int tx = 1, x_threads = 32, x_tiles = 1;    // x pass: columns per block
  int x_blocks_per_instance = 1;
  size_t z_smem = 0, y_smem = 0, x_smem = 0;
};

// Tile and block sizes of the three passes for complex values of elem_bytes bytes.
LaunchShape plan_launch(const GridDesc& g, int elem_bytes);
cudaError_t configure_kernels();

// Pointers are batch base pointers; the kernels process instance b when it is not done
// and its phase matches the precision T (float: phase 0, double: phase 1). Instance b
// reads the Lame fields of structure b / g.lame_group and the medium med[b / g.lame_group].
// mode 0: eps = eps_bar (or eps0 if given); mode 1: eps += r / N from spec; mode 2: keep
// eps and the stored shift (continuation in another precision, or after the Anderson
// combine); mode 3: Anderson residual into the rings (see ls_kernels.cu).
template <typename T>
void launch_zpass(const GridDesc& g, const LaunchShape& ls, int mode, int batch, const T* lambda,
                  const T* mu, T* eps, cplx<T>* spec, const double* eps_bar, const T* eps0,
                  InstanceState* st, const Medium* med, const AndersonArgs<T>& aa, cudaStream_t s);
// Gram-row partials [batch][nblk][depth+2] of the newest residual of every instance in
// `phase` (depth+1 products and the block's max |r|; r: the residual ring
// [batch][depth+1][6][nv], FP16 with per-slot scales in the FP32 phase).
template <typename T>
void launch_anderson_gram(long long nv, int nblk, int depth, int phase, int batch,
                          const InstanceState* st, const typename ResRing<T>::type* r,
                          double* partials, cudaStream_t s);
// eps = sum_s alpha_s g_s for every instance in `phase` (g: [batch][depth+1][6][nv]);
// with `inject` ([batch][6][nv]) the first update of a solve sets eps = inject instead.
template <typename T>
void launch_anderson_combine(long long nv, int depth, int phase, int batch, const InstanceState* st,
                             const T* g, const double* alpha, T* eps, cudaStream_t s,
                             const T* inject = nullptr);
// Anderson coefficients of every instance in `phase` from the Gram-row partials (and, in
// the FP32 phase, the newest residual's max |r| into the instance state).
void launch_anderson_solve(int nzblk, int depth, int phase, int batch, InstanceState* st,
                           const double* partials, double* amat, double* alpha, cudaStream_t s);
template <typename T>
void launch_ypass(const GridDesc& g, const LaunchShape& ls, bool inverse, int batch, cplx<T>* spec,
                  const InstanceState* st, cudaStream_t s);
template <typename T>
void launch_xpass(const GridDesc& g, const LaunchShape& ls, int batch, cplx<T>* spec,
                  const Medium* med, InstanceState* st, double* partials, cudaStream_t s);
void launch_finalize(const LaunchShape& ls, int phase, int batch, InstanceState* st,
                     const double* partials, double* history, int history_len,
                     const SolveParams& sp, cudaStream_t s);
// e0_ref (optional, device double[batch]): reference criteria for the stop threshold.
void launch_reset_state(int batch, int phase, InstanceState* st, cudaStream_t s,
                        const double* e0_ref = nullptr);
// min/max and FP64 means of each of nstruct Lame field pairs ([structure][nv]) ->
// reference media med[structure]; scratch: 6 * max(1024, nstruct) doubles.
template <typename TL>
void launch_medium(long long nv, int nstruct, const TL* lambda, const TL* mu, double* scratch,
                   Medium* med, cudaStream_t s);
// out = in for instances in phase 1 (if only_running: and not done).
template <typename Tin, typename Tout>
void launch_convert_fields(long long n_per_instance, int batch, int only_running,
                           const InstanceState* st, const Tin* in, Tout* out, cudaStream_t s);
template <typename Tin, typename Tout>
void launch_convert(long long n, const Tin* in, Tout* out, cudaStream_t s);
// sigma = C : eps for the instances in `phase`; if mean != nullptr also the FP64 mean of
// sigma per instance and component ([batch][6]); scratch: batch * 6 * 1024 doubles.
template <typename T, typename TS>
void launch_stress(const GridDesc& g, int phase, int batch, const InstanceState* st,
                   const T* lambda, const T* mu, const T* eps, TS* sigma, double* scratch,
                   double* mean, cudaStream_t s);

}  // namespace lsb
