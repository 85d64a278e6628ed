// Kernel launchers of the Lippmann-Schwinger solver (implemented in ls_kernels.cu).
#pragma once

#include "ls_types.cuh"

namespace lsb {

constexpr int kVPT = 16;  // complex values per thread in the shared-memory FFTs
constexpr long long kPassElems = 6144;  // complex values per block (48 KB of shared memory)

struct LaunchShape {
  int lines_per_block = 1;  // z pass
  int z_threads = 32;
  int z_blocks = 1;
  int ty = 1, y_threads = 32, y_tiles = 1;    // y pass: columns per block
  int tx = 1, x_threads = 32, x_tiles = 1;    // x pass: columns per block
  int x_blocks_per_instance = 1;
  size_t z_smem = 0, y_smem = 0, x_smem = 0;
};

LaunchShape plan_launch(const GridDesc& g);
cudaError_t configure_kernels(const LaunchShape& ls);

// eps/sigma/spec/state/partials are batch base pointers; `batch` instances run.
// mode 0: eps = eps_bar (or eps0 if given); mode 1: eps += r / N from spec.
void launch_zpass(const GridDesc& g, const LaunchShape& ls, int mode, int batch,
                  const float* lambda, const float* mu, float* eps, float2* spec,
                  const float* eps_bar, const float* eps0, const InstanceState* st,
                  const SolveParams& sp, cudaStream_t s);
void launch_ypass(const GridDesc& g, const LaunchShape& ls, bool inverse, int batch,
                  float2* spec, const InstanceState* st, cudaStream_t s);
void launch_xpass(const GridDesc& g, const LaunchShape& ls, int batch, float2* spec,
                  const Medium* med, InstanceState* st, double* partials, cudaStream_t s);
void launch_finalize(const GridDesc& g, const LaunchShape& ls, int batch, InstanceState* st,
                     const double* partials, double* history, int history_len,
                     const SolveParams& sp, cudaStream_t s);
void launch_reset_state(int batch, InstanceState* st, cudaStream_t s);
// min/max of the Lame fields -> reference medium. `scratch` holds 4 * 1024 floats.
void launch_medium(long long nv, const float* lambda, const float* mu, float* scratch,
                   Medium* med, cudaStream_t s);
// sigma = C : eps for every instance; if mean != nullptr also the FP64 mean of sigma
// per instance and component ([batch][6]); `scratch` holds batch * 6 * 1024 doubles.
void launch_stress(const GridDesc& g, int batch, const float* lambda, const float* mu,
                   const float* eps, float* sigma, double* scratch, double* mean,
                   cudaStream_t s);

}  // namespace lsb
