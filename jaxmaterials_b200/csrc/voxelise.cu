// GPU voxelisation of layered fibre composites: the reference's
// LayeredFibresDatasetGenerator.material_properties (src/jaxmaterials/data/data.py:267-314)
// for many samples per call, bit-identical to its numpy evaluation.
//
// The fibres are infinite cylinders along x (orientation 0) or y (orientation 1), so
// whether a voxel lies in a fibre depends only on (x, z) or (y, z). Pass 1 counts, for
// every sample, orientation and point (u, z) of the two cross-section grids, the fibres
// that contain it (FP64 predicate without contraction, as numpy evaluates it). Pass 2
// writes every voxel from the two counts of its (x, z) and (y, z) points: the additions of
// the reference (void once, then the same fibre increment once per containing fibre) are
// replayed in order, each rounded to the output type. Pass 2 is a pure HBM write stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "../../include/lippmann_schwinger.h"
#include "ls_solver_impl.cuh"

using namespace lsb::detail;

namespace {

struct VoxGrid {
  int nx, ny, nz, amax;
  double h[3];          // L_d / n_d, as the reference's meshgrid spacing
  double d_void, z_top; // void where z < d_void or z > z_top
};

struct VoxValues {
  double material[2];  // mu, lambda
  double dvoid[2];     // void - material
  double dfibre[2];    // fibre - material
};

// counts[(s * 2 + o) * amax + a][k] = number of fibres of orientation o in sample s that
// contain (u, z) = (h_o (a + 1/2), h_z (k + 1/2)). Block = 128 consecutive k of one (a, s, o).
__global__ void __launch_bounds__(128) count_kernel(VoxGrid g, int s0, const int* __restrict__ off,
                                                    const double4* __restrict__ fib,
                                                    int* __restrict__ counts) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = blockIdx.y;
  const int so = blockIdx.z;  // local sample * 2 + orientation
  const int s = s0 + (so >> 1), o = so & 1;
  const int na = o ? g.ny : g.nx;
  if (k >= g.nz || a >= na) return;
  const double u = __dmul_rn(g.h[o], 0.5 + (double)a);
  const double z = __dmul_rn(g.h[2], 0.5 + (double)k);
  int c = 0;
  for (int f = off[s]; f < off[s + 1]; ++f) {
    const double4 F = fib[f];  // (u0, z0, r^2, orientation)
    if ((int)F.w != o) continue;
    const double du = __dsub_rn(u, F.x);
    const double dz = __dsub_rn(z, F.y);
    c += __dadd_rn(__dmul_rn(du, du), __dmul_rn(dz, dz)) < F.z ? 1 : 0;
  }
  counts[((size_t)so * g.amax + a) * g.nz + k] = c;
}

__device__ __forceinline__ float add_rounded(float x, double d) {
  return __double2float_rn(__dadd_rn((double)x, d));
}
__device__ __forceinline__ double add_rounded(double x, double d) { return __dadd_rn(x, d); }

template <typename T>
__device__ __forceinline__ T from_double(double v);
template <>
__device__ __forceinline__ float from_double<float>(double v) { return __double2float_rn(v); }
template <>
__device__ __forceinline__ double from_double<double>(double v) { return v; }

// out[s][c][i][j][k], c = 0 mu, 1 lambda; grid (blocks over voxels, local sample).
template <typename T>
__global__ void __launch_bounds__(256) fill_kernel(VoxGrid g, VoxValues v, int s0,
                                                   const int* __restrict__ counts,
                                                   T* __restrict__ out) {
  const long long nv = (long long)g.nx * g.ny * g.nz;
  const int sl = blockIdx.y;
  const int* c0 = counts + (size_t)(2 * sl) * g.amax * g.nz;
  const int* c1 = counts + (size_t)(2 * sl + 1) * g.amax * g.nz;
  T* o = out + (size_t)(s0 + sl) * 2 * nv;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < nv;
       idx += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(idx % g.nz);
    const long long ij = idx / g.nz;
    const int j = (int)(ij % g.ny), i = (int)(ij / g.ny);
    const double z = __dmul_rn(g.h[2], 0.5 + (double)k);
    const bool vd = (z < g.d_void) || (z > g.z_top);
    const int n = c0[(size_t)i * g.nz + k] + c1[(size_t)j * g.nz + k];
#pragma unroll
    for (int f = 0; f < 2; ++f) {
      T x = from_double<T>(v.material[f]);
      if (vd) x = add_rounded(x, v.dvoid[f]);
      for (int t = 0; t < n; ++t) x = add_rounded(x, v.dfibre[f]);
      o[(size_t)f * nv + idx] = x;
    }
  }
}

}  // namespace

extern "C" int lsb_voxelise_fibres(int nsamples, const int voxels[3], const double extents[3],
                                   double d_void, double z_top_void, const double values[6],
                                   const int* fibre_offsets, const double* fibres, int elem_size,
                                   void* d_out, void* stream) {
  if (nsamples < 0) return fail(-1, "nsamples must be >= 0");
  if (nsamples == 0) return 0;
  if (!voxels || !extents || !values || !fibre_offsets || !d_out)
    return fail(-1, "null argument");
  if (elem_size != 4 && elem_size != 8) return fail(-1, "elem_size must be 4 or 8");
  for (int d = 0; d < 3; ++d) {
    if (voxels[d] < 1 || voxels[d] > 65535) return fail(-1, "voxels[%d] = %d outside [1, 65535]", d, voxels[d]);
    if (!(extents[d] > 0.0)) return fail(-1, "extents[%d] must be positive", d);
  }
  if (fibre_offsets[0] != 0) return fail(-1, "fibre_offsets[0] must be 0");
  for (int s = 0; s < nsamples; ++s)
    if (fibre_offsets[s + 1] < fibre_offsets[s]) return fail(-1, "fibre_offsets must not decrease");
  const int total = fibre_offsets[nsamples];
  if (total > 0 && !fibres) return fail(-1, "null fibres");
  for (int f = 0; f < total; ++f) {
    const double w = fibres[4 * f + 3];
    if (w != 0.0 && w != 1.0) return fail(-1, "fibre %d: orientation must be 0 or 1", f);
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  VoxGrid g;
  g.nx = voxels[0];
  g.ny = voxels[1];
  g.nz = voxels[2];
  g.amax = std::max(g.nx, g.ny);
  for (int d = 0; d < 3; ++d) g.h[d] = extents[d] / (double)voxels[d];
  g.d_void = d_void;
  g.z_top = z_top_void;
  VoxValues v;
  for (int f = 0; f < 2; ++f) {
    v.material[f] = values[4 + f];
    v.dvoid[f] = values[f] - values[4 + f];
    v.dfibre[f] = values[2 + f] - values[4 + f];
  }
  // samples per chunk: the count tables of a chunk stay below 64 MB
  const size_t per_sample = (size_t)2 * g.amax * g.nz * sizeof(int);
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>({(size_t)nsamples, (64u << 20) / per_sample, 32767}));
  int* d_off = nullptr;
  double4* d_fib = nullptr;
  int* d_cnt = nullptr;
  auto release = [&]() {
    if (d_off) cudaFreeAsync(d_off, st);
    if (d_fib) cudaFreeAsync(d_fib, st);
    if (d_cnt) cudaFreeAsync(d_cnt, st);
  };
  cudaError_t e = cudaMallocAsync((void**)&d_off, sizeof(int) * (nsamples + 1), st);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&d_fib, sizeof(double4) * std::max(total, 1), st);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&d_cnt, per_sample * chunk, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_off, fibre_offsets, sizeof(int) * (nsamples + 1), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && total > 0)
    e = cudaMemcpyAsync(d_fib, fibres, sizeof(double4) * total, cudaMemcpyHostToDevice, st);
  const long long nv = (long long)g.nx * g.ny * g.nz;
  for (int s0 = 0; e == cudaSuccess && s0 < nsamples; s0 += chunk) {
    const int ns = std::min(chunk, nsamples - s0);
    count_kernel<<<dim3((g.nz + 127) / 128, g.amax, 2 * ns), 128, 0, st>>>(g, s0, d_off, d_fib, d_cnt);
    const dim3 grid((unsigned)std::min<long long>((nv + 255) / 256, 2048), ns);
    if (elem_size == 4)
      fill_kernel<float><<<grid, 256, 0, st>>>(g, v, s0, d_cnt, static_cast<float*>(d_out));
    else
      fill_kernel<double><<<grid, 256, 0, st>>>(g, v, s0, d_cnt, static_cast<double*>(d_out));
    e = cudaGetLastError();
  }
  release();
  if (e != cudaSuccess) return fail(-2, "voxelise: %s", cudaGetErrorString(e));
  return 0;
}
