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
#include <cstdint>
#include <cstring>
#include <mutex>
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
// contain (u, z) = (h_o (a + 1/2), h_z (k + 1/2)). Block = 128 consecutive k of one (a, s, o);
// off[2 s + o] .. off[2 s + o + 1] - 1 are the records of sample s with orientation o.
__global__ void __launch_bounds__(128) count_kernel(VoxGrid g, int s0, const int* __restrict__ off,
                                                    const double4* __restrict__ fib,
                                                    int* __restrict__ counts) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = blockIdx.y;
  const int so = blockIdx.z;  // local sample * 2 + orientation
  const int o = so & 1;
  const int na = o ? g.ny : g.nx;
  if (k >= g.nz || a >= na) return;
  const double u = __dmul_rn(g.h[o], 0.5 + (double)a);
  const double z = __dmul_rn(g.h[2], 0.5 + (double)k);
  int c = 0;
  const int f1 = off[2 * s0 + so + 1];
  for (int f = off[2 * s0 + so]; f < f1; ++f) {
    const double4 F = fib[f];  // (u0, z0, r^2, orientation)
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

template <typename T, int V>
struct VecOf;
template <>
struct VecOf<float, 4> { using type = float4; };
template <>
struct VecOf<double, 2> { using type = double2; };

template <typename T>
__device__ __forceinline__ T voxel_value(const VoxValues& v, int f, bool vd, int n) {
  T x = from_double<T>(v.material[f]);
  if (vd) x = add_rounded(x, v.dvoid[f]);
  for (int t = 0; t < n; ++t) x = add_rounded(x, v.dfibre[f]);
  return x;
}

// out[s][c][i][j][k], c = 0 mu, 1 lambda. Each thread writes V consecutive voxels of a
// z-line (V divides nz) per step of a grid-stride loop, reading their counts as one vector
// (the count tables start 256-byte aligned and their rows hold nz ints); grid (blocks,
// local sample).
template <typename T, int V>
__global__ void __launch_bounds__(256) fill_kernel(VoxGrid g, VoxValues v, int s0,
                                                   const int* __restrict__ counts,
                                                   T* __restrict__ out) {
  const int nv = g.nx * g.ny * g.nz;  // < 2^31 (checked on the host)
  const int nq = nv / V;
  const int sl = blockIdx.y;
  const int* c0 = counts + (size_t)(2 * sl) * g.amax * g.nz;
  const int* c1 = counts + (size_t)(2 * sl + 1) * g.amax * g.nz;
  T* o = out + (size_t)(s0 + sl) * 2 * nv;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
    const int e0 = q * V;
    const int line = e0 / g.nz, k0 = e0 - line * g.nz;
    const int i = line / g.ny, j = line - i * g.ny;
    int n0[V], n1[V];
    if constexpr (V == 4) {
      const int4 a = *reinterpret_cast<const int4*>(c0 + i * g.nz + k0);
      const int4 b = *reinterpret_cast<const int4*>(c1 + j * g.nz + k0);
      n0[0] = a.x; n0[1] = a.y; n0[2] = a.z; n0[3] = a.w;
      n1[0] = b.x; n1[1] = b.y; n1[2] = b.z; n1[3] = b.w;
    } else if constexpr (V == 2) {
      const int2 a = *reinterpret_cast<const int2*>(c0 + i * g.nz + k0);
      const int2 b = *reinterpret_cast<const int2*>(c1 + j * g.nz + k0);
      n0[0] = a.x; n0[1] = a.y;
      n1[0] = b.x; n1[1] = b.y;
    } else {
      n0[0] = c0[i * g.nz + k0];
      n1[0] = c1[j * g.nz + k0];
    }
    T val[2][V];
#pragma unroll
    for (int u = 0; u < V; ++u) {
      const int k = k0 + u;
      const double z = __dmul_rn(g.h[2], 0.5 + (double)k);
      const bool vd = (z < g.d_void) || (z > g.z_top);
      const int n = n0[u] + n1[u];
      val[0][u] = voxel_value<T>(v, 0, vd, n);
      val[1][u] = voxel_value<T>(v, 1, vd, n);
    }
#pragma unroll
    for (int f = 0; f < 2; ++f) {
      if constexpr (V == 1) {
        o[(size_t)f * nv + e0] = val[f][0];
      } else {
        typename VecOf<T, V>::type w;
        T* wp = reinterpret_cast<T*>(&w);
#pragma unroll
        for (int u = 0; u < V; ++u) wp[u] = val[f][u];
        *reinterpret_cast<typename VecOf<T, V>::type*>(o + (size_t)f * nv + e0) = w;
      }
    }
  }
}

template <typename T, int V>
void launch_fill(const VoxGrid& g, const VoxValues& v, int s0, int ns, const int* cnt, T* out,
                 cudaStream_t st) {
  const long long nq = (long long)g.nx * g.ny * g.nz / V;
  const dim3 grid((unsigned)std::min<long long>((nq + 255) / 256, 148 * 8), ns);
  fill_kernel<T, V><<<grid, 256, 0, st>>>(g, v, s0, cnt, out);
}

// Device scratch of lsb_voxelise_fibres (record offsets, records, count tables), one
// growing buffer per device, reused across calls; calls are serialised on the host and
// ordered on the device by the event of the previous call.
constexpr int kMaxVoxDevices = 64;
struct VoxScratch {
  void* buf = nullptr;
  size_t bytes = 0;
  cudaEvent_t done = nullptr;
};
std::mutex g_vox_mu;
VoxScratch g_vox[kMaxVoxDevices];

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
  if ((long long)voxels[0] * voxels[1] * voxels[2] > 0x7fffffffLL)
    return fail(-1, "nx * ny * nz must stay below 2^31");
  // records grouped by (sample, orientation): off2[2 s + o] .. off2[2 s + o + 1] - 1 (the
  // fields depend only on how many fibres contain a point, not on their order)
  std::vector<int> off2(2 * (size_t)nsamples + 1, 0);
  std::vector<double> grouped((size_t)4 * std::max(total, 1));
  {
    size_t w = 0;
    for (int s = 0; s < nsamples; ++s)
      for (int o = 0; o < 2; ++o) {
        for (int f = fibre_offsets[s]; f < fibre_offsets[s + 1]; ++f)
          if ((int)fibres[4 * f + 3] == o) {
            std::memcpy(&grouped[4 * w], &fibres[4 * f], 4 * sizeof(double));
            ++w;
          }
        off2[2 * s + o + 1] = (int)w;
      }
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
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t b_off = up(sizeof(int) * off2.size());
  const size_t b_fib = up(sizeof(double4) * std::max(total, 1));
  const size_t need = b_off + b_fib + per_sample * chunk;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxVoxDevices)
    return fail(-2, "voxelise: no usable device");
  std::lock_guard<std::mutex> lock(g_vox_mu);
  VoxScratch& sc = g_vox[dev];
  if (sc.bytes < need) {
    // cudaFree synchronises the device, so no earlier call still uses the old buffer;
    // the buffer grows with headroom so that similar calls do not reallocate
    if (sc.buf) cudaFree(sc.buf);
    sc.buf = nullptr;
    sc.bytes = 0;
    const size_t bytes = std::max(need + need / 2, (size_t)1 << 20);
    e = cudaMalloc(&sc.buf, bytes);
    if (e != cudaSuccess) return fail(-3, "voxelise: cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    sc.bytes = bytes;
  }
  if (!sc.done) {
    e = cudaEventCreateWithFlags(&sc.done, cudaEventDisableTiming);
    if (e != cudaSuccess) return fail(-2, "voxelise: %s", cudaGetErrorString(e));
  } else {
    // the previous call (maybe on another stream) must be done with the scratch
    e = cudaStreamWaitEvent(st, sc.done, 0);
  }
  int* d_off = reinterpret_cast<int*>(sc.buf);
  double4* d_fib = reinterpret_cast<double4*>(static_cast<char*>(sc.buf) + b_off);
  int* d_cnt = reinterpret_cast<int*>(static_cast<char*>(sc.buf) + b_off + b_fib);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_off, off2.data(), sizeof(int) * off2.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && total > 0)
    e = cudaMemcpyAsync(d_fib, grouped.data(), sizeof(double4) * total, cudaMemcpyHostToDevice, st);
  // 16-byte stores where the z-lines (and so every sample's fields) keep 16-byte alignment
  const bool vec = reinterpret_cast<uintptr_t>(d_out) % 16 == 0 &&
                   g.nz % (elem_size == 4 ? 4 : 2) == 0;
  for (int s0 = 0; e == cudaSuccess && s0 < nsamples; s0 += chunk) {
    const int ns = std::min(chunk, nsamples - s0);
    count_kernel<<<dim3((g.nz + 127) / 128, g.amax, 2 * ns), 128, 0, st>>>(g, s0, d_off, d_fib, d_cnt);
    if (elem_size == 4) {
      float* out = static_cast<float*>(d_out);
      vec ? launch_fill<float, 4>(g, v, s0, ns, d_cnt, out, st) : launch_fill<float, 1>(g, v, s0, ns, d_cnt, out, st);
    } else {
      double* out = static_cast<double*>(d_out);
      vec ? launch_fill<double, 2>(g, v, s0, ns, d_cnt, out, st) : launch_fill<double, 1>(g, v, s0, ns, d_cnt, out, st);
    }
    e = cudaGetLastError();
  }
  // (the host staging vectors are pageable: their copies were taken before returning)
  if (e == cudaSuccess) e = cudaEventRecord(sc.done, st);
  if (e != cudaSuccess) return fail(-2, "voxelise: %s", cudaGetErrorString(e));
  return 0;
}
