// lsb_solve_noalloc: the FP32 solve of lsb_solve without any device or pinned-host
// allocation, for callers that cannot call cudaMalloc.
//
// Who needs this: a caller running inside a framework that owns every byte of device
// memory (a framework caching allocator, or a custom-operator interface that forbids
// allocation while the operator runs), or a latency-critical caller that must not pay
// cudaMalloc's implicit device synchronisation. Such callers still pass their inputs and
// outputs; everything else the solve needs (spectrum, partial sums, per-instance state,
// reference medium, twiddle and wave-vector tables) is carved from one file-scope device
// array of LSB_NOALLOC_SCRATCH_BYTES bytes that every GPU loading the library keeps
// until the process exits.
//
// Contract:
// * the first call on a device (and the first call after the device's context was
//   destroyed, e.g. by cudaDeviceReset) resolves the array's device address with
//   cudaGetSymbolAddress, with that device current, and caches it with the context's id;
//   make that first call before any stream capture starts on the device;
// * all work, the table upload included, is ordered on the caller's stream; the call
//   returns after that stream has finished the solve;
// * every call reuses the same array and leaves the previous call's contents in it: the
//   per-call state is cleared by the call itself (the tables are uploaded again whenever
//   the grid differs from the previous call's on that device), and calls whose GPU work
//   overlaps in time (other streams, other host threads, other processes sharing the
//   context) race on the array and must not be issued;
// * grids and batches whose scratch exceeds the array, and batches above
//   LSB_NOALLOC_MAX_BATCH, are rejected with an error;
// * FP32 fields only, plain Moulinec-Suquet iteration, stop rule of the reference C
//   signature, stall detection as LSB_PREC_FP32 (status LSB_STALLED); no criterion
//   history is kept.
#include <cuda.h>

#include <cstring>
#include <mutex>

#include "../../include/lippmann_schwinger.h"
#include "ls_solver_impl.cuh"

using namespace lsb::detail;

namespace {

constexpr size_t kScratchBytes = LSB_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;
constexpr int kMaxBatch = LSB_NOALLOC_MAX_BATCH;

// The scratch array. Host code never dereferences this symbol: its host-side name is only
// a handle, and the device address comes from cudaGetSymbolAddress in device_base().
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct DeviceCache {
  unsigned char* base = nullptr;     // device address of the array in context `ctx_id`
  unsigned long long ctx_id = 0;
  int tables[3] = {0, 0, 0};         // grid whose tables the array holds (0: none)
};

std::mutex g_mutex;
DeviceCache g_dev[kMaxDevices];
InstanceState g_host_state[kMaxBatch];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Id of the current context (0 if the driver does not provide one). Context ids are unique
// over the life of the process, so a reset device gets a new id.
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    looked_up = true;
    void* f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault) == cudaSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault) == cudaSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current && get_id && get_current(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, &id) == CUDA_SUCCESS)
    return id;
  return 0;
}

// Device address of the array on `dev` (current), resolved once per device and context.
int device_base(int dev, DeviceCache** cache) {
  if (dev < 0 || dev >= kMaxDevices) return fail(-1, "device %d outside [0, %d)", dev, kMaxDevices);
  // make the device's primary context current (initialising it if needed) before reading
  // its id
  cudaError_t e = cudaSetDevice(dev);
  if (e != cudaSuccess) return fail(-2, "cudaSetDevice(%d): %s", dev, cudaGetErrorString(e));
  DeviceCache& c = g_dev[dev];
  const unsigned long long id = current_context_id();
  if (!c.base || id != c.ctx_id) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return fail(-2, "cudaGetSymbolAddress of the scratch array failed on device %d: %s", dev,
                  cudaGetErrorString(e));
    c.base = static_cast<unsigned char*>(p);
    c.ctx_id = id;
    c.tables[0] = c.tables[1] = c.tables[2] = 0;  // a new context holds no tables
  }
  *cache = &c;
  return 0;
}

// Bump allocator over the scratch array (256-byte aligned pieces).
struct Carver {
  unsigned char* base;
  size_t used = 0;
  template <typename P>
  void take(P*& out, size_t bytes) {
    out = reinterpret_cast<P*>(base + used);
    used += (bytes + 255) / 256 * 256;
  }
};

}  // namespace

extern "C" int lsb_solve_noalloc(const int voxels[3], const double extents[3], int batch,
                                 const float* d_lambda, const float* d_mu, const float* eps_bar,
                                 float* d_eps, float* d_sigma, double* mean_sigma, float rtol,
                                 float atol, int maxiter, int* iters, int* status,
                                 double* residual, void* stream) {
  if (!voxels || !extents || !eps_bar || !d_lambda || !d_mu || !d_eps || !iters || !status)
    return fail(-1, "null argument");
  if (batch < 1 || batch > kMaxBatch)
    return fail(-1, "batch %d outside [1, %d] (LSB_NOALLOC_MAX_BATCH)", batch, kMaxBatch);
  std::lock_guard<std::mutex> lock(g_mutex);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(-2, "cudaGetDevice: %s", cudaGetErrorString(e));
  DeviceCache* cache = nullptr;
  int rc = device_base(dev, &cache);
  if (rc) return rc;

  lsb_solver s;           // points into the scratch array; frees nothing when it goes away
  s.owns_memory = false;
  s.use_graphs = false;  // graph instantiation allocates
  s.xtuned = true;       // default x-pass tiles (the partials below are sized for them)
  s.device = dev;
  s.batch_cap = batch;
  s.depth = 0;
  s.precision = kPrecFP32;
  s.h_state = g_host_state;
  s.stream = static_cast<cudaStream_t>(stream);
  s.tiled_allowed = false;  // one spectrum buffer: the strided x pass
  rc = plan_grid(&s, voxels, extents);
  if (rc) return rc;
  const GridDesc& g = s.g;
  const size_t B = (size_t)batch;
  const size_t ntw = (size_t)(g.nx + g.ny + g.nz);
  Carver c{cache->base};
  // the tables first: their place depends only on the grid, so an unchanged grid keeps them
  c.take(s.d_tw32, sizeof(float2) * ntw);
  c.take(s.d_tw64, sizeof(double2) * ntw);
  c.take(s.d_tables, sizeof(double) * 2 * (size_t)(g.nx + g.ny + g.nzh));
  c.take(s.d_spec32, sizeof(float2) * B * 6 * g.nm);
  c.take(s.d_partials, sizeof(double) * B * s.sh32.x_blocks_per_instance);
  c.take(s.d_state, sizeof(InstanceState) * B);
  c.take(s.d_medium, sizeof(Medium) * B);
  c.take(s.d_epsbar, sizeof(double) * B * 6);
  c.take(s.d_scratch, sizeof(double) * 6 * 1024);
  c.take(s.d_mean_scratch, sizeof(double) * B * 6 * 1024);
  c.take(s.d_mean, sizeof(double) * B * 6);
  if (c.used > kScratchBytes)
    return fail(-1, "grid %dx%dx%d with batch %d needs %zu bytes of scratch, more than the %zu "
                "bytes of the static array (use lsb_solve)", g.nx, g.ny, g.nz, batch, c.used,
                kScratchBytes);
  const int key[3] = {g.nx, g.ny, g.nz};
  const bool have = std::memcmp(cache->tables, key, sizeof(key)) == 0;
  // forget the cached grid until the new upload has been issued
  if (!have) cache->tables[0] = cache->tables[1] = cache->tables[2] = 0;
  rc = upload_tables(&s, have ? TableUpload::kNone : TableUpload::kAsync);
  if (rc) return rc;
  if (!have) std::memcpy(cache->tables, key, sizeof(key));
  std::vector<double> eb(eps_bar, eps_bar + 6 * batch);
  return solve_f32(&s, batch, d_lambda, d_mu, eb.data(), nullptr, d_eps, d_sigma, mean_sigma,
                   rtol, atol, maxiter, LSB_RULE_CUDA, iters, status, residual);
}
