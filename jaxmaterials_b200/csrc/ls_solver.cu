// Host side of liblippmannschwinger.so: plans, device buffers, the iteration driver and
// the C ABI declared in include/lippmann_schwinger.h.
//
// The iteration never waits on the host per step: kernels read the per-instance state
// written by finalize_kernel, so the host enqueues iterations in growing chunks and reads
// the small states back once per chunk. Precision (lsb_set_precision):
//   FP32   FP32 fields and FFTs throughout (FP64 norms); may stall at the FP32 floor;
//   MIXED  FP32 until the criterion stalls near the tolerance, then the stalled
//          instances continue from their iterate with FP64 fields and FFTs (default);
//   FP64   FP64 fields and FFTs from the start.
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/lippmann_schwinger.h"
#include "ls_solver_impl.cuh"

using namespace lsb;

namespace {
thread_local std::string g_last_error;
}  // namespace

namespace lsb {
namespace detail {

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define LSB_CUDA(expr)                                                                    \
  do {                                                                                    \
    cudaError_t _e = (expr);                                                              \
    if (_e != cudaSuccess)                                                                \
      return fail(-2, "%s:%d: %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(_e)); \
  } while (0)

#define LSB_TRY(expr)        \
  do {                       \
    int _rc = (expr);        \
    if (_rc != 0) return _rc; \
  } while (0)

// Radices for a length-n Stockham plan: 8s first, then 4, 2, 3, 5, then remaining primes.
bool factorize(int n, Plan1D& p) {
  p.n = n;
  p.nst = 0;
  int m = n;
  auto push = [&](int r) {
    if (p.nst >= kMaxStages) return false;
    p.radix[p.nst++] = r;
    return true;
  };
  while (m % 8 == 0) { if (!push(8)) return false; m /= 8; }
  while (m % 4 == 0) { if (!push(4)) return false; m /= 4; }
  while (m % 2 == 0) { if (!push(2)) return false; m /= 2; }
  while (m % 3 == 0) { if (!push(3)) return false; m /= 3; }
  while (m % 5 == 0) { if (!push(5)) return false; m /= 5; }
  for (int f = 7; m > 1; f += 2) {
    while (m % f == 0) { if (!push(f)) return false; m /= f; }
    if (f * f > m && m > 1) { if (!push(m)) return false; m = 1; }
  }
  return true;
}

int structures_of(lsb_solver* s, int batch) {
  const int group = s->lame_group > 0 ? s->lame_group : batch;
  if (batch % group != 0)
    return fail(-1, "batch %d is not a multiple of %d instances per Lame field pair", batch, group);
  s->g.lame_group = group;
  return batch / group;
}

bool shape_fits(const LaunchShape& sh) {
  return sh.z_threads <= kMaxThreads && sh.y_threads <= kMaxThreads && sh.x_threads <= kMaxThreads;
}

}  // namespace detail
}  // namespace lsb

using namespace lsb::detail;



namespace {

int ensure_history(lsb_solver* s, int len) {
  if (len <= s->history_len || !s->owns_memory) return 0;
  cudaFree(s->d_history);
  s->d_history = nullptr;
  LSB_CUDA(cudaMalloc(&s->d_history, sizeof(double) * (size_t)s->batch_cap * len));
  s->history_len = len;
  return 0;
}

// FP64 work buffers, and FP64 copies of `nstruct` Lame field pairs when nstruct > 0.
// Points s->g at the damage field of lsb_set_damage for a solve over nstruct structures,
// converting the caller's field into the other precision (the mixed-precision continuation
// and the FP64 solve read FP64, the FP32 passes FP32).
int prepare_damage(lsb_solver* s, int nstruct) {
  GridDesc& g = s->g;
  g.dmg32 = nullptr;
  g.dmg64 = nullptr;
  g.dmg_k = s->dmg_k;
  if (!s->dmg_user) return 0;
  const long long n = (long long)nstruct * g.nv;
  const size_t bytes = (size_t)n * (s->dmg_elem == 4 ? sizeof(double) : sizeof(float));
  if (bytes > s->dmg_conv_bytes) {
    if (s->d_dmg_conv) cudaFree(s->d_dmg_conv);
    s->d_dmg_conv = nullptr;
    s->dmg_conv_bytes = 0;
    LSB_CUDA(cudaMalloc(&s->d_dmg_conv, bytes));
    s->dmg_conv_bytes = bytes;
  }
  if (s->dmg_elem == 4) {
    g.dmg32 = static_cast<const float*>(s->dmg_user);
    g.dmg64 = static_cast<const double*>(s->d_dmg_conv);
    launch_convert<float, double>(n, g.dmg32, static_cast<double*>(s->d_dmg_conv), s->stream);
  } else {
    g.dmg64 = static_cast<const double*>(s->dmg_user);
    g.dmg32 = static_cast<const float*>(s->d_dmg_conv);
    launch_convert<double, float>(n, g.dmg64, static_cast<float*>(s->d_dmg_conv), s->stream);
  }
  ++s->launches;
  LSB_CUDA(cudaGetLastError());
  return 0;
}

int ensure_fp64(lsb_solver* s, int nstruct) {
  const size_t B = (size_t)s->batch_cap;
  if (!s->d_spec64) {
    LSB_CUDA(cudaMalloc(&s->d_eps64, sizeof(double) * B * 6 * s->g.nv));
    LSB_CUDA(cudaMalloc(&s->d_spec64, sizeof(double2) * B * 6 * s->g.nm));
  }
  if (nstruct > s->lame64_structs) {
    cudaFree(s->d_lame64);
    s->d_lame64 = nullptr;
    s->lame64_structs = 0;
    LSB_CUDA(cudaMalloc(&s->d_lame64, sizeof(double) * 2 * (size_t)nstruct * s->g.nv));
    s->lame64_structs = nstruct;
  }
  return 0;
}

int ensure_fp64_rings(lsb_solver* s) {
  if (s->depth == 0 || s->d_aa_g64) return 0;
  const size_t n = (size_t)s->batch_cap * (s->depth + 1) * 6 * s->g.nv;
  LSB_CUDA(cudaMalloc(&s->d_aa_g64, sizeof(double) * n));
  LSB_CUDA(cudaMalloc(&s->d_aa_r64, sizeof(double) * n));
  return 0;
}

template <typename T>
AndersonArgs<T> anderson_args(lsb_solver* s, bool on) {
  AndersonArgs<T> a;
  a.depth = on ? s->depth : 0;
  if constexpr (sizeof(T) == 4) {
    a.g = s->d_aa_g32;
    a.r = s->d_aa_r32;
  } else {
    a.g = s->d_aa_g64;
    a.r = s->d_aa_r64;
  }
  a.partials = s->d_aa_partials;
  a.alpha = s->d_aa_alpha;
  return a;
}

}  // namespace

namespace lsb {
namespace detail {

int plan_grid(lsb_solver* s, const int voxels[3], const double extents[3]) {
  for (int d = 0; d < 3; ++d) {
    if (voxels[d] < 1 || voxels[d] > kMaxDim)
      return fail(-1, "voxels[%d] = %d outside [1, %d]", d, voxels[d], kMaxDim);
    if (!(extents[d] > 0.0) || !std::isfinite(extents[d]))
      return fail(-1, "extents[%d] must be positive and finite", d);
  }
  GridDesc& g = s->g;
  g.nx = voxels[0];
  g.ny = voxels[1];
  g.nz = voxels[2];
  g.nzh = g.nz / 2 + 1;
  g.nv = (long long)g.nx * g.ny * g.nz;
  g.nm = (long long)g.nx * g.ny * g.nzh;
  g.Lx = extents[0];
  g.Ly = extents[1];
  g.Lz = extents[2];
  if (!factorize(g.nx, g.px) || !factorize(g.ny, g.py) || !factorize(g.nz, g.pz))
    return fail(-1, "grid extent has too many prime factors");
  s->sh32 = plan_launch(g, sizeof(float2));
  s->x_blocks_generic32 = s->sh32.x_blocks_per_instance;
  s->sh64 = plan_launch(g, sizeof(double2));
  s->fast32 = fast::supported(g);
  s->tiled = s->tiled_allowed && s->fast32 && fast::tiled_supported(g);
  s->slab = s->slab_allowed && s->tiled && fast::slab_supported(g);
  if (s->tiled) s->sh32.x_blocks_per_instance = fast::x_tiles_tiled(g);
  else if (s->fast32) s->sh32.x_blocks_per_instance = fast::x_tiles(g, s->xvariant) * g.ny;
  if (!shape_fits(s->sh32) || !shape_fits(s->sh64))
    return fail(-1, "grid %dx%dx%d needs FFT blocks above %d threads", g.nx, g.ny, g.nz, kMaxThreads);
  cudaError_t e = configure_kernels();
  if (e == cudaSuccess) e = fast::configure();
  if (e != cudaSuccess) return fail(-2, "kernel configuration: %s", cudaGetErrorString(e));
  return 0;
}

int upload_tables(lsb_solver* s, TableUpload how) {
  GridDesc& g = s->g;
  const size_t ntw = (size_t)(g.nx + g.ny + g.nz);
  if (how != TableUpload::kNone) {
    // twiddles exp(-2 pi i k / n) and the sin/cos tables of the modified wave vectors,
    // both evaluated in FP64 (fourier.py:29-31: xi_d / 2 = pi k_d / N_d)
    std::vector<float2> tw32;
    std::vector<double2> tw64;
    for (int n : {g.nx, g.ny, g.nz})
      for (int k = 0; k < n; ++k) {
        double a = -2.0 * M_PI * (double)k / (double)n;
        double c = std::cos(a), sn = std::sin(a);
        tw32.push_back(make_float2((float)c, (float)sn));
        tw64.push_back(make_double2(c, sn));
      }
    std::vector<double> tab;
    auto add_tab = [&](int n, int count) {
      for (int k = 0; k < count; ++k) tab.push_back(std::sin((2.0 * M_PI * k / n) / 2.0));
      for (int k = 0; k < count; ++k) tab.push_back(std::cos((2.0 * M_PI * k / n) / 2.0));
    };
    add_tab(g.nx, g.nx);
    add_tab(g.ny, g.ny);
    add_tab(g.nz, g.nzh);
    // (an asynchronous copy from pageable memory returns once the data is staged, so the
    // vectors may go out of scope)
    auto copy = [&](void* dst, const void* src, size_t bytes) {
      return how == TableUpload::kAsync
                 ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s->stream)
                 : cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
    };
    if (copy(s->d_tw32, tw32.data(), sizeof(float2) * ntw) != cudaSuccess ||
        copy(s->d_tw64, tw64.data(), sizeof(double2) * ntw) != cudaSuccess ||
        copy(s->d_tables, tab.data(), sizeof(double) * tab.size()) != cudaSuccess)
      return fail(-2, "upload of twiddle tables failed");
  }
  g.px.tw = s->d_tw32;
  g.py.tw = s->d_tw32 + g.nx;
  g.pz.tw = s->d_tw32 + g.nx + g.ny;
  g.px.tw64 = s->d_tw64;
  g.py.tw64 = s->d_tw64 + g.nx;
  g.pz.tw64 = s->d_tw64 + g.nx + g.ny;
  g.sx = s->d_tables;
  g.cx = g.sx + g.nx;
  g.sy = g.cx + g.nx;
  g.cy = g.sy + g.ny;
  g.sz = g.cy + g.ny;
  g.cz = g.sz + g.nzh;
  return 0;
}

}  // namespace detail
}  // namespace lsb

namespace {

int create_impl(lsb_solver** out, const int voxels[3], const double extents[3], int batch, int depth) {
  if (!out || !voxels || !extents) return fail(-1, "null argument");
  *out = nullptr;
  if (batch < 1) return fail(-1, "batch must be >= 1");
  if (depth < 0 || depth > kMaxDepth) return fail(-1, "Anderson depth %d outside [0, %d]", depth, kMaxDepth);
  auto* s = new lsb_solver();
  s->batch_cap = batch;
  s->depth = depth;
  // LSB_DEVICE_LOOP=0: host-polled graph replays instead of the conditional-node loop
  // (profilers cannot see the kernels of graphs that hold conditional nodes)
  if (const char* env = std::getenv("LSB_DEVICE_LOOP")) s->use_loop = std::string(env) != "0";
  cudaGetDevice(&s->device);
  int rc = plan_grid(s, voxels, extents);
  if (rc) {
    delete s;
    return rc;
  }
  const GridDesc& g = s->g;
  auto alloc = [&](void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) rc = fail(-3, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    return e == cudaSuccess;
  };
  const size_t B = (size_t)batch;
  // room for the partials of either x-pass tile variant
  const size_t xblk = (size_t)std::max({s->sh32.x_blocks_per_instance, s->sh64.x_blocks_per_instance,
                                        s->x_blocks_generic32,
                                        s->fast32 ? fast::x_tiles(g, 1) * g.ny : 0,
                                        s->fast32 && fast::tiled_supported(g) ? fast::x_tiles_tiled(g) : 0});
  const size_t ntw = (size_t)(g.nx + g.ny + g.nz);
  bool ok = alloc((void**)&s->d_eps32, sizeof(float) * B * 6 * g.nv) &&
            alloc((void**)&s->d_spec32, sizeof(float2) * B * 6 * g.nm) &&
            (!s->tiled || alloc((void**)&s->d_tspec32, sizeof(float2) * B * 6 * g.nm)) &&
            alloc((void**)&s->d_partials, sizeof(double) * B * xblk) &&
            alloc((void**)&s->d_state, sizeof(InstanceState) * B) &&
            alloc((void**)&s->d_medium, sizeof(Medium) * B) &&
            alloc((void**)&s->d_epsbar, sizeof(double) * B * 6) &&
            alloc((void**)&s->d_scratch, sizeof(double) * 6 * std::max<size_t>(1024, B)) &&
            alloc((void**)&s->d_mean_scratch, sizeof(double) * B * 6 * 1024) &&
            alloc((void**)&s->d_mean, sizeof(double) * B * 6) &&
            alloc((void**)&s->d_tw32, sizeof(float2) * ntw) &&
            alloc((void**)&s->d_tw64, sizeof(double2) * ntw) &&
            alloc((void**)&s->d_tables, sizeof(double) * 2 * (size_t)(g.nx + g.ny + g.nzh));
  if (!ok) {
    delete s;
    return rc;
  }
  if (depth > 0) {
    const size_t M1 = (size_t)depth + 1;
    s->aa_zblocks = std::max(std::max(s->sh32.z_blocks, s->sh64.z_blocks),
                             s->fast32 ? fast::z_blocks(g) : 0);
    ok = alloc((void**)&s->d_aa_g32, sizeof(float) * B * M1 * 6 * g.nv) &&
         alloc((void**)&s->d_aa_r32, sizeof(__half) * B * M1 * 6 * g.nv) &&
         alloc((void**)&s->d_aa_partials, sizeof(double) * B * s->aa_zblocks * (M1 + 1)) &&
         alloc((void**)&s->d_aa_mat, sizeof(double) * B * M1 * M1) &&
         alloc((void**)&s->d_aa_alpha, sizeof(double) * B * M1);
    if (!ok) {
      delete s;
      return rc;
    }
  }
  if (cudaMallocHost(&s->h_state, sizeof(InstanceState) * B) != cudaSuccess) {
    delete s;
    return fail(-3, "cudaMallocHost failed");
  }
  rc = upload_tables(s);
  if (rc) {
    delete s;
    return rc;
  }
  *out = s;
  return 0;
}

SolveParams make_params(const lsb_solver* s, double rtol, double atol, int maxiter, int rule) {
  SolveParams sp;
  sp.rtol = rtol;
  sp.atol = atol;
  sp.maxiter = maxiter;
  sp.rule = rule;
  sp.nv = s->g.nv;
  sp.precision = s->precision;
  sp.stall_window = s->stall_window;
  sp.stall_improve = 0.98;
  sp.stall_near = 4.0;
  return sp;
}

// The fused slab pass runs this FP32 solve's y and z passes (isotropic law only).
inline bool use_slab(const lsb_solver* s) { return s->slab && !s->g.cf32 && !s->g.dmg32; }

template <typename T>
void pass_slab(lsb_solver* s, int mode, int batch, const T* lam, const T* mu, T* eps,
               const T* eps0, const AndersonArgs<T>& aa) {
  if constexpr (sizeof(T) == 4) {
    const cudaError_t e = fast::launch_slab(s->g, mode, batch, lam, mu, eps, s->d_tspec32, s->d_epsbar,
                                            eps0, s->d_state, s->d_medium, aa, s->stream);
    if (e != cudaSuccess && s->launch_error == cudaSuccess) s->launch_error = e;
  }
}

// The first launch error recorded since the last call (cleared), or cudaGetLastError().
inline cudaError_t take_launch_error(lsb_solver* s) {
  const cudaError_t e = s->launch_error;
  s->launch_error = cudaSuccess;
  const cudaError_t last = cudaGetLastError();
  return e != cudaSuccess ? e : last;
}

// Pass dispatch: FP32 fields use the compile-time-size passes when every extent is a
// supported power of two, the generic passes otherwise.
template <typename T>
void pass_z(lsb_solver* s, int mode, int batch, const T* lam, const T* mu, T* eps, cplx<T>* spec,
            const T* eps0, const AndersonArgs<T>& aa) {
  if constexpr (sizeof(T) == 4) {
    if (use_fast32(s)) {
      fast::launch_zpass(s->g, mode, batch, lam, mu, eps, spec, s->d_epsbar, eps0, s->d_state,
                         s->d_medium, aa, s->stream);
      return;
    }
  }
  launch_zpass<T>(s->g, sizeof(T) == 8 ? s->sh64 : s->sh32, mode, batch, lam, mu, eps, spec,
                  s->d_epsbar, eps0, s->d_state, s->d_medium, aa, s->stream);
}

template <typename T>
void pass_y(lsb_solver* s, bool inverse, int batch, cplx<T>* spec) {
  if constexpr (sizeof(T) == 4) {
    if (use_fast32(s)) {
      fast::launch_ypass(s->g, s->yvariant, inverse, batch, spec, s->tiled ? s->d_tspec32 : nullptr,
                         s->d_state, s->stream);
      return;
    }
  }
  launch_ypass<T>(s->g, sizeof(T) == 8 ? s->sh64 : s->sh32, inverse, batch, spec, s->d_state, s->stream);
}

template <typename T>
void pass_x(lsb_solver* s, int batch, cplx<T>* spec) {
  if constexpr (sizeof(T) == 4) {
    if (use_fast32(s)) {
      if (s->tiled) {
        fast::launch_xpass_tiled(s->g, batch, s->d_tspec32, s->d_medium, s->d_state, s->d_partials,
                                 s->stream);
        return;
      }
      fast::launch_xpass(s->g, s->xvariant, batch, spec, s->d_medium, s->d_state, s->d_partials,
                         s->stream);
      return;
    }
  }
  launch_xpass<T>(s->g, sizeof(T) == 8 ? s->sh64 : s->sh32, batch, spec, s->d_medium, s->d_state,
                  s->d_partials, s->stream);
}

// Runs the loop of precision T for every instance in its phase until none is left there.
// init_mode: 0 (eps from eps_bar / eps0) or 2 (continue from eps in place).
// With `anderson` the update is Anderson mixing of depth s->depth (rings of precision T).
// Start of a phase's device-driven loop inside a larger graph: resets the evaluation count
// and opens the loop only if an instance of `phase` is running (the loop's default is
// closed). One warp.
__global__ void loop_arm_kernel(cudaGraphConditionalHandle handle, const InstanceState* __restrict__ st,
                                int batch, int phase, int* count) {
  int any = 0;
  for (int b = threadIdx.x; b < batch; b += 32) any |= (!st[b].done && st[b].phase == phase) ? 1 : 0;
  any = __any_sync(0xffffffffu, any);
  if (threadIdx.x == 0) {
    *count = 0;
    cudaGraphSetConditional(handle, any ? 1u : 0u);
  }
}

// Moves a phase's work to the solver's graph stream (ordered after everything already on
// the caller's stream) and back (the caller's stream waits for the phase); owns the graph.
// End of one body execution of a phase's device-driven loop: counts the evaluations and
// keeps the loop going while an instance of `phase` is still running and fewer than
// max_evals evaluations have run (the hard cap that makes the loop terminate even if no
// instance stops). One warp.
__global__ void loop_check_kernel(cudaGraphConditionalHandle handle, const InstanceState* __restrict__ st,
                                  int batch, int phase, int* count, int max_evals) {
  int any = 0;
  for (int b = threadIdx.x; b < batch; b += 32) any |= (!st[b].done && st[b].phase == phase) ? 1 : 0;
  any = __any_sync(0xffffffffu, any);
  if (threadIdx.x == 0) {
    const int c = *count + 1;
    *count = c;
    cudaGraphSetConditional(handle, (any && c < max_evals) ? 1u : 0u);
  }
}

struct GraphPhase {
  lsb_solver* s;
  cudaStream_t user;
  bool on = false;
  bool loop = false;  // the graph is a device-driven WHILE loop over the iteration
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  explicit GraphPhase(lsb_solver* solver) : s(solver), user(solver->stream) {
    if (!s->use_graphs) return;
    // (the graph stream takes the caller's stream priority)
    int prio = 0;
    if (cudaStreamGetPriority(user, &prio) != cudaSuccess) {
      cudaGetLastError();
      prio = 0;
    }
    if (!s->graph_stream &&
        cudaStreamCreateWithPriority(&s->graph_stream, cudaStreamNonBlocking, prio) != cudaSuccess) {
      s->graph_stream = nullptr;
      cudaGetLastError();
      return;
    }
    if ((!s->ev_in && cudaEventCreateWithFlags(&s->ev_in, cudaEventDisableTiming) != cudaSuccess) ||
        (!s->ev_out && cudaEventCreateWithFlags(&s->ev_out, cudaEventDisableTiming) != cudaSuccess)) {
      cudaGetLastError();
      return;
    }
    if (cudaEventRecord(s->ev_in, user) != cudaSuccess ||
        cudaStreamWaitEvent(s->graph_stream, s->ev_in, 0) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    s->stream = s->graph_stream;
    on = true;
  }
  // Captures one enqueue() into a graph; on any failure the phase runs without it.
  template <typename F>
  void capture(F&& enqueue) {
    if (!on) return;
    if (cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    enqueue();
    cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
    if (e == cudaSuccess && graph) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) {
      if (exec) cudaGraphExecDestroy(exec);
      if (graph) cudaGraphDestroy(graph);
      exec = nullptr;
      graph = nullptr;
      cudaGetLastError();
    }
  }
  // Builds a graph of one conditional WHILE node whose body is one enqueue() followed by
  // loop_check_kernel, so that a single launch runs the phase to its end; on any failure
  // nothing is kept (capture() or the host-polled loop remains).
  template <typename F>
  bool capture_loop(F&& enqueue, int batch, int phase, int max_evals) {
    if (!on) return false;
    if (!s->d_loop_count && cudaMalloc(&s->d_loop_count, sizeof(int)) != cudaSuccess) {
      s->d_loop_count = nullptr;
      cudaGetLastError();
      return false;
    }
    cudaGraph_t g = nullptr;
    cudaGraphConditionalHandle handle;
    cudaGraphNode_t node;
    cudaGraphNodeParams params = {};
    bool ok = cudaGraphCreate(&g, 0) == cudaSuccess &&
              cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) {
      params.type = cudaGraphNodeTypeConditional;
      params.conditional.handle = handle;
      params.conditional.type = cudaGraphCondTypeWhile;
      params.conditional.size = 1;
      ok = cudaGraphAddNode(&node, g, nullptr, 0, &params) == cudaSuccess;
    }
    if (ok) {
      cudaGraph_t body = params.conditional.phGraph_out[0];
      ok = cudaStreamBeginCaptureToGraph(s->stream, body, nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      if (ok) {
        enqueue();
        loop_check_kernel<<<1, 32, 0, s->stream>>>(handle, s->d_state, batch, phase, s->d_loop_count,
                                                   max_evals);
        cudaGraph_t captured = nullptr;
        ok = cudaStreamEndCapture(s->stream, &captured) == cudaSuccess;
      }
    }
    if (ok) ok = cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
    if (!ok) {
      if (exec) cudaGraphExecDestroy(exec);
      if (g) cudaGraphDestroy(g);
      exec = nullptr;
      cudaGetLastError();
      return false;
    }
    graph = g;
    loop = true;
    return true;
  }
  ~GraphPhase() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (on) {
      cudaEventRecord(s->ev_out, s->stream);
      cudaStreamWaitEvent(user, s->ev_out, 0);
      s->stream = user;
    }
  }
};

// Records an event on the solver's stream after each launch of one iteration (profiling).
struct StepTimer {
  cudaStream_t st;
  std::vector<cudaEvent_t> ev;        // ev[0] before the first launch, ev[k] after launch k
  std::vector<const char*> names;     // names[k - 1]: kernel of launch k
  size_t next = 1;
  void mark(const char* name) {
    if (next < ev.size()) cudaEventRecord(ev[next], st);
    if (names.size() < next) names.push_back(name);
    ++next;
  }
};

// Blocks per instance of the Anderson Gram-row kernel: about four 16-byte element groups
// per thread (fewer left the 64^3 Gram row dominated by its block reductions), at most 2048
// and within the z-block-sized partials buffer.
int gram_blocks(const lsb_solver* s) {
  return (int)std::max<long long>(
      1, std::min<long long>({(long long)s->aa_zblocks, 2048LL, (6 * s->g.nv + 4095) / 4096}));
}

// One iteration of precision T: x pass, criterion and stop decision, inverse y pass, then
// either the plain update (z pass mode 1) or the Anderson update (residual rings, Gram
// row, coefficients, combine, stress of the combined iterate), and the forward y pass.
template <typename T>
void enqueue_iteration(lsb_solver* s, int batch, const T* lam, const T* mu, T* eps, cplx<T>* spec,
                       const AndersonArgs<T>& aa, const SolveParams& sp, const LaunchShape& sh,
                       int phase, const T* inject, StepTimer* tm) {
  cudaStream_t st = s->stream;
  auto mark = [&](const char* name) {
    if (tm) tm->mark(name);
  };
  pass_x<T>(s, batch, spec);
  mark("x pass");
  launch_finalize(sh, phase, batch, s->d_state, s->d_partials, s->d_history, s->history_len, sp, st);
  mark("finalize");
  if (sizeof(T) == 4 && use_slab(s)) {
    if (aa.depth > 0) {
      const int gblk = gram_blocks(s);
      pass_slab<T>(s, 3, batch, lam, mu, eps, nullptr, aa);
      mark("slab residual rings");
      launch_anderson_gram<T>(s->g.nv, gblk, s->depth, phase, batch, s->d_state, aa.r,
                              s->d_aa_partials, st);
      mark("anderson gram");
      launch_anderson_solve(gblk, s->depth, phase, batch, s->d_state, s->d_aa_partials,
                            s->d_aa_mat, s->d_aa_alpha, st);
      mark("anderson solve");
      launch_anderson_combine<T>(s->g.nv, s->depth, phase, batch, s->d_state, aa.g, s->d_aa_alpha,
                                 eps, st, inject);
      mark("anderson combine");
      pass_slab<T>(s, 2, batch, lam, mu, eps, nullptr, aa);
      mark("slab stress");
    } else {
      pass_slab<T>(s, 1, batch, lam, mu, eps, nullptr, aa);
      mark("slab update");
    }
    return;
  }
  pass_y<T>(s, true, batch, spec);
  mark("y pass inverse");
  if (aa.depth > 0) {
    const int gblk = gram_blocks(s);
    pass_z<T>(s, 3, batch, lam, mu, eps, spec, nullptr, aa);
    mark("z pass residual rings");
    launch_anderson_gram<T>(s->g.nv, gblk, s->depth, phase, batch, s->d_state, aa.r,
                            s->d_aa_partials, st);
    mark("anderson gram");
    launch_anderson_solve(gblk, s->depth, phase, batch, s->d_state, s->d_aa_partials,
                          s->d_aa_mat, s->d_aa_alpha, st);
    mark("anderson solve");
    launch_anderson_combine<T>(s->g.nv, s->depth, phase, batch, s->d_state, aa.g, s->d_aa_alpha,
                               eps, st, inject);
    mark("anderson combine");
    pass_z<T>(s, 2, batch, lam, mu, eps, spec, nullptr, aa);
    mark("z pass stress");
  } else {
    pass_z<T>(s, 1, batch, lam, mu, eps, spec, nullptr, aa);
    mark("z pass update");
  }
  pass_y<T>(s, false, batch, spec);
  mark("y pass forward");
}

// Kernels launched by one iteration.
inline long long iteration_launches(bool mix, bool slab) {
  return slab ? (mix ? 7LL : 3LL) : (mix ? 9LL : 5LL);
}

// Runs the loop of precision T for every instance in its phase until none is left there.
// init_mode: 0 (eps from eps_bar / eps0) or 2 (continue from eps in place).
// With `anderson` the update is Anderson mixing of depth s->depth (rings of precision T).
// One iteration is captured into a CUDA graph and replayed (s->use_graphs).
template <typename T>
int run_phase(lsb_solver* s, int batch, const T* lam, const T* mu, T* eps, cplx<T>* spec,
              const T* eps0, int init_mode, const SolveParams& sp, bool anderson,
              const T* inject = nullptr) {
  LaunchShape sh = sizeof(T) == 8 ? s->sh64 : s->sh32;
  if (sizeof(T) == 4 && !use_fast32(s)) sh.x_blocks_per_instance = s->x_blocks_generic32;
  const int phase = sizeof(T) == 8 ? 1 : 0;
  GraphPhase gp(s);
  cudaStream_t st = s->stream;
  const AndersonArgs<T> aa = anderson_args<T>(s, anderson && s->depth > 0);
  const bool mix = aa.depth > 0;
  const bool slab = sizeof(T) == 4 && use_slab(s);
  if (slab) {
    pass_slab<T>(s, init_mode, batch, lam, mu, eps, eps0, aa);
    s->launches += 1;
  } else {
    pass_z<T>(s, init_mode, batch, lam, mu, eps, spec, eps0, aa);
    pass_y<T>(s, false, batch, spec);
    s->launches += 2;
  }
  LSB_CUDA(take_launch_error(s));
  auto iteration = [&]() {
    enqueue_iteration<T>(s, batch, lam, mu, eps, spec, aa, sp, sh, phase, inject, nullptr);
  };
  const long long max_evals = (long long)sp.maxiter + 2;
  // one launch runs the whole phase: a WHILE node over the iteration, stopped on the device
  if (s->use_loop && gp.capture_loop(iteration, batch, phase, (int)max_evals)) {
    LSB_CUDA(cudaMemsetAsync(s->d_loop_count, 0, sizeof(int), st));
    LSB_CUDA(cudaGraphLaunch(gp.exec, st));
    int evals = 0;
    LSB_CUDA(cudaMemcpyAsync(s->h_state, s->d_state, sizeof(InstanceState) * batch,
                             cudaMemcpyDeviceToHost, st));
    LSB_CUDA(cudaMemcpyAsync(&evals, s->d_loop_count, sizeof(int), cudaMemcpyDeviceToHost, st));
    LSB_CUDA(cudaStreamSynchronize(st));
    LSB_CUDA(take_launch_error(s));
    s->launches += (iteration_launches(mix, slab) + 1) * evals;
    for (int b = 0; b < batch; ++b)
      if (!s->h_state[b].done && s->h_state[b].phase == phase)
        return fail(-4, "internal: iteration loop stopped after %d evaluations with instance %d running",
                    evals, b);
    return 0;
  }
  gp.capture(iteration);
  long long launched = 0;
  int chunk = 1;
  for (;;) {
    int n = (int)std::min<long long>(chunk, max_evals - launched);
    for (int i = 0; i < n; ++i) {
      if (gp.exec) {
        LSB_CUDA(cudaGraphLaunch(gp.exec, st));
      } else {
        iteration();
      }
    }
    launched += n;
    s->launches += iteration_launches(mix, slab) * n;
    LSB_CUDA(take_launch_error(s));
    LSB_CUDA(cudaMemcpyAsync(s->h_state, s->d_state, sizeof(InstanceState) * batch,
                             cudaMemcpyDeviceToHost, st));
    LSB_CUDA(cudaStreamSynchronize(st));
    bool left = false;
    for (int b = 0; b < batch; ++b) left = left || (!s->h_state[b].done && s->h_state[b].phase == phase);
    if (!left) return 0;
    if (launched >= max_evals) return fail(-4, "internal: iteration driver did not terminate");
    chunk = std::min(chunk * 2, 32);
  }
}

// ---- autotuner of the FP32 pass configuration
//
// Candidates for a grid of the compile-time-size passes: the tiled spectrum layout
// between the y and x passes (when the solver holds its buffer), the fused slab pass
// over it (ny == nz, isotropic law), and the strided x pass with either tile variant.
// Each runs the solve's own iteration (Anderson when depth > 0) on this solver's buffers
// from a fresh state: the initial pass, depth + 2 untimed iterations that fill the
// Anderson rings, then kTuneReps timed iterations (CUDA events on the solver's stream,
// tolerances 0 so that every pass does its full work). The fastest is kept; the choice is
// timed on at most 24 of the solve's instances and remembered per (device, grid, depth, law)
// for the process and in a cache file
// (LSB_TUNE_CACHE, else $HOME/.cache/jaxmaterials_b200/tune.tsv; an empty value or "0"
// disables the file), so that later processes skip the timing.
struct TuneChoice {
  int tiled, xvariant, slab, yvariant;
};
constexpr int kTuneReps = 3;

std::mutex g_tune_mu;
std::map<std::string, TuneChoice>* g_tune = nullptr;

std::string tune_path() {
  const char* env = std::getenv("LSB_TUNE_CACHE");
  if (env) return (env[0] == '\0' || std::string(env) == "0") ? std::string() : std::string(env);
  const char* home = std::getenv("HOME");
  if (!home || !home[0]) return std::string();
  return std::string(home) + "/.cache/jaxmaterials_b200/tune.tsv";
}

void tune_load_locked() {
  if (g_tune) return;
  g_tune = new std::map<std::string, TuneChoice>();
  const std::string path = tune_path();
  if (path.empty()) return;
  std::ifstream in(path);
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    std::string key;
    TuneChoice c{};
    if (std::getline(ls, key, '\t') && (ls >> c.tiled >> c.xvariant >> c.slab >> c.yvariant)) (*g_tune)[key] = c;
  }
}

void tune_store_locked(const std::string& key, const TuneChoice& c, float ms) {
  (*g_tune)[key] = c;
  const std::string path = tune_path();
  if (path.empty()) return;
  const size_t slash = path.rfind('/');
  if (slash != std::string::npos) {
    // create the directory chain (ignore failures: the choice then stays in memory only)
    std::string dir = path.substr(0, slash);
    for (size_t k = 1; k <= dir.size(); ++k)
      if (k == dir.size() || dir[k] == '/') mkdir(dir.substr(0, k).c_str(), 0755);
  }
  std::ofstream out(path, std::ios::app);
  if (out)
    out << key << '\t' << c.tiled << '\t' << c.xvariant << '\t' << c.slab << '\t' << c.yvariant << '\t' << ms
        << '\n';
}

std::string tune_key(const lsb_solver* s) {
  cudaDeviceProp prop;
  std::string dev = "device";
  if (cudaGetDeviceProperties(&prop, s->device) == cudaSuccess)
    dev = std::string(prop.name) + "/" + std::to_string(prop.multiProcessorCount);
  const char* law = s->g.cf32 ? "aniso" : (s->g.dmg32 ? "damage" : "iso");
  char buf[256];
  // (|y: the entries that carry the y-pass variant)
  std::snprintf(buf, sizeof(buf), "%s|%dx%dx%d|m%d|%s|y", dev.c_str(), s->g.nx, s->g.ny, s->g.nz,
                s->depth, law);
  return buf;
}

void apply_choice(lsb_solver* s, const TuneChoice& c) {
  s->tiled = c.tiled && s->d_tspec32 != nullptr && fast::tiled_supported(s->g);
  s->slab = c.slab && s->tiled && fast::slab_supported(s->g);
  s->xvariant = c.xvariant;
  s->yvariant = c.yvariant;
  if (s->tiled) s->sh32.x_blocks_per_instance = fast::x_tiles_tiled(s->g);
  else s->sh32.x_blocks_per_instance = fast::x_tiles(s->g, s->xvariant) * s->g.ny;
}

// Times kTuneReps iterations of the current configuration (see above); ms per iteration.
int time_config(lsb_solver* s, int batch, const float* d_lambda, const float* d_mu, float* d_eps,
                int nstruct, float* ms_out) {
  cudaStream_t st = s->stream;
  SolveParams sp = make_params(s, 0.0, 0.0, 0x3fffffff, LSB_RULE_CUDA);
  sp.precision = kPrecFP32;
  sp.stall_window = 0;
  LaunchShape sh = s->sh32;
  launch_reset_state(batch, 0, s->d_state, st);
  launch_medium<float>(s->g.nv, nstruct, d_lambda, d_mu, s->d_scratch, s->d_medium, st);
  const AndersonArgs<float> aa = anderson_args<float>(s, s->depth > 0);
  if (use_slab(s)) {
    pass_slab<float>(s, 0, batch, d_lambda, d_mu, d_eps, nullptr, aa);
  } else {
    pass_z<float>(s, 0, batch, d_lambda, d_mu, d_eps, s->d_spec32, nullptr, aa);
    pass_y<float>(s, false, batch, s->d_spec32);
  }
  for (int i = 0; i < s->depth + 2; ++i)
    enqueue_iteration<float>(s, batch, d_lambda, d_mu, d_eps, s->d_spec32, aa, sp, sh, 0, nullptr, nullptr);
  cudaEvent_t ev[2];
  LSB_CUDA(cudaEventCreate(&ev[0]));
  LSB_CUDA(cudaEventCreate(&ev[1]));
  cudaEventRecord(ev[0], st);
  for (int i = 0; i < kTuneReps; ++i)
    enqueue_iteration<float>(s, batch, d_lambda, d_mu, d_eps, s->d_spec32, aa, sp, sh, 0, nullptr, nullptr);
  cudaEventRecord(ev[1], st);
  cudaError_t e = cudaEventSynchronize(ev[1]);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev[0], ev[1]);
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (e == cudaSuccess) e = take_launch_error(s);
  if (e != cudaSuccess) return fail(-2, "pass tuning: %s", cudaGetErrorString(e));
  s->launches += (long long)(s->depth + 2 + kTuneReps) * iteration_launches(s->depth > 0, use_slab(s)) + 4;
  *ms_out = ms / kTuneReps;
  return 0;
}

// Chooses the pass configuration of the fast FP32 passes (see above). Runs once per solver
// unless the caller fixed the configuration (lsb_tile_variant, lsb_set_tiled, lsb_set_slab);
// leaves the per-instance state to be reset by the solve.
int tune_passes(lsb_solver* s, int batch, const float* d_lambda, const float* d_mu, float* d_eps,
                int nstruct) {
  if (!use_fast32(s)) return 0;  // the generic passes have one configuration
  s->xtuned = true;
  const std::string key = tune_key(s);
  // up to 24 instances (structures_of has set g.lame_group for the solve's batch): enough
  // for the small grids' ranking to be that of their large batches
  const int tb = std::min(batch, 24);
  nstruct = (tb + s->g.lame_group - 1) / s->g.lame_group;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    tune_load_locked();
    auto f = g_tune->find(key);
    if (f != g_tune->end()) {
      apply_choice(s, f->second);
      return 0;
    }
  }
  // (each configuration with either y-pass column count, except the slab pass, which has
  // no y pass of its own)
  std::vector<TuneChoice> cand;
  if (s->d_tspec32 && fast::tiled_supported(s->g)) {
    cand.push_back({1, 0, 0, 0});
    cand.push_back({1, 0, 0, 1});
    if (fast::slab_supported(s->g) && !s->g.cf32 && !s->g.dmg32) cand.push_back({1, 0, 1, 0});
  }
  cand.push_back({0, 0, 0, 0});
  cand.push_back({0, 0, 0, 1});
  if (fast::x_tiles(s->g, 0) != fast::x_tiles(s->g, 1)) {
    cand.push_back({0, 1, 0, 0});
    cand.push_back({0, 1, 0, 1});
  }
  TuneChoice best = cand[0];
  float best_ms = 0.f;
  if (cand.size() > 1) {
    for (size_t k = 0; k < cand.size(); ++k) {
      apply_choice(s, cand[k]);
      float ms = 0.f;
      LSB_TRY(time_config(s, tb, d_lambda, d_mu, d_eps, nstruct, &ms));
      if (k == 0 || ms < best_ms) {
        best_ms = ms;
        best = cand[k];
      }
    }
  }
  apply_choice(s, best);
  std::lock_guard<std::mutex> lock(g_tune_mu);
  tune_store_locked(key, best, best_ms);
  return 0;
}

}  // namespace

namespace lsb {
namespace detail {

// Full solve with FP32 inputs/outputs. d_eps (FP32) is the FP32 work buffer and output.
int solve_f32(lsb_solver* s, int batch, const float* d_lambda, const float* d_mu,
              const double* eps_bar, const float* d_eps0, float* d_eps, float* d_sigma,
              double* mean_sigma, double rtol, double atol, int maxiter, int rule, int* iters,
              int* status, double* residual) {
  if (!s) return fail(-1, "null solver");
  if (batch < 1 || batch > s->batch_cap) return fail(-1, "batch %d outside [1, %d]", batch, s->batch_cap);
  if (!d_lambda || !d_mu || !eps_bar || !iters || !status || !d_eps) return fail(-1, "null argument");
  if (maxiter < 0) return fail(-1, "maxiter must be >= 0");
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != s->device) return fail(-1, "solver was created on device %d, current is %d", s->device, cur);
  const GridDesc& g = s->g;
  cudaStream_t st = s->stream;
  const int nstruct = structures_of(s, batch);
  if (nstruct < 0) return nstruct;
  LSB_TRY(prepare_damage(s, nstruct));
  LSB_TRY(prepare_aniso(s, nstruct));
  LSB_TRY(ensure_history(s, maxiter + 8));
  const SolveParams sp = make_params(s, rtol, atol, maxiter, rule);
  const bool fp64_start = s->precision == kPrecFP64;
  if (s->precision != kPrecFP32) LSB_TRY(ensure_fp64(s, nstruct));

  LSB_CUDA(cudaMemcpyAsync(s->d_epsbar, eps_bar, sizeof(double) * 6 * batch, cudaMemcpyHostToDevice, st));
  if (!s->xtuned && !fp64_start) LSB_TRY(tune_passes(s, batch, d_lambda, d_mu, d_eps, nstruct));
  if (s->d_history)
    LSB_CUDA(cudaMemsetAsync(s->d_history, 0, sizeof(double) * (size_t)batch * s->history_len, st));
  launch_reset_state(batch, fp64_start ? 1 : 0, s->d_state, st, s->use_e0ref ? s->d_e0ref : nullptr);
  launch_medium<float>(g.nv, nstruct, d_lambda, d_mu, s->d_scratch, s->d_medium, st);
  s->launches += 3;
  bool any64 = fp64_start;
  if (!fp64_start) {
    // a warm start either starts the iteration or (warm_history) enters the Anderson
    // history as the second iterate, after the cold start's
    const bool hist = s->warm_history && d_eps0 && s->depth > 0;
    LSB_TRY(run_phase<float>(s, batch, d_lambda, d_mu, d_eps, s->d_spec32, hist ? nullptr : d_eps0,
                             0, sp, true, hist ? d_eps0 : nullptr));
    for (int b = 0; b < batch; ++b) any64 = any64 || (s->h_state[b].phase == 1 && !s->h_state[b].done);
  }
  if (any64) {
    const long long n6 = 6 * g.nv;
    const long long nl = (long long)nstruct * g.nv;
    launch_convert<float, double>(nl, d_lambda, s->d_lame64, st);
    launch_convert<float, double>(nl, d_mu, s->d_lame64 + nl, st);
    s->launches += 2;
    if (fp64_start && d_eps0) {
      launch_convert_fields<float, double>(n6, batch, 1, s->d_state, d_eps0, s->d_eps64, st);
      s->launches += 1;
    } else if (!fp64_start) {
      launch_convert_fields<float, double>(n6, batch, 1, s->d_state, d_eps, s->d_eps64, st);
      s->launches += 1;
    }
    const int init_mode = fp64_start ? (d_eps0 ? 2 : 0) : 2;
    // FP64 from the start runs Anderson in FP64; the continuation after an FP32 stall is
    // a few plain updates from the FP32 iterate.
    if (fp64_start) LSB_TRY(ensure_fp64_rings(s));
    LSB_TRY(run_phase<double>(s, batch, s->d_lame64, s->d_lame64 + nl, s->d_eps64, s->d_spec64,
                              nullptr, init_mode, sp, fp64_start));
    launch_convert_fields<double, float>(n6, batch, 0, s->d_state, s->d_eps64, d_eps, st);
    launch_stress<double, float>(g, 1, batch, s->d_state, s->d_lame64, s->d_lame64 + nl, s->d_eps64,
                                 d_sigma, s->d_mean_scratch, s->d_mean, st);
    s->launches += 3;
  }
  launch_stress<float, float>(g, 0, batch, s->d_state, d_lambda, d_mu, d_eps, d_sigma,
                              s->d_mean_scratch, s->d_mean, st);
  s->launches += 2;
  LSB_CUDA(take_launch_error(s));
  if (mean_sigma)
    LSB_CUDA(cudaMemcpyAsync(mean_sigma, s->d_mean, sizeof(double) * 6 * batch, cudaMemcpyDeviceToHost, st));
  LSB_CUDA(cudaMemcpyAsync(s->h_state, s->d_state, sizeof(InstanceState) * batch, cudaMemcpyDeviceToHost, st));
  LSB_CUDA(cudaStreamSynchronize(st));
  for (int b = 0; b < batch; ++b) {
    iters[b] = s->h_state[b].iter;
    status[b] = s->h_state[b].status;
    if (residual) residual[b] = s->h_state[b].e;
  }
  s->last_batch = batch;
  return 0;
}

// Appends the device work of one FP32-start solve of `batch` instances (the sequence of
// solve_f32: reset, media, initial pass, the FP32 loop, the FP64 continuation of stalled
// instances, the means of the stresses) to `graph`, after the nodes in `deps`; both loops
// are conditional WHILE nodes opened and stopped on the device. The mean stresses and the
// instance states are copied into the pinned h_mean ([batch][6]) and h_state ([batch]) at
// the end. *last receives the terminal nodes, *bodies (if given) the loops' body graphs.
// The caller has prepared the solver
// (prepare_graph_solve) and owns the two capture streams. Returns 0 or a negative code
// (the graph is then unusable).
int append_solve_f32(lsb_solver* s, cudaGraph_t graph, const std::vector<cudaGraphNode_t>& deps,
                     cudaStream_t cap, cudaStream_t body_st, int batch, const float* d_lambda,
                     const float* d_mu, double rtol, double atol, int maxiter, double* h_mean,
                     InstanceState* h_state, std::vector<cudaGraphNode_t>* last,
                     std::vector<cudaGraph_t>* bodies) {
  const GridDesc& g = s->g;
  const int nstruct = structures_of(s, batch);
  if (nstruct < 0) return nstruct;
  if (!s->d_loop_count) LSB_CUDA(cudaMalloc(&s->d_loop_count, sizeof(int)));
  const SolveParams sp = make_params(s, rtol, atol, maxiter, LSB_RULE_CUDA);
  const int max_evals = maxiter + 2;
  cudaStream_t saved = s->stream;
  s->stream = cap;
  LSB_CUDA(cudaStreamBeginCaptureToGraph(cap, graph, deps.empty() ? nullptr : deps.data(), nullptr,
                                         deps.size(), cudaStreamCaptureModeThreadLocal));
  // one conditional WHILE node at the capture's current position, opened by
  // loop_arm_kernel; its body (one iteration and loop_check_kernel) captured on body_st
  auto add_loop = [&](auto iteration, int phase) -> bool {
    cudaGraphConditionalHandle h;
    if (cudaGraphConditionalHandleCreate(&h, graph, 0, cudaGraphCondAssignDefault) != cudaSuccess) return false;
    loop_arm_kernel<<<1, 32, 0, cap>>>(h, s->d_state, batch, phase, s->d_loop_count);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* cur = nullptr;
    size_t ncur = 0;
    if (cudaStreamGetCaptureInfo(cap, &cs, nullptr, nullptr, &cur, &ncur) != cudaSuccess ||
        cs != cudaStreamCaptureStatusActive)
      return false;
    cudaGraphNodeParams params = {};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = h;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t node;
    std::vector<cudaGraphNode_t> cdeps(cur, cur + ncur);
    if (cudaGraphAddNode(&node, graph, cdeps.data(), cdeps.size(), &params) != cudaSuccess) return false;
    cudaGraph_t body = params.conditional.phGraph_out[0];
    if (bodies) bodies->push_back(body);
    if (cudaStreamBeginCaptureToGraph(body_st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess)
      return false;
    s->stream = body_st;
    iteration();
    loop_check_kernel<<<1, 32, 0, body_st>>>(h, s->d_state, batch, phase, s->d_loop_count, max_evals);
    s->stream = cap;
    cudaGraph_t captured = nullptr;
    if (cudaStreamEndCapture(body_st, &captured) != cudaSuccess) return false;
    return cudaStreamUpdateCaptureDependencies(cap, &node, 1, cudaStreamSetCaptureDependencies) == cudaSuccess;
  };
  bool ok = true;
  if (s->d_history) cudaMemsetAsync(s->d_history, 0, sizeof(double) * (size_t)batch * s->history_len, cap);
  launch_reset_state(batch, 0, s->d_state, cap, nullptr);
  launch_medium<float>(g.nv, nstruct, d_lambda, d_mu, s->d_scratch, s->d_medium, cap);
  {
    LaunchShape sh = s->sh32;
    if (!use_fast32(s)) sh.x_blocks_per_instance = s->x_blocks_generic32;
    const AndersonArgs<float> aa = anderson_args<float>(s, s->depth > 0);
    float* eps = s->d_eps32;
    if (use_slab(s)) {
      pass_slab<float>(s, 0, batch, d_lambda, d_mu, eps, nullptr, aa);
    } else {
      pass_z<float>(s, 0, batch, d_lambda, d_mu, eps, s->d_spec32, nullptr, aa);
      pass_y<float>(s, false, batch, s->d_spec32);
    }
    ok = add_loop([&]() { enqueue_iteration<float>(s, batch, d_lambda, d_mu, eps, s->d_spec32, aa, sp, sh, 0,
                                                  nullptr, nullptr); }, 0);
  }
  if (ok && s->precision == kPrecMixed) {
    // continuation of the instances that stalled in FP32 (every kernel below skips the
    // others; with none, the FP64 loop does not open)
    const long long n6 = 6 * g.nv;
    const long long nl = (long long)nstruct * g.nv;
    launch_convert<float, double>(nl, d_lambda, s->d_lame64, cap);
    launch_convert<float, double>(nl, d_mu, s->d_lame64 + nl, cap);
    launch_convert_fields<float, double>(n6, batch, 1, s->d_state, s->d_eps32, s->d_eps64, cap);
    const double* lam64 = s->d_lame64;
    const double* mu64 = s->d_lame64 + nl;
    LaunchShape sh = s->sh64;
    const AndersonArgs<double> aa = anderson_args<double>(s, false);
    pass_z<double>(s, 2, batch, lam64, mu64, s->d_eps64, s->d_spec64, nullptr, aa);
    pass_y<double>(s, false, batch, s->d_spec64);
    ok = add_loop([&]() { enqueue_iteration<double>(s, batch, lam64, mu64, s->d_eps64, s->d_spec64, aa, sp,
                                                   sh, 1, nullptr, nullptr); }, 1);
    if (ok) {
      launch_convert_fields<double, float>(n6, batch, 0, s->d_state, s->d_eps64, s->d_eps32, cap);
      launch_stress<double, float>(g, 1, batch, s->d_state, lam64, mu64, s->d_eps64, nullptr,
                                   s->d_mean_scratch, s->d_mean, cap);
    }
  }
  if (ok) {
    launch_stress<float, float>(g, 0, batch, s->d_state, d_lambda, d_mu, s->d_eps32, nullptr,
                                s->d_mean_scratch, s->d_mean, cap);
    cudaMemcpyAsync(h_mean, s->d_mean, sizeof(double) * 6 * batch, cudaMemcpyDeviceToHost, cap);
    cudaMemcpyAsync(h_state, s->d_state, sizeof(InstanceState) * batch, cudaMemcpyDeviceToHost, cap);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* cur = nullptr;
    size_t ncur = 0;
    ok = cudaStreamGetCaptureInfo(cap, &cs, nullptr, nullptr, &cur, &ncur) == cudaSuccess &&
         cs == cudaStreamCaptureStatusActive;
    if (ok) last->assign(cur, cur + ncur);
  }
  cudaGraph_t captured = nullptr;
  const cudaError_t e = cudaStreamEndCapture(cap, &captured);
  s->stream = saved;
  if (!ok || e != cudaSuccess) {
    const cudaError_t le = cudaGetLastError();
    return fail(-2, "building the dataset graph failed (%s)",
                cudaGetErrorString(e != cudaSuccess ? e : le));
  }
  return 0;
}

// Prepares a solver for append_solve_f32: unit loads (six per structure) in d_epsbar, the
// criterion history, the FP64 buffers of the mixed-precision continuation, and the pass
// configuration (autotuned on the fields at d_lambda / d_mu, the first structures').
int prepare_graph_solve(lsb_solver* s, int batch, const float* d_lambda, const float* d_mu, int maxiter) {
  const int nstruct = structures_of(s, batch);
  if (nstruct < 0) return nstruct;
  LSB_TRY(ensure_history(s, maxiter + 8));
  if (s->precision != kPrecFP32) LSB_TRY(ensure_fp64(s, nstruct));
  std::vector<double> eb(6 * (size_t)batch, 0.0);
  for (int b = 0; b < batch; ++b) eb[6 * b + b % 6] = 1.0;
  LSB_CUDA(cudaMemcpy(s->d_epsbar, eb.data(), sizeof(double) * eb.size(), cudaMemcpyHostToDevice));
  if (!s->xtuned) LSB_TRY(tune_passes(s, batch, d_lambda, d_mu, s->d_eps32, nstruct));
  LSB_CUDA(cudaStreamSynchronize(s->stream));
  return 0;
}

}  // namespace detail
}  // namespace lsb

namespace {

// Full solve with FP64 inputs/outputs (FP64 fields throughout).
int solve_f64(lsb_solver* s, int batch, const double* d_lambda, const double* d_mu,
              const double* eps_bar, const double* d_eps0, double* d_eps, double* d_sigma,
              double* mean_sigma, double rtol, double atol, int maxiter, int rule, int* iters,
              int* status, double* residual) {
  if (!s) return fail(-1, "null solver");
  if (batch < 1 || batch > s->batch_cap) return fail(-1, "batch %d outside [1, %d]", batch, s->batch_cap);
  if (!d_lambda || !d_mu || !eps_bar || !iters || !status || !d_eps) return fail(-1, "null argument");
  if (maxiter < 0) return fail(-1, "maxiter must be >= 0");
  const GridDesc& g = s->g;
  cudaStream_t st = s->stream;
  const int nstruct = structures_of(s, batch);
  if (nstruct < 0) return nstruct;
  LSB_TRY(prepare_damage(s, nstruct));
  LSB_TRY(prepare_aniso(s, nstruct));
  LSB_TRY(ensure_history(s, maxiter + 8));
  LSB_TRY(ensure_fp64(s, 0));
  const SolveParams sp = make_params(s, rtol, atol, maxiter, rule);
  LSB_CUDA(cudaMemcpyAsync(s->d_epsbar, eps_bar, sizeof(double) * 6 * batch, cudaMemcpyHostToDevice, st));
  LSB_CUDA(cudaMemsetAsync(s->d_history, 0, sizeof(double) * (size_t)batch * s->history_len, st));
  launch_reset_state(batch, 1, s->d_state, st, s->use_e0ref ? s->d_e0ref : nullptr);
  launch_medium<double>(g.nv, nstruct, d_lambda, d_mu, s->d_scratch, s->d_medium, st);
  s->launches += 3;
  LSB_TRY(ensure_fp64_rings(s));
  const bool hist = s->warm_history && d_eps0 && s->depth > 0;
  LSB_TRY(run_phase<double>(s, batch, d_lambda, d_mu, d_eps, s->d_spec64, hist ? nullptr : d_eps0,
                            0, sp, true, hist ? d_eps0 : nullptr));
  launch_stress<double, double>(g, 1, batch, s->d_state, d_lambda, d_mu, d_eps, d_sigma,
                                s->d_mean_scratch, s->d_mean, st);
  s->launches += 2;
  LSB_CUDA(take_launch_error(s));
  if (mean_sigma)
    LSB_CUDA(cudaMemcpyAsync(mean_sigma, s->d_mean, sizeof(double) * 6 * batch, cudaMemcpyDeviceToHost, st));
  LSB_CUDA(cudaMemcpyAsync(s->h_state, s->d_state, sizeof(InstanceState) * batch, cudaMemcpyDeviceToHost, st));
  LSB_CUDA(cudaStreamSynchronize(st));
  for (int b = 0; b < batch; ++b) {
    iters[b] = s->h_state[b].iter;
    status[b] = s->h_state[b].status;
    if (residual) residual[b] = s->h_state[b].e;
  }
  s->last_batch = batch;
  return 0;
}

// Cache for the reference-signature entry point: one solver per (grid, device).
struct AbiCache {
  std::mutex mu;
  lsb_solver* solver = nullptr;
  int voxels[3] = {0, 0, 0};
  double extents[3] = {0, 0, 0};
  float* d_lame = nullptr;   // [2][nv]
  float* d_fields = nullptr; // [2][6][nv] eps, sigma
  size_t nv = 0;
  void release() {
    if (solver) delete solver;
    solver = nullptr;
    cudaFree(d_lame);
    cudaFree(d_fields);
    d_lame = d_fields = nullptr;
    nv = 0;
  }
};

AbiCache& abi_cache() {
  static AbiCache c;
  return c;
}

}  // namespace

extern "C" {

int lsb_version(void) { return 2; }

const char* lsb_last_error(void) { return g_last_error.c_str(); }

int lsb_create(lsb_solver** out, const int voxels[3], const double extents[3], int batch, int depth) {
  g_last_error.clear();
  return create_impl(out, voxels, extents, batch, depth);
}

void lsb_destroy(lsb_solver* solver) { delete solver; }

int lsb_set_stream(lsb_solver* solver, void* stream) {
  if (!solver) return fail(-1, "null solver");
  solver->stream = (cudaStream_t)stream;
  return 0;
}

int lsb_set_reference_e0(lsb_solver* solver, int batch, const double* e0) {
  if (!solver) return fail(-1, "null solver");
  if (!e0) {
    solver->use_e0ref = false;
    return 0;
  }
  if (batch < 1 || batch > solver->batch_cap) return fail(-1, "batch %d outside [1, %d]", batch, solver->batch_cap);
  for (int b = 0; b < batch; ++b)
    if (!(e0[b] > 0.0) || !std::isfinite(e0[b])) return fail(-1, "e0[%d] must be positive and finite", b);
  if (!solver->d_e0ref) LSB_CUDA(cudaMalloc(&solver->d_e0ref, sizeof(double) * solver->batch_cap));
  LSB_CUDA(cudaMemcpy(solver->d_e0ref, e0, sizeof(double) * batch, cudaMemcpyHostToDevice));
  solver->use_e0ref = true;
  return 0;
}

int lsb_tile_variant(lsb_solver* solver, int variant) {
  if (!solver) return fail(-1, "null solver");
  if (variant < -1 || variant > 1) return fail(-1, "tile variant %d outside [-1, 1]", variant);
  if (variant >= 0) {
    if (!solver->fast32) return solver->xvariant;
    solver->xvariant = variant;
    solver->xtuned = true;
    if (!solver->tiled)
      solver->sh32.x_blocks_per_instance = fast::x_tiles(solver->g, variant) * solver->g.ny;
  }
  return solver->xvariant;
}

int lsb_y_variant(lsb_solver* solver, int variant) {
  if (!solver) return fail(-1, "null solver");
  if (variant < -1 || variant > 1) return fail(-1, "y-pass variant %d outside [-1, 1]", variant);
  if (variant >= 0 && solver->fast32) {
    solver->yvariant = variant;
    solver->xtuned = true;  // the caller's choice: no autotuning
  }
  return solver->yvariant;
}

int lsb_pass_config(lsb_solver* solver, int* out) {
  if (!solver || !out) return fail(-1, "null argument");
  out[0] = solver->tiled ? 1 : 0;
  out[1] = solver->xvariant;
  out[2] = solver->slab ? 1 : 0;
  out[3] = solver->xtuned ? 1 : 0;
  return 0;
}

int lsb_set_slab(lsb_solver* solver, int on) {
  if (!solver) return fail(-1, "null solver");
  solver->xtuned = true;  // the caller's choice: no autotuning
  solver->slab_allowed = on != 0;
  solver->slab = solver->slab_allowed && solver->tiled && fast::slab_supported(solver->g);
  return solver->slab ? 1 : 0;
}

int lsb_set_tiled(lsb_solver* solver, int on) {
  if (!solver) return fail(-1, "null solver");
  lsb_solver* s = solver;
  s->xtuned = true;  // the caller's choice: no autotuning
  const bool want = on != 0 && s->fast32 && fast::tiled_supported(s->g);
  if (want && !s->d_tspec32) {
    if (!s->owns_memory) return fail(-1, "this solver cannot allocate the tiled spectrum");
    LSB_CUDA(cudaMalloc(&s->d_tspec32, sizeof(float2) * (size_t)s->batch_cap * 6 * s->g.nm));
  }
  s->tiled = want;
  s->slab = s->tiled && s->slab_allowed && fast::slab_supported(s->g);
  if (s->tiled) s->sh32.x_blocks_per_instance = fast::x_tiles_tiled(s->g);
  else if (s->fast32) s->sh32.x_blocks_per_instance = fast::x_tiles(s->g, s->xvariant) * s->g.ny;
  return s->tiled ? 1 : 0;
}

int lsb_set_warm_history(lsb_solver* solver, int on) {
  if (!solver) return fail(-1, "null solver");
  if (on && solver->depth == 0) return fail(-1, "a warm start in the Anderson history needs depth >= 1");
  solver->warm_history = on != 0;
  return 0;
}

int lsb_set_device_loop(lsb_solver* solver, int on) {
  if (!solver) return fail(-1, "null solver");
  solver->use_loop = on != 0;
  return 0;
}

int lsb_set_graphs(lsb_solver* solver, int on) {
  if (!solver) return fail(-1, "null solver");
  solver->use_graphs = on != 0;
  return 0;
}

int lsb_set_lame_group(lsb_solver* solver, int instances_per_field) {
  if (!solver) return fail(-1, "null solver");
  if (instances_per_field < 0) return fail(-1, "instances_per_field must be >= 0");
  solver->lame_group = instances_per_field;
  return 0;
}

int lsb_set_precision(lsb_solver* solver, int precision, int stall_window) {
  if (!solver) return fail(-1, "null solver");
  if (precision < LSB_PREC_FP32 || precision > LSB_PREC_FP64) return fail(-1, "unknown precision %d", precision);
  if (stall_window < 0) return fail(-1, "stall_window must be >= 0");
  solver->precision = precision;
  solver->stall_window = stall_window;
  return 0;
}

int lsb_solve(lsb_solver* solver, int batch, const float* d_lambda, const float* d_mu,
              const float* eps_bar, const float* d_eps0, float* d_eps, float* d_sigma,
              double* mean_sigma, float rtol, float atol, int maxiter, int rule, int* iters,
              int* status, double* residual) {
  g_last_error.clear();
  if (!eps_bar) return fail(-1, "null argument");
  if (batch < 1 || (solver && batch > solver->batch_cap)) return fail(-1, "batch %d out of range", batch);
  std::vector<double> eb(eps_bar, eps_bar + 6 * batch);
  return solve_f32(solver, batch, d_lambda, d_mu, eb.data(), d_eps0, d_eps, d_sigma, mean_sigma,
                   rtol, atol, maxiter, rule, iters, status, residual);
}

int lsb_solve_f64(lsb_solver* solver, int batch, const double* d_lambda, const double* d_mu,
                  const double* eps_bar, const double* d_eps0, double* d_eps, double* d_sigma,
                  double* mean_sigma, double rtol, double atol, int maxiter, int rule, int* iters,
                  int* status, double* residual) {
  g_last_error.clear();
  return solve_f64(solver, batch, d_lambda, d_mu, eps_bar, d_eps0, d_eps, d_sigma, mean_sigma,
                   rtol, atol, maxiter, rule, iters, status, residual);
}

int lsb_set_damage(lsb_solver* solver, const void* d_damage, int elem_size, double k) {
  g_last_error.clear();
  if (!solver) return fail(-1, "null solver");
  if (d_damage && elem_size != 4 && elem_size != 8) return fail(-1, "elem_size must be 4 or 8");
  if (!std::isfinite(k)) return fail(-1, "k must be finite");
  solver->dmg_user = d_damage;
  solver->dmg_elem = d_damage ? elem_size : 4;
  solver->dmg_k = k;
  return 0;
}

long long lsb_kernel_launches(lsb_solver* solver) { return solver ? solver->launches : -1; }

int lsb_fp64_iters(lsb_solver* solver, int* out) {
  if (!solver || !out) return fail(-1, "null argument");
  for (int b = 0; b < solver->last_batch; ++b) {
    const InstanceState& st = solver->h_state[b];
    out[b] = st.switched ? st.iter - st.switch_iter : (st.phase == 1 ? st.iter : 0);
  }
  return 0;
}

int lsb_profile_step(lsb_solver* s, int batch, const float* d_lambda, const float* d_mu,
                     float* d_eps, int reps, float* ms_out, int max_kernels, char* names,
                     int names_len) {
  g_last_error.clear();
  if (!s || !d_lambda || !d_mu || !d_eps || !ms_out || !names) return fail(-1, "null argument");
  if (batch < 1 || batch > s->batch_cap) return fail(-1, "batch %d outside [1, %d]", batch, s->batch_cap);
  if (reps < 1 || max_kernels < 1 || names_len < 1) return fail(-1, "reps, max_kernels and names_len must be >= 1");
  const GridDesc& g = s->g;
  LaunchShape sh = s->sh32;
  if (!use_fast32(s)) sh.x_blocks_per_instance = s->x_blocks_generic32;
  cudaStream_t st = s->stream;
  // tolerances 0 and no stall detection: every pass does its full work
  SolveParams sp = make_params(s, 0.0, 0.0, 0x3fffffff, LSB_RULE_CUDA);
  sp.precision = kPrecFP32;
  sp.stall_window = 0;
  std::vector<double> eb(6 * batch, 0.0);
  for (int b = 0; b < batch; ++b) eb[6 * b + (b % 6)] = 1.0;
  LSB_CUDA(cudaMemcpyAsync(s->d_epsbar, eb.data(), sizeof(double) * eb.size(), cudaMemcpyHostToDevice, st));
  const int nstruct = structures_of(s, batch);
  if (nstruct < 0) return nstruct;
  LSB_TRY(prepare_damage(s, nstruct));
  LSB_TRY(prepare_aniso(s, nstruct));
  if (!s->xtuned) LSB_TRY(tune_passes(s, batch, d_lambda, d_mu, d_eps, nstruct));
  sh = s->sh32;  // (the tuned configuration's x-pass blocks)
  if (!use_fast32(s)) sh.x_blocks_per_instance = s->x_blocks_generic32;
  launch_reset_state(batch, 0, s->d_state, st);
  launch_medium<float>(g.nv, nstruct, d_lambda, d_mu, s->d_scratch, s->d_medium, st);
  const AndersonArgs<float> aa = anderson_args<float>(s, s->depth > 0);
  if (use_slab(s)) {
    pass_slab<float>(s, 0, batch, d_lambda, d_mu, d_eps, nullptr, aa);
  } else {
    pass_z<float>(s, 0, batch, d_lambda, d_mu, d_eps, s->d_spec32, nullptr, aa);
    pass_y<float>(s, false, batch, s->d_spec32);
  }
  // warm-up iterations: the Anderson rings fill up, so that the timed ones do full work
  for (int i = 0; i < s->depth + 2; ++i)
    enqueue_iteration<float>(s, batch, d_lambda, d_mu, d_eps, s->d_spec32, aa, sp, sh, 0, nullptr, nullptr);
  StepTimer tm{st};
  tm.ev.resize((size_t)max_kernels + 1);
  for (auto& e : tm.ev) LSB_CUDA(cudaEventCreate(&e));
  std::vector<double> acc(max_kernels, 0.0);
  size_t count = 0;
  for (int r = 0; r < reps; ++r) {
    tm.next = 1;
    cudaEventRecord(tm.ev[0], st);
    enqueue_iteration<float>(s, batch, d_lambda, d_mu, d_eps, s->d_spec32, aa, sp, sh, 0, nullptr, &tm);
    count = std::min(tm.next - 1, (size_t)max_kernels);
    LSB_CUDA(cudaEventSynchronize(tm.ev[count]));
    for (size_t k = 0; k < count; ++k) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, tm.ev[k], tm.ev[k + 1]);
      acc[k] += ms;
    }
  }
  for (auto& e : tm.ev) cudaEventDestroy(e);
  LSB_CUDA(take_launch_error(s));
  std::string joined;
  for (size_t k = 0; k < count; ++k) {
    ms_out[k] = (float)(acc[k] / reps);
    if (k) joined += ",";
    joined += tm.names[k];
  }
  std::snprintf(names, (size_t)names_len, "%s", joined.c_str());
  return (int)count;
}

int lsb_history(lsb_solver* solver, double* out, int len) {
  if (!solver || !out) return fail(-1, "null argument");
  if (len > solver->history_len) return fail(-1, "len %d > stored %d", len, solver->history_len);
  for (int b = 0; b < solver->last_batch; ++b)
    LSB_CUDA(cudaMemcpy(out + (size_t)b * len, solver->d_history + (size_t)b * solver->history_len,
                        sizeof(double) * len, cudaMemcpyDeviceToHost));
  return 0;
}

int lsb_c_eff(const float* lambda, const float* mu, const int voxels[3], const double extents[3],
              float rtol, float atol, int maxiter, int depth, double* c_eff, int* iters) {
  g_last_error.clear();
  if (!lambda || !mu || !c_eff || !iters) return fail(-1, "null argument");
  lsb_solver* s = nullptr;
  int rc = create_impl(&s, voxels, extents, 6, depth);
  if (rc) return rc;
  const size_t nv = (size_t)s->g.nv;
  float *d_l = nullptr, *d_m = nullptr;
  auto cleanup = [&]() {
    cudaFree(d_l);
    cudaFree(d_m);
    delete s;
  };
  if (cudaMalloc(&d_l, sizeof(float) * nv) != cudaSuccess || cudaMalloc(&d_m, sizeof(float) * nv) != cudaSuccess) {
    cleanup();
    return fail(-3, "cudaMalloc failed");
  }
  cudaMemcpy(d_l, lambda, sizeof(float) * nv, cudaMemcpyHostToDevice);
  cudaMemcpy(d_m, mu, sizeof(float) * nv, cudaMemcpyHostToDevice);
  double eb[36] = {0};
  for (int k = 0; k < 6; ++k) eb[6 * k + k] = 1.0;
  int status[6];
  rc = solve_f32(s, 6, d_l, d_m, eb, nullptr, s->d_eps32, nullptr, c_eff, rtol, atol, maxiter,
                 LSB_RULE_CUDA, iters, status, nullptr);
  cleanup();
  return rc;
}

void lippmann_schwinger_release(void) {
  AbiCache& c = abi_cache();
  std::lock_guard<std::mutex> lock(c.mu);
  c.release();
}

int lippmann_schwinger_solve(float* lambda, float* mu, float* epsilon_bar, float* epsilon,
                             float* sigma, int* voxels, float* extents, float rtol, float atol,
                             int maxiter, int verbose) {
  g_last_error.clear();
  if (!lambda || !mu || !epsilon_bar || !epsilon || !sigma || !voxels || !extents)
    return fail(-1, "null argument");
  AbiCache& c = abi_cache();
  std::lock_guard<std::mutex> lock(c.mu);
  int dev = 0;
  cudaGetDevice(&dev);
  const double ext[3] = {extents[0], extents[1], extents[2]};
  bool same = c.solver && c.solver->device == dev &&
              std::memcmp(c.voxels, voxels, sizeof(c.voxels)) == 0 &&
              std::memcmp(c.extents, ext, sizeof(c.extents)) == 0;
  if (!same) {
    c.release();
    int rc = create_impl(&c.solver, voxels, ext, 1, 0);
    if (rc) return rc;
    std::memcpy(c.voxels, voxels, sizeof(c.voxels));
    std::memcpy(c.extents, ext, sizeof(c.extents));
    c.nv = (size_t)c.solver->g.nv;
    if (cudaMalloc(&c.d_lame, sizeof(float) * 2 * c.nv) != cudaSuccess ||
        cudaMalloc(&c.d_fields, sizeof(float) * 12 * c.nv) != cudaSuccess) {
      c.release();
      return fail(-3, "cudaMalloc failed");
    }
  }
  const size_t nv = c.nv;
  cudaStream_t st = c.solver->stream;
  LSB_CUDA(cudaMemcpyAsync(c.d_lame, lambda, sizeof(float) * nv, cudaMemcpyHostToDevice, st));
  LSB_CUDA(cudaMemcpyAsync(c.d_lame + nv, mu, sizeof(float) * nv, cudaMemcpyHostToDevice, st));
  int it = 0, status = 0;
  double e = 0.0;
  double eb[6];
  for (int k = 0; k < 6; ++k) eb[k] = epsilon_bar[k];
  int rc = solve_f32(c.solver, 1, c.d_lame, c.d_lame + nv, eb, nullptr, c.d_fields,
                     c.d_fields + 6 * nv, nullptr, rtol, atol, maxiter, LSB_RULE_CUDA, &it,
                     &status, &e);
  if (rc) return rc;
  LSB_CUDA(cudaMemcpyAsync(epsilon, c.d_fields, sizeof(float) * 6 * nv, cudaMemcpyDeviceToHost, st));
  LSB_CUDA(cudaMemcpyAsync(sigma, c.d_fields + 6 * nv, sizeof(float) * 6 * nv, cudaMemcpyDeviceToHost, st));
  LSB_CUDA(cudaStreamSynchronize(st));
  if (verbose > 0) {
    std::vector<double> hist(c.solver->history_len);
    lsb_history(c.solver, hist.data(), c.solver->history_len);
    const double e0 = hist[0] != 0.0 ? hist[0] : 1.0;
    if (verbose > 1) {
      printf("==== Lippmann Schwinger solver ====\n");
      printf("  iteration           ||r||   ||r||/||r_0||\n");
      for (int i = 0; i < (int)hist.size() && (i == 0 || hist[i] != 0.0); ++i)
        printf("     %4d          %8.4e  %8.4e\n", i, hist[i], hist[i] / e0);
      printf("  ");
    } else {
      printf("  LS ");
    }
    printf("%s after %4d its, ||r|| = %6.3e ||r||/||r_0|| = %6.3e\n",
           status == LSB_CONVERGED ? "converged" : "failed to converge", it, e, e / e0);
  }
  return it;
}

}  // extern "C"
