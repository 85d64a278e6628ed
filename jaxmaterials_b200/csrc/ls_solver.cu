// Host side of liblippmannschwinger.so: plans, device buffers, the iteration driver and
// the C ABI declared in include/lippmann_schwinger.h.
//
// The iteration never waits on the host per step: kernels read the per-instance stop flag
// written by finalize_kernel, so the host enqueues iterations in growing chunks and reads
// the 64-byte states back once per chunk.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lippmann_schwinger.h"
#include "ls_kernels.cuh"

using namespace lsb;

namespace {

thread_local std::string g_last_error;

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

}  // namespace

struct lsb_solver {
  int device = 0;
  int batch_cap = 0;
  int depth = 0;
  GridDesc g{};
  LaunchShape shape{};
  cudaStream_t stream = nullptr;
  // device buffers
  float* d_eps = nullptr;          // [batch][6][nv] working strain (when caller gives none)
  float2* d_spec = nullptr;        // [batch][6][nm]
  double* d_partials = nullptr;    // [batch][x blocks]
  InstanceState* d_state = nullptr;
  Medium* d_medium = nullptr;
  float* d_epsbar = nullptr;       // [batch][6]
  float* d_mm_scratch = nullptr;   // min/max partials
  double* d_mean_scratch = nullptr;
  double* d_mean = nullptr;        // [batch][6]
  double* d_history = nullptr;     // [batch][history_len]
  int history_len = 0;
  int last_batch = 0;
  float2* d_tw = nullptr;
  double* d_tables = nullptr;
  InstanceState* h_state = nullptr;  // pinned
  long long launches = 0;            // kernels enqueued by this solver

  ~lsb_solver() {
    cudaFree(d_eps);
    cudaFree(d_spec);
    cudaFree(d_partials);
    cudaFree(d_state);
    cudaFree(d_medium);
    cudaFree(d_epsbar);
    cudaFree(d_mm_scratch);
    cudaFree(d_mean_scratch);
    cudaFree(d_mean);
    cudaFree(d_history);
    cudaFree(d_tw);
    cudaFree(d_tables);
    if (h_state) cudaFreeHost(h_state);
  }
};

namespace {

int ensure_history(lsb_solver* s, int len) {
  if (len <= s->history_len) return 0;
  cudaFree(s->d_history);
  s->d_history = nullptr;
  LSB_CUDA(cudaMalloc(&s->d_history, sizeof(double) * (size_t)s->batch_cap * len));
  s->history_len = len;
  return 0;
}

int create_impl(lsb_solver** out, const int voxels[3], const float extents[3], int batch, int depth) {
  if (!out || !voxels || !extents) return fail(-1, "null argument");
  *out = nullptr;
  for (int d = 0; d < 3; ++d) {
    if (voxels[d] < 1 || voxels[d] > kMaxDim)
      return fail(-1, "voxels[%d] = %d outside [1, %d]", d, voxels[d], kMaxDim);
    if (!(extents[d] > 0.f) || !std::isfinite(extents[d]))
      return fail(-1, "extents[%d] must be positive and finite", d);
  }
  if (batch < 1) return fail(-1, "batch must be >= 1");
  if (depth != 0) return fail(-1, "Anderson depth %d not supported by this build", depth);
  auto* s = new lsb_solver();
  s->batch_cap = batch;
  s->depth = depth;
  cudaGetDevice(&s->device);
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
  if (!factorize(g.nx, g.px) || !factorize(g.ny, g.py) || !factorize(g.nz, g.pz)) {
    delete s;
    return fail(-1, "grid extent has too many prime factors");
  }
  s->shape = plan_launch(g);
  const LaunchShape& sh = s->shape;
  if (sh.z_threads > kMaxThreads || sh.y_threads > kMaxThreads || sh.x_threads > kMaxThreads) {
    delete s;
    return fail(-1, "grid %dx%dx%d needs FFT blocks above %d threads", g.nx, g.ny, g.nz, kMaxThreads);
  }
  int rc = 0;
  auto alloc = [&](void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) rc = fail(-3, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    return e == cudaSuccess;
  };
  const size_t B = (size_t)batch;
  bool ok = alloc((void**)&s->d_eps, sizeof(float) * B * 6 * g.nv) &&
            alloc((void**)&s->d_spec, sizeof(float2) * B * 6 * g.nm) &&
            alloc((void**)&s->d_partials, sizeof(double) * B * sh.x_blocks_per_instance) &&
            alloc((void**)&s->d_state, sizeof(InstanceState) * B) &&
            alloc((void**)&s->d_medium, sizeof(Medium)) &&
            alloc((void**)&s->d_epsbar, sizeof(float) * B * 6) &&
            alloc((void**)&s->d_mm_scratch, sizeof(float) * 4 * 1024) &&
            alloc((void**)&s->d_mean_scratch, sizeof(double) * B * 6 * 1024) &&
            alloc((void**)&s->d_mean, sizeof(double) * B * 6) &&
            alloc((void**)&s->d_tw, sizeof(float2) * (size_t)(g.nx + g.ny + g.nz)) &&
            alloc((void**)&s->d_tables, sizeof(double) * 2 * (size_t)(g.nx + g.ny + g.nzh));
  if (!ok) {
    delete s;
    return rc;
  }
  if (cudaMallocHost(&s->h_state, sizeof(InstanceState) * B) != cudaSuccess) {
    delete s;
    return fail(-3, "cudaMallocHost failed");
  }
  // twiddles exp(-2 pi i k / n) and the sin/cos tables of the modified wave vectors,
  // both evaluated in FP64 (fourier.py:29-31: xi_d / 2 = pi k_d / N_d)
  std::vector<float2> tw;
  for (int n : {g.nx, g.ny, g.nz})
    for (int k = 0; k < n; ++k) {
      double a = -2.0 * M_PI * (double)k / (double)n;
      tw.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
    }
  std::vector<double> tab;
  auto add_tab = [&](int n, int count) {
    for (int k = 0; k < count; ++k) tab.push_back(std::sin((2.0 * M_PI * k / n) / 2.0));
    for (int k = 0; k < count; ++k) tab.push_back(std::cos((2.0 * M_PI * k / n) / 2.0));
  };
  add_tab(g.nx, g.nx);
  add_tab(g.ny, g.ny);
  add_tab(g.nz, g.nzh);
  if (cudaMemcpy(s->d_tw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(s->d_tables, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    delete s;
    return fail(-2, "upload of twiddle tables failed");
  }
  g.px.tw = s->d_tw;
  g.py.tw = s->d_tw + g.nx;
  g.pz.tw = s->d_tw + g.nx + g.ny;
  g.sx = s->d_tables;
  g.cx = g.sx + g.nx;
  g.sy = g.cx + g.nx;
  g.cy = g.sy + g.ny;
  g.sz = g.cy + g.ny;
  g.cz = g.sz + g.nzh;
  cudaError_t e = configure_kernels(sh);
  if (e != cudaSuccess) {
    delete s;
    return fail(-2, "kernel configuration: %s", cudaGetErrorString(e));
  }
  *out = s;
  return 0;
}

int solve_impl(lsb_solver* s, int batch, const float* d_lambda, const float* d_mu,
               const float* eps_bar, const float* d_eps0, float* d_eps, float* d_sigma,
               double* mean_sigma, float rtol, float atol, int maxiter, int rule, int* iters,
               int* status, double* residual) {
  if (!s) return fail(-1, "null solver");
  if (batch < 1 || batch > s->batch_cap) return fail(-1, "batch %d outside [1, %d]", batch, s->batch_cap);
  if (!d_lambda || !d_mu || !eps_bar || !iters || !status) return fail(-1, "null argument");
  if (maxiter < 0) return fail(-1, "maxiter must be >= 0");
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != s->device) return fail(-1, "solver was created on device %d, current is %d", s->device, cur);
  const GridDesc& g = s->g;
  const LaunchShape& sh = s->shape;
  cudaStream_t st = s->stream;
  float* eps = d_eps ? d_eps : s->d_eps;
  if (ensure_history(s, maxiter + 1)) return -3;
  SolveParams sp;
  sp.rtol = rtol;
  sp.atol = atol;
  sp.maxiter = maxiter;
  sp.rule = rule;
  sp.inv_nv = (float)(1.0 / (double)g.nv);

  LSB_CUDA(cudaMemcpyAsync(s->d_epsbar, eps_bar, sizeof(float) * 6 * batch, cudaMemcpyHostToDevice, st));
  LSB_CUDA(cudaMemsetAsync(s->d_history, 0, sizeof(double) * (size_t)batch * s->history_len, st));
  launch_reset_state(batch, s->d_state, st);
  launch_medium(g.nv, d_lambda, d_mu, s->d_mm_scratch, s->d_medium, st);
  launch_zpass(g, sh, 0, batch, d_lambda, d_mu, eps, s->d_spec, s->d_epsbar, d_eps0, s->d_state, sp, st);
  launch_ypass(g, sh, false, batch, s->d_spec, s->d_state, st);
  s->launches += 5;
  LSB_CUDA(cudaGetLastError());

  long long launched = 0;
  const long long max_evals = (long long)maxiter + 1;
  int chunk = 1;
  for (;;) {
    int n = (int)std::min<long long>(chunk, max_evals - launched);
    for (int i = 0; i < n; ++i) {
      launch_xpass(g, sh, batch, s->d_spec, s->d_medium, s->d_state, s->d_partials, st);
      launch_finalize(g, sh, batch, s->d_state, s->d_partials, s->d_history, s->history_len, sp, st);
      launch_ypass(g, sh, true, batch, s->d_spec, s->d_state, st);
      launch_zpass(g, sh, 1, batch, d_lambda, d_mu, eps, s->d_spec, s->d_epsbar, nullptr, s->d_state, sp, st);
      launch_ypass(g, sh, false, batch, s->d_spec, s->d_state, st);
    }
    launched += n;
    s->launches += 5LL * n;
    LSB_CUDA(cudaGetLastError());
    LSB_CUDA(cudaMemcpyAsync(s->h_state, s->d_state, sizeof(InstanceState) * batch, cudaMemcpyDeviceToHost, st));
    LSB_CUDA(cudaStreamSynchronize(st));
    bool all = true;
    for (int b = 0; b < batch; ++b) all = all && s->h_state[b].done;
    if (all) break;
    if (launched >= max_evals) return fail(-4, "internal: iteration driver did not terminate");
    chunk = std::min(chunk * 2, 32);
  }
  launch_stress(g, batch, d_lambda, d_mu, eps, d_sigma, s->d_mean_scratch, mean_sigma ? s->d_mean : nullptr, st);
  s->launches += mean_sigma ? 2 : 1;
  LSB_CUDA(cudaGetLastError());
  if (mean_sigma)
    LSB_CUDA(cudaMemcpyAsync(mean_sigma, s->d_mean, sizeof(double) * 6 * batch, cudaMemcpyDeviceToHost, st));
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
  float extents[3] = {0, 0, 0};
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

int lsb_version(void) { return 1; }

const char* lsb_last_error(void) { return g_last_error.c_str(); }

int lsb_create(lsb_solver** out, const int voxels[3], const float extents[3], int batch, int depth) {
  g_last_error.clear();
  return create_impl(out, voxels, extents, batch, depth);
}

void lsb_destroy(lsb_solver* solver) { delete solver; }

int lsb_set_stream(lsb_solver* solver, void* stream) {
  if (!solver) return fail(-1, "null solver");
  solver->stream = (cudaStream_t)stream;
  return 0;
}

int lsb_solve(lsb_solver* solver, int batch, const float* d_lambda, const float* d_mu,
              const float* eps_bar, const float* d_eps0, float* d_eps, float* d_sigma,
              double* mean_sigma, float rtol, float atol, int maxiter, int rule, int* iters,
              int* status, double* residual) {
  g_last_error.clear();
  if (!d_eps) return fail(-1, "d_eps must not be null");
  return solve_impl(solver, batch, d_lambda, d_mu, eps_bar, d_eps0, d_eps, d_sigma, mean_sigma,
                    rtol, atol, maxiter, rule, iters, status, residual);
}

long long lsb_kernel_launches(lsb_solver* solver) { return solver ? solver->launches : -1; }

int lsb_profile_passes(lsb_solver* s, int batch, const float* d_lambda, const float* d_mu,
                       float* d_eps, int reps, float* ms_out) {
  g_last_error.clear();
  if (!s || !d_lambda || !d_mu || !d_eps || !ms_out) return fail(-1, "null argument");
  if (batch < 1 || batch > s->batch_cap) return fail(-1, "batch %d outside [1, %d]", batch, s->batch_cap);
  if (reps < 1) return fail(-1, "reps must be >= 1");
  const GridDesc& g = s->g;
  const LaunchShape& sh = s->shape;
  cudaStream_t st = s->stream;
  SolveParams sp;
  sp.rtol = 0.f;
  sp.atol = 0.f;  // never converges: every pass does its full work
  sp.maxiter = 0x3fffffff;
  sp.rule = LSB_RULE_CUDA;
  sp.inv_nv = (float)(1.0 / (double)g.nv);
  std::vector<float> eb(6 * batch, 0.f);
  for (int b = 0; b < batch; ++b) eb[6 * b + (b % 6)] = 1.f;
  if (ensure_history(s, 1)) return -3;
  LSB_CUDA(cudaMemcpyAsync(s->d_epsbar, eb.data(), sizeof(float) * eb.size(), cudaMemcpyHostToDevice, st));
  launch_reset_state(batch, s->d_state, st);
  launch_medium(g.nv, d_lambda, d_mu, s->d_mm_scratch, s->d_medium, st);
  launch_zpass(g, sh, 0, batch, d_lambda, d_mu, d_eps, s->d_spec, s->d_epsbar, nullptr, s->d_state, sp, st);
  launch_ypass(g, sh, false, batch, s->d_spec, s->d_state, st);
  cudaEvent_t ev[6];
  for (auto& e : ev) LSB_CUDA(cudaEventCreate(&e));
  double acc[5] = {0, 0, 0, 0, 0};
  for (int r = 0; r < reps; ++r) {
    cudaEventRecord(ev[0], st);
    launch_xpass(g, sh, batch, s->d_spec, s->d_medium, s->d_state, s->d_partials, st);
    cudaEventRecord(ev[1], st);
    launch_finalize(g, sh, batch, s->d_state, s->d_partials, nullptr, 0, sp, st);
    cudaEventRecord(ev[2], st);
    launch_ypass(g, sh, true, batch, s->d_spec, s->d_state, st);
    cudaEventRecord(ev[3], st);
    launch_zpass(g, sh, 1, batch, d_lambda, d_mu, d_eps, s->d_spec, s->d_epsbar, nullptr, s->d_state, sp, st);
    cudaEventRecord(ev[4], st);
    launch_ypass(g, sh, false, batch, s->d_spec, s->d_state, st);
    cudaEventRecord(ev[5], st);
    LSB_CUDA(cudaEventSynchronize(ev[5]));
    for (int k = 0; k < 5; ++k) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
      acc[k] += ms;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  LSB_CUDA(cudaGetLastError());
  for (int k = 0; k < 5; ++k) ms_out[k] = (float)(acc[k] / reps);
  return 0;
}

int lsb_history(lsb_solver* solver, double* out, int len) {
  if (!solver || !out) return fail(-1, "null argument");
  if (len > solver->history_len) return fail(-1, "len %d > stored %d", len, solver->history_len);
  for (int b = 0; b < solver->last_batch; ++b)
    LSB_CUDA(cudaMemcpy(out + (size_t)b * len, solver->d_history + (size_t)b * solver->history_len,
                        sizeof(double) * len, cudaMemcpyDeviceToHost));
  return 0;
}

int lsb_c_eff(const float* lambda, const float* mu, const int voxels[3], const float extents[3],
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
  float eb[36] = {0};
  for (int k = 0; k < 6; ++k) eb[6 * k + k] = 1.f;
  int status[6];
  rc = solve_impl(s, 6, d_l, d_m, eb, nullptr, s->d_eps, nullptr, c_eff, rtol, atol, maxiter,
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
  bool same = c.solver && c.solver->device == dev &&
              std::memcmp(c.voxels, voxels, sizeof(c.voxels)) == 0 &&
              std::memcmp(c.extents, extents, sizeof(c.extents)) == 0;
  if (!same) {
    c.release();
    int rc = create_impl(&c.solver, voxels, extents, 1, 0);
    if (rc) return rc;
    std::memcpy(c.voxels, voxels, sizeof(c.voxels));
    std::memcpy(c.extents, extents, sizeof(c.extents));
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
  int rc = solve_impl(c.solver, 1, c.d_lame, c.d_lame + nv, epsilon_bar, nullptr, c.d_fields,
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
      for (int i = 0; i <= it && i < (int)hist.size(); ++i)
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
