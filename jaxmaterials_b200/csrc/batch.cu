// lsb_c_eff_batch: effective stiffness of many microstructures of uneven grid sizes, six
// unit load cases each -- the dataset loop of src/jaxmaterials/data/data.py:178-186 run
// as batched solves on one GPU.
//
// Schedule. Structures are grouped into buckets of equal grid (voxels and extents). Inside
// a bucket one solver holds `chunk` structures x 6 load cases; instance b reads the Lame
// fields of structure b / 6 and its own reference medium, and retires at its own
// convergence (kernels skip retired instances). The chunk is the largest that fits the
// bucket's share of the memory budget (share proportional to the bucket's voxels); the
// chunks of a bucket are evened out so that the last one is not a small remainder.
// Default: the whole dataset is ONE CUDA graph launch (run_dataset_graph): each bucket a
// chain of its chunks' solves, whose iteration loops are conditional WHILE nodes stopped on
// the device, the buckets independent branches with priorities by grid size; the host
// waits once. Fallback (and LSB_BATCH_GRAPH=0): each bucket on its own host thread and
// stream, one graph launch per chunk and phase.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lippmann_schwinger.h"
#include "ls_solver_impl.cuh"

using namespace lsb::detail;

namespace {

struct Bucket {
  int voxels[3];
  double extents[3];
  std::vector<int> members;  // structure indices in input order
  double voxels_total = 0.0;
};

// Device bytes one structure (6 instances) needs in a solver of the given configuration:
// fields, spectra and Anderson rings, the criterion history (maxiter + 8 values per
// instance), and upper bounds of the x-pass and Gram-row partials (one value per (ky, kz)
// column and per (x, y) line and slot).
size_t bytes_per_structure(const int v[3], int depth, int precision, int maxiter) {
  const size_t nv = (size_t)v[0] * v[1] * v[2];
  const size_t nm = (size_t)v[0] * v[1] * (v[2] / 2 + 1);
  const size_t partials = 8 * ((size_t)v[1] * (v[2] / 2 + 1) +
                               (depth > 0 ? (size_t)v[0] * v[1] * (depth + 2) : 0));
  const size_t history = 8 * ((size_t)maxiter + 8);
  // rings: g in FP32 and r in FP16, m+1 slots of 6 nv each
  const size_t inst32 = 24 * nv + 48 * nm + (depth > 0 ? (size_t)(depth + 1) * 36 * nv : 0) +
                        6 * 1024 * 8 + partials + history;
  size_t inst64 = 0;
  if (precision != LSB_PREC_FP32) {
    inst64 = 48 * nv + 96 * nm;
    if (precision == LSB_PREC_FP64 && depth > 0) inst64 += 2 * (size_t)(depth + 1) * 48 * nv;
  }
  const size_t lame = 8 * nv + (precision != LSB_PREC_FP32 ? 16 * nv : 0);
  return 6 * (inst32 + inst64) + lame;
}

struct BucketResult {
  int rc = 0;
  std::string error;
};

void run_bucket(const Bucket& bk, int device, size_t budget, int depth, int precision,
                double rtol, double atol, int maxiter, const float* const* lambda,
                const float* const* mu, double* c_eff, int* iters, int* status, int priority,
                BucketResult* out) {
  auto fail_here = [&](int rc) {
    out->rc = rc;
    out->error = lsb_last_error();
  };
  cudaSetDevice(device);
  const long long nv = (long long)bk.voxels[0] * bk.voxels[1] * bk.voxels[2];
  const int n = (int)bk.members.size();
  const size_t per = bytes_per_structure(bk.voxels, depth, precision, maxiter);
  int chunk = (int)std::max<size_t>(1, std::min<size_t>(budget / per, (size_t)n));
  const int nchunks = (n + chunk - 1) / chunk;
  chunk = (n + nchunks - 1) / nchunks;

  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, priority) != cudaSuccess) {
    out->rc = -2;
    out->error = "cudaStreamCreate failed";
    return;
  }
  lsb_solver* s = nullptr;
  float* d_lame = nullptr;
  int rc = lsb_create(&s, bk.voxels, bk.extents, 6 * chunk, depth);
  if (rc) {
    fail_here(rc);
    cudaStreamDestroy(st);
    return;
  }
  s->stream = st;
  s->precision = precision;
  s->lame_group = 6;
  if (cudaMalloc(&d_lame, sizeof(float) * 2 * (size_t)chunk * nv) != cudaSuccess) {
    out->rc = -3;
    out->error = "cudaMalloc of the Lame fields of one chunk failed";
  }
  std::vector<double> eb(36 * (size_t)chunk, 0.0), mean(36 * (size_t)chunk);
  for (int j = 0; j < chunk; ++j)
    for (int k = 0; k < 6; ++k) eb[36 * j + 7 * k] = 1.0;
  std::vector<int> it(6 * chunk), stt(6 * chunk);
  // LSB_BATCH_TRACE: one line per bucket on stderr (grid, structures, chunking, time, FP64
  // continuations)
  const bool trace = std::getenv("LSB_BATCH_TRACE") != nullptr;
  const auto t_start = std::chrono::steady_clock::now();
  long long switched = 0, updates = 0;
  for (int c0 = 0; c0 < n && out->rc == 0; c0 += chunk) {
    const int c = std::min(chunk, n - c0);
    for (int j = 0; j < c; ++j) {
      const int m = bk.members[c0 + j];
      cudaMemcpyAsync(d_lame + (size_t)j * nv, lambda[m], sizeof(float) * nv,
                      cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(d_lame + (size_t)(c + j) * nv, mu[m], sizeof(float) * nv,
                      cudaMemcpyHostToDevice, st);
    }
    rc = solve_f32(s, 6 * c, d_lame, d_lame + (size_t)c * nv, eb.data(), nullptr, s->d_eps32,
                   nullptr, mean.data(), rtol, atol, maxiter, LSB_RULE_CUDA, it.data(),
                   stt.data(), nullptr);
    if (rc) {
      fail_here(rc);
      break;
    }
    if (trace)
      for (int k = 0; k < 6 * c; ++k) {
        switched += s->h_state[k].switched;
        updates += s->h_state[k].iter;
      }
    for (int j = 0; j < c; ++j) {
      const int m = bk.members[c0 + j];
      std::memcpy(c_eff + 36 * (size_t)m, mean.data() + 36 * (size_t)j, sizeof(double) * 36);
      std::memcpy(iters + 6 * (size_t)m, it.data() + 6 * (size_t)j, sizeof(int) * 6);
      std::memcpy(status + 6 * (size_t)m, stt.data() + 6 * (size_t)j, sizeof(int) * 6);
    }
  }
  if (trace) {
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    std::fprintf(stderr, "lsb_c_eff_batch: grid %dx%dx%d structures %d chunk %d (%d chunks) %.3f s, "
                 "%lld updates, %lld instances continued in FP64\n", bk.voxels[0], bk.voxels[1],
                 bk.voxels[2], n, chunk, nchunks, sec, updates, switched);
  }
  cudaFree(d_lame);
  lsb_destroy(s);
  cudaStreamDestroy(st);
}

// ---- one graph for the whole dataset
//
// Every bucket gets its solver at once (chunk sized to the bucket's share of the budget,
// as above) and its structures' Lame fields are copied to the device up front; the solves
// of all chunks are then appended to ONE CUDA graph -- each bucket a chain of its chunks'
// solves (append_solve_f32: device-opened and device-stopped WHILE loops over the
// iterations, FP32 then the FP64 continuation), the buckets independent branches whose
// kernel nodes carry the bucket's priority (smallest grid highest) -- which is
// instantiated and launched once. The host waits once, for the whole dataset. Returns
// kNoGraph (and leaves nothing behind) when this schedule does not apply: a bucket whose
// share cannot hold one structure, the Lame fields above a third of the budget, or a graph
// call that failed; the caller then runs the threaded schedule.
constexpr int kNoGraph = 1;

struct GraphBucket {
  lsb_solver* s = nullptr;
  cudaStream_t st = nullptr;
  float* d_lame = nullptr;  // [2][members][nv]: lambda of every member, then mu
  int chunk = 0;
  double* h_mean = nullptr;          // [6 members][6] in the pinned result buffer
  InstanceState* h_state = nullptr;  // [6 members]
};

void set_priority(cudaGraph_t g, int prio) {
  size_t n = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) return;
  std::vector<cudaGraphNode_t> nodes(n);
  if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return;
  cudaLaunchAttributeValue v = {};
  v.priority = prio;
  for (cudaGraphNode_t nd : nodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
      cudaGraphKernelNodeSetAttribute(nd, cudaLaunchAttributePriority, &v);
  }
}

int run_dataset_graph(const std::vector<Bucket>& buckets, int device, size_t budget, int depth,
                      int precision, double rtol, double atol, int maxiter,
                      const float* const* lambda, const float* const* mu,
                      const std::vector<int>& priority, double* c_eff, int* iters, int* status,
                      bool trace) {
  double total = 0.0, lame_bytes = 0.0;
  for (const Bucket& b : buckets) {
    total += b.voxels_total;
    lame_bytes += 8.0 * b.voxels_total;
  }
  if (lame_bytes > (double)budget / 3.0) return kNoGraph;
  const size_t rest = budget - (size_t)lame_bytes;
  std::vector<GraphBucket> gb(buckets.size());
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cap = nullptr, body = nullptr, run = nullptr;
  unsigned char* h_res = nullptr;  // pinned: every structure's means and states
  int rc = 0;
  std::vector<std::pair<const char*, double>> times;  // (step, seconds) for the trace
  auto tick = [&](const char* what) {
    static thread_local auto last = std::chrono::steady_clock::now();
    const auto now = std::chrono::steady_clock::now();
    if (what) times.emplace_back(what, std::chrono::duration<double>(now - last).count());
    last = now;
  };
  tick(nullptr);
  auto cleanup = [&]() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    tick("graph release");
    for (GraphBucket& b : gb) {
      cudaFree(b.d_lame);
      if (b.s) lsb_destroy(b.s);
      if (b.st) cudaStreamDestroy(b.st);
    }
    tick("solvers release");
    if (h_res) cudaFreeHost(h_res);
    if (cap) cudaStreamDestroy(cap);
    if (body) cudaStreamDestroy(body);
    if (run) cudaStreamDestroy(run);
    cudaGetLastError();
  };
  size_t nmembers = 0;
  for (const Bucket& b : buckets) nmembers += b.members.size();
  if (cudaMallocHost(&h_res, (sizeof(double) * 36 + sizeof(InstanceState) * 6) * nmembers) != cudaSuccess) {
    cudaGetLastError();
    return kNoGraph;
  }
  {
    size_t off = 0;
    for (size_t k = 0; k < buckets.size(); ++k) {
      gb[k].h_mean = reinterpret_cast<double*>(h_res) + 36 * off;
      off += buckets[k].members.size();
    }
    off = 0;
    InstanceState* hs = reinterpret_cast<InstanceState*>(h_res + sizeof(double) * 36 * nmembers);
    for (size_t k = 0; k < buckets.size(); ++k) {
      gb[k].h_state = hs + 6 * off;
      off += buckets[k].members.size();
    }
  }
  // solvers, Lame fields on the device and tuned passes, one host thread per bucket (the
  // buckets' uploads from pageable memory and allocations proceed in parallel)
  for (size_t k = 0; k < buckets.size(); ++k) {
    const Bucket& bk = buckets[k];
    const size_t per = bytes_per_structure(bk.voxels, depth, precision, maxiter);
    const size_t share = (size_t)((double)rest * bk.voxels_total / total);
    if (share < per) {
      cleanup();
      return kNoGraph;
    }
    const int n = (int)bk.members.size();
    const int chunk = (int)std::min<size_t>(share / per, (size_t)n);
    const int nchunks = (n + chunk - 1) / chunk;
    gb[k].chunk = (n + nchunks - 1) / nchunks;
  }
  std::vector<int> setup_rc(buckets.size(), 0);
  std::vector<std::string> setup_err(buckets.size());
  auto set_up = [&](size_t k) {
    cudaSetDevice(device);
    const Bucket& bk = buckets[k];
    GraphBucket& b = gb[k];
    const long long nv = (long long)bk.voxels[0] * bk.voxels[1] * bk.voxels[2];
    const int n = (int)bk.members.size();
    if (cudaStreamCreateWithPriority(&b.st, cudaStreamNonBlocking, priority[k]) != cudaSuccess ||
        cudaMalloc(&b.d_lame, sizeof(float) * 2 * (size_t)n * nv) != cudaSuccess) {
      cudaGetLastError();
      setup_rc[k] = kNoGraph;
      return;
    }
    for (int j = 0; j < n; ++j) {
      const int m = bk.members[j];
      cudaMemcpyAsync(b.d_lame + (size_t)j * nv, lambda[m], sizeof(float) * nv, cudaMemcpyHostToDevice, b.st);
      cudaMemcpyAsync(b.d_lame + (size_t)(n + j) * nv, mu[m], sizeof(float) * nv, cudaMemcpyHostToDevice, b.st);
    }
    int r = lsb_create(&b.s, bk.voxels, bk.extents, 6 * b.chunk, depth);
    if (r == 0) {
      b.s->stream = b.st;
      b.s->precision = precision;
      b.s->lame_group = 6;
      r = prepare_graph_solve(b.s, 6 * b.chunk, b.d_lame, b.d_lame + (size_t)n * nv, maxiter);
    }
    if (r) {
      setup_rc[k] = r;
      setup_err[k] = lsb_last_error();
    }
  };
  {
    std::vector<std::thread> th;
    for (size_t k = 0; k < buckets.size(); ++k) th.emplace_back(set_up, k);
    for (auto& t : th) t.join();
  }
  for (size_t k = 0; k < buckets.size() && rc == 0; ++k)
    if (setup_rc[k]) {
      rc = setup_rc[k] == kNoGraph ? kNoGraph
                                   : fail(setup_rc[k], "bucket %dx%dx%d: %s", buckets[k].voxels[0],
                                          buckets[k].voxels[1], buckets[k].voxels[2], setup_err[k].c_str());
    }
  tick("solvers, fields, tuning");
  if (rc == 0 &&
      (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess ||
       cudaStreamCreateWithFlags(&body, cudaStreamNonBlocking) != cudaSuccess ||
       cudaStreamCreateWithFlags(&run, cudaStreamNonBlocking) != cudaSuccess || cudaGraphCreate(&graph, 0) != cudaSuccess))
    rc = kNoGraph;
  // one branch per bucket: its chunks' solves in sequence
  std::set<cudaGraphNode_t> seen;  // root nodes of the buckets already appended
  for (size_t k = 0; k < buckets.size() && rc == 0; ++k) {
    const Bucket& bk = buckets[k];
    GraphBucket& b = gb[k];
    const long long nv = (long long)bk.voxels[0] * bk.voxels[1] * bk.voxels[2];
    const int n = (int)bk.members.size();
    std::vector<cudaGraphNode_t> deps, last;
    std::vector<cudaGraph_t> bodies;
    for (int c0 = 0; c0 < n && rc == 0; c0 += b.chunk) {
      const int c = std::min(b.chunk, n - c0);
      rc = append_solve_f32(b.s, graph, deps, cap, body, 6 * c, b.d_lame + (size_t)c0 * nv,
                            b.d_lame + (size_t)(n + c0) * nv, rtol, atol, maxiter, b.h_mean + 36 * (size_t)c0,
                            b.h_state + 6 * (size_t)c0, &last, &bodies);
      deps = last;
    }
    if (rc) {
      // a graph that cannot be built leaves the dataset to the threaded schedule
      if (trace) std::fprintf(stderr, "lsb_c_eff_batch: graph build failed (%s)\n", lsb_last_error());
      rc = kNoGraph;
      break;
    }
    // this bucket's kernel nodes (the ones added since the previous bucket, and the loop
    // bodies) get its priority
    size_t n_now = 0;
    cudaGraphGetNodes(graph, nullptr, &n_now);
    std::vector<cudaGraphNode_t> all(n_now);
    cudaGraphGetNodes(graph, all.data(), &n_now);
    cudaLaunchAttributeValue v = {};
    v.priority = priority[k];
    for (size_t i = 0; i < n_now; ++i) {
      if (!seen.insert(all[i]).second) continue;
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(all[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
        cudaGraphKernelNodeSetAttribute(all[i], cudaLaunchAttributePriority, &v);
    }
    for (cudaGraph_t bg : bodies) set_priority(bg, priority[k]);
  }
  tick("graph build");
  if (rc == 0 && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) rc = kNoGraph;
  tick("instantiate");
  if (rc == 0) {
    cudaError_t e = cudaGraphLaunch(exec, run);
    if (e == cudaSuccess) e = cudaStreamSynchronize(run);
    if (e != cudaSuccess) rc = fail(-2, "dataset graph: %s", cudaGetErrorString(e));
  }
  tick("run");
  if (rc == 0) {
    for (size_t k = 0; k < buckets.size(); ++k) {
      const Bucket& bk = buckets[k];
      const GraphBucket& b = gb[k];
      for (size_t j = 0; j < bk.members.size(); ++j) {
        const int m = bk.members[j];
        std::memcpy(c_eff + 36 * (size_t)m, b.h_mean + 36 * j, sizeof(double) * 36);
        for (int q = 0; q < 6; ++q) {
          iters[6 * (size_t)m + q] = b.h_state[6 * j + q].iter;
          status[6 * (size_t)m + q] = b.h_state[6 * j + q].status;
        }
      }
    }
  }
  cleanup();
  tick("release");
  if (trace && rc == 0) {
    std::fprintf(stderr, "lsb_c_eff_batch: one graph over %zu buckets:", buckets.size());
    for (auto& t : times) std::fprintf(stderr, " %s %.3f s,", t.first, t.second);
    std::fprintf(stderr, "\n");
    for (size_t k = 0; k < buckets.size(); ++k)
      std::fprintf(stderr, "  grid %dx%dx%d structures %zu chunk %d priority %d\n", buckets[k].voxels[0],
                   buckets[k].voxels[1], buckets[k].voxels[2], buckets[k].members.size(), gb[k].chunk,
                   priority[k]);
  }
  return rc;
}

}  // namespace

extern "C" int lsb_c_eff_batch(int nstruct, const int* voxels, const double* extents,
                               const float* const* lambda, const float* const* mu, int depth,
                               int precision, float rtol, float atol, int maxiter,
                               double memory_gb, double* c_eff, int* iters, int* status) {
  if (nstruct < 0) return fail(-1, "nstruct must be >= 0");
  if (nstruct == 0) return 0;
  if (!voxels || !extents || !lambda || !mu || !c_eff || !iters || !status)
    return fail(-1, "null argument");
  if (depth < 0 || depth > kMaxDepth) return fail(-1, "Anderson depth %d outside [0, %d]", depth, kMaxDepth);
  if (precision < LSB_PREC_FP32 || precision > LSB_PREC_FP64) return fail(-1, "unknown precision %d", precision);
  if (maxiter < 0) return fail(-1, "maxiter must be >= 0");
  for (int i = 0; i < nstruct; ++i)
    if (!lambda[i] || !mu[i]) return fail(-1, "null Lame field of structure %d", i);

  // buckets of equal grid, in order of first appearance
  std::vector<Bucket> buckets;
  std::map<std::vector<double>, int> index;
  for (int i = 0; i < nstruct; ++i) {
    const int* v = voxels + 3 * i;
    const double* e = extents + 3 * i;
    std::vector<double> key = {(double)v[0], (double)v[1], (double)v[2], e[0], e[1], e[2]};
    auto f = index.find(key);
    int b;
    if (f == index.end()) {
      b = (int)buckets.size();
      index[key] = b;
      Bucket nb;
      std::memcpy(nb.voxels, v, sizeof(nb.voxels));
      std::memcpy(nb.extents, e, sizeof(nb.extents));
      buckets.push_back(nb);
    } else {
      b = f->second;
    }
    buckets[b].members.push_back(i);
    buckets[b].voxels_total += (double)v[0] * v[1] * v[2];
  }

  int device = 0;
  cudaGetDevice(&device);
  size_t budget;
  if (memory_gb > 0.0) {
    budget = (size_t)(memory_gb * 1e9);
  } else {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return fail(-2, "cudaMemGetInfo failed");
    budget = (size_t)(0.7 * (double)free_b);
  }
  double total = 0.0;
  for (const Bucket& b : buckets) total += b.voxels_total;

  // Stream priorities: the smaller a bucket's grid, the higher its priority, so that the
  // short kernels of small grids are not queued behind the blocks of the large ones (each
  // small-grid iteration is a chain of short dependent launches); the small buckets then
  // finish early and the large ones keep the GPU.
  int least = 0, greatest = 0;
  if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) {
    cudaGetLastError();
    least = greatest = 0;
  }
  std::vector<double> sizes;
  for (const Bucket& b : buckets) sizes.push_back((double)b.voxels[0] * b.voxels[1] * b.voxels[2]);
  std::vector<double> sorted_sizes = sizes;
  std::sort(sorted_sizes.begin(), sorted_sizes.end());
  sorted_sizes.erase(std::unique(sorted_sizes.begin(), sorted_sizes.end()), sorted_sizes.end());
  auto priority_of = [&](size_t b) {
    // rank 0 (smallest grid) -> greatest priority (numerically lowest), clamped to the range
    const int rank = (int)(std::lower_bound(sorted_sizes.begin(), sorted_sizes.end(), sizes[b]) -
                           sorted_sizes.begin());
    return std::min(least, greatest + rank);
  };
  // One graph for the whole dataset (LSB_BATCH_GRAPH=0: the threaded schedule below; FP64
  // solves, which start in FP64, also take the threaded schedule: the graph's solves start
  // in FP32).
  const char* gmode = std::getenv("LSB_BATCH_GRAPH");
  if (!(gmode && gmode[0] == '0' && gmode[1] == 0) && precision != LSB_PREC_FP64) {
    std::vector<int> prio(buckets.size());
    for (size_t b = 0; b < buckets.size(); ++b) prio[b] = priority_of(b);
    const int grc = run_dataset_graph(buckets, device, budget, depth, precision, (double)rtol, (double)atol,
                                      maxiter, lambda, mu, prio, c_eff, iters, status,
                                      std::getenv("LSB_BATCH_TRACE") != nullptr);
    if (grc != kNoGraph) return grc;
  }
  // Buckets whose share of the budget holds at least one structure run concurrently, one
  // host thread each; the others run afterwards one at a time with the whole budget.
  std::vector<BucketResult> res(buckets.size());
  std::vector<std::thread> threads;
  std::vector<size_t> serial;
  for (size_t b = 0; b < buckets.size(); ++b) {
    const size_t share = (size_t)((double)budget * buckets[b].voxels_total / total);
    if (share < bytes_per_structure(buckets[b].voxels, depth, precision, maxiter)) {
      serial.push_back(b);
      continue;
    }
    threads.emplace_back(run_bucket, std::cref(buckets[b]), device, share, depth, precision,
                         (double)rtol, (double)atol, maxiter, lambda, mu, c_eff, iters, status,
                         priority_of(b), &res[b]);
  }
  for (auto& t : threads) t.join();
  for (size_t b : serial)
    run_bucket(buckets[b], device, budget, depth, precision, (double)rtol, (double)atol, maxiter,
               lambda, mu, c_eff, iters, status, priority_of(b), &res[b]);
  for (size_t b = 0; b < buckets.size(); ++b)
    if (res[b].rc)
      return fail(res[b].rc, "bucket %dx%dx%d: %s", buckets[b].voxels[0], buckets[b].voxels[1],
                  buckets[b].voxels[2], res[b].error.c_str());
  return 0;
}
