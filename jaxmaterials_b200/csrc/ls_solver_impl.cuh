// Internal declarations shared by the host-side translation units of the library
// (the solver handle and the driver entry points).
#pragma once

#include <cstdarg>
#include <vector>

#include "fast_passes.cuh"
#include "ls_kernels.cuh"

using namespace lsb;  // internal header: only the library's own translation units include it

struct lsb_solver {
  // Device buffers, launch shapes and plans of one grid; see ls_solver.cu.
  int device = 0;
  int batch_cap = 0;
  int depth = 0;
  int precision = kPrecMixed;
  int stall_window = 8;
  // instances per (lambda, mu) field pair: 0 = every instance of a solve shares one pair;
  // k > 0 = instance b uses structure b / k of [structure][nv] Lame arrays
  int lame_group = 0;
  bool fast32 = false;   // FP32 passes with compile-time lengths (fast_passes.cu)
  // the fast passes keep the spectrum between the y and x passes in the tiled layout
  // (d_tspec32); tiled_allowed = false keeps the strided x pass (no second spectrum buffer)
  bool tiled = false;
  bool tiled_allowed = true;
  // the fused slab pass (inverse y + z + forward y per x-plane) replaces the y and z passes
  // of FP32 solves over the tiled layout with the isotropic law
  bool slab = false;
  bool slab_allowed = false;  // measured slower than the separate passes (opt-in)
  cudaError_t launch_error = cudaSuccess;  // first failed cluster launch since the last check
  int xvariant = 0;      // x-pass tile variant of the fast passes (chosen by timing)
  int yvariant = 0;      // y-pass column-count variant of the fast passes (chosen by timing)
  bool xtuned = false;   // xvariant has been chosen
  bool warm_history = false;  // d_eps0 enters the Anderson history instead of starting it
  GridDesc g{};
  LaunchShape sh32{}, sh64{};
  cudaStream_t stream = nullptr;
  // The iterations of a phase are captured once into a CUDA graph (one iteration) and
  // replayed; capture needs a stream of our own, ordered after/before `stream` by events.
  bool use_graphs = true;
  cudaStream_t graph_stream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  int* d_loop_count = nullptr;   // evaluations of the device-driven iteration loop
  bool use_loop = true;          // one WHILE-node graph launch per phase (else host-polled)
  // FP32 work buffers
  float* d_eps32 = nullptr;      // [batch][6][nv] (used when the caller passes no strain buffer)
  float2* d_spec32 = nullptr;    // [batch][6][nm]
  float2* d_tspec32 = nullptr;   // [batch][6][nm], tiled layout (tiled solvers only)
  // FP64 work buffers, allocated on first use
  double* d_eps64 = nullptr;
  double2* d_spec64 = nullptr;
  double* d_lame64 = nullptr;    // [2][structures][nv]
  int lame64_structs = 0;        // structures d_lame64 holds
  // Anderson acceleration (depth > 0): rings of g = eps + r and r, Gram matrices, coefficients
  float* d_aa_g32 = nullptr;     // [batch][m+1][6][nv]
  __half* d_aa_r32 = nullptr;    // FP16, per-slot power-of-two scales (InstanceState)
  double* d_aa_g64 = nullptr;    // FP64 rings, allocated for FP64 runs
  double* d_aa_r64 = nullptr;
  double* d_aa_partials = nullptr;  // [batch][z blocks][m+2]: Gram-row sums, block max abs r
  double* d_aa_mat = nullptr;    // [batch][m+1][m+1]
  double* d_aa_alpha = nullptr;  // [batch][m+1]
  int aa_zblocks = 0;
  // shared
  double* d_partials = nullptr;  // [batch][x blocks]
  InstanceState* d_state = nullptr;
  Medium* d_medium = nullptr;    // [structures]
  double* d_epsbar = nullptr;    // [batch][6]
  double* d_e0ref = nullptr;     // [batch_cap] reference criteria (lsb_set_reference_e0)
  // damage extension (lsb_set_damage): the caller's field, its element size, k, and the
  // copy in the other precision for the passes of that precision
  const void* dmg_user = nullptr;
  int dmg_elem = 4;
  double dmg_k = 0.0;
  void* d_dmg_conv = nullptr;
  size_t dmg_conv_bytes = 0;
  // anisotropic stiffness (lsb_set_anisotropic): the caller's field, its element size, an
  // optional caller C^0, the copy in the other precision and the per-structure C^0
  const void* aniso_user = nullptr;
  int aniso_elem = 4;
  bool aniso_c0_given = false;
  double aniso_c0[21] = {};
  void* d_cf_conv = nullptr;
  size_t cf_conv_bytes = 0;
  double* d_c0 = nullptr;        // [batch_cap][21]
  double* d_c0_part = nullptr;   // min/max partials of the C^0 reduction
  int x_blocks_generic32 = 1;    // x-pass partials per instance of the generic FP32 pass
  // phase-field work buffers (lsb_phase_field_solve), allocated on first use
  void* d_pf_w = nullptr;
  void* d_pf_chi = nullptr;
  void* d_pf_part = nullptr;
  void* d_pf_state = nullptr;
  void* h_pf_state = nullptr;  // pinned
  bool use_e0ref = false;
  double* d_scratch = nullptr;   // 6 * max(1024, batch_cap)
  double* d_mean_scratch = nullptr;
  double* d_mean = nullptr;      // [batch][6]
  double* d_history = nullptr;   // [batch][history_len]
  int history_len = 0;
  int last_batch = 0;
  float2* d_tw32 = nullptr;
  double2* d_tw64 = nullptr;
  double* d_tables = nullptr;
  InstanceState* h_state = nullptr;  // pinned
  long long launches = 0;            // kernels enqueued by this solver
  // false for a solver whose buffers point into memory it does not own (they are never
  // freed, and the criterion history is not kept)
  bool owns_memory = true;

  ~lsb_solver() {
    if (!owns_memory) return;
    void* bufs[] = {d_eps32, d_spec32, d_tspec32, d_eps64, d_spec64, d_lame64, d_partials, d_state, d_medium,
                    d_epsbar, d_scratch, d_mean_scratch, d_mean, d_history, d_tw32, d_tw64,
                    d_tables, d_aa_g32, d_aa_r32, d_aa_g64, d_aa_r64, d_aa_partials, d_aa_mat,
                    d_aa_alpha, d_e0ref, d_dmg_conv, d_pf_w, d_pf_chi, d_pf_part, d_pf_state,
                    d_cf_conv, d_c0, d_c0_part, d_loop_count};
    for (void* p : bufs) cudaFree(p);
    if (h_state) cudaFreeHost(h_state);
    if (h_pf_state) cudaFreeHost(h_pf_state);
    if (graph_stream) cudaStreamDestroy(graph_stream);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
  }
};

namespace lsb {
namespace detail {

// Records a formatted message for lsb_last_error() and returns `code`.
int fail(int code, const char* fmt, ...);
// Radices of a length-n Stockham plan; false when n has too many prime factors.
bool factorize(int n, Plan1D& p);
// Fills s->g from voxels/extents, plans the launches and checks block sizes.
int plan_grid(lsb_solver* s, const int voxels[3], const double extents[3]);
// How upload_tables fills the table buffers: blocking copies, copies on s->stream, or no
// copy (the buffers already hold this grid's tables).
enum class TableUpload { kBlocking, kAsync, kNone };
// Uploads the twiddle and sin/cos tables into s->d_tw32/d_tw64/d_tables and points the
// plans of s->g at them (the buffers must be sized for the grid).
int upload_tables(lsb_solver* s, TableUpload how = TableUpload::kBlocking);
// Sets s->g.lame_group for a solve of `batch` instances and returns the number of Lame
// field pairs the solve reads (negative with an error message when batch does not split).
int structures_of(lsb_solver* s, int batch);
// Points s->g at the anisotropic stiffness of lsb_set_anisotropic (both precisions) and
// its reference stiffness C^0 for a solve over nstruct structures (aniso.cu).
int prepare_aniso(lsb_solver* s, int nstruct);
// The compile-time-size FP32 passes apply (every extent supported).
inline bool use_fast32(const lsb_solver* s) { return s->fast32; }
// Full FP32-input solve (see lsb_solve); d_eps is the FP32 work buffer and output.
int solve_f32(lsb_solver* s, int batch, const float* d_lambda, const float* d_mu,
              const double* eps_bar, const float* d_eps0, float* d_eps, float* d_sigma,
              double* mean_sigma, double rtol, double atol, int maxiter, int rule, int* iters,
              int* status, double* residual);

// Dataset graphs (batch.cu): see ls_solver.cu.
int prepare_graph_solve(lsb_solver* s, int batch, const float* d_lambda, const float* d_mu, int maxiter);
int append_solve_f32(lsb_solver* s, cudaGraph_t graph, const std::vector<cudaGraphNode_t>& deps,
                     cudaStream_t cap, cudaStream_t body_st, int batch, const float* d_lambda,
                     const float* d_mu, double rtol, double atol, int maxiter, double* h_mean,
                     InstanceState* h_state, std::vector<cudaGraphNode_t>* last,
                     std::vector<cudaGraph_t>* bodies);

}  // namespace detail
}  // namespace lsb
