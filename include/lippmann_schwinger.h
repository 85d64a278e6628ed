/* C ABI of liblippmannschwinger.so, the B200 (sm_100a) Lippmann-Schwinger solver.
 *
 * Drop-in for the reference library built from cuda/src (yang-chen-2022/JaxMaterials):
 * the first entry point has the reference's exact signature and meaning; the others are
 * additive. No function takes or returns torch or other framework types.
 *
 * Conventions shared by every entry point:
 *   - fields are float32, C order, z fastest: Lame fields [nx][ny][nz]; strain and
 *     stress [6][nx][ny][nz] in Voigt order (xx, yy, zz, xy, xz, yz) with TENSOR shear
 *     entries (eps_xy, not gamma_xy = 2 eps_xy);
 *   - voxels = (nx, ny, nz), extents = (Lx, Ly, Lz) (cuda/src/common.hh:73-91); the
 *     reference signature takes float extents, the handle API double extents (FP64
 *     runs resolve the grid spacing to FP64);
 *   - the criterion is e = sqrt(<|div sigma|^2>) / |<sigma>| evaluated in Fourier space
 *     (cuda/src/lippmann_schwinger.hh:76-89) and the loop stops when
 *     e < max(rtol * e0, atol), e0 being e at the first iterate.
 *   - a negative return value is an error; lsb_last_error() describes it.
 */
#ifndef LIPPMANN_SCHWINGER_B200_H
#define LIPPMANN_SCHWINGER_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces lippmann_schwinger_solve (cuda/src/lippmann_schwinger.hh:176-184,
 * cuda/src/lippmann_schwinger.cu:236-257), bound by ctypes in
 * src/jaxmaterials/solver/lippmann_schwinger.py:284-322.
 *
 * lambda, mu:   host float[nx*ny*nz]  (lambda FIRST, as in the C signature)
 * epsilon_bar:  host float[6]          macroscopic strain
 * epsilon, sigma: caller-allocated host float[6*nx*ny*nz], overwritten with the
 *               solution and sigma = C : epsilon
 * Returns the number of updates performed; == maxiter means "not converged", as in the
 * reference. Negative on error (the reference only printed errors). Runs in
 * LSB_PREC_MIXED precision, so the tolerance is met even where FP32 round-off alone
 * would stall above it. Device buffers are
 * cached between calls with the same grid on the same device; see
 * lippmann_schwinger_release(). */
int lippmann_schwinger_solve(float *lambda, float *mu, float *epsilon_bar,
                             float *epsilon, float *sigma, int *voxels, float *extents,
                             float rtol, float atol, int maxiter, int verbose);

/* No reference counterpart: frees the buffers cached by lippmann_schwinger_solve. */
void lippmann_schwinger_release(void);

/* ------------------------------------------------------------------ handle API
 * Additive exports (no reference counterpart). A solver owns the device buffers of one
 * grid and a batch capacity; every solve takes DEVICE pointers and runs on the
 * solver's stream. Instances of one call share lambda and mu (e.g. the six load cases
 * of an effective-stiffness computation). */
typedef struct lsb_solver lsb_solver;

/* Statuses written to status[] by the solve calls. */
enum {
  LSB_CONVERGED = 1,
  LSB_MAXITER = 2,
  LSB_NONFINITE = 3,
  LSB_STALLED = 4, /* FP32 round-off floor above the tolerance (LSB_PREC_FP32 only) */
  LSB_TIMEOUT = 5  /* a kernel's bounded wait for its own asynchronous copies ran out and the
                    * instance was abandoned; the solver's device buffers are then suspect:
                    * destroy the solver and create a new one */
};

/* Field precision of the iteration (norms and the stop decision are always FP64):
 * LSB_PREC_FP32   FP32 fields and FFTs; a solve whose criterion stalls on FP32
 *                 round-off above the tolerance ends with LSB_STALLED;
 * LSB_PREC_MIXED  FP32 fields until the criterion stalls near the tolerance, then the
 *                 stalled instances continue from their iterate with FP64 fields (default);
 * LSB_PREC_FP64   FP64 fields from the start. */
enum { LSB_PREC_FP32 = 0, LSB_PREC_MIXED = 1, LSB_PREC_FP64 = 2 };

/* Stop rules: LSB_RULE_CUDA stops when e < max(rtol e0, atol)
 * (cuda/src/lippmann_schwinger.cu:205); LSB_RULE_JAX when e <= max(rtol e0, atol)
 * (src/jaxmaterials/solver/lippmann_schwinger.py:196-206). */
enum { LSB_RULE_CUDA = 0, LSB_RULE_JAX = 1 };

/* Creates a solver for voxels/extents with room for `batch` instances and Anderson
 * depth `depth` (0 = plain Moulinec-Suquet iteration) on the current CUDA device. */
int lsb_create(lsb_solver **out, const int voxels[3], const double extents[3], int batch,
               int depth);
void lsb_destroy(lsb_solver *solver);
/* Stream (cudaStream_t passed as void*) for all later work; NULL = legacy default. */
int lsb_set_stream(lsb_solver *solver, void *stream);

/* Precision mode (LSB_PREC_*) and the stall window: the number of criterion evaluations
 * without a 2% improvement, while the criterion is within 4x of the tolerance, after
 * which FP32 round-off is taken to have stalled the iteration (default 8; 0 disables). */
int lsb_set_precision(lsb_solver *solver, int precision, int stall_window);

/* No reference counterpart. Reference criteria for the stop rule of later solves: with
 * e0 (host double[batch], positive) instance b stops when e < max(rtol * e0[b], atol)
 * instead of using its own first criterion. A warm-started solve given the criterion of
 * the cold start (the residual of a maxiter = 0 solve from eps_bar) thereby stops at the
 * same absolute residual as the cold solve. e0 = NULL clears it. */
int lsb_set_reference_e0(lsb_solver *solver, int batch, const double *e0);

/* No reference counterpart. on != 0 (Anderson depth >= 1 only): the warm start d_eps0 of
 * later solves does not start the iteration; the iteration starts from eps_bar, and its
 * first update sets eps = d_eps0, so that the cold start's and the warm start's residuals
 * are both in the Anderson history and the mixing weighs them (a poor warm start then
 * costs about one update instead of slowing the solve). The criterion e0 is the cold
 * start's. d_eps0 must be eps_bar plus a compatible field (see lsb_solve). */
int lsb_set_warm_history(lsb_solver *solver, int on);

/* No reference counterpart. Tile variant of the FP32 x pass (extents 32-128: 0 = the
 * wide tile, 1 = half as many kz columns per block with twice the resident blocks). By
 * default the solver times both on its first FP32 solve and keeps the faster. variant =
 * 0 or 1 fixes it, -1 only queries. Returns the variant in use (0 before tuning). */
int lsb_tile_variant(lsb_solver *solver, int variant);

/* No reference counterpart. Variant of the FP32 y pass: kz columns per block (0: 8 at
 * extent 128 and 16 elsewhere, 1: the other of 8 and 16; the results are the same). By
 * default the solver's autotuner times both with each x-pass configuration on its first
 * FP32 solve. variant = 0 or 1 fixes it (and the other choices), -1 only queries. Returns
 * the variant in use. */
int lsb_y_variant(lsb_solver *solver, int variant);

/* No reference counterpart. Layout of the FP32 spectrum between the y and x passes:
 * on = 1 (where it applies: every extent in {16, 32, 48, 64, 96, 128}, ny a power of two) keeps
 * it in contiguous x tiles of 8 kz columns in a second spectrum buffer, so that the x pass
 * reads one contiguous chunk per component and tile; on = 0 keeps the cuFFT layout
 * throughout and the strided x pass (lsb_tile_variant). Both give bit-identical results.
 * Returns 1 if the tiled layout is in use after the call, 0 if not. */
int lsb_set_tiled(lsb_solver *solver, int on);

/* No reference counterpart. Fused slab pass: on = 1 runs the inverse y DFT, the z pass and
 * the forward y DFT of every x-plane in one kernel (a thread-block cluster of nz / 16
 * blocks per plane, the plane's half spectrum in distributed shared memory), for FP32
 * solves with the isotropic law over the tiled layout with ny == nz; on = 0 (the default:
 * at 128^3 the fused pass is measured slower than the separate passes) keeps the separate
 * y and z passes. Both give bit-identical results. Returns 1 if the slab pass is in use
 * after the call, 0 if not. */
int lsb_set_slab(lsb_solver *solver, int on);

/* No reference counterpart. FP32 pass configuration of the solver: out (host int[4]) =
 * tiled layout in use, x-pass tile variant of the strided layout, slab pass in use, and
 * whether the configuration is settled (by the autotuner on the first FP32 solve or
 * profile, or by the caller through lsb_tile_variant / lsb_set_tiled / lsb_set_slab).
 * The autotuner times every candidate configuration on the solve's own iteration and
 * keeps the fastest; its choices are cached per (device, grid, Anderson depth, law) in
 * the file named by the environment variable LSB_TUNE_CACHE (default
 * $HOME/.cache/jaxmaterials_b200/tune.tsv; empty or "0": no file). */
int lsb_pass_config(lsb_solver *solver, int *out);

/* No reference counterpart. on != 0 (default): each phase of a solve captures one
 * iteration's launches into a CUDA graph on a stream of the solver's own (ordered after
 * the work already on the solver's stream, and that stream waits for it) and replays it;
 * on = 0 launches the kernels one by one on the solver's stream. */
int lsb_set_graphs(lsb_solver *solver, int on);

/* No reference counterpart. on = 1 (default, with graphs on): each phase of a solve is one
 * launch of a graph whose conditional WHILE node repeats the captured iteration until no
 * instance of the phase is running (decided on the device after every iteration, capped
 * at maxiter + 2 evaluations); the host waits once. on = 0: the host replays the iteration
 * graph in growing chunks and reads the instance states after each chunk. Both give
 * bit-identical results. The environment variable LSB_DEVICE_LOOP=0 sets the default of
 * new solvers to 0 (kernel profilers do not see the kernels of graphs that hold
 * conditional nodes). */
int lsb_set_device_loop(lsb_solver *solver, int on);

/* No reference counterpart. Groups instances by microstructure: with
 * instances_per_field = k > 0, instance b of a solve reads the Lame fields of structure
 * b / k from d_lambda, d_mu laid out [batch / k][nv] (and gets that structure's own
 * reference medium), so one launch sequence solves several structures, e.g. the six
 * unit load cases of batch/6 structures with k = 6. batch must then be a multiple of k.
 * k = 0 (default): every instance shares one field pair [nv]. */
int lsb_set_lame_group(lsb_solver *solver, int instances_per_field);

/* Solves `batch` instances that share d_lambda, d_mu (device float[nv]), or, after
 * lsb_set_lame_group(solver, k), read structure b / k of [batch / k][nv] arrays.
 * eps_bar:   host float[batch*6]
 * d_eps0:    optional device float[batch*6*nv] warm start (NULL: eps = eps_bar). The
 *            updates only add compatible fields, so a warm start must itself be
 *            eps_bar + a compatible zero-mean field (the symmetric gradient of a periodic
 *            displacement, in this discretisation); an arbitrary field converges to an
 *            equilibrium that keeps its incompatible part. One update of the homogeneous
 *            medium lambda = 0, mu = 1/2 from eps0 gives eps1 = eps_bar + (I - P)(eps0 -
 *            eps_bar), P the projection onto compatible fields, so eps0 + eps_bar - eps1 is
 *            the compatible part (Solver.project_compatible in the Python package).
 * d_eps:     device float[batch*6*nv] output strain
 * d_sigma:   optional device float[batch*6*nv] output stress sigma(eps)
 * mean_sigma: optional host double[batch*6], mean stress per instance (FP64 sums)
 * iters, status: host int[batch]; residual: optional host double[batch] final e.
 * Blocks the calling thread until every instance has stopped. */
int lsb_solve(lsb_solver *solver, int batch, const float *d_lambda, const float *d_mu,
              const float *eps_bar, const float *d_eps0, float *d_eps, float *d_sigma,
              double *mean_sigma, float rtol, float atol, int maxiter, int rule,
              int *iters, int *status, double *residual);

/* FP64 variant of lsb_solve (the reference's dtype=float64 path,
 * src/jaxmaterials/solver/lippmann_schwinger.py:146-265): FP64 Lame fields, strain,
 * stress and FFTs on the device; eps_bar host double[batch*6]. */
int lsb_solve_f64(lsb_solver *solver, int batch, const double *d_lambda, const double *d_mu,
                  const double *eps_bar, const double *d_eps0, double *d_eps, double *d_sigma,
                  double *mean_sigma, double rtol, double atol, int maxiter, int rule,
                  int *iters, int *status, double *residual);

/* Criterion history of the last solve: host double[batch*len], e after every
 * evaluation (0 for evaluations that did not happen). len <= maxiter + 1. */
int lsb_history(lsb_solver *solver, double *out, int len);

/* No reference counterpart: number of kernels this solver has enqueued so far. */
long long lsb_kernel_launches(lsb_solver *solver);

/* No reference counterpart: updates of each instance of the last solve that ran with FP64
 * fields (after a mixed-precision switch, or all of them for an FP64 solve); out is host
 * int[batch of that solve]. */
int lsb_fp64_iters(lsb_solver *solver, int *out);

/* No reference counterpart: times every kernel of one FP32 iteration, as the solve runs it
 * (Anderson when the solver's depth > 0, plain otherwise), with CUDA events on the
 * solver's stream, averaged over `reps` iterations that never stop (tolerances 0), after
 * depth + 2 untimed iterations that fill the Anderson rings. Writes the mean milliseconds
 * of each launch to ms_out (host float[max_kernels]) and their kernel names, comma
 * separated, to names (host char[names_len]); returns the number of launches per
 * iteration (or a negative error). d_eps (device float[batch*6*nv]) is the strain work
 * buffer. */
int lsb_profile_step(lsb_solver *solver, int batch, const float *d_lambda, const float *d_mu,
                     float *d_eps, int reps, float *ms_out, int max_kernels, char *names,
                     int names_len);

/* Effective stiffness from the six unit macroscopic strains (the caller in
 * src/jaxmaterials/data/data.py:178-186): row k of c_eff (host double[36]) is the mean
 * stress for eps_bar = e_k. Host lambda/mu float[nv]; iters host int[6]. */
int lsb_c_eff(const float *lambda, const float *mu, const int voxels[3],
              const double extents[3], float rtol, float atol, int maxiter, int depth,
              double *c_eff, int *iters);

/* Effective stiffness of a dataset: the loop over structures of
 * src/jaxmaterials/data/data.py:148-186 (six unit-strain solves per structure, row k of
 * C = mean stress for e_k) as batched solves on the current device. Structure i has
 * voxels[3*i..3*i+2], extents[3*i..3*i+2] and host Lame fields lambda[i], mu[i]
 * (float[nv_i]); grids may differ between structures. Structures of equal grid run
 * together (instance b of a launch reads structure b / 6, each with its own reference
 * medium and its own convergence), different grids concurrently: the whole dataset is one
 * CUDA graph launch (one branch per grid; environment LSB_BATCH_GRAPH=0, or a budget too
 * small for it, selects one host thread and stream per grid instead; same results).
 * depth: Anderson depth; precision: LSB_PREC_*; memory_gb: device memory the call may
 * use (<= 0: 70% of the free memory). Outputs: c_eff host double[nstruct*36],
 * iters and status host int[nstruct*6]. */
int lsb_c_eff_batch(int nstruct, const int *voxels, const double *extents,
                    const float *const *lambda, const float *const *mu, int depth,
                    int precision, float rtol, float atol, int maxiter, double memory_gb,
                    double *c_eff, int *iters, int *status);

/* No reference counterpart. lsb_solve without any allocation, for callers that cannot
 * call cudaMalloc: code running inside a framework that owns all device memory (a
 * caching allocator, or a custom-operator interface that forbids allocation while it
 * runs) and latency-critical callers that must not pay cudaMalloc's implicit device
 * synchronisation. Inputs and outputs are the caller's (device pointers as in lsb_solve,
 * eps_bar host float[batch*6]); all other scratch comes from one static device array of
 * LSB_NOALLOC_SCRATCH_BYTES bytes per GPU, kept until the process exits (a 32^3 grid
 * with 6 load cases needs about 5.5 MB of it). Grids whose scratch does not fit, and
 * batches above LSB_NOALLOC_MAX_BATCH instances, are rejected with an error. The first
 * call on a device (and the first after its context was reset) looks up the array's
 * address (cudaGetSymbolAddress); make that call before any stream capture on the device.
 * All work is ordered on `stream` (the twiddle tables are uploaded on it, only when the
 * grid differs from the previous call's), and the call returns once that stream has
 * finished the solve. Every call reuses the array: calls whose GPU work overlaps in time
 * race and must not be issued. FP32 fields, plain iteration, stop rule LSB_RULE_CUDA,
 * FP32 stall detection (status LSB_STALLED), no criterion history. */
#define LSB_NOALLOC_SCRATCH_BYTES (8u << 20)
#define LSB_NOALLOC_MAX_BATCH 64
int lsb_solve_noalloc(const int voxels[3], const double extents[3], int batch,
                      const float *d_lambda, const float *d_mu, const float *eps_bar,
                      float *d_eps, float *d_sigma, double *mean_sigma, float rtol,
                      float atol, int maxiter, int *iters, int *status, double *residual,
                      void *stream);

/* No reference counterpart (the reference differentiates only forward-mode through
 * JAX, src/driver.py:73-76). Gradient of a loss L of the effective stiffness M (row k =
 * mean stress for the unit strain e_k, as lsb_c_eff) with respect to the Lame fields:
 * d_eps holds the six converged strain fields of one microstructure, device
 * [6 load cases][6][nv] (the output of a batch-6 lsb_solve with eps_bar = identity);
 * dl_dc is host double[36] = dL/dM (row-major). Writes device d_dlambda[nv], d_dmu[nv].
 * The six forward solutions are their own adjoints (the operator is self-adjoint in the
 * energy inner product), so no further solve is needed. Runs on `stream`. */
int lsb_ceff_gradient(const int voxels[3], const float *d_eps, const double *dl_dc,
                      float *d_dlambda, float *d_dmu, void *stream);
/* FP64 variant of lsb_ceff_gradient (fields of lsb_solve_f64). */
int lsb_ceff_gradient_f64(const int voxels[3], const double *d_eps, const double *dl_dc,
                          double *d_dlambda, double *d_dmu, void *stream);

/* Message of the last error on this thread ("" if none). */
const char *lsb_last_error(void);
/* Library ABI version. */
int lsb_version(void);

/* No reference counterpart as a library call: voxelises layered fibre composites on the
 * GPU, as the reference's LayeredFibresDatasetGenerator.material_properties
 * (src/jaxmaterials/data/data.py:267-314) does on the host, for `nsamples` structures at once, with identical results (bit for bit, FP64 predicates).
 *
 * Voxel (i, j, k) has centre (h_x (i + 1/2), h_y (j + 1/2), h_z (k + 1/2)), h_d = L_d / n_d.
 * Every field starts at the matrix value; voxels with z < d_void or z > z_top_void get
 * (void - matrix) added once; then (fibre - matrix) is added once for every fibre that
 * contains the voxel: a fibre record (u0, z0, r2, orientation) contains it when
 * (u - u0)^2 + (z - z0)^2 < r2 with u = x (orientation 0) or y (orientation 1). Each
 * addition is rounded to the output type, as numpy's in-place additions are.
 *
 * voxels[3], extents[3]: grid; d_void, z_top_void: void-layer bounds (z_top_void is L_z -
 * d_void as the caller computes it); values[6] = (mu_void, lambda_void, mu_fibre,
 * lambda_fibre, mu_material, lambda_material); fibre_offsets (host int[nsamples + 1]):
 * sample s owns records fibre_offsets[s] .. fibre_offsets[s+1]-1 of fibres (host
 * double[4 * total]); elem_size 4 (float) or 8 (double); d_out (device) receives
 * [nsamples][2][nx][ny][nz], channel 0 = mu, 1 = lambda (the reference's order); stream: a
 * cudaStream_t or NULL. Returns 0, or a negative code with lsb_last_error(). */
int lsb_voxelise_fibres(int nsamples, const int voxels[3], const double extents[3],
                        double d_void, double z_top_void, const double values[6],
                        const int *fibre_offsets, const double *fibres, int elem_size,
                        void *d_out, void *stream);

/* ---- Damage extension (src/jaxmaterials/solver/lippmann_schwinger.py:36-100, 330-547).
 * Voigt components (v0..v5) of strain and stress sit in the 3 x 3 tensor as
 * [[v0, v5, v4], [v5, v1, v3], [v4, v3, v2]] (src/jaxmaterials/utilities.py:65-85). */

/* Replaces elasticity_solve's stress law (lippmann_schwinger.py:330-455): from the next
 * solve on, every stress evaluation of `solver` uses compute_sigma_damaged
 * (lippmann_schwinger.py:36-75), sigma = ((1 - d)^2 + k) sigma+ + sigma-, where sigma+-
 * are the stresses of the strain's tension and compression parts (spectral split, trace
 * split at 0). d_damage: device [structures][nv] in the layout of the Lame fields (elem_size
 * 4 = float, 8 = double; the other precision is derived per solve); NULL restores the linear
 * law. The field must stay valid while solves use it. Returns 0 or a negative code. */
int lsb_set_damage(lsb_solver *solver, const void *d_damage, int elem_size, double k);

/* Replaces compute_sigma_damaged (lippmann_schwinger.py:36-75) as a standalone call:
 * sigma [batch][6][nv] from eps [batch][6][nv] and lambda, mu, d [nv] (device; d may be
 * NULL: no degradation); elem_size 4 or 8; stream: cudaStream_t or NULL. */
int lsb_damage_stress(long long nv, int batch, const void *d_eps, const void *d_lambda,
                      const void *d_mu, const void *d_damage, double k, void *d_sigma,
                      int elem_size, void *stream);

/* Replaces compute_strain_energy (lippmann_schwinger.py:78-100) and the history update of
 * the staggered scheme (tests/phasefield.py: HH = max(HH, psi)): psi+ = 1/2 lambda
 * <tr eps>+^2 + mu sum <eig>+^2 from eps [6][nv]; writes psi (if d_psi) and/or
 * history = max(history, psi) (if d_history). Device pointers; elem_size 4 or 8. */
int lsb_strain_energy(long long nv, const void *d_eps, const void *d_lambda, const void *d_mu,
                      void *d_psi, void *d_history, int elem_size, void *stream);

/* Replaces phase_field_solve (lippmann_schwinger.py:457-547) on the grid of `solver` and on
 * its stream: d = F^-1[F[chi] / (A0 + |xi~|^2)], chi = B - (A - A0) d with A = 1/lc^2 +
 * 2H/(gc lc), B = 2H/(gc lc), A0 = (min A + max A)/2, until ||chi_new - chi|| <= tolerance
 * ||chi_new|| or maxiter updates. d_history (H) [nv], d_damage [nv] in: previous damage,
 * out: new damage (device, elem_size 4 or 8). Writes the updates done to *iters and the last
 * residual to *residual (either may be NULL). */
int lsb_phase_field_solve(lsb_solver *solver, const void *d_history, void *d_damage, double gc,
                          double lc, double tolerance, int maxiter, int elem_size, int *iters,
                          double *residual);

/* ---- Anisotropic stiffness (the derivation of doc/linear_elasticity.tex:372-402 and
 * doc/anisotropic.py; the reference has no solver for it).
 * From the next solve on, `solver` uses the stiffness field d_stiffness: device
 * [structures][21][nv] (layout of the Lame fields, 21 entries per voxel) holding the
 * independent entries C_0..C_20 of the symmetric 6 x 6 Voigt matrix in the numbering of
 * doc/anisotropic.py:150-185 (C_0..C_5 the diagonal, then (0,1), (0,2), (1,2), (0,3), (0,4),
 * (0,5), (1,3), (1,4), (1,5), (2,3), (2,4), (2,5), (3,4), (3,5), (4,5)), Voigt order (xx, yy,
 * zz, xy, xz, yz), tensor shear: sigma_a = sum_b C_ab w_b eps_b, w = (1, 1, 1, 2, 2, 2).
 * Gamma^0 follows from the reference stiffness C^0 through the inverse of the acoustic
 * matrix K_ki = C^0_kjil xi_j xi_l; c0 (host double[21]) fixes C^0 for every structure,
 * NULL takes (min + max) / 2 of every entry over each structure. The lambda/mu arguments of
 * the solves then do not enter the law (they must still be valid device arrays of the Lame
 * layout, e.g. two entries of the stiffness field). The generic passes run
 * (no compile-time-size FP32 passes). NULL restores the isotropic law; cannot be combined
 * with lsb_set_damage. */
int lsb_set_anisotropic(lsb_solver *solver, const void *d_stiffness, int elem_size,
                        const double *c0);

#ifdef __cplusplus
}
#endif

#endif /* LIPPMANN_SCHWINGER_B200_H */
