/*
 * clgpu.h -- C ABI of libclgpu, the B200 (sm_100a) implementation of the
 * Clarabel GPU interior-point hot path.
 *
 * Two levels of entry points:
 *
 *  1. Solver level.  Replaces the GPU branch of Clarabel.Solver / setup! /
 *     solve! (src/solver.jl:5-17, :129-195, :231-422 of the CuClarabel tree)
 *     for one problem (the plain path) or for a batch of independent problems
 *     solved in lock step (the batched path).  Problem data is passed as host
 *     CSC arrays exactly as the reference's CPU-side constructor receives it
 *     (P upper triangle, src/solver.jl:618-630).
 *
 *  2. Cone level.  Replaces the CompositeConeGPU method table
 *     (src/gpucones/coneops_compositecone_gpu.jl) for callers that keep their
 *     own IPM loop: every vector argument is a DEVICE pointer borrowed for the
 *     duration of the call, laid out in the reference's order (cones sorted
 *     zero, nonnegative, second-order, exponential, power, PSD; the same order
 *     rule as src/gpucones/compositecone_type_gpu.jl:75-79).
 *
 * Conventions: every function returns int status, 0 = success, > 0 =
 * numerical failure (maps to NUMERICAL_ERROR / the Dual-scaling fallback of
 * the reference), < 0 = argument or CUDA error.  A cudaStream_t may be passed
 * as NULL (legacy default stream).  Handles are not thread safe; use one
 * handle per host thread or stream.  The library never frees caller memory.
 */
#ifndef CLGPU_H
#define CLGPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *clgpu_stream_t; /* == cudaStream_t */

/* cone type codes, reference order of src/cones/cone_api.jl:93-108 */
enum {
  CLGPU_CONE_ZERO = 0,
  CLGPU_CONE_NONNEG = 1,
  CLGPU_CONE_SOC = 2,
  CLGPU_CONE_EXP = 3,
  CLGPU_CONE_POW = 4,
  CLGPU_CONE_PSD = 5 /* dim = side n of the n x n matrix */
};

/* direct_solve_method (src/settings.jl:113-114, gpu_solver_list of
 * src/Clarabel.jl:27).  The reference names :cudss and :cudssmixed; this
 * library's own batched LDL^T takes their place with the same precision
 * policy: CLGPU_METHOD_MIXED factors in FP32 arithmetic and stores the
 * factor in FP32, refinement in FP64 (directldl_mixed_cudss.jl:42-78).
 * CLGPU_METHOD_MIXED_F64ELIM is this library's variant of it: the
 * elimination in FP64, the factor stored and applied in FP32, refinement in
 * FP64 (the same factor bytes for the solves, a more accurate factor).  Both
 * set the static regularisation to sqrt(eps(Float32)) (src/solver.jl:609-611);
 * instances on the supernodal factorisation factor in FP32 under both. */
enum {
  CLGPU_METHOD_FP64 = 0 /* :cudss */,
  CLGPU_METHOD_MIXED = 1 /* :cudssmixed */,
  CLGPU_METHOD_MIXED_F64ELIM = 2
};

/* mirrors Settings (src/settings.jl:70-148), numeric fields only */
typedef struct {
  int max_iter;
  double time_limit;
  double max_step_fraction;
  double tol_gap_abs, tol_gap_rel, tol_feas, tol_infeas_abs, tol_infeas_rel,
      tol_ktratio;
  double reduced_tol_gap_abs, reduced_tol_gap_rel, reduced_tol_feas,
      reduced_tol_infeas_abs, reduced_tol_infeas_rel, reduced_tol_ktratio;
  int equilibrate_enable, equilibrate_max_iter;
  double equilibrate_min_scaling, equilibrate_max_scaling;
  double linesearch_backtrack_step, min_switch_step_length,
      min_terminate_step_length;
  int static_regularization_enable;
  double static_regularization_constant, static_regularization_proportional;
  int dynamic_regularization_enable;
  double dynamic_regularization_eps, dynamic_regularization_delta;
  int iterative_refinement_enable;
  double iterative_refinement_reltol, iterative_refinement_abstol;
  int iterative_refinement_max_iter;
  double iterative_refinement_stop_ratio;
  int direct_solve_method; /* CLGPU_METHOD_* */
  int soc_threshold;       /* src/settings.jl:147 */
  int verbose;
  int setup_threads;       /* host threads for per-instance setup; 0 = all */
  int fused_solves;        /* 1: kkt_update!'s constant-rhs solve shares the
                              affine solve's launch (same results); 0: its own */
  int device_setup;        /* 1: Ruiz equilibration and the KKT values computed
                              on the device at setup (bitwise the host's
                              result); 0: on the host.  Problems whose
                              matrices hold repeated or unsorted entries are
                              equilibrated on the host either way. */
  int autotune;            /* 1: time the SOC / NN launch shapes at setup and
                              keep the fastest (every shape gives the same
                              bits); 0: default shapes, no timing launches
                              (for solvers set up while others run) */
} clgpu_settings;

/* mirrors DefaultInfo (src/types.jl:227-255) plus solution scalars */
typedef struct {
  int status; /* SolverStatus, src/statuscodes.jl:24-36 */
  int iterations;
  double obj_val, obj_val_dual;
  double cost_primal, cost_dual;
  double res_primal, res_dual, res_primal_inf, res_dual_inf;
  double gap_abs, gap_rel, ktratio, mu, sigma, step_length;
  double solve_time;
} clgpu_info;

/* one problem instance, host memory, borrowed for the create call */
typedef struct {
  int n, m;
  const int *Pp, *Pi;  /* P (n x n) CSC, upper triangle used */
  const double *Px;
  const double *q;     /* n */
  const int *Ap, *Ai;  /* A (m x n) CSC */
  const double *Ax;
  const double *b;     /* m */
  int ncones;
  const int *cone_types;    /* CLGPU_CONE_* (any order) */
  const int *cone_dims;     /* zero/nonneg/soc: dim; psd: side n; exp/pow: 3 */
  const double *cone_params;/* power-cone alpha, else ignored (may be NULL) */
} clgpu_problem;

typedef struct clgpu_solver clgpu_solver;
typedef struct clgpu_cones clgpu_cones;

/* src/settings.jl defaults */
int clgpu_default_settings(clgpu_settings *s);

/* ---------------------------------------------------------------- solver */
/* Solver(P,q,A,b,cones,settings) + setup! for nprob >= 1 instances
 * (src/solver.jl:5-17, :129-195).  nprob == 1 is the plain path. */
int clgpu_solver_create(const clgpu_problem *probs, int nprob,
                        const clgpu_settings *settings, clgpu_solver **out);
/* solve! (src/solver.jl:231-422) for every instance, on the given stream;
 * returns after the stream work has completed. */
int clgpu_solver_solve(clgpu_solver *h, clgpu_stream_t stream);
/* DefaultInfo of one instance after solve */
int clgpu_solver_get_info(clgpu_solver *h, int inst, clgpu_info *info);
/* solution (unscaled, user row order) of one instance into HOST buffers;
 * any pointer may be NULL.  src/solution.jl:2-50 */
int clgpu_solver_get_solution(clgpu_solver *h, int inst, double *x, double *s,
                              double *z);
/* all instances at once: x/s/z concatenated in instance order (sum n / sum m),
 * info array of nprob entries; any pointer may be NULL */
int clgpu_solver_get_solutions(clgpu_solver *h, double *x, double *s,
                               double *z, clgpu_info *info);
/* The same x / s / z without a copy: pointers into the handle's pinned host
 * staging, which the next solve overwrites (no reference counterpart; the
 * reference's solver.solution is likewise refilled by every solve!).  Any
 * pointer may be NULL; -1 before the first solve. */
int clgpu_solver_get_solution_views(const clgpu_solver *h, const double **x,
                                    const double **s, const double **z);
/* update_data! for every instance (src/data_updating.jl:26-120): new values
 * with the sparsity given at setup, concatenated over the instances in
 * instance order, HOST pointers -- Px: the entries of each instance's P in
 * the CSC order given at setup (entries below the diagonal are read and
 * ignored), q, Ax: A's entries in CSC order, b: rows in the caller's order.
 * A NULL pointer leaves that part unchanged.  The equilibration computed at
 * setup is reused, as in the reference; the unscaled norms of q and b are
 * recomputed.  Returns after the values are on the device; -11 when the
 * setup matrices held repeated entries (their values were summed). */
int clgpu_solver_update_data(clgpu_solver *h, const double *Px, const double *q,
                             const double *Ax, const double *b, clgpu_stream_t st);
/* update_q! / update_b! of one instance (same sizes) before the next solve
 * (src/data_updating.jl:155-185); NULL leaves that vector unchanged */
int clgpu_solver_update_qb(clgpu_solver *h, int inst, const double *q,
                           const double *b);
/* device-memory footprint of the handle in bytes */
long long clgpu_solver_device_bytes(const clgpu_solver *h);
/* The launch shapes the setup autotuner chose for this batch (see
 * clgpu_cones_get_launch_shapes); tuning hook, no reference counterpart. */
int clgpu_solver_get_launch_shapes(const clgpu_solver *h, int *nn_block, int *soc_variants);
/* number of kernel launches issued by the last solve */
long long clgpu_solver_launch_count(const clgpu_solver *h);
/* timing of the last solve: total ms and the per-kernel-class ms measured
 * with CUDA events (0 if profiling was not requested) */
int clgpu_solver_set_profiling(clgpu_solver *h, int enable);
int clgpu_solver_get_profile(const clgpu_solver *h, double *ms_total,
                             double *ms_factor, double *ms_solve,
                             double *ms_cones, double *ms_residual,
                             int *passes);
/* per-phase device time of the last profiled solve (CUDA events on the solve
 * stream), ms[6]: ms[0] LDL factorisation, ms[1] one-side LDL solves +
 * refinement, ms[2] KKT refresh (Hs scatter), ms[3] residual kernels, ms[4]
 * update_scaling, ms[5] two-side LDL solves (constant + affine rhs, see
 * fused_solves); calls[6] receives the number of timed launches of each
 * phase.  No reference counterpart (the reference times host phases with
 * TimerOutputs). */
int clgpu_solver_get_phase_times(const clgpu_solver *h, double *ms,
                                 long long *calls);
/* algorithmic bytes of the last profiled solve, bytes[3]: bytes[0] all LDL
 * factorisations, bytes[1] all one-side LDL solves, bytes[2] all two-side
 * solves, with refinement (each stream pass reads its entries, values and
 * chunk words once per side; vectors once per use).  Divided by the phase
 * times this gives the achieved bandwidth.  No reference counterpart. */
int clgpu_solver_get_phase_bytes(const clgpu_solver *h, double *bytes);
/* Supernodal factorisation of the large instances (those whose KKT work
 * vector exceeds the single-warp kernels' 48 KB), per launch kind, summed
 * over the solves since profiling was switched on: device ms (each launch
 * bracketed by CUDA events), algorithmic flops and launches, CLGPU_SN_KINDS
 * entries each (any pointer may be NULL).  Kinds: 0 small fronts, 1 front
 * assembly, 2 diagonal blocks, 3 panel TRSM, 4 trailing update (FP64 DMMA /
 * FP32 FMA tiles), 5-9 forward substitution (small fronts, gather,
 * diagonal blocks, matrix-vector, scatter), 10-14 backward substitution
 * (small fronts, gather, partial sums, diagonal blocks, scatter).  Returns 1
 * when the solver has no such instance.  No reference counterpart. */
#define CLGPU_SN_KINDS 15
/* The numeric setup as the solve sees it, copied to HOST buffers (any may
 * be NULL): equilibration d (sum n), e (sum m, type-major rows), c (one per
 * instance), the scaled q and b (the same layouts) and the stored KKT values
 * (*kkt_nnz of them, the library's permuted order); before the first solve.
 * A diagnostic with no reference counterpart: it lets a test compare the
 * device equilibration (device_setup = 1) with the host's bit for bit. */
int clgpu_solver_debug_setup(const clgpu_solver *h, double *d, double *e, double *c, double *q,
                             double *b, double *Kx, long long *kkt_nnz);
int clgpu_solver_get_sn_profile(const clgpu_solver *h, double *ms, double *flops,
                                long long *calls);
/* Iterative refinement of those instances since profiling was switched on:
 * counts[3] = {solves, refinement sweeps, solves that stopped above the
 * tolerance (stop ratio or sweep limit)}, *worst = the largest final
 * |e|_inf / (abstol + reltol |b|_inf) among the latter.  1 when the solver
 * has no such instance.  A diagnostic with no reference counterpart. */
int clgpu_solver_get_sn_refinement(const clgpu_solver *h, long long *counts, double *worst);
int clgpu_solver_destroy(clgpu_solver *h);

/* ------------------------------------------------ serving (continuous batching)
 * The instances of a solver are slots with fixed structure (P, A sparsity,
 * cones).  admit starts new solves in idle slots, with new q / b values when
 * given (packed slot by slot in the order of `slots`; NULL keeps the current
 * values; copied before return), while other slots are mid-solve: the
 * starting points are computed on a stream of the library's own, overlapping
 * the next step, and the slots join the step after it (at once when nothing
 * else runs).  step runs one IPM iteration of every running slot and lists
 * the slots that finished in it (ascending); *nrunning counts running and
 * admitted slots.  collect post-processes finished slots, copies their
 * x / s / z (packed slot by slot in user order) and infos to the host, and
 * makes them idle again.  At most one admit between two steps.  A slot's
 * result is exactly that of solving it alone.  The first admit makes every
 * slot idle; clgpu_solver_solve leaves serving.  Returns 0, -1 on a bad
 * argument, -2 on a bad or repeated slot, -3 when admitting a slot that is
 * running, admitted or not yet collected, -4 on a second admit before a
 * step.  No reference counterpart (the reference has no serving loop;
 * config 5 of the benchmark plan). */
int clgpu_serve_admit(clgpu_solver *h, const int *slots, int n, const double *q,
                      const double *b, clgpu_stream_t stream);
int clgpu_serve_step(clgpu_solver *h, clgpu_stream_t stream, int *finished,
                     int *nfinished, int *nrunning);
int clgpu_serve_collect(clgpu_solver *h, const int *slots, int n, double *x, double *s,
                        double *z, clgpu_info *info, clgpu_stream_t stream);

/* --------------------------------------------------------------- cones */
/* CompositeConeGPU{T}(cones, soc_threshold)
 * (src/gpucones/compositecone_type_gpu.jl:72-216).  Cones must be sorted
 * by type (zero, nonneg, soc, exp, pow, psd); returns -2 otherwise. */
int clgpu_cones_create(int ncones, const int *types, const int *dims,
                       const double *params, int soc_threshold,
                       clgpu_cones **out);
int clgpu_cones_destroy(clgpu_cones *h);
int clgpu_cones_numel(const clgpu_cones *h);
int clgpu_cones_degree(const clgpu_cones *h);
/* length of the packed Hsblocks vector (rng_blocks, compositecone_type.jl:251) */
int clgpu_cones_hs_len(const clgpu_cones *h);
/* Kernel-time profiling of the cone operations: a profiling hook with no
 * counterpart in the reference.  With profiling on, each operation below
 * brackets its own kernel launches (not its scalar copies or its final
 * synchronisation) with CUDA events, and clgpu_cones_last_kernel_ms returns
 * the device time of the last completed operation in milliseconds
 * (step_length: both launch groups summed). */
int clgpu_cones_set_profiling(clgpu_cones *h, int enable);
/* Launch shapes (a tuning hook with no counterpart in the reference): the
 * threads per block of the nonnegative-cone kernels and, for the
 * CLGPU_SOC_SHAPED_OPS SOC operations update_scaling, affine_ds,
 * combined_ds_shift, Δs_from_Δz_offset, step_length and mul_Hs (in that
 * order), 0 = one lane group per cone or v = 1..3 = shared-memory tiles of
 * 32, 64 or 128 cones of dim <= 16.  clgpu_cones_create and
 * clgpu_solver_create time the candidates on their own cone layout and keep
 * the fastest (a few ms, with temporary device scratch of up to 160 MB plus
 * five vectors of the cone rows, freed before they return; like the rest of
 * set-up, call them outside stream capture); every shape gives the same
 * results.  set: nn_block 0 keeps the current block size, soc_variants NULL
 * keeps the SOC variants; -1 on an invalid shape. */
#define CLGPU_SOC_SHAPED_OPS 6
int clgpu_cones_get_launch_shapes(const clgpu_cones *h, int *nn_block, int *soc_variants);
int clgpu_cones_set_launch_shapes(clgpu_cones *h, int nn_block, const int *soc_variants);
int clgpu_cones_last_kernel_ms(const clgpu_cones *h, double *ms);
/* update_scaling! (coneops_compositecone_gpu.jl:185); strategy 0 PrimalDual,
 * 1 Dual; returns 1 if a cone is not strictly interior */
int clgpu_update_scaling(clgpu_cones *h, const double *s, const double *z,
                         double mu, int strategy, clgpu_stream_t st);
/* set_identity_scaling! (:161) */
int clgpu_set_identity_scaling(clgpu_cones *h, clgpu_stream_t st);
/* get_Hs! (:252) into the packed reference layout */
int clgpu_get_Hs(clgpu_cones *h, double *Hsblocks, clgpu_stream_t st);
/* mul_Hs! (:315) y = Hs x */
int clgpu_mul_Hs(clgpu_cones *h, double *y, const double *x,
                 clgpu_stream_t st);
/* affine_ds! (:409) */
int clgpu_affine_ds(clgpu_cones *h, double *ds, const double *s,
                    clgpu_stream_t st);
/* combined_ds_shift! (:458).  step_z/step_s are read only here (the
 * reference overwrites them with W dz and W^{-T} ds as scratch). */
int clgpu_combined_ds_shift(clgpu_cones *h, double *shift,
                            const double *step_z, const double *step_s,
                            const double *z, double sigma_mu,
                            clgpu_stream_t st);
/* Δs_from_Δz_offset! (:515) */
int clgpu_ds_from_dz_offset(clgpu_cones *h, double *out, const double *ds,
                            const double *z, clgpu_stream_t st);
/* step_length (:566): returns the common step in *alpha (host) */
int clgpu_step_length(clgpu_cones *h, const double *dz, const double *ds,
                      const double *z, const double *s, double alpha_max,
                      double max_step_fraction, double backtrack_step,
                      double alpha_min, double *alpha, clgpu_stream_t st);
/* compute_barrier (:650) */
int clgpu_compute_barrier(clgpu_cones *h, const double *z, const double *s,
                          const double *dz, const double *ds, double alpha,
                          double *barrier, clgpu_stream_t st);
/* margins (:42): pd 0 primal, 1 dual */
int clgpu_margins(clgpu_cones *h, const double *z, int pd, double *alpha,
                  double *beta, clgpu_stream_t st);
/* Margins without a handle and without any device allocation: no
 * counterpart in the reference.  Same result as clgpu_margins on a handle
 * made from the same (types, dims) with clgpu_cones_create.  The cone layout
 * and the per-cone temporaries live in a fixed static device array, so at
 * most CLGPU_MARGINS_STATIC_MAX_CONES second-order plus PSD cones are
 * accepted (CLGPU_ERR_STATIC_TOO_LARGE above that).  The first call on each
 * device looks up that array's address and should come before any stream
 * capture.  Every call is synchronous: it copies the layout through host
 * staging, synchronises the stream and reads the two results back before it
 * returns.  The array is shared per device: overlapping calls race. */
#define CLGPU_MARGINS_STATIC_MAX_CONES 32768
#define CLGPU_ERR_STATIC_TOO_LARGE (-20)
int clgpu_margins_static(int ncones, const int *types, const int *dims,
                         const double *z, int pd, double *alpha, double *beta,
                         clgpu_stream_t st);
/* mul_Hs_diag! (:365): y = Hs x like clgpu_mul_Hs, except on the rows of
 * the sparse (expanded, dim > soc_threshold) second-order cones, which are
 * left as the caller had them: the reference's refinement residual adds
 * their diagonal and rank-2 parts from the KKT matrix
 * (kktsolver_directldl_gpu.jl:454-480). */
int clgpu_mul_Hs_diag(clgpu_cones *h, double *y, const double *x, clgpu_stream_t st);
/* rectify_equilibration! (:21): delta = 1, and mean(e over the cone) / e on
 * the rows of every second-order, exponential, power and PSD cone; device
 * vectors of length numel.  *any_changed (host, may be NULL) = 1 when such
 * a cone exists, as the reference's return value. */
int clgpu_rectify_equilibration(clgpu_cones *h, double *delta, const double *e,
                                int *any_changed, clgpu_stream_t st);
/* The Hs -> KKT refresh of kktsolver_update! (kktsolver_directldl_gpu.jl:
 * 181-214 with update_KKT_sparse_soc_parallel!, :490-548): writes -Hs into
 * the caller's KKT values (device) at hs_map[k] for entry k of the packed
 * Hsblocks layout (clgpu_cones_hs_len entries), and for the sparse
 * second-order cones the expansion entries: per cone (in order) its values
 * [-eta^2 v; -eta^2 u] (2 dim values) at vu_map[j] and vut_map[j], j running
 * over the concatenated 2 dim slots of the sparse cones, and -eta^2, +eta^2
 * at D_map[2 i], D_map[2 i + 1] for the i-th sparse cone.  Maps are the
 * reference's GPUDataMap fields Hsblocks, vu, vut, D made 0-based (device
 * int32).  kkt_vals32 (may be NULL) receives the same values in FP32 (the
 * :cudssmixed matrix copy). */
int clgpu_refresh_kkt(clgpu_cones *h, double *kkt_vals, const int *hs_map, const int *vu_map,
                      const int *vut_map, const int *D_map, float *kkt_vals32,
                      clgpu_stream_t st);
/* step_length (:566) with its scalars in DEVICE memory and no host
 * synchronisation: *alpha = the common step from the start value
 * *alpha_max (both device pointers); asymmetric cones cap it at
 * max_step_fraction and backtrack as clgpu_step_length does.  Returns once
 * the work is queued. */
int clgpu_step_length_device(clgpu_cones *h, const double *dz, const double *ds,
                             const double *z, const double *s, const double *alpha_max,
                             double max_step_fraction, double backtrack_step, double alpha_min,
                             double *alpha, clgpu_stream_t st);
/* scaled_unit_shift! (:81) */
int clgpu_scaled_unit_shift(clgpu_cones *h, double *z, double alpha, int pd,
                            clgpu_stream_t st);
/* unit_initialization! (:115) */
int clgpu_unit_initialization(clgpu_cones *h, double *z, double *s,
                              clgpu_stream_t st);

/* ------------------------------------------------------------ KKT level
 * The direct LDL solver of a KKT matrix the caller assembles and refreshes
 * itself: the AbstractDirectLDLSolver protocol (ldlsolver_constructor /
 * refactor! / solve!, directldl_cudss.jl:30-59) together with
 * _kktsolver_regularize_and_refactor! and the refined solve of
 * GPULDLKKTSolver (kktsolver_directldl_gpu.jl:216-260, :300-413).
 * create: N x N symmetric pattern as a full CSR (both triangles, 0-based,
 * HOST arrays, every row with its diagonal; -2 otherwise, -4 on a repeated
 * entry), Dsigns (+1 / -1 per row, host) and the settings'
 * regularisation, refinement and direct_solve_method (CLGPU_METHOD_MIXED:
 * FP32 factor and substitutions, FP64 refinement); orders the matrix and
 * plans the supernodal factorisation.
 * refactor: Kx (DEVICE, values in the create pattern's CSR order) is
 * copied, its diagonal shifted by eps Dsigns (eps = static_c + static_prop
 * max|diag|, returned in *eps when not NULL) and factored; returns 0, or 1
 * when a pivot is not finite (is_success = false in the reference).
 * solve: x = K \ b with iterative refinement against the unshifted K (b, x
 * DEVICE vectors of length N; may not alias); 0, 1 on a non-finite result,
 * -2 before a successful refactor.  Both synchronise the stream. */
typedef struct clgpu_ldl clgpu_ldl;
int clgpu_ldl_create(int N, const int *Kp, const int *Kj, const signed char *Dsigns,
                     const clgpu_settings *settings, clgpu_ldl **out);
int clgpu_ldl_refactor(clgpu_ldl *h, const double *Kx, double *eps, clgpu_stream_t st);
int clgpu_ldl_solve(clgpu_ldl *h, const double *b, double *x, clgpu_stream_t st);
int clgpu_ldl_destroy(clgpu_ldl *h);

/* residuals_update! (src/residuals.jl:39-75, the GPU form): P full
 * symmetric n x n, A m x n and At = A' (n x m) as CSR, all DEVICE arrays;
 * q, b, x, s, z device vectors; tau, kappa device scalars.  Writes Px, rx_inf
 * = -A' z, rz_inf = A x + s, rx = rx_inf - Px - q tau, rz = rz_inf - b tau
 * and dots[5] = {q.x, b.z, s.z, x.Px, r_tau = q.x + b.z + kappa + x.Px /
 * tau} in device memory.  work: device scratch of clgpu_residuals_work_len()
 * doubles (the per-block partial sums; every reduction runs in a fixed
 * order).  Returns once the work is queued. */
int clgpu_residuals(int n, int m, const int *Pp, const int *Pj, const double *Px,
                    const int *Ap, const int *Aj, const double *Ax, const int *Atp,
                    const int *Atj, const double *Atx, const double *q, const double *b,
                    const double *x, const double *s, const double *z, const double *tau,
                    const double *kappa, double *rx, double *rz, double *rx_inf, double *rz_inf,
                    double *Px_out, double *dots, double *work, clgpu_stream_t st);
int clgpu_residuals_work_len(void);
/* variables_add_step! (src/variables.jl:146-158): x += alpha dx, s += alpha
 * ds, z += alpha dz, tau += alpha dtau, kappa += alpha dkappa; every
 * argument in device memory, alpha included.  Returns once queued. */
int clgpu_add_step(int n, int m, double *x, double *s, double *z, double *tau, double *kappa,
                   const double *dx, const double *ds, const double *dz, const double *dtau,
                   const double *dkappa, const double *alpha, clgpu_stream_t st);

/* --------------------------------------------------------------- checks */
/* The scaling state of the last update_scaling, copied to HOST buffers (any
 * may be NULL); a diagnostic with no reference counterpart, used to check the
 * reference's cone identities (test/UnitTests/test_coneops_secondordercone.jl,
 * test_coneops_psdtrianglecone.jl) on the device's numbers.
 *  second-order cones: w and lambda (one value per SOC row, cones in order),
 *    u and v of the rank-2 form W'W = eta^2 (D + u u' - v v') (per SOC row,
 *    zero on dense cones), eta and d = D[0,0] (one per cone);
 *  PSD cones: R and Rinv (n x n, column-major, cone k from k nmax^2) and
 *    lambda (cone k from k nmax), nmax = the largest side (returned). */
int clgpu_cones_debug_scaling(const clgpu_cones *h, double *soc_w, double *soc_lambda,
                              double *soc_u, double *soc_v, double *soc_eta, double *soc_d,
                              double *psd_R, double *psd_Rinv, double *psd_lambda,
                              int *psd_nmax);
/* Host-only replay of the device factorisation on the structures prepared
 * for one instance: validates the ordering, the symbolic factorisation and
 * every index map, then factors a quasi-definite test matrix on the KKT
 * pattern and returns the solve residual.  No reference counterpart
 * (diagnostic); needs no GPU. */
/* Host-only view of the SOC tiling (diagnostic, no reference counterpart):
 * for n second-order cones with first rows off[k] and dimensions dim[k],
 * writes the tiles the kernels would use for tiles of at most max_cones
 * cones and max_rows rows as [c0, c1) pairs into tiles (room for cap
 * pairs) and returns the number of tiles, or -1 on bad arguments or too
 * little room.  Needs no GPU. */
int clgpu_debug_soc_tiles(const int *off, const int *dim, int n, int max_cones,
                          int max_rows, int *tiles, int cap);
int clgpu_debug_check_instance(const clgpu_problem *prob,
                               const clgpu_settings *settings, double *resid);
/* Host-only view of the factorisation path setup picks for one instance
 * (diagnostic, no reference counterpart): *supernodal = 1 for the
 * supernodal (dense-front) LDL^T, 0 for the single-warp kernels, and the
 * factor's strictly-lower entries.  Needs no GPU. */
int clgpu_debug_instance_path(const clgpu_problem *prob, const clgpu_settings *settings,
                              int *supernodal, long long *factor_entries);
/* Host replay of one instance's streamed-factorisation op stream (the 8-byte
 * records, chunk words and per-level counts that setup uploads for
 * k_ldl_factor_stream) on a quasi-definite matrix with the instance's KKT
 * pattern, compared with a dense LDL^T of the same permuted matrix
 * (diagnostic, no reference counterpart): *resid = largest difference of
 * the L and D entries relative to the largest |D|.  Returns 0, or -3 when
 * the instance does not take the streamed path, -4 when N > 2000, other
 * negative codes for structure errors.  Needs no GPU. */
int clgpu_debug_factor_stream(const clgpu_problem *prob, const clgpu_settings *settings,
                              double *resid);
/* Counters of the process-wide page-locked host pool that setup arrays,
 * upload staging and result staging come from (diagnostic, no reference
 * counterpart): out[0] buffers served from the pool, out[1] page-locked
 * allocations made, out[2] bytes page-locked in all (the pool never
 * shrinks), out[3] failed allocations (heap memory used instead).  Needs no
 * GPU. */
int clgpu_debug_pinned_stats(long long *out);

#ifdef __cplusplus
}
#endif
#endif
