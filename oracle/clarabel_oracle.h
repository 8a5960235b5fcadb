/*
 * clarabel_oracle.h -- CPU restatement of the Clarabel interior-point path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the B200
 * implementation in cuclarabel_b200/.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline legs may load it.  The product never links,
 * imports or calls anything here.
 *
 * What it restates (paths relative to the CuClarabel project root):
 *   src/solver.jl:231-582          IPM loop, strategy checkpoints, backtracking
 *   src/variables.jl               mu, step rhs, add_step, initialisation, unscale
 *   src/residuals.jl:1-37          residual update
 *   src/info.jl                    info update, termination, post-process
 *   src/kktsystem.jl:57-210        constant rhs, initial point, reduced KKT solve
 *   src/kktsolvers/kktsolver_directldl.jl:199-467
 *                                  Hs refresh, static regularisation, IR
 *   src/kktsolvers/direct-ldl/directldl_kkt_assembly.jl:15-175,
 *   src/kktsolvers/direct-ldl/directldl_datamaps.jl:183-254
 *                                  triu KKT with sparse SOC expansion
 *   src/problemdata.jl:196-284     Ruiz equilibration
 *   src/cones/ (all but genpow)    all cone operations
 *   src/utils/mathutils.jl         helpers
 * Third-party arithmetic that is not in the reference tree: QDLDL.jl 0.4.1
 * (Project.toml:42) does the CPU LDL^T with dynamic regularisation, and AMD.jl
 * does its ordering.  Their published algorithms are restated in
 * clarabel_oracle.cpp (up-looking LDL^T with elimination tree; the ordering
 * is a minimum-degree ordering of this file's own design, which only changes
 * rounding).
 *
 * Parity pin: the oracle is checked against the golden values in the
 * reference's own tests (test/OptTests/basic_*.jl), committed under
 * tests/golden/.
 */
#ifndef CLARABEL_ORACLE_H
#define CLARABEL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* cone type codes (same as the B200 library) */
enum {
  OR_CONE_ZERO = 0,
  OR_CONE_NONNEG = 1,
  OR_CONE_SOC = 2,
  OR_CONE_EXP = 3,
  OR_CONE_POW = 4,
  OR_CONE_PSD = 5
};

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
  int verbose;
  /* 0: Ruiz cost scaling as the CPU path (mean of triu column norms of P,
   *    src/problemdata.jl:250-251); 1: as the GPU path (mean of full-P row
   *    norms, src/problemdata.jl:337-338) */
  int gpu_equilibration;
  /* 1: round L, D to FP32 after every factorisation (models a factor held
   *    in single precision; refinement stays FP64)
   * 2: the factorisation in FP32 arithmetic (the KKT values rounded to FP32,
   *    every operation of the elimination an FP32 one), as the FP32 sparse
   *    factorisation of the reference's mixed form
   *    (directldl_mixed_cudss.jl:42-78); refinement stays FP64 */
  int factor_fp32;
} oracle_settings;

typedef struct {
  int status; /* SolverStatus codes, src/statuscodes.jl:24-36 */
  int iterations;
  double obj_val, obj_val_dual;
  double cost_primal, cost_dual;
  double res_primal, res_dual, res_primal_inf, res_dual_inf;
  double gap_abs, gap_rel, ktratio, mu, sigma, step_length;
  double solve_time;
  /* iterative refinement over the run: solves, refinement sweeps, solves
   * that ended above abstol + reltol |b|, worst final |e| / that tolerance */
  int ir_solves, ir_sweeps, ir_unconverged;
  double ir_worst_ratio;
} oracle_info;

void oracle_default_settings(oracle_settings *s);

/* Solve min 1/2 x'Px + q'x  s.t. Ax + s = b, s in K.
 * P: upper triangle, CSC (n x n).  A: CSC (m x n).  Cones in the caller's
 * order (the CPU path accepts any order).  Returns 0 on success of the call
 * (the solver status is in info->status), <0 on argument errors. */
int oracle_solve(int n, int m, const int *Pp, const int *Pi, const double *Px,
                 const double *q, const int *Ap, const int *Ai,
                 const double *Ax, const double *b, int ncones,
                 const int *cone_types, const int *cone_dims,
                 const double *cone_params, const oracle_settings *settings,
                 double *x, double *s, double *z, oracle_info *info);

/* Solver object: setup once (equilibration, KKT assembly, ordering,
 * symbolic factorisation), then run the interior-point solve any number of
 * times, each from the default start (src/solver.jl:5-17, :231-422). */
typedef struct oracle_solver oracle_solver;
oracle_solver *oracle_solver_create(int n, int m, const int *Pp, const int *Pi,
                                    const double *Px, const double *q, const int *Ap,
                                    const int *Ai, const double *Ax, const double *b,
                                    int ncones, const int *cone_types, const int *cone_dims,
                                    const double *cone_params,
                                    const oracle_settings *settings);
int oracle_solver_run(oracle_solver *h, double *x, double *s, double *z, oracle_info *info);
void oracle_solver_destroy(oracle_solver *h);

/* ---- per-cone-operation entry points for kernel-level parity tests ---- */
typedef struct oracle_cones oracle_cones;
oracle_cones *oracle_cones_create(int ncones, const int *types,
                                  const int *dims, const double *params);
void oracle_cones_destroy(oracle_cones *c);
int oracle_cones_numel(const oracle_cones *c);
int oracle_cones_degree(const oracle_cones *c);
int oracle_cones_hs_len(const oracle_cones *c);
int oracle_update_scaling(oracle_cones *c, const double *s, const double *z,
                          double mu, int strategy);
void oracle_set_identity_scaling(oracle_cones *c);
void oracle_get_Hs(oracle_cones *c, double *Hsblocks);
void oracle_mul_Hs(oracle_cones *c, double *y, const double *x);
void oracle_affine_ds(oracle_cones *c, double *ds, const double *s);
void oracle_combined_ds_shift(oracle_cones *c, double *shift, double *step_z,
                              double *step_s, const double *z, double sigma_mu);
void oracle_ds_from_dz_offset(oracle_cones *c, double *out, const double *ds,
                              const double *z);
double oracle_step_length(oracle_cones *c, const double *dz, const double *ds,
                          const double *z, const double *s, double alpha_max,
                          double max_step_fraction, double backtrack_step,
                          double alpha_min);
double oracle_compute_barrier(oracle_cones *c, const double *z,
                              const double *s, const double *dz,
                              const double *ds, double alpha);
void oracle_margins(oracle_cones *c, const double *z, int pd, double *alpha,
                    double *beta);
void oracle_scaled_unit_shift(oracle_cones *c, double *z, double alpha, int pd);
void oracle_unit_initialization(oracle_cones *c, double *z, double *s);
/* read back per-cone scaling state: which = 0 w, 1 lambda (per element,
 * numel entries; PSD lambda is n per cone packed at the cone's first n
 * slots), 2 eta (one per cone, SOC only else 0), 3 sparse-SOC d/u/v packed
 * as [d, u(dim), v(dim)] per sparse SOC cone. Returns entries written. */
int oracle_get_state(oracle_cones *c, int which, double *out);

#ifdef __cplusplus
}
#endif
#endif
