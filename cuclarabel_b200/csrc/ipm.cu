// ipm.cu -- device-resident homogeneous-embedding IPM for a batch of
// independent problems (B = 1 is the plain path).
//
// The iteration, termination and strategy logic follow src/solver.jl:231-582,
// src/variables.jl, src/residuals.jl, src/info.jl and src/kktsystem_gpu.jl of
// the CuClarabel tree.  Every scalar of the reference loop (tau, kappa, mu,
// sigma, alpha, status, scaling strategy, ...) is a per-instance device value
// and every host-side decision of the reference is an instance kernel with one
// thread per instance, so a whole pass over the loop body is issued without a
// single device->host copy.  The host reads one counter per pass (how many
// instances are still running).
//
// Lock-step semantics: an instance that would "continue" in the reference
// (new scaling strategy) sets its skip flag and sits out the rest of the pass;
// an instance that would "break" sets done and is frozen.  All vector kernels
// read the per-instance active mask.
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <thread>

#include "cones.cuh"
#include "devbuf.hpp"
#include "pinned.hpp"
#include "ldl.cuh"
#include "equilibrate.cuh"
#include "sn_exec.cuh"
#include "setup.hpp"

namespace clgpu {

static constexpr int TB = 256;
static constexpr int kRedThreads = 128;  // threads of the per-instance reduction blocks
static inline int nblk(long long n) { return n <= 0 ? 1 : (int)((n + TB - 1) / TB); }

// masks for k_set_mask
enum MaskMode { M_PASS = 0, M_SYM, M_ASYM, M_SYM_QP, M_SYM_LP, M_BT, M_ALL_UNDONE };

struct Dev {
  int B = 0, nx = 0, mz = 0;
  // data
  const int *Pp, *Pj, *Ap, *Aj, *Atp, *Atj;
  const double *Px, *Ax, *Atx;
  const double *q, *b, *d, *dinv, *e, *einv, *negq;
  const int *col_inst, *row_inst;
  const int *xoff;              // [B+1]
  const int *zbeg, *zcnt;       // [6*B] per instance and cone type: global z rows
  // variables
  double *x, *s, *z, *px, *ps, *pz;       // current, previous
  double *rhs_x, *rhs_s, *rhs_z;          // step_rhs
  double *dx, *ds, *dz;                   // step_lhs
  double *rx, *rz, *rx_inf, *rz_inf, *Px_; // residuals
  double *x1, *z1, *x2, *z2, *workz, *wconic, *zerox, *zeroz;
  double *S;
  int *I;
  int *active;
  int *counter;
};
__device__ __forceinline__ double &SF(const Dev &d, int f, int i) { return d.S[f * d.B + i]; }
__device__ __forceinline__ int &IF(const Dev &d, int f, int i) { return d.I[f * d.B + i]; }

// per-instance constants kept beside the scalar block
struct InstConst {
  const int *degree;
  const int *sym;
};

struct SettingsDev {
  int max_iter;
  double time_limit, max_step_fraction;
  double tol_gap_abs, tol_gap_rel, tol_feas, tol_infeas_abs, tol_infeas_rel, tol_ktratio;
  double r_gap_abs, r_gap_rel, r_feas, r_infeas_abs, r_infeas_rel, r_ktratio;
  double bt_step, min_switch, min_terminate;
};

// =============================================================== masks
// sel (optional): only instances with sel[i] != 0 can be active (serving
// admits a subset while other instances are mid-solve)
__global__ void k_set_mask(Dev d, InstConst ic, int mode, const int *sel) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B) return;
  // with sel (admitting), the selected slots stay marked done until they are
  // activated at a step boundary, so they count as undone here
  bool undone = sel ? true : IF(d, I_DONE, i) == 0;
  bool v = false;
  switch (mode) {
    case M_PASS: v = undone && IF(d, I_SKIP, i) == 0; break;
    case M_SYM: v = undone && ic.sym[i]; break;
    case M_ASYM: v = undone && !ic.sym[i]; break;
    case M_SYM_QP: v = undone && ic.sym[i] && IF(d, I_PNNZ, i); break;
    case M_SYM_LP: v = undone && ic.sym[i] && !IF(d, I_PNNZ, i); break;
    case M_BT: v = undone && IF(d, I_SKIP, i) == 0 && IF(d, I_BT_ACTIVE, i); break;
    case M_ALL_UNDONE: v = undone; break;
  }
  if (sel && !sel[i]) v = false;
  d.active[i] = v ? 1 : 0;
}

__global__ void k_zero_fields(Dev d, int f0, int nf, double v) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nf * d.B) return;
  d.S[f0 * d.B + t] = v;
}

// =============================================================== init
__global__ void k_init_state(Dev d, const double *c, const double *normq,
                             const double *normb, const int *pnnz, const int *sel) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || (sel && !sel[i])) return;
  for (int f = 0; f < NUM_SCALARS; ++f) SF(d, f, i) = 0.0;
  for (int f = 0; f < NUM_INTS; ++f) IF(d, f, i) = 0;
  SF(d, F_TAU, i) = 1.0;
  SF(d, F_KAPPA, i) = 1.0;
  SF(d, F_SIGMA, i) = 1.0;
  SF(d, F_MU, i) = kDMax;
  const double inf = CUDART_INF;
  SF(d, F_PREV_COST_P, i) = inf;
  SF(d, F_PREV_COST_D, i) = inf;
  SF(d, F_PREV_RES_P, i) = inf;
  SF(d, F_PREV_RES_D, i) = inf;
  SF(d, F_PREV_GAP_ABS, i) = inf;
  SF(d, F_PREV_GAP_REL, i) = inf;
  SF(d, F_EQ_C, i) = c[i];
  SF(d, F_NORMQ, i) = normq[i];
  SF(d, F_NORMB, i) = normb[i];
  IF(d, I_PNNZ, i) = pnnz[i];
  IF(d, I_SCALING, i) = 0;  // PrimalDual (every supported cone allows it)
  IF(d, I_KKT_OK, i) = 1;
  IF(d, I_SCALE_OK, i) = 1;
  // an admitted slot (sel) stays out of the running passes until activated
  if (sel) IF(d, I_DONE, i) = 1;
}

// x = 0 for the asymmetric (unit) start, tau = kappa = 1
__global__ void k_zero_x_masked(Dev d) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= d.nx) return;
  if (!d.active[d.col_inst[j]]) return;
  d.x[j] = 0.0;
}
__global__ void k_negate_s_masked(Dev d) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= d.mz) return;
  if (!d.active[d.row_inst[g]]) return;
  d.s[g] = -d.s[g];
}
__global__ void k_s_from_neg_z_masked(Dev d) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= d.mz) return;
  if (!d.active[d.row_inst[g]]) return;
  d.s[g] = -d.z[g];
}
// _shift_to_cone_interior! (variables.jl:276-304): two shift amounts per
// instance from the margins
__global__ void k_shift_amounts(Dev d, InstConst ic, int fmin, int fsum, int fa1, int fa2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || !d.active[i]) return;
  double mm = SF(d, fmin, i), pm = SF(d, fsum, i);
  int deg = ic.degree[i];
  double target = fmax(1.0, 0.1 * pm / deg);
  double a1, a2;
  if (mm <= 0) {
    a1 = -mm;
    a2 = target;
  } else if (mm < target) {
    a1 = target - mm;
    a2 = 0.0;
  } else {
    a1 = 0.0;
    a2 = 0.0;
  }
  SF(d, fa1, i) = a1;
  SF(d, fa2, i) = a2;
}
__global__ void k_set_tau_kappa_one(Dev d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || !d.active[i]) return;
  SF(d, F_TAU, i) = 1.0;
  SF(d, F_KAPPA, i) = 1.0;
}

// =============================================================== residuals
// Deterministic per-instance block reduction: every thread accumulates a
// fixed strided subset in a fixed order, warps reduce by shuffles, warp
// partials are combined in warp order.  Results do not depend on the batch.
template <int NV, int NTH>
__device__ __forceinline__ void block_reduce_store(double (&acc)[NV], double *S, int B,
                                                   const int (&field)[NV], int inst) {
  __shared__ double red[NTH / 32][NV];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double t = warp_sum(acc[v]);
    if (lane == 0) red[wid][v] = t;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double t = 0;
    for (int w = 0; w < NTH / 32; ++w) t += red[w][threadIdx.x];
    S[field[threadIdx.x] * B + inst] = t;
  }
}

// residuals.jl:39-75 fused with the scaled norms of info.jl:66-133; one
// block per instance
template <int NTH>
__global__ void __launch_bounds__(NTH) k_residuals(Dev d) {
  const int i = blockIdx.x;
  if (!d.active[i]) return;
  double acc[12];
#pragma unroll
  for (int v = 0; v < 12; ++v) acc[v] = 0.0;
  const double tau = SF(d, F_TAU, i);
  for (int j = d.xoff[i] + threadIdx.x; j < d.xoff[i + 1]; j += NTH) {
    double px = 0;
    for (int p = d.Pp[j]; p < d.Pp[j + 1]; ++p) px += d.Px[p] * d.x[d.Pj[p]];
    double atz = 0;
    for (int p = d.Atp[j]; p < d.Atp[j + 1]; ++p) atz += d.Atx[p] * d.z[d.Atj[p]];
    const double rxinf = -atz;
    const double xj = d.x[j];
    const double rx = rxinf - px - d.q[j] * tau;
    d.Px_[j] = px;
    d.rx_inf[j] = rxinf;
    d.rx[j] = rx;
    acc[0] += d.q[j] * xj;
    acc[1] += xj * px;
    double t = d.d[j] * xj;
    acc[2] += t * t;
    t = d.dinv[j] * rxinf;
    acc[3] += t * t;
    t = d.dinv[j] * px;
    acc[4] += t * t;
    t = d.dinv[j] * rx;
    acc[5] += t * t;
  }
  for (int ty = 0; ty < 6; ++ty) {
    const int g0 = d.zbeg[6 * i + ty], g1 = g0 + d.zcnt[6 * i + ty];
    for (int g = g0 + threadIdx.x; g < g1; g += NTH) {
      double ax = 0;
      for (int p = d.Ap[g]; p < d.Ap[g + 1]; ++p) ax += d.Ax[p] * d.x[d.Aj[p]];
      const double sg = d.s[g], zg = d.z[g];
      const double rzinf = ax + sg;
      const double rz = rzinf - d.b[g] * tau;
      d.rz_inf[g] = rzinf;
      d.rz[g] = rz;
      acc[6] += d.b[g] * zg;
      acc[7] += sg * zg;
      double t = d.e[g] * zg;
      acc[8] += t * t;
      t = d.einv[g] * sg;
      acc[9] += t * t;
      t = d.einv[g] * rzinf;
      acc[10] += t * t;
      t = d.einv[g] * rz;
      acc[11] += t * t;
    }
  }
  const int fields[12] = {F_DOT_QX, F_DOT_XPX, F_NRM_X, F_NRM_RXINF, F_NRM_PX, F_NRM_RX,
                          F_DOT_BZ, F_DOT_SZ, F_NRM_Z, F_NRM_S, F_NRM_RZINF, F_NRM_RZ};
  block_reduce_store<12, NTH>(acc, d.S, d.B, fields, i);
}

__device__ void check_convergence(const Dev &d, int i, double tga, double tgr, double tf,
                                  double tia, double tir, double tkt, int ss, int ps,
                                  int ds) {
  double kt = SF(d, F_KTRATIO, i);
  double gabs = SF(d, F_GAP_ABS, i), grel = SF(d, F_GAP_REL, i);
  double rp = SF(d, F_RES_P, i), rd = SF(d, F_RES_D, i);
  if (kt <= 1.0 && ((gabs < tga || grel < tgr) && rp < tf && rd < tf)) {
    IF(d, I_STATUS, i) = ss;
  } else if (kt > 1000. / tkt) {
    double bz = SF(d, F_DOT_BZ, i), qx = SF(d, F_DOT_QX, i);
    if (bz < -tia && SF(d, F_RES_PINF, i) < -tir * bz)
      IF(d, I_STATUS, i) = ps;
    else if (qx < -tia && SF(d, F_RES_DINF, i) < -tir * qx)
      IF(d, I_STATUS, i) = ds;
  }
}

// mu, info_update!, info_check_termination!, insufficient-progress checkpoint
// (solver.jl:267-295, info.jl:66-190, solver.jl:521-540)
__global__ void k_info_termination(Dev d, InstConst ic, SettingsDev st, double elapsed,
                                   int *reset_flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B) return;
  reset_flag[i] = 0;
  if (!d.active[i]) return;
  double tau = SF(d, F_TAU, i), kappa = SF(d, F_KAPPA, i);
  double mu = (SF(d, F_DOT_SZ, i) + tau * kappa) / (ic.degree[i] + 1);
  SF(d, F_MU, i) = mu;
  double tinv = 1.0 / tau;
  double cinv = 1.0 / SF(d, F_EQ_C, i);
  double xPx = SF(d, F_DOT_XPX, i) * tinv * tinv / 2;
  double cp = (SF(d, F_DOT_QX, i) * tinv + xPx) * cinv;
  double cd = (-SF(d, F_DOT_BZ, i) * tinv - xPx) * cinv;
  SF(d, F_COST_P, i) = cp;
  SF(d, F_COST_D, i) = cd;
  double normx = sqrt(SF(d, F_NRM_X, i));
  double normz = sqrt(SF(d, F_NRM_Z, i)) * cinv;
  double norms = sqrt(SF(d, F_NRM_S, i));
  SF(d, F_RES_PINF, i) = (sqrt(SF(d, F_NRM_RXINF, i)) * cinv) / fmax(1.0, normz);
  SF(d, F_RES_DINF, i) = fmax(sqrt(SF(d, F_NRM_PX, i)) / fmax(1.0, normx),
                              sqrt(SF(d, F_NRM_RZINF, i)) / fmax(1.0, normx + norms));
  normx *= tinv;
  normz *= tinv;
  norms *= tinv;
  SF(d, F_RES_P, i) = sqrt(SF(d, F_NRM_RZ, i)) * tinv /
                      fmax(1.0, SF(d, F_NORMB, i) + normx + norms);
  SF(d, F_RES_D, i) = sqrt(SF(d, F_NRM_RX, i)) * tinv * cinv /
                      fmax(1.0, SF(d, F_NORMQ, i) + normx + normz);
  double gabs = fabs(cp - cd);
  SF(d, F_GAP_ABS, i) = gabs;
  SF(d, F_GAP_REL, i) = gabs / fmax(1.0, fmin(fabs(cp), fabs(cd)));
  SF(d, F_KTRATIO, i) = kappa * tinv;
  // info_save_scalars(mu, alpha, sigma, iter)
  SF(d, F_SOLVE_TIME, i) = elapsed;
  int iter = IF(d, I_ITER, i);
  // termination
  IF(d, I_STATUS, i) = ST_UNSOLVED;
  check_convergence(d, i, st.tol_gap_abs, st.tol_gap_rel, st.tol_feas, st.tol_infeas_abs,
                    st.tol_infeas_rel, st.tol_ktratio, ST_SOLVED, ST_PRIMAL_INFEASIBLE,
                    ST_DUAL_INFEASIBLE);
  double rd = SF(d, F_RES_D, i), rp = SF(d, F_RES_P, i);
  double prd = SF(d, F_PREV_RES_D, i), prp = SF(d, F_PREV_RES_P, i);
  double kt = SF(d, F_KTRATIO, i);
  if (IF(d, I_STATUS, i) == ST_UNSOLVED && iter > 1 && (rd > prd || rp > prp)) {
    if (kt < 100 * kDEps &&
        (SF(d, F_PREV_GAP_ABS, i) < st.tol_gap_abs || SF(d, F_PREV_GAP_REL, i) < st.tol_gap_rel))
      IF(d, I_STATUS, i) = ST_INSUFFICIENT_PROGRESS;
    if (kt < 1.0) {
      if ((rd > 100 * st.tol_feas && rd > 100 * prd) || (rp > 100 * st.tol_feas && rp > 100 * prp))
        IF(d, I_STATUS, i) = ST_INSUFFICIENT_PROGRESS;
    }
  }
  if (IF(d, I_STATUS, i) == ST_UNSOLVED) {
    if (st.max_iter == iter)
      IF(d, I_STATUS, i) = ST_MAX_ITERATIONS;
    else if (elapsed > st.time_limit)
      IF(d, I_STATUS, i) = ST_MAX_TIME;
  }
  int status = IF(d, I_STATUS, i);
  if (status != ST_UNSOLVED) {
    if (status != ST_INSUFFICIENT_PROGRESS) {
      IF(d, I_DONE, i) = 1;
    } else {
      // info_reset_to_prev_iterate
      SF(d, F_COST_P, i) = SF(d, F_PREV_COST_P, i);
      SF(d, F_COST_D, i) = SF(d, F_PREV_COST_D, i);
      SF(d, F_RES_P, i) = SF(d, F_PREV_RES_P, i);
      SF(d, F_RES_D, i) = SF(d, F_PREV_RES_D, i);
      SF(d, F_GAP_ABS, i) = SF(d, F_PREV_GAP_ABS, i);
      SF(d, F_GAP_REL, i) = SF(d, F_PREV_GAP_REL, i);
      SF(d, F_TAU, i) = SF(d, F_PREV_TAU, i);
      SF(d, F_KAPPA, i) = SF(d, F_PREV_KAPPA, i);
      reset_flag[i] = 1;
      if (!ic.sym[i] && IF(d, I_SCALING, i) == 0) {
        IF(d, I_STATUS, i) = ST_UNSOLVED;
        IF(d, I_SCALING, i) = 1;
        IF(d, I_SKIP, i) = 1;
      } else {
        IF(d, I_DONE, i) = 1;
      }
    }
  }
  // record for the final "alpha == 0" re-save
  SF(d, F_SIGMA_MU, i) = 0;
}

__global__ void k_reset_vars(Dev d, const int *reset_flag) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < d.nx && reset_flag[d.col_inst[t]]) d.x[t] = d.px[t];
  if (t < d.mz && reset_flag[d.row_inst[t]]) {
    d.s[t] = d.ps[t];
    d.z[t] = d.pz[t];
  }
}

// after update_scaling (solver.jl:300-313)
__global__ void k_after_scaling(Dev d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || !d.active[i]) return;
  if (!IF(d, I_SCALE_OK, i)) {
    IF(d, I_STATUS, i) = ST_NUMERICAL_ERROR;
    IF(d, I_DONE, i) = 1;
    return;
  }
  IF(d, I_ITER, i) += 1;
  IF(d, I_KKT_OK, i) = 1;
}

// ======================================================== update_data!
// New problem values scaled with the equilibration computed at setup (d, e,
// c), as _update_matrix / _update_vector do (data_updating.jl:185-300), and
// written into every device copy: the full P, A, A^T and the KKT matrix.
__global__ void k_update_P(Dev d, const int4 *__restrict__ map, const int2 *__restrict__ xy,
                           const double *__restrict__ in, long long n, const double *c,
                           double *Kx) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int2 rc = xy[t];
  if (rc.x < 0) return;  // below the diagonal: ignored, as at setup
  const int4 m = map[t];
  const double v = in[t] * d.d[rc.x] * d.d[rc.y] * c[d.col_inst[rc.x]];
  double *Px = const_cast<double *>(d.Px);
  if (m.x >= 0) Px[m.x] = v;
  if (m.y >= 0) Px[m.y] = v;
  if (m.z >= 0) Kx[m.z] = v;
  if (m.w >= 0) Kx[m.w] = v;
}
__global__ void k_update_A(Dev d, const int4 *__restrict__ map, const int2 *__restrict__ xy,
                           const double *__restrict__ in, long long n, double *Kx) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int4 m = map[t];
  const int2 rc = xy[t];  // global row, global column
  const double v = in[t] * d.e[rc.x] * d.d[rc.y];
  const_cast<double *>(d.Atx)[m.x] = v;
  const_cast<double *>(d.Ax)[m.y] = v;
  if (m.z >= 0) Kx[m.z] = v;
  if (m.w >= 0) Kx[m.w] = v;
}
__global__ void k_update_q(Dev d, const double *__restrict__ in, int lo, int hi,
                           const double *c) {
  const int j = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= hi) return;
  const double v = in[j] * d.d[j] * c[d.col_inst[j]];
  const_cast<double *>(d.q)[j] = v;
  const_cast<double *>(d.negq)[j] = -v;
}
__global__ void k_update_b(Dev d, const double *__restrict__ in, int lo, int hi,
                           const int *zmap) {
  const int u = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= hi) return;
  const int g = zmap[u];
  const_cast<double *>(d.b)[g] = in[u] * d.e[g];
}
// unscaled infinity norms of the new q / b of instances [lo, hi) (the
// reference flushes them on update and recomputes them in solve!)
template <int NTH>
__global__ void __launch_bounds__(NTH)
    k_update_norms(const double *__restrict__ inq, const double *__restrict__ inb,
                   const int *xoff, const int *moff, int lo, double *normq, double *normb) {
  const int i = lo + blockIdx.x;
  __shared__ double red[2][NTH / 32];
  double mq = 0, mb = 0;
  if (inq)
    for (int j = xoff[i] + threadIdx.x; j < xoff[i + 1]; j += NTH) mq = fmax(mq, fabs(inq[j]));
  if (inb)
    for (int u = moff[i] + threadIdx.x; u < moff[i + 1]; u += NTH) mb = fmax(mb, fabs(inb[u]));
  mq = warp_max(mq);
  mb = warp_max(mb);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = mq;
    red[1][threadIdx.x >> 5] = mb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < NTH / 32; ++w) {
      mq = fmax(mq, red[0][w]);
      mb = fmax(mb, red[1][w]);
    }
    if (inq) normq[i] = mq;
    if (inb) normb[i] = mb;
  }
}

// ============================================================ KKT glue
// workz = dsc - rhs_z (kktsystem_gpu.jl:168)
__global__ void k_workz(Dev d, const double *dsc) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= d.mz || !d.active[d.row_inst[g]]) return;
  d.workz[g] = dsc[g] - d.rhs_z[g];
}
// the three P products and seven dots of the tau solve
// (kktsystem_gpu.jl:179-200); one block per instance
template <int NTH>
__global__ void __launch_bounds__(NTH) k_tau_dots(Dev d) {
  const int i = blockIdx.x;
  if (!d.active[i] || !IF(d, I_KKT_OK, i)) return;
  double acc[7];
#pragma unroll
  for (int v = 0; v < 7; ++v) acc[v] = 0.0;
  const double tau = SF(d, F_TAU, i);
  for (int j = d.xoff[i] + threadIdx.x; j < d.xoff[i + 1]; j += NTH) {
    double px1 = 0, pxm = 0, px2 = 0;
    for (int p = d.Pp[j]; p < d.Pp[j + 1]; ++p) {
      const int k = d.Pj[p];
      const double v = d.Px[p];
      px1 += v * d.x1[k];
      pxm += v * (d.x[k] / tau - d.x2[k]);
      px2 += v * d.x2[k];
    }
    const double xi = d.x[j] / tau;
    acc[0] += d.q[j] * d.x1[j];
    acc[1] += xi * px1;
    acc[2] += d.q[j] * d.x2[j];
    acc[3] += (xi - d.x2[j]) * pxm;
    acc[4] += d.x2[j] * px2;
  }
  for (int ty = 0; ty < 6; ++ty) {
    const int g0 = d.zbeg[6 * i + ty], g1 = g0 + d.zcnt[6 * i + ty];
    for (int g = g0 + threadIdx.x; g < g1; g += NTH) {
      acc[5] += d.b[g] * d.z1[g];
      acc[6] += d.b[g] * d.z2[g];
    }
  }
  const int fields[7] = {F_DOT_Q_X1, F_DOT_XI_PX1, F_DOT_Q_X2, F_QF1, F_QF2, F_DOT_B_Z1,
                         F_DOT_B_Z2};
  block_reduce_store<7, NTH>(acc, d.S, d.B, fields, i);
}
__global__ void k_tau_solve(Dev d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || !d.active[i] || !IF(d, I_KKT_OK, i)) return;
  double tau = SF(d, F_TAU, i), kappa = SF(d, F_KAPPA, i);
  double num = SF(d, F_RHS_TAU, i) - SF(d, F_RHS_KAPPA, i) / tau + SF(d, F_DOT_Q_X1, i) +
               SF(d, F_DOT_B_Z1, i) + 2 * SF(d, F_DOT_XI_PX1, i);
  double den = kappa / tau - SF(d, F_DOT_Q_X2, i) - SF(d, F_DOT_B_Z2, i);
  den += SF(d, F_QF1, i) - SF(d, F_QF2, i);
  SF(d, F_STEP_TAU, i) = num / den;
}
__global__ void k_lhs_xz(Dev d) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < d.nx) {
    int inst = d.col_inst[t];
    if (d.active[inst] && IF(d, I_KKT_OK, inst))
      d.dx[t] = d.x1[t] + SF(d, F_STEP_TAU, inst) * d.x2[t];
  }
  if (t < d.mz) {
    int inst = d.row_inst[t];
    if (d.active[inst] && IF(d, I_KKT_OK, inst))
      d.dz[t] = d.z1[t] + SF(d, F_STEP_TAU, inst) * d.z2[t];
  }
}
// ds = -(Hs dz + dsc); dkappa (kktsystem_gpu.jl:213-220)
__global__ void k_lhs_s(Dev d, const double *dsc) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= d.mz) return;
  int inst = d.row_inst[g];
  if (!d.active[inst] || !IF(d, I_KKT_OK, inst)) return;
  d.ds[g] = -(d.ds[g] + dsc[g]);
}
__global__ void k_lhs_kappa(Dev d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || !d.active[i] || !IF(d, I_KKT_OK, i)) return;
  double tau = SF(d, F_TAU, i);
  SF(d, F_STEP_KAPPA, i) = -(SF(d, F_RHS_KAPPA, i) + SF(d, F_KAPPA, i) * SF(d, F_STEP_TAU, i)) / tau;
}

// affine rhs (variables.jl:161-175)
__global__ void k_affine_rhs(Dev d) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < d.nx && d.active[d.col_inst[t]]) d.rhs_x[t] = d.rx[t];
  if (t < d.mz && d.active[d.row_inst[t]]) d.rhs_z[t] = d.rz[t];
  if (t < d.B && d.active[t]) {
    double rtau = SF(d, F_DOT_QX, t) + SF(d, F_DOT_BZ, t) + SF(d, F_KAPPA, t) +
                  SF(d, F_DOT_XPX, t) / SF(d, F_TAU, t);
    SF(d, F_RTAU, t) = rtau;
    SF(d, F_RHS_TAU, t) = rtau;
    SF(d, F_RHS_KAPPA, t) = SF(d, F_TAU, t) * SF(d, F_KAPPA, t);
  }
}

// ============================================================ step length
// variables.jl:14-43
__global__ void k_step_prep(Dev d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || !d.active[i] || !IF(d, I_KKT_OK, i)) return;
  double dt = SF(d, F_STEP_TAU, i), dk = SF(d, F_STEP_KAPPA, i);
  double at = dt < 0 ? -SF(d, F_TAU, i) / dt : kDMax;
  double ak = dk < 0 ? -SF(d, F_KAPPA, i) / dk : kDMax;
  SF(d, F_STEP_SYM, i) = fmin(fmin(at, ak), 1.0);
}
__global__ void k_step_mid(Dev d, InstConst ic, double msf) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || !d.active[i] || !IF(d, I_KKT_OK, i)) return;
  double a = SF(d, F_STEP_SYM, i);
  if (!ic.sym[i]) a = fmin(a, msf);
  SF(d, F_STEP_SYM, i) = a;
  SF(d, F_STEP, i) = a;
}
__global__ void k_step_final(Dev d, int combined, double msf, int out_field) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || !d.active[i] || !IF(d, I_KKT_OK, i)) return;
  double a = SF(d, F_STEP, i);
  if (combined) a *= msf;
  SF(d, out_field, i) = a;
}

// sigma, mfac and the combined tau/kappa rhs (solver.jl:344-357,
// variables.jl:218-258)
__global__ void k_combined_scalars(Dev d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || !d.active[i] || !IF(d, I_KKT_OK, i)) return;
  double a = SF(d, F_ALPHA_AFF, i);
  double sigma = (1 - a) * (1 - a) * (1 - a);
  SF(d, F_SIGMA, i) = sigma;
  double mfac = IF(d, I_ITER, i) > 1 ? 1.0 : a;
  SF(d, F_MFAC, i) = mfac;
  double mu = SF(d, F_MU, i);
  double sm = sigma * mu;
  SF(d, F_SIGMA_MU, i) = sm;
  double dt = SF(d, F_STEP_TAU, i), dk = SF(d, F_STEP_KAPPA, i);
  SF(d, F_RHS_TAU, i) = (1 - sigma) * SF(d, F_RTAU, i);
  SF(d, F_RHS_KAPPA, i) = -sm + mfac * dt * dk + SF(d, F_TAU, i) * SF(d, F_KAPPA, i);
}
__global__ void k_combined_pre(Dev d) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < d.nx) {
    int inst = d.col_inst[t];
    if (d.active[inst] && IF(d, I_KKT_OK, inst))
      d.rhs_x[t] = (1 - SF(d, F_SIGMA, inst)) * d.rx[t];
  }
  if (t < d.mz) {
    int inst = d.row_inst[t];
    if (d.active[inst] && IF(d, I_KKT_OK, inst)) {
      double mf = SF(d, F_MFAC, inst);
      if (mf != 1.0) d.dz[t] *= mf;
    }
  }
}
// d.s += shift (held in rhs_z) ; d.z = (1-sigma) rz
__global__ void k_combined_post(Dev d) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= d.mz) return;
  int inst = d.row_inst[g];
  if (!d.active[inst] || !IF(d, I_KKT_OK, inst)) return;
  d.rhs_s[g] += d.rhs_z[g];
  d.rhs_z[g] = (1 - SF(d, F_SIGMA, inst)) * d.rz[g];
}

// _strategy_checkpoint_numerical_error (solver.jl:543-557)
__global__ void k_check_numerical(Dev d, InstConst ic) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || !d.active[i]) return;
  if (IF(d, I_KKT_OK, i)) return;
  SF(d, F_ALPHA, i) = 0.0;
  if (!ic.sym[i] && IF(d, I_SCALING, i) == 0) {
    IF(d, I_SCALING, i) = 1;
    IF(d, I_SKIP, i) = 1;
  } else {
    IF(d, I_STATUS, i) = ST_NUMERICAL_ERROR;
    IF(d, I_DONE, i) = 1;
  }
}

// barrier backtracking setup (solver.jl:449-485)
__global__ void k_bt_setup(Dev d, InstConst ic) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B) return;
  bool bt = d.active[i] && !ic.sym[i] && IF(d, I_SCALING, i) == 1;
  IF(d, I_BT_ACTIVE, i) = bt ? 1 : 0;
  if (bt) atomicAdd(d.counter + 1, 1);
}
// dot_shifted (mathutils.jl:23-43) per instance, deterministic
template <int NTH>
__global__ void __launch_bounds__(NTH) k_dot_shifted(Dev d) {
  const int i = blockIdx.x;
  if (!d.active[i]) return;
  double acc[1] = {0.0};
  const double a = SF(d, F_ALPHA, i);
  for (int ty = 0; ty < 6; ++ty) {
    const int g0 = d.zbeg[6 * i + ty], g1 = g0 + d.zcnt[6 * i + ty];
    for (int g = g0 + threadIdx.x; g < g1; g += NTH)
      acc[0] += (d.z[g] + a * d.dz[g]) * (d.s[g] + a * d.ds[g]);
  }
  const int fields[1] = {F_TAU_NUM};
  block_reduce_store<1, NTH>(acc, d.S, d.B, fields, i);
}
__global__ void k_bt_central(Dev d, InstConst ic) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || !d.active[i]) return;
  double a = SF(d, F_ALPHA, i);
  double cc = ic.degree[i] + 1;
  double ct = SF(d, F_TAU, i) + a * SF(d, F_STEP_TAU, i);
  double ck = SF(d, F_KAPPA, i) + a * SF(d, F_STEP_KAPPA, i);
  double mu = (SF(d, F_TAU_NUM, i) + ct * ck) / cc;
  SF(d, F_BARRIER, i) = cc * logsafe(mu) - logsafe(ct) - logsafe(ck);
}
__global__ void k_bt_check(Dev d, double step) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || !d.active[i]) return;
  if (SF(d, F_BARRIER, i) < 1.0) {
    IF(d, I_BT_ACTIVE, i) = 0;
  } else {
    SF(d, F_ALPHA, i) *= step;
    atomicAdd(d.counter + 1, 1);
  }
}

// _strategy_checkpoint_small_step (solver.jl:560-573)
__global__ void k_check_small_step(Dev d, InstConst ic, SettingsDev st) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || !d.active[i]) return;
  double a = SF(d, F_ALPHA, i);
  if (!ic.sym[i] && IF(d, I_SCALING, i) == 0 && a < st.min_switch) {
    IF(d, I_SCALING, i) = 1;
    SF(d, F_ALPHA, i) = 0.0;
    IF(d, I_SKIP, i) = 1;
  } else if (a <= fmax(0.0, st.min_terminate)) {
    IF(d, I_STATUS, i) = ST_INSUFFICIENT_PROGRESS;
    SF(d, F_ALPHA, i) = 0.0;
    IF(d, I_DONE, i) = 1;
  }
}

// info_save_prev_iterate + variables_add_step! (solver.jl:389-391)
__global__ void k_add_step(Dev d) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < d.nx) {
    int inst = d.col_inst[t];
    if (d.active[inst]) {
      double a = SF(d, F_ALPHA, inst);
      d.px[t] = d.x[t];
      d.x[t] += a * d.dx[t];
    }
  }
  if (t < d.mz) {
    int inst = d.row_inst[t];
    if (d.active[inst]) {
      double a = SF(d, F_ALPHA, inst);
      d.ps[t] = d.s[t];
      d.pz[t] = d.z[t];
      d.s[t] += a * d.ds[t];
      d.z[t] += a * d.dz[t];
    }
  }
}
__global__ void k_add_step_scalars(Dev d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || !d.active[i]) return;
  SF(d, F_PREV_COST_P, i) = SF(d, F_COST_P, i);
  SF(d, F_PREV_COST_D, i) = SF(d, F_COST_D, i);
  SF(d, F_PREV_RES_P, i) = SF(d, F_RES_P, i);
  SF(d, F_PREV_RES_D, i) = SF(d, F_RES_D, i);
  SF(d, F_PREV_GAP_ABS, i) = SF(d, F_GAP_ABS, i);
  SF(d, F_PREV_GAP_REL, i) = SF(d, F_GAP_REL, i);
  SF(d, F_PREV_TAU, i) = SF(d, F_TAU, i);
  SF(d, F_PREV_KAPPA, i) = SF(d, F_KAPPA, i);
  double a = SF(d, F_ALPHA, i);
  SF(d, F_TAU, i) += a * SF(d, F_STEP_TAU, i);
  SF(d, F_KAPPA, i) += a * SF(d, F_STEP_KAPPA, i);
}
__global__ void k_count_running(Dev d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B) return;
  if (IF(d, I_DONE, i) == 0) {
    IF(d, I_SKIP, i) = 0;
    atomicAdd(d.counter, 1);
  }
}

// ============================================================ post-process
// info_post_process! + solution_post_process! + variables_unscale!
// (info.jl:275-291, solution.jl:2-50, variables.jl:373-403)
__global__ void k_post_status(Dev d, SettingsDev st, const int *sel) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B || (sel && !sel[i])) return;
  int s = IF(d, I_STATUS, i);
  if (s == ST_NUMERICAL_ERROR || s == ST_INSUFFICIENT_PROGRESS || s == ST_MAX_ITERATIONS ||
      s == ST_MAX_TIME)
    check_convergence(d, i, st.r_gap_abs, st.r_gap_rel, st.r_feas, st.r_infeas_abs,
                      st.r_infeas_rel, st.r_ktratio, ST_ALMOST_SOLVED,
                      ST_ALMOST_PRIMAL_INFEASIBLE, ST_ALMOST_DUAL_INFEASIBLE);
}
__device__ __forceinline__ bool status_infeasible(int s) {
  return s == ST_PRIMAL_INFEASIBLE || s == ST_DUAL_INFEASIBLE ||
         s == ST_ALMOST_PRIMAL_INFEASIBLE || s == ST_ALMOST_DUAL_INFEASIBLE;
}
// out_x: instance-concatenated; out_s/out_z: instance-concatenated in user row
// order, zmap[k] = global type-major row of output slot k
__global__ void k_unscale(Dev d, const int *zmap, const int *zinst, double *ox, double *os,
                          double *oz, const int *sel) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < d.nx && !(sel && !sel[d.col_inst[t]])) {
    int inst = d.col_inst[t];
    int s = IF(d, I_STATUS, inst);
    double sinv = status_infeasible(s) ? 1.0 / SF(d, F_KAPPA, inst) : 1.0 / SF(d, F_TAU, inst);
    ox[t] = d.x[t] * d.d[t] * sinv;
  }
  if (t < d.mz && !(sel && !sel[zinst[t]])) {
    int g = zmap[t];
    int inst = zinst[t];
    int s = IF(d, I_STATUS, inst);
    double sinv = status_infeasible(s) ? 1.0 / SF(d, F_KAPPA, inst) : 1.0 / SF(d, F_TAU, inst);
    double c = SF(d, F_EQ_C, inst);
    oz[t] = d.z[g] * d.e[g] * (sinv / c);
    os[t] = d.s[g] * d.einv[g] * sinv;
  }
}

}  // namespace clgpu

// ====================================================================== host
using namespace clgpu;

struct clgpu_solver {
  clgpu_settings st{};
  int B = 0, nx = 0, mz = 0;
  bool mixed = false;    // factor stored in FP32
  bool arith32 = false;  // and eliminated in FP32 arithmetic
  DevArena arena;
  Dev dv{};
  ConeSet cs{};
  KKTMapDev map{};
  KKTDev kk{};
  LDLParams lp{};
  SettingsDev sd{};
  InstConst ic{};
  int *d_reset = nullptr;
  double *d_c = nullptr, *d_normq = nullptr, *d_normb = nullptr;
  int *d_pnnz = nullptr;
  int *d_zmap = nullptr, *d_zinst = nullptr, *d_moff = nullptr;
  double *d_out = nullptr;  // nx + 2*mz
  int *h_counter = nullptr;  // pinned
  std::vector<int> h_n, h_m, h_xoff, h_moff;
  bool any_asym = false, any_sym = false;
  long long kkt_nnz = 0;              // stored KKT entries over all instances
  bool any_sn = false;                // class-3 (supernodal) instances present
  std::unique_ptr<SnExec> sn;         // their factorisation
  std::vector<clgpu_info> info;
  double *h_sol = nullptr;  // pinned host copy of x, s, z (concatenated), nx + 2*mz
  bool solved = false;
  long long launches = 0;
  bool profiling = false;
  // per-phase device time of the last solve (ms): factor, one-side ldl
  // solves, KKT refresh, residual kernels, update_scaling alone, two-side ldl
  // solves
  static constexpr int kPhases = 6;
  double prof[kPhases] = {0, 0, 0, 0, 0, 0};
  long long prof_calls[kPhases] = {0, 0, 0, 0, 0, 0};
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<int, int>>> ev_marks;  // class, (ev begin, ev end)
  size_t ev_next = 0;
  int prof_open = -1, prof_open_ev = -1;
  int passes = 0;
  double last_ms = 0;
  double *d_prof_bytes = nullptr;  // [3B] algorithmic bytes (profiling)
  // update_data!: maps from the caller's value arrays to the device copies,
  // and staging buffers for the new values
  bool upd_ok = false;
  long long upd_np = 0, upd_na = 0;
  std::vector<long long> h_pu_off;
  int4 *d_upd_pmap = nullptr, *d_upd_amap = nullptr;
  int2 *d_upd_pxy = nullptr, *d_upd_axy = nullptr;
  double *d_in_P = nullptr, *d_in_A = nullptr, *d_in_q = nullptr, *d_in_b = nullptr;
  double prof_bytes[3] = {0, 0, 0};  // factor, one-side, two-side solves (last profiled solve)
  // serving (continuous batching): instances are slots; mask_sel restricts
  // the masks to the slots being started; d_run flags the running slots;
  // d_list / h_list carry slot lists; slot_state: 0 idle, 1 running, 2
  // finished (awaiting collect)
  // Admissions run on their own stream (st_admit) through views (dv_admit,
  // cs_admit) whose active mask is separate, overlapping the running pass;
  // an admitted batch joins at the step after the one it was admitted
  // before (fresh -> aged -> activated), so it never joins a pass midway.
  const int *mask_sel = nullptr;
  int *d_sel = nullptr, *d_sel_admit = nullptr, *d_run = nullptr, *d_active_admit = nullptr;
  int *d_list = nullptr, *d_list_admit = nullptr, *d_list_collect = nullptr,
      *d_list_act = nullptr;
  int *h_list = nullptr, *h_list_admit = nullptr, *h_list_collect = nullptr,
      *h_list_act = nullptr;
  double *d_info = nullptr, *h_info = nullptr, *h_stage = nullptr;
  bool serving = false;
  // the pass as a CUDA graph (index 1: with the serving finished-list)
  bool use_graphs = true;
  int solves_done = 0;  // completed clgpu_solver_solve calls
  cudaGraphExec_t pass_exec[2] = {nullptr, nullptr};
  long long pass_launches = 0;
  Dev dv_admit{};
  ConeSet cs_admit{};
  cudaStream_t st_admit = nullptr;
  cudaEvent_t ev_admit[2] = {nullptr, nullptr};  // alternate between admissions
  int ev_fresh = 0, ev_aged = 0;                 // event of the fresh / aged batch
  std::vector<int> fresh, aged;  // admitted slots awaiting activation
  std::vector<int> slot_state;   // 0 idle, 1 running, 2 finished, 3 admitted
  std::vector<std::chrono::steady_clock::time_point> slot_t0;
  ~clgpu_solver() {
    for (auto ex : pass_exec)
      if (ex) cudaGraphExecDestroy(ex);
    if (h_counter) pinned_give(h_counter);
    if (st_admit) {
      cudaStreamSynchronize(st_admit);
      cudaStreamDestroy(st_admit);
    }
    for (auto ev : ev_admit)
      if (ev) cudaEventDestroy(ev);
    for (int *p : {h_list, h_list_admit, h_list_collect, h_list_act})
      if (p) pinned_give(p);
    if (h_info) pinned_give(h_info);
    if (h_stage) pinned_give(h_stage);
    if (h_sol) pinned_give(h_sol);
    for (auto e : ev_pool) cudaEventDestroy(e);
  }
  int next_event() {
    if (ev_next == ev_pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      ev_pool.push_back(e);
    }
    return (int)ev_next++;
  }
  void prof_begin(int cls, cudaStream_t st) {
    if (!profiling) return;
    int e = next_event();
    cudaEventRecord(ev_pool[e], st);
    prof_open = cls;
    prof_open_ev = e;
  }
  void prof_end(cudaStream_t st) {
    if (!profiling || prof_open < 0) return;
    int e = next_event();
    cudaEventRecord(ev_pool[e], st);
    ev_marks.push_back({prof_open, {prof_open_ev, e}});
    prof_open = -1;
  }
  void prof_collect() {
    if (d_prof_bytes) {
      std::vector<double> hb(3 * (size_t)B);
      cudaMemcpy(hb.data(), d_prof_bytes, hb.size() * sizeof(double), cudaMemcpyDeviceToHost);
      for (int c = 0; c < 3; ++c) {
        prof_bytes[c] = 0;
        for (int i = 0; i < B; ++i) prof_bytes[c] += hb[(size_t)c * B + i];
      }
    }
    for (int c = 0; c < kPhases; ++c) {
      prof[c] = 0;
      prof_calls[c] = 0;
    }
    for (auto &m : ev_marks) {
      float ms = 0;
      cudaEventElapsedTime(&ms, ev_pool[m.second.first], ev_pool[m.second.second]);
      prof[m.first] += ms;
      prof_calls[m.first] += 1;
    }
    ev_marks.clear();
    ev_next = 0;
  }
};

static SettingsDev make_sd(const clgpu_settings &s) {
  SettingsDev d;
  d.max_iter = s.max_iter;
  d.time_limit = s.time_limit;
  d.max_step_fraction = s.max_step_fraction;
  d.tol_gap_abs = s.tol_gap_abs;
  d.tol_gap_rel = s.tol_gap_rel;
  d.tol_feas = s.tol_feas;
  d.tol_infeas_abs = s.tol_infeas_abs;
  d.tol_infeas_rel = s.tol_infeas_rel;
  d.tol_ktratio = s.tol_ktratio;
  d.r_gap_abs = s.reduced_tol_gap_abs;
  d.r_gap_rel = s.reduced_tol_gap_rel;
  d.r_feas = s.reduced_tol_feas;
  d.r_infeas_abs = s.reduced_tol_infeas_abs;
  d.r_infeas_rel = s.reduced_tol_infeas_rel;
  d.r_ktratio = s.reduced_tol_ktratio;
  d.bt_step = s.linesearch_backtrack_step;
  d.min_switch = s.min_switch_step_length;
  d.min_terminate = s.min_terminate_step_length;
  return d;
}

extern "C" int clgpu_default_settings(clgpu_settings *s) {
  if (!s) return -1;
  std::memset(s, 0, sizeof(*s));
  s->max_iter = 200;
  s->time_limit = INFINITY;
  s->max_step_fraction = 0.99;
  s->tol_gap_abs = 1e-8;
  s->tol_gap_rel = 1e-8;
  s->tol_feas = 1e-8;
  s->tol_infeas_abs = 1e-8;
  s->tol_infeas_rel = 1e-8;
  s->tol_ktratio = 1e-6;
  s->reduced_tol_gap_abs = 5e-5;
  s->reduced_tol_gap_rel = 5e-5;
  s->reduced_tol_feas = 1e-4;
  s->reduced_tol_infeas_abs = 5e-12;
  s->reduced_tol_infeas_rel = 5e-5;
  s->reduced_tol_ktratio = 1e-4;
  s->equilibrate_enable = 1;
  s->equilibrate_max_iter = 10;
  s->equilibrate_min_scaling = 1e-4;
  s->equilibrate_max_scaling = 1e4;
  s->linesearch_backtrack_step = 0.8;
  s->min_switch_step_length = 1e-2;
  s->min_terminate_step_length = 1e-4;
  s->static_regularization_enable = 1;
  s->static_regularization_constant = 1e-8;
  s->static_regularization_proportional = kDEps * kDEps;
  s->dynamic_regularization_enable = 1;
  s->dynamic_regularization_eps = 1e-13;
  s->dynamic_regularization_delta = 2e-7;
  s->iterative_refinement_enable = 1;
  s->iterative_refinement_reltol = 1e-12;
  s->iterative_refinement_abstol = 1e-12;
  s->iterative_refinement_max_iter = 10;
  s->iterative_refinement_stop_ratio = 5;
  s->direct_solve_method = CLGPU_METHOD_FP64;
  s->soc_threshold = 5;
  s->verbose = 0;
  s->setup_threads = 0;
  s->fused_solves = 1;
  s->device_setup = 1;
  s->autotune = 1;
  return 0;
}

// Builds every device structure of a batch from prepared instances.
// Runs f(i) for i in [0, n) on nth host threads (blocks of 16 indices).
template <class F>
static void par_for(int n, int nth, F f) {
  if (nth <= 1 || n < 64) {
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<int> next{0};
  std::vector<std::thread> th;
  for (int t = 0; t < nth; ++t)
    th.emplace_back([&]() {
      for (int i0; (i0 = next.fetch_add(16)) < n;)
        for (int i = i0; i < std::min(n, i0 + 16); ++i) f(i);
    });
  for (auto &t : th) t.join();
}

// Exclusive prefix sum of counts[0..n) into off[0..n] (off[n] = total).
template <class T>
static std::vector<long long> prefix(const std::vector<T> &counts) {
  std::vector<long long> off(counts.size() + 1, 0);
  for (size_t i = 0; i < counts.size(); ++i) off[i + 1] = off[i] + (long long)counts[i];
  return off;
}

// Concatenates the prepared instances into the batch layout and uploads it.
// Every per-instance copy runs on nth host threads: offsets first (prefix
// sums over instances), then each instance fills its own disjoint slices.
// First-fit-decreasing packing of instances into blocks of `slots` warps:
// items in decreasing order of need (stable), each placed in the first block
// with a free slot and room for it; a block's needs sum to at most cap.
// pinst / poff receive per slot the instance (-1: idle) and its byte offset in
// the block's shared memory.  Returns the number of blocks.
template <typename Need>
static int ffd_pack(std::vector<int> items, Need need, long long cap, int slots,
                    std::vector<int> &pinst, std::vector<int> &poff) {
  std::stable_sort(items.begin(), items.end(), [&](int a, int b) { return need(a) > need(b); });
  std::vector<long long> used;
  std::vector<int> cnt;
  pinst.clear();
  poff.clear();
  size_t first_open = 0;
  for (int i : items) {
    const long long s_i = need(i);
    size_t b = first_open;
    while (b < used.size() && (cnt[b] == slots || used[b] + s_i > cap)) ++b;
    if (b == used.size()) {
      used.push_back(0);
      cnt.push_back(0);
      for (int w = 0; w < slots; ++w) {
        pinst.push_back(-1);
        poff.push_back(0);
      }
    }
    pinst[(size_t)slots * b + cnt[b]] = i;
    poff[(size_t)slots * b + cnt[b]] = (int)used[b];
    used[b] += s_i;
    ++cnt[b];
    while (first_open < used.size() &&
           (cnt[first_open] == slots || used[first_open] + need(items.back()) > cap))
      ++first_open;
  }
  return (int)used.size();
}

// KKT position of every L entry (i, j), i > j, in the instance's permuted
// full CSR (rows sorted, pattern symmetric), offset by kb; -1 when K has no
// such entry.  Walking the rows r in order meets the entries (c, r) of each
// row c in increasing r, so tpos[t] (the position of entry t's transpose) is
// one pass with a cursor per row; row j scattered into a stamped map then
// gives (j, i), and tpos its transpose (i, j).  Linear in nnz(K) + nnz(L).
struct FactorOpScratch {
  std::vector<int4> lev;
  std::vector<int> nodes, cnt, segs, rowpos, rowstamp, tpos, cur;
  std::vector<int> wch[kFactorWarps];
  int stamp = 0;
  void fit(int n, int nk) {
    if ((int)rowpos.size() < n) {
      rowpos.resize(n);
      rowstamp.assign(n, 0);
      cur.resize(n);
      stamp = 0;
    }
    if ((int)tpos.size() < nk) tpos.resize(nk);
  }
};

static void l_kkt_positions(const Prepared &p, long long kb, int *Lkpos, FactorOpScratch &sc) {
  const int Ni = p.N;
  sc.fit(Ni, (int)p.Kj.size());
  int *rowpos = sc.rowpos.data(), *rowstamp = sc.rowstamp.data();
  int *tpos = sc.tpos.data(), *cur = sc.cur.data();
  for (int r = 0; r < Ni; ++r) cur[r] = p.Kp[r];
  for (int r = 0; r < Ni; ++r)
    for (int t = p.Kp[r]; t < p.Kp[r + 1]; ++t) tpos[t] = cur[p.Kj[t]]++;
  for (int j = 0; j < Ni; ++j) {
    const int st = ++sc.stamp;
    for (int t = p.Kp[j]; t < p.Kp[j + 1]; ++t) {
      rowpos[p.Kj[t]] = t;
      rowstamp[p.Kj[t]] = st;
    }
    for (int q = p.Lp[j]; q < p.Lp[j + 1]; ++q) {
      const int r = p.Li[q];
      Lkpos[q] = rowstamp[r] == st ? (int)(kb + tpos[rowpos[r]]) : -1;
    }
  }
}

// Number of ops of the instance's streamed factorisation: one per (j, k)
// pair of its row structure and per entry of L(:,k) below row j, and one
// pivot per column.
static long long factor_op_count(const Prepared &p) {
  long long t = p.N;
  for (size_t r = 0; r < p.Rk.size(); ++r) t += p.Lp[p.Rk[r] + 1] - p.Rpos[r];
  return t;
}

// The streamed factorisation's ops of one instance, written to op (exactly
// factor_op_count(p) of them), level by level:
//  - the level's updates grouped by target (a segment per target), targets
//    increasing: first the diagonal targets j (update d_j -= U(j,k)^2 / d_k,
//    {j, Ni + pjk, Ni + pjk, k}), then the column targets Ni + q (update
//    L(i,j) -= L(i,k) U(j,k), {Ni + q, Ni + pp, Ni + pjk, k}); a segment keeps
//    its ops in generation order (the pairs (j, k) in row-structure order);
//  - split into kFactorWarps parts of about equal length at segment starts,
//    each op's .w or'd with min(position in segment, kPosMax) << 16 and the
//    last-of-segment bit, each part cut into chunk words;
//  - then the level's pivots (t = j, a = sign + 1) in kFactorWarps contiguous
//    parts.
// Each op is packed into 8 bytes (fop_pack).
// The column ranges of L follow the node order, so sorting the level's nodes
// and bucketing each column by q (counting sort) lists the groups in target
// order without a comparison sort.  Returns false when the structure of
// L(:,k) below j is not inside L(:,j) (not reached for a valid symbolic
// factorisation) or a part's chunk count leaves its 16-bit field.
static bool build_factor_ops(const Prepared &p, uint2 *op, int *flcnt, std::vector<int> &chk,
                             std::array<int, kFactorWarps + 1> &woff, FactorOpScratch &sc) {
  constexpr int W = kFactorWarps;
  const int Ni = p.N;
  const int nl = (int)p.lvl_ptr.size() - 1;
  const int *lp = p.lvl_ptr.data();
  sc.fit(Ni, 0);
  int *rowpos = sc.rowpos.data(), *rowstamp = sc.rowstamp.data();
  auto &lev = sc.lev;
  auto &nodes = sc.nodes;
  auto &cnt = sc.cnt;
  auto &segs = sc.segs;
  for (int w = 0; w < W; ++w) sc.wch[w].clear();
  long long nops = 0;
  bool bad = false;
  auto put_chunks = [&](int w, long long c0, long long c1, bool pivot) {
    int n = 0;
    for (long long c = c0; c < c1; c += kChunk, ++n) {
      const int cn = (int)std::min<long long>(kChunk, c1 - c);
      const int steps =
          pivot ? 0 : chunk_scan_steps<2>(cn, [&](int e) { return fop_pos(op[c + e]); });
      sc.wch[w].push_back((int)(c | ((long long)steps << kStepShift) |
                                ((long long)(cn - 1) << kCntShift) |
                                (pivot ? (long long)1 << 31 : 0LL)));
    }
    return n;
  };
  for (int l = 0; l < nl && !bad; ++l) {
    nodes.assign(p.lvl_nodes.begin() + lp[l], p.lvl_nodes.begin() + lp[l + 1]);
    std::sort(nodes.begin(), nodes.end());
    size_t nlev = 0;
    for (int j : nodes)
      for (int r = p.Rp[j]; r < p.Rp[j + 1]; ++r) nlev += p.Lp[p.Rk[r] + 1] - p.Rpos[r];
    if (lev.size() < nlev) lev.resize(nlev);
    segs.clear();
    int f = 0;
    for (int j : nodes) {
      if (p.Rp[j + 1] > p.Rp[j]) segs.push_back(f);
      for (int r = p.Rp[j]; r < p.Rp[j + 1]; ++r) {
        const int pjk = p.Rpos[r];
        lev[f++] = make_int4(j, Ni + pjk, Ni + pjk, p.Rk[r]);
      }
    }
    for (int j : nodes) {
      if (p.Rp[j + 1] == p.Rp[j]) continue;
      const int q0 = p.Lp[j], qe = p.Lp[j + 1], len = qe - q0;
      if ((int)cnt.size() < len + 1) cnt.resize(len + 1);
      std::fill(cnt.begin(), cnt.begin() + len + 1, 0);
      const int st = ++sc.stamp;
      for (int q = q0; q < qe; ++q) {
        rowpos[p.Li[q]] = q - q0;
        rowstamp[p.Li[q]] = st;
      }
      for (int r = p.Rp[j]; r < p.Rp[j + 1] && !bad; ++r) {
        const int k = p.Rk[r];
        for (int pp = p.Rpos[r] + 1; pp < p.Lp[k + 1]; ++pp) {
          const int row = p.Li[pp];
          if (rowstamp[row] != st) {
            bad = true;
            break;
          }
          cnt[rowpos[row] + 1]++;
        }
      }
      if (bad) break;
      for (int a = 0; a < len; ++a) {
        if (cnt[a + 1]) segs.push_back(f + cnt[a]);
        cnt[a + 1] += cnt[a];
      }
      for (int r = p.Rp[j]; r < p.Rp[j + 1]; ++r) {
        const int k = p.Rk[r], pjk = p.Rpos[r];
        for (int pp = pjk + 1; pp < p.Lp[k + 1]; ++pp) {
          const int a = rowpos[p.Li[pp]];
          lev[f + cnt[a]++] = make_int4(Ni + q0 + a, Ni + pp, Ni + pjk, k);
        }
      }
      f += cnt[len - 1];  // bucket ends after placement
    }
    if (bad) break;
    const int nseg = (int)segs.size();
    segs.push_back(f);
    int sb[W + 1];
    sb[0] = 0;
    sb[W] = nseg;
    for (int w = 1; w < W; ++w) {
      const int ideal = (int)((size_t)f * w / W);
      const int g = (int)(std::lower_bound(segs.begin(), segs.end(), ideal) - segs.begin());
      sb[w] = std::min(nseg, std::max(sb[w - 1], g));
    }
    int nop[W], npv[W];
    for (int w = 0; w < W; ++w) {
      const long long start = nops;
      for (int g = sb[w]; g < sb[w + 1]; ++g) {
        const int s0 = segs[g], s1 = segs[g + 1];
        for (int t = s0; t < s1; ++t) {
          const int4 o4 = lev[t];
          op[nops++] = fop_pack(o4.x, o4.y, o4.z, o4.w, std::min(t - s0, kPosMax),
                                t == s1 - 1 ? 1 : 0);
        }
      }
      nop[w] = put_chunks(w, start, nops, false);
    }
    const int np = lp[l + 1] - lp[l];
    for (int w = 0; w < W; ++w) {
      const long long start = nops;
      for (int t = lp[l] + np * w / W; t < lp[l] + np * (w + 1) / W; ++t) {
        const int j = p.lvl_nodes[t];
        op[nops++] = fop_pack(j, (int)p.Dsign[j] + 1, 0, 0, 0, 0);
      }
      npv[w] = put_chunks(w, start, nops, true);
    }
    for (int w = 0; w < W; ++w) {
      if (nop[w] > 0xffff || npv[w] > 0xffff) bad = true;
      flcnt[(size_t)l * W + w] = nop[w] | (npv[w] << 16);
    }
  }
  chk.clear();
  woff[0] = 0;
  for (int w = 0; w < W; ++w) {
    chk.insert(chk.end(), sc.wch[w].begin(), sc.wch[w].end());
    woff[w + 1] = (int)chk.size();
  }
  return !bad;
}

static int build_batch(clgpu_solver *h, std::vector<Prepared> &prep, int nth) {
  DevArena &A = h->arena;
  const int B = (int)prep.size();
  h->B = B;
  auto tmark = std::chrono::steady_clock::now();
  auto mark = [&](const char *what) {  // setup timing, printed when verbose
    if (!h->st.verbose) return;
    auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "clgpu setup: %-22s %8.1f ms\n", what,
                 std::chrono::duration<double, std::milli>(now - tmark).count());
    tmark = now;
  };
  // ---------------- sizes and offsets
  std::vector<int> xoff(B + 1, 0), moff(B + 1, 0);
  for (int i = 0; i < B; ++i) {
    xoff[i + 1] = xoff[i] + prep[i].n;
    moff[i + 1] = moff[i] + prep[i].m;
  }
  const int nx = xoff[B], mz = moff[B];
  h->nx = nx;
  h->mz = mz;
  h->h_xoff = xoff;
  h->h_moff = moff;
  // type-major global rows: instance i's rows of type t start at tcur[6i+t]
  std::vector<long long> type_total(6, 0);
  for (auto &p : prep)
    for (int t = 0; t < 6; ++t) type_total[t] += p.type_rows[t];
  std::vector<int> type_begin(7, 0);
  for (int t = 0; t < 6; ++t) type_begin[t + 1] = type_begin[t] + (int)type_total[t];
  std::vector<int> tcur(6 * (size_t)B);
  {
    std::vector<int> cursor(type_begin.begin(), type_begin.end() - 1);
    for (int i = 0; i < B; ++i)
      for (int t = 0; t < 6; ++t) {
        tcur[6 * i + t] = cursor[t];
        cursor[t] += prep[i].type_rows[t];
      }
  }
  std::vector<std::vector<int>> grow(B);  // local type-major row -> global row
  std::vector<int> row_inst(mz), col_inst(nx);
  par_for(B, nth, [&](int i) {
    auto &p = prep[i];
    grow[i].resize(p.m);
    int lr = 0;
    for (int t = 0; t < 6; ++t)
      for (int k = 0; k < p.type_rows[t]; ++k) grow[i][lr++] = tcur[6 * i + t] + k;
    for (int g : grow[i]) row_inst[g] = i;
    for (int j = xoff[i]; j < xoff[i + 1]; ++j) col_inst[j] = i;
  });
  // ---------------- problem data in global CSR form
  std::vector<long long> pcnt(B), acnt(B);
  for (int i = 0; i < B; ++i) {
    pcnt[i] = prep[i].Pfull.p[prep[i].n];
    acnt[i] = prep[i].A.p[prep[i].n];
  }
  const auto poffs = prefix(pcnt), aoffs = prefix(acnt);
  if (poffs[B] > 2000000000LL || aoffs[B] > 2000000000LL) return -4;
  std::vector<int> Pp(nx + 1, 0), Ap(mz + 1, 0), Atp(nx + 1, 0);
  hvec<int> Pj(poffs[B]), Aj(aoffs[B]), Atj(aoffs[B]);
  hvec<double> Pxv(poffs[B]), Axv(aoffs[B]), Atxv(aoffs[B]), q(nx), negq(nx), b(mz), dd(nx),
      ddinv(nx), ee(mz), eeinv(mz);
  std::vector<int> arow_cnt(mz, 0);
  par_for(B, nth, [&](int i) {
    auto &p = prep[i];
    // P: full symmetric CSC == CSR by symmetry
    const long long pb = poffs[i];
    for (int j = 0; j < p.n; ++j) {
      for (int k = p.Pfull.p[j]; k < p.Pfull.p[j + 1]; ++k) {
        Pj[pb + k] = xoff[i] + p.Pfull.i[k];
        Pxv[pb + k] = p.Pfull.x[k];
      }
      Pp[xoff[i] + j + 1] = (int)(pb + p.Pfull.p[j + 1]);
      q[xoff[i] + j] = p.q[j];
      negq[xoff[i] + j] = -p.q[j];
      dd[xoff[i] + j] = p.d[j];
      ddinv[xoff[i] + j] = 1.0 / p.d[j];
    }
    // A^T rows = A columns (CSC of A), column indices = global rows
    std::vector<int> local_of_user(p.m);
    for (int lr = 0; lr < p.m; ++lr) local_of_user[p.user_row_of[lr]] = lr;
    const long long ab = aoffs[i];
    for (int j = 0; j < p.n; ++j) {
      for (int k = p.A.p[j]; k < p.A.p[j + 1]; ++k) {
        const int g = grow[i][local_of_user[p.A.i[k]]];
        Atj[ab + k] = g;
        Atxv[ab + k] = p.A.x[k];
        arow_cnt[g]++;  // rows belong to this instance only
      }
      Atp[xoff[i] + j + 1] = (int)(ab + p.A.p[j + 1]);
    }
    for (int lr = 0; lr < p.m; ++lr) {
      const int g = grow[i][lr], ur = p.user_row_of[lr];
      b[g] = p.b[ur];
      ee[g] = p.e[ur];
      eeinv[g] = 1.0 / p.e[ur];
    }
  });
  // A rows (global, type-major order) from A^T, columns ascending per row
  for (int g = 0; g < mz; ++g) Ap[g + 1] = Ap[g] + arow_cnt[g];
  hvec<int> acsr(aoffs[B]);  // A CSR position of every A^T (= caller CSC) entry
  {
    std::vector<int> next(Ap.begin(), Ap.end() - 1);
    par_for(B, nth, [&](int i) {  // an instance touches only its own rows
      for (int j = xoff[i]; j < xoff[i + 1]; ++j)
        for (int k = Atp[j]; k < Atp[j + 1]; ++k) {
          const int qd = next[Atj[k]]++;
          Aj[qd] = j;
          Axv[qd] = Atxv[k];
          acsr[k] = qd;
        }
    });
  }
  // ---------------- per-instance constants
  std::vector<double> c(B), nq(B), nb(B);
  std::vector<int> pnnz(B), deg(B), sym(B);
  for (int i = 0; i < B; ++i) {
    c[i] = prep[i].c;
    nq[i] = prep[i].normq;
    nb[i] = prep[i].normb;
    pnnz[i] = prep[i].p_nnz > 0 ? 1 : 0;
    deg[i] = prep[i].degree;
    sym[i] = prep[i].symmetric ? 1 : 0;
    if (sym[i]) h->any_sym = true; else h->any_asym = true;
  }
  // ---------------- cones (type lists, instance by instance)
  ConeSet &cs = h->cs;
  cs.B = B;
  cs.m_total = mz;
  cs.zero_begin = type_begin[0];
  cs.n_zero = (int)type_total[0];
  cs.nn_begin = type_begin[1];
  cs.n_nn = (int)type_total[1];
  cs.soc_begin = type_begin[2];
  cs.soc_rows = (int)type_total[2];
  cs.exp_begin = type_begin[3];
  cs.pow_begin = type_begin[4];
  cs.psd_begin = type_begin[5];
  std::vector<int> nsoc(B), nexp(B), npow(B), npsd(B);
  int soc_maxdim = 0, psd_nmax = 0;
  for (int i = 0; i < B; ++i) {
    nsoc[i] = prep[i].type_cones[2];
    nexp[i] = prep[i].type_cones[3];
    npow[i] = prep[i].type_cones[4];
    npsd[i] = prep[i].type_cones[5];
    for (size_t k = 0; k < prep[i].ctype.size(); ++k) {
      if (prep[i].ctype[k] == CLGPU_CONE_SOC) soc_maxdim = std::max(soc_maxdim, prep[i].cdim[k]);
      if (prep[i].ctype[k] == CLGPU_CONE_PSD) psd_nmax = std::max(psd_nmax, prep[i].cdim[k]);
    }
  }
  if (psd_nmax > kPsdMaxSide) return -3;  // warp-per-cone kernels, matrices in shared memory
  const auto osoc = prefix(nsoc), oexp = prefix(nexp), opow = prefix(npow), opsd = prefix(npsd);
  std::vector<int> soc_off(osoc[B]), soc_dim(osoc[B]), soc_inst(osoc[B]), soc_sparse(osoc[B]),
      exp_inst(oexp[B]), pow_inst(opow[B]), psd_off(opsd[B]), psd_n(opsd[B]), psd_inst(opsd[B]);
  std::vector<double> pow_alpha(opow[B]);
  par_for(B, nth, [&](int i) {
    auto &p = prep[i];
    long long a = osoc[i], e = oexp[i], w = opow[i], s = opsd[i];
    for (size_t k = 0; k < p.ctype.size(); ++k) {
      const int t = p.ctype[k], g = p.m ? grow[i][p.cstart[k]] : 0;
      if (t == CLGPU_CONE_SOC) {
        soc_off[a] = g;
        soc_dim[a] = p.cdim[k];
        soc_inst[a] = i;
        soc_sparse[a] = p.cdim[k] > h->st.soc_threshold ? 1 : 0;
        ++a;
      } else if (t == CLGPU_CONE_EXP) {
        exp_inst[e++] = i;
      } else if (t == CLGPU_CONE_POW) {
        pow_inst[w] = i;
        pow_alpha[w++] = p.cparam[k];
      } else if (t == CLGPU_CONE_PSD) {
        psd_off[s] = g;
        psd_n[s] = p.cdim[k];
        psd_inst[s++] = i;
      }
    }
  });
  cs.n_soc = (int)osoc[B];
  cs.n_exp = (int)oexp[B];
  cs.n_pow = (int)opow[B];
  cs.n_psd = (int)opsd[B];
  int G = 2;
  while (G < soc_maxdim && G < 32) G <<= 1;
  cs.soc_group = G;
  cs.psd_nmax = std::max(psd_nmax, 1);
  {
    // per-instance ranges of each cone type (cones are stored instance by
    // instance inside each type list)
    std::vector<int> rnn(2 * (size_t)B), rsoc(2 * (size_t)B), rexp(2 * (size_t)B),
        rpow(2 * (size_t)B), rpsd(2 * (size_t)B);
    for (int i = 0; i < B; ++i) {
      rnn[2 * i] = tcur[6 * i + 1] - type_begin[1];
      rnn[2 * i + 1] = prep[i].type_rows[1];
      rsoc[2 * i] = (int)osoc[i];
      rsoc[2 * i + 1] = nsoc[i];
      rexp[2 * i] = (int)oexp[i];
      rexp[2 * i + 1] = nexp[i];
      rpow[2 * i] = (int)opow[i];
      rpow[2 * i + 1] = npow[i];
      rpsd[2 * i] = (int)opsd[i];
      rpsd[2 * i + 1] = npsd[i];
    }
    cs.rng_nn = A.upload(rnn);
    cs.rng_soc = A.upload(rsoc);
    cs.rng_exp = A.upload(rexp);
    cs.rng_pow = A.upload(rpow);
    cs.rng_psd = A.upload(rpsd);
  }
  cs.row_inst = A.upload(row_inst);
  cs.soc_off = A.upload(soc_off);
  cs.soc_dim = A.upload(soc_dim);
  cs.soc_inst = A.upload(soc_inst);
  cs.soc_sparse = A.upload(soc_sparse);
  {
    const int nsc = (int)soc_off.size();
    for (int v = 1; v <= kSocTileShapes; ++v) {
      std::vector<int> tiles =
          soc_tiles(soc_off.data(), soc_dim.data(), nsc, soc_tile_cones(v), soc_tile_rows(v));
      cs.soc_ntiles[v] = (int)tiles.size() / 2;
      cs.soc_tile[v] = A.upload(tiles);
    }
    cs.soc_ntiles[0] = 0;
    cs.soc_tile[0] = nullptr;
    cones_default_shapes(cs);
  }
  cs.exp_inst = A.upload(exp_inst);
  cs.pow_inst = A.upload(pow_inst);
  cs.pow_alpha = A.upload(pow_alpha);
  cs.psd_off = A.upload(psd_off);
  cs.psd_n = A.upload(psd_n);
  cs.psd_inst = A.upload(psd_inst);
  cs.nn_w = A.alloc<double>(cs.n_nn);
  cs.nn_lambda = A.alloc<double>(cs.n_nn);
  cs.soc_w = A.alloc<double>(cs.soc_rows);
  cs.soc_lambda = A.alloc<double>(cs.soc_rows);
  cs.soc_u = A.alloc<double>(cs.soc_rows);
  cs.soc_v = A.alloc<double>(cs.soc_rows);
  cs.soc_eta = A.alloc<double>(cs.n_soc);
  cs.soc_d = A.alloc<double>(cs.n_soc);
  cs.exp_Hd = A.alloc<double>(9 * (size_t)cs.n_exp);
  cs.exp_Hs = A.alloc<double>(9 * (size_t)cs.n_exp);
  cs.exp_grad = A.alloc<double>(3 * (size_t)cs.n_exp);
  cs.exp_z = A.alloc<double>(3 * (size_t)cs.n_exp);
  cs.pow_Hd = A.alloc<double>(9 * (size_t)cs.n_pow);
  cs.pow_Hs = A.alloc<double>(9 * (size_t)cs.n_pow);
  cs.pow_grad = A.alloc<double>(3 * (size_t)cs.n_pow);
  cs.pow_z = A.alloc<double>(3 * (size_t)cs.n_pow);
  size_t nn2 = (size_t)cs.psd_nmax * cs.psd_nmax;
  cs.psd_R = A.alloc<double>(nn2 * cs.n_psd);
  cs.psd_Rinv = A.alloc<double>(nn2 * cs.n_psd);
  cs.psd_lam = A.alloc<double>((size_t)cs.psd_nmax * cs.n_psd);
  cs.cone_tmp = A.alloc<double>((size_t)cs.n_soc + cs.n_exp + cs.n_pow + cs.n_psd);
  cs.cone_tmp2 = A.alloc<double>((size_t)cs.n_soc + cs.n_exp + cs.n_pow + cs.n_psd);
  mark("data + cones");
  // ---------------- KKT arrays (concatenate with global positions)
  std::vector<int> N(B), voff(B + 1, 0), poff(B, 0), nlev(B);
  std::vector<long long> kcnt(B), lcnt(B), lvcnt(B);
  for (int i = 0; i < B; ++i) {
    N[i] = prep[i].N;
    voff[i + 1] = voff[i] + N[i];
    poff[i] = voff[i] + i;
    kcnt[i] = (long long)prep[i].Kj.size();
    lcnt[i] = (long long)prep[i].Li.size();
    lvcnt[i] = (long long)prep[i].lvl_ptr.size();
    nlev[i] = (int)prep[i].lvl_ptr.size() - 1;
  }
  const auto kof = prefix(kcnt), lof = prefix(lcnt), lvof = prefix(lvcnt);
  const long long knz = kof[B], lnz = lof[B];
  if (knz > 2000000000LL || lnz > 2000000000LL) return -4;
  std::vector<int> lvl_off(B);
  for (int i = 0; i < B; ++i) lvl_off[i] = (int)lvof[i];
  const int VT = voff[B], PT = voff[B] + B;
  hvec<int> Kp(PT), Kj((size_t)knz), Kdiag(VT), Lp(PT), Li((size_t)lnz), Rp(PT), Rk((size_t)lnz),
      Rpos((size_t)lnz), gsrc(VT), lvl_ptr(lvof[B]), lvl_nodes(VT);
  hvec<double> Kx((size_t)knz);
  hvec<signed char> Dsign(VT);
  const int tsize = 8;  // work vectors are FP64 in both precision forms
  int max_small = 0;
  bool has_small = false, has_large = false;
  // kernel class: single warp when the work vector fits the shared-memory
  // budget and the streams fit the chunk-word offsets
  std::vector<int> cls(B);
  for (int i = 0; i < B; ++i) {
    const bool fits = (long long)N[i] * tsize <= 48 * 1024 &&
                      (long long)prep[i].Li.size() <= (long long)kStartMask &&
                      (long long)prep[i].Kj.size() <= (long long)kStartMask;
    cls[i] = prep[i].supernodal ? 3 : (fits ? 1 : 2);
    if (cls[i] == 3) {
      h->any_sn = true;
    } else if (fits) {
      has_small = true;
      max_small = std::max(max_small, N[i]);
    } else {
      has_large = true;
    }
  }
  par_for(B, nth, [&](int i) {
    auto &p = prep[i];
    const int n = p.n, m = p.m;
    const long long kb = kof[i], lb = lof[i];
    for (int r = 0; r <= N[i]; ++r) {
      Kp[poff[i] + r] = (int)(kb + p.Kp[r]);
      Lp[poff[i] + r] = (int)(lb + p.Lp[r]);
      Rp[poff[i] + r] = (int)(lb + p.Rp[r]);
    }
    std::copy(p.Kj.begin(), p.Kj.end(), Kj.begin() + kb);
    std::copy(p.Kx.begin(), p.Kx.end(), Kx.begin() + kb);
    std::copy(p.Li.begin(), p.Li.end(), Li.begin() + lb);
    std::copy(p.Rk.begin(), p.Rk.end(), Rk.begin() + lb);
    for (size_t k = 0; k < p.Rpos.size(); ++k) Rpos[lb + k] = (int)(lb + p.Rpos[k]);
    std::copy(p.lvl_ptr.begin(), p.lvl_ptr.end(), lvl_ptr.begin() + lvof[i]);
    std::copy(p.lvl_nodes.begin(), p.lvl_nodes.end(), lvl_nodes.begin() + voff[i]);
    for (int r = 0; r < N[i]; ++r) {
      Kdiag[voff[i] + r] = (int)(kb + p.Kdiag[r]);
      Dsign[voff[i] + r] = p.Dsign[r];
      const int o = p.perm[r];
      gsrc[voff[i] + r] = o < n ? xoff[i] + o : (o < n + m ? -grow[i][o - n] - 2 : -1);
    }
  });
  // refresh maps in global cone order (type lists, instance by instance)
  std::vector<long long> c_nn(B), c_sde(B), c_srow(B), c_exp(B), c_pow(B), c_pse(B);
  for (int i = 0; i < B; ++i) {
    auto &p = prep[i];
    c_nn[i] = (long long)p.nn_pos.size();
    c_srow[i] = (long long)p.socs_diag.size();
    c_exp[i] = (long long)p.exp_pos.size();
    c_pow[i] = (long long)p.pow_pos.size();
    long long de = 0, pe = 0;
    size_t sc = 0, pc = 0;
    for (size_t k = 0; k < p.ctype.size(); ++k) {
      if (p.ctype[k] == CLGPU_CONE_SOC) {
        if (p.socd_start[sc] >= 0) de += (long long)p.cdim[k] * (p.cdim[k] + 1) / 2;
        ++sc;
      } else if (p.ctype[k] == CLGPU_CONE_PSD) {
        const long long t = (long long)p.cdim[k] * (p.cdim[k] + 1) / 2;
        pe += t * (t + 1) / 2;
        ++pc;
      }
    }
    c_sde[i] = de;
    c_pse[i] = pe;
  }
  const auto o_nn = prefix(c_nn), o_sde = prefix(c_sde), o_srow = prefix(c_srow),
             o_exp = prefix(c_exp), o_pow = prefix(c_pow), o_pse = prefix(c_pse);
  std::vector<int> nn_pos(o_nn[B]), socd_off(osoc[B]), socd_pos(2 * o_sde[B]),
      socs_diag(o_srow[B]), socs_uv(4 * o_srow[B]), socs_D(2 * osoc[B]), exp_pos(o_exp[B]),
      pow_pos(o_pow[B]), psdo(opsd[B]), psd_pos(2 * o_pse[B]);
  par_for(B, nth, [&](int i) {
    auto &p = prep[i];
    const int kb = Kp[poff[i]];
    auto addk = [&](int v) { return v < 0 ? -1 : v + kb; };
    for (long long t = 0; t < c_nn[i]; ++t) nn_pos[o_nn[i] + t] = addk(p.nn_pos[t]);
    long long sc_g = osoc[i], de = o_sde[i];
    size_t sc = 0;
    for (size_t k = 0; k < p.ctype.size(); ++k) {
      if (p.ctype[k] != CLGPU_CONE_SOC) continue;
      const int st0 = p.socd_start[sc];
      if (st0 < 0) {
        socd_off[sc_g] = 0;
      } else {
        socd_off[sc_g] = (int)de;
        const int dim = p.cdim[k], t = dim * (dim + 1) / 2;
        for (int e2 = 0; e2 < t; ++e2) {
          socd_pos[2 * (de + e2)] = addk(p.socd_pos[2 * (st0 + e2)]);
          socd_pos[2 * (de + e2) + 1] = addk(p.socd_pos[2 * (st0 + e2) + 1]);
        }
        de += t;
      }
      socs_D[2 * sc_g] = addk(p.socs_D[2 * sc]);
      socs_D[2 * sc_g + 1] = addk(p.socs_D[2 * sc + 1]);
      ++sc;
      ++sc_g;
    }
    for (long long t = 0; t < c_srow[i]; ++t) socs_diag[o_srow[i] + t] = addk(p.socs_diag[t]);
    for (long long t = 0; t < 4 * c_srow[i]; ++t)
      socs_uv[4 * o_srow[i] + t] = addk(p.socs_uv[t]);
    for (long long t = 0; t < c_exp[i]; ++t) exp_pos[o_exp[i] + t] = addk(p.exp_pos[t]);
    for (long long t = 0; t < c_pow[i]; ++t) pow_pos[o_pow[i] + t] = addk(p.pow_pos[t]);
    long long pe = o_pse[i], pc_g = opsd[i];
    size_t pc = 0;
    for (size_t k = 0; k < p.ctype.size(); ++k) {
      if (p.ctype[k] != CLGPU_CONE_PSD) continue;
      const int st0 = p.psd_start[pc++];
      const long long t = (long long)p.cdim[k] * (p.cdim[k] + 1) / 2, tt = t * (t + 1) / 2;
      psdo[pc_g++] = (int)pe;
      for (long long e2 = 0; e2 < tt; ++e2) {
        psd_pos[2 * (pe + e2)] = addk(p.psd_pos[2 * (st0 + e2)]);
        psd_pos[2 * (pe + e2) + 1] = addk(p.psd_pos[2 * (st0 + e2) + 1]);
      }
      pe += tt;
    }
  });
  // value-update maps (update_data!): global positions
  {
    std::vector<long long> pu(B);
    bool upd = true;
    for (int i = 0; i < B; ++i) {
      pu[i] = prep[i].p_user_nnz;
      upd = upd && prep[i].updatable;
    }
    const auto opu = prefix(pu);
    hvec<int4> pmap(opu[B]), amap(aoffs[B]);
    hvec<int2> pxy(opu[B]), axy(aoffs[B]);
    par_for(B, nth, [&](int i) {
      const auto &p = prep[i];
      const int pb = (int)poffs[i], kb = (int)kof[i];
      auto g = [](int v, int base) { return v < 0 ? -1 : v + base; };
      for (long long t = 0; t < pu[i]; ++t) {
        const int *m4 = p.pmap.data() + 4 * t;
        pmap[opu[i] + t] = make_int4(g(m4[0], pb), g(m4[1], pb), g(m4[2], kb), g(m4[3], kb));
        const int r = p.pxy[2 * t], c = p.pxy[2 * t + 1];
        pxy[opu[i] + t] = r < 0 ? make_int2(-1, -1) : make_int2(xoff[i] + r, xoff[i] + c);
      }
      for (int j = 0; j < p.n; ++j)
        for (int k = p.A.p[j]; k < p.A.p[j + 1]; ++k) {
          const long long t = aoffs[i] + k;
          amap[t] = make_int4((int)t, acsr[t], g(p.amapk[2 * k], kb), g(p.amapk[2 * k + 1], kb));
          axy[t] = make_int2(Atj[t], xoff[i] + j);
        }
    });
    h->upd_ok = upd;
    h->upd_np = opu[B];
    h->upd_na = aoffs[B];
    h->h_pu_off.assign(opu.begin(), opu.end());
    h->d_upd_pmap = A.upload(pmap);
    h->d_upd_pxy = A.upload(pxy);
    h->d_upd_amap = A.upload(amap);
    h->d_upd_axy = A.upload(axy);
    h->d_in_P = A.alloc<double>(std::max<long long>(opu[B], 1), false);
    h->d_in_A = A.alloc<double>(std::max<long long>(aoffs[B], 1), false);
    h->d_in_q = A.alloc<double>(std::max(nx, 1), false);
    h->d_in_b = A.alloc<double>(std::max(mz, 1), false);
  }
  mark("kkt concat + maps");
  KKTMapDev &mp = h->map;
  mp.nn_pos = A.upload(nn_pos);
  mp.socd_off = A.upload(socd_off);
  mp.socd_pos = A.upload(socd_pos);
  mp.socs_diag = A.upload(socs_diag);
  mp.socs_uv = A.upload(socs_uv);
  mp.socs_D = A.upload(socs_D);
  mp.exp_pos = A.upload(exp_pos);
  mp.pow_pos = A.upload(pow_pos);
  mp.psd_off = A.upload(psdo);
  mp.psd_pos = A.upload(psd_pos);
  KKTDev &kk = h->kk;
  kk.B = B;
  kk.prof_bytes = nullptr;
  h->d_prof_bytes = A.alloc<double>(3 * (size_t)B);
  kk.N = A.upload(N);
  kk.voff = A.upload(voff);
  kk.poff = A.upload(poff);
  kk.Kp = A.upload(Kp);
  kk.Kj = A.upload(Kj);
  kk.Kx = A.upload(Kx);
  h->kkt_nnz = knz;
  kk.Kdiag = A.upload(Kdiag);
  kk.Dsign = A.upload(Dsign);
  kk.gsrc = A.upload(gsrc);
  kk.Lp = A.upload(Lp);
  kk.Li = A.upload(Li);
  kk.Rp = A.upload(Rp);
  kk.Rk = A.upload(Rk);
  kk.Rpos = A.upload(Rpos);
  kk.lvl_off = A.upload(lvl_off);
  kk.nlev = A.upload(nlev);
  kk.lvl_ptr = A.upload(lvl_ptr);
  kk.lvl_nodes = A.upload(lvl_nodes);
  mark("kkt upload");
  // ---------------- substitution schedules (block instances) and streams
  // (single-warp instances)
  kk.fsched = kk.bsched = nullptr;
  if (has_large) {
    std::vector<int4> fsched(VT), bsched(VT);
    par_for(B, nth, [&](int i) {
      const int *lp = lvl_ptr.data() + lvl_off[i];
      const int *nodes = lvl_nodes.data() + voff[i];
      for (int l = 0; l < nlev[i]; ++l)
        for (int t = lp[l]; t < lp[l + 1]; ++t) {
          const int j = nodes[t];
          fsched[voff[i] + t] = make_int4(j, Rp[poff[i] + j], Rp[poff[i] + j + 1], 0);
          const int bp = N[i] - lp[l + 1] + (t - lp[l]);
          bsched[voff[i] + bp] = make_int4(j, Lp[poff[i] + j], Lp[poff[i] + j + 1], 0);
        }
    });
    kk.fsched = A.upload(fsched);
    kk.bsched = A.upload(bsched);
  }
  hvec<int2> fent((size_t)lnz), bent((size_t)lnz), kent((size_t)knz);
  hvec<int> fpos((size_t)lnz), bpos((size_t)lnz), flev(lvl_ptr.size()), blev(lvl_ptr.size());
  std::vector<int> nchf(B, 0), nchb(B, 0), nchk(B, 0);
  // encode segment positions: .x = seg | min(pos, kSPosMax) << 16 | last << kSLastBit
  auto encode = [](int2 *e, long long n) {
    long long q = 0;
    while (q < n) {
      long long r = q;
      while (r + 1 < n && e[r + 1].x == e[q].x) ++r;
      for (long long t = q; t <= r; ++t) {
        const int pos = (int)std::min<long long>(t - q, kSPosMax);
        e[t].x = (e[t].x & 0xffff) | (pos << 16) | ((t == r ? 1 : 0) << kSLastBit);
      }
      q = r + 1;
    }
  };
  auto nchunks = [](const int *lev, int nl) {
    int n = 0;
    for (int l = 0; l < nl; ++l) n += (lev[l + 1] - lev[l] + kSChunk - 1) / kSChunk;
    return n;
  };
  par_for(B, nth, [&](int i) {
    const auto &p = prep[i];
    const int nl = nlev[i];
    const int *lp = p.lvl_ptr.data();
    const long long base = Lp[poff[i]];
    long long f = base;
    for (int l = 0; l < nl; ++l) {
      flev[lvl_off[i] + l] = (int)f;
      for (int t = lp[l]; t < lp[l + 1]; ++t) {
        const int node = p.lvl_nodes[t];
        for (int r = p.Rp[node]; r < p.Rp[node + 1]; ++r) {
          fent[f] = make_int2(node, p.Rk[r]);
          fpos[f] = (int)(base + p.Rpos[r]);
          ++f;
        }
      }
    }
    flev[lvl_off[i] + nl] = (int)f;
    long long g = base;
    for (int l = nl - 1, t2 = 0; l >= 0; --l, ++t2) {
      blev[lvl_off[i] + t2] = (int)g;
      for (int t = lp[l]; t < lp[l + 1]; ++t) {
        const int node = p.lvl_nodes[t];
        for (int q = p.Lp[node]; q < p.Lp[node + 1]; ++q) {
          bent[g] = make_int2(node, p.Li[q]);
          bpos[g] = (int)(base + q);
          ++g;
        }
      }
    }
    blev[lvl_off[i] + nl] = (int)g;
    const long long kbase = Kp[poff[i]];
    for (int r = 0; r < N[i]; ++r)
      for (int q = p.Kp[r]; q < p.Kp[r + 1]; ++q) kent[kbase + q] = make_int2(r, p.Kj[q]);
    if (cls[i] == 1) {
      encode(fent.data() + base, f - base);
      encode(bent.data() + base, g - base);
      encode(kent.data() + kbase, (long long)p.Kj.size());
      nchf[i] = nchunks(flev.data() + lvl_off[i], nl);
      nchb[i] = nchunks(blev.data() + lvl_off[i], nl);
      nchk[i] = ((int)p.Kj.size() + kSChunk - 1) / kSChunk;
    }
  });
  mark("  streams: entries");
  // chunk tables: start relative to the stream base | scan steps <<
  // kStepShift | (count - 1) << kCntShift
  const auto ofch = prefix(nchf), obch = prefix(nchb), okch = prefix(nchk);
  hvec<int> fch(ofch[B]), bch(obch[B]), kch(okch[B]);
  std::vector<int> fch_off(B + 1), bch_off(B + 1), kch_off(B + 1);
  for (int i = 0; i <= B; ++i) {
    fch_off[i] = (int)ofch[i];
    bch_off[i] = (int)obch[i];
    kch_off[i] = (int)okch[i];
  }
  par_for(B, nth, [&](int i) {
    auto put = [](int *out, const int *lev, int nl, long long base, const int2 *ent) {
      for (int l = 0; l < nl; ++l)
        for (long long c = lev[l]; c < lev[l + 1]; c += kSChunk) {
          const int cnt = (int)std::min<long long>(kSChunk, lev[l + 1] - c);
          const int steps = chunk_scan_steps<kSK>(
              cnt, [&](int e) { return (ent[c + e].x >> 16) & kSPosMax; });
          *out++ = (int)((c - base) | ((long long)steps << kStepShift) |
                         ((long long)(cnt - 1) << kCntShift));
        }
    };
    if (cls[i] != 1) return;
    const long long base = Lp[poff[i]], kbase = Kp[poff[i]];
    put(fch.data() + ofch[i], flev.data() + lvl_off[i], nlev[i], base, fent.data());
    put(bch.data() + obch[i], blev.data() + lvl_off[i], nlev[i], base, bent.data());
    const int klev[2] = {(int)kbase, (int)(kbase + prep[i].Kj.size())};
    put(kch.data() + okch[i], klev, 1, kbase, kent.data());
  });
  // setup statistics (verbose): scan steps per chunk of each stream kind
  auto step_stats = [&](const char *name, const int *w, size_t n, bool factor) {
    if (!h->st.verbose) return;
    long long hist[8] = {0, 0, 0, 0, 0, 0, 0, 0}, nc = 0, ne = 0;
    for (size_t c = 0; c < n; ++c) {
      if (factor && ((unsigned)w[c] >> 31)) continue;  // pivot chunks take no scan
      ++hist[((unsigned)w[c] >> kStepShift) & 7u];
      ++nc;
      ne += (((unsigned)w[c] >> kCntShift) & (factor ? 63u : 127u)) + 1;
    }
    double mean = 0;
    for (int q = 0; q < 8; ++q) mean += q * (double)hist[q];
    std::fprintf(stderr,
                 "clgpu setup: %-6s chunks %lld, entries/chunk %.1f, scan steps mean %.2f "
                 "[%lld %lld %lld %lld %lld %lld]\n",
                 name, nc, nc ? (double)ne / nc : 0.0, nc ? mean / nc : 0.0, hist[0], hist[1],
                 hist[2], hist[3], hist[4], hist[5]);
  };
  step_stats("fwd", fch.data(), fch.size(), false);
  step_stats("bwd", bch.data(), bch.size(), false);
  step_stats("resid", kch.data(), kch.size(), false);
  mark("  streams: chunks + upload");
  // streamed factorisation: op streams, pivots and chunk tables, split over
  // the kFactorWarps warps of the instance's block level by level
  {
    constexpr long long kFactorSmemBytes = 96 * 1024;
    constexpr int W = kFactorWarps;
    const long long ring_bytes = (long long)W * kFRingSlots * kChunk * (long long)sizeof(uint2);
    std::vector<int> fs(B, 0);
    std::vector<long long> nch(B, 0);
    std::vector<std::vector<int>> ich(B);
    std::vector<std::array<int, W + 1>> iwoff(B);
    hvec<int> flcnt((size_t)lvof[B] * W);
    hvec<int> Lkpos((size_t)lnz);
    // instances on the streamed factorisation, their op counts, and the
    // streams written in place at their final offsets
    std::vector<long long> ocnt(B, 0);
    par_for(B, nth, [&](int i) {
      const auto &p = prep[i];
      // (the op words address at most kFopMaxPos work-vector positions)
      if (cls[i] != 1 || (N[i] + (long long)p.Li.size()) * 8 + ring_bytes > kFactorSmemBytes ||
          N[i] + (long long)p.Li.size() > kFopMaxPos)
        return;
      fs[i] = 1;
      ocnt[i] = factor_op_count(p);
    });
    const auto oop = prefix(ocnt);
    if (oop[B] > 2000000000LL) return -4;
    hvec<uint2> fop(std::max<long long>(oop[B], 1));
    par_for(B, nth, [&](int i) {
      thread_local FactorOpScratch sc;
      const auto &p = prep[i];
      l_kkt_positions(p, kof[i], Lkpos.data() + lof[i], sc);
      if (!fs[i]) return;
      bool ok = build_factor_ops(p, fop.data() + oop[i], flcnt.data() + (size_t)lvl_off[i] * W,
                                 ich[i], iwoff[i], sc);
      // an op stream longer than the chunk words address, or a structure
      // mismatch, falls back to the level-scheduled single-warp factorisation
      if (ocnt[i] > (long long)kStartMask) ok = false;
      if (!ok) {
        fs[i] = 0;
        ich[i].clear();
        for (int w = 0; w <= W; ++w) iwoff[i][w] = 0;
      }
      nch[i] = (long long)ich[i].size();
    });
    const auto och = prefix(nch);
    if (och[B] > 2000000000LL) return -4;
    hvec<int> foch(std::max<long long>(och[B], 1));
    std::vector<int> fop_base(B), fwoff((size_t)B * (W + 1));
    bool any_fs = false;
    for (int i = 0; i < B; ++i) {
      fop_base[i] = (int)oop[i];
      for (int w = 0; w <= W; ++w) fwoff[(size_t)i * (W + 1) + w] = (int)(och[i] + iwoff[i][w]);
      if (fs[i]) any_fs = true;
    }
    par_for(B, nth, [&](int i) {
      std::copy(ich[i].begin(), ich[i].end(), foch.begin() + och[i]);
    });
    step_stats("factor", foch.data(), foch.size(), true);
    mark("  factor ops: build");
    kk.fstream = A.upload(fs);
    kk.fop_base = A.upload(fop_base);
    kk.foch = A.upload(foch);
    kk.fwoff = A.upload(fwoff);
    kk.flcnt = A.upload(flcnt);
    kk.fop = A.upload(fop);
    kk.Lkpos = A.upload(Lkpos);
    mark("  factor ops: upload");
    kk.has_fstream = any_fs ? 1 : 0;
    kk.has_small_legacy = 0;
    for (int i = 0; i < B; ++i)
      if (cls[i] == 1 && !fs[i]) kk.has_small_legacy = 1;
    // launch list: streamed instances by decreasing shared-memory need (the
    // largest start first); one block each, sized for the largest
    {
      auto need = [&](int i) {
        return ((((long long)N[i] + (long long)prep[i].Li.size()) * 8 + 15) & ~15LL) +
               ring_bytes;
      };
      std::vector<int> items;
      for (int i = 0; i < B; ++i)
        if (fs[i]) items.push_back(i);
      std::stable_sort(items.begin(), items.end(),
                       [&](int a, int b) { return need(a) > need(b); });
      kk.fs_count = (int)items.size();
      kk.fs_smem = items.empty() ? 0 : (int)need(items[0]);
      kk.fs_inst = A.upload(items);
    }
  }
  kk.cls = A.upload(cls);
  // ---------------- supernodal instances: plan and numeric storage
  kk.sn = nullptr;
  if (h->any_sn) {
    std::vector<SnInstance> sin;
    int vlo = VT, vhi = 0;
    for (int i = 0; i < B; ++i)
      if (cls[i] == 3) {
        sin.push_back({&prep[i].sym, prep[i].Kp.data(), prep[i].Kj.data(), kof[i], voff[i], i});
        vlo = std::min(vlo, voff[i]);
        vhi = std::max(vhi, voff[i + 1]);
      }
    SnPlan plan;
    std::string err;
    if (!sn_build_plan(sin, plan, &err)) return -4;
    std::vector<int> vinst(vhi - vlo, -1);
    for (int i = 0; i < B; ++i)
      if (cls[i] == 3)
        for (int v = voff[i]; v < voff[i + 1]; ++v) vinst[v - vlo] = i;
    h->sn.reset(new SnExec());
    if (!sn_exec_create(plan, h->mixed, B, vlo, vhi - vlo, vinst, A, *h->sn)) return -5;
    kk.sn = h->sn.get();
    mark("supernodal plan");
  }
  // pack single-warp solves into blocks of kSolveWarps warps: each warp needs
  // its work vector (N FP64 values) and its ring (entries + FP64 values);
  // bins sized so kSolveBlocksPerSM blocks fit an SM's shared memory
  // (two-side solves: two work vectors per warp)
  for (int nr = 1; nr <= 2; ++nr) {
    auto need = [&](int i) {
      return nr * (((long long)N[i] * 8 + 15) & ~15LL) +
             (long long)kSRingSlots * kSChunk * (long long)(sizeof(int2) + sizeof(double));
    };
    std::vector<int> items, pinst, poffv;
    for (int i = 0; i < B; ++i)
      if (cls[i] == 1) items.push_back(i);
    long long cap = ((228LL * 1024) / kSolveBlocksPerSM - 1024) & ~15LL;
    for (int i : items) cap = std::max(cap, need(i));
    const int nb = ffd_pack(items, need, cap, kSolveWarps, pinst, poffv);
    if (nr == 1) {
      kk.spack_blocks = nb;
      kk.spack_inst = A.upload(pinst);
      kk.spack_off = A.upload(poffv);
      kk.spack_smem = (int)cap;
    } else {
      kk.spack2_blocks = nb;
      kk.spack2_inst = A.upload(pinst);
      kk.spack2_off = A.upload(poffv);
      kk.spack2_smem = (int)cap;
    }
  }
  kk.fch = A.upload(fch);
  kk.bch = A.upload(bch);
  kk.kch = A.upload(kch);
  kk.fch_off = A.upload(fch_off);
  kk.bch_off = A.upload(bch_off);
  kk.kch_off = A.upload(kch_off);
  kk.fent = A.upload(fent);
  kk.bent = A.upload(bent);
  kk.fpos = A.upload(fpos);
  kk.bpos = A.upload(bpos);
  kk.flev = A.upload(flev);
  kk.blev = A.upload(blev);
  kk.kent = A.upload(kent);
  if (h->mixed) {
    kk.LxF = A.alloc<float>((size_t)lnz);
    kk.LxB = A.alloc<float>((size_t)lnz);
    kk.LxR = has_large ? A.alloc<float>((size_t)lnz) : nullptr;
    kk.Lx = A.alloc<float>((size_t)lnz);
    kk.D = A.alloc<float>(VT);
    kk.Dinv = A.alloc<float>(VT);
    kk.Lacc = A.alloc<double>((size_t)lnz);
    kk.Dacc = A.alloc<double>(VT);
  } else {
    kk.LxF = A.alloc<double>((size_t)lnz);
    kk.LxB = A.alloc<double>((size_t)lnz);
    kk.LxR = has_large ? A.alloc<double>((size_t)lnz) : nullptr;
    kk.Lx = A.alloc<double>((size_t)lnz);
    kk.D = A.alloc<double>(VT);
    kk.Dinv = A.alloc<double>(VT);
    kk.Lacc = nullptr;
    kk.Dacc = nullptr;
  }
  mark("schedules + streams");
  kk.yf = A.alloc<double>(VT);
  kk.w = A.alloc<double>(VT);
  kk.max_small_N = max_small;
  kk.has_small = has_small;
  kk.has_large = has_large;
  kk.b = A.alloc<double>(VT);
  kk.x = A.alloc<double>(VT);
  kk.e = A.alloc<double>(VT);
  kk.b2 = A.alloc<double>(VT);
  kk.x2 = A.alloc<double>(VT);
  kk.e2 = A.alloc<double>(VT);
  kk.dx = A.alloc<double>(VT);
  // ---------------- vectors and scalars
  Dev &dv = h->dv;
  dv.B = B;
  dv.nx = nx;
  dv.mz = mz;
  dv.Pp = A.upload(Pp);
  dv.Pj = A.upload(Pj);
  dv.Px = A.upload(Pxv);
  dv.Ap = A.upload(Ap);
  dv.Aj = A.upload(Aj);
  dv.Ax = A.upload(Axv);
  dv.Atp = A.upload(Atp);
  dv.Atj = A.upload(Atj);
  dv.Atx = A.upload(Atxv);
  dv.q = A.upload(q);
  dv.negq = A.upload(negq);
  dv.b = A.upload(b);
  dv.d = A.upload(dd);
  dv.dinv = A.upload(ddinv);
  dv.e = A.upload(ee);
  dv.einv = A.upload(eeinv);
  dv.col_inst = A.upload(col_inst);
  dv.row_inst = cs.row_inst;
  {
    std::vector<int> zb(6 * (size_t)B, 0), zc(6 * (size_t)B, 0);
    for (int i = 0; i < B; ++i) {
      int lr = 0;
      for (int t = 0; t < 6; ++t) {
        int cnt = prep[i].type_rows[t];
        zc[6 * i + t] = cnt;
        zb[6 * i + t] = cnt > 0 ? grow[i][lr] : 0;
        lr += cnt;
      }
    }
    dv.xoff = A.upload(xoff);
    dv.zbeg = A.upload(zb);
    dv.zcnt = A.upload(zc);
  }
  double **xv[] = {&dv.x, &dv.px, &dv.rhs_x, &dv.dx, &dv.rx, &dv.rx_inf, &dv.Px_, &dv.x1,
                   &dv.x2, &dv.zerox};
  for (auto p : xv) *p = A.alloc<double>(nx);
  double **zv[] = {&dv.s, &dv.z, &dv.ps, &dv.pz, &dv.rhs_s, &dv.rhs_z, &dv.ds, &dv.dz,
                   &dv.rz, &dv.rz_inf, &dv.z1, &dv.z2, &dv.workz, &dv.wconic, &dv.zeroz};
  for (auto p : zv) *p = A.alloc<double>(mz);
  dv.S = A.alloc<double>((size_t)NUM_SCALARS * B);
  dv.I = A.alloc<int>((size_t)NUM_INTS * B);
  dv.active = A.alloc<int>(B);
  dv.counter = A.alloc<int>(4);
  cs.inst_active = dv.active;
  h->ic.degree = A.upload(deg);
  h->ic.sym = A.upload(sym);
  cs.inst_sym = h->ic.sym;
  h->d_reset = A.alloc<int>(B);
  // per-instance constants for init
  h->d_c = A.upload(c);
  // ---------------- numeric setup on the device: Ruiz equilibration, the
  // cost scaling, rectification and the KKT values of the instances whose
  // equilibration the host left undone (bitwise the host's result)
  {
    std::vector<int> on(B, 0);
    bool any = false;
    for (int i = 0; i < B; ++i) {
      on[i] = prep[i].eq_deferred ? 1 : 0;
      any = any || on[i];
    }
    if (any) {
      std::vector<int2> rc;
      for (size_t k = 0; k < soc_off.size(); ++k)
        if (on[soc_inst[k]]) rc.push_back(make_int2(soc_off[k], soc_dim[k]));
      for (size_t k = 0; k < exp_inst.size(); ++k)
        if (on[exp_inst[k]]) rc.push_back(make_int2(cs.exp_begin + 3 * (int)k, 3));
      for (size_t k = 0; k < pow_inst.size(); ++k)
        if (on[pow_inst[k]]) rc.push_back(make_int2(cs.pow_begin + 3 * (int)k, 3));
      for (size_t k = 0; k < psd_off.size(); ++k)
        if (on[psd_inst[k]]) rc.push_back(make_int2(psd_off[k], psd_n[k] * (psd_n[k] + 1) / 2));
      EqDev q{};
      q.B = B;
      q.nx = nx;
      q.mz = mz;
      q.xoff = dv.xoff;
      q.col_inst = dv.col_inst;
      q.row_inst = dv.row_inst;
      q.Pp = dv.Pp;
      q.Pj = dv.Pj;
      q.Px = const_cast<double *>(dv.Px);
      q.Ap = dv.Ap;
      q.Aj = dv.Aj;
      q.Ax = const_cast<double *>(dv.Ax);
      q.Atp = dv.Atp;
      q.Atj = dv.Atj;
      q.Atx = const_cast<double *>(dv.Atx);
      q.q = const_cast<double *>(dv.q);
      q.b = const_cast<double *>(dv.b);
      q.negq = const_cast<double *>(dv.negq);
      q.d = const_cast<double *>(dv.d);
      q.dinv = const_cast<double *>(dv.dinv);
      q.e = const_cast<double *>(dv.e);
      q.einv = const_cast<double *>(dv.einv);
      q.c = h->d_c;
      q.dw = A.alloc<double>(nx);
      q.ew = A.alloc<double>(mz);
      q.ct = A.alloc<double>(B);
      q.cflag = A.alloc<int>(B);
      q.on = A.upload(on);
      q.rcone = A.upload(rc);
      q.nrc = (int)rc.size();
      EqParams ep{h->st.equilibrate_enable, h->st.equilibrate_max_iter,
                  h->st.equilibrate_min_scaling, h->st.equilibrate_max_scaling};
      if (A.err != cudaSuccess) return -5;
      equilibrate_on_device(q, ep, h->d_upd_pmap, h->d_upd_pxy, h->upd_np, h->d_upd_amap,
                            h->d_upd_axy, h->upd_na, h->kk.Kx, 0);
      // setup runs on the legacy stream: waiting for it (not for the whole
      // device) leaves other solvers' streams running
      cudaError_t e = cudaStreamSynchronize(0);
      if (e == cudaSuccess) e = cudaGetLastError();
      if (e != cudaSuccess) return -1000 - (int)e;
      A.settle();
    }
    mark("device equilibration");
  }
  h->d_normq = A.upload(nq);
  h->d_normb = A.upload(nb);
  h->d_pnnz = A.upload(pnnz);
  // output map (user order)
  std::vector<int> zmap(mz), zinst(mz);
  for (int i = 0; i < B; ++i)
    for (int lr = 0; lr < prep[i].m; ++lr) {
      int ur = prep[i].user_row_of[lr];
      zmap[moff[i] + ur] = grow[i][lr];
      zinst[moff[i] + ur] = i;
    }
  h->d_zmap = A.upload(zmap);
  h->d_moff = A.upload(moff);
  h->d_zinst = A.upload(zinst);
  h->d_out = A.alloc<double>((size_t)nx + 2 * (size_t)mz);
  h->h_n.resize(B);
  h->h_m.resize(B);
  for (int i = 0; i < B; ++i) {
    h->h_n[i] = prep[i].n;
    h->h_m[i] = prep[i].m;
  }
  pinned_take(&h->h_counter, 4 * sizeof(int));
  // serving buffers
  h->d_sel = A.alloc<int>(B);
  h->d_sel_admit = A.alloc<int>(B);
  h->d_run = A.alloc<int>(B);
  h->d_active_admit = A.alloc<int>(B);
  h->d_list = A.alloc<int>(B);
  h->d_list_admit = A.alloc<int>(B);
  h->d_list_collect = A.alloc<int>(B);
  h->d_list_act = A.alloc<int>(B);
  h->d_info = A.alloc<double>((size_t)B * (NUM_SCALARS + NUM_INTS));
  pinned_take(&h->h_list, (size_t)B * sizeof(int));
  pinned_take(&h->h_list_admit, (size_t)B * sizeof(int));
  pinned_take(&h->h_list_collect, (size_t)B * sizeof(int));
  pinned_take(&h->h_list_act, (size_t)B * sizeof(int));
  pinned_take(&h->h_info, (size_t)B * (NUM_SCALARS + NUM_INTS) * sizeof(double));
  pinned_take(&h->h_stage, ((size_t)nx + (size_t)mz) * sizeof(double));
  pinned_take(&h->h_sol, ((size_t)nx + 2 * (size_t)mz) * sizeof(double));
  h->slot_state.assign(B, 0);
  h->slot_t0.assign(B, std::chrono::steady_clock::now());
  if (A.err != cudaSuccess) return -1000 - (int)A.err;
  cudaError_t e = cudaStreamSynchronize(0);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return -1000 - (int)e;
  A.settle();  // the uploads have completed: their host sources go back to the pool
  mark("scratch + tail");
  return 0;
}

// Host replay of one instance's streamed-factorisation op stream (the
// records, chunk words and level counts build_batch uploads) on a
// quasi-definite matrix with the instance's KKT pattern, against a dense
// LDL^T of the same permuted matrix.  The replay follows the kernel's
// schedule: per level, every warp part's update chunks (a segment's sum is
// subtracted from its target at the segment's last record, carried across
// chunk boundaries), then every part's pivot chunks (V[j] becomes 1/d_j);
// at the end L(i,j) = U(i,j) / d_j.  *resid receives the largest difference
// of L and D entries relative to the largest |D|.  Returns 0, -2 when the
// instance cannot be prepared, -3 when it does not take the streamed path,
// -4 when it is too large for the dense reference (N > 2000), or a negative
// structure code.
extern "C" int clgpu_debug_factor_stream(const clgpu_problem *pb, const clgpu_settings *st,
                                         double *resid) {
  using namespace clgpu;
  constexpr int W = kFactorWarps;
  if (!pb) return -1;
  SetupOptions opt;
  if (st) {
    opt.soc_threshold = st->soc_threshold;
    opt.equilibrate_enable = st->equilibrate_enable;
    opt.equilibrate_max_iter = st->equilibrate_max_iter;
  }
  Prepared p;
  if (!prepare_instance(*pb, opt, p)) return -2;
  const int N = p.N, nli = (int)p.Li.size();
  if (p.supernodal || N + nli > kFopMaxPos) return -3;
  if (N > 2000) return -4;
  FactorOpScratch sc;
  std::vector<int> Lkpos(nli);
  l_kkt_positions(p, 0, Lkpos.data(), sc);
  const int nl = (int)p.lvl_ptr.size() - 1;
  std::vector<uint2> ops(factor_op_count(p));
  std::vector<int> flcnt((size_t)nl * W), chk;
  std::array<int, W + 1> woff;
  if (!build_factor_ops(p, ops.data(), flcnt.data(), chk, woff, sc)) return -5;
  // the quasi-definite test matrix of clgpu_debug_check_instance
  const int knz = (int)p.Kj.size();
  std::vector<double> Kx(knz, 0.0);
  for (int r = 0; r < N; ++r)
    for (int q = p.Kp[r]; q < p.Kp[r + 1]; ++q) {
      const int c = p.Kj[q];
      if (c != r) Kx[q] = 0.01 * std::sin(1.0 + r + 7.0 * c) * std::sin(1.0 + c + 7.0 * r);
    }
  for (int r = 0; r < N; ++r) Kx[p.Kdiag[r]] = p.Dsign[r] * 2.0;
  // replay
  std::vector<double> V(N + nli, 0.0), D(N, 0.0);
  for (int j = 0; j < N; ++j) V[j] = Kx[p.Kdiag[j]];
  for (int q = 0; q < nli; ++q) V[N + q] = Lkpos[q] >= 0 ? Kx[Lkpos[q]] : 0.0;
  int cur[W];
  for (int w = 0; w < W; ++w) cur[w] = woff[w];
  auto chunk = [&](int w, bool pivot_expected, double &acc) {
    if (cur[w] >= woff[w + 1]) return -6;
    const unsigned word = (unsigned)chk[cur[w]++];
    const bool pivot = (word >> 31) != 0;
    if (pivot != pivot_expected) return -7;
    const int p0 = (int)(word & kStartMask), cnt = (int)((word >> kCntShift) & 63u) + 1;
    if (p0 + cnt > (int)ops.size()) return -8;
    for (int e = 0; e < cnt; ++e) {
      const uint2 o = ops[p0 + e];
      const int t = fop_t(o), a = fop_a(o);
      if (t >= N + nli || a >= N + nli) return -9;
      if (pivot) {
        const int sgn = a - 1;
        if (t >= N || (sgn != 1 && sgn != -1) || sgn != p.Dsign[t]) return -10;
        D[t] = V[t];
        V[t] = 1.0 / V[t];
      } else {
        const int b = fop_b(o), k = fop_k(o);
        if (b >= N + nli || k >= N) return -11;
        if (fop_pos(o) == 0) acc = 0.0;
        acc += V[a] * V[b] * V[k];
        if (fop_last(o)) V[t] -= acc;
      }
    }
    return 0;
  };
  for (int l = 0; l < nl; ++l) {
    for (int w = 0; w < W; ++w) {
      double acc = 0.0;
      const int nop = flcnt[(size_t)l * W + w] & 0xffff;
      for (int c = 0; c < nop; ++c)
        if (int rc = chunk(w, false, acc)) return rc;
    }
    for (int w = 0; w < W; ++w) {
      double acc = 0.0;
      const int npv = (flcnt[(size_t)l * W + w] >> 16) & 0xffff;
      for (int c = 0; c < npv; ++c)
        if (int rc = chunk(w, true, acc)) return rc;
    }
  }
  for (int w = 0; w < W; ++w)
    if (cur[w] != woff[w + 1]) return -12;  // every chunk replayed
  // dense LDL^T of the same permuted matrix
  std::vector<double> Ad((size_t)N * N, 0.0), Ld((size_t)N * N, 0.0), Dd(N, 0.0);
  for (int r = 0; r < N; ++r)
    for (int q = p.Kp[r]; q < p.Kp[r + 1]; ++q) Ad[(size_t)r * N + p.Kj[q]] = Kx[q];
  for (int j = 0; j < N; ++j) {
    double dj = Ad[(size_t)j * N + j];
    for (int k = 0; k < j; ++k) dj -= Ld[(size_t)j * N + k] * Ld[(size_t)j * N + k] * Dd[k];
    Dd[j] = dj;
    for (int i = j + 1; i < N; ++i) {
      double v = Ad[(size_t)i * N + j];
      for (int k = 0; k < j; ++k) v -= Ld[(size_t)i * N + k] * Ld[(size_t)j * N + k] * Dd[k];
      Ld[(size_t)i * N + j] = v / dj;
    }
  }
  double dmax = 0.0, err = 0.0;
  for (int j = 0; j < N; ++j) dmax = std::max(dmax, std::fabs(Dd[j]));
  for (int j = 0; j < N; ++j) {
    err = std::max(err, std::fabs(D[j] - Dd[j]));
    for (int q = p.Lp[j]; q < p.Lp[j + 1]; ++q)
      err = std::max(err, std::fabs(V[N + q] * V[j] - Ld[(size_t)p.Li[q] * N + j]));
  }
  if (resid) *resid = err / std::max(dmax, 1e-300);
  return 0;
}

extern "C" int clgpu_solver_create(const clgpu_problem *probs, int nprob,
                                   const clgpu_settings *settings, clgpu_solver **out) {
  if (!probs || nprob < 1 || !out) return -1;
  auto *h = new clgpu_solver();
  if (settings)
    h->st = *settings;
  else
    clgpu_default_settings(&h->st);
  if (h->st.direct_solve_method < CLGPU_METHOD_FP64 ||
      h->st.direct_solve_method > CLGPU_METHOD_MIXED_F64ELIM) {
    delete h;
    return -1;
  }
  h->mixed = h->st.direct_solve_method != CLGPU_METHOD_FP64;
  h->arith32 = h->st.direct_solve_method == CLGPU_METHOD_MIXED;
  if (h->mixed) h->st.static_regularization_constant = std::sqrt(1.1920928955078125e-07);
  SetupOptions opt;
  opt.soc_threshold = h->st.soc_threshold;
  opt.equilibrate_enable = h->st.equilibrate_enable;
  opt.equilibrate_max_iter = h->st.equilibrate_max_iter;
  opt.equilibrate_min_scaling = h->st.equilibrate_min_scaling;
  opt.equilibrate_max_scaling = h->st.equilibrate_max_scaling;
  opt.defer_equilibration = h->st.device_setup != 0;
  std::vector<Prepared> prep(nprob);
  std::vector<int> okv(nprob, 0);
  int nth = h->st.setup_threads > 0 ? h->st.setup_threads
                                    : (int)std::max(1u, std::thread::hardware_concurrency());
  nth = std::min(nth, nprob);
  auto t_prep = std::chrono::steady_clock::now();
  {
    std::vector<std::thread> th;
    std::atomic<int> next{0};
    for (int t = 0; t < nth; ++t)
      th.emplace_back([&]() {
        while (true) {
          int i = next.fetch_add(1);
          if (i >= nprob) break;
          okv[i] = prepare_instance(probs[i], opt, prep[i]) ? 1 : 0;
        }
      });
    for (auto &t : th) t.join();
  }
  for (int i = 0; i < nprob; ++i)
    if (!okv[i]) {
      if (h->st.verbose)
        std::fprintf(stderr, "clgpu: instance %d rejected: %s\n", i, prep[i].error.c_str());
      delete h;
      return -2;
    }
  if (h->st.verbose)
    std::fprintf(stderr, "clgpu setup: %-22s %8.1f ms (%d threads)\n", "prepare instances",
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() -
                                                           t_prep).count(), nth);
  int rc = build_batch(h, prep, nth);
  if (rc != 0) {
    delete h;
    return rc;
  }
  h->lp.static_reg = h->st.static_regularization_enable;
  h->lp.static_c = h->st.static_regularization_constant;
  h->lp.static_prop = h->st.static_regularization_proportional;
  h->lp.dyn_reg = h->st.dynamic_regularization_enable;
  h->lp.dyn_eps = h->st.dynamic_regularization_eps;
  h->lp.dyn_delta = h->st.dynamic_regularization_delta;
  h->lp.ir_enable = h->st.iterative_refinement_enable;
  h->lp.ir_maxiter = h->st.iterative_refinement_max_iter;
  h->lp.ir_reltol = h->st.iterative_refinement_reltol;
  h->lp.ir_abstol = h->st.iterative_refinement_abstol;
  h->lp.ir_stopratio = h->st.iterative_refinement_stop_ratio;
  h->sd = make_sd(h->st);
  h->info.assign(nprob, clgpu_info{});
  // launch shapes of the nonnegative and SOC kernels, timed on this batch
  const auto t_at = std::chrono::steady_clock::now();
  rc = h->st.autotune ? cones_autotune(h->cs, 0) : 0;
  if (rc != 0) {
    delete h;
    return rc;
  }
  if (h->st.verbose)
    std::fprintf(stderr, "clgpu setup: %-22s %8.1f ms\n", "launch-shape timing",
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() -
                                                           t_at).count());
  *out = h;
  return 0;
}

// ------------------------------------------------------------ solve phases
struct Phase {
  clgpu_solver *h;
  cudaStream_t st;
  // the views the kernels run on (default: the solver's own); serving admits
  // through views whose active mask is separate from the running passes'
  Dev *dp = nullptr;
  ConeSet *cp = nullptr;
  Dev &D() { return dp ? *dp : h->dv; }
  ConeSet &C() { return cp ? *cp : h->cs; }
  void mask(int mode) {
    k_set_mask<<<nblk(h->B), TB, 0, st>>>(D(), h->ic, mode, h->mask_sel);
    h->launches++;
  }
  void zero(int f0, int nf, double v = 0.0) {
    k_zero_fields<<<nblk((long long)nf * h->B), TB, 0, st>>>(D(), f0, nf, v);
    h->launches++;
  }
  // kkt_update! without its constant-rhs solve: Hs refresh, regularise +
  // refactor
  void kkt_refactor() {
    h->prof_begin(2, st);
    cones_refresh_kkt(C(), h->map, h->kk.Kx, st);
    h->prof_end(st);
    int *ok = D().I + I_KKT_OK * h->B;
    h->prof_begin(0, st);
    ldl_factor(h->kk, h->mixed, h->lp, D().active, ok, D().S + F_KKT_EPS * h->B, st,
               h->arith32);
    h->prof_end(st);
    h->launches += 8;
  }
  // kkt_update!: refresh, refactor, constant rhs solve [x2; z2] = K \ [-q; b]
  void kkt_update() {
    kkt_refactor();
    int *ok = D().I + I_KKT_OK * h->B;
    h->prof_begin(1, st);
    ldl_solve(h->kk, h->mixed, h->lp, D().active, D().negq, D().b, D().x2, D().z2, ok, st);
    h->prof_end(st);
    h->launches += 4;
  }
  // kkt_solve! (kktsystem_gpu.jl:139-227).  with_constant: also solve the
  // constant rhs of kkt_update! in the same launch (it depends on neither
  // side's result, and each side's result is exactly that of its own solve)
  void kkt_solve(bool affine, bool with_constant = false) {
    Dev &dv = h->dv;
    const double *dsc;
    if (affine) {
      dsc = dv.s;
    } else {
      cones_ds_from_dz_offset(h->cs, dv.wconic, dv.rhs_s, dv.z, st);
      dsc = dv.wconic;
    }
    k_workz<<<nblk(dv.mz), TB, 0, st>>>(dv, dsc);
    int *ok = dv.I + I_KKT_OK * h->B;
    h->prof_begin(with_constant ? 5 : 1, st);
    if (with_constant)
      ldl_solve2(h->kk, h->mixed, h->lp, dv.active, dv.negq, dv.b, dv.x2, dv.z2, dv.rhs_x,
                 dv.workz, dv.x1, dv.z1, ok, st);
    else
      ldl_solve(h->kk, h->mixed, h->lp, dv.active, dv.rhs_x, dv.workz, dv.x1, dv.z1, ok, st);
    h->prof_end(st);
    k_tau_dots<kRedThreads><<<h->B, kRedThreads, 0, st>>>(dv);
    k_tau_solve<<<nblk(h->B), TB, 0, st>>>(dv);
    k_lhs_xz<<<nblk(std::max(dv.nx, dv.mz)), TB, 0, st>>>(dv);
    cones_mul_Hs(h->cs, dv.ds, dv.dz, st);
    k_lhs_s<<<nblk(dv.mz), TB, 0, st>>>(dv, dsc);
    k_lhs_kappa<<<nblk(h->B), TB, 0, st>>>(dv);
    h->launches += 30;
  }
  void step_length(bool combined, int out_field) {
    Dev &dv = h->dv;
    k_step_prep<<<nblk(h->B), TB, 0, st>>>(dv);
    cones_step_length_sym(h->cs, dv.dz, dv.ds, dv.z, dv.s, dv.S + F_STEP_SYM * h->B, st);
    k_step_mid<<<nblk(h->B), TB, 0, st>>>(dv, h->ic, h->st.max_step_fraction);
    if (h->any_asym)
      cones_step_length_asym(h->cs, dv.dz, dv.ds, dv.z, dv.s, dv.S + F_STEP_SYM * h->B,
                             dv.S + F_STEP * h->B, h->st.linesearch_backtrack_step,
                             h->st.min_terminate_step_length, st);
    k_step_final<<<nblk(h->B), TB, 0, st>>>(dv, combined ? 1 : 0, h->st.max_step_fraction,
                                           out_field);
    h->launches += 8;
  }
  void residuals() {
    Dev &dv = h->dv;
    h->prof_begin(3, st);
    k_residuals<kRedThreads><<<h->B, kRedThreads, 0, st>>>(dv);
    h->prof_end(st);
    h->launches += 4;
  }
  int read_counter(int which) {
    cudaMemcpyAsync(h->h_counter, h->dv.counter, 4 * sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    return h->h_counter[which];
  }
};

// solver_default_start! (solver.jl:425-446) for every instance, or with
// h->mask_sel set only for the selected ones (the others are untouched)
static void ipm_start(clgpu_solver *h, Phase &P, cudaStream_t st) {
  Dev &dv = P.D();
  ConeSet &cs = P.C();
  const int B = h->B;
  // (re)initialise every per-instance scalar; solve! may be called repeatedly
  k_init_state<<<nblk(B), TB, 0, st>>>(dv, h->d_c, h->d_normq, h->d_normb, h->d_pnnz,
                                        h->mask_sel);
  P.mask(M_ALL_UNDONE);
  if (h->any_sym) {
    P.mask(M_SYM);
    cones_set_identity_scaling(cs, st);
    P.kkt_update();
    // QP instances: [x; z] = K \ [-q; b], s = -z
    P.mask(M_SYM_QP);
    ldl_solve(h->kk, h->mixed, h->lp, dv.active, dv.negq, dv.b, dv.x, dv.z,
              dv.I + I_KKT_OK * B, st);
    k_s_from_neg_z_masked<<<nblk(dv.mz), TB, 0, st>>>(dv);
    // LP instances: [x; -s] = K \ [0; b], then z from K \ [-q; 0]
    P.mask(M_SYM_LP);
    ldl_solve(h->kk, h->mixed, h->lp, dv.active, dv.zerox, dv.b, dv.x, dv.s,
              dv.I + I_KKT_OK * B, st);
    k_negate_s_masked<<<nblk(dv.mz), TB, 0, st>>>(dv);
    ldl_solve(h->kk, h->mixed, h->lp, dv.active, dv.negq, dv.zeroz, nullptr, dv.z,
              dv.I + I_KKT_OK * B, st);
    // shift s (primal) and z (dual) into the cone interior
    P.mask(M_SYM);
    for (int pd = 0; pd < 2; ++pd) {
      double *v = pd == 0 ? dv.s : dv.z;
      k_zero_fields<<<nblk(B), TB, 0, st>>>(dv, F_MARGIN_MIN, 1, kDMax);
      P.zero(F_MARGIN_SUM, 1);
      cones_margins(cs, v, pd, dv.S + F_MARGIN_MIN * B, dv.S + F_MARGIN_SUM * B, st);
      k_shift_amounts<<<nblk(B), TB, 0, st>>>(dv, h->ic, F_MARGIN_MIN, F_MARGIN_SUM, F_TAU_NUM,
                                              F_TAU_DEN);
      cones_scaled_unit_shift(cs, v, dv.S + F_TAU_NUM * B, pd, st);
      cones_scaled_unit_shift(cs, v, dv.S + F_TAU_DEN * B, pd, st);
    }
    k_set_tau_kappa_one<<<nblk(B), TB, 0, st>>>(dv);
  }
  if (h->any_asym) {
    P.mask(M_ASYM);
    cones_unit_initialization(cs, dv.z, dv.s, st);
    k_zero_x_masked<<<nblk(dv.nx), TB, 0, st>>>(dv);
    k_set_tau_kappa_one<<<nblk(B), TB, 0, st>>>(dv);
  }
}

// slots that finished in the pass just run: flagged running, now done
__global__ void k_serve_finished(Dev d, int *run, int *list, int *count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B) return;
  if (run[i] && IF(d, I_DONE, i)) {
    run[i] = 0;
    list[atomicAdd(count, 1)] = i;
  }
}

// the kernels of one pass of the IPM loop (solver.jl:265-393) over every
// running instance, up to the running count (dv.counter[0]) and, serving,
// the list of slots that finished in it (dv.counter[2], h->d_list)
static void ipm_pass_kernels(clgpu_solver *h, Phase &P, cudaStream_t st, double elapsed,
                             bool serve) {
  Dev &dv = h->dv;
  const int B = h->B;
  P.mask(M_PASS);
  P.residuals();
  k_info_termination<<<nblk(B), TB, 0, st>>>(dv, h->ic, h->sd, elapsed, h->d_reset);
  k_reset_vars<<<nblk(std::max(dv.nx, dv.mz)), TB, 0, st>>>(dv, h->d_reset);
  P.mask(M_PASS);
  // update_scaling
  h->prof_begin(4, st);
  cones_update_scaling(h->cs, dv.s, dv.z, dv.S + F_MU * B, dv.I + I_SCALING * B,
                       dv.I + I_SCALE_OK * B, st);
  h->prof_end(st);
  k_after_scaling<<<nblk(B), TB, 0, st>>>(dv);
  P.mask(M_PASS);
  // KKT update and affine step; the affine rhs needs nothing from the new
  // factor, so kkt_update!'s constant solve runs with the affine solve
  const bool fused = h->st.fused_solves != 0;
  if (fused)
    P.kkt_refactor();
  else
    P.kkt_update();
  k_affine_rhs<<<nblk(std::max(std::max(dv.nx, dv.mz), B)), TB, 0, st>>>(dv);
  cones_affine_ds(h->cs, dv.rhs_s, dv.s, st);
  P.kkt_solve(true, fused);
  P.step_length(false, F_ALPHA_AFF);
  k_combined_scalars<<<nblk(B), TB, 0, st>>>(dv);
  k_combined_pre<<<nblk(std::max(dv.nx, dv.mz)), TB, 0, st>>>(dv);
  cones_combined_ds_shift(h->cs, dv.rhs_z, dv.dz, dv.ds, dv.S + F_SIGMA_MU * B, st);
  k_combined_post<<<nblk(dv.mz), TB, 0, st>>>(dv);
  P.kkt_solve(false);
  k_check_numerical<<<nblk(B), TB, 0, st>>>(dv, h->ic);
  P.mask(M_PASS);
  P.step_length(true, F_ALPHA);
  if (h->any_asym) {
    cudaMemsetAsync(dv.counter + 1, 0, sizeof(int), st);
    k_bt_setup<<<nblk(B), TB, 0, st>>>(dv, h->ic);
    if (P.read_counter(1) > 0) {
      P.mask(M_BT);
      for (int j = 0; j < 50; ++j) {
        P.zero(F_BARRIER, 1);
        k_dot_shifted<kRedThreads><<<B, kRedThreads, 0, st>>>(dv);
        k_bt_central<<<nblk(B), TB, 0, st>>>(dv, h->ic);
        cones_barrier(h->cs, dv.z, dv.s, dv.dz, dv.ds, dv.S + F_ALPHA * B,
                      dv.I + I_BT_ACTIVE * B, dv.S + F_BARRIER * B, st);
        cudaMemsetAsync(dv.counter + 1, 0, sizeof(int), st);
        k_bt_check<<<nblk(B), TB, 0, st>>>(dv, h->st.linesearch_backtrack_step);
        P.mask(M_BT);
        if (P.read_counter(1) == 0) break;
      }
      P.mask(M_PASS);
    }
  }
  k_check_small_step<<<nblk(B), TB, 0, st>>>(dv, h->ic, h->sd);
  P.mask(M_PASS);
  k_add_step<<<nblk(std::max(dv.nx, dv.mz)), TB, 0, st>>>(dv);
  k_add_step_scalars<<<nblk(B), TB, 0, st>>>(dv);
  cudaMemsetAsync(dv.counter, 0, 3 * sizeof(int), st);
  k_count_running<<<nblk(B), TB, 0, st>>>(dv);
  if (serve) k_serve_finished<<<nblk(B), TB, 0, st>>>(dv, h->d_run, h->d_list, dv.counter + 2);
  h->launches += 25;
}

// One pass of the IPM loop over every running instance; returns how many are
// still running.  serve: also lists the slots that finished in this pass in
// h->h_list (count in *nfin).  Without host decisions inside the pass (no
// asymmetric-cone backtracking, no profiling or tracing, no time limit) the
// pass is captured once as a CUDA graph and replayed: one launch instead of
// ~60.  A solver's first solve launches kernel by kernel: capturing and
// instantiating the graph costs more than the launches of one solve, so a
// solver used once (a cold pass) never pays it; the second solve captures.
// The serving steps capture at once (their lanes warm up before serving, and
// no capture may be open while other threads allocate).
static int ipm_pass(clgpu_solver *h, Phase &P, cudaStream_t st, double elapsed, bool serve,
                    int *nfin) {
  Dev &dv = h->dv;
  const int B = h->B;
  const bool graph = h->use_graphs && !h->any_asym && !h->any_sn && !h->profiling && !h->st.verbose &&
                     !std::isfinite(h->st.time_limit) && h->mask_sel == nullptr &&
                     (serve || h->solves_done > 0);
  bool done = false;
  if (graph) {
    cudaGraphExec_t &ex = h->pass_exec[serve ? 1 : 0];
    if (!ex) {
      cudaGraph_t g = nullptr;
      const long long l0 = h->launches;
      if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        ipm_pass_kernels(h, P, st, 0.0, serve);
        if (cudaStreamEndCapture(st, &g) == cudaSuccess && g) {
          if (cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) ex = nullptr;
          cudaGraphDestroy(g);
        }
      }
      h->pass_launches = h->launches - l0;
      h->launches = l0;
      if (!ex) {
        cudaGetLastError();     // clear the failed capture's error
        h->use_graphs = false;  // and launch kernel by kernel from now on
      }
    }
    if (ex) {
      cudaGraphLaunch(ex, st);
      h->launches += h->pass_launches;
      done = true;
    }
  }
  if (!done) ipm_pass_kernels(h, P, st, elapsed, serve);
  const int running = P.read_counter(0);
  if (serve) {
    *nfin = h->h_counter[2];
    if (*nfin > 0) {
      cudaMemcpyAsync(h->h_list, h->d_list, (size_t)*nfin * sizeof(int),
                      cudaMemcpyDeviceToHost, st);
      cudaStreamSynchronize(st);
      std::sort(h->h_list, h->h_list + *nfin);
    }
  }
  if (h->st.verbose) {
    // per-pass trace of instance 0 (same columns as the CPU oracle's)
    double sv[NUM_SCALARS];
    int iv[NUM_INTS];
    for (int f = 0; f < NUM_SCALARS; ++f)
      cudaMemcpy(&sv[f], dv.S + (size_t)f * B, sizeof(double), cudaMemcpyDeviceToHost);
    for (int f = 0; f < NUM_INTS; ++f)
      cudaMemcpy(&iv[f], dv.I + (size_t)f * B, sizeof(int), cudaMemcpyDeviceToHost);
    std::fprintf(stderr,
                 "%3d  %+.8e  %+.8e  %.2e %.2e %.2e %.2e %.2e  a=%.3e st=%d sc=%d ok=%d\n",
                 iv[I_ITER], sv[F_COST_P], sv[F_COST_D], sv[F_GAP_REL], sv[F_RES_P],
                 sv[F_RES_D], sv[F_KTRATIO], sv[F_MU], sv[F_ALPHA], iv[I_STATUS],
                 iv[I_SCALING], iv[I_KKT_OK]);
  }
  return running;
}

// DefaultInfo of instance i from its scalar / integer fields
template <typename SF_, typename IF_>
static void fill_info(clgpu_info &inf, SF_ s, IF_ iv, double solve_time) {
  inf.status = iv(I_STATUS);
  inf.iterations = iv(I_ITER);
  inf.cost_primal = s(F_COST_P);
  inf.cost_dual = s(F_COST_D);
  bool infeas = inf.status == ST_PRIMAL_INFEASIBLE || inf.status == ST_DUAL_INFEASIBLE ||
                inf.status == ST_ALMOST_PRIMAL_INFEASIBLE ||
                inf.status == ST_ALMOST_DUAL_INFEASIBLE;
  inf.obj_val = infeas ? NAN : inf.cost_primal;
  inf.obj_val_dual = infeas ? NAN : inf.cost_dual;
  inf.res_primal = s(F_RES_P);
  inf.res_dual = s(F_RES_D);
  inf.res_primal_inf = s(F_RES_PINF);
  inf.res_dual_inf = s(F_RES_DINF);
  inf.gap_abs = s(F_GAP_ABS);
  inf.gap_rel = s(F_GAP_REL);
  inf.ktratio = s(F_KTRATIO);
  inf.mu = s(F_MU);
  inf.sigma = s(F_SIGMA);
  inf.step_length = s(F_ALPHA);
  inf.solve_time = solve_time;
}

extern "C" int clgpu_solver_solve(clgpu_solver *h, clgpu_stream_t stream) {
  if (!h) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  auto t0 = std::chrono::steady_clock::now();
  Phase P{h, st};
  Dev &dv = h->dv;
  const int B = h->B;
  h->launches = 0;
  if (h->st_admit) cudaStreamSynchronize(h->st_admit);  // no admission in flight
  h->serving = false;
  h->fresh.clear();
  h->aged.clear();
  h->mask_sel = nullptr;
  std::fill(h->slot_state.begin(), h->slot_state.end(), 0);
  if (h->profiling && h->d_prof_bytes)
    cudaMemsetAsync(h->d_prof_bytes, 0, 3 * (size_t)B * sizeof(double), st);
  h->kk.prof_bytes = h->profiling ? h->d_prof_bytes : nullptr;
  cudaEvent_t ev0, ev1;
  cudaEventCreate(&ev0);
  cudaEventCreate(&ev1);
  cudaEventRecord(ev0, st);
  ipm_start(h, P, st);
  // ----------------------------------------------------------- main loop
  int passes = 0;
  const int max_passes = 4 * (h->st.max_iter + 5);
  while (passes < max_passes) {
    ++passes;
    double elapsed =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (ipm_pass(h, P, st, elapsed, false, nullptr) == 0) break;
  }
  h->passes = passes;
  ++h->solves_done;
  if (h->profiling) {
    cudaStreamSynchronize(st);
    h->prof_collect();
  }
  // post-process
  k_post_status<<<nblk(B), TB, 0, st>>>(dv, h->sd, nullptr);
  double *ox = h->d_out, *os = ox + dv.nx, *oz = os + dv.mz;
  k_unscale<<<nblk(std::max(dv.nx, dv.mz)), TB, 0, st>>>(dv, h->d_zmap, h->d_zinst, ox, os, oz,
                                                        nullptr);
  cudaEventRecord(ev1, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return -1000 - (int)e;
  e = cudaGetLastError();
  if (e != cudaSuccess) return -1000 - (int)e;
  float ms = 0;
  cudaEventElapsedTime(&ms, ev0, ev1);
  h->last_ms = ms;
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  // copy results back into pinned staging (the info scalars reuse the
  // serving info buffer: a solve ends serving)
  double *S = h->h_info;
  int *I = reinterpret_cast<int *>(h->h_info + (size_t)NUM_SCALARS * B);
  cudaMemcpyAsync(S, dv.S, (size_t)NUM_SCALARS * B * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(I, dv.I, (size_t)NUM_INTS * B * sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(h->h_sol, h->d_out, ((size_t)dv.nx + 2 * (size_t)dv.mz) * sizeof(double),
                  cudaMemcpyDeviceToHost, st);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return -1000 - (int)e;
  double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  for (int i = 0; i < B; ++i)
    fill_info(
        h->info[i], [&](int f) { return S[(size_t)f * B + i]; },
        [&](int f) { return I[(size_t)f * B + i]; }, elapsed);
  h->solved = true;
  return 0;
}

// ------------------------------------------------------------- serving
__global__ void k_serve_mark_idle(Dev d, int *run) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.B) return;
  IF(d, I_DONE, i) = 1;
  run[i] = 0;
}
// sel[i] = 1 for the listed slots (sel zeroed before)
__global__ void k_serve_set(const int *list, int n, int *sel) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) sel[list[t]] = 1;
}
// the listed (admitted, started) slots join the running passes
__global__ void k_serve_activate(Dev d, const int *list, int n, int *run) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  IF(d, I_DONE, list[t]) = 0;
  run[list[t]] = 1;
}
// scalar and integer fields of the listed slots, packed slot by slot
__global__ void k_serve_gather_info(Dev d, const int *list, int n, double *out) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = list[t];
  double *o = out + (size_t)t * (NUM_SCALARS + NUM_INTS);
  for (int f = 0; f < NUM_SCALARS; ++f) o[f] = SF(d, f, i);
  for (int f = 0; f < NUM_INTS; ++f) o[NUM_SCALARS + f] = (double)IF(d, f, i);
}

// list -> device (through pinned host memory) and sel = its indicator
static void serve_upload_list(const int *slots, int n, int *h_buf, int *d_buf, int *d_sel,
                              int B, cudaStream_t st) {
  std::memcpy(h_buf, slots, (size_t)n * sizeof(int));
  cudaMemcpyAsync(d_buf, h_buf, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(d_sel, 0, (size_t)B * sizeof(int), st);
  k_serve_set<<<nblk(n), TB, 0, st>>>(d_buf, n, d_sel);
}

extern "C" int clgpu_serve_admit(clgpu_solver *h, const int *slots, int n, const double *q,
                                 const double *b, clgpu_stream_t stream) {
  if (!h || n < 0 || (n > 0 && !slots)) return -1;
  if (n == 0) return 0;
  Dev &dv = h->dv;
  std::vector<char> seen(h->B, 0);
  for (int k = 0; k < n; ++k) {
    const int i = slots[k];
    if (i < 0 || i >= h->B || seen[i]) return -2;
    if (h->serving && h->slot_state[i] != 0) return -3;  // running, pending or not collected
    seen[i] = 1;
  }
  if (h->serving && !h->fresh.empty()) return -4;  // one admission per step
  if (!h->serving) {
    cudaStream_t cst = (cudaStream_t)stream;
    k_serve_mark_idle<<<nblk(h->B), TB, 0, cst>>>(dv, h->d_run);
    if (!h->st_admit) {
      cudaStreamCreateWithFlags(&h->st_admit, cudaStreamNonBlocking);
      for (auto &ev : h->ev_admit) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    }
    h->dv_admit = dv;
    h->dv_admit.active = h->d_active_admit;
    h->cs_admit = h->cs;
    h->cs_admit.inst_active = h->d_active_admit;
    std::fill(h->slot_state.begin(), h->slot_state.end(), 0);
    h->fresh.clear();
    h->aged.clear();
    h->serving = true;
    h->kk.prof_bytes = nullptr;
    cudaError_t e = cudaStreamSynchronize(cst);
    if (e != cudaSuccess) return -1000 - (int)e;
  }
  cudaStream_t st = h->st_admit;
  // the previous admission's buffers are free once it completed
  const int ev = h->ev_fresh ^ 1;
  cudaEventSynchronize(h->ev_admit[h->ev_fresh]);
  // new q / b values (packed slot by slot, staged in pinned memory), scaled
  // with the setup equilibration
  long long qo = 0, bo = 0;
  double *hq = h->h_stage, *hb = h->h_stage + dv.nx;
  for (int k = 0; k < n; ++k) {
    const int i = slots[k];
    const int x0 = h->h_xoff[i], x1 = h->h_xoff[i + 1];
    const int m0 = h->h_moff[i], m1 = h->h_moff[i + 1];
    if (q && x1 > x0) {
      std::memcpy(hq + x0, q + qo, (size_t)(x1 - x0) * sizeof(double));
      cudaMemcpyAsync(h->d_in_q + x0, hq + x0, (size_t)(x1 - x0) * sizeof(double),
                      cudaMemcpyHostToDevice, st);
      k_update_q<<<nblk(x1 - x0), TB, 0, st>>>(dv, h->d_in_q, x0, x1, h->d_c);
    }
    if (b && m1 > m0) {
      std::memcpy(hb + m0, b + bo, (size_t)(m1 - m0) * sizeof(double));
      cudaMemcpyAsync(h->d_in_b + m0, hb + m0, (size_t)(m1 - m0) * sizeof(double),
                      cudaMemcpyHostToDevice, st);
      k_update_b<<<nblk(m1 - m0), TB, 0, st>>>(dv, h->d_in_b, m0, m1, h->d_zmap);
    }
    if (q || b)
      k_update_norms<128><<<1, 128, 0, st>>>(q ? h->d_in_q : nullptr, b ? h->d_in_b : nullptr,
                                             dv.xoff, h->d_moff, i, h->d_normq, h->d_normb);
    qo += x1 - x0;
    bo += m1 - m0;
  }
  // the starting point of the admitted slots, through the admission views
  serve_upload_list(slots, n, h->h_list_admit, h->d_list_admit, h->d_sel_admit, h->B, st);
  Phase P{h, st, &h->dv_admit, &h->cs_admit};
  h->mask_sel = h->d_sel_admit;
  ipm_start(h, P, st);
  h->mask_sel = nullptr;
  cudaEventRecord(h->ev_admit[ev], st);
  h->ev_fresh = ev;
  const auto now = std::chrono::steady_clock::now();
  for (int k = 0; k < n; ++k) {
    h->slot_state[slots[k]] = 3;
    h->slot_t0[slots[k]] = now;
    h->fresh.push_back(slots[k]);
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : -1000 - (int)e;
}

extern "C" int clgpu_serve_step(clgpu_solver *h, clgpu_stream_t stream, int *finished,
                                int *nfinished, int *nrunning) {
  if (!h || !h->serving) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  int active = 0;
  for (int v : h->slot_state) active += v == 1;
  // the batch admitted before the previous step joins now; so does a fresh
  // one when nothing else runs (there is no pass for it to overlap)
  std::vector<int> join = h->aged;
  int wait_ev = h->ev_aged;
  h->aged.clear();
  if (active == 0 && join.empty() && !h->fresh.empty()) {
    join.swap(h->fresh);
    wait_ev = h->ev_fresh;
  }
  if (!join.empty()) {
    cudaStreamWaitEvent(st, h->ev_admit[wait_ev], 0);
    std::memcpy(h->h_list_act, join.data(), join.size() * sizeof(int));
    cudaMemcpyAsync(h->d_list_act, h->h_list_act, join.size() * sizeof(int),
                    cudaMemcpyHostToDevice, st);
    k_serve_activate<<<nblk((int)join.size()), TB, 0, st>>>(h->dv, h->d_list_act,
                                                           (int)join.size(), h->d_run);
    for (int i : join) h->slot_state[i] = 1;
  }
  Phase P{h, st};
  int nfin = 0;
  const int running = ipm_pass(h, P, st, 0.0, true, &nfin);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return -1000 - (int)e;
  for (int k = 0; k < nfin; ++k) {
    h->slot_state[h->h_list[k]] = 2;
    if (finished) finished[k] = h->h_list[k];
  }
  // the fresh batch has overlapped this pass; it joins the next one
  h->aged.swap(h->fresh);
  h->fresh.clear();
  h->ev_aged = h->ev_fresh;
  if (nfinished) *nfinished = nfin;
  if (nrunning) *nrunning = running + (int)h->aged.size();
  return 0;
}

extern "C" int clgpu_serve_collect(clgpu_solver *h, const int *slots, int n, double *x,
                                   double *s, double *z, clgpu_info *info,
                                   clgpu_stream_t stream) {
  if (!h || !h->serving || n < 0 || (n > 0 && !slots)) return -1;
  if (n == 0) return 0;
  for (int k = 0; k < n; ++k)
    if (slots[k] < 0 || slots[k] >= h->B || h->slot_state[slots[k]] != 2) return -2;
  cudaStream_t st = (cudaStream_t)stream;
  Dev &dv = h->dv;
  serve_upload_list(slots, n, h->h_list_collect, h->d_list_collect, h->d_sel, h->B, st);
  k_post_status<<<nblk(h->B), TB, 0, st>>>(dv, h->sd, h->d_sel);
  double *ox = h->d_out, *os = ox + dv.nx, *oz = os + dv.mz;
  k_unscale<<<nblk(std::max(dv.nx, dv.mz)), TB, 0, st>>>(dv, h->d_zmap, h->d_zinst, ox, os, oz,
                                                        h->d_sel);
  k_serve_gather_info<<<nblk(n), TB, 0, st>>>(dv, h->d_list_collect, n, h->d_info);
  constexpr int NF = NUM_SCALARS + NUM_INTS;
  cudaMemcpyAsync(h->h_info, h->d_info, (size_t)n * NF * sizeof(double),
                  cudaMemcpyDeviceToHost, st);
  long long xo = 0, mo = 0;
  for (int k = 0; k < n; ++k) {
    const int i = slots[k];
    const int nx_i = h->h_n[i], m_i = h->h_m[i];
    if (x && nx_i)
      cudaMemcpyAsync(x + xo, ox + h->h_xoff[i], (size_t)nx_i * sizeof(double),
                      cudaMemcpyDeviceToHost, st);
    if (s && m_i)
      cudaMemcpyAsync(s + mo, os + h->h_moff[i], (size_t)m_i * sizeof(double),
                      cudaMemcpyDeviceToHost, st);
    if (z && m_i)
      cudaMemcpyAsync(z + mo, oz + h->h_moff[i], (size_t)m_i * sizeof(double),
                      cudaMemcpyDeviceToHost, st);
    xo += nx_i;
    mo += m_i;
  }
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return -1000 - (int)e;
  const auto now = std::chrono::steady_clock::now();
  for (int k = 0; k < n; ++k) {
    const int i = slots[k];
    const double *o = h->h_info + (size_t)k * NF;
    const double t = std::chrono::duration<double>(now - h->slot_t0[i]).count();
    clgpu_info inf{};
    fill_info(
        inf, [&](int f) { return o[f]; }, [&](int f) { return (int)o[NUM_SCALARS + f]; }, t);
    if (info) info[k] = inf;
    h->info[i] = inf;
    h->slot_state[i] = 0;
  }
  return 0;
}

extern "C" int clgpu_solver_get_info(clgpu_solver *h, int inst, clgpu_info *info) {
  if (!h || !info || inst < 0 || inst >= h->B) return -1;
  *info = h->info[inst];
  return 0;
}

extern "C" int clgpu_solver_get_solution(clgpu_solver *h, int inst, double *x, double *s,
                                         double *z) {
  if (!h || inst < 0 || inst >= h->B || !h->solved) return -1;
  const double *ox = h->h_sol, *os = ox + h->nx, *oz = os + h->mz;
  int n = h->h_n[inst], m = h->h_m[inst];
  if (x) std::memcpy(x, ox + h->h_xoff[inst], n * sizeof(double));
  if (s) std::memcpy(s, os + h->h_moff[inst], m * sizeof(double));
  if (z) std::memcpy(z, oz + h->h_moff[inst], m * sizeof(double));
  return 0;
}

extern "C" int clgpu_solver_get_solutions(clgpu_solver *h, double *x, double *s, double *z,
                                          clgpu_info *info) {
  if (!h || !h->solved) return -1;
  const double *ox = h->h_sol, *os = ox + h->nx, *oz = os + h->mz;
  // large batches: the three copies split over a few host threads
  struct Part {
    double *dst;
    const double *src;
    size_t n;
  };
  std::vector<Part> parts;
  const size_t chunk = (size_t)1 << 18;  // 2 MB
  for (auto pr : {Part{x, ox, (size_t)h->nx}, Part{s, os, (size_t)h->mz},
                  Part{z, oz, (size_t)h->mz}})
    if (pr.dst)
      for (size_t o = 0; o < pr.n; o += chunk)
        parts.push_back({pr.dst + o, pr.src + o, std::min(chunk, pr.n - o)});
  const int np = (int)parts.size(), nth = std::min(8, np);
  if (nth <= 1) {
    for (auto &pr : parts) std::memcpy(pr.dst, pr.src, pr.n * sizeof(double));
  } else {
    std::atomic<int> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < nth; ++t)
      th.emplace_back([&]() {
        for (int k; (k = next.fetch_add(1)) < np;)
          std::memcpy(parts[k].dst, parts[k].src, parts[k].n * sizeof(double));
      });
    for (auto &t : th) t.join();
  }
  if (info) std::memcpy(info, h->info.data(), h->B * sizeof(clgpu_info));
  return 0;
}

extern "C" int clgpu_solver_get_launch_shapes(const clgpu_solver *h, int *nn_block,
                                              int *soc_variants) {
  if (!h) return -1;
  if (nn_block) *nn_block = h->cs.nn_block;
  if (soc_variants)
    for (int op = 0; op < kSocOps; ++op) soc_variants[op] = h->cs.soc_variant[op];
  return 0;
}
extern "C" int clgpu_solver_get_solution_views(const clgpu_solver *h, const double **x,
                                               const double **s, const double **z) {
  if (!h || !h->solved || !h->h_sol) return -1;
  if (x) *x = h->h_sol;
  if (s) *s = h->h_sol + h->nx;
  if (z) *z = h->h_sol + h->nx + h->mz;
  return 0;
}
extern "C" long long clgpu_solver_device_bytes(const clgpu_solver *h) {
  return h ? h->arena.bytes : -1;
}
extern "C" long long clgpu_solver_launch_count(const clgpu_solver *h) {
  return h ? h->launches : -1;
}
extern "C" int clgpu_solver_set_profiling(clgpu_solver *h, int enable) {
  if (!h) return -1;
  h->profiling = enable != 0;
  if (h->sn) sn_set_profiling(*h->sn, enable != 0);
  return 0;
}
extern "C" int clgpu_solver_debug_setup(const clgpu_solver *h, double *d, double *e, double *c,
                                        double *q, double *b, double *Kx, long long *kkt_nnz) {
  if (!h) return -1;
  const Dev &dv = h->dv;
  struct {
    double *dst;
    const double *src;
    size_t n;
  } cp[] = {{d, dv.d, (size_t)h->nx},       {e, dv.e, (size_t)h->mz},
            {c, h->d_c, (size_t)h->B},      {q, dv.q, (size_t)h->nx},
            {b, dv.b, (size_t)h->mz},       {Kx, h->kk.Kx, (size_t)h->kkt_nnz}};
  for (auto &x : cp)
    if (x.dst && x.n) {
      cudaError_t err = cudaMemcpy(x.dst, x.src, x.n * sizeof(double), cudaMemcpyDeviceToHost);
      if (err != cudaSuccess) return -1000 - (int)err;
    }
  if (kkt_nnz) *kkt_nnz = h->kkt_nnz;
  return 0;
}
extern "C" int clgpu_solver_get_sn_refinement(const clgpu_solver *h, long long *counts,
                                               double *worst) {
  if (!h) return -1;
  if (!h->sn) return 1;
  if (counts) {
    counts[0] = h->sn->ir_solves;
    counts[1] = h->sn->ir_sweeps;
    counts[2] = h->sn->ir_unconverged;
  }
  if (worst) *worst = h->sn->ir_worst;
  return 0;
}
extern "C" int clgpu_solver_get_sn_profile(const clgpu_solver *h, double *ms, double *flops,
                                           long long *calls) {
  if (!h) return -1;
  if (!h->sn) return 1;
  sn_get_profile(*h->sn, ms, flops, calls);
  return 0;
}
extern "C" int clgpu_solver_get_profile(const clgpu_solver *h, double *ms_total,
                                        double *ms_factor, double *ms_solve, double *ms_cones,
                                        double *ms_residual, int *passes) {
  if (!h) return -1;
  if (ms_total) *ms_total = h->last_ms;
  if (ms_factor) *ms_factor = h->prof[0];
  if (ms_solve) *ms_solve = h->prof[1];
  if (ms_cones) *ms_cones = h->prof[2];
  if (ms_residual) *ms_residual = h->prof[3];
  if (passes) *passes = h->passes;
  return 0;
}
extern "C" int clgpu_solver_get_phase_times(const clgpu_solver *h, double *ms, long long *calls) {
  if (!h) return -1;
  for (int c = 0; c < clgpu_solver::kPhases; ++c) {
    if (ms) ms[c] = h->prof[c];
    if (calls) calls[c] = h->prof_calls[c];
  }
  return 0;
}
extern "C" int clgpu_solver_get_phase_bytes(const clgpu_solver *h, double *bytes) {
  if (!h || !bytes) return -1;
  for (int c = 0; c < 3; ++c) bytes[c] = h->prof_bytes[c];
  return 0;
}
extern "C" int clgpu_solver_update_data(clgpu_solver *h, const double *Px, const double *q,
                                        const double *Ax, const double *b,
                                        clgpu_stream_t stream) {
  if (!h) return -1;
  if ((Px || Ax) && !h->upd_ok) return -11;  // repeated matrix entries at setup
  cudaStream_t st = (cudaStream_t)stream;
  Dev &dv = h->dv;
  if (Px && h->upd_np > 0) {
    cudaMemcpyAsync(h->d_in_P, Px, (size_t)h->upd_np * sizeof(double), cudaMemcpyHostToDevice,
                    st);
    k_update_P<<<nblk(h->upd_np), TB, 0, st>>>(dv, h->d_upd_pmap, h->d_upd_pxy, h->d_in_P,
                                                h->upd_np, h->d_c, h->kk.Kx);
  }
  if (Ax && h->upd_na > 0) {
    cudaMemcpyAsync(h->d_in_A, Ax, (size_t)h->upd_na * sizeof(double), cudaMemcpyHostToDevice,
                    st);
    k_update_A<<<nblk(h->upd_na), TB, 0, st>>>(dv, h->d_upd_amap, h->d_upd_axy, h->d_in_A,
                                                h->upd_na, h->kk.Kx);
  }
  if (q && dv.nx > 0) {
    cudaMemcpyAsync(h->d_in_q, q, (size_t)dv.nx * sizeof(double), cudaMemcpyHostToDevice, st);
    k_update_q<<<nblk(dv.nx), TB, 0, st>>>(dv, h->d_in_q, 0, dv.nx, h->d_c);
  }
  if (b && dv.mz > 0) {
    cudaMemcpyAsync(h->d_in_b, b, (size_t)dv.mz * sizeof(double), cudaMemcpyHostToDevice, st);
    k_update_b<<<nblk(dv.mz), TB, 0, st>>>(dv, h->d_in_b, 0, dv.mz, h->d_zmap);
  }
  if (q || b)
    k_update_norms<128><<<h->B, 128, 0, st>>>(q ? h->d_in_q : nullptr, b ? h->d_in_b : nullptr,
                                              dv.xoff, h->d_moff, 0, h->d_normq, h->d_normb);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // caller buffers consumed
  return e == cudaSuccess ? 0 : -1000 - (int)e;
}
extern "C" int clgpu_solver_update_qb(clgpu_solver *h, int inst, const double *q,
                                      const double *b) {
  if (!h || inst < 0 || inst >= h->B) return -1;
  Dev &dv = h->dv;
  const int x0 = h->h_xoff[inst], x1 = h->h_xoff[inst + 1];
  const int m0 = h->h_moff[inst], m1 = h->h_moff[inst + 1];
  if (q && x1 > x0) {
    cudaMemcpy(h->d_in_q + x0, q, (size_t)(x1 - x0) * sizeof(double), cudaMemcpyHostToDevice);
    k_update_q<<<nblk(x1 - x0), TB>>>(dv, h->d_in_q, x0, x1, h->d_c);
  }
  if (b && m1 > m0) {
    cudaMemcpy(h->d_in_b + m0, b, (size_t)(m1 - m0) * sizeof(double), cudaMemcpyHostToDevice);
    k_update_b<<<nblk(m1 - m0), TB>>>(dv, h->d_in_b, m0, m1, h->d_zmap);
  }
  if (q || b)
    k_update_norms<128><<<1, 128>>>(q ? h->d_in_q : nullptr, b ? h->d_in_b : nullptr, dv.xoff,
                                    h->d_moff, inst, h->d_normq, h->d_normb);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  return e == cudaSuccess ? 0 : -1000 - (int)e;
}
extern "C" int clgpu_solver_destroy(clgpu_solver *h) {
  if (!h) return -1;
  delete h;
  return 0;
}
