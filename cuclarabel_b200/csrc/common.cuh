// common.cuh -- shared device helpers and data layout for libclgpu.
//
// Layout (one batch = B independent problem instances, B = 1 for the plain
// path):
//   * x vectors are concatenated per instance (xoff[i] .. xoff[i+1]).
//   * s/z vectors use a TYPE-MAJOR global row order: all zero-cone rows of all
//     instances, then all nonnegative rows, then SOC rows, exp rows, pow rows,
//     PSD rows.  Inside one type block rows are ordered by instance, then by
//     cone.  Every cone kernel therefore streams one contiguous range, and
//     row_inst[g] gives the owning instance of global row g.
//   * per-instance scalars live in device arrays (struct-of-arrays, see
//     InstScalars), so a whole IPM pass runs without host round trips.
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include <cfloat>
#include <cmath>

namespace clgpu {

enum ConeType { CONE_ZERO = 0, CONE_NONNEG = 1, CONE_SOC = 2, CONE_EXP = 3,
                CONE_POW = 4, CONE_PSD = 5 };

constexpr double kDMax = DBL_MAX;
constexpr double kDEps = 2.220446049250313e-16;
// largest PSD side: one warp per cone, its matrices (7 of side n for
// update_scaling) in shared memory
constexpr int kPsdMaxSide = 48;

// src/utils/mathutils.jl:12 (logsafe)
__device__ __forceinline__ double logsafe(double v) {
  return v < 0 ? -kDMax : log(v);
}

// Device-side description of all cones of a batch.
struct ConeSet {
  int B;            // instances
  int m_total;      // total s/z rows
  const int *row_inst;  // [m_total]
  // nonnegative: rows [nn_begin, nn_begin + n_nn)
  int nn_begin, n_nn;
  int zero_begin, n_zero;
  // second-order cones
  int n_soc;            // number of cones
  int soc_begin, soc_rows;
  int soc_group;        // lanes per cone (power of two, <= 32)
  const int *soc_off;   // [n_soc] global row of first element
  const int *soc_dim;   // [n_soc]
  const int *soc_inst;  // [n_soc]
  const int *soc_sparse;// [n_soc] 1 if dim > soc_threshold
  // Launch shapes, chosen per cone set by cones_autotune: threads per block
  // of the nonnegative kernels, and for each tiled SOC operation its
  // variant, 0 = lane groups, v = 1..3 = shared-memory tiles of 32 << (v-1)
  // cones (8 rows per cone) over the cones of dim <= 16.
  int nn_block;
  int soc_variant[6];  // indexed by SocOp (cones.cuh)
  int soc_ntiles[4];         // tiles per shape v = 1..3 ([0] unused)
  const int *soc_tile[4];    // [2*soc_ntiles[v]] first and one-past-last cone
  int soc_skip_lo, soc_skip_hi;  // lane-group kernels leave these dims alone
  // exponential / power cones (3 rows each, contiguous)
  int n_exp, exp_begin;
  int n_pow, pow_begin;
  const int *exp_inst, *pow_inst;
  const double *pow_alpha;  // [n_pow]
  // PSD triangle cones
  int n_psd, psd_begin;
  const int *psd_off, *psd_n, *psd_inst;
  int psd_nmax;
  // state
  double *nn_w, *nn_lambda;           // [n_nn]
  double *soc_w, *soc_lambda;         // [soc_rows] (indexed g - soc_begin)
  double *soc_eta, *soc_d;            // [n_soc]
  double *soc_u, *soc_v;              // [soc_rows]
  double *exp_Hd, *exp_Hs, *exp_grad, *exp_z;  // 9,9,3,3 per cone
  double *pow_Hd, *pow_Hs, *pow_grad, *pow_z;
  double *psd_R, *psd_Rinv, *psd_lam;  // nmax^2, nmax^2, nmax per cone
  // per-instance flags
  const int *inst_active;  // [B] nonzero -> instance takes part
  const int *inst_sym;     // [B] 1 if every cone of the instance is symmetric
  // per-instance ranges (cones of each type are stored instance by instance):
  // [2*i] first index, [2*i+1] count -- nonneg rows (element index), SOC,
  // exp, pow and PSD cones (cone index)
  const int *rng_nn, *rng_soc, *rng_exp, *rng_pow, *rng_psd;
  // per-cone scratch for deterministic per-instance reductions, indexed
  // soc | exp | pow | psd (n_soc + n_exp + n_pow + n_psd entries each)
  double *cone_tmp, *cone_tmp2;
};

// KKT value positions touched by the Hs refresh (global indices into the
// concatenated per-instance permuted full KKT value array).
struct KKTMapDev {
  const int *nn_pos;         // [n_nn] diagonal position of each NN row
  const int *socd_off;       // [n_soc] start into socd_pos (dense cones) or -1
  const int *socd_pos;       // pairs (upper, lower) per triu entry
  const int *socs_diag;      // [soc_rows] diag position (sparse cones) or -1
  const int *socs_uv;        // [soc_rows*4] v up, v lo, u up, u lo (sparse)
  const int *socs_D;         // [n_soc*2] extra diagonal positions (sparse)
  const int *exp_pos;        // [n_exp*12]
  const int *pow_pos;        // [n_pow*12]
  const int *psd_off;        // [n_psd] start into psd_pos
  const int *psd_pos;        // pairs per triu entry of the t x t block
};

// per-instance scalar fields (doubles), stored field-major: S[f*B + i]
enum ScalarField {
  F_TAU = 0, F_KAPPA, F_MU, F_SIGMA, F_ALPHA, F_ALPHA_AFF,
  F_DOT_QX, F_DOT_BZ, F_DOT_SZ, F_DOT_XPX, F_RTAU,
  F_COST_P, F_COST_D, F_RES_P, F_RES_D, F_RES_PINF, F_RES_DINF,
  F_GAP_ABS, F_GAP_REL, F_KTRATIO,
  F_PREV_COST_P, F_PREV_COST_D, F_PREV_RES_P, F_PREV_RES_D, F_PREV_GAP_ABS,
  F_PREV_GAP_REL, F_PREV_TAU, F_PREV_KAPPA,
  F_EQ_C, F_NORMQ, F_NORMB,
  // reductions (zeroed before use)
  F_NRM_X, F_NRM_Z, F_NRM_S, F_NRM_RXINF, F_NRM_PX, F_NRM_RZINF, F_NRM_RZ,
  F_NRM_RX,
  F_MARGIN_MIN, F_MARGIN_SUM, F_STEP_SYM, F_STEP, F_BARRIER,
  // step direction scalars
  F_STEP_TAU, F_STEP_KAPPA, F_RHS_TAU, F_RHS_KAPPA,
  F_TAU_NUM, F_TAU_DEN,
  F_DOT_Q_X1, F_DOT_B_Z1, F_DOT_XI_PX1, F_DOT_Q_X2, F_DOT_B_Z2,
  F_QF1, F_QF2, F_KKT_EPS, F_SIGMA_MU, F_MFAC,
  F_SOLVE_TIME,
  NUM_SCALARS
};
// per-instance integer fields: I[f*B + i]
enum IntField {
  I_STATUS = 0, I_ITER, I_SCALING, I_DONE, I_SKIP, I_KKT_OK, I_SCALE_OK,
  I_SYM, I_PNNZ, I_BT_ACTIVE, I_ALPHA_ZERO_EXIT,
  NUM_INTS
};

// SolverStatus codes, src/statuscodes.jl:24-36
enum Status { ST_UNSOLVED = 0, ST_SOLVED, ST_PRIMAL_INFEASIBLE,
  ST_DUAL_INFEASIBLE, ST_ALMOST_SOLVED, ST_ALMOST_PRIMAL_INFEASIBLE,
  ST_ALMOST_DUAL_INFEASIBLE, ST_MAX_ITERATIONS, ST_MAX_TIME,
  ST_NUMERICAL_ERROR, ST_INSUFFICIENT_PROGRESS };

// ---------------------------------------------------------------- atomics
// atomic min for non-negative doubles (IEEE order == unsigned int order)
__device__ __forceinline__ void atomic_min_nonneg(double *addr, double v) {
  if (!(v >= 0)) v = 0;  // NaN or negative -> 0 (caller guarantees >= 0)
  atomicMin(reinterpret_cast<unsigned long long *>(addr),
            (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
  if (!(v >= 0)) v = 0;
  atomicMax(reinterpret_cast<unsigned long long *>(addr),
            (unsigned long long)__double_as_longlong(v));
}
// generic atomic min (any sign) via CAS
__device__ __forceinline__ void atomic_min_any(double *addr, double v) {
  unsigned long long *a = reinterpret_cast<unsigned long long *>(addr);
  unsigned long long old = *a, assumed;
  do {
    assumed = old;
    if (__longlong_as_double(assumed) <= v) return;
    old = atomicCAS(a, assumed, (unsigned long long)__double_as_longlong(v));
  } while (old != assumed);
}

__device__ __forceinline__ double warp_sum(double v, unsigned mask = 0xffffffffu) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// reduce within aligned groups of G lanes (G power of two)
template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double group_sum_dyn(double v, int G) {
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Warp-aggregated per-instance atomic add.  All 32 lanes must call it (lanes
// without a contribution pass inst = -1).
__device__ __forceinline__ void seg_atomic_add(double *base, int stride_unused,
                                               int inst, double v) {
  (void)stride_unused;
  unsigned full = 0xffffffffu;
  int first = __shfl_sync(full, inst, 0);
  bool uniform = __all_sync(full, inst == first);
  if (uniform) {
    if (first < 0) return;
    double s = warp_sum(v);
    if ((threadIdx.x & 31) == 0) atomicAdd(base + first, s);
  } else if (inst >= 0) {
    atomicAdd(base + inst, v);
  }
}
__device__ __forceinline__ void seg_atomic_min_nonneg(double *base, int inst,
                                                      double v) {
  unsigned full = 0xffffffffu;
  int first = __shfl_sync(full, inst, 0);
  bool uniform = __all_sync(full, inst == first);
  if (uniform) {
    if (first < 0) return;
    double s = warp_min(v);
    if ((threadIdx.x & 31) == 0) atomic_min_nonneg(base + first, s);
  } else if (inst >= 0) {
    atomic_min_nonneg(base + inst, v);
  }
}
// Atomic min of a non-negative value that skips the atomic when the stored
// value is already no larger.  The stored value only decreases, so a stale
// read can only let an unneeded atomic through; the result is the same.
// Thousands of blocks folding into one instance's step length would
// otherwise queue on a single address.
__device__ __forceinline__ void atomic_min_nonneg_filtered(double *addr, double v) {
  if (!(v >= 0)) v = 0;
  if (v < __ldcg(addr)) atomic_min_nonneg(addr, v);
}

// Block-aggregated per-instance min: every thread of the block must call it
// (threads without a value pass inst = -1); blockDim.x is a multiple of 32.
// Warps whose contributing lanes share one instance are reduced in the warp,
// then runs of equal instances across the block's warps in one thread, so a
// block whose rows all belong to one instance issues one filtered atomic.
__device__ __forceinline__ void block_seg_min_nonneg(double *base, int inst, double v) {
  __shared__ int s_inst[32];
  __shared__ double s_val[32];
  const unsigned full = 0xffffffffu;
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (inst < 0) v = CUDART_INF;
  else if (!(v >= 0)) v = 0;  // NaN or negative -> 0, as atomic_min_nonneg
  int lead = inst;
  for (int o = 16; o > 0; o >>= 1) lead = max(lead, __shfl_xor_sync(full, lead, o));
  bool uniform = __all_sync(full, inst < 0 || inst == lead);
  if (!uniform) {
    if (inst >= 0) atomic_min_nonneg_filtered(base + inst, v);
    lead = -1;
  }
  double m = warp_min(v);
  if (lane == 0) {
    s_inst[wid] = lead;
    s_val[wid] = m;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int cur = -1;
    double cm = CUDART_INF;
    for (int w = 0; w < nw; ++w) {
      int iw = s_inst[w];
      if (iw < 0) continue;
      if (iw != cur) {
        if (cur >= 0) atomic_min_nonneg_filtered(base + cur, cm);
        cur = iw;
        cm = s_val[w];
      } else {
        cm = fmin(cm, s_val[w]);
      }
    }
    if (cur >= 0) atomic_min_nonneg_filtered(base + cur, cm);
  }
}
__device__ __forceinline__ void seg_atomic_max_nonneg(double *base, int inst,
                                                      double v) {
  unsigned full = 0xffffffffu;
  int first = __shfl_sync(full, inst, 0);
  bool uniform = __all_sync(full, inst == first);
  if (uniform) {
    if (first < 0) return;
    double s = warp_max(v);
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(base + first, s);
  } else if (inst >= 0) {
    atomic_max_nonneg(base + inst, v);
  }
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

#define CLGPU_CHECK(expr)                                      \
  do {                                                         \
    cudaError_t _e = (expr);                                   \
    if (_e != cudaSuccess) return (int)-1000 - (int)_e;        \
  } while (0)

}  // namespace clgpu
