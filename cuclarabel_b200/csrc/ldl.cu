// ldl.cu -- batched sparse LDL^T numeric factorisation and solves (sm_100a).
//
// One thread block per instance.  Instances whose KKT dimension fits keep
// their dense work vector in shared memory and run on a single warp (NT=32:
// __syncwarp between dependent steps); larger instances run on 256 threads
// with the work vector in global scratch.
//
// Both the factorisation and the triangular solves are scheduled by
// elimination-tree levels (computed once by the symbolic phase): a column
// depends only on columns of lower levels, so every column of a level is
// processed concurrently and one barrier separates levels.  The KKT trees of
// the interior-point systems are bushy (height ~ N/10), which turns the
// O(N) chain of dependent steps into O(height).
//
// Factorisation, left-looking:
//   * wide level (>= NT/2 columns): one thread per column.  The column's
//     entries are accumulated in place: the lower part of K(:,j) and every
//     update column k (k in row j of L) are merged into column j's sorted
//     row list (the etree guarantees struct(L(j+1:,k)) is a subset of
//     struct(L(:,j))).
//   * narrow level: the whole block cooperates on one column through a dense
//     accumulator indexed by row; the update columns are applied one after
//     another with the threads spread over each column's rows.
// No floating-point atomics are used, so the factor of an instance is
// bitwise identical whether it is solved alone or inside any batch.
// Static regularisation (kktsolver_directldl_gpu.jl:216-260: eps = c +
// prop*||diag||_inf, diag +/- eps by the expected sign) is applied when the
// diagonal is read, so the stored KKT keeps its true diagonal for the
// refinement residual; dynamic regularisation follows the CPU path
// (sign*D(j) <= eps_dyn -> D(j) = sign*delta).
//
// Solve: forward substitution gathers each row of L (row pattern), backward
// substitution gathers each column, both level by level; then iterative
// refinement against the unregularised KKT exactly as
// kktsolver_directldl_gpu.jl:349-409.  In the mixed-precision form (the
// reference's :cudssmixed) L and D are STORED in FP32; accumulation,
// substitution arithmetic, the refinement residual and the iterate are FP64.
#include <type_traits>
#include "ldl.cuh"

namespace clgpu {

static constexpr int kSmallNT = 32;
static constexpr int kLargeNT = 256;
static constexpr int kSmemLimitBytes = 48 * 1024;

template <int NT>
__device__ __forceinline__ void bar_sync() {
  if (NT == 32)
    __syncwarp();
  else
    __syncthreads();
}

template <int NT>
__device__ __forceinline__ double block_sum(double v, double *red) {
  v = warp_sum(v);
  if (NT == 32) return v;
  int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < NT / 32; ++i) t += red[i];
    red[NT / 32] = t;
  }
  __syncthreads();
  return red[NT / 32];
}
template <int NT>
__device__ __forceinline__ double block_max(double v, double *red) {
  v = warp_max(v);
  if (NT == 32) return v;
  int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = red[0];
    for (int i = 1; i < NT / 32; ++i) t = fmax(t, red[i]);
    red[NT / 32] = t;
  }
  __syncthreads();
  return red[NT / 32];
}

// class of an instance: 1 = small (single warp, smem), 2 = large
__device__ __forceinline__ int inst_class(int N) {
  return (long long)N * (long long)sizeof(double) <= kSmemLimitBytes ? 1 : 2;
}

// Dynamic regularisation of pivot dj (kktsolver_directldl.jl:224-229 via
// QDLDL's Dsigns check): the FP64 pivot the elimination continues with.
__device__ __forceinline__ double pivot_value(double dj, signed char sg, const LDLParams &prm) {
  if (prm.dyn_reg) {
    const double sgn = double(sg);
    if (sgn * dj <= prm.dyn_eps) dj = prm.dyn_delta * sgn;
  }
  return dj;
}
// Stores pivot j: D and Dinv in the storage type T (Dinv is the inverse of
// the stored pivot so the solves see a consistent pair) and the FP64 pivot
// in Dacc, which aliases D in FP64 mode.  False if a stored value is not
// finite.
template <typename T>
__device__ __forceinline__ bool store_pivot(T *D, T *Dinv, double *Dacc, int j, double dj) {
  const T djs = T(dj);
  const T dis = T(1.0 / double(djs));
  D[j] = djs;
  Dinv[j] = dis;
  Dacc[j] = dj;
  return isfinite(double(djs)) && isfinite(double(dis));
}
// Stores factor entry q: the storage copy, and the FP64 value the rest of the
// elimination reads when the two differ.
template <typename T>
__device__ __forceinline__ void store_l(T *Lx, double *Lacc, int q, double v) {
  Lx[q] = T(v);
  if (!std::is_same<T, double>::value) Lacc[q] = v;
}

template <typename T, int NT, bool SMEM>
__global__ void __launch_bounds__(NT) k_ldl_factor(KKTDev k, LDLParams prm, const int *run,
                                                   int *ok, double *eps_out) {
  int inst = blockIdx.x;
  if (!run[inst]) return;
  int N = k.N[inst];
  if (inst_class(N) != (SMEM ? 1 : 2)) return;
  __shared__ double red[NT / 32 + 1];
  extern __shared__ __align__(16) unsigned char sm_raw[];
  const int vo = k.voff[inst], po = k.poff[inst];
  double *w = SMEM ? reinterpret_cast<double *>(sm_raw) : k.w + vo;
  T *Lx = reinterpret_cast<T *>(k.Lx);
  // FP64 factor values the elimination reads (aliases Lx / D in FP64 mode)
  double *Lacc = k.Lacc ? k.Lacc : reinterpret_cast<double *>(k.Lx);
  T *D = reinterpret_cast<T *>(k.D) + vo;
  T *Dinv = reinterpret_cast<T *>(k.Dinv) + vo;
  double *Dacc = (k.Dacc ? k.Dacc : reinterpret_cast<double *>(k.D)) + vo;
  const int *Kp = k.Kp + po, *Lp = k.Lp + po, *Rp = k.Rp + po;
  const int *Kdiag = k.Kdiag + vo;
  const int *nodes = k.lvl_nodes + vo;
  const int *lptr = k.lvl_ptr + k.lvl_off[inst];
  const int nlev = k.nlev[inst];
  const signed char *sg = k.Dsign + vo;
  const int tid = threadIdx.x;
  for (int i = tid; i < N; i += NT) w[i] = 0.0;
  double eps = 0;
  if (prm.static_reg) {
    double mx = 0;
    for (int i = tid; i < N; i += NT) mx = fmax(mx, fabs(k.Kx[Kdiag[i]]));
    mx = block_max<NT>(mx, red);
    eps = prm.static_c + prm.static_prop * mx;
  }
  bar_sync<NT>();
  bool finite = true;
  for (int l = 0; l < nlev; ++l) {
    const int a = lptr[l], b = lptr[l + 1];
    if (b - a >= NT / 2) {
      // ---- wide level: one thread per column, merge into the column
      for (int idx = a + tid; idx < b; idx += NT) {
        const int j = nodes[idx];
        const int q0 = Lp[j], q1 = Lp[j + 1];
        for (int q = q0; q < q1; ++q) Lacc[q] = 0.0;
        double dj = 0.0;
        int q = q0;
        for (int p = Kp[j]; p < Kp[j + 1]; ++p) {
          int c = k.Kj[p];
          if (c < j) continue;
          if (c == j) {
            dj = k.Kx[p] + (sg[j] > 0 ? eps : -eps);
            continue;
          }
          while (q < q1 && k.Li[q] != c) ++q;
          if (q < q1) Lacc[q] = k.Kx[p];
        }
        for (int r = Rp[j]; r < Rp[j + 1]; ++r) {
          const int kk = k.Rk[r], pos = k.Rpos[r];
          const double ljk = Lacc[pos];
          const double f = ljk * Dacc[kk];
          dj -= ljk * f;
          const int pe = Lp[kk + 1];
          q = q0;
          for (int p = pos + 1; p < pe; ++p) {
            const int i = k.Li[p];
            while (q < q1 && k.Li[q] != i) ++q;
            if (q < q1) Lacc[q] -= Lacc[p] * f;
          }
        }
        dj = pivot_value(dj, sg[j], prm);
        const double dinv = 1.0 / dj;
        if (!isfinite(dinv)) finite = false;
        for (int qq = q0; qq < q1; ++qq) store_l(Lx, Lacc, qq, Lacc[qq] * dinv);
        if (!store_pivot(D, Dinv, Dacc, j, dj)) finite = false;
      }
      bar_sync<NT>();
    } else {
      // ---- narrow level: the block cooperates on each column
      for (int idx = a; idx < b; ++idx) {
        const int j = nodes[idx];
        for (int p = Kp[j] + tid; p < Kp[j + 1]; p += NT) {
          int c = k.Kj[p];
          if (c > j)
            w[c] = k.Kx[p];
          else if (c == j)
            w[c] = k.Kx[p] + (sg[j] > 0 ? eps : -eps);
        }
        bar_sync<NT>();
        // update columns applied one after another (threads over the rows
        // of each update column, fixed order: the result is bitwise
        // reproducible and independent of the batch composition)
        const int r0 = Rp[j], r1 = Rp[j + 1];
        for (int rb = r0; rb < r1; rb += 32) {
          const int lane = tid & 31;
          int mypos = 0, myend = 0;
          double myf = 0.0, myl = 0.0;
          if (rb + lane < r1) {
            const int kk = k.Rk[rb + lane];
            mypos = k.Rpos[rb + lane];
            myend = Lp[kk + 1];
            myl = Lacc[mypos];
            myf = myl * Dacc[kk];
          }
          const int cnt = min(32, r1 - rb);
          for (int t = 0; t < cnt; ++t) {
            const int pos = __shfl_sync(0xffffffffu, mypos, t);
            const int pe = __shfl_sync(0xffffffffu, myend, t);
            const double f = __shfl_sync(0xffffffffu, myf, t);
            const double ljk = __shfl_sync(0xffffffffu, myl, t);
            if (tid == 0) w[j] -= ljk * f;
            for (int p = pos + 1 + tid; p < pe; p += NT) w[k.Li[p]] -= Lacc[p] * f;
            bar_sync<NT>();
          }
        }
        const double dj = pivot_value(w[j], sg[j], prm);
        const double dinv = 1.0 / dj;
        if (!isfinite(dinv)) finite = false;
        for (int q = Lp[j] + tid; q < Lp[j + 1]; q += NT) {
          const int i = k.Li[q];
          store_l(Lx, Lacc, q, w[i] * dinv);
          w[i] = 0.0;
        }
        bar_sync<NT>();
        if (tid == 0) {
          if (!store_pivot(D, Dinv, Dacc, j, dj)) finite = false;
          w[j] = 0.0;
        }
        bar_sync<NT>();
      }
    }
  }
  double bad = block_max<NT>(finite ? 0.0 : 1.0, red);
  if (tid == 0) {
    if (bad > 0) ok[inst] = 0;
    if (eps_out) eps_out[inst] = eps;
  }
}

// y <- L^{-T} D^{-1} L^{-1} y, level-scheduled gathers
template <typename T, int NT>
__device__ void ldl_trisolve(const KKTDev &k, int inst, int N, int vo, int po, double *y,
                             double *red) {
  const T *Lx = reinterpret_cast<const T *>(k.Lx);
  const T *Dinv = reinterpret_cast<const T *>(k.Dinv) + vo;
  const int *Lp = k.Lp + po, *Rp = k.Rp + po;
  const int *nodes = k.lvl_nodes + vo;
  const int *lptr = k.lvl_ptr + k.lvl_off[inst];
  const int nlev = k.nlev[inst];
  const int tid = threadIdx.x;
  // forward: y_i -= sum_k L(i,k) y_k over the row pattern of i
  for (int l = 0; l < nlev; ++l) {
    const int a = lptr[l], b = lptr[l + 1];
    if (b - a >= NT / 2) {
      for (int idx = a + tid; idx < b; idx += NT) {
        const int i = nodes[idx];
        double t = y[i];
        for (int r = Rp[i]; r < Rp[i + 1]; ++r) t -= double(Lx[k.Rpos[r]]) * y[k.Rk[r]];
        y[i] = t;
      }
      bar_sync<NT>();
    } else {
      for (int idx = a; idx < b; ++idx) {
        const int i = nodes[idx];
        double t = 0.0;
        for (int r = Rp[i] + tid; r < Rp[i + 1]; r += NT)
          t += double(Lx[k.Rpos[r]]) * y[k.Rk[r]];
        t = block_sum<NT>(t, red);
        if (tid == 0) y[i] -= t;
        bar_sync<NT>();
      }
    }
  }
  for (int i = tid; i < N; i += NT) y[i] *= double(Dinv[i]);
  bar_sync<NT>();
  // backward: y_j -= sum_i L(i,j) y_i over column j (ancestors)
  for (int l = nlev - 1; l >= 0; --l) {
    const int a = lptr[l], b = lptr[l + 1];
    if (b - a >= NT / 2) {
      for (int idx = a + tid; idx < b; idx += NT) {
        const int j = nodes[idx];
        double t = y[j];
        for (int p = Lp[j]; p < Lp[j + 1]; ++p) t -= double(Lx[p]) * y[k.Li[p]];
        y[j] = t;
      }
      bar_sync<NT>();
    } else {
      for (int idx = a; idx < b; ++idx) {
        const int j = nodes[idx];
        double t = 0.0;
        for (int p = Lp[j] + tid; p < Lp[j + 1]; p += NT) t += double(Lx[p]) * y[k.Li[p]];
        t = block_sum<NT>(t, red);
        if (tid == 0) y[j] -= t;
        bar_sync<NT>();
      }
    }
  }
}

// e = b - K xi ; returns ||e||_inf (non-finite -> +inf)
template <int NT>
__device__ double refine_error(const KKTDev &k, int N, int po, const double *b,
                               const double *xi, double *e, double *red) {
  const int *Kp = k.Kp + po;
  double mx = 0;
  bool bad = false;
  for (int r = threadIdx.x; r < N; r += NT) {
    double t = 0;
    for (int p = Kp[r]; p < Kp[r + 1]; ++p) t += k.Kx[p] * xi[k.Kj[p]];
    double er = b[r] - t;
    e[r] = er;
    if (!isfinite(er)) bad = true;
    mx = fmax(mx, fabs(er));
  }
  mx = block_max<NT>(mx, red);
  double anybad = block_max<NT>(bad ? 1.0 : 0.0, red);
  return anybad > 0 ? CUDART_INF : mx;
}

template <typename T, int NT, bool SMEM>
__global__ void __launch_bounds__(NT) k_ldl_solve(KKTDev k, LDLParams prm, const int *run,
                                                  const double *rx, const double *rz,
                                                  double *lx, double *lz, int *ok) {
  int inst = blockIdx.x;
  if (!run[inst] || !ok[inst]) return;
  int N = k.N[inst];
  if (inst_class(N) != (SMEM ? 1 : 2)) return;
  __shared__ double red[NT / 32 + 1];
  extern __shared__ __align__(16) unsigned char sm_raw[];
  int vo = k.voff[inst], po = k.poff[inst];
  int tid = threadIdx.x;
  double *y = SMEM ? reinterpret_cast<double *>(sm_raw) : k.yf + vo;
  double *b = k.b + vo, *x = k.x + vo, *e = k.e + vo, *dx = k.dx + vo;
  const int *gs = k.gsrc + vo;
  double nb = 0;
  for (int i = tid; i < N; i += NT) {
    int g = gs[i];
    double v = g >= 0 ? rx[g] : (g == -1 ? 0.0 : rz[-g - 2]);
    b[i] = v;
    y[i] = v;
    nb = fmax(nb, fabs(v));
  }
  double normb = block_max<NT>(nb, red);
  bar_sync<NT>();
  ldl_trisolve<T, NT>(k, inst, N, vo, po, y, red);
  for (int i = tid; i < N; i += NT) x[i] = y[i];
  bar_sync<NT>();
  bool good = true;
  if (prm.ir_enable) {
    double norme = refine_error<NT>(k, N, po, b, x, e, red);
    if (!isfinite(norme)) good = false;
    for (int it = 0; good && it < prm.ir_maxiter; ++it) {
      if (norme <= prm.ir_abstol + prm.ir_reltol * normb) break;
      double last = norme;
      for (int i = tid; i < N; i += NT) y[i] = e[i];
      bar_sync<NT>();
      ldl_trisolve<T, NT>(k, inst, N, vo, po, y, red);
      for (int i = tid; i < N; i += NT) dx[i] = y[i] + x[i];
      bar_sync<NT>();
      norme = refine_error<NT>(k, N, po, b, dx, e, red);
      if (!isfinite(norme)) {
        good = false;
        break;
      }
      double ratio = last / norme;
      if (ratio < prm.ir_stopratio) {
        if (ratio > 1.0) {
          double *t = x;
          x = dx;
          dx = t;
        }
        break;
      }
      double *t = x;
      x = dx;
      dx = t;
    }
  } else {
    double bad = 0;
    for (int i = tid; i < N; i += NT)
      if (!isfinite(x[i])) bad = 1;
    if (block_max<NT>(bad, red) > 0) good = false;
  }
  if (!good) {
    if (tid == 0) ok[inst] = 0;
    return;
  }
  for (int i = tid; i < N; i += NT) {
    int g = gs[i];
    if (g >= 0) {
      if (lx) lx[g] = x[i];
    } else if (g <= -2) {
      if (lz) lz[-g - 2] = x[i];
    }
  }
}

// dynamic shared memory = the largest single-warp instance's work vector
template <typename T>
static void launch_factor(const KKTDev &k, const LDLParams &p, const int *run, int *ok,
                          double *eps_out, cudaStream_t st) {
  size_t sm = ((size_t)k.max_small_N * sizeof(double) + 15) & ~(size_t)15;
  if (k.has_small)
    k_ldl_factor<T, kSmallNT, true><<<k.B, kSmallNT, sm, st>>>(k, p, run, ok, eps_out);
  if (k.has_large)
    k_ldl_factor<T, kLargeNT, false><<<k.B, kLargeNT, 0, st>>>(k, p, run, ok, eps_out);
}
template <typename T>
static void launch_solve(const KKTDev &k, const LDLParams &p, const int *run,
                         const double *rx, const double *rz, double *lx, double *lz, int *ok,
                         cudaStream_t st) {
  size_t sm = ((size_t)k.max_small_N * sizeof(double) + 15) & ~(size_t)15;
  if (k.has_small)
    k_ldl_solve<T, kSmallNT, true><<<k.B, kSmallNT, sm, st>>>(k, p, run, rx, rz, lx, lz, ok);
  if (k.has_large)
    k_ldl_solve<T, kLargeNT, false><<<k.B, kLargeNT, 0, st>>>(k, p, run, rx, rz, lx, lz, ok);
}

static bool g_attr_done = false;
static void set_attrs() {
  if (g_attr_done) return;
  cudaFuncSetAttribute(k_ldl_factor<double, kSmallNT, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimitBytes);
  cudaFuncSetAttribute(k_ldl_factor<float, kSmallNT, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimitBytes);
  cudaFuncSetAttribute(k_ldl_solve<double, kSmallNT, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimitBytes);
  cudaFuncSetAttribute(k_ldl_solve<float, kSmallNT, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimitBytes);
  g_attr_done = true;
}

void ldl_factor(const KKTDev &k, bool fp32, const LDLParams &p, const int *run, int *ok,
                double *eps_out, cudaStream_t st) {
  set_attrs();
  if (fp32)
    launch_factor<float>(k, p, run, ok, eps_out, st);
  else
    launch_factor<double>(k, p, run, ok, eps_out, st);
}

void ldl_solve(const KKTDev &k, bool fp32, const LDLParams &p, const int *run,
               const double *rx, const double *rz, double *lx, double *lz, int *ok,
               cudaStream_t st) {
  set_attrs();
  if (fp32)
    launch_solve<float>(k, p, run, rx, rz, lx, lz, ok, st);
  else
    launch_solve<double>(k, p, run, rx, rz, lx, lz, ok, st);
}

}  // namespace clgpu
