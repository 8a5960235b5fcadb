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
#include "sn_exec.cuh"

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
// FP32 operations on FP32 values held in FP64 slots (the mixed form's
// elimination)
__device__ __forceinline__ double f32r(double x) { return double(float(x)); }
__device__ __forceinline__ double f32mul(double a, double b) {
  return double(__fmul_rn(float(a), float(b)));
}
__device__ __forceinline__ double f32add(double a, double b) {
  return double(__fadd_rn(float(a), float(b)));
}
__device__ __forceinline__ double f32sub(double a, double b) {
  return double(__fsub_rn(float(a), float(b)));
}
// the pivot the FP32 elimination continues with: its stored inverse
__device__ __forceinline__ double f32inv(double dj) {
  return double(float(1.0 / double(float(dj))));
}

template <typename T, int NT, bool SMEM, bool AR32 = false>
__global__ void __launch_bounds__(NT, NT == 32 ? 20 : 4) k_ldl_factor(KKTDev k, LDLParams prm, const int *run,
                                                   int *ok, double *eps_out) {
  int inst = blockIdx.x;
  if (!run[inst]) return;
  int N = k.N[inst];
  if (k.cls[inst] != (SMEM ? 1 : 2)) return;
  if (SMEM && k.has_fstream && k.fstream[inst]) return;  // streamed factorisation
  // AR32: FP32 arithmetic throughout (see k_ldl_factor_stream)
  static_assert(!AR32 || std::is_same<T, float>::value, "FP32 arithmetic stores FP32");
  constexpr bool F32 = AR32;
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
            if constexpr (F32)
              dj = f32add(f32r(k.Kx[p]), f32r(sg[j] > 0 ? eps : -eps));
            else
              dj = k.Kx[p] + (sg[j] > 0 ? eps : -eps);
            continue;
          }
          while (q < q1 && k.Li[q] != c) ++q;
          if (q < q1) Lacc[q] = F32 ? f32r(k.Kx[p]) : k.Kx[p];
        }
        for (int r = Rp[j]; r < Rp[j + 1]; ++r) {
          const int kk = k.Rk[r], pos = k.Rpos[r];
          const double ljk = Lacc[pos];
          double f;
          if constexpr (F32) {
            f = f32mul(ljk, Dacc[kk]);
            dj = f32sub(dj, f32mul(ljk, f));
          } else {
            f = ljk * Dacc[kk];
            dj -= ljk * f;
          }
          const int pe = Lp[kk + 1];
          q = q0;
          for (int p = pos + 1; p < pe; ++p) {
            const int i = k.Li[p];
            while (q < q1 && k.Li[q] != i) ++q;
            if (q < q1) {
              if constexpr (F32)
                Lacc[q] = f32sub(Lacc[q], f32mul(Lacc[p], f));
              else
                Lacc[q] -= Lacc[p] * f;
            }
          }
        }
        dj = pivot_value(dj, sg[j], prm);
        if (F32) dj = f32r(dj);
        const double dinv = F32 ? f32inv(dj) : 1.0 / dj;
        if (!isfinite(dinv)) finite = false;
        for (int qq = q0; qq < q1; ++qq)
          store_l(Lx, Lacc, qq, F32 ? f32mul(Lacc[qq], dinv) : Lacc[qq] * dinv);
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
            w[c] = F32 ? f32r(k.Kx[p]) : k.Kx[p];
          else if (c == j)
            w[c] = F32 ? f32add(f32r(k.Kx[p]), f32r(sg[j] > 0 ? eps : -eps))
                       : k.Kx[p] + (sg[j] > 0 ? eps : -eps);
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
            myf = F32 ? f32mul(myl, Dacc[kk]) : myl * Dacc[kk];
          }
          const int cnt = min(32, r1 - rb);
          for (int t = 0; t < cnt; ++t) {
            const int pos = __shfl_sync(0xffffffffu, mypos, t);
            const int pe = __shfl_sync(0xffffffffu, myend, t);
            const double f = __shfl_sync(0xffffffffu, myf, t);
            const double ljk = __shfl_sync(0xffffffffu, myl, t);
            if constexpr (F32) {
              if (tid == 0) w[j] = f32sub(w[j], f32mul(ljk, f));
              for (int p = pos + 1 + tid; p < pe; p += NT)
                w[k.Li[p]] = f32sub(w[k.Li[p]], f32mul(Lacc[p], f));
            } else {
              if (tid == 0) w[j] -= ljk * f;
              for (int p = pos + 1 + tid; p < pe; p += NT) w[k.Li[p]] -= Lacc[p] * f;
            }
            bar_sync<NT>();
          }
        }
        double dj = pivot_value(w[j], sg[j], prm);
        if (F32) dj = f32r(dj);
        const double dinv = F32 ? f32inv(dj) : 1.0 / dj;
        if (!isfinite(dinv)) finite = false;
        for (int q = Lp[j] + tid; q < Lp[j + 1]; q += NT) {
          const int i = k.Li[q];
          store_l(Lx, Lacc, q, F32 ? f32mul(w[i], dinv) : w[i] * dinv);
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
  // copies of L in the order the substitutions read it (every level ended
  // with a barrier, so all of Lx is written): level-ordered streams for the
  // single-warp solve, row order for the block solve
  if (SMEM) {
    T *LxF = reinterpret_cast<T *>(k.LxF), *LxB = reinterpret_cast<T *>(k.LxB);
    for (int r = Lp[0] + tid; r < Lp[N]; r += NT) {
      LxF[r] = Lx[k.fpos[r]];
      LxB[r] = Lx[k.bpos[r]];
    }
  } else {
    T *LxR = reinterpret_cast<T *>(k.LxR);
    const int rbeg = Rp[0], rend = Rp[N];
    for (int r = rbeg + tid; r < rend; r += NT) LxR[r] = Lx[k.Rpos[r]];
  }
  double bad = block_max<NT>(finite ? 0.0 : 1.0, red);
  if (k.prof_bytes && tid == 0) {
    // algorithmic bytes: K (indices + values) and the symbolic structure read
    // once, L, D, D^-1 and the substitution copies of L written once
    const double nl = Lp[N] - Lp[0], nk = Kp[N] - Kp[0], ts = sizeof(T);
    k.prof_bytes[inst] += 12.0 * nk + 16.0 * N + 12.0 * nl + ts * (nl + 2.0 * N) +
                          (SMEM ? nl * (8.0 + 2.0 * ts) : nl * (4.0 + ts));
  }
  if (tid == 0) {
    if (bad > 0) ok[inst] = 0;
    if (eps_out) eps_out[inst] = eps;
  }
}

// One node at a time over a run of consecutive narrow levels [a, e) of a
// schedule: y[node] -= sum_r V[r] * y[I[r]] over the node's entries
// [s.y, s.z), the block sharing each sum.  Nothing but y depends on the
// previous node, so each thread loads its first entry of the NEXT node (and
// that node's schedule record) before it reduces the current one; thread t
// accumulates entries s.y + t, s.y + t + NT, ... in order, as a plain loop
// would, so the result does not depend on the prefetch.
template <typename T, int NT>
__device__ __forceinline__ void narrow_run(const int4 *__restrict__ sched, int a, int e,
                                           const T *__restrict__ V,
                                           const int *__restrict__ I, double *y,
                                           double *red, int tid) {
  int4 s = sched[a];
  double pv = 0.0;
  int pk = -1;
  if (s.y + tid < s.z) {
    pv = double(V[s.y + tid]);
    pk = I[s.y + tid];
  }
  for (int idx = a; idx < e; ++idx) {
    int4 sn = make_int4(0, 0, 0, 0);
    if (idx + 1 < e) sn = sched[idx + 1];
    double nv = 0.0;
    int nk = -1;
    if (sn.y + tid < sn.z) {
      nv = double(V[sn.y + tid]);
      nk = I[sn.y + tid];
    }
    double t = 0.0;
    if (pk >= 0) t += pv * y[pk];
    for (int r = s.y + tid + NT; r < s.z; r += NT) t += double(V[r]) * y[I[r]];
    t = block_sum<NT>(t, red);
    if (tid == 0) y[s.x] -= t;
    bar_sync<NT>();
    s = sn;
    pv = nv;
    pk = nk;
  }
}

// y <- L^{-T} D^{-1} L^{-1} y, level-scheduled gathers.  Wide levels: one
// thread per node walks the node's row (forward) or column (backward).
// Runs of narrow levels: narrow_run.
template <typename T, int NT>
__device__ void ldl_trisolve(const KKTDev &k, int inst, int N, int vo, double *y,
                             double *red, int tid) {
  const T *Lx = reinterpret_cast<const T *>(k.Lx);
  const T *LxR = reinterpret_cast<const T *>(k.LxR);
  const T *Dinv = reinterpret_cast<const T *>(k.Dinv) + vo;
  const int4 *fs = k.fsched + vo, *bs = k.bsched + vo;
  const int *lptr = k.lvl_ptr + k.lvl_off[inst];
  const int nlev = k.nlev[inst];
  // forward: y_i -= sum_k L(i,k) y_k over the row pattern of i
  for (int l = 0; l < nlev;) {
    const int a = lptr[l], b = lptr[l + 1];
    if (b - a >= NT / 2) {
      for (int idx = a + tid; idx < b; idx += NT) {
        const int4 sc = fs[idx];
        double t = y[sc.x];
        for (int r = sc.y; r < sc.z; ++r) t -= double(LxR[r]) * y[k.Rk[r]];
        y[sc.x] = t;
      }
      bar_sync<NT>();
      ++l;
      continue;
    }
    int l2 = l + 1;
    while (l2 < nlev && lptr[l2 + 1] - lptr[l2] < NT / 2) ++l2;
    narrow_run<T, NT>(fs, a, lptr[l2], LxR, k.Rk, y, red, tid);
    l = l2;
  }
  for (int i = tid; i < N; i += NT) y[i] *= double(Dinv[i]);
  bar_sync<NT>();
  // backward: y_j -= sum_i L(i,j) y_i over column j (ancestors), root first
  for (int l = nlev - 1; l >= 0;) {
    const int a = N - lptr[l + 1], b = N - lptr[l];
    if (b - a >= NT / 2) {
      for (int idx = a + tid; idx < b; idx += NT) {
        const int4 sc = bs[idx];
        double t = y[sc.x];
        for (int p = sc.y; p < sc.z; ++p) t -= double(Lx[p]) * y[k.Li[p]];
        y[sc.x] = t;
      }
      bar_sync<NT>();
      --l;
      continue;
    }
    int l2 = l - 1;
    while (l2 >= 0 && lptr[l2 + 1] - lptr[l2] < NT / 2) --l2;
    narrow_run<T, NT>(bs, a, N - lptr[l2 + 1], Lx, k.Li, y, red, tid);
    l = l2;
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
__global__ void __launch_bounds__(NT, NT == 32 ? 20 : 4) k_ldl_solve(KKTDev k, LDLParams prm, const int *run,
                                                  const double *rx, const double *rz,
                                                  double *lx, double *lz, int *ok) {
  int inst = blockIdx.x;
  if (!run[inst] || !ok[inst]) return;
  int N = k.N[inst];
  if (k.cls[inst] != (SMEM ? 1 : 2)) return;
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
  ldl_trisolve<T, NT>(k, inst, N, vo, y, red, tid);
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
      ldl_trisolve<T, NT>(k, inst, N, vo, y, red, tid);
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

// ------------------------------------------------------------------------
// Single-warp solve.  Each substitution pass, and the refinement residual,
// streams its nonzeros in chunks of at most kSChunk entries of one level.
// None of a chunk's entries or values depends on earlier results, so they
// are copied into a shared-memory ring kSRing chunks ahead with cp.async: the
// warp's global-memory latency overlaps the reduction of the chunks before.
// Within a chunk the products are summed per segment (a node of the pass,
// or a KKT row) by a segmented warp scan; a segment running into the next
// chunk of the same level carries its partial sum across, so every segment
// is written once.  Chunks never straddle a level, and a level's writes are
// complete (__syncwarp) before the next level gathers them.  The summation
// order depends only on the instance's own layout, never on the batch.

constexpr int kSRing = kSRingSlots;

template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem_dst, const void *gsrc) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(gsrc), "n"(BYTES));
}

// The stream kernels spell their products and sums with __dmul_rn /
// __dadd_rn / __dsub_rn: the compiler never fuses those into FMAs, so every
// value is rounded the same way whatever the surrounding code (one or two
// right-hand sides, unrolling), and results do not depend on code shape.

// Segmented sums of one chunk held two entries per lane: A = entry 2 lane,
// B = entry 2 lane + 1, with products xA, xB and positions in their segments
// pA, pB (clamped to 63).  Returns sA / sB: the sum of A's / B's segment from
// its start up to A / B, including lower lanes and, for a segment continued
// from the previous chunk, the carry.  The lane scan runs over each lane's
// tail value (its part of B's segment); a lane adds lane l-d's value while
// d does not pass the lane that holds the start of B's segment.  After the
// steps d = 1 .. 2^(s-1) a lane has summed min(reach, 2^s - 1) lanes back, so
// the chunk's nsteps (from its chunk word, the same on every lane) steps
// complete every segment and the remaining steps are skipped.
__device__ __forceinline__ void seg_scan2(double xA, double xB, int pA, int pB, int lane,
                                          double carry, int nsteps, double &sA, double &sB) {
  if (lane == 0 && pA > 0) xA = __dadd_rn(xA, carry);
  double v = pB > 0 ? __dadd_rn(xA, xB) : xB;
  const int reach = pB > 0 ? lane - ((2 * lane + 1 - pB) >> 1) : 0;  // lanes back
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    if (s >= nsteps) break;
    const int d = 1 << s;
    const double o = __shfl_up_sync(0xffffffffu, v, d);
    if (d <= reach && d <= lane) v = __dadd_rn(v, o);
  }
  sB = v;
  const double prev = __shfl_up_sync(0xffffffffu, v, 1);
  sA = (pA > 0 && lane > 0) ? __dadd_rn(xA, prev) : xA;
}
// The same scan in FP32 arithmetic (the mixed form's factorisation).
__device__ __forceinline__ void seg_scan2(float xA, float xB, int pA, int pB, int lane,
                                          float carry, int nsteps, float &sA, float &sB) {
  if (lane == 0 && pA > 0) xA = __fadd_rn(xA, carry);
  float v = pB > 0 ? __fadd_rn(xA, xB) : xB;
  const int reach = pB > 0 ? lane - ((2 * lane + 1 - pB) >> 1) : 0;
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    if (s >= nsteps) break;
    const int d = 1 << s;
    const float o = __shfl_up_sync(0xffffffffu, v, d);
    if (d <= reach && d <= lane) v = __fadd_rn(v, o);
  }
  sB = v;
  const float prev = __shfl_up_sync(0xffffffffu, v, 1);
  sA = (pA > 0 && lane > 0) ? __fadd_rn(xA, prev) : xA;
}

// Segmented sums of one solve chunk held kSK consecutive entries per lane
// (entries kSK lane .. kSK lane + kSK - 1), with products x and positions in
// their segments p (clamped to kSPosMax, zero for entries past the chunk).
// Returns s: for every entry the sum of its segment from the segment's start
// up to the entry, including lower lanes and, for a segment continued from
// the previous chunk, the carry.  Each lane first sums its own entries
// (a segment restarts where p = 0), the lane scan then runs over each lane's
// tail value with the reach rule of seg_scan2, and an entry whose segment
// began below its lane (p > its index in the lane) adds the lower lane's
// total.  nsteps doubling steps complete every segment of the chunk.
__device__ __forceinline__ void seg_scan4(double (&x)[kSK], const int (&p)[kSK], int lane,
                                          double carry, int nsteps, double (&s)[kSK]) {
  if (lane == 0 && p[0] > 0) x[0] = __dadd_rn(x[0], carry);
  s[0] = x[0];
#pragma unroll
  for (int j = 1; j < kSK; ++j) s[j] = p[j] > 0 ? __dadd_rn(s[j - 1], x[j]) : x[j];
  double v = s[kSK - 1];
  const int pt = p[kSK - 1];
  const int reach = pt > 0 ? lane - ((kSK * lane + kSK - 1 - pt) >> kSKShift) : 0;
#pragma unroll
  for (int t = 0; t < 5; ++t) {
    if (t >= nsteps) break;
    const int d = 1 << t;
    const double o = __shfl_up_sync(0xffffffffu, v, d);
    if (d <= reach && d <= lane) v = __dadd_rn(v, o);
  }
  const double prev = __shfl_up_sync(0xffffffffu, v, 1);
#pragma unroll
  for (int j = 0; j < kSK - 1; ++j)
    if (p[j] > j && lane > 0) s[j] = __dadd_rn(s[j], prev);
  s[kSK - 1] = v;
}

// Ring slot layout of the 8-byte items (entries, FP64 values) of a solve
// chunk: lane l holds entries 4l .. 4l+3, which it reads as two 16-byte
// pairs; pair (4l, 4l+1) is stored in 16-byte unit l and pair (4l+2, 4l+3)
// in unit 32 + l, so each of the two reads is contiguous across the warp
// (conflict-free) instead of striding 32 bytes (two-way conflicts).
__device__ __forceinline__ int ring_pos8(int e) {
  return 2 * (((e >> 1) & 1) * 32 + (e >> 2)) + (e & 1);
}
// lane's kSK values of the ring as FP64 (two 16-byte or one 16-byte shared
// load); FP32 values keep the plain order (one contiguous float4 per lane)
__device__ __forceinline__ void ring_vals(const double *rv, int lane, double (&v)[kSK]) {
  const double2 a = reinterpret_cast<const double2 *>(rv)[lane];
  const double2 b = reinterpret_cast<const double2 *>(rv)[32 + lane];
  v[0] = a.x;
  v[1] = a.y;
  v[2] = b.x;
  v[3] = b.y;
}
__device__ __forceinline__ void ring_vals(const float *rv, int lane, double (&v)[kSK]) {
  const float4 a = reinterpret_cast<const float4 *>(rv)[lane];
  v[0] = a.x;
  v[1] = a.y;
  v[2] = a.z;
  v[3] = a.w;
}

// One pass over an encoded stream (entries ent / values val from stream
// position base), chunk by chunk as listed in chunks[0..nch), for each
// right-hand side r < NR whose bit is set in act:
//   RESID = false:  y_r[seg] -= sum val * y_r[idx]     (out_r == y_r)
//   RESID = true:   out_r[seg] = sum val * y_r[idx]
// A chunk's entries and values are read once for all right-hand sides; each
// side's arithmetic is exactly that of a single-side pass.  Chunk words are
// read 32 at a time, one per lane, two blocks ahead of use.  The ring copies
// are coalesced (lane l copies entries l, l + 32, ...); each lane then reads
// its kSK consecutive entries with 16-byte shared loads.
template <typename T, bool RESID, int NR>
__device__ void ring_pass(const int *__restrict__ chunks, int nch, int base,
                          const int2 *__restrict__ ent, const T *__restrict__ val,
                          double *const (&yin)[NR], double *const (&outin)[NR], int2 *re, T *rv,
                          int lane, unsigned act) {
  static_assert(kSK == 4, "ring_pass reads four entries per lane");
  const unsigned full = 0xffffffffu;
  if (nch == 0) return;
  // register copies of the side pointers (the caller's arrays may live in
  // local memory; every index below is a compile-time constant)
  double *y[NR], *out[NR];
  bool on[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    y[r] = yin[r];
    out[r] = outin[r];
    on[r] = (act >> r) & 1u;
  }
  int d0 = lane < nch ? chunks[lane] : 0;
  int d1 = lane + 32 < nch ? chunks[lane + 32] : 0;
  int d2 = lane + 64 < nch ? chunks[lane + 64] : 0;
  int blk = 0;  // d0 holds chunks [32 blk, 32 blk + 32)
  auto word = [&](int c) {
    const int r = c - 32 * blk;  // 0 <= r < 64
    return (unsigned)__shfl_sync(full, r < 32 ? d0 : d1, r & 31);
  };
  auto issue = [&](int c, int slot) {
    if (c < nch) {
      const unsigned w = word(c);
      const int p = base + (int)(w & kStartMask);
      const int cnt = (int)((w >> kCntShift) & 127u) + 1;
      int2 *rd = re + slot * kSChunk;
      T *vd = rv + slot * kSChunk;
#pragma unroll
      for (int h = 0; h < kSK; ++h) {
        const int e = lane + 32 * h;
        if (e < cnt) {
          const int pe = ring_pos8(e);
          cp_async<8>(&rd[pe], &ent[p + e]);
          cp_async<sizeof(T)>(&vd[sizeof(T) == 8 ? pe : e], &val[p + e]);
        }
      }
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };
#pragma unroll
  for (int c = 0; c < kSRing; ++c) issue(c, c);
  double carry[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) carry[r] = 0.0;
  unsigned wnext = word(0);  // each chunk's word is read one chunk ahead
  for (int c = 0; c < nch; ++c) {
    if (c > 0 && (c & 31) == 0) {
      ++blk;
      d0 = d1;
      d1 = d2;
      const int q = 32 * (blk + 2) + lane;
      d2 = q < nch ? chunks[q] : 0;
    }
    const unsigned wc = wnext;
    const int cnt = (int)((wc >> kCntShift) & 127u) + 1;
    const int nsteps = (int)((wc >> kStepShift) & 7u);
    asm volatile("cp.async.wait_group %0;\n" ::"n"(kSRing - 1));
    __syncwarp();
    const int slot = c & (kSRing - 1);
    const int4 *r4 = reinterpret_cast<const int4 *>(re + slot * kSChunk);
    const int4 ea = r4[lane], eb = r4[32 + lane];
    const int sg[kSK] = {ea.x, ea.z, eb.x, eb.z};
    const int ix[kSK] = {ea.y, ea.w, eb.y, eb.w};
    double vv[kSK];
    ring_vals(rv + slot * kSChunk, lane, vv);
    int p[kSK], gi[kSK];
    bool ok[kSK], wr[kSK];
#pragma unroll
    for (int j = 0; j < kSK; ++j) {
      ok[j] = kSK * lane + j < cnt;
      p[j] = ok[j] ? (sg[j] >> 16) & kSPosMax : 0;
      gi[j] = ok[j] ? ix[j] : 0;
      wr[j] = ok[j] && ((sg[j] >> kSLastBit) & 1);
    }
    const int jl = (cnt - 1) & (kSK - 1), ll = (cnt - 1) >> kSKShift;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      if (!on[r]) continue;
      double x[kSK], sm[kSK], yo[kSK];
      // a segment's target is written once per pass, by its last entry, so
      // its old value can be read before the scan, off the dependent chain
      if (!RESID) {
#pragma unroll
        for (int j = 0; j < kSK; ++j) yo[j] = wr[j] ? out[r][sg[j] & 0xffff] : 0.0;
      }
#pragma unroll
      for (int j = 0; j < kSK; ++j) {
        const double yv = y[r][gi[j]];
        x[j] = ok[j] ? __dmul_rn(vv[j], yv) : 0.0;
      }
      seg_scan4(x, p, lane, carry[r], nsteps, sm);
#pragma unroll
      for (int j = 0; j < kSK; ++j)
        if (wr[j]) {
          if (RESID)
            out[r][sg[j] & 0xffff] = sm[j];
          else
            out[r][sg[j] & 0xffff] = __dsub_rn(yo[j], sm[j]);
        }
      // partial sum of the segment of the chunk's last entry (used by the
      // next chunk only if its first entry continues that segment)
      const double cs = jl == 0 ? sm[0] : jl == 1 ? sm[1] : jl == 2 ? sm[2] : sm[3];
      carry[r] = __shfl_sync(full, cs, ll);
    }
    __syncwarp();
    issue(c + kSRing, slot);
    if (c + 1 < nch) wnext = word(c + 1);  // before the block rotation: c + 1 - 32 blk <= 32
  }
  asm volatile("cp.async.wait_all;\n" ::);
  __syncwarp();
}

// Vector loops of the single-warp solve: each lane handles elements
// lane, lane + 32, ...; kVecU of them are loaded before any is used so the
// loads of one lane are in flight together rather than one round trip each.
constexpr int kVecU = 8;
#define VEC_LOOP(i, N, BODY_LOAD, BODY_USE)                       \
  for (int i##0 = lane; i##0 < (N); i##0 += 32 * kVecU) {         \
    _Pragma("unroll") for (int u = 0; u < kVecU; ++u) {           \
      const int i = i##0 + 32 * u;                                \
      if (i < (N)) { BODY_LOAD }                                  \
    }                                                             \
    _Pragma("unroll") for (int u = 0; u < kVecU; ++u) {           \
      const int i = i##0 + 32 * u;                                \
      if (i < (N)) { BODY_USE }                                   \
    }                                                             \
  }

// Right-hand sides of one solve launch: side r gathers its rhs from rx[r] /
// rz[r] and scatters its solution to lx[r] / lz[r] (either may be null).
template <int NR>
struct SolveIO {
  const double *rx[NR], *rz[NR];
  double *lx[NR], *lz[NR];
};

// Warps of a block solve different instances (the packing tables); they
// share nothing but the block's shared memory, each in its own slice, and
// never synchronise with one another.  A warp solves NR right-hand sides with
// one factor: every stream pass serves all sides still refining, and each
// side follows the refinement rules on its own, so its result is exactly
// that of a single-side solve.
template <typename T, int NR>
__global__ void __launch_bounds__(32 * kSolveWarps, kSolveBlocksPerSM)
    k_ldl_solve_warp(KKTDev k, LDLParams prm, const int *run, SolveIO<NR> io, int *ok) {
  const int slot = blockIdx.x * kSolveWarps + (threadIdx.x >> 5);
  const int inst = NR == 1 ? k.spack_inst[slot] : k.spack2_inst[slot];
  if (inst < 0 || !run[inst] || !ok[inst]) return;
  const int N = k.N[inst];
  extern __shared__ __align__(16) unsigned char sm_raw[];
  unsigned char *smw = sm_raw + (NR == 1 ? k.spack_off[slot] : k.spack2_off[slot]);
  const size_t ybytes = ((size_t)N * 8 + 15) & ~(size_t)15;
  double *y[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) y[r] = reinterpret_cast<double *>(smw + r * ybytes);
  int2 *re = reinterpret_cast<int2 *>(smw + NR * ybytes);
  T *rv = reinterpret_cast<T *>(re + kSRing * kSChunk);
  const int vo = k.voff[inst], po = k.poff[inst], lane = threadIdx.x & 31;
  double *b[NR], *x[NR], *e[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    b[r] = (r == 0 ? k.b : k.b2) + vo;
    x[r] = (r == 0 ? k.x : k.x2) + vo;
    e[r] = (r == 0 ? k.e : k.e2) + vo;
  }
  const int *__restrict__ gs = k.gsrc + vo;
  const int lbase = k.Lp[po], kbase = k.Kp[po];
  const int *fch = k.fch + k.fch_off[inst], *bch = k.bch + k.bch_off[inst],
            *kch = k.kch + k.kch_off[inst];
  const int nfch = k.fch_off[inst + 1] - k.fch_off[inst];
  const int nbch = k.bch_off[inst + 1] - k.bch_off[inst];
  const int nkch = k.kch_off[inst + 1] - k.kch_off[inst];
  const T *LxF = reinterpret_cast<const T *>(k.LxF), *LxB = reinterpret_cast<const T *>(k.LxB);
  const T *__restrict__ Dinv = reinterpret_cast<const T *>(k.Dinv) + vo;
  double normb[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    const double *__restrict__ rx = io.rx[r], *__restrict__ rz = io.rz[r];
    double nb = 0;
    int g[kVecU];
    double v[kVecU];
    for (int i0 = lane; i0 < N; i0 += 32 * kVecU) {
#pragma unroll
      for (int u = 0; u < kVecU; ++u) {
        const int i = i0 + 32 * u;
        g[u] = i < N ? gs[i] : -1;
      }
#pragma unroll
      for (int u = 0; u < kVecU; ++u)
        v[u] = g[u] >= 0 ? rx[g[u]] : (g[u] == -1 ? 0.0 : rz[-g[u] - 2]);
#pragma unroll
      for (int u = 0; u < kVecU; ++u) {
        const int i = i0 + 32 * u;
        if (i < N) {
          b[r][i] = v[u];
          y[r][i] = v[u];
          nb = fmax(nb, fabs(v[u]));
        }
      }
    }
    normb[r] = warp_max(nb);
  }
  __syncwarp();
  double tv[kVecU];
  int ntri = 0, nres = 0, nir = 0;  // side-passes (profiling)
  auto popc = [](unsigned m) { return __popc(m); };
  auto trisolve = [&](unsigned m) {
    ntri += popc(m);
    ring_pass<T, false, NR>(fch, nfch, lbase, k.fent, LxF, y, y, re, rv, lane, m);
#pragma unroll
    for (int r = 0; r < NR; ++r)
      if ((m >> r) & 1u) {
        double *yr = y[r];
        VEC_LOOP(i, N, tv[u] = double(Dinv[i]);, yr[i] *= tv[u];)
      }
    __syncwarp();
    ring_pass<T, false, NR>(bch, nbch, lbase, k.bent, LxB, y, y, re, rv, lane, m);
  };
  // e_r = b_r - K y_r; norme[r] = ||e_r||_inf (+inf when not finite)
  auto residual = [&](unsigned m, double (&norme)[NR]) {
    nres += popc(m);
    ring_pass<double, true, NR>(kch, nkch, kbase, k.kent, k.Kx, y, e, re,
                                reinterpret_cast<double *>(rv), lane, m);
    __syncwarp();
#pragma unroll
    for (int r = 0; r < NR; ++r)
      if ((m >> r) & 1u) {
        double mx = 0.0;
        bool bad = false;
        double tb[kVecU];
        double *br = b[r], *er = e[r];
        VEC_LOOP(i, N, tb[u] = br[i]; tv[u] = er[i];, {
          const double ev = tb[u] - tv[u];
          er[i] = ev;
          if (!isfinite(ev)) bad = true;
          mx = fmax(mx, fabs(ev));
        })
        __syncwarp();
        mx = warp_max(mx);
        norme[r] = __any_sync(0xffffffffu, bad) ? CUDART_INF : mx;
      }
  };
  // The per-side loops of the refinement stay rolled (unroll 1): with them
  // unrolled, the two-side build skipped every refinement sweep (its results
  // then differed from the one-side solve's); rolled, each side's result is
  // bitwise that of the one-side kernel, which the two-side parity test checks.
  const unsigned all = (1u << NR) - 1u;
  trisolve(all);
  bool good = true;
  if (prm.ir_enable) {
    // x keeps the accepted iterate; y holds the candidate the residual reads
    double norme[NR], last[NR];
    residual(all, norme);
    unsigned m = 0;
#pragma unroll 1
    for (int r = 0; r < NR; ++r) {
      for (int i = lane; i < N; i += 32) x[r][i] = y[r][i];
      if (!isfinite(norme[r]))
        good = false;
      else
        m |= 1u << r;
    }
    __syncwarp();
    if (!good) m = 0;
    for (int it = 0; m && it < prm.ir_maxiter; ++it) {
#pragma unroll 1
      for (int r = 0; r < NR; ++r)
        if (((m >> r) & 1u) && norme[r] <= prm.ir_abstol + prm.ir_reltol * normb[r])
          m &= ~(1u << r);
      if (!m) break;
#pragma unroll 1
      for (int r = 0; r < NR; ++r)
        if ((m >> r) & 1u) {
          last[r] = norme[r];
          ++nir;
          double *yr = y[r], *er = e[r];
          VEC_LOOP(i, N, tv[u] = er[i];, yr[i] = tv[u];)
        }
      __syncwarp();
      trisolve(m);
#pragma unroll 1
      for (int r = 0; r < NR; ++r)
        if ((m >> r) & 1u) {
          double *yr = y[r], *xr = x[r];
          VEC_LOOP(i, N, tv[u] = xr[i];, yr[i] += tv[u];)
        }
      __syncwarp();
      residual(m, norme);
#pragma unroll 1
      for (int r = 0; r < NR; ++r)
        if ((m >> r) & 1u) {
          if (!isfinite(norme[r])) {
            good = false;
            m &= ~(1u << r);
            continue;
          }
          // kktsolver_directldl_gpu.jl:390-400: keep the candidate if it
          // improved on the last error; stop when the improvement ratio is
          // below stopratio
          const double ratio = last[r] / norme[r];
          if (ratio > 1.0 || ratio >= prm.ir_stopratio)
            for (int i = lane; i < N; i += 32) x[r][i] = y[r][i];
          if (ratio < prm.ir_stopratio) m &= ~(1u << r);
        }
      __syncwarp();
      if (!good) break;
    }
  } else {
    bool bad = false;
#pragma unroll 1
    for (int r = 0; r < NR; ++r)
      for (int i = lane; i < N; i += 32) {
        x[r][i] = y[r][i];
        if (!isfinite(y[r][i])) bad = true;
      }
    if (__any_sync(0xffffffffu, bad)) good = false;
    __syncwarp();
  }
  if (k.prof_bytes && lane == 0) {
    // algorithmic bytes: every stream pass reads its entries, values and
    // chunk words once per side-pass; vectors are read / written once per use
    const double nl = k.Lp[po + N] - lbase, nk = k.Kp[po + N] - kbase, ts = sizeof(T);
    k.prof_bytes[(NR == 1 ? 1 : 2) * (size_t)k.B + inst] +=
        NR * 20.0 * N                                               // rhs gather, b
        + ntri * (2.0 * nl * (8 + ts) + 4.0 * (nfch + nbch) + ts * N)  // substitutions
        + nres * (16.0 * nk + 4.0 * nkch + 24.0 * N)                // residuals
        + nir * 24.0 * N + NR * 8.0 * N                             // refinement vectors
        + NR * 20.0 * N;                                            // result scatter
  }
  if (!good) {
    if (lane == 0) ok[inst] = 0;
    return;
  }
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    double *lx = io.lx[r], *lz = io.lz[r], *xr = x[r];
    int g[kVecU];
    VEC_LOOP(i, N, g[u] = gs[i]; tv[u] = xr[i];, {
      if (g[u] >= 0) {
        if (lx) lx[g[u]] = tv[u];
      } else if (g[u] <= -2) {
        if (lz) lz[-g[u] - 2] = tv[u];
      }
    })
  }
}
#undef VEC_LOOP

// ------------------------------------------------------------------------
// Streamed factorisation, one instance per block of kFactorWarps warps.
// Shared memory holds V = [d_j, then 1/d_j once pivot j is taken (N) | U = L D
// (nnz(L))], initialised from the KKT matrix (static regularisation on the
// diagonal), and one cp.async ring per warp.  Each warp streams its own part
// of every level: op chunks subtract V[a] V[b] V[k] from V[t] through a
// segmented warp scan (the carry rule of the substitutions; a part never
// splits a target's updates, so each V[t] has one writer), pivot chunks take
// the warp's pivots of the level (dynamic regularisation, D and D^-1 in the
// storage type, 1/d_j kept in V).  The block synchronises after a level's
// updates (its pivots read them) and after its pivots (the next level's
// updates read them).  Updates of a level only read columns and pivots of
// lower levels, all final.  At the end L = U / d is written in CSC order and
// in the two substitution-stream orders.
// T is the storage type of L, D and D^-1.  AR32 (with T = float) is the
// mixed form: the factorisation itself runs in FP32 arithmetic (the KKT
// values rounded to FP32, every product, sum and pivot inverse an FP32
// operation; V keeps FP32 values in its FP64 slots), as the FP32 sparse
// factorisation of the reference's mixed form does.  T = float without
// AR32 eliminates in FP64 and stores the factor in FP32.
constexpr int kFRing = kFRingSlots;

template <typename T, bool AR32 = false>
__global__ void __launch_bounds__(32 * kFactorWarps, 6)
    k_ldl_factor_stream(KKTDev k, LDLParams prm, const int *run, int *ok, double *eps_out) {
  constexpr int NT = 32 * kFactorWarps;
  static_assert(!AR32 || std::is_same<T, float>::value, "FP32 arithmetic stores FP32");
  constexpr bool F32 = AR32;
  using A = typename std::conditional<AR32, float, double>::type;  // elimination arithmetic
  const int inst = k.fs_inst[blockIdx.x];
  if (!run[inst]) return;  // the whole block
  __shared__ double red[kFactorWarps + 1];
  const unsigned full = 0xffffffffu;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int N = k.N[inst], vo = k.voff[inst], po = k.poff[inst];
  const int lbase = k.Lp[po], nl = k.Lp[po + N] - lbase;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  double *V = reinterpret_cast<double *>(sm_raw);
  uint2 *ring = reinterpret_cast<uint2 *>(sm_raw + (((size_t)(N + nl) * 8 + 15) & ~(size_t)15)) +
                warp * kFRing * kChunk;
  const signed char *sg = k.Dsign + vo;
  const int *Kdiag = k.Kdiag + vo;
  T *D = reinterpret_cast<T *>(k.D) + vo;
  T *Dinv = reinterpret_cast<T *>(k.Dinv) + vo;
  // diagonal of K into V (loads of kU elements in flight per thread), then
  // the static regularisation eps = c + prop * max |diag(K)| on it
  constexpr int kU = 8;
  double mx = 0.0;
  for (int j0 = tid; j0 < N; j0 += NT * kU) {
    int kd[kU];
    double kv[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) kd[u] = j0 + NT * u < N ? Kdiag[j0 + NT * u] : -1;
#pragma unroll
    for (int u = 0; u < kU; ++u) kv[u] = kd[u] >= 0 ? k.Kx[kd[u]] : 0.0;
#pragma unroll
    for (int u = 0; u < kU; ++u)
      if (kd[u] >= 0) {
        V[j0 + NT * u] = F32 ? double(float(kv[u])) : kv[u];
        mx = fmax(mx, fabs(kv[u]));
      }
  }
  double eps = 0.0;
  mx = block_max<NT>(mx, red);  // synchronises the block
  if (prm.static_reg) eps = prm.static_c + prm.static_prop * mx;
  if constexpr (F32) {
    const float ef = float(eps);
    for (int j = tid; j < N; j += NT) V[j] = double(__fadd_rn(float(V[j]), sg[j] > 0 ? ef : -ef));
  } else {
    for (int j = tid; j < N; j += NT) V[j] += sg[j] > 0 ? eps : -eps;
  }
  {
    const int *kp = k.Lkpos + lbase;
    int pos[8];
    for (int e0 = tid; e0 < nl; e0 += NT * 8) {
#pragma unroll
      for (int u = 0; u < 8; ++u) pos[u] = e0 + NT * u < nl ? kp[e0 + NT * u] : -1;
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (e0 + NT * u < nl) {
          const double kx = pos[u] >= 0 ? k.Kx[pos[u]] : 0.0;
          V[N + e0 + NT * u] = F32 ? double(float(kx)) : kx;
        }
    }
  }
  __syncthreads();
  // ---- this warp's op / pivot stream, level by level
  const int *wo = k.fwoff + (size_t)inst * (kFactorWarps + 1);
  const int *chunks = k.foch + wo[warp];
  const int nch = wo[warp + 1] - wo[warp];
  const uint2 *ops = k.fop + k.fop_base[inst];
  const int *lc = k.flcnt + (size_t)k.lvl_off[inst] * kFactorWarps + warp;
  const int nlev = k.nlev[inst];
  bool finite = true;
  double nent = 0.0;  // stream entries (profiling)
  int d0 = lane < nch ? chunks[lane] : 0;
  int d1 = lane + 32 < nch ? chunks[lane + 32] : 0;
  int d2 = lane + 64 < nch ? chunks[lane + 64] : 0;
  int blk = 0;
  auto word = [&](int c) {
    const int r = c - 32 * blk;
    return (unsigned)__shfl_sync(full, r < 32 ? d0 : d1, r & 31);
  };
  auto issue = [&](int c, int slot) {
    if (c < nch) {
      const unsigned w = word(c);
      const int p0 = (int)(w & kStartMask), cnt = (int)((w >> kCntShift) & 63u) + 1;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int e = 2 * lane + h;
        if (e < cnt) {
          const unsigned dst =
              static_cast<unsigned>(__cvta_generic_to_shared(&ring[slot * kChunk + h * 32 + lane]));
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst),
                       "l"(&ops[p0 + e]));
        }
      }
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };
#pragma unroll
  for (int c = 0; c < kFRing; ++c) issue(c, c);
  int c = 0;
  A carry = A(0);
  // one chunk of the stream: updates (segmented scan, one write per target)
  // or pivots
  auto step = [&]() {
    if (c >= nch) return;  // the level counts and the chunk list agree; never taken
    if (c > 0 && (c & 31) == 0) {
      ++blk;
      d0 = d1;
      d1 = d2;
      const int q = 32 * (blk + 2) + lane;
      d2 = q < nch ? chunks[q] : 0;
    }
    const unsigned w = word(c);
    const int cnt = (int)((w >> kCntShift) & 63u) + 1;
    const bool pivot = (w >> 31) != 0;
    nent += cnt;
    asm volatile("cp.async.wait_group %0;\n" ::"n"(kFRing - 1));
    __syncwarp();
    const int slot = c & (kFRing - 1);
    const int eA = 2 * lane, eB = eA + 1;
    const bool vA = eA < cnt, vB = eB < cnt;
    // entry 2 lane + h sits at h * 32 + lane: both reads contiguous across the warp
    static_assert(kChunk == 64, "two ring entries per lane");
    const uint2 oA = vA ? ring[slot * kChunk + lane] : make_uint2(0u, 0u);
    const uint2 oB = vB ? ring[slot * kChunk + 32 + lane] : make_uint2(0u, 0u);
    if (pivot) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const uint2 o = h ? oB : oA;
        if (h ? vB : vA) {
          const int j = fop_t(o);
          const double dj = pivot_value(V[j], (signed char)(fop_a(o) - 1), prm);
          const T djs = T(dj);
          const T dis = T(1.0 / double(djs));
          D[j] = djs;
          Dinv[j] = dis;
          // FP32: the stored pivot and its stored inverse are the
          // elimination's values
          const double r = F32 ? double(dis) : 1.0 / dj;
          if (!isfinite(r) || !isfinite(double(djs)) || !isfinite(double(dis))) finite = false;
          V[j] = r;
        }
      }
      carry = A(0);
    } else {
      // each target is written once per level (by its last update), so its
      // old value is read before the scan, off the dependent chain
      const int tAi = fop_t(oA), tBi = fop_t(oB);
      const bool wA = vA && fop_last(oA), wB = vB && fop_last(oB);
      const A tA = wA ? A(V[tAi]) : A(0), tB = wB ? A(V[tBi]) : A(0);
      A xA, xB, sA, sB;
      if constexpr (F32) {
        xA = vA ? __fmul_rn(__fmul_rn(float(V[fop_a(oA)]), float(V[fop_b(oA)])),
                            float(V[fop_k(oA)]))
                : 0.f;
        xB = vB ? __fmul_rn(__fmul_rn(float(V[fop_a(oB)]), float(V[fop_b(oB)])),
                            float(V[fop_k(oB)]))
                : 0.f;
      } else {
        xA = vA ? __dmul_rn(__dmul_rn(V[fop_a(oA)], V[fop_b(oA)]), V[fop_k(oA)]) : 0.0;
        xB = vB ? __dmul_rn(__dmul_rn(V[fop_a(oB)], V[fop_b(oB)]), V[fop_k(oB)]) : 0.0;
      }
      seg_scan2(xA, xB, fop_pos(oA), fop_pos(oB), lane, carry,
                (int)((w >> kStepShift) & 7u), sA, sB);
      if constexpr (F32) {
        if (wA) V[tAi] = double(__fsub_rn(tA, sA));
        if (wB) V[tBi] = double(__fsub_rn(tB, sB));
      } else {
        if (wA) V[tAi] = __dsub_rn(tA, sA);
        if (wB) V[tBi] = __dsub_rn(tB, sB);
      }
      const int ll = (cnt - 1) >> 1;
      carry = __shfl_sync(full, ((cnt - 1) & 1) ? sB : sA, ll);
    }
    __syncwarp();
    issue(c + kFRing, slot);
    ++c;
  };
  for (int l = 0; l < nlev; ++l) {
    const int cw = lc[(size_t)l * kFactorWarps];
    const int nop = cw & 0xffff, npv = (cw >> 16) & 0xffff;
    for (int q = 0; q < nop; ++q) step();
    __syncthreads();  // the level's updates before its pivots
    for (int q = 0; q < npv; ++q) step();
    __syncthreads();  // the level's pivots before the next level's updates
  }
  asm volatile("cp.async.wait_all;\n" ::);
  // ---- L = U / d into CSC order and the two substitution-stream orders
  {
    T *Lx = reinterpret_cast<T *>(k.Lx), *LxF = reinterpret_cast<T *>(k.LxF),
      *LxB = reinterpret_cast<T *>(k.LxB);
    for (int e0 = tid; e0 < nl; e0 += NT * kU) {
      int2 be[kU], fe[kU];
      int bq[kU], fq[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int e = e0 + NT * u;
        if (e < nl) {
          be[u] = k.bent[lbase + e];
          bq[u] = k.bpos[lbase + e];
          fe[u] = k.fent[lbase + e];
          fq[u] = k.fpos[lbase + e];
        }
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int e = e0 + NT * u;
        if (e < nl) {
          if constexpr (F32) {
            const float l = __fmul_rn(float(V[N + (bq[u] - lbase)]), float(V[be[u].x & 0xffff]));
            Lx[bq[u]] = l;
            LxB[lbase + e] = l;
            LxF[lbase + e] = __fmul_rn(float(V[N + (fq[u] - lbase)]), float(V[fe[u].y]));
          } else {
            const double l = V[N + (bq[u] - lbase)] * V[be[u].x & 0xffff];
            Lx[bq[u]] = T(l);
            LxB[lbase + e] = T(l);
            LxF[lbase + e] = T(V[N + (fq[u] - lbase)] * V[fe[u].y]);
          }
        }
      }
    }
  }
  const int bad = __syncthreads_or(finite ? 0 : 1);
  if (k.prof_bytes && lane == 0) {
    // the op stream (8 B per entry) and chunk words of this warp; thread 0
    // adds the K diagonal and L-position values (8 + 4 B each), L written
    // three times with the stream indices read, D and D^-1 written
    const double ts = sizeof(T);
    double by = 8.0 * nent + 4.0 * nch;
    if (tid == 0) by += 12.0 * N + 12.0 * nl + nl * (3.0 * ts + 16.0) + 2.0 * ts * N;
    atomicAdd(&k.prof_bytes[inst], by);
  }
  if (tid == 0) {
    if (bad) ok[inst] = 0;
    if (eps_out) eps_out[inst] = eps;
  }
}

// dynamic shared memory = the largest single-warp instance's work vector
template <typename T, bool AR32>
static void launch_factor(const KKTDev &k, const LDLParams &p, const int *run, int *ok,
                          double *eps_out, cudaStream_t st) {
  size_t sm = ((size_t)k.max_small_N * sizeof(double) + 15) & ~(size_t)15;
  if (k.has_fstream)
    k_ldl_factor_stream<T, AR32><<<k.fs_count, 32 * kFactorWarps, k.fs_smem, st>>>(
        k, p, run, ok, eps_out);
  if (k.has_small_legacy)
    k_ldl_factor<T, kSmallNT, true, AR32><<<k.B, kSmallNT, sm, st>>>(k, p, run, ok, eps_out);
  if (k.has_large)
    k_ldl_factor<T, kLargeNT, false, AR32><<<k.B, kLargeNT, 0, st>>>(k, p, run, ok, eps_out);
}
template <typename T>
static void launch_solve(const KKTDev &k, const LDLParams &p, const int *run,
                         const double *rx, const double *rz, double *lx, double *lz, int *ok,
                         cudaStream_t st) {
  if (k.has_small) {
    SolveIO<1> io{{rx}, {rz}, {lx}, {lz}};
    k_ldl_solve_warp<T, 1><<<k.spack_blocks, 32 * kSolveWarps, k.spack_smem, st>>>(k, p, run,
                                                                                 io, ok);
  }
  if (k.has_large)
    k_ldl_solve<T, kLargeNT, false><<<k.B, kLargeNT, 0, st>>>(k, p, run, rx, rz, lx, lz, ok);
}
template <typename T>
static void launch_solve2(const KKTDev &k, const LDLParams &p, const int *run,
                          const double *rx0, const double *rz0, double *lx0, double *lz0,
                          const double *rx1, const double *rz1, double *lx1, double *lz1,
                          int *ok, cudaStream_t st) {
  if (k.has_small) {
    SolveIO<2> io{{rx0, rx1}, {rz0, rz1}, {lx0, lx1}, {lz0, lz1}};
    k_ldl_solve_warp<T, 2><<<k.spack2_blocks, 32 * kSolveWarps, k.spack2_smem, st>>>(k, p, run,
                                                                                   io, ok);
  }
  if (k.has_large) {
    k_ldl_solve<T, kLargeNT, false><<<k.B, kLargeNT, 0, st>>>(k, p, run, rx0, rz0, lx0, lz0, ok);
    k_ldl_solve<T, kLargeNT, false><<<k.B, kLargeNT, 0, st>>>(k, p, run, rx1, rz1, lx1, lz1, ok);
  }
}

static bool g_attr_done = false;
static void set_attrs() {
  if (g_attr_done) return;
  auto stream_attrs = [](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024 + 64);
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
  };
  stream_attrs(k_ldl_factor_stream<double, false>);
  stream_attrs(k_ldl_factor_stream<float, false>);
  stream_attrs(k_ldl_factor_stream<float, true>);
  cudaFuncSetAttribute(k_ldl_factor<double, kSmallNT, true, false>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimitBytes);
  cudaFuncSetAttribute(k_ldl_factor<float, kSmallNT, true, false>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimitBytes);
  cudaFuncSetAttribute(k_ldl_factor<float, kSmallNT, true, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimitBytes);
  // the packed kernels size their blocks for the SM's full shared memory
  auto solve_attrs = [](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kSolveSmemMax);
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
  };
  solve_attrs(k_ldl_solve_warp<double, 1>);
  solve_attrs(k_ldl_solve_warp<float, 1>);
  solve_attrs(k_ldl_solve_warp<double, 2>);
  solve_attrs(k_ldl_solve_warp<float, 2>);
  g_attr_done = true;
}

void ldl_factor(const KKTDev &k, bool fp32, const LDLParams &p, const int *run, int *ok,
                double *eps_out, cudaStream_t st, bool arith32) {
  set_attrs();
  if (fp32 && arith32)
    launch_factor<float, true>(k, p, run, ok, eps_out, st);
  else if (fp32)
    launch_factor<float, false>(k, p, run, ok, eps_out, st);
  else
    launch_factor<double, false>(k, p, run, ok, eps_out, st);
  if (k.sn) sn_factor(*k.sn, k, p, run, ok, eps_out, st);
}

void ldl_solve(const KKTDev &k, bool fp32, const LDLParams &p, const int *run,
               const double *rx, const double *rz, double *lx, double *lz, int *ok,
               cudaStream_t st) {
  set_attrs();
  if (fp32)
    launch_solve<float>(k, p, run, rx, rz, lx, lz, ok, st);
  else
    launch_solve<double>(k, p, run, rx, rz, lx, lz, ok, st);
  if (k.sn) sn_solve(*k.sn, k, p, run, rx, rz, lx, lz, ok, st);
}

void ldl_solve2(const KKTDev &k, bool fp32, const LDLParams &p, const int *run,
                const double *rx0, const double *rz0, double *lx0, double *lz0,
                const double *rx1, const double *rz1, double *lx1, double *lz1, int *ok,
                cudaStream_t st) {
  set_attrs();
  if (fp32)
    launch_solve2<float>(k, p, run, rx0, rz0, lx0, lz0, rx1, rz1, lx1, lz1, ok, st);
  else
    launch_solve2<double>(k, p, run, rx0, rz0, lx0, lz0, rx1, rz1, lx1, lz1, ok, st);
  if (k.sn) {
    sn_solve(*k.sn, k, p, run, rx0, rz0, lx0, lz0, ok, st);
    sn_solve(*k.sn, k, p, run, rx1, rz1, lx1, lz1, ok, st);
  }
}

}  // namespace clgpu
