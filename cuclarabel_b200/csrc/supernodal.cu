// supernodal.cu -- numeric supernodal (multifrontal) LDL^T and solves.
//
// Plays cuDSS's numeric role for the large problems: refactor! every IPM
// iteration (src/kktsolvers/gpu/directldl_cudss.jl:37-46; FP32 for
// :cudssmixed, directldl_mixed_cudss.jl:42-60) and solve! with the FP64
// iterative refinement of kktsolver_directldl_gpu.jl:349-410.  The plan
// (front layout, maps, per-level launch lists) comes from supernodal.cpp.
//
// Factorisation, level by level from the leaves (every task list of a
// level is one launch):
//   small fronts  one block assembles the front in shared memory (original
//                 entries, children's Schur complements), eliminates its
//                 pivots and writes L, D and the Schur complement back;
//   blocked       k_sn_assemble zeroes and assembles column ranges of the
//   fronts        front (a task owns its columns, so children are added in a
//                 fixed order without atomics), then per panel of K <= 128
//                 pivots: k_sn_diag factors the K x K diagonal block,
//                 k_sn_trsm solves every 128-row tile below by triangular
//                 substitution (W = A L11^-T, L = W D^-1), and
//                 k_sn_update_* subtracts L W^T from every lower tile of the
//                 trailing matrix.  FP64 tiles run on the tensor cores (DMMA,
//                 mma.sync m8n8k4), FP32 tiles (mixed form) on FMA units;
//                 both stage their operands with cp.async.
// Solve: forward substitution leaves first (small fronts one warp each,
// blocked fronts panel by panel: diagonal solve then a matrix-vector
// update of the rows below), D^-1, backward substitution roots first.
// Every reduction runs in a fixed order: results do not depend on timing.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "ldl.cuh"
#include "sn_exec.cuh"
#include "pinned.hpp"

namespace clgpu {

namespace {

// trailing update tiles: 128 rows x kUpdCols columns, k in chunks of kUpdKC
constexpr int kUpdCols = 64;
constexpr int kUpdKC = 16;
constexpr int kUpdStages = 3;
constexpr int kUpdLdA = kSnNB + 4;     // shared row strides (elements): 4 mod 16 (FP64
constexpr int kUpdLdB = kUpdCols + 4;  // banks), so DMMA fragment loads are conflict-free
static_assert(kSnKPad % kUpdKC == 0, "panel widths are whole update chunks");
constexpr int kDiagThreads = 256;
constexpr int kTrsmThreads = 256;
constexpr int kAsmThreads = 256;
constexpr int kSmallThreads = 128;
constexpr int kVecThreads = 128;
constexpr int kGemvThreads = 256;
constexpr int kDiagSolveThreads = 512;

// two consecutive elements of a front (8- or 16-byte aligned pairs)
template <typename T>
struct Pair {
  T x, y;
};
__device__ __forceinline__ Pair<double> load_pair(const double *p) {
  const double2 w = *reinterpret_cast<const double2 *>(p);
  return {w.x, w.y};
}
__device__ __forceinline__ Pair<float> load_pair(const float *p) {
  const float2 w = *reinterpret_cast<const float2 *>(p);
  return {w.x, w.y};
}
__device__ __forceinline__ void store_pair(double *p, Pair<double> w) {
  *reinterpret_cast<double2 *>(p) = make_double2(w.x, w.y);
}
__device__ __forceinline__ void store_pair(float *p, Pair<float> w) {
  *reinterpret_cast<float2 *>(p) = make_float2(w.x, w.y);
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
// D(8x8) += A(8x4) B(4x8), FP64 tensor cores.  Fragments: a = A[lane/4][lane%4],
// b = B[lane%4][lane/4], (c0, c1) = C[lane/4][2 (lane%4) + {0, 1}].
__device__ __forceinline__ void dmma884(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// dynamic regularisation (QDLDL's Dsigns rule, kktsolver_directldl.jl:224-229)
__device__ __forceinline__ double sn_pivot(double dj, int sg, const LDLParams &prm) {
  if (prm.dyn_reg && double(sg) * dj <= prm.dyn_eps) dj = prm.dyn_delta * double(sg);
  return dj;
}
__device__ __forceinline__ int pivot_sign(const KKTDev &k, int g) {
  return g >= 0 ? int(k.Dsign[g]) : 1;
}

// ------------------------------------------------------------------ eps
// static regulariser per instance: c + prop * max |diag(K)|
// (_compute_regularizer, kktsolver_directldl.jl:299-313)
__global__ void k_sn_eps(SnDev d, KKTDev k, LDLParams prm, const int *insts, const int *run,
                         double *eps_out) {
  const int inst = insts[blockIdx.x];
  if (!run[inst]) return;
  __shared__ double red[kAsmThreads / 32];
  double mx = 0;
  if (prm.static_reg)
    for (int v = k.voff[inst] + threadIdx.x; v < k.voff[inst + 1]; v += kAsmThreads)
      mx = fmax(mx, fabs(k.Kx[k.Kdiag[v]]));
  mx = warp_max(mx);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kAsmThreads / 32; ++w) mx = fmax(mx, red[w]);
    mx = fmax(mx, red[0]);
    const double eps = prm.static_reg ? prm.static_c + prm.static_prop * mx : 0.0;
    d.eps[inst] = eps;
    if (eps_out) eps_out[inst] = eps;
  }
}

// --------------------------------------------------------- small fronts
// One block per front of at most kSnSmallMax rows: assemble in shared
// memory, eliminate the ncol pivots (right-looking), write back.
template <typename T>
__global__ void __launch_bounds__(kSmallThreads) k_sn_small(SnDev d, KKTDev k, LDLParams prm,
                                                           int base, const int *run, int *ok) {
  const int s = d.tasks[base + blockIdx.x].x, inst = d.inst[s];
  if (!run[inst]) return;
  extern __shared__ __align__(16) unsigned char sraw[];
  const int ld = d.ld[s], nc = d.ncol[s], tid = threadIdx.x;
  T *f = reinterpret_cast<T *>(sraw);
  T *col = f + ld * ld;
  for (int i = tid; i < ld * ld; i += kSmallThreads) f[i] = T(0);
  __syncthreads();
  const int2 *am = d.amap;
  for (int q = d.acol[d.cbase[s]] + tid; q < d.acol[d.cbase[s] + nc]; q += kSmallThreads)
    f[am[q].y] = T(k.Kx[am[q].x]);
  __syncthreads();
  const double eps = d.eps[inst];
  for (int c = tid; c < nc; c += kSmallThreads) {
    const int g = d.col0g[s] + c;
    f[c * ld + c] += T(k.Dsign[g] > 0 ? eps : -eps);
  }
  __syncthreads();
  const T *F = reinterpret_cast<const T *>(d.F);
  for (int a = d.ch_ptr[s]; a < d.ch_ptr[s + 1]; ++a) {
    const int c = d.ch[a], cn = d.nrow[c], cld = d.ld[c], cu = d.u0[c];
    const int *rel = d.rel + d.rel_off[c];
    const T *cf = F + d.foff[c];
    for (int q = 0; q < cn; ++q) {
      const int pc = rel[q];
      for (int r = q + tid; r < cn; r += kSmallThreads)
        f[pc * ld + rel[r]] += cf[(long long)(cu + q) * cld + cu + r];
    }
    __syncthreads();
  }
  bool bad = false;
  for (int j = 0; j < nc; ++j) {
    const int g = d.col0g[s] + j;
    const T dj = T(sn_pivot(double(f[j * ld + j]), k.Dsign[g], prm));
    for (int i = j + 1 + tid; i < ld; i += kSmallThreads) col[i] = f[j * ld + i];
    __syncthreads();
    {
      // rank-1 update of the trailing lower triangle: 16 x 8 threads
      const int tx = tid & 15, ty = tid >> 4;
      for (int r = j + 1 + ty; r < ld; r += kSmallThreads / 16) {
        const T cr = col[r];
        for (int i = j + 1 + tx; i < ld; i += 16)
          if (i >= r) f[r * ld + i] -= (col[i] / dj) * cr;
      }
    }
    for (int i = j + 1 + tid; i < ld; i += kSmallThreads) f[j * ld + i] = col[i] / dj;
    if (tid == 0) {
      f[j * ld + j] = dj;
      const double di = 1.0 / double(dj);
      d.Dinv[g] = di;
      if (!isfinite(di) || !isfinite(double(dj))) bad = true;
    }
    __syncthreads();
  }
  T *out = reinterpret_cast<T *>(d.F) + d.foff[s];
  for (int i = tid; i < ld * ld; i += kSmallThreads) {
    const int c = i / ld, r = i % ld;
    if (r >= c) out[i] = f[i];
  }
  if (bad) ok[inst] = 0;
}

// ------------------------------------------------------- blocked fronts
// Assembly of columns [ca, cb) of a blocked front: zero (rows c..ld), the
// original entries (+ static regularisation), unit dummy pivots, then the
// Schur complements of the children that touch these columns, in child
// order (the plan lists them per 32-column chunk with their entry ranges).
template <typename T>
__global__ void __launch_bounds__(kAsmThreads) k_sn_assemble(SnDev d, KKTDev k, int base,
                                                            const int *run) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, ca = t.y, cb = t.z, inst = d.inst[s];
  if (!run[inst]) return;
  const long long ld = d.ld[s];
  const int nc = d.ncol[s], u0 = d.u0[s], tid = threadIdx.x;
  T *f = reinterpret_cast<T *>(d.F) + d.foff[s];
  for (int c = ca; c < cb; ++c)
    for (long long r = c + tid; r < ld; r += kAsmThreads) f[c * ld + r] = T(0);
  __syncthreads();
  const double eps = d.eps[inst];
  const int ce = min(cb, nc);
  if (ca < ce) {
    const int2 *am = d.amap;
    for (int q = d.acol[d.cbase[s] + ca] + tid; q < d.acol[d.cbase[s] + ce]; q += kAsmThreads) {
      const int2 e = am[q];
      double v = k.Kx[e.x];
      const int c = e.y / (int)ld, r = e.y - c * (int)ld;
      if (r == c) v += k.Dsign[d.col0g[s] + c] > 0 ? eps : -eps;
      f[e.y] = T(v);
    }
  }
  for (int c = max(ca, nc) + tid; c < min(cb, u0); c += kAsmThreads) f[c * ld + c] = T(1);
  __syncthreads();
  const T *F = reinterpret_cast<const T *>(d.F);
  // the children touching columns [ca, cb), in child order (plan)
  for (int a = d.cl_ptr[t.w]; a < d.cl_ptr[t.w + 1]; ++a) {
    const int4 cq = d.clist[a];
    const int c = cq.x, qa = cq.y, qb = cq.z, cn = d.nrow[c], cu = d.u0[c];
    const long long cld = d.ld[c];
    const int *rel = d.rel + d.rel_off[c];
    const T *cf = F + d.foff[c];
    for (int q = qa; q < qb; ++q) {
      const long long pc = rel[q];
      const T *src = cf + (cu + q) * cld + cu;
      // four rows per thread per round, their loads issued before any add
      // (the parent positions of one column are distinct)
      for (int r0 = q + tid; r0 < cn; r0 += 4 * kAsmThreads) {
        int rr[4];
        T sv[4], fv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int r = r0 + u * kAsmThreads;
          rr[u] = r < cn ? rel[r] : 0;
          sv[u] = r < cn ? src[r] : T(0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (r0 + u * kAsmThreads < cn) fv[u] = f[pc * ld + rr[u]];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (r0 + u * kAsmThreads < cn) f[pc * ld + rr[u]] = fv[u] + sv[u];
      }
    }
    __syncthreads();
  }
}

// Diagonal block of a panel: factor the K x K block (the static shift was
// applied at assembly), write L11 and D to the front and 1/d to the
// workspace.  Blocked right-looking LDL^T in 32-column blocks, every column
// kept unscaled until the end (L(:, j) = a(:, j) / d_j is written last):
//   1. one warp factors the 32 x 32 diagonal block (lane i owns row i; step
//      j subtracts a(i, j) (a(k, j) / d_j) from a(i, k), j < k <= i), with
//      the pivot rule applied to each pivot as it becomes final;
//   2. every row below the block (one thread each, the row in registers)
//      takes the same 32 steps against the block's columns;
//   3. the trailing lower triangle -= X D^-1 X^T over the block's 32
//      columns, 6 x 6 outputs per thread.
// Three barriers per column block instead of one per pivot.  Pivot signs
// and D's global positions are staged first.
constexpr int kDiagNB = 32;
template <typename T>
__global__ void __launch_bounds__(kDiagThreads) k_sn_diag(SnDev d, KKTDev k, LDLParams prm,
                                                         int base, const int *run, int *ok) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16, inst = d.inst[s];
  if (!run[inst]) return;
  extern __shared__ __align__(16) unsigned char sraw[];
  T *blk = reinterpret_cast<T *>(sraw);       // K x K, column-major, stride K
  T *wsc = blk + kSnNB * kSnNB;               // scaled block columns, [kDiagNB][kSnNB]
  __shared__ double dinv[kSnNB];
  __shared__ T dd[kSnNB];
  __shared__ int gix[kSnNB], sgn[kSnNB];
  const long long ld = d.ld[s];
  T *f = reinterpret_cast<T *>(d.F) + d.foff[s];
  T *ws = reinterpret_cast<T *>(d.W) + d.woff[s];
  const int *fi = d.fidx + d.fix_off[s];
  const int tid = threadIdx.x;
  // stage the block by row pairs (16-byte loads for FP64), a fixed trip
  // count so that many loads are in flight; the strict upper part is not
  // read by the factorisation below
#pragma unroll 8
  for (int it = 0; it < kSnNB * kSnNB / 2 / kDiagThreads; ++it) {
    const int p = tid + it * kDiagThreads, c = p >> 6, r = (p & 63) * 2;
    if (c < K && r < K) store_pair(blk + c * K + r, load_pair(f + (k0 + c) * ld + k0 + r));
  }
  for (int j = tid; j < K; j += kDiagThreads) {
    const int g = fi[k0 + j];
    gix[j] = g;
    sgn[j] = pivot_sign(k, g);
  }
  __syncthreads();
  for (int b0 = 0; b0 < K; b0 += kDiagNB) {
    const int nb = min(kDiagNB, K - b0);
    // 1. the diagonal block, one warp
    if (tid < 32) {
      const int i = tid;
      for (int j = 0; j < nb; ++j) {
        const T dj = T(sn_pivot(double(blk[(b0 + j) * K + b0 + j]), sgn[b0 + j], prm));
        const double di = 1.0 / double(dj);
        if (i == 0) {
          dd[b0 + j] = dj;
          dinv[b0 + j] = di;
        }
        if (i > j && i < nb) {
          const T *cj = blk + (b0 + j) * K + b0;
          const T li = cj[i] * T(di);
          for (int q = j + 1; q <= i; ++q) blk[(b0 + q) * K + b0 + i] -= li * cj[q];
        }
        __syncwarp();
      }
    }
    __syncthreads();
    const int rb = b0 + nb, m = K - rb;  // rows below the block
    if (m <= 0) break;
    // 2. the rows below, one thread each
    if (tid < m) {
      const int r = rb + tid;
      T x[kDiagNB];
#pragma unroll
      for (int j = 0; j < kDiagNB; ++j) x[j] = j < nb ? blk[(b0 + j) * K + r] : T(0);
#pragma unroll
      for (int j = 0; j < kDiagNB; ++j) {
        if (j < nb) {
          const T lj = x[j] * T(dinv[b0 + j]);
#pragma unroll
          for (int q = j + 1; q < kDiagNB; ++q)
            if (q < nb) x[q] -= lj * blk[(b0 + j) * K + b0 + q];
        }
      }
#pragma unroll
      for (int j = 0; j < kDiagNB; ++j)
        if (j < nb) {
          blk[(b0 + j) * K + r] = x[j];
          wsc[j * kSnNB + tid] = x[j] * T(dinv[b0 + j]);
        }
    }
    __syncthreads();
    // 3. trailing lower triangle: a(r, c) -= sum_j x(r, j) (x(c, j) / d_j)
    {
      const int tx = tid & 15, ty = tid >> 4;
      T acc[6][6];
#pragma unroll
      for (int u = 0; u < 6; ++u)
#pragma unroll
        for (int v = 0; v < 6; ++v) acc[u][v] = T(0);
      for (int j = 0; j < nb; ++j) {
        T xa[6], wb[6];
#pragma unroll
        for (int u = 0; u < 6; ++u) {
          const int rr = ty + 16 * u, cc = tx + 16 * u;
          xa[u] = rr < m ? blk[(b0 + j) * K + rb + rr] : T(0);
          wb[u] = cc < m ? wsc[j * kSnNB + cc] : T(0);
        }
#pragma unroll
        for (int u = 0; u < 6; ++u)
#pragma unroll
          for (int v = 0; v < 6; ++v) acc[u][v] += xa[u] * wb[v];
      }
#pragma unroll
      for (int u = 0; u < 6; ++u)
#pragma unroll
        for (int v = 0; v < 6; ++v) {
          const int rr = ty + 16 * u, cc = tx + 16 * v;
          if (rr < m && cc <= rr) blk[(rb + cc) * K + rb + rr] -= acc[u][v];
        }
    }
    __syncthreads();
  }
#pragma unroll 8
  for (int it = 0; it < kSnNB * kSnNB / kDiagThreads; ++it) {
    const int p = tid + it * kDiagThreads, c = p >> 7, r = p & (kSnNB - 1);
    if (c < K && r < K && r >= c)
      f[(k0 + c) * ld + k0 + r] = r > c ? blk[c * K + r] * T(dinv[c]) : dd[c];
  }
  bool bad = false;
  for (int j = tid; j < kSnNB; j += kDiagThreads) {
    if (j < K) {
      const double di = dinv[j];
      if (gix[j] >= 0) d.Dinv[gix[j]] = di;
      ws[j] = T(di);
      if (!isfinite(di) || !isfinite(double(dd[j]))) bad = true;
    } else {
      ws[j] = T(0);
    }
  }
  if (bad) ok[inst] = 0;
}

// one column block of the TRSM below: (a) then (b), NB columns from b0
template <typename T, int NB>
__device__ __forceinline__ void trsm_block(T *X, const T *Lr, int b0, int K, int m, int half) {
  if (half == 0) {
    T x[NB];
#pragma unroll
    for (int j = 0; j < NB; ++j) x[j] = X[(b0 + j) * kSnNB + m];
#pragma unroll
    for (int q = 1; q < NB; ++q) {
      const T *lq = Lr + (b0 + q) * (b0 + q - 1) / 2 + b0;
      T acc = x[q];
#pragma unroll
      for (int j = 0; j < q; ++j) acc -= x[j] * lq[j];
      x[q] = acc;
    }
#pragma unroll
    for (int j = 0; j < NB; ++j) X[(b0 + j) * kSnNB + m] = x[j];
  }
  __syncthreads();
  if (b0 + NB < K) {
    T x[NB];
#pragma unroll
    for (int j = 0; j < NB; ++j) x[j] = X[(b0 + j) * kSnNB + m];
    for (int q = b0 + NB + half; q < K; q += kTrsmThreads / kSnNB) {
      const T *lq = Lr + q * (q - 1) / 2 + b0;
      T acc = T(0);
#pragma unroll
      for (int j = 0; j < NB; ++j) acc += x[j] * lq[j];
      X[q * kSnNB + m] -= acc;
    }
  }
  __syncthreads();
}

// TRSM of a panel's row tile: rows r0..r0+127 of panel [k0, k0+K),
// W = A L11^-T by substitution, then L = W D^-1: L overwrites A in the
// front, W goes to the workspace for the trailing update.  Blocked by 32
// columns: (a) each row (one thread) solves the block's 32 columns in
// registers against the block's unit lower triangle (row-oriented: w(m, q)
// = a(m, q) - sum_{j<q} w(m, j) L11(q, j)); (b) the later columns of the
// row take the block's contribution, sum_j w(m, j) L11(q, j), the two
// halves of the thread block splitting the columns.  Two barriers per
// column block.  The tile (K x 128, column-major) and the strict lower triangle
// of L11 packed by rows (row q at q (q - 1) / 2) sit in shared memory.
template <typename T>
__global__ void __launch_bounds__(kTrsmThreads) k_sn_trsm(SnDev d, int base, const int *run) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16, r0 = t.z;
  if (!run[d.inst[s]]) return;
  extern __shared__ __align__(16) unsigned char sraw[];
  T *X = reinterpret_cast<T *>(sraw);  // column q of the tile at X + q kSnNB
  T *Lr = X + K * kSnNB;               // L11(q, j), j < q, at Lr[q (q - 1) / 2 + j]
  const long long ld = d.ld[s];
  T *f = reinterpret_cast<T *>(d.F) + d.foff[s];
  const T *ws = reinterpret_cast<const T *>(d.W) + d.woff[s];
  T *wr = reinterpret_cast<T *>(d.W) + d.woff[s] + kSnNB;
  const int tid = threadIdx.x;
  // stage the tile and L11 by row pairs, fixed trip counts (many 16-byte
  // loads in flight)
#pragma unroll 8
  for (int it = 0; it < kSnNB * kSnNB / 2 / kTrsmThreads; ++it) {
    const int p = tid + it * kTrsmThreads, q = p >> 6, m = (p & 63) * 2;
    if (q < K) store_pair(X + q * kSnNB + m, load_pair(f + (k0 + q) * ld + r0 + m));
  }
#pragma unroll 8
  for (int it = 0; it < kSnNB * kSnNB / 2 / kTrsmThreads; ++it) {
    const int p = tid + it * kTrsmThreads, j = p >> 6, q = (p & 63) * 2;
    if (j < K && q + 1 > j && q < K) {
      const Pair<T> w = load_pair(f + (k0 + j) * ld + k0 + q);
      if (q > j) Lr[q * (q - 1) / 2 + j] = w.x;
      Lr[(q + 1) * q / 2 + j] = w.y;  // q + 1 > j
    }
  }
  __syncthreads();
  const int m = tid & (kSnNB - 1), half = tid / kSnNB;
  for (int b0 = 0; b0 < K; b0 += 32) {
    // K is a multiple of 16, so a block has 32 or 16 columns
    if (K - b0 >= 32)
      trsm_block<T, 32>(X, Lr, b0, K, m, half);
    else
      trsm_block<T, 16>(X, Lr, b0, K, m, half);
  }
#pragma unroll 4
  for (int it = 0; it < kSnNB * kSnNB / kTrsmThreads; ++it) {
    const int idx = tid + it * kTrsmThreads, q = idx >> 7, mm = idx & (kSnNB - 1);
    if (q < K) {
      const T w = X[idx];
      wr[(long long)q * ld + r0 + mm] = w;
      f[(k0 + q) * ld + r0 + mm] = w * ws[q];
    }
  }
}

// Trailing update of the blocked fronts, one 128 x 64 tile per block:
// front tile (r0, c0) -= L(r0.., panel) W(c0.., :)^T, entries on or below
// the diagonal only (r0 + m >= c0 + n).  K (a multiple of kSnKPad = 16) is
// streamed in chunks of kUpdKC through a kUpdStages-deep cp.async pipeline.
// FP64: 8 warps as 4 (rows) x 2 (columns), warp tile 32 x 32 of m8n8k4
// DMMA; 120 registers, so two blocks (16 warps) are resident per SM and
// one block's prologue and epilogue overlap the other's main loop.  The
// accumulators start from the front tile itself (its loads are issued
// before the operand pipeline fills, so their latency is hidden) and the
// products are subtracted as they come (W fragments negated), so the
// epilogue only stores.
constexpr int kUpdThreads = 256;
__global__ void __launch_bounds__(kUpdThreads, 2) k_sn_update_f64(SnDev d, int base, const int *run) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16, r0 = t.z, c0 = t.w;
  if (!run[d.inst[s]]) return;
  const long long ld = d.ld[s];
  double *f = reinterpret_cast<double *>(d.F) + d.foff[s];
  const double *Ag = f + k0 * ld + r0;
  const double *Bg = reinterpret_cast<const double *>(d.W) + d.woff[s] + kSnNB + c0;
  extern __shared__ __align__(16) unsigned char sraw[];
  double *sm = reinterpret_cast<double *>(sraw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 3, wn = warp >> 2;
  // accumulator (mi, ni, h) is front entry (r0 + m, c0 + n); the whole
  // tile lies inside the front (entries above the diagonal are read and
  // left unchanged)
  double acc[4][4][2];
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int h = 0; h < 2; ++h)
        acc[mi][ni][h] = f[(long long)(c0 + wn * 32 + ni * 8 + 2 * (lane & 3) + h) * ld + r0 +
                           wm * 32 + mi * 8 + (lane >> 2)];
  const int nchunks = K / kUpdKC;
  constexpr int kStage = kUpdKC * (kUpdLdA + kUpdLdB);
  auto load = [&](int chunk, int stage) {
    double *As = sm + stage * kStage, *Bs = As + kUpdKC * kUpdLdA;
    // A: kUpdKC columns x 64 pieces of 16 B; B: kUpdKC x 32
    for (int p = tid; p < kUpdKC * 64; p += kUpdThreads) {
      const int q = p >> 6, m = (p & 63) * 2;
      cp_async16(As + q * kUpdLdA + m, Ag + ((long long)chunk * kUpdKC + q) * ld + m);
    }
    for (int p = tid; p < kUpdKC * 32; p += kUpdThreads) {
      const int q = p >> 5, n = (p & 31) * 2;
      cp_async16(Bs + q * kUpdLdB + n, Bg + ((long long)chunk * kUpdKC + q) * ld + n);
    }
  };
#pragma unroll
  for (int st = 0; st < kUpdStages - 1; ++st) {
    if (st < nchunks) load(st, st);
    cp_async_commit();
  }
  for (int c = 0; c < nchunks; ++c) {
    cp_async_wait<kUpdStages - 2>();
    __syncthreads();
    const int nx = c + kUpdStages - 1;
    if (nx < nchunks) load(nx, nx % kUpdStages);
    cp_async_commit();
    const double *As = sm + (c % kUpdStages) * kStage;
    const double *Bs = As + kUpdKC * kUpdLdA;
#pragma unroll
    for (int kk = 0; kk < kUpdKC; kk += 4) {
      const int q = kk + (lane & 3);
      double a[4], b[4];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) a[mi] = As[q * kUpdLdA + wm * 32 + mi * 8 + (lane >> 2)];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) b[ni] = -Bs[q * kUpdLdB + wn * 32 + ni * 8 + (lane >> 2)];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) dmma884(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
    }
  }
  cp_async_wait<0>();
  const bool diag = r0 < c0 + 64;  // the tile reaches above the diagonal
#pragma unroll
  for (int mi = 0; mi < 4; ++mi) {
    const int m = wm * 32 + mi * 8 + (lane >> 2);
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int n = wn * 32 + ni * 8 + 2 * (lane & 3) + h;
        if (!diag || r0 + m >= c0 + n) f[(long long)(c0 + n) * ld + r0 + m] = acc[mi][ni][h];
      }
  }
}

// FP32 form: 16 x 8 threads, each 8 x 8 outputs (rows ty*4 + {0..3} and
// 64 + ty*4 + {0..3}; columns tx*4 + {0..3} and 32 + tx*4 + {0..3}), FMA units.
__global__ void __launch_bounds__(128, 2) k_sn_update_f32(SnDev d, int base, const int *run) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16, r0 = t.z, c0 = t.w;
  if (!run[d.inst[s]]) return;
  const long long ld = d.ld[s];
  float *f = reinterpret_cast<float *>(d.F) + d.foff[s];
  const float *Ag = f + k0 * ld + r0;
  const float *Bg = reinterpret_cast<const float *>(d.W) + d.woff[s] + kSnNB + c0;
  extern __shared__ __align__(16) unsigned char sraw[];
  float *sm = reinterpret_cast<float *>(sraw);
  const int tid = threadIdx.x, tx = tid & 7, ty = tid >> 3;
  // accumulators start from the front tile (as in the FP64 kernel)
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j)
      acc[i][j] = f[(long long)(c0 + (j < 4 ? 0 : 32) + tx * 4 + (j & 3)) * ld + r0 +
                    (i < 4 ? 0 : 64) + ty * 4 + (i & 3)];
  const int nchunks = K / kUpdKC;
  constexpr int kStage = kUpdKC * (kUpdLdA + kUpdLdB);
  auto load = [&](int chunk, int stage) {
    float *As = sm + stage * kStage, *Bs = As + kUpdKC * kUpdLdA;
    for (int p = tid; p < kUpdKC * 32; p += 128) {  // 16 B = 4 floats
      const int q = p >> 5, m = (p & 31) * 4;
      cp_async16(As + q * kUpdLdA + m, Ag + ((long long)chunk * kUpdKC + q) * ld + m);
    }
    for (int p = tid; p < kUpdKC * 16; p += 128) {
      const int q = p >> 4, n = (p & 15) * 4;
      cp_async16(Bs + q * kUpdLdB + n, Bg + ((long long)chunk * kUpdKC + q) * ld + n);
    }
  };
#pragma unroll
  for (int st = 0; st < kUpdStages - 1; ++st) {
    if (st < nchunks) load(st, st);
    cp_async_commit();
  }
  for (int c = 0; c < nchunks; ++c) {
    cp_async_wait<kUpdStages - 2>();
    __syncthreads();
    const int nx = c + kUpdStages - 1;
    if (nx < nchunks) load(nx, nx % kUpdStages);
    cp_async_commit();
    const float *As = sm + (c % kUpdStages) * kStage;
    const float *Bs = As + kUpdKC * kUpdLdA;
#pragma unroll
    for (int q = 0; q < kUpdKC; ++q) {
      const float4 a0 = *reinterpret_cast<const float4 *>(As + q * kUpdLdA + ty * 4);
      const float4 a1 = *reinterpret_cast<const float4 *>(As + q * kUpdLdA + 64 + ty * 4);
      const float4 b0 = *reinterpret_cast<const float4 *>(Bs + q * kUpdLdB + tx * 4);
      const float4 b1 = *reinterpret_cast<const float4 *>(Bs + q * kUpdLdB + 32 + tx * 4);
      const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(-a[i], b[j], acc[i][j]);
    }
  }
  cp_async_wait<0>();
  const bool diag = r0 < c0 + 64;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int m = (i < 4 ? 0 : 64) + ty * 4 + (i & 3);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int n = (j < 4 ? 0 : 32) + tx * 4 + (j & 3);
      if (!diag || r0 + m >= c0 + n) f[(long long)(c0 + n) * ld + r0 + m] = acc[i][j];
    }
  }
}

// ------------------------------------------------------------------ solves
// vector index of plan entry g (global vector index)
__device__ __forceinline__ int vix(const SnDev &d, int g) { return g - d.vbase; }

// small fronts, one warp each: forward substitution
template <typename T>
__global__ void __launch_bounds__(256) k_sn_fwd_small(SnDev d, int base, int count) {
  __shared__ double vs[8][kSnSmallMax];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ti = blockIdx.x * 8 + w;
  if (ti >= count) return;
  const int s = d.tasks[base + ti].x;
  if (!d.srun[d.inst[s]]) return;
  const int ld = d.ld[s], nc = d.ncol[s];
  double *v = vs[w];
  double *y = d.y;
  for (int i = lane; i < ld; i += 32) v[i] = i < nc ? y[vix(d, d.col0g[s] + i)] : 0.0;
  __syncwarp();
  for (int a = d.ch_ptr[s]; a < d.ch_ptr[s + 1]; ++a) {
    const int c = d.ch[a], cn = d.nrow[c];
    const int *rel = d.rel + d.rel_off[c];
    const double *u = d.U + d.uoff[c];
    for (int q = lane; q < cn; q += 32) v[rel[q]] += u[q];
    __syncwarp();
  }
  const T *f = reinterpret_cast<const T *>(d.F) + d.foff[s];
  // lane holds rows lane + 32 r (ld <= 128); column j + 1 is loaded while
  // column j is applied, so the dependent chain waits on shared memory only
  double cur[4], nxt[4];
  auto column = [&](int j, double (&o)[4]) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int i = lane + 32 * r;
      o[r] = (j < nc && i > j && i < ld) ? double(f[j * ld + i]) : 0.0;
    }
  };
  column(0, cur);
  for (int j = 0; j < nc; ++j) {
    column(j + 1, nxt);
    const double vj = v[j];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int i = lane + 32 * r;
      if (i > j && i < ld) v[i] -= cur[r] * vj;
      cur[r] = nxt[r];
    }
    __syncwarp();
  }
  for (int i = lane; i < nc; i += 32) y[vix(d, d.col0g[s] + i)] = v[i];
  double *uo = d.U + d.uoff[s];
  for (int q = lane; q < ld - nc; q += 32) uo[q] = v[nc + q];
}

// small fronts, one warp each: backward substitution
template <typename T>
__global__ void __launch_bounds__(256) k_sn_bwd_small(SnDev d, int base, int count) {
  __shared__ double vs[8][kSnSmallMax];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ti = blockIdx.x * 8 + w;
  if (ti >= count) return;
  const int s = d.tasks[base + ti].x;
  if (!d.srun[d.inst[s]]) return;
  const int ld = d.ld[s], nc = d.ncol[s];
  const int *fi = d.fidx + d.fix_off[s];
  double *v = vs[w];
  double *y = d.y;
  for (int i = lane; i < ld; i += 32) v[i] = y[vix(d, fi[i])];
  __syncwarp();
  const T *f = reinterpret_cast<const T *>(d.F) + d.foff[s];
  // column j - 1 is loaded while column j's dot product runs
  double cur[4], nxt[4];
  auto column = [&](int j, double (&o)[4]) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int i = lane + 32 * r;
      o[r] = (j >= 0 && i > j && i < ld) ? double(f[j * ld + i]) : 0.0;
    }
  };
  column(nc - 1, cur);
  for (int j = nc - 1; j >= 0; --j) {
    column(j - 1, nxt);
    double t = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int i = lane + 32 * r;
      if (i > j && i < ld) t += cur[r] * v[i];
      cur[r] = nxt[r];
    }
    t = warp_sum(t);
    if (lane == 0) v[j] -= t;
    __syncwarp();
  }
  for (int i = lane; i < nc; i += 32) y[vix(d, d.col0g[s] + i)] = v[i];
}

// blocked fronts: positions [ca, cb) of the work vector v (ld) from y and
// the contributions of the children touching them (in child order); one
// warp per 32-position chunk
__global__ void __launch_bounds__(256) k_sn_fwd_gather(SnDev d, int base, int count) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ti = blockIdx.x * 8 + w;
  if (ti >= count) return;
  const int4 t = d.tasks[base + ti];
  const int s = t.x, ca = t.y, cb = t.z;
  if (!d.srun[d.inst[s]]) return;
  const int nc = d.ncol[s];
  double *v = d.S + d.soff[s];
  const int i = ca + lane;
  if (i < cb) v[i] = i < nc ? d.y[vix(d, d.col0g[s] + i)] : 0.0;
  __syncwarp();
  for (int a = d.cl_ptr[t.w]; a < d.cl_ptr[t.w + 1]; ++a) {
    const int4 cq = d.clist[a];
    const int *rel = d.rel + d.rel_off[cq.x];
    const double *u = d.U + d.uoff[cq.x];
    for (int q = cq.y + lane; q < cq.z; q += 32) v[rel[q]] += u[q];
    __syncwarp();
  }
}

// forward: v[k..k+K) <- L11^-1 v[k..k+K).  L11 is first copied to shared
// memory (coalesced pairs), then one warp runs the K dependent steps with x
// in registers.
template <typename T>
__global__ void __launch_bounds__(kDiagSolveThreads) k_sn_fwd_diag(SnDev d, int base) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16;
  if (!d.srun[d.inst[s]]) return;
  extern __shared__ __align__(16) unsigned char sraw[];
  T *Ls = reinterpret_cast<T *>(sraw);  // column j at Ls + j kSnNB
  const long long ld = d.ld[s];
  double *v = d.S + d.soff[s] + k0;
  const T *f = reinterpret_cast<const T *>(d.F) + d.foff[s] + k0 * ld + k0;
  // stage L11 by pairs of rows (K, ld and the front offsets are even); a
  // fixed trip count, so the loads are unrolled and many are in flight
#pragma unroll 8
  for (int it = 0; it < kSnNB * kSnNB / 2 / kDiagSolveThreads; ++it) {
    const int p = threadIdx.x + it * kDiagSolveThreads, j = p >> 6, i = (p & 63) * 2;
    if (j < K && i < K) store_pair(Ls + j * kSnNB + i, load_pair(f + j * ld + i));
  }
  __syncthreads();
  if (threadIdx.x >= 32) return;
  // one warp: lane owns rows lane + 32 r; x_j is final when step j starts
  // and is broadcast from its owner
  const int lane = threadIdx.x;
  double xr[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) xr[r] = lane + 32 * r < K ? v[lane + 32 * r] : 0.0;
#pragma unroll
  for (int sb = 0; sb < 4; ++sb) {
    if (32 * sb >= K) break;
#pragma unroll
    for (int jj = 0; jj < 32; ++jj) {
      const int j = 32 * sb + jj;
      const double xj = __shfl_sync(0xffffffffu, xr[sb], jj);
#pragma unroll
      for (int r = sb; r < 4; ++r) {
        const int i = 32 * r + lane;
        if (i > j && i < K) xr[r] -= double(Ls[j * kSnNB + i]) * xj;
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
    if (lane + 32 * r < K) v[lane + 32 * r] = xr[r];
}

// forward: v[r0..r0+128) -= L(r0.., panel) v[k..k+K).  Thread (rp, g) takes
// rows 2 rp, 2 rp + 1 and columns g, g + 4, ...; the four column groups'
// sums are added in group order.
template <typename T>
__global__ void __launch_bounds__(kGemvThreads) k_sn_fwd_gemv(SnDev d, int base) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16, r0 = t.z;
  if (!d.srun[d.inst[s]]) return;
  __shared__ double x[kSnNB];
  __shared__ __align__(16) double acc[4][kSnNB];
  const long long ld = d.ld[s];
  double *v = d.S + d.soff[s];
  const int tid = threadIdx.x, rp = tid & 63, g = tid >> 6;
  if (tid < K) x[tid] = v[k0 + tid];
  __syncthreads();
  const T *fp = reinterpret_cast<const T *>(d.F) + d.foff[s] + k0 * ld + r0 + 2 * rp;
  double a0 = 0.0, a1 = 0.0;
#pragma unroll 8
  for (int q = g; q < K; q += 4) {
    const Pair<T> w = load_pair(fp + q * ld);
    const double xq = x[q];
    a0 += double(w.x) * xq;
    a1 += double(w.y) * xq;
  }
  reinterpret_cast<double2 *>(acc[g])[rp] = make_double2(a0, a1);
  __syncthreads();
  if (tid < kSnNB) v[r0 + tid] -= (acc[0][tid] + acc[1][tid]) + (acc[2][tid] + acc[3][tid]);
}

__global__ void __launch_bounds__(kVecThreads) k_sn_fwd_scatter(SnDev d, int base) {
  const int s = d.tasks[base + blockIdx.x].x;
  if (!d.srun[d.inst[s]]) return;
  const int nc = d.ncol[s], nr = d.nrow[s], u0 = d.u0[s];
  const double *v = d.S + d.soff[s];
  for (int i = threadIdx.x; i < nc; i += kVecThreads) d.y[vix(d, d.col0g[s] + i)] = v[i];
  double *uo = d.U + d.uoff[s];
  for (int q = threadIdx.x; q < nr; q += kVecThreads) uo[q] = v[u0 + q];
}

__global__ void __launch_bounds__(kVecThreads) k_sn_bwd_gather(SnDev d, int base) {
  const int s = d.tasks[base + blockIdx.x].x;
  if (!d.srun[d.inst[s]]) return;
  const int ld = d.ld[s];
  const int *fi = d.fidx + d.fix_off[s];
  double *v = d.S + d.soff[s];
  for (int i = threadIdx.x; i < ld; i += kVecThreads) {
    const int g = fi[i];
    v[i] = g >= 0 ? d.y[vix(d, g)] : 0.0;
  }
}

// backward: partial sums over the row tile r0: p[q] = sum_m L(r0 + m, k + q) v[r0 + m].
// Thread (rp, g) takes rows 2 rp, 2 rp + 1 and columns g, g + 4, ...; each
// column's 64 products are summed by a fixed butterfly in the two warps of
// its group, then the two warp sums in order.
template <typename T>
__global__ void __launch_bounds__(kGemvThreads) k_sn_bwd_partial(SnDev d, int base) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16, r0 = t.z;
  if (!d.srun[d.inst[s]]) return;
  __shared__ double red[2][kSnNB];
  const long long ld = d.ld[s];
  const double *v = d.S + d.soff[s] + r0;
  double *part = d.S + d.soff[s] + ld + r0;  // tile r0's partials at [r0, r0 + K)
  const int tid = threadIdx.x, rp = tid & 63, g = tid >> 6, lane = tid & 31, h = rp >> 5;
  const double2 vm = reinterpret_cast<const double2 *>(v)[rp];
  const T *fp = reinterpret_cast<const T *>(d.F) + d.foff[s] + k0 * ld + r0 + 2 * rp;
  for (int c0 = 0; 4 * c0 < K; c0 += 8) {
    double pr[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int q = g + 4 * (c0 + u);
      pr[u] = 0.0;
      if (q < K) {
        const Pair<T> w = load_pair(fp + q * ld);
        pr[u] = double(w.x) * vm.x + double(w.y) * vm.y;
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
      for (int u = 0; u < 8; ++u) pr[u] += __shfl_xor_sync(0xffffffffu, pr[u], off);
    if (lane == 0)
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int q = g + 4 * (c0 + u);
        if (q < K) red[h][q] = pr[u];
      }
  }
  __syncthreads();
  if (tid < K) part[tid] = red[0][tid] + red[1][tid];
}

// backward: v[k..k+K) <- L11^-T (v[k..k+K) - sum of the tiles' partials),
// the partials summed in a fixed order (kParts interleaved runs of tiles,
// then the runs in order).  L11 is staged transposed (row i of L11
// contiguous, stride kSnNB + 1), then one warp runs the chain: lane owns
// x_j for j = lane + 32 r; x_i is final when step i (descending) starts,
// is broadcast from its owner, and L(i, j) x_i leaves every x_j, j < i.
template <typename T>
__global__ void __launch_bounds__(kDiagSolveThreads) k_sn_bwd_diag(SnDev d, int base) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16;
  if (!d.srun[d.inst[s]]) return;
  extern __shared__ __align__(16) unsigned char sraw[];
  T *LT = reinterpret_cast<T *>(sraw);  // LT[i (kSnNB + 1) + j] = L(i, j)
  constexpr int KP = kSnNB + 1;
  constexpr int kParts = kDiagSolveThreads / kSnNB;  // threads per partial sum
  __shared__ double a[kParts][kSnNB];
  const long long ld = d.ld[s];
  double *v = d.S + d.soff[s];
  const double *part = v + ld;
  const int e = k0 + K;
  const T *f = reinterpret_cast<const T *>(d.F) + d.foff[s] + k0 * ld + k0;
#pragma unroll 8
  for (int it = 0; it < kSnNB * kSnNB / 2 / kDiagSolveThreads; ++it) {
    const int p = threadIdx.x + it * kDiagSolveThreads, j = p >> 6, i = (p & 63) * 2;
    if (j < K && i < K) {
      const Pair<T> w = load_pair(f + j * ld + i);
      LT[i * KP + j] = w.x;
      LT[(i + 1) * KP + j] = w.y;
    }
  }
  // the tiles' partials of column q: thread (q, h) sums tiles h, h + kParts,
  // ... in order; the kParts sums are then added in order
  {
    const int q = threadIdx.x & (kSnNB - 1), h = threadIdx.x / kSnNB;
    double acc = 0.0;
    if (q < K)
#pragma unroll 8
      for (long long r0 = e + (long long)h * kSnNB; r0 < ld; r0 += kParts * kSnNB)
        acc += part[r0 + q];
    a[h][q] = acc;
  }
  __syncthreads();
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  double xr[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int j = lane + 32 * r;
    double sum = 0.0;
#pragma unroll
    for (int h = 0; h < kParts; ++h) sum += a[h][j];
    xr[r] = j < K ? v[k0 + j] - sum : 0.0;
  }
#pragma unroll
  for (int sb = 3; sb >= 0; --sb) {
    if (32 * sb >= K) continue;
#pragma unroll
    for (int jj = 31; jj >= 0; --jj) {
      const int i = 32 * sb + jj;
      if (i >= K) continue;  // uniform over the warp
      const double xi = __shfl_sync(0xffffffffu, xr[sb], jj);
#pragma unroll
      for (int r = 0; r <= sb; ++r) {
        const int j = 32 * r + lane;
        if (j < i) xr[r] -= double(LT[i * KP + j]) * xi;
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
    if (lane + 32 * r < K) v[k0 + lane + 32 * r] = xr[r];
}

__global__ void __launch_bounds__(kVecThreads) k_sn_bwd_scatter(SnDev d, int base) {
  const int s = d.tasks[base + blockIdx.x].x;
  if (!d.srun[d.inst[s]]) return;
  const int nc = d.ncol[s];
  const double *v = d.S + d.soff[s];
  for (int i = threadIdx.x; i < nc; i += kVecThreads) d.y[vix(d, d.col0g[s] + i)] = v[i];
}

// y <- D^-1 y over the plan's running instances
__global__ void k_sn_dscale(SnDev d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.vcount) return;
  const int inst = d.vinst[i];
  if (inst < 0 || !d.srun[inst]) return;
  d.y[i] *= d.Dinv[d.vbase + i];
}

// ------------------------------------------------------------- refinement
__device__ __forceinline__ void nrm_max(unsigned long long *a, double v) {
  if (!(v >= 0.0)) v = CUDART_INF;  // NaN counts as infinite
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

// b, y from the right-hand side (rx by x index, rz by z row; gsrc codes);
// |b|_inf; zeroes |e|_inf
__global__ void k_sn_rhs(SnDev d, KKTDev k, const double *rx, const double *rz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.vcount) return;
  const int inst = d.vinst[i];
  if (inst < 0 || !d.srun[inst]) return;
  const int g = k.gsrc[d.vbase + i];
  const double v = g >= 0 ? rx[g] : (g == -1 ? 0.0 : rz[-g - 2]);
  d.b[i] = v;
  d.y[i] = v;
  nrm_max(d.nrm + 2 * inst, fabs(v));
}

// e = b - K xs, |e|_inf (K with its true diagonal)
__global__ void k_sn_resid(SnDev d, KKTDev k, const double *xs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.vcount) return;
  const int inst = d.vinst[i];
  if (inst < 0 || !d.srun[inst]) return;
  const int vb = k.voff[inst], r = d.vbase + i - vb;
  const int *kp = k.Kp + k.poff[inst];
  double t = 0;
  for (int p = kp[r]; p < kp[r + 1]; ++p) t += k.Kx[p] * xs[vb + k.Kj[p] - d.vbase];
  const double e = d.b[i] - t;
  d.e[i] = e;
  nrm_max(d.nrm + 2 * inst + 1, fabs(e));
}

__global__ void k_sn_zero_nrm(SnDev d, int which, int B) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < B && d.srun[i]) d.nrm[2 * i + which] = 0ull;
}

// mode 0: x = y; 1: y = e; 2: xn = x + y; 3: x = xn
__global__ void k_sn_vec(SnDev d, int mode) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.vcount) return;
  const int inst = d.vinst[i];
  if (inst < 0 || !d.srun[inst]) return;
  switch (mode) {
    case 0: d.x[i] = d.y[i]; break;
    case 1: d.y[i] = d.e[i]; break;
    case 2: d.xn[i] = d.x[i] + d.y[i]; break;
    default: d.x[i] = d.xn[i]; break;
  }
}

// solution scatter (permuted -> x index / z row)
__global__ void k_sn_out(SnDev d, KKTDev k, double *lx, double *lz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.vcount) return;
  const int inst = d.vinst[i];
  if (inst < 0 || !d.srun[inst]) return;
  const int g = k.gsrc[d.vbase + i];
  if (g >= 0) {
    if (lx) lx[g] = d.x[i];
  } else if (g <= -2) {
    if (lz) lz[-g - 2] = d.x[i];
  }
}

__global__ void k_sn_flags(const int *insts, int n, const int *run, const int *ok, int *flags) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a < n) flags[a] = (run[insts[a]] && ok[insts[a]]) ? 1 : 0;
}

__global__ void k_sn_clear_ok(const int *insts, const int *bad, int n, int *ok) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a < n && bad[a]) ok[insts[a]] = 0;
}

inline int nb256(long long n) { return n <= 0 ? 1 : (int)((n + 255) / 256); }

template <typename T>
size_t diag_smem() {  // the block and the scaled columns of one column block
  return (size_t)kSnNB * kSnNB * sizeof(T) + (size_t)kDiagNB * kSnNB * sizeof(T);
}
template <typename T>
size_t trsm_smem() {  // the tile (kSnNB x kSnNB) and the packed strict lower L11
  return (size_t)kSnNB * kSnNB * sizeof(T) + (size_t)kSnNB * (kSnNB - 1) / 2 * sizeof(T);
}
template <typename T>
size_t gemm_smem() {
  return (size_t)kUpdStages * kUpdKC * (kUpdLdA + kUpdLdB) * sizeof(T);
}

template <typename T>
void set_sn_attrs() {
  static bool done = false;
  if (done) return;
  cudaFuncSetAttribute(k_sn_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)diag_smem<T>());
  cudaFuncSetAttribute(k_sn_small<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)((kSnSmallMax * kSnSmallMax + kSnSmallMax) * sizeof(T)));
  cudaFuncSetAttribute(k_sn_trsm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)trsm_smem<T>());
  cudaFuncSetAttribute(k_sn_fwd_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(kSnNB * kSnNB * sizeof(T)));
  cudaFuncSetAttribute(k_sn_bwd_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(kSnNB * (kSnNB + 1) * sizeof(T)));
  if (sizeof(T) == 8)
    cudaFuncSetAttribute(k_sn_update_f64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)gemm_smem<double>());
  else
    cudaFuncSetAttribute(k_sn_update_f32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)gemm_smem<float>());
  done = true;
}

// profiling: an event pair around one launch
void prof_begin(SnExec &ex, const SnLaunch &L, cudaStream_t st) {
  if (!ex.prof.on) return;
  auto &P = ex.prof;
  const size_t k = P.kinds.size();
  while (P.pool.size() < 2 * k + 2) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) {
      P.on = false;
      return;
    }
    P.pool.push_back(e);
  }
  P.kinds.push_back(L.kind);
  P.flops[L.kind] += L.flops;
  P.calls[L.kind]++;
  cudaEventRecord(P.pool[2 * k], st);
}
void prof_end(SnExec &ex, cudaStream_t st) {
  if (!ex.prof.on || ex.prof.kinds.empty()) return;
  cudaEventRecord(ex.prof.pool[2 * ex.prof.kinds.size() - 1], st);
}
// sum the recorded pairs (waits for the last one)
void prof_collect(SnExec &ex) {
  auto &P = ex.prof;
  if (!P.on || P.kinds.empty()) return;
  cudaEventSynchronize(P.pool[2 * P.kinds.size() - 1]);
  for (size_t k = 0; k < P.kinds.size(); ++k) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, P.pool[2 * k], P.pool[2 * k + 1]) == cudaSuccess)
      P.ms[P.kinds[k]] += t;
  }
  P.kinds.clear();
}

template <typename T>
void run_factor(SnExec &ex, const KKTDev &k, const LDLParams &p, const int *run, int *ok,
                cudaStream_t st) {
  set_sn_attrs<T>();
  const SnDev &d = ex.d;
  for (const SnLaunch &L : ex.fact) {
    prof_begin(ex, L, st);
    switch (L.kind) {
      case SN_SMALL_FACTOR:
        k_sn_small<T><<<L.count, kSmallThreads, (L.smem + kSnSmallMax) * sizeof(T), st>>>(
            d, k, p, L.begin, run, ok);
        break;
      case SN_ASSEMBLE:
        k_sn_assemble<T><<<L.count, kAsmThreads, 0, st>>>(d, k, L.begin, run);
        break;
      case SN_DIAG:
        k_sn_diag<T><<<L.count, kDiagThreads, diag_smem<T>(), st>>>(d, k, p, L.begin, run, ok);
        break;
      case SN_TRSM:
        k_sn_trsm<T><<<L.count, kTrsmThreads, trsm_smem<T>(), st>>>(d, L.begin, run);
        break;
      case SN_UPDATE:
        if (sizeof(T) == 8)
          k_sn_update_f64<<<L.count, kUpdThreads, gemm_smem<double>(), st>>>(d, L.begin, run);
        else
          k_sn_update_f32<<<L.count, 128, gemm_smem<float>(), st>>>(d, L.begin, run);
        break;
      default:
        break;
    }
    prof_end(ex, st);
    ex.launches++;
  }
  prof_collect(ex);
}

// one pass y <- K^-1 y for the instances with srun set
template <typename T>
void run_solve_pass(SnExec &ex, cudaStream_t st) {
  set_sn_attrs<T>();
  const SnDev &d = ex.d;
  for (const SnLaunch &L : ex.fwd) {
    prof_begin(ex, L, st);
    switch (L.kind) {
      case SN_FWD_SMALL: k_sn_fwd_small<T><<<(L.count + 7) / 8, 256, 0, st>>>(d, L.begin, L.count); break;
      case SN_FWD_GATHER: k_sn_fwd_gather<<<(L.count + 7) / 8, 256, 0, st>>>(d, L.begin, L.count); break;
      case SN_FWD_DIAG:
        k_sn_fwd_diag<T><<<L.count, kDiagSolveThreads, kSnNB * kSnNB * sizeof(T), st>>>(d, L.begin);
        break;
      case SN_FWD_GEMV: k_sn_fwd_gemv<T><<<L.count, kGemvThreads, 0, st>>>(d, L.begin); break;
      case SN_FWD_SCATTER: k_sn_fwd_scatter<<<L.count, kVecThreads, 0, st>>>(d, L.begin); break;
      default: break;
    }
    prof_end(ex, st);
    ex.launches++;
  }
  k_sn_dscale<<<nb256(d.vcount), 256, 0, st>>>(d);
  for (const SnLaunch &L : ex.bwd) {
    prof_begin(ex, L, st);
    switch (L.kind) {
      case SN_BWD_SMALL: k_sn_bwd_small<T><<<(L.count + 7) / 8, 256, 0, st>>>(d, L.begin, L.count); break;
      case SN_BWD_GATHER: k_sn_bwd_gather<<<L.count, kVecThreads, 0, st>>>(d, L.begin); break;
      case SN_BWD_PARTIAL: k_sn_bwd_partial<T><<<L.count, kGemvThreads, 0, st>>>(d, L.begin); break;
      case SN_BWD_DIAG:
        k_sn_bwd_diag<T><<<L.count, kDiagSolveThreads, kSnNB * (kSnNB + 1) * sizeof(T), st>>>(
            d, L.begin);
        break;
      case SN_BWD_SCATTER: k_sn_bwd_scatter<<<L.count, kVecThreads, 0, st>>>(d, L.begin); break;
      default: break;
    }
    prof_end(ex, st);
    ex.launches++;
  }
  ex.launches++;
  prof_collect(ex);
}

// one pass, replayed from a CUDA graph when possible (direct launches while
// profiling or if capturing failed)
template <typename T>
void solve_pass(SnExec &ex, cudaStream_t st) {
  if (!ex.prof.on && !ex.g_pass && !ex.graph_failed) {
    set_sn_attrs<T>();
    bool ok = ex.cap || cudaStreamCreateWithFlags(&ex.cap, cudaStreamNonBlocking) == cudaSuccess;
    cudaGraph_t g = nullptr;
    const long long before = ex.launches;
    if (ok) ok = cudaStreamBeginCapture(ex.cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      run_solve_pass<T>(ex, ex.cap);
      ok = cudaStreamEndCapture(ex.cap, &g) == cudaSuccess && g;
    }
    if (ok) ok = cudaGraphInstantiate(&ex.g_pass, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    ex.pass_launches = ex.launches - before;
    ex.launches = before;
    if (!ok) {
      ex.g_pass = nullptr;
      ex.graph_failed = true;
      cudaGetLastError();  // clear a capture error; the pass runs directly
    }
  }
  if (!ex.prof.on && ex.g_pass) {
    cudaGraphLaunch(ex.g_pass, st);
    ex.launches += ex.pass_launches;
  } else {
    run_solve_pass<T>(ex, st);
  }
}

}  // namespace

void sn_set_profiling(SnExec &ex, bool on) {
  ex.prof.on = on;
  ex.prof.kinds.clear();
  if (on) {
    ex.ir_solves = ex.ir_sweeps = ex.ir_unconverged = 0;
    ex.ir_worst = 0.0;
  }
  if (on)
    for (int k = 0; k < SN_KINDS; ++k) {
      ex.prof.ms[k] = ex.prof.flops[k] = 0.0;
      ex.prof.calls[k] = 0;
    }
}

void sn_get_profile(const SnExec &ex, double *ms, double *flops, long long *calls) {
  for (int k = 0; k < SN_KINDS; ++k) {
    if (ms) ms[k] = ex.prof.ms[k];
    if (flops) flops[k] = ex.prof.flops[k];
    if (calls) calls[k] = ex.prof.calls[k];
  }
}

SnExec::~SnExec() {
  if (g_pass) cudaGraphExecDestroy(g_pass);
  if (cap) cudaStreamDestroy(cap);
  for (cudaEvent_t e : prof.pool) cudaEventDestroy(e);
  if (h_srun) pinned_give(h_srun);
  if (h_flags) pinned_give(h_flags);
  if (h_nrm) pinned_give(h_nrm);
}

bool sn_exec_create(const SnPlan &P, bool fp32, int B, int vbase, int vcount,
                    const std::vector<int> &vinst, DevArena &A, SnExec &ex) {
  ex.fp32 = fp32;
  ex.B = B;
  ex.fact = P.fact;
  ex.fwd = P.fwd;
  ex.bwd = P.bwd;
  ex.insts = P.insts;
  ex.small_smem = P.small_smem_max;
  ex.flops = P.flops;
  SnDev &d = ex.d;
  d.inst = A.upload(P.inst);
  d.col0g = A.upload(P.col0g);
  d.ncol = A.upload(P.ncol);
  d.nrow = A.upload(P.nrow);
  d.u0 = A.upload(P.u0);
  d.ld = A.upload(P.ld);
  d.cbase = A.upload(P.cbase);
  d.fix_off = A.upload(P.fix_off);
  d.rel_off = A.upload(P.rel_off);
  d.ch_ptr = A.upload(P.ch_ptr);
  d.ch = A.upload(P.ch);
  d.uoff = A.upload(P.uoff);
  d.fidx = A.upload(P.fidx);
  d.rel = A.upload(P.rel);
  d.acol = A.upload(P.acol);
  d.foff = A.upload(P.foff);
  d.woff = A.upload(P.woff);
  d.soff = A.upload(P.soff);
  d.amap = reinterpret_cast<const int2 *>(A.upload(P.amap));
  d.tasks = reinterpret_cast<const int4 *>(A.upload(P.tasks));
  d.cl_ptr = A.upload(P.cl_ptr);
  d.clist = reinterpret_cast<const int4 *>(A.upload(P.clist));
  const size_t ts = fp32 ? 4 : 8;
  d.F = fp32 ? (void *)A.alloc<float>(P.f_elems) : (void *)A.alloc<double>(P.f_elems);
  d.W = fp32 ? (void *)A.alloc<float>(P.w_elems) : (void *)A.alloc<double>(P.w_elems);
  (void)ts;
  d.S = A.alloc<double>(P.s_elems);
  d.U = A.alloc<double>(P.u_elems);
  d.Dinv = A.alloc<double>((size_t)vbase + vcount);
  d.eps = A.alloc<double>(B);
  d.srun = A.alloc<int>(B);
  d.nrm = A.alloc<unsigned long long>(2 * (size_t)B);
  d.b = A.alloc<double>(vcount);
  d.x = A.alloc<double>(vcount);
  d.xn = A.alloc<double>(vcount);
  d.e = A.alloc<double>(vcount);
  d.y = A.alloc<double>(vcount);
  d.vinst = A.upload(vinst);
  d.vbase = vbase;
  d.vcount = vcount;
  ex.d_insts = A.upload(P.insts);
  ex.d_flags = A.alloc<int>(B);
  if (pinned_take(&ex.h_srun, sizeof(int) * B) != cudaSuccess) return false;
  if (pinned_take(&ex.h_flags, sizeof(int) * B) != cudaSuccess) return false;
  if (pinned_take(&ex.h_nrm, sizeof(unsigned long long) * 2 * B) != cudaSuccess) return false;
  return A.err == cudaSuccess;
}

void sn_factor(SnExec &ex, const KKTDev &k, const LDLParams &p, const int *run, int *ok,
               double *eps_out, cudaStream_t st) {
  if (ex.insts.empty()) return;
  k_sn_eps<<<(int)ex.insts.size(), kAsmThreads, 0, st>>>(ex.d, k, p, ex.d_insts, run, eps_out);
  ex.launches++;
  if (ex.fp32)
    run_factor<float>(ex, k, p, run, ok, st);
  else
    run_factor<double>(ex, k, p, run, ok, st);
}

void sn_solve(SnExec &ex, const KKTDev &k, const LDLParams &p, const int *run, const double *rx,
              const double *rz, double *lx, double *lz, int *ok, cudaStream_t st) {
  const int n = (int)ex.insts.size();
  if (n == 0) return;
  SnDev &d = ex.d;
  const int B = ex.B;
  auto pass = [&]() {
    if (ex.fp32)
      solve_pass<float>(ex, st);
    else
      solve_pass<double>(ex, st);
  };
  auto upload_srun = [&](const std::vector<char> &on) {
    cudaStreamSynchronize(st);  // the previous upload has left the staging
    for (int i = 0; i < B; ++i) ex.h_srun[i] = 0;
    for (int a = 0; a < n; ++a) ex.h_srun[ex.insts[a]] = on[a] ? 1 : 0;
    cudaMemcpyAsync(d.srun, ex.h_srun, sizeof(int) * B, cudaMemcpyHostToDevice, st);
  };
  auto read_nrm = [&]() {
    cudaMemcpyAsync(ex.h_nrm, d.nrm, sizeof(unsigned long long) * 2 * B, cudaMemcpyDeviceToHost,
                    st);
    cudaStreamSynchronize(st);
  };
  auto as_double = [](unsigned long long u) {
    double v;
    memcpy(&v, &u, sizeof(v));
    return v;
  };
  // instances taking part: run and ok
  k_sn_flags<<<nb256(n), 256, 0, st>>>(ex.d_insts, n, run, ok, ex.d_flags);
  cudaMemcpyAsync(ex.h_flags, ex.d_flags, sizeof(int) * n, cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  std::vector<char> act(n), live(n), bad(n, 0);
  bool any = false;
  for (int a = 0; a < n; ++a) {
    act[a] = ex.h_flags[a] != 0;
    any = any || act[a];
  }
  if (!any) return;
  upload_srun(act);
  k_sn_zero_nrm<<<nb256(B), 256, 0, st>>>(d, 0, B);
  k_sn_zero_nrm<<<nb256(B), 256, 0, st>>>(d, 1, B);
  k_sn_rhs<<<nb256(d.vcount), 256, 0, st>>>(d, k, rx, rz);
  pass();
  k_sn_vec<<<nb256(d.vcount), 256, 0, st>>>(d, 0);  // x = y
  k_sn_resid<<<nb256(d.vcount), 256, 0, st>>>(d, k, d.x);
  read_nrm();
  std::vector<double> normb(n), norme(n);
  for (int a = 0; a < n; ++a) {
    if (!act[a]) continue;
    const int i = ex.insts[a];
    normb[a] = as_double(ex.h_nrm[2 * i]);
    norme[a] = as_double(ex.h_nrm[2 * i + 1]);
    if (!std::isfinite(norme[a])) bad[a] = 1;  // non-finite solution
    live[a] = act[a] && !bad[a] && p.ir_enable;
  }
  // iterative refinement (kktsolver_directldl_gpu.jl:349-410): stop at the
  // tolerance, after ir_maxiter sweeps, or when a sweep improves the error
  // by less than ir_stopratio (keeping the better iterate)
  for (int it = 0; p.ir_enable && it < p.ir_maxiter; ++it) {
    std::vector<char> cont(n, 0);
    bool anyc = false;
    for (int a = 0; a < n; ++a) {
      if (!live[a]) continue;
      if (norme[a] <= p.ir_abstol + p.ir_reltol * normb[a]) {
        live[a] = 0;
        continue;
      }
      cont[a] = 1;
      anyc = true;
    }
    if (!anyc) break;
    ex.ir_sweeps++;
    upload_srun(cont);
    k_sn_vec<<<nb256(d.vcount), 256, 0, st>>>(d, 1);  // y = e
    pass();
    k_sn_vec<<<nb256(d.vcount), 256, 0, st>>>(d, 2);  // xn = x + y
    k_sn_zero_nrm<<<nb256(B), 256, 0, st>>>(d, 1, B);
    k_sn_resid<<<nb256(d.vcount), 256, 0, st>>>(d, k, d.xn);
    read_nrm();
    std::vector<char> accept(n, 0);
    bool anya = false;
    for (int a = 0; a < n; ++a) {
      if (!cont[a]) continue;
      const double ne = as_double(ex.h_nrm[2 * ex.insts[a] + 1]);
      if (!std::isfinite(ne)) {
        bad[a] = 1;
        live[a] = 0;
        continue;
      }
      const double ratio = norme[a] / ne;
      if (ratio < p.ir_stopratio) {
        live[a] = 0;
        if (ratio > 1.0) accept[a] = 1;
      } else {
        accept[a] = 1;
      }
      if (accept[a]) {
        norme[a] = ne;
        anya = true;
      }
    }
    if (anya) {
      upload_srun(accept);
      k_sn_vec<<<nb256(d.vcount), 256, 0, st>>>(d, 3);  // x = xn
    }
  }
  std::vector<char> good(n);
  for (int a = 0; a < n; ++a) good[a] = act[a] && !bad[a];
  for (int a = 0; a < n; ++a) {
    if (!act[a]) continue;
    ex.ir_solves++;
    const double tol = p.ir_abstol + p.ir_reltol * normb[a];
    if (p.ir_enable && !bad[a] && norme[a] > tol) {
      ex.ir_unconverged++;
      ex.ir_worst = std::max(ex.ir_worst, norme[a] / tol);
    }
  }
  upload_srun(good);
  k_sn_out<<<nb256(d.vcount), 256, 0, st>>>(d, k, lx, lz);
  bool anybad = false;
  for (int a = 0; a < n; ++a) {
    ex.h_flags[a] = bad[a];
    anybad = anybad || bad[a];
  }
  if (anybad) {
    cudaMemcpyAsync(ex.d_flags, ex.h_flags, sizeof(int) * n, cudaMemcpyHostToDevice, st);
    k_sn_clear_ok<<<nb256(n), 256, 0, st>>>(ex.d_insts, ex.d_flags, n, ok);
  }
  cudaStreamSynchronize(st);  // pinned staging is reused by the next call
}

}  // namespace clgpu
