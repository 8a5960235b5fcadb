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
      for (int r = q + tid; r < cn; r += kAsmThreads) f[pc * ld + rel[r]] += src[r];
    }
    __syncthreads();
  }
}

// Diagonal block of a panel: factor the K x K block (right-looking, the
// static shift was applied at assembly), write L11 and D to the front and
// 1/d to the workspace.
template <typename T>
__global__ void __launch_bounds__(kDiagThreads) k_sn_diag(SnDev d, KKTDev k, LDLParams prm,
                                                         int base, const int *run, int *ok) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16, inst = d.inst[s];
  if (!run[inst]) return;
  extern __shared__ __align__(16) unsigned char sraw[];
  T *blk = reinterpret_cast<T *>(sraw);  // K x K, column-major, stride K
  T *col = blk + K * K;
  const long long ld = d.ld[s];
  T *f = reinterpret_cast<T *>(d.F) + d.foff[s];
  T *ws = reinterpret_cast<T *>(d.W) + d.woff[s];
  const int *fi = d.fidx + d.fix_off[s];
  const int tid = threadIdx.x;
  for (int idx = tid; idx < K * K; idx += kDiagThreads) {
    const int c = idx / K, r = idx - c * K;
    blk[idx] = r >= c ? f[(k0 + c) * ld + k0 + r] : T(0);
  }
  __syncthreads();
  bool bad = false;
  for (int j = 0; j < K; ++j) {
    const T dj = T(sn_pivot(double(blk[j * K + j]), pivot_sign(k, fi[k0 + j]), prm));
    for (int i = j + 1 + tid; i < K; i += kDiagThreads) col[i] = blk[j * K + i];
    __syncthreads();
    // rank-1 update of the trailing lower triangle: 16 x 16 threads, thread
    // (tx, ty) takes columns j+1+ty, +16, ... and rows i >= r, i = j+1+tx, +16, ...
    {
      const int tx = tid & 15, ty = tid >> 4;
      for (int r = j + 1 + ty; r < K; r += 16) {
        const T cr = col[r];
        for (int i = j + 1 + tx; i < K; i += 16)
          if (i >= r) blk[r * K + i] -= (col[i] / dj) * cr;
      }
    }
    for (int i = j + 1 + tid; i < K; i += kDiagThreads) blk[j * K + i] = col[i] / dj;
    if (tid == 0) {
      blk[j * K + j] = dj;
      const double di = 1.0 / double(dj);
      const int g = fi[k0 + j];
      if (g >= 0) d.Dinv[g] = di;
      ws[j] = T(di);
      if (!isfinite(di) || !isfinite(double(dj))) bad = true;
    }
    __syncthreads();
  }
  for (int idx = tid; idx < K * K; idx += kDiagThreads) {
    const int c = idx / K, r = idx - c * K;
    if (r >= c) f[(k0 + c) * ld + k0 + r] = blk[idx];
  }
  for (int j = K + tid; j < kSnNB; j += kDiagThreads) ws[j] = T(0);
  if (bad && tid == 0) ok[inst] = 0;
}

// TRSM of a panel's row tile: rows r0..r0+127 of panel [k0, k0+K),
// W = A L11^-T by column-oriented substitution (after step j column j of W
// is final and is subtracted, times L11(t, j), from every later column t),
// then L = W D^-1: L overwrites A in the front, W goes to the workspace for
// the trailing update.  The tile (K x 128) and the strict lower triangle of
// L11 (packed by columns) sit in shared memory.
template <typename T>
__global__ void __launch_bounds__(kTrsmThreads) k_sn_trsm(SnDev d, int base, const int *run) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16, r0 = t.z;
  if (!run[d.inst[s]]) return;
  extern __shared__ __align__(16) unsigned char sraw[];
  T *X = reinterpret_cast<T *>(sraw);  // column q of the tile at X + q kSnNB
  T *Lp = X + K * kSnNB;               // column j of L11 below the diagonal at Lp + cs(j)
  const long long ld = d.ld[s];
  T *f = reinterpret_cast<T *>(d.F) + d.foff[s];
  const T *ws = reinterpret_cast<const T *>(d.W) + d.woff[s];
  T *wr = reinterpret_cast<T *>(d.W) + d.woff[s] + kSnNB;
  const int tid = threadIdx.x;
  auto cs = [K](int j) { return j * (K - 1) - j * (j - 1) / 2; };
  for (int idx = tid; idx < K * kSnNB; idx += kTrsmThreads) {
    const int q = idx / kSnNB, m = idx - q * kSnNB;
    X[idx] = f[(k0 + q) * ld + r0 + m];
  }
  for (int j = 0; j < K; ++j)
    for (int i = j + 1 + tid; i < K; i += kTrsmThreads) Lp[cs(j) + i - j - 1] = f[(k0 + j) * ld + k0 + i];
  __syncthreads();
  const int m = tid & (kSnNB - 1), half = tid / kSnNB;
  for (int j = 0; j + 1 < K; ++j) {
    const T xj = X[j * kSnNB + m];
    const T *lc = Lp + cs(j) - j - 1;
    for (int q = j + 1 + half; q < K; q += kTrsmThreads / kSnNB) X[q * kSnNB + m] -= xj * lc[q];
    __syncthreads();
  }
  for (int idx = tid; idx < K * kSnNB; idx += kTrsmThreads) {
    const int q = idx / kSnNB, mm = idx - q * kSnNB;
    const T w = X[idx];
    wr[(long long)q * ld + r0 + mm] = w;
    f[(k0 + q) * ld + r0 + mm] = w * ws[q];
  }
}

// Trailing update of the blocked fronts, one 128 x 64 tile per block:
// front tile (r0, c0) -= L(r0.., panel) W(c0.., :)^T, entries on or below
// the diagonal only (r0 + m >= c0 + n).  K (a multiple of kSnKPad = 16) is
// streamed in chunks of kUpdKC through a kUpdStages-deep cp.async pipeline;
// two blocks are resident per SM, so one's prologue and epilogue overlap the
// other's main loop.
// FP64: 4 warps as 2 (rows) x 2 (columns), warp tile 64 x 32 of m8n8k4 DMMA.
__global__ void __launch_bounds__(128, 2) k_sn_update_f64(SnDev d, int base, const int *run) {
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
  const int wm = warp & 1, wn = warp >> 1;
  double acc[8][4][2];
#pragma unroll
  for (int mi = 0; mi < 8; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
  const int nchunks = K / kUpdKC;
  constexpr int kStage = kUpdKC * (kUpdLdA + kUpdLdB);
  auto load = [&](int chunk, int stage) {
    double *As = sm + stage * kStage, *Bs = As + kUpdKC * kUpdLdA;
    // A: kUpdKC columns x 64 pieces of 16 B; B: kUpdKC x 32
    for (int p = tid; p < kUpdKC * 64; p += 128) {
      const int q = p >> 6, m = (p & 63) * 2;
      cp_async16(As + q * kUpdLdA + m, Ag + ((long long)chunk * kUpdKC + q) * ld + m);
    }
    for (int p = tid; p < kUpdKC * 32; p += 128) {
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
      double a[8], b[4];
#pragma unroll
      for (int mi = 0; mi < 8; ++mi) a[mi] = As[q * kUpdLdA + wm * 64 + mi * 8 + (lane >> 2)];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) b[ni] = Bs[q * kUpdLdB + wn * 32 + ni * 8 + (lane >> 2)];
#pragma unroll
      for (int mi = 0; mi < 8; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) dmma884(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
    }
  }
  cp_async_wait<0>();
  const bool diag = r0 < c0 + 64;  // the tile reaches above the diagonal
#pragma unroll
  for (int mi = 0; mi < 8; ++mi) {
    const int m = wm * 64 + mi * 8 + (lane >> 2);
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int n = wn * 32 + ni * 8 + 2 * (lane & 3) + h;
        if (!diag || r0 + m >= c0 + n) f[(long long)(c0 + n) * ld + r0 + m] -= acc[mi][ni][h];
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
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
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
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
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
      if (!diag || r0 + m >= c0 + n) f[(long long)(c0 + n) * ld + r0 + m] -= acc[i][j];
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

// forward: v[k..k+K) <- L11^-1 v[k..k+K).  L11's strict lower triangle is
// first copied to shared memory (coalesced), so the K dependent steps read
// shared memory only.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_sn_fwd_diag(SnDev d, int base) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16;
  if (!d.srun[d.inst[s]]) return;
  extern __shared__ __align__(16) unsigned char sraw[];
  T *Ls = reinterpret_cast<T *>(sraw);  // K x K, column-major, stride K
  __shared__ double x[kSnNB];
  const long long ld = d.ld[s];
  double *v = d.S + d.soff[s] + k0;
  const T *f = reinterpret_cast<const T *>(d.F) + d.foff[s] + k0 * ld + k0;
  const int i = threadIdx.x;
  for (int j = 0; j < K; ++j)
    if (i < K) Ls[j * K + i] = f[j * ld + i];
  if (i < K) x[i] = v[i];
  __syncthreads();
  double xi = i < K ? x[i] : 0.0;
  for (int j = 0; j < K; ++j) {
    if (i == j) x[j] = xi;
    __syncthreads();
    if (i > j && i < K) xi -= double(Ls[j * K + i]) * x[j];
  }
  if (i < K) v[i] = xi;
}
// forward: v[r0..r0+128) -= L(r0.., panel) v[k..k+K)
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_sn_fwd_gemv(SnDev d, int base) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16, r0 = t.z;
  if (!d.srun[d.inst[s]]) return;
  __shared__ double x[kSnNB];
  const long long ld = d.ld[s];
  double *v = d.S + d.soff[s];
  if (threadIdx.x < K) x[threadIdx.x] = v[k0 + threadIdx.x];
  __syncthreads();
  const T *f = reinterpret_cast<const T *>(d.F) + d.foff[s] + k0 * ld + r0 + threadIdx.x;
  double acc = 0;
  for (int q = 0; q < K; ++q) acc += double(f[q * ld]) * x[q];
  v[r0 + threadIdx.x] -= acc;
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

// backward: partial sums over the row tile r0: p[q] = sum_m L(r0 + m, k + q) v[r0 + m]
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_sn_bwd_partial(SnDev d, int base) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16, r0 = t.z;
  if (!d.srun[d.inst[s]]) return;
  const long long ld = d.ld[s];
  const double *v = d.S + d.soff[s] + r0;
  double *part = d.S + d.soff[s] + ld + r0;  // tile r0's partials at [r0, r0 + K)
  const T *f = reinterpret_cast<const T *>(d.F) + d.foff[s] + k0 * ld + r0;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double vm[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) vm[e] = v[lane * 4 + e];
  for (int q = w; q < K; q += kVecThreads / 32) {
    const T *fc = f + q * ld + lane * 4;
    double acc = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) acc += double(fc[e]) * vm[e];
    acc = warp_sum(acc);
    if (lane == 0) part[q] = acc;
  }
}

// backward: v[k..k+K) <- L11^-T (v[k..k+K) - sum of the tiles' partials),
// the partials summed in tile order; L11 staged in shared memory, then one
// warp runs the K dependent column dot products
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_sn_bwd_diag(SnDev d, int base) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16;
  if (!d.srun[d.inst[s]]) return;
  extern __shared__ __align__(16) unsigned char sraw[];
  T *Ls = reinterpret_cast<T *>(sraw);  // K x K, column-major, stride K
  __shared__ double x[kSnNB];
  const long long ld = d.ld[s];
  double *v = d.S + d.soff[s];
  const double *part = v + ld;
  const int q = threadIdx.x, e = k0 + K;
  const T *f = reinterpret_cast<const T *>(d.F) + d.foff[s] + k0 * ld + k0;
  for (int j = 0; j < K; ++j)
    if (q < K) Ls[j * K + q] = f[j * ld + q];
  if (q < K) {
    double a = v[k0 + q];
    for (long long r0 = e; r0 < ld; r0 += kSnNB) a -= part[r0 + q];
    x[q] = a;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    for (int j = K - 1; j >= 0; --j) {
      double acc = 0;
      for (int i = j + 1 + lane; i < K; i += 32) acc += double(Ls[j * K + i]) * x[i];
      acc = warp_sum(acc);
      if (lane == 0) x[j] -= acc;
      __syncwarp();
    }
  }
  __syncthreads();
  if (q < K) v[k0 + q] = x[q];
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
size_t diag_smem() {
  return (size_t)kSnNB * kSnNB * sizeof(T) + kSnNB * sizeof(T);
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
                       (int)(kSnNB * kSnNB * sizeof(T)));
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
          k_sn_update_f64<<<L.count, 128, gemm_smem<double>(), st>>>(d, L.begin, run);
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
        k_sn_fwd_diag<T><<<L.count, kVecThreads, kSnNB * kSnNB * sizeof(T), st>>>(d, L.begin);
        break;
      case SN_FWD_GEMV: k_sn_fwd_gemv<T><<<L.count, kVecThreads, 0, st>>>(d, L.begin); break;
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
      case SN_BWD_PARTIAL: k_sn_bwd_partial<T><<<L.count, kVecThreads, 0, st>>>(d, L.begin); break;
      case SN_BWD_DIAG:
        k_sn_bwd_diag<T><<<L.count, kVecThreads, kSnNB * kSnNB * sizeof(T), st>>>(d, L.begin);
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
  for (cudaEvent_t e : prof.pool) cudaEventDestroy(e);
  if (h_srun) cudaFreeHost(h_srun);
  if (h_flags) cudaFreeHost(h_flags);
  if (h_nrm) cudaFreeHost(h_nrm);
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
  if (cudaMallocHost(&ex.h_srun, sizeof(int) * B) != cudaSuccess) return false;
  if (cudaMallocHost(&ex.h_flags, sizeof(int) * B) != cudaSuccess) return false;
  if (cudaMallocHost(&ex.h_nrm, sizeof(unsigned long long) * 2 * B) != cudaSuccess) return false;
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
      run_solve_pass<float>(ex, st);
    else
      run_solve_pass<double>(ex, st);
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
