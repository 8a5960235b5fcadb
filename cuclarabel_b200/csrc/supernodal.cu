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
//                 pivots: k_sn_diag factors the K x K diagonal block and
//                 inverts its unit L, k_sn_gemm<TRSM> forms W = A Linv^T and
//                 L = W D^-1 for every 128-row tile below, and
//                 k_sn_gemm<UPDATE> subtracts L W^T from every lower tile of
//                 the trailing matrix.  FP64 tiles run on the tensor cores
//                 (DMMA, mma.sync m8n8k4), FP32 tiles (mixed form) on FMA
//                 units; both stage their operands with cp.async.
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

constexpr int kGemmKC = 8;       // k per pipeline stage
constexpr int kGemmStages = 4;   // cp.async stages
constexpr int kGemmLd = kSnNB + 4;  // shared row stride (elements): conflict-free fragments
constexpr int kDiagThreads = 256;
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
    const int rem = ld - j - 1;
    for (int idx = tid; idx < rem * rem; idx += kSmallThreads) {
      const int r = j + 1 + idx / rem, i = j + 1 + idx % rem;
      if (i >= r) f[r * ld + i] -= (col[i] / dj) * col[r];
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
// children's Schur complements in order.
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
  for (int a = d.ch_ptr[s]; a < d.ch_ptr[s + 1]; ++a) {
    const int c = d.ch[a], cn = d.nrow[c], cu = d.u0[c];
    const long long cld = d.ld[c];
    const int *rel = d.rel + d.rel_off[c];
    // child columns whose parent position lies in [ca, cb): rel is increasing
    int lo = 0, hi = cn;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (rel[mid] < ca) lo = mid + 1; else hi = mid;
    }
    const int qa = lo;
    hi = cn;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (rel[mid] < cb) lo = mid + 1; else hi = mid;
    }
    const int qb = lo;
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
// static shift was applied at assembly), write L11 and D, and the inverse
// of the unit L11 (zero-padded to kSnNB x kSnNB) and 1/d to the workspace.
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
    const int rem = K - j - 1;
    for (int idx = tid; idx < rem * rem; idx += kDiagThreads) {
      const int r = j + 1 + idx / rem, i = j + 1 + idx % rem;
      if (i >= r) blk[r * K + i] -= (col[i] / dj) * col[r];
    }
    for (int i = j + 1 + tid; i < K; i += kDiagThreads) blk[j * K + i] = col[i] / dj;
    if (tid == 0) {
      blk[j * K + j] = dj;
      const double di = 1.0 / double(dj);
      const int g = fi[k0 + j];
      if (g >= 0) d.Dinv[g] = di;
      ws[kSnNB * kSnNB + j] = T(di);
      if (!isfinite(di) || !isfinite(double(dj))) bad = true;
    }
    __syncthreads();
  }
  for (int idx = tid; idx < K * K; idx += kDiagThreads) {
    const int c = idx / K, r = idx - c * K;
    if (r >= c) f[(k0 + c) * ld + k0 + r] = blk[idx];
  }
  for (int j = K + tid; j < kSnNB; j += kDiagThreads) ws[kSnNB * kSnNB + j] = T(0);
  __syncthreads();
  // in-place inverse of the unit lower L11: after step t row t of X = L^-1
  // is final; rows below subtract L(r, t) times it
  for (int tt = 0; tt + 1 < K; ++tt) {
    for (int r = tt + 1 + tid; r < K; r += kDiagThreads) col[r] = blk[tt * K + r];
    __syncthreads();
    const int w = tt + 1, cnt = (K - 1 - tt) * w;
    for (int idx = tid; idx < cnt; idx += kDiagThreads) {
      const int r = tt + 1 + idx / w, c = idx % w;
      if (c == tt)
        blk[tt * K + r] = -col[r];
      else
        blk[c * K + r] -= col[r] * blk[c * K + tt];
    }
    __syncthreads();
  }
  for (int idx = tid; idx < kSnNB * kSnNB; idx += kDiagThreads) {
    const int q = idx / kSnNB, n = idx - q * kSnNB;  // Linv(n, q) at n + q kSnNB
    T v = T(0);
    if (n < K && q < K) v = n == q ? T(1) : (n > q ? blk[q * K + n] : T(0));
    ws[idx] = v;
  }
  if (bad && tid == 0) ok[inst] = 0;
}

// 128 x 128 tile products of the blocked fronts.
//   TRSM   (MODE 0): rows r0.. of panel [k, k+K): W = A Linv^T -> workspace,
//                    L = W diag(1/d) -> front (in place of A)
//   UPDATE (MODE 1): front tile (r0, c0) -= L(r0.., panel) W(c0.., :)^T,
//                    lower triangle only on a diagonal tile
// FP64: 8 warps as 2 (rows) x 4 (columns), warp tile 64 x 32 of m8n8k4 DMMA.
template <int MODE>
__global__ void __launch_bounds__(256, 1) k_sn_gemm_f64(SnDev d, int base, const int *run) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16, r0 = t.z, c0 = t.w;
  if (!run[d.inst[s]]) return;
  const long long ld = d.ld[s];
  double *f = reinterpret_cast<double *>(d.F) + d.foff[s];
  double *ws = reinterpret_cast<double *>(d.W) + d.woff[s];
  double *wr = ws + kSnNB * kSnNB + kSnNB;
  const double *Ag = f + k0 * ld + r0;
  const double *Bg = MODE == 0 ? ws : wr + c0;
  const long long ldb = MODE == 0 ? kSnNB : ld;
  extern __shared__ __align__(16) unsigned char sraw[];
  double *sm = reinterpret_cast<double *>(sraw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  double acc[8][4][2];
#pragma unroll
  for (int mi = 0; mi < 8; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
  const int nchunks = K / kGemmKC;
  auto load = [&](int chunk, int stage) {
    double *As = sm + stage * 2 * kGemmKC * kGemmLd, *Bs = As + kGemmKC * kGemmLd;
    for (int p = tid; p < kGemmKC * (kSnNB / 2); p += 256) {
      const int q = p / (kSnNB / 2), m = (p % (kSnNB / 2)) * 2;
      const long long kq = (long long)chunk * kGemmKC + q;
      cp_async16(As + q * kGemmLd + m, Ag + kq * ld + m);
      cp_async16(Bs + q * kGemmLd + m, Bg + kq * ldb + m);
    }
  };
#pragma unroll
  for (int st = 0; st < kGemmStages - 1; ++st) {
    if (st < nchunks) load(st, st);
    cp_async_commit();
  }
  for (int c = 0; c < nchunks; ++c) {
    cp_async_wait<kGemmStages - 2>();
    __syncthreads();
    const int nx = c + kGemmStages - 1;
    if (nx < nchunks) load(nx, nx % kGemmStages);
    cp_async_commit();
    const double *As = sm + (c % kGemmStages) * 2 * kGemmKC * kGemmLd;
    const double *Bs = As + kGemmKC * kGemmLd;
#pragma unroll
    for (int kk = 0; kk < kGemmKC; kk += 4) {
      const int row = (kk + (lane & 3)) * kGemmLd + (lane >> 2);
      double a[8], b[4];
#pragma unroll
      for (int mi = 0; mi < 8; ++mi) a[mi] = As[row + wm * 64 + mi * 8];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) b[ni] = Bs[row + wn * 32 + ni * 8];
#pragma unroll
      for (int mi = 0; mi < 8; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) dmma884(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  const double *dinv = ws + kSnNB * kSnNB;
#pragma unroll
  for (int mi = 0; mi < 8; ++mi) {
    const int m = wm * 64 + mi * 8 + (lane >> 2);
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int n = wn * 32 + ni * 8 + 2 * (lane & 3) + h;
        const double v = acc[mi][ni][h];
        if (MODE == 0) {
          if (n < K) {
            wr[(long long)n * ld + r0 + m] = v;
            f[(long long)(k0 + n) * ld + r0 + m] = v * dinv[n];
          }
        } else {
          if (r0 != c0 || m >= n) f[(long long)(c0 + n) * ld + r0 + m] -= v;
        }
      }
  }
}

// FP32 form: 16 x 16 threads, each 8 x 8 outputs (rows ty*4 + {0..3} and
// 64 + ty*4 + {0..3}, columns likewise with tx), FMA units.
template <int MODE>
__global__ void __launch_bounds__(256) k_sn_gemm_f32(SnDev d, int base, const int *run) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16, r0 = t.z, c0 = t.w;
  if (!run[d.inst[s]]) return;
  const long long ld = d.ld[s];
  float *f = reinterpret_cast<float *>(d.F) + d.foff[s];
  float *ws = reinterpret_cast<float *>(d.W) + d.woff[s];
  float *wr = ws + kSnNB * kSnNB + kSnNB;
  const float *Ag = f + k0 * ld + r0;
  const float *Bg = MODE == 0 ? ws : wr + c0;
  const long long ldb = MODE == 0 ? kSnNB : ld;
  extern __shared__ __align__(16) unsigned char sraw[];
  float *sm = reinterpret_cast<float *>(sraw);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
  const int nchunks = K / kGemmKC;
  auto load = [&](int chunk, int stage) {
    float *As = sm + stage * 2 * kGemmKC * kGemmLd, *Bs = As + kGemmKC * kGemmLd;
    const int q = tid / (kSnNB / 4), m = (tid % (kSnNB / 4)) * 4;  // 8 x 32 pieces
    const long long kq = (long long)chunk * kGemmKC + q;
    cp_async16(As + q * kGemmLd + m, Ag + kq * ld + m);
    cp_async16(Bs + q * kGemmLd + m, Bg + kq * ldb + m);
  };
#pragma unroll
  for (int st = 0; st < kGemmStages - 1; ++st) {
    if (st < nchunks) load(st, st);
    cp_async_commit();
  }
  for (int c = 0; c < nchunks; ++c) {
    cp_async_wait<kGemmStages - 2>();
    __syncthreads();
    const int nx = c + kGemmStages - 1;
    if (nx < nchunks) load(nx, nx % kGemmStages);
    cp_async_commit();
    const float *As = sm + (c % kGemmStages) * 2 * kGemmKC * kGemmLd;
    const float *Bs = As + kGemmKC * kGemmLd;
#pragma unroll
    for (int q = 0; q < kGemmKC; ++q) {
      const float4 a0 = *reinterpret_cast<const float4 *>(As + q * kGemmLd + ty * 4);
      const float4 a1 = *reinterpret_cast<const float4 *>(As + q * kGemmLd + 64 + ty * 4);
      const float4 b0 = *reinterpret_cast<const float4 *>(Bs + q * kGemmLd + tx * 4);
      const float4 b1 = *reinterpret_cast<const float4 *>(Bs + q * kGemmLd + 64 + tx * 4);
      const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  const float *dinv = ws + kSnNB * kSnNB;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int m = (i < 4 ? 0 : 64) + ty * 4 + (i & 3);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int n = (j < 4 ? 0 : 64) + tx * 4 + (j & 3);
      const float v = acc[i][j];
      if (MODE == 0) {
        if (n < K) {
          wr[(long long)n * ld + r0 + m] = v;
          f[(long long)(k0 + n) * ld + r0 + m] = v * dinv[n];
        }
      } else {
        if (r0 != c0 || m >= n) f[(long long)(c0 + n) * ld + r0 + m] -= v;
      }
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
  for (int j = 0; j < nc; ++j) {
    const double vj = v[j];
    for (int i = j + 1 + lane; i < ld; i += 32) v[i] -= double(f[j * ld + i]) * vj;
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
  for (int j = nc - 1; j >= 0; --j) {
    double t = 0;
    for (int i = j + 1 + lane; i < ld; i += 32) t += double(f[j * ld + i]) * v[i];
    t = warp_sum(t);
    if (lane == 0) v[j] -= t;
    __syncwarp();
  }
  for (int i = lane; i < nc; i += 32) y[vix(d, d.col0g[s] + i)] = v[i];
}

// blocked fronts: work vector v (ld) from y and the children's contributions
__global__ void __launch_bounds__(kVecThreads) k_sn_fwd_gather(SnDev d, int base) {
  const int s = d.tasks[base + blockIdx.x].x;
  if (!d.srun[d.inst[s]]) return;
  const int ld = d.ld[s], nc = d.ncol[s];
  double *v = d.S + d.soff[s];
  for (int i = threadIdx.x; i < ld; i += kVecThreads) v[i] = i < nc ? d.y[vix(d, d.col0g[s] + i)] : 0.0;
  __syncthreads();
  for (int a = d.ch_ptr[s]; a < d.ch_ptr[s + 1]; ++a) {
    const int c = d.ch[a], cn = d.nrow[c];
    const int *rel = d.rel + d.rel_off[c];
    const double *u = d.U + d.uoff[c];
    for (int q = threadIdx.x; q < cn; q += kVecThreads) v[rel[q]] += u[q];
    __syncthreads();
  }
}

// forward: v[k..k+K) <- L11^-1 v[k..k+K)
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_sn_fwd_diag(SnDev d, int base) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16;
  if (!d.srun[d.inst[s]]) return;
  __shared__ double x[kSnNB];
  const long long ld = d.ld[s];
  double *v = d.S + d.soff[s] + k0;
  const T *f = reinterpret_cast<const T *>(d.F) + d.foff[s] + k0 * ld + k0;
  const int i = threadIdx.x;
  if (i < K) x[i] = v[i];
  __syncthreads();
  for (int j = 0; j < K; ++j) {
    if (i > j && i < K) x[i] -= double(f[j * ld + i]) * x[j];
    __syncthreads();
  }
  if (i < K) v[i] = x[i];
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

// backward: v[k..k+K) <- L11^-T (v[k..k+K) - sum of the tiles' partials)
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_sn_bwd_diag(SnDev d, int base) {
  const int4 t = d.tasks[base + blockIdx.x];
  const int s = t.x, k0 = t.y & 0xffff, K = t.y >> 16;
  if (!d.srun[d.inst[s]]) return;
  __shared__ double x[kSnNB];
  const long long ld = d.ld[s];
  double *v = d.S + d.soff[s];
  const double *part = v + ld;
  const int q = threadIdx.x, e = k0 + K;
  if (q < K) {
    double a = v[k0 + q];
    for (long long r0 = e; r0 < ld; r0 += kSnNB) a -= part[r0 + q];
    x[q] = a;
  }
  __syncthreads();
  const T *f = reinterpret_cast<const T *>(d.F) + d.foff[s] + k0 * ld + k0;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    for (int j = K - 1; j >= 0; --j) {
      double acc = 0;
      for (int i = j + 1 + lane; i < K; i += 32) acc += double(f[j * ld + i]) * x[i];
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
size_t gemm_smem() {
  return (size_t)kGemmStages * 2 * kGemmKC * kGemmLd * sizeof(T);
}

template <typename T>
void set_sn_attrs() {
  static bool done = false;
  if (done) return;
  cudaFuncSetAttribute(k_sn_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)diag_smem<T>());
  cudaFuncSetAttribute(k_sn_small<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)((kSnSmallMax * kSnSmallMax + kSnSmallMax) * sizeof(T)));
  if (sizeof(T) == 8) {
    cudaFuncSetAttribute(k_sn_gemm_f64<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)gemm_smem<double>());
    cudaFuncSetAttribute(k_sn_gemm_f64<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)gemm_smem<double>());
  }
  done = true;
}

template <typename T>
void run_factor(SnExec &ex, const KKTDev &k, const LDLParams &p, const int *run, int *ok,
                cudaStream_t st) {
  set_sn_attrs<T>();
  const SnDev &d = ex.d;
  for (const SnLaunch &L : ex.fact) {
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
        if (sizeof(T) == 8)
          k_sn_gemm_f64<0><<<L.count, 256, gemm_smem<double>(), st>>>(d, L.begin, run);
        else
          k_sn_gemm_f32<0><<<L.count, 256, gemm_smem<float>(), st>>>(d, L.begin, run);
        break;
      case SN_UPDATE:
        if (sizeof(T) == 8)
          k_sn_gemm_f64<1><<<L.count, 256, gemm_smem<double>(), st>>>(d, L.begin, run);
        else
          k_sn_gemm_f32<1><<<L.count, 256, gemm_smem<float>(), st>>>(d, L.begin, run);
        break;
      default:
        break;
    }
    ex.launches++;
  }
}

// one pass y <- K^-1 y for the instances with srun set
template <typename T>
void run_solve_pass(SnExec &ex, cudaStream_t st) {
  const SnDev &d = ex.d;
  for (const SnLaunch &L : ex.fwd) {
    switch (L.kind) {
      case SN_FWD_SMALL: k_sn_fwd_small<T><<<(L.count + 7) / 8, 256, 0, st>>>(d, L.begin, L.count); break;
      case SN_FWD_GATHER: k_sn_fwd_gather<<<L.count, kVecThreads, 0, st>>>(d, L.begin); break;
      case SN_FWD_DIAG: k_sn_fwd_diag<T><<<L.count, kVecThreads, 0, st>>>(d, L.begin); break;
      case SN_FWD_GEMV: k_sn_fwd_gemv<T><<<L.count, kVecThreads, 0, st>>>(d, L.begin); break;
      case SN_FWD_SCATTER: k_sn_fwd_scatter<<<L.count, kVecThreads, 0, st>>>(d, L.begin); break;
      default: break;
    }
    ex.launches++;
  }
  k_sn_dscale<<<nb256(d.vcount), 256, 0, st>>>(d);
  for (const SnLaunch &L : ex.bwd) {
    switch (L.kind) {
      case SN_BWD_SMALL: k_sn_bwd_small<T><<<(L.count + 7) / 8, 256, 0, st>>>(d, L.begin, L.count); break;
      case SN_BWD_GATHER: k_sn_bwd_gather<<<L.count, kVecThreads, 0, st>>>(d, L.begin); break;
      case SN_BWD_PARTIAL: k_sn_bwd_partial<T><<<L.count, kVecThreads, 0, st>>>(d, L.begin); break;
      case SN_BWD_DIAG: k_sn_bwd_diag<T><<<L.count, kVecThreads, 0, st>>>(d, L.begin); break;
      case SN_BWD_SCATTER: k_sn_bwd_scatter<<<L.count, kVecThreads, 0, st>>>(d, L.begin); break;
      default: break;
    }
    ex.launches++;
  }
  ex.launches++;
}

}  // namespace

SnExec::~SnExec() {
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
