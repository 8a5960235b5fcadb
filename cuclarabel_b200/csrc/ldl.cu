// ldl.cu -- batched sparse LDL^T numeric factorisation and solves (sm_100a).
//
// One thread block per instance.  Instances whose KKT dimension fits keep
// their dense work vector in shared memory and run on a single warp (NT=32:
// __syncwarp between dependent steps, no block barriers); larger instances
// run on 256 threads with the work vector in global scratch.
//
// Factorisation: left-looking by columns on the permuted matrix.  For column
// j the lower part of K(:,j) (row j of the symmetric permuted CSR, entries
// with col >= j) is scattered into w, every earlier column k with L(j,k) != 0
// is applied as w(j:) -= L(j:,k) * (L(j,k) D(k)) (the (k, pos) list of row j
// is precomputed by the symbolic phase), then D(j) = w(j) and
// L(j+1:,j) = w / D(j).  Static regularisation (kktsolver_directldl_gpu.jl:
// 216-260: eps = c + prop*||diag||_inf, diag +/- eps by the expected sign)
// is applied inside the scatter so the stored KKT keeps its true diagonal
// for the refinement residual; dynamic regularisation follows the CPU path
// (sign*D(j) <= eps_dyn -> D(j) = sign*delta).
//
// Solve: forward (column-oriented scatter), diagonal, backward (column dot
// products with a warp reduction), then iterative refinement against the
// unregularised KKT exactly as kktsolver_directldl_gpu.jl:349-409.  In the
// mixed-precision form L, D and the triangular solves are FP32 while the
// refinement residual, the right-hand side and the iterate stay FP64.
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
__device__ __forceinline__ int inst_class(int N, int tsize) {
  return (long long)N * tsize <= kSmemLimitBytes ? 1 : 2;
}

template <typename T, int NT, bool SMEM>
__global__ void __launch_bounds__(NT) k_ldl_factor(KKTDev k, LDLParams prm, const int *run,
                                                   int *ok, double *eps_out) {
  int inst = blockIdx.x;
  if (!run[inst]) return;
  int N = k.N[inst];
  if (inst_class(N, sizeof(T)) != (SMEM ? 1 : 2)) return;
  __shared__ double red[NT / 32 + 1];
  extern __shared__ __align__(16) unsigned char sm_raw[];
  int vo = k.voff[inst], po = k.poff[inst];
  T *w = SMEM ? reinterpret_cast<T *>(sm_raw) : reinterpret_cast<T *>(k.w) + vo;
  T *Lx = reinterpret_cast<T *>(k.Lx);
  T *D = reinterpret_cast<T *>(k.D) + vo;
  T *Dinv = reinterpret_cast<T *>(k.Dinv) + vo;
  const int *Kp = k.Kp + po, *Lp = k.Lp + po, *Rp = k.Rp + po;
  const int *Kdiag = k.Kdiag + vo;
  const signed char *sg = k.Dsign + vo;
  int tid = threadIdx.x, lane = tid & 31;
  if (SMEM)
    for (int i = tid; i < N; i += NT) w[i] = T(0);
  // static regulariser from the true diagonal
  double eps = 0;
  if (prm.static_reg) {
    double mx = 0;
    for (int i = tid; i < N; i += NT) mx = fmax(mx, fabs(k.Kx[Kdiag[i]]));
    mx = block_max<NT>(mx, red);
    eps = prm.static_c + prm.static_prop * mx;
  }
  bar_sync<NT>();
  bool finite = true;
  for (int j = 0; j < N; ++j) {
    // scatter the lower part of column j (row j, cols >= j)
    for (int p = Kp[j] + tid; p < Kp[j + 1]; p += NT) {
      int c = k.Kj[p];
      if (c > j)
        w[c] = T(k.Kx[p]);
      else if (c == j)
        w[c] = T(k.Kx[p] + (sg[j] > 0 ? eps : -eps));
    }
    bar_sync<NT>();
    // left-looking updates from the columns in row j of L
    int q0 = Rp[j], q1 = Rp[j + 1];
    for (int qb = q0; qb < q1; qb += 32) {
      int myk = 0, mypos = 0, myend = 0;
      T myf = T(0);
      if (qb + lane < q1) {
        myk = k.Rk[qb + lane];
        mypos = k.Rpos[qb + lane];
        myend = Lp[myk + 1];
        myf = Lx[mypos] * D[myk];
      }
      int cnt = min(32, q1 - qb);
      for (int t = 0; t < cnt; ++t) {
        int pos = __shfl_sync(0xffffffffu, mypos, t);
        int end = __shfl_sync(0xffffffffu, myend, t);
        T f = __shfl_sync(0xffffffffu, myf, t);
        for (int p = pos + tid; p < end; p += NT) w[k.Li[p]] -= Lx[p] * f;
        bar_sync<NT>();
      }
    }
    T dj = w[j];
    if (prm.dyn_reg) {
      T sgn = T(sg[j]);
      if (sgn * dj <= T(prm.dyn_eps)) dj = T(prm.dyn_delta) * sgn;
    }
    T dinv = T(1) / dj;
    if (!isfinite((double)dinv)) finite = false;
    for (int p = Lp[j] + tid; p < Lp[j + 1]; p += NT) {
      int i = k.Li[p];
      Lx[p] = w[i] * dinv;
      w[i] = T(0);
    }
    if (tid == 0) {
      D[j] = dj;
      Dinv[j] = dinv;
      w[j] = T(0);
    }
    bar_sync<NT>();
  }
  if (tid == 0) {
    if (!finite) ok[inst] = 0;
    if (eps_out) eps_out[inst] = eps;
  }
}

// y <- L^{-T} D^{-1} L^{-1} y  (y in factor precision)
template <typename T, int NT>
__device__ void ldl_trisolve(const KKTDev &k, int N, int vo, int po, T *y, double *red) {
  const T *Lx = reinterpret_cast<const T *>(k.Lx);
  const T *Dinv = reinterpret_cast<const T *>(k.Dinv) + vo;
  const int *Lp = k.Lp + po;
  int tid = threadIdx.x;
  for (int j = 0; j < N; ++j) {
    T yj = y[j];
    for (int p = Lp[j] + tid; p < Lp[j + 1]; p += NT) y[k.Li[p]] -= Lx[p] * yj;
    bar_sync<NT>();
  }
  for (int i = tid; i < N; i += NT) y[i] *= Dinv[i];
  bar_sync<NT>();
  for (int j = N - 1; j >= 0; --j) {
    double t = 0;
    for (int p = Lp[j] + tid; p < Lp[j + 1]; p += NT) t += double(Lx[p] * y[k.Li[p]]);
    t = block_sum<NT>(t, red);
    if (tid == 0) y[j] -= T(t);
    bar_sync<NT>();
  }
}

// e = b - K xi ; returns ||e||_inf (NaN/Inf propagate)
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
  if (inst_class(N, sizeof(T)) != (SMEM ? 1 : 2)) return;
  __shared__ double red[NT / 32 + 1];
  extern __shared__ __align__(16) unsigned char sm_raw[];
  int vo = k.voff[inst], po = k.poff[inst];
  int tid = threadIdx.x;
  T *y = SMEM ? reinterpret_cast<T *>(sm_raw) : reinterpret_cast<T *>(k.yf) + vo;
  double *b = k.b + vo, *x = k.x + vo, *e = k.e + vo, *dx = k.dx + vo;
  const int *gs = k.gsrc + vo;
  // gather the right-hand side in permuted order
  double nb = 0;
  for (int i = tid; i < N; i += NT) {
    int g = gs[i];
    double v = g >= 0 ? rx[g] : (g == -1 ? 0.0 : rz[-g - 2]);
    b[i] = v;
    y[i] = T(v);
    nb = fmax(nb, fabs(v));
  }
  double normb = block_max<NT>(nb, red);
  bar_sync<NT>();
  ldl_trisolve<T, NT>(k, N, vo, po, y, red);
  for (int i = tid; i < N; i += NT) x[i] = double(y[i]);
  bar_sync<NT>();
  bool good = true;
  if (prm.ir_enable) {
    double norme = refine_error<NT>(k, N, po, b, x, e, red);
    if (!isfinite(norme)) good = false;
    for (int it = 0; good && it < prm.ir_maxiter; ++it) {
      if (norme <= prm.ir_abstol + prm.ir_reltol * normb) break;
      double last = norme;
      for (int i = tid; i < N; i += NT) y[i] = T(e[i]);
      bar_sync<NT>();
      ldl_trisolve<T, NT>(k, N, vo, po, y, red);
      for (int i = tid; i < N; i += NT) dx[i] = double(y[i]) + x[i];
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
  size_t sm = ((size_t)k.max_small_N * sizeof(T) + 15) & ~(size_t)15;
  if (k.has_small)
    k_ldl_factor<T, kSmallNT, true><<<k.B, kSmallNT, sm, st>>>(k, p, run, ok, eps_out);
  if (k.has_large)
    k_ldl_factor<T, kLargeNT, false><<<k.B, kLargeNT, 0, st>>>(k, p, run, ok, eps_out);
}
template <typename T>
static void launch_solve(const KKTDev &k, const LDLParams &p, const int *run,
                         const double *rx, const double *rz, double *lx, double *lz, int *ok,
                         cudaStream_t st) {
  size_t sm = ((size_t)k.max_small_N * sizeof(T) + 15) & ~(size_t)15;
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
