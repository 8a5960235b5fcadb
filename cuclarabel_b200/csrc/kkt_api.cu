// kkt_api.cu -- KKT- and variable-level C ABI for callers that keep their
// own IPM loop (the reference's solve! in Julia) and call this library for
// the linear algebra underneath it:
//
//   clgpu_ldl_*        the AbstractDirectLDLSolver protocol with the
//                      regularise-and-refactor and refined-solve steps of
//                      GPULDLKKTSolver (kktsolver_directldl_gpu.jl:216-260,
//                      :300-413; directldl_cudss.jl:30-59): analysis at
//                      create, static regularisation + numeric factorisation
//                      at refactor, solve with FP64 iterative refinement
//                      against the unshifted matrix.  The factorisation is
//                      the supernodal LDL^T of supernodal.cu for every size.
//   clgpu_residuals    residuals_update! (src/residuals.jl:39-75), GPU form
//   clgpu_add_step     variables_add_step! (src/variables.jl:146-158)
//
// Every pointer argument of the numeric calls is device memory; the
// residual dot products and the step scalars stay on the device, so a loop
// of these calls needs no host synchronisation (clgpu_ldl_refactor and
// clgpu_ldl_solve report their status, so they synchronise).
#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "../../include/clgpu.h"
#include "devbuf.hpp"
#include "ldl.cuh"
#include "setup.hpp"
#include "sn_exec.cuh"

using namespace clgpu;

struct clgpu_ldl {
  int N = 0;
  DevArena arena;
  KKTDev kk{};
  LDLParams lp{};
  std::unique_ptr<SnExec> sn;
  const int *d_src = nullptr;  // permuted CSR position -> caller's CSR position
  int *d_run = nullptr, *d_ok = nullptr;
  double *d_eps = nullptr;
  int nnz = 0;
  bool factored = false;
};

namespace {

__global__ void k_gather_vals(const double *src_vals, const int *src, int n, double *kx) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) kx[p] = src_vals[src[p]];
}

int cuda_status(cudaError_t e) { return e == cudaSuccess ? 0 : -1000 - (int)e; }

}  // namespace

extern "C" int clgpu_ldl_create(int N, const int *Kp, const int *Kj, const signed char *Dsigns,
                                const clgpu_settings *settings, clgpu_ldl **out) {
  if (!out || N <= 0 || !Kp || !Kj || !Dsigns) return -1;
  clgpu_settings st;
  clgpu_default_settings(&st);
  if (settings) st = *settings;
  const int nnz = Kp[N];
  if (nnz <= 0) return -1;
  for (int r = 0; r < N; ++r)
    if (Kp[r + 1] < Kp[r]) return -1;
  for (int q = 0; q < nnz; ++q)
    if (Kj[q] < 0 || Kj[q] >= N) return -1;
  for (int r = 0; r < N; ++r)
    if (Dsigns[r] != 1 && Dsigns[r] != -1) return -1;
  // symmetric pattern (off-diagonal graph) and the diagonal of every row
  std::vector<int> xadj(N + 1, 0), adj;
  adj.reserve(nnz);
  std::vector<char> hasdiag(N, 0);
  for (int r = 0; r < N; ++r) {
    for (int q = Kp[r]; q < Kp[r + 1]; ++q) {
      if (Kj[q] == r) hasdiag[r] = 1;
      else adj.push_back(Kj[q]);
    }
    xadj[r + 1] = (int)adj.size();
  }
  for (int r = 0; r < N; ++r)
    if (!hasdiag[r]) return -2;  // every row needs its diagonal entry (the regularisation target)
  auto h = std::unique_ptr<clgpu_ldl>(new clgpu_ldl());
  h->N = N;
  h->nnz = nnz;
  std::vector<int> perm;
  SnSymbolic sym;
  std::string err;
  if (!sn_analyse(N, xadj, adj, perm, sym, &err)) return -3;
  std::vector<int> ip(N);
  for (int k = 0; k < N; ++k) ip[perm[k]] = k;
  // permuted CSR, columns sorted, each value's position in the caller's CSR
  std::vector<int> P(N + 1, 0), J(nnz), src(nnz), Kd(N, -1), gsrc(N);
  std::vector<signed char> ds(N);
  {
    std::vector<std::vector<std::pair<int, int>>> rows(N);
    for (int r = 0; r < N; ++r)
      for (int q = Kp[r]; q < Kp[r + 1]; ++q) rows[ip[r]].push_back({ip[Kj[q]], q});
    int w = 0;
    for (int k = 0; k < N; ++k) {
      auto &R = rows[k];
      std::sort(R.begin(), R.end());
      for (size_t a = 0; a < R.size(); ++a) {
        if (a > 0 && R[a].first == R[a - 1].first) return -4;  // repeated entry
        J[w] = R[a].first;
        src[w] = R[a].second;
        if (R[a].first == k) Kd[k] = w;
        ++w;
      }
      P[k + 1] = w;
      ds[k] = Dsigns[perm[k]];
      gsrc[k] = perm[k];
    }
  }
  std::vector<SnInstance> in{{&sym, P.data(), J.data(), 0, 0, 0}};
  SnPlan plan;
  if (!sn_build_plan(in, plan, &err)) return -3;
  DevArena &A = h->arena;
  KKTDev &k = h->kk;
  std::vector<int> voff{0, N}, poff{0}, Nv{N};
  k.B = 1;
  k.N = A.upload(Nv);
  k.voff = A.upload(voff);
  k.poff = A.upload(poff);
  k.Kp = A.upload(P);
  k.Kj = A.upload(J);
  k.Kx = A.alloc<double>(nnz);
  k.Kdiag = A.upload(Kd);
  k.Dsign = A.upload(ds);
  k.gsrc = A.upload(gsrc);
  h->d_src = A.upload(src);
  std::vector<int> one{1};
  h->d_run = A.upload(one);
  h->d_ok = A.alloc<int>(1);
  h->d_eps = A.alloc<double>(1);
  std::vector<int> vinst(N, 0);
  h->sn.reset(new SnExec());
  const bool mixed = st.direct_solve_method == CLGPU_METHOD_MIXED ||
                     st.direct_solve_method == CLGPU_METHOD_MIXED_F64ELIM;
  if (!sn_exec_create(plan, mixed, 1, 0, N, vinst, A, *h->sn)) return cuda_status(A.err ? A.err : cudaErrorMemoryAllocation);
  k.sn = h->sn.get();
  if (A.err != cudaSuccess) return cuda_status(A.err);
  // the arena's zero fills run on the legacy stream: finished before any
  // stream of the caller's uses the handle
  if (cudaError_t se = cudaStreamSynchronize(0)) return cuda_status(se);
  A.settle();
  LDLParams &lp = h->lp;
  lp.static_reg = st.static_regularization_enable;
  lp.static_c = st.static_regularization_constant;
  lp.static_prop = st.static_regularization_proportional;
  lp.dyn_reg = st.dynamic_regularization_enable;
  lp.dyn_eps = st.dynamic_regularization_eps;
  lp.dyn_delta = st.dynamic_regularization_delta;
  lp.ir_enable = st.iterative_refinement_enable;
  lp.ir_maxiter = st.iterative_refinement_max_iter;
  lp.ir_reltol = st.iterative_refinement_reltol;
  lp.ir_abstol = st.iterative_refinement_abstol;
  lp.ir_stopratio = st.iterative_refinement_stop_ratio;
  *out = h.release();
  return 0;
}

extern "C" int clgpu_ldl_destroy(clgpu_ldl *h) {
  if (!h) return -1;
  delete h;
  return 0;
}

extern "C" int clgpu_ldl_refactor(clgpu_ldl *h, const double *Kx, double *eps,
                                  clgpu_stream_t stream) {
  if (!h || !Kx) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  k_gather_vals<<<(h->nnz + 255) / 256, 256, 0, st>>>(Kx, h->d_src, h->nnz, h->kk.Kx);
  const int one = 1;
  cudaMemcpyAsync(h->d_ok, &one, sizeof(int), cudaMemcpyHostToDevice, st);
  sn_factor(*h->sn, h->kk, h->lp, h->d_run, h->d_ok, h->d_eps, st);
  int ok = 0;
  double e = 0;
  cudaMemcpyAsync(&ok, h->d_ok, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&e, h->d_eps, sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaError_t err = cudaStreamSynchronize(st);
  if (err == cudaSuccess) err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_status(err);
  if (eps) *eps = e;
  h->factored = ok != 0;
  return ok ? 0 : 1;
}

extern "C" int clgpu_ldl_solve(clgpu_ldl *h, const double *b, double *x, clgpu_stream_t stream) {
  if (!h || !b || !x) return -1;
  if (!h->factored) return -2;
  cudaStream_t st = (cudaStream_t)stream;
  const int one = 1;
  cudaMemcpyAsync(h->d_ok, &one, sizeof(int), cudaMemcpyHostToDevice, st);
  sn_solve(*h->sn, h->kk, h->lp, h->d_run, b, nullptr, x, nullptr, h->d_ok, st);
  int ok = 0;
  cudaMemcpyAsync(&ok, h->d_ok, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaError_t err = cudaStreamSynchronize(st);
  if (err == cudaSuccess) err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_status(err);
  return ok ? 0 : 1;
}

// ------------------------------------------------------------- residuals
namespace {

constexpr int kResBlocks = 512;  // fixed grid: partial sums in a fixed order
constexpr int kResThreads = 256;

__device__ double csr_row(const int *p, const int *j, const double *v, const double *x, int r) {
  double t = 0;
  for (int q = p[r]; q < p[r + 1]; ++q) t += v[q] * x[j[q]];
  return t;
}

// Px, rx_inf = -A' z, rz_inf = A x + s, and per-block partial dot products
// {q.x, b.z, s.z, x.Px} into part[4 * kResBlocks]
__global__ void __launch_bounds__(kResThreads) k_res_main(
    int n, int m, const int *Pp, const int *Pj, const double *Pv, const int *Ap, const int *Aj,
    const double *Av, const int *Atp, const int *Atj, const double *Atv, const double *q,
    const double *b, const double *x, const double *s, const double *z, double *Pxo,
    double *rx_inf, double *rz_inf, double *part) {
  double a[4] = {0, 0, 0, 0};
  const int stride = gridDim.x * kResThreads;
  for (int i = blockIdx.x * kResThreads + threadIdx.x; i < n; i += stride) {
    const double px = csr_row(Pp, Pj, Pv, x, i);
    Pxo[i] = px;
    rx_inf[i] = -csr_row(Atp, Atj, Atv, z, i);
    a[0] += q[i] * x[i];
    a[3] += x[i] * px;
  }
  for (int i = blockIdx.x * kResThreads + threadIdx.x; i < m; i += stride) {
    rz_inf[i] = csr_row(Ap, Aj, Av, x, i) + s[i];
    a[1] += b[i] * z[i];
    a[2] += s[i] * z[i];
  }
  __shared__ double red[4][kResThreads / 32];
  for (int k = 0; k < 4; ++k) {
    double v = a[k];
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0;
    for (int w = 0; w < kResThreads / 32; ++w) v += red[threadIdx.x][w];
    part[threadIdx.x * kResBlocks + blockIdx.x] = v;
  }
}

// rx, rz and the dots {qx, bz, sz, xPx, r_tau} (one block, fixed order)
__global__ void __launch_bounds__(kResThreads) k_res_finish(
    int n, int m, const double *q, const double *b, const double *tau, const double *kappa,
    const double *Pxo, const double *rx_inf, const double *rz_inf, double *rx, double *rz,
    const double *part, double *dots) {
  const double t = *tau;
  for (int i = blockIdx.x * kResThreads + threadIdx.x; i < n; i += gridDim.x * kResThreads)
    rx[i] = rx_inf[i] - Pxo[i] - q[i] * t;
  for (int i = blockIdx.x * kResThreads + threadIdx.x; i < m; i += gridDim.x * kResThreads)
    rz[i] = rz_inf[i] - b[i] * t;
  if (blockIdx.x != 0) return;
  __shared__ double red[4];
  if (threadIdx.x < 4) {
    double v = 0;
    for (int k = 0; k < kResBlocks; ++k) v += part[threadIdx.x * kResBlocks + k];
    red[threadIdx.x] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    dots[0] = red[0];
    dots[1] = red[1];
    dots[2] = red[2];
    dots[3] = red[3];
    dots[4] = red[0] + red[1] + *kappa + red[3] / t;
  }
}

__global__ void k_add_step_vec(int n, double *v, const double *dv, const double *alpha) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] += *alpha * dv[i];
}
__global__ void k_add_step_scal(double *tau, double *kappa, const double *dtau,
                                const double *dkappa, const double *alpha) {
  *tau += *alpha * *dtau;
  *kappa += *alpha * *dkappa;
}

}  // namespace

extern "C" int clgpu_residuals(int n, int m, const int *Pp, const int *Pj, const double *Px,
                               const int *Ap, const int *Aj, const double *Ax, const int *Atp,
                               const int *Atj, const double *Atx, const double *q,
                               const double *b, const double *x, const double *s,
                               const double *z, const double *tau, const double *kappa,
                               double *rx, double *rz, double *rx_inf, double *rz_inf,
                               double *Pxo, double *dots, double *work, clgpu_stream_t stream) {
  if (n < 0 || m < 0 || !tau || !kappa || !dots || !work) return -1;
  if (n > 0 && (!Pp || !Pj || !Atp || !Atj || !q || !x || !rx || !rx_inf || !Pxo)) return -1;
  if (m > 0 && (!Ap || !Aj || !b || !s || !z || !rz || !rz_inf)) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  k_res_main<<<kResBlocks, kResThreads, 0, st>>>(n, m, Pp, Pj, Px, Ap, Aj, Ax, Atp, Atj, Atx, q,
                                                 b, x, s, z, Pxo, rx_inf, rz_inf, work);
  const int nb = std::max(1, std::min(kResBlocks, (std::max(n, m) + kResThreads - 1) / kResThreads));
  k_res_finish<<<nb, kResThreads, 0, st>>>(n, m, q, b, tau, kappa, Pxo, rx_inf, rz_inf, rx, rz,
                                           work, dots);
  return cuda_status(cudaGetLastError());
}

extern "C" int clgpu_residuals_work_len(void) { return 4 * kResBlocks; }

extern "C" int clgpu_add_step(int n, int m, double *x, double *s, double *z, double *tau,
                              double *kappa, const double *dx, const double *ds,
                              const double *dz, const double *dtau, const double *dkappa,
                              const double *alpha, clgpu_stream_t stream) {
  if (n < 0 || m < 0 || !tau || !kappa || !dtau || !dkappa || !alpha) return -1;
  if ((n > 0 && (!x || !dx)) || (m > 0 && (!s || !z || !ds || !dz))) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  if (n > 0) k_add_step_vec<<<(n + 255) / 256, 256, 0, st>>>(n, x, dx, alpha);
  if (m > 0) {
    k_add_step_vec<<<(m + 255) / 256, 256, 0, st>>>(m, s, ds, alpha);
    k_add_step_vec<<<(m + 255) / 256, 256, 0, st>>>(m, z, dz, alpha);
  }
  k_add_step_scal<<<1, 1, 0, st>>>(tau, kappa, dtau, dkappa, alpha);
  return cuda_status(cudaGetLastError());
}
