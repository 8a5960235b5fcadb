// cones_api.cu -- cone-level C ABI (the CompositeConeGPU method table of
// src/gpucones/coneops_compositecone_gpu.jl), one problem, device pointers
// borrowed from the caller in the reference's sorted cone order.
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/clgpu.h"
#include "cones.cuh"
#include "devbuf.hpp"

using namespace clgpu;

struct clgpu_cones {
  DevArena arena;
  ConeSet cs{};
  int numel = 0, degree = 0, hs_len = 0;
  bool symmetric = true;
  int *d_nn_blk = nullptr, *d_soc_blk = nullptr, *d_exp_blk = nullptr, *d_pow_blk = nullptr,
      *d_psd_blk = nullptr;
  double *d_scal = nullptr;  // small scalar workspace [8]
  int *d_iscal = nullptr;    // [4]
  double *d_save = nullptr;  // [soc_rows] rows kept by mul_Hs_diag
  double *d_hs = nullptr;    // [hs_len] Hs blocks for refresh_kkt
  int n_sparse = 0, sparse_rows = 0;
  // kernel-time profiling: events around an operation's launches only
  bool prof = false;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  double last_ms = 0.0;
  ~clgpu_cones() {
    for (auto &e : ev)
      if (e) cudaEventDestroy(e);
  }
};

// Marks the start (k even) or end (k odd) of an operation's launch group
// when profiling is on; step_length has two groups (k = 0..3).
static void prof_mark(clgpu_cones *h, int k, cudaStream_t st) {
  if (h->prof) cudaEventRecord(h->ev[k], st);
}
// After the stream has been synchronised: the operation's kernel time.
static void prof_collect(clgpu_cones *h, int groups) {
  if (!h->prof) return;
  double ms = 0.0;
  for (int p = 0; p < groups; ++p) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, h->ev[2 * p], h->ev[2 * p + 1]) == cudaSuccess) ms += t;
  }
  h->last_ms = ms;
}

extern "C" int clgpu_cones_create(int ncones, const int *types, const int *dims,
                                  const double *params, int soc_threshold,
                                  clgpu_cones **out) {
  if (!out || ncones < 0 || (ncones > 0 && (!types || !dims))) return -1;
  for (int c = 1; c < ncones; ++c)
    if (types[c] < types[c - 1]) return -2;  // compositecone_type_gpu.jl:75-79
  auto *h = new clgpu_cones();
  ConeSet &cs = h->cs;
  DevArena &A = h->arena;
  std::vector<int> row_inst, soc_off, soc_dim, soc_inst, soc_sparse, exp_inst, pow_inst,
      psd_off, psd_n, psd_inst, nn_blk, soc_blk, exp_blk, pow_blk, psd_blk;
  std::vector<double> pow_alpha;
  int row = 0, blk = 0, soc_max = 0, psd_max = 1;
  int tbeg[6] = {-1, -1, -1, -1, -1, -1}, trows[6] = {0, 0, 0, 0, 0, 0};
  for (int c = 0; c < ncones; ++c) {
    int t = types[c], d = dims[c];
    if (t < 0 || t > 5 || d < 0) {
      delete h;
      return -1;
    }
    int nv = (t == 3 || t == 4) ? 3 : (t == 5 ? d * (d + 1) / 2 : d);
    if (tbeg[t] < 0) tbeg[t] = row;
    trows[t] += nv;
    bool sparse = (t == 2 && d > soc_threshold);
    bool diag = (t == 0 || t == 1 || sparse);
    int bl = diag ? nv : nv * (nv + 1) / 2;
    switch (t) {
      case 0: h->degree += 0; break;
      case 1:
        for (int k = 0; k < nv; ++k) nn_blk.push_back(blk + k);
        h->degree += d;
        break;
      case 2:
        soc_off.push_back(row);
        soc_dim.push_back(d);
        soc_inst.push_back(0);
        soc_sparse.push_back(sparse ? 1 : 0);
        soc_blk.push_back(blk);
        soc_max = std::max(soc_max, d);
        h->degree += 1;
        break;
      case 3:
        exp_inst.push_back(0);
        exp_blk.push_back(blk);
        h->degree += 3;
        h->symmetric = false;
        break;
      case 4:
        pow_inst.push_back(0);
        pow_alpha.push_back(params ? params[c] : 0.5);
        pow_blk.push_back(blk);
        h->degree += 3;
        h->symmetric = false;
        break;
      case 5:
        if (d > kPsdMaxSide) {
          delete h;
          return -3;
        }
        psd_off.push_back(row);
        psd_n.push_back(d);
        psd_inst.push_back(0);
        psd_blk.push_back(blk);
        psd_max = std::max(psd_max, d);
        h->degree += d;
        break;
    }
    row += nv;
    blk += bl;
  }
  for (int r = 0; r < row; ++r) row_inst.push_back(0);
  h->numel = row;
  h->hs_len = blk;
  cs.B = 1;
  cs.m_total = row;
  cs.zero_begin = tbeg[0] < 0 ? 0 : tbeg[0];
  cs.n_zero = trows[0];
  cs.nn_begin = tbeg[1] < 0 ? 0 : tbeg[1];
  cs.n_nn = trows[1];
  cs.soc_begin = tbeg[2] < 0 ? 0 : tbeg[2];
  cs.soc_rows = trows[2];
  cs.exp_begin = tbeg[3] < 0 ? 0 : tbeg[3];
  cs.pow_begin = tbeg[4] < 0 ? 0 : tbeg[4];
  cs.psd_begin = tbeg[5] < 0 ? 0 : tbeg[5];
  cs.n_soc = (int)soc_off.size();
  cs.n_exp = (int)exp_inst.size();
  cs.n_pow = (int)pow_inst.size();
  cs.n_psd = (int)psd_off.size();
  int G = 2;
  while (G < soc_max && G < 32) G <<= 1;
  cs.soc_group = G;
  cs.psd_nmax = psd_max;
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
  size_t nn2 = (size_t)psd_max * psd_max;
  cs.psd_R = A.alloc<double>(nn2 * cs.n_psd);
  cs.psd_Rinv = A.alloc<double>(nn2 * cs.n_psd);
  cs.psd_lam = A.alloc<double>((size_t)psd_max * cs.n_psd);
  cs.cone_tmp = A.alloc<double>((size_t)cs.n_soc + cs.n_exp + cs.n_pow + cs.n_psd);
  cs.cone_tmp2 = A.alloc<double>((size_t)cs.n_soc + cs.n_exp + cs.n_pow + cs.n_psd);
  {
    std::vector<int> rnn = {0, cs.n_nn}, rsoc = {0, cs.n_soc}, rexp = {0, cs.n_exp},
                     rpow = {0, cs.n_pow}, rpsd = {0, cs.n_psd};
    cs.rng_nn = A.upload(rnn);
    cs.rng_soc = A.upload(rsoc);
    cs.rng_exp = A.upload(rexp);
    cs.rng_pow = A.upload(rpow);
    cs.rng_psd = A.upload(rpsd);
  }
  cs.inst_active = nullptr;
  h->d_nn_blk = A.upload(nn_blk);
  h->d_soc_blk = A.upload(soc_blk);
  h->d_exp_blk = A.upload(exp_blk);
  h->d_pow_blk = A.upload(pow_blk);
  h->d_psd_blk = A.upload(psd_blk);
  h->d_scal = A.alloc<double>(8);
  h->d_iscal = A.alloc<int>(4);
  h->d_save = A.alloc<double>(cs.soc_rows);
  h->d_hs = A.alloc<double>(blk);
  for (size_t c = 0; c < soc_sparse.size(); ++c)
    if (soc_sparse[c]) {
      h->n_sparse++;
      h->sparse_rows += soc_dim[c];
    }
  int one = 1;
  cudaMemcpy(h->d_iscal + 2, &one, sizeof(int), cudaMemcpyHostToDevice);  // bt active
  if (A.err != cudaSuccess) {
    int e = -1000 - (int)A.err;
    delete h;
    return e;
  }
  int rc = cones_autotune(cs, 0);  // launch shapes timed on this cone set
  if (rc != 0) {
    delete h;
    return rc;
  }
  // the arena's zero fills run on the legacy stream: finished before any
  // stream of the caller's can read the handle's state
  cudaError_t se = cudaStreamSynchronize(0);
  if (se != cudaSuccess) {
    delete h;
    return -1000 - (int)se;
  }
  A.settle();
  *out = h;
  return 0;
}

extern "C" int clgpu_cones_destroy(clgpu_cones *h) {
  if (!h) return -1;
  delete h;
  return 0;
}
extern "C" int clgpu_cones_numel(const clgpu_cones *h) { return h ? h->numel : -1; }
extern "C" int clgpu_cones_degree(const clgpu_cones *h) { return h ? h->degree : -1; }
extern "C" int clgpu_cones_hs_len(const clgpu_cones *h) { return h ? h->hs_len : -1; }

extern "C" int clgpu_cones_get_launch_shapes(const clgpu_cones *h, int *nn_block,
                                             int *soc_variants) {
  if (!h) return -1;
  if (nn_block) *nn_block = h->cs.nn_block;
  if (soc_variants)
    for (int op = 0; op < kSocOps; ++op) soc_variants[op] = h->cs.soc_variant[op];
  return 0;
}
extern "C" int clgpu_cones_set_launch_shapes(clgpu_cones *h, int nn_block,
                                             const int *soc_variants) {
  if (!h) return -1;
  if (nn_block != 0 && (nn_block < 32 || nn_block > 1024 || nn_block % 32 != 0)) return -1;
  if (soc_variants)
    for (int op = 0; op < kSocOps; ++op)
      if (soc_variants[op] < 0 || soc_variants[op] > kSocTileShapes) return -1;
  if (nn_block) h->cs.nn_block = nn_block;
  if (soc_variants)
    for (int op = 0; op < kSocOps; ++op) h->cs.soc_variant[op] = soc_variants[op];
  return 0;
}
extern "C" int clgpu_cones_set_profiling(clgpu_cones *h, int enable) {
  if (!h) return -1;
  if (enable && !h->ev[0])
    for (auto &e : h->ev)
      if (cudaEventCreate(&e) != cudaSuccess) return -1;
  h->prof = enable != 0;
  h->last_ms = 0.0;
  return 0;
}
extern "C" int clgpu_cones_last_kernel_ms(const clgpu_cones *h, double *ms) {
  if (!h || !ms) return -1;
  *ms = h->last_ms;
  return 0;
}

__global__ void k_fill(double *v, int n, double a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = a;
}

static int finish(cudaStream_t st) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return -1000 - (int)e;
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return -1000 - (int)e;
  return 0;
}
static int finish_prof(clgpu_cones *h, cudaStream_t st) {
  int rc = finish(st);
  if (rc == 0) prof_collect(h, 1);
  return rc;
}

extern "C" int clgpu_update_scaling(clgpu_cones *h, const double *s, const double *z,
                                    double mu, int strategy, clgpu_stream_t stream) {
  if (!h) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  int iv[2] = {strategy, 1};
  cudaMemcpyAsync(h->d_scal, &mu, sizeof(double), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(h->d_iscal, iv, 2 * sizeof(int), cudaMemcpyHostToDevice, st);
  prof_mark(h, 0, st);
  cones_update_scaling(h->cs, s, z, h->d_scal, h->d_iscal, h->d_iscal + 1, st);
  prof_mark(h, 1, st);
  int ok = 0;
  cudaMemcpyAsync(&ok, h->d_iscal + 1, sizeof(int), cudaMemcpyDeviceToHost, st);
  int rc = finish(st);
  if (rc) return rc;
  prof_collect(h, 1);
  return ok ? 0 : 1;
}
extern "C" int clgpu_set_identity_scaling(clgpu_cones *h, clgpu_stream_t stream) {
  if (!h) return -1;
  cones_set_identity_scaling(h->cs, (cudaStream_t)stream);
  return finish((cudaStream_t)stream);
}
extern "C" int clgpu_get_Hs(clgpu_cones *h, double *Hs, clgpu_stream_t stream) {
  if (!h) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(Hs, 0, (size_t)std::max(h->hs_len, 1) * sizeof(double), st);
  prof_mark(h, 0, st);
  cones_get_Hs(h->cs, h->d_nn_blk, h->d_soc_blk, h->d_exp_blk, h->d_pow_blk, h->d_psd_blk, Hs,
               st);
  prof_mark(h, 1, st);
  return finish_prof(h, st);
}
extern "C" int clgpu_mul_Hs(clgpu_cones *h, double *y, const double *x, clgpu_stream_t stream) {
  if (!h) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  prof_mark(h, 0, st);
  cones_mul_Hs(h->cs, y, x, st);
  prof_mark(h, 1, st);
  return finish_prof(h, st);
}
extern "C" int clgpu_affine_ds(clgpu_cones *h, double *ds, const double *s,
                               clgpu_stream_t stream) {
  if (!h) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  prof_mark(h, 0, st);
  cones_affine_ds(h->cs, ds, s, st);
  prof_mark(h, 1, st);
  return finish_prof(h, st);
}
extern "C" int clgpu_combined_ds_shift(clgpu_cones *h, double *shift, const double *step_z,
                                       const double *step_s, const double *z, double sigma_mu,
                                       clgpu_stream_t stream) {
  if (!h) return -1;
  (void)z;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemcpyAsync(h->d_scal + 1, &sigma_mu, sizeof(double), cudaMemcpyHostToDevice, st);
  prof_mark(h, 0, st);
  cones_combined_ds_shift(h->cs, shift, step_z, step_s, h->d_scal + 1, st);
  prof_mark(h, 1, st);
  return finish_prof(h, st);
}
extern "C" int clgpu_ds_from_dz_offset(clgpu_cones *h, double *out, const double *ds,
                                       const double *z, clgpu_stream_t stream) {
  if (!h) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  prof_mark(h, 0, st);
  cones_ds_from_dz_offset(h->cs, out, ds, z, st);
  prof_mark(h, 1, st);
  return finish_prof(h, st);
}
extern "C" int clgpu_step_length(clgpu_cones *h, const double *dz, const double *ds,
                                 const double *z, const double *s, double alpha_max,
                                 double max_step_fraction, double backtrack_step,
                                 double alpha_min, double *alpha, clgpu_stream_t stream) {
  if (!h || !alpha) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemcpyAsync(h->d_scal + 2, &alpha_max, sizeof(double), cudaMemcpyHostToDevice, st);
  prof_mark(h, 0, st);
  cones_step_length_sym(h->cs, dz, ds, z, s, h->d_scal + 2, st);
  prof_mark(h, 1, st);
  double a = 0;
  cudaMemcpyAsync(&a, h->d_scal + 2, sizeof(double), cudaMemcpyDeviceToHost, st);
  int rc = finish(st);
  if (rc) return rc;
  int groups = 1;
  if (!h->symmetric) {
    a = std::min(a, max_step_fraction);
    cudaMemcpyAsync(h->d_scal + 2, &a, sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(h->d_scal + 3, &a, sizeof(double), cudaMemcpyHostToDevice, st);
    prof_mark(h, 2, st);
    cones_step_length_asym(h->cs, dz, ds, z, s, h->d_scal + 2, h->d_scal + 3, backtrack_step,
                           alpha_min, st);
    prof_mark(h, 3, st);
    cudaMemcpyAsync(&a, h->d_scal + 3, sizeof(double), cudaMemcpyDeviceToHost, st);
    rc = finish(st);
    if (rc) return rc;
    groups = 2;
  }
  prof_collect(h, groups);
  *alpha = a;
  return 0;
}
extern "C" int clgpu_compute_barrier(clgpu_cones *h, const double *z, const double *s,
                                     const double *dz, const double *ds, double alpha,
                                     double *barrier, clgpu_stream_t stream) {
  if (!h || !barrier) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  double init[2] = {alpha, 0.0};
  cudaMemcpyAsync(h->d_scal + 4, init, 2 * sizeof(double), cudaMemcpyHostToDevice, st);
  cones_barrier(h->cs, z, s, dz, ds, h->d_scal + 4, h->d_iscal + 2, h->d_scal + 5, st);
  cudaMemcpyAsync(barrier, h->d_scal + 5, sizeof(double), cudaMemcpyDeviceToHost, st);
  return finish(st);
}
extern "C" int clgpu_margins(clgpu_cones *h, const double *z, int pd, double *alpha,
                             double *beta, clgpu_stream_t stream) {
  if (!h) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  cones_margins(h->cs, z, pd, h->d_scal + 6, h->d_scal + 7, st);
  double out[2];
  cudaMemcpyAsync(out, h->d_scal + 6, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
  int rc = finish(st);
  if (rc) return rc;
  if (alpha) *alpha = out[0];
  if (beta) *beta = out[1];
  return 0;
}
extern "C" int clgpu_scaled_unit_shift(clgpu_cones *h, double *z, double alpha, int pd,
                                       clgpu_stream_t stream) {
  if (!h) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemcpyAsync(h->d_scal, &alpha, sizeof(double), cudaMemcpyHostToDevice, st);
  cones_scaled_unit_shift(h->cs, z, h->d_scal, pd, st);
  return finish(st);
}
extern "C" int clgpu_unit_initialization(clgpu_cones *h, double *z, double *s,
                                         clgpu_stream_t stream) {
  if (!h) return -1;
  cones_unit_initialization(h->cs, z, s, (cudaStream_t)stream);
  return finish((cudaStream_t)stream);
}

// ------------------------------------------------ KKT-level cone operations
// Rows of the sparse (expanded) second-order cones: dir 0 saves y there,
// dir 1 puts the saved values back.
__global__ void k_sparse_soc_rows(ConeSet cs, double *y, double *save, int dir) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cs.n_soc || !cs.soc_sparse[c]) return;
  const int off = cs.soc_off[c], d = cs.soc_dim[c];
  for (int i = 0; i < d; ++i) {
    if (dir == 0)
      save[off + i - cs.soc_begin] = y[off + i];
    else
      y[off + i] = save[off + i - cs.soc_begin];
  }
}

extern "C" int clgpu_mul_Hs_diag(clgpu_cones *h, double *y, const double *x,
                                 clgpu_stream_t stream) {
  if (!h || (h->numel > 0 && (!y || !x))) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = (h->cs.n_soc + 127) / 128;
  if (h->n_sparse) k_sparse_soc_rows<<<nb, 128, 0, st>>>(h->cs, y, h->d_save, 0);
  cones_mul_Hs(h->cs, y, x, st);
  if (h->n_sparse) k_sparse_soc_rows<<<nb, 128, 0, st>>>(h->cs, y, h->d_save, 1);
  return finish(st);
}

// delta = mean(e over the cone) / e for every cone without elementwise
// scaling (second-order, exponential, power, PSD), 1 elsewhere
// (rectify_equilibration!, coneops_compositecone_gpu.jl:21-39 and
// mathutils_gpu.jl:41-55)
__global__ void k_rectify(ConeSet cs, double *delta, const double *e) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nrec = cs.n_soc + cs.n_exp + cs.n_pow + cs.n_psd;
  if (c >= nrec) return;
  int off, len;
  if (c < cs.n_soc) {
    off = cs.soc_off[c];
    len = cs.soc_dim[c];
  } else if (c < cs.n_soc + cs.n_exp) {
    off = cs.exp_begin + 3 * (c - cs.n_soc);
    len = 3;
  } else if (c < cs.n_soc + cs.n_exp + cs.n_pow) {
    off = cs.pow_begin + 3 * (c - cs.n_soc - cs.n_exp);
    len = 3;
  } else {
    const int k = c - cs.n_soc - cs.n_exp - cs.n_pow;
    off = cs.psd_off[k];
    len = cs.psd_n[k] * (cs.psd_n[k] + 1) / 2;
  }
  if (len == 0) return;
  double mean = 0;
  for (int i = 0; i < len; ++i) mean += e[off + i];
  mean /= len;
  for (int i = 0; i < len; ++i) delta[off + i] = mean / e[off + i];
}

extern "C" int clgpu_rectify_equilibration(clgpu_cones *h, double *delta, const double *e,
                                           int *any_changed, clgpu_stream_t stream) {
  if (!h || (h->numel > 0 && (!delta || !e))) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  const ConeSet &cs = h->cs;
  const int nrec = cs.n_soc + cs.n_exp + cs.n_pow + cs.n_psd;
  if (h->numel > 0) {
    k_fill<<<(h->numel + 255) / 256, 256, 0, st>>>(delta, h->numel, 1.0);
    if (nrec > 0) k_rectify<<<(nrec + 127) / 128, 128, 0, st>>>(cs, delta, e);
  }
  if (any_changed) *any_changed = nrec > 0 ? 1 : 0;
  return finish(st);
}

// -Hs into the caller's KKT values, and the sparse-SOC expansion entries
// (the reference's vut values [-eta^2 v; -eta^2 u] per cone and -/+ eta^2 on
// the two extra diagonals)
__global__ void k_scatter_neg(const double *hs, const int *map, int n, double *kv, float *kv32) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double v = -hs[k];
  kv[map[k]] = v;
  if (kv32) kv32[map[k]] = float(v);
}
__global__ void k_sparse_soc_kkt(ConeSet cs, const int *vu, const int *vut, const int *D,
                                 double *kv, float *kv32) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cs.n_soc || !cs.soc_sparse[c]) return;
  // position of this cone among the sparse ones and its first expansion entry
  int sidx = 0, base = 0;
  for (int q = 0; q < c; ++q)
    if (cs.soc_sparse[q]) {
      ++sidx;
      base += 2 * cs.soc_dim[q];
    }
  const int off = cs.soc_off[c] - cs.soc_begin, d = cs.soc_dim[c];
  const double eta = cs.soc_eta[c], e2 = eta * eta;
  auto put = [&](int pos, double v) {
    kv[pos] = v;
    if (kv32) kv32[pos] = float(v);
  };
  for (int i = 0; i < d; ++i) {
    const double vv = -e2 * cs.soc_v[off + i], uu = -e2 * cs.soc_u[off + i];
    put(vu[base + i], vv);
    put(vut[base + i], vv);
    put(vu[base + d + i], uu);
    put(vut[base + d + i], uu);
  }
  put(D[2 * sidx], -e2);
  put(D[2 * sidx + 1], e2);
}

extern "C" int clgpu_refresh_kkt(clgpu_cones *h, double *kkt_vals, const int *hs_map,
                                 const int *vu_map, const int *vut_map, const int *D_map,
                                 float *kkt_vals32, clgpu_stream_t stream) {
  if (!h || !kkt_vals || (h->hs_len > 0 && !hs_map)) return -1;
  if (h->n_sparse > 0 && (!vu_map || !vut_map || !D_map)) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  if (h->hs_len > 0) {
    cudaMemsetAsync(h->d_hs, 0, (size_t)h->hs_len * sizeof(double), st);
    cones_get_Hs(h->cs, h->d_nn_blk, h->d_soc_blk, h->d_exp_blk, h->d_pow_blk, h->d_psd_blk,
                 h->d_hs, st);
    k_scatter_neg<<<(h->hs_len + 255) / 256, 256, 0, st>>>(h->d_hs, hs_map, h->hs_len, kkt_vals,
                                                          kkt_vals32);
  }
  if (h->n_sparse > 0)
    k_sparse_soc_kkt<<<(h->cs.n_soc + 127) / 128, 128, 0, st>>>(h->cs, vu_map, vut_map, D_map,
                                                               kkt_vals, kkt_vals32);
  return finish(st);
}

__global__ void k_min_scalar(double *a, double cap) { *a = fmin(*a, cap); }

extern "C" int clgpu_step_length_device(clgpu_cones *h, const double *dz, const double *ds,
                                        const double *z, const double *s,
                                        const double *alpha_max, double max_step_fraction,
                                        double backtrack_step, double alpha_min, double *alpha,
                                        clgpu_stream_t stream) {
  if (!h || !alpha_max || !alpha) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemcpyAsync(alpha, alpha_max, sizeof(double), cudaMemcpyDeviceToDevice, st);
  cones_step_length_sym(h->cs, dz, ds, z, s, alpha, st);
  if (!h->symmetric) {
    k_min_scalar<<<1, 1, 0, st>>>(alpha, max_step_fraction);
    cudaMemcpyAsync(h->d_scal + 2, alpha, sizeof(double), cudaMemcpyDeviceToDevice, st);
    cones_step_length_asym(h->cs, dz, ds, z, s, h->d_scal + 2, alpha, backtrack_step, alpha_min,
                           st);
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : -1000 - (int)e;
}

extern "C" int clgpu_cones_debug_scaling(const clgpu_cones *h, double *soc_w,
                                         double *soc_lambda, double *soc_u, double *soc_v,
                                         double *soc_eta, double *soc_d, double *psd_R,
                                         double *psd_Rinv, double *psd_lambda, int *psd_nmax) {
  if (!h) return -1;
  const ConeSet &cs = h->cs;
  const size_t nr = (size_t)cs.soc_rows, nc = (size_t)cs.n_soc;
  const size_t n2 = (size_t)cs.psd_nmax * cs.psd_nmax * cs.n_psd;
  const size_t nl = (size_t)cs.psd_nmax * cs.n_psd;
  struct {
    double *dst;
    const double *src;
    size_t n;
  } copies[] = {{soc_w, cs.soc_w, nr},          {soc_lambda, cs.soc_lambda, nr},
                {soc_u, cs.soc_u, nr},          {soc_v, cs.soc_v, nr},
                {soc_eta, cs.soc_eta, nc},      {soc_d, cs.soc_d, nc},
                {psd_R, cs.psd_R, n2},          {psd_Rinv, cs.psd_Rinv, n2},
                {psd_lambda, cs.psd_lam, nl}};
  for (auto &c : copies)
    if (c.dst && c.n) {
      cudaError_t e = cudaMemcpy(c.dst, c.src, c.n * sizeof(double), cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) return -1000 - (int)e;
    }
  if (psd_nmax) *psd_nmax = cs.psd_nmax;
  return 0;
}

extern "C" int clgpu_debug_soc_tiles(const int *off, const int *dim, int n, int max_cones,
                                     int max_rows, int *tiles, int cap) {
  if (n < 0 || (n > 0 && (!off || !dim)) || max_cones < 1 || max_rows < 1 || cap < 0 ||
      (cap > 0 && !tiles))
    return -1;
  std::vector<int> t = soc_tiles(off, dim, n, max_cones, max_rows);
  const int nt = (int)t.size() / 2;
  if (nt > cap) return -1;
  for (size_t i = 0; i < t.size(); ++i) tiles[i] = t[i];
  return nt;
}
