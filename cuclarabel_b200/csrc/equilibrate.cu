// equilibrate.cu -- data equilibration and KKT value assembly on the device.
//
// The reference equilibrates on the GPU at setup (data_equilibrate!, GPU
// form: src/problemdata.jl:286-374 with the row-norm kernels of
// src/utils/mathutils_gpu.jl:13-213, rectify_equilibration! of
// coneops_compositecone_gpu.jl:21) and assembles the KKT values on the GPU
// (_assemble_full_kkt_matrix, directgpu_kkt_assembly.jl:69-170).  Here the
// host keeps the structural part of setup (patterns, ordering, symbolic
// factorisation, maps), which needs no values, and the device does the
// numeric part for every instance at once:
//
//   per Ruiz iteration  column norms of [P; A] and row norms of A (max, so
//                       independent of order), the scalings 1/sqrt clipped
//                       against the accumulated ones, P, A, A', q, b scaled
//                       in place, then the cost scaling from the mean of
//                       P's column norms (summed in column order by one
//                       thread per instance) and |q|_inf;
//   rectify             delta = mean(e over the cone) / e on second-order,
//                       exponential, power and PSD rows;
//   assembly            every P and A value written to its KKT positions.
//
// Every floating-point operation is the one the host setup (setup.cpp)
// performs, in the same order, so the device result equals the host's bit
// for bit (tested).
#include <cmath>

#include "equilibrate.cuh"

namespace clgpu {

namespace {

__device__ __forceinline__ double clip_d(double s, double lo, double hi) {
  return s < lo ? lo : (s > hi ? hi : s);
}

// column norms of [P; A] (into dw) and row norms of A (into ew)
__global__ void k_eq_norms(EqDev q) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < q.nx && q.on[q.col_inst[j]]) {
    double v = 0.0;
    for (int k = q.Pp[j]; k < q.Pp[j + 1]; ++k) v = fmax(v, fabs(q.Px[k]));
    for (int k = q.Atp[j]; k < q.Atp[j + 1]; ++k) v = fmax(v, fabs(q.Atx[k]));
    q.dw[j] = v;
  }
  if (j < q.mz && q.on[q.row_inst[j]]) {
    double v = 0.0;
    for (int k = q.Ap[j]; k < q.Ap[j + 1]; ++k) v = fmax(v, fabs(q.Ax[k]));
    q.ew[j] = v;
  }
}

// the scalings: 0 -> 1, 1 / sqrt, clipped against the accumulated ones
__global__ void k_eq_vecs(EqDev q, double smin, double smax) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < q.nx && q.on[q.col_inst[j]]) {
    double v = q.dw[j];
    v = v == 0.0 ? 1.0 : v;
    v = 1.0 / sqrt(v);
    q.dw[j] = clip_d(v, smin / q.d[j], smax / q.d[j]);
  }
  if (j < q.mz && q.on[q.row_inst[j]]) {
    double v = q.ew[j];
    v = v == 0.0 ? 1.0 : v;
    v = 1.0 / sqrt(v);
    q.ew[j] = clip_d(v, smin / q.e[j], smax / q.e[j]);
  }
}

// P (column j) *= dw_i dw_j, A' (row j) *= ew_i dw_j, q *= dw, d *= dw;
// A (row i) *= ew_i dw_j, b *= ew, e *= ew
__global__ void k_eq_scale(EqDev q) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < q.nx && q.on[q.col_inst[j]]) {
    const double dj = q.dw[j];
    for (int k = q.Pp[j]; k < q.Pp[j + 1]; ++k) q.Px[k] *= q.dw[q.Pj[k]] * dj;
    for (int k = q.Atp[j]; k < q.Atp[j + 1]; ++k) q.Atx[k] *= q.ew[q.Atj[k]] * dj;
    q.q[j] *= dj;
    q.d[j] *= dj;
  }
  if (j < q.mz && q.on[q.row_inst[j]]) {
    const double ei = q.ew[j];
    for (int k = q.Ap[j]; k < q.Ap[j + 1]; ++k) q.Ax[k] *= ei * q.dw[q.Aj[k]];
    q.b[j] *= ei;
    q.e[j] *= ei;
  }
}

// P's column norms after the scaling (into dw)
__global__ void k_eq_pnorms(EqDev q) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= q.nx || !q.on[q.col_inst[j]]) return;
  double v = 0.0;
  for (int k = q.Pp[j]; k < q.Pp[j + 1]; ++k) v = fmax(v, fabs(q.Px[k]));
  q.dw[j] = v;
}

// cost scaling factor of each instance (one thread per instance: the mean
// of P's column norms summed in column order, |q|_inf); ct = 1 when skipped
__global__ void k_eq_cost(EqDev q, double smin, double smax) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= q.B || !q.on[i]) return;
  const int x0 = q.xoff[i], x1 = q.xoff[i + 1], n = x1 - x0;
  double mean = 0.0, infq = 0.0;
  for (int j = x0; j < x1; ++j) mean += q.dw[j];
  mean = n > 0 ? mean / n : 0.0;
  for (int j = x0; j < x1; ++j) infq = fmax(infq, fabs(q.q[j]));
  double ct = 1.0;
  bool apply = false;
  if (mean != 0.0 && infq != 0.0) {
    const double sc = fmax(infq, mean);
    ct = clip_d(1.0 / sc, smin / q.c[i], smax / q.c[i]);
    apply = true;
  }
  q.ct[i] = ct;
  q.cflag[i] = apply ? 1 : 0;
  if (apply) q.c[i] *= ct;
}

__global__ void k_eq_cost_apply(EqDev q) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= q.nx) return;
  const int i = q.col_inst[j];
  if (!q.on[i] || !q.cflag[i]) return;
  const double ct = q.ct[i];
  for (int k = q.Pp[j]; k < q.Pp[j + 1]; ++k) q.Px[k] *= ct;
  q.q[j] *= ct;
}

// rectify_equilibration!: delta over each second-order / exp / pow / PSD
// cone (the cone's rows summed in order), applied to A's rows, A' columns,
// b and e
__global__ void k_eq_rectify(EqDev q) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= q.nrc) return;
  const int2 rc = q.rcone[c];  // first global row, rows
  if (!q.on[q.row_inst[rc.x]] || rc.y == 0) return;
  double mu = 0.0;
  for (int k = 0; k < rc.y; ++k) mu += q.e[rc.x + k];
  mu /= rc.y;
  for (int k = 0; k < rc.y; ++k) q.ew[rc.x + k] = mu / q.e[rc.x + k];
}
__global__ void k_eq_rectify_apply(EqDev q) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < q.nx && q.on[q.col_inst[j]])
    for (int k = q.Atp[j]; k < q.Atp[j + 1]; ++k) q.Atx[k] *= q.ew[q.Atj[k]];
  if (j < q.mz && q.on[q.row_inst[j]]) {
    const double dl = q.ew[j];
    for (int k = q.Ap[j]; k < q.Ap[j + 1]; ++k) q.Ax[k] *= dl;
    q.b[j] *= dl;
    q.e[j] *= dl;
  }
}
__global__ void k_eq_fill(double *v, int n, double a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) v[j] = a;
}

// inverses, -q, and the KKT values of P and A (update_data!'s maps)
__global__ void k_eq_finish(EqDev q) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < q.nx && q.on[q.col_inst[j]]) {
    q.dinv[j] = 1.0 / q.d[j];
    q.negq[j] = -q.q[j];
  }
  if (j < q.mz && q.on[q.row_inst[j]]) q.einv[j] = 1.0 / q.e[j];
}
__global__ void k_eq_kkt_P(EqDev q, const int4 *map, const int2 *xy, long long n, double *Kx) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int2 rc = xy[t];
  if (rc.x < 0 || !q.on[q.col_inst[rc.x]]) return;
  const int4 m = map[t];
  const double v = q.Px[m.x];
  if (m.z >= 0) Kx[m.z] = v;
  if (m.w >= 0) Kx[m.w] = v;
}
__global__ void k_eq_kkt_A(EqDev q, const int4 *map, const int2 *xy, long long n, double *Kx) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  if (!q.on[q.col_inst[xy[t].y]]) return;
  const int4 m = map[t];
  const double v = q.Atx[m.x];
  if (m.z >= 0) Kx[m.z] = v;
  if (m.w >= 0) Kx[m.w] = v;
}

inline int nb(long long n) { return n <= 0 ? 1 : (int)((n + 255) / 256); }

}  // namespace

void equilibrate_on_device(const EqDev &q, const EqParams &p, const int4 *pmap,
                           const int2 *pxy, long long np, const int4 *amap, const int2 *axy,
                           long long na, double *Kx, cudaStream_t st) {
  const int nv = q.nx > q.mz ? q.nx : q.mz;
  if (p.enable) {
    for (int it = 0; it < p.max_iter; ++it) {
      k_eq_norms<<<nb(nv), 256, 0, st>>>(q);
      k_eq_vecs<<<nb(nv), 256, 0, st>>>(q, p.smin, p.smax);
      k_eq_scale<<<nb(nv), 256, 0, st>>>(q);
      k_eq_pnorms<<<nb(q.nx), 256, 0, st>>>(q);
      k_eq_cost<<<nb(q.B), 256, 0, st>>>(q, p.smin, p.smax);
      k_eq_cost_apply<<<nb(q.nx), 256, 0, st>>>(q);
    }
    if (q.nrc > 0) {
      k_eq_fill<<<nb(q.mz), 256, 0, st>>>(q.ew, q.mz, 1.0);
      k_eq_rectify<<<nb(q.nrc), 256, 0, st>>>(q);
      k_eq_rectify_apply<<<nb(nv), 256, 0, st>>>(q);
    }
  }
  k_eq_finish<<<nb(nv), 256, 0, st>>>(q);
  if (np > 0) k_eq_kkt_P<<<nb(np), 256, 0, st>>>(q, pmap, pxy, np, Kx);
  if (na > 0) k_eq_kkt_A<<<nb(na), 256, 0, st>>>(q, amap, axy, na, Kx);
}

}  // namespace clgpu
