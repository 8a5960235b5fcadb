// cones.cu -- per-cone kernels for sm_100a.
//
// Reference behaviour followed (CuClarabel tree):
//   nonnegative  src/gpucones/coneops_nncone_gpu.jl (CPU twin src/cones/coneops_nncone.jl)
//   second-order src/gpucones/coneops_socone_gpu.jl (CPU twin coneops_socone.jl:372-814)
//   exponential  src/gpucones/coneops_expcone_gpu.jl (CPU twin coneops_expcone.jl)
//   power        src/gpucones/coneops_powcone_gpu.jl (CPU twin coneops_powcone.jl)
//   nonsym share src/gpucones/coneops_nonsymmetric_common_gpu.jl
//   PSD triangle src/gpucones/coneops_psdtrianglecone_gpu.jl (CPU twin coneops_psdtrianglecone.jl)
//
// Mapping to the hardware (not a translation of the reference's one thread
// per cone):
//   * nonnegative rows: one thread per row over a contiguous type-major range
//     (coalesced FP64 streams);
//   * second-order cones: a group of G lanes per cone (G = next power of two
//     of the largest cone dim, <= 32), elements strided across the group,
//     norms/dots by shuffle reductions inside the group;
//   * exponential/power cones: one thread per cone (FP64 transcendental work);
//   * PSD cones: one warp per cone with its n x n matrices in shared memory
//     (Cholesky, one-sided Jacobi SVD, Jacobi eigenvalues, small GEMMs).  The
//     t x t Hs block is never stored: the KKT refresh evaluates the symmetric
//     Kronecker product entries from R R^T on the fly.
#include <algorithm>
#include <cstdio>

#include "cones.cuh"

namespace clgpu {

static constexpr int kBlock = 256;
static constexpr int kNNRows = 4;  // rows per thread of k_nn_affine_ds, single-problem k_nn_step
static constexpr int kPsdWarps = 2;  // warps (cones) per PSD block

__device__ __forceinline__ bool active_inst(const ConeSet &cs, int inst) {
  return cs.inst_active == nullptr || cs.inst_active[inst] != 0;
}
// Instance of row g: a single problem streams no row-to-instance index.
__device__ __forceinline__ int row_instance(const ConeSet &cs, int g) {
  return cs.B == 1 ? 0 : cs.row_inst[g];
}
// Row g belongs to a running instance; the row's instance is looked up only
// when there is an active mask.
__device__ __forceinline__ bool active_row(const ConeSet &cs, int g) {
  return cs.inst_active == nullptr || cs.inst_active[row_instance(cs, g)] != 0;
}

// =================================================================== NN
__global__ void k_nn_update_scaling(ConeSet cs, const double *__restrict__ s,
                                    const double *__restrict__ z) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= cs.n_nn) return;
  int g = cs.nn_begin + e;
  if (!active_row(cs, g)) return;
  double si = s[g], zi = z[g];
  cs.nn_lambda[e] = sqrt(si * zi);
  cs.nn_w[e] = sqrt(si / zi);
}

// =================================================================== SOC
// group helpers --------------------------------------------------------
template <int G>
struct SocCtx {
  int c, lane, off, dim, inst;
  bool valid;
  __device__ SocCtx(const ConeSet &cs) {
    int gid = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    lane = threadIdx.x & (G - 1);
    valid = gid < cs.n_soc;
    c = valid ? gid : cs.n_soc - 1;
    off = cs.soc_off[c];
    dim = cs.soc_dim[c];
    inst = cs.soc_inst[c];
    if (valid && !active_inst(cs, inst)) valid = false;
    if (valid && dim >= cs.soc_skip_lo && dim <= cs.soc_skip_hi) valid = false;
  }
};
#define SOC_FOR(i) for (int i = ctx.lane; i < ctx.dim; i += G)

template <int G>
__device__ __forceinline__ double soc_tail_sq(const double *x, const SocCtx<G> &ctx) {
  double t = 0;
  SOC_FOR(i) if (i > 0) t += x[i] * x[i];
  return group_sum<G>(t);
}
template <int G>
__device__ __forceinline__ double soc_tail_dot(const double *x, const double *y,
                                               const SocCtx<G> &ctx) {
  double t = 0;
  SOC_FOR(i) if (i > 0) t += x[i] * y[i];
  return group_sum<G>(t);
}
// (x0 - |x1|)(x0 + |x1|), coneops_socone.jl:716-720
__device__ __forceinline__ double soc_res(double x0, double x1sq) {
  double n1 = sqrt(x1sq);
  return (x0 - n1) * (x0 + n1);
}

// coneops_socone.jl:372-451 (and the sparse d/u/v of
// coneops_socone_gpu.jl:338-470, kept unscaled as on the CPU side)
template <int G>
__global__ void k_soc_update_scaling(ConeSet cs, const double *__restrict__ s_,
                                     const double *__restrict__ z_, int *scale_ok) {
  SocCtx<G> ctx(cs);
  const double *s = s_ + ctx.off, *z = z_ + ctx.off;
  int r = ctx.off - cs.soc_begin;
  double *w = cs.soc_w + r, *lam = cs.soc_lambda + r;
  double s0 = s[0], z0 = z[0];
  double zs = soc_res(z0, soc_tail_sq<G>(z, ctx));
  double ss = soc_res(s0, soc_tail_sq<G>(s, ctx));
  double zscale = zs > 0.0 ? sqrt(zs) : 0.0;
  double sscale = ss > 0.0 ? sqrt(ss) : 0.0;
  bool fail = (zscale == 0.0 || sscale == 0.0);
  if (fail) {
    if (ctx.valid && ctx.lane == 0) scale_ok[ctx.inst] = 0;
    zscale = sscale = 1.0;  // keep lanes in lock step; results discarded
  }
  double eta = sqrt(sscale / zscale);
  // w = s/sscale + (z0, -z1)/zscale, with the three scalings' reciprocals
  // taken once per cone (the tile kernel below does the same, so both
  // forms agree bit for bit)
  const double isc = 1.0 / sscale, izc = 1.0 / zscale;
  double wl[4];  // per-lane cache (dim <= 4*G handled in registers)
  int k = 0;
  double w1sq_a = 0;
  SOC_FOR(i) {
    double wi = __dadd_rn(__dmul_rn(s[i], isc), __dmul_rn(i == 0 ? z[i] : -z[i], izc));
    if (k < 4) wl[k] = wi;
    ++k;
    if (i > 0) w1sq_a += wi * wi;
  }
  double w0pre = __dadd_rn(__dmul_rn(s0, isc), __dmul_rn(z0, izc));
  double wres = soc_res(w0pre, group_sum<G>(w1sq_a));
  double wscale = wres > 0.0 ? sqrt(wres) : 0.0;
  if (wscale == 0.0) {
    if (ctx.valid && ctx.lane == 0) scale_ok[ctx.inst] = 0;
    fail = true;
    wscale = 1.0;
  }
  double w1sq = 0;
  const double iwc = 1.0 / wscale;
  k = 0;
  SOC_FOR(i) {
    double wi = __dmul_rn(k < 4 ? wl[k]
                                : __dadd_rn(__dmul_rn(s[i], isc),
                                            __dmul_rn(i == 0 ? z[i] : -z[i], izc)),
                          iwc);
    if (k < 4) wl[k] = wi;
    ++k;
    if (i > 0) w1sq += wi * wi;
  }
  w1sq = group_sum<G>(w1sq);
  double w0 = sqrt(1 + w1sq);
  double gamma = 0.5 * wscale;
  double c1 = __dmul_rn(__dadd_rn(gamma, __dmul_rn(z0, izc)), isc);
  double c2 = __dmul_rn(__dadd_rn(gamma, __dmul_rn(s0, isc)), izc);
  double inv = 1.0 / __dadd_rn(w0pre, 2 * gamma);
  double sc = sqrt(sscale * zscale);
  bool sparse = cs.soc_sparse[ctx.c] != 0;
  double u0 = 0, u1 = 0, v1 = 0, dd = 0;
  if (sparse) {
    double wsq = w0 * w0 + w1sq;
    double wsqinv = 1 / wsq;
    dd = wsqinv / 2;
    u0 = sqrt(wsq - dd);
    u1 = 2 * w0 / u0;
    v1 = sqrt(2 * (2 + wsqinv) / (2 * wsq - wsqinv));
  }
  if (!ctx.valid || fail) return;
  k = 0;
  SOC_FOR(i) {
    double wi = (k < 4) ? wl[k]
                        : __dmul_rn(__dadd_rn(__dmul_rn(s[i], isc),
                                              __dmul_rn(i == 0 ? z[i] : -z[i], izc)),
                                    iwc);
    ++k;
    if (i == 0) {
      w[0] = w0;
      lam[0] = gamma * sc;
      if (sparse) {
        cs.soc_u[r] = u0;
        cs.soc_v[r] = 0.0;
      }
    } else {
      w[i] = wi;
      lam[i] = ((c1 * s[i] + c2 * z[i]) * inv) * sc;
      if (sparse) {
        cs.soc_u[r + i] = u1 * wi;
        cs.soc_v[r + i] = v1 * wi;
      }
    }
  }
  if (ctx.lane == 0) {
    cs.soc_eta[ctx.c] = eta;
    if (sparse) cs.soc_d[ctx.c] = dd;
  }
}

// =============================================================== exp / pow
struct M3 {
  double a[9];  // column-major
  __device__ double &operator()(int i, int j) { return a[i + 3 * j]; }
  __device__ double operator()(int i, int j) const { return a[i + 3 * j]; }
};

// coneops_expcone.jl:655-711 (Wright omega; the third Taylor term keeps the
// reference's unassigned "q * zinv" statement)
__device__ double wright_omega(double z) {
  if (z < 0) return CUDART_INF;
  double w;
  if (z < 1.0 + 3.141592653589793) {
    double zm1 = z - 1.0, p = zm1;
    w = 1 + 0.5 * p;
    p *= zm1;
    w += (1 / 16.0) * p;
    p *= zm1;
    w -= (1 / 192.0) * p;
    p *= zm1;
    w -= (1 / 3072.0) * p;
    p *= zm1;
    w += (13 / 61440.0) * p;
  } else {
    double logz = logsafe(z), zinv = 1.0 / z;
    w = z - logz;
    double q = logz * zinv;
    w += q;
    q *= zinv;
    w += q * (logz / 2 - 1.0);
    w += q * (logz * logz / 3. - (3 / 2.) * logz + 1.0);
  }
  double r = z - w - logsafe(w);
  for (int i = 0; i < 2; ++i) {
    double wp1 = w + 1.0;
    double t = wp1 * (wp1 + (2. * r) / 3.0);
    w *= 1 + (r / wp1) * (t - 0.5 * r) / (t - r);
    double wp2 = wp1 * wp1, wp6 = wp2 * wp2 * wp2;
    r = (2 * w * w - 8 * w - 1) / (72.0 * wp6) * r * r * r * r;
  }
  return w;
}

struct ExpOps {
  __device__ static void grad_primal(const double *s, double *g, double) {
    double o = wright_omega(1 - s[0] / s[1] - logsafe(s[1] / s[2]));
    g[0] = 1.0 / ((o - 1.0) * s[1]);
    g[1] = g[0] + g[0] * logsafe(o * s[1] / s[2]) - 1.0 / s[1];
    g[2] = o / ((1.0 - o) * s[2]);
  }
  __device__ static void dual_grad_H(const double *z, double *grad, M3 &H, double) {
    double l = logsafe(-z[2] / z[0]);
    double r = -z[0] * l - z[0] + z[1];
    double c2 = 1.0 / r;
    grad[0] = c2 * l - 1 / z[0];
    grad[1] = -c2;
    grad[2] = (c2 * z[0] - 1) / z[2];
    H(0, 0) = ((r * r - z[0] * r + l * l * z[0] * z[0]) / (r * z[0] * z[0] * r));
    H(0, 1) = (-l / (r * r));
    H(1, 0) = H(0, 1);
    H(1, 1) = (1 / (r * r));
    H(0, 2) = ((z[1] - z[0]) / (r * r * z[2]));
    H(2, 0) = H(0, 2);
    H(1, 2) = (-z[0] / (r * r * z[2]));
    H(2, 1) = H(1, 2);
    H(2, 2) = ((r * r - z[0] * r + z[0] * z[0]) / (r * r * z[2] * z[2]));
  }
  __device__ static bool primal_feasible(const double *s, double) {
    if (s[2] > 0 && s[1] > 0) {
      double res = s[1] * logsafe(s[2] / s[1]) - s[0];
      if (res > 0) return true;
    }
    return false;
  }
  __device__ static bool dual_feasible(const double *z, double) {
    if (z[2] > 0 && z[0] < 0) {
      double res = z[1] - z[0] - z[0] * logsafe(-z[2] / z[0]);
      if (res > 0) return true;
    }
    return false;
  }
  __device__ static double barrier_dual(const double *z, double) {
    double l = logsafe(-z[2] / z[0]);
    return -logsafe(-z[2] * z[0]) - logsafe(z[1] - z[0] - z[0] * l);
  }
  __device__ static double barrier_primal(const double *s, double) {
    double o = wright_omega(1 - s[0] / s[1] - logsafe(s[1] / s[2]));
    o = (o - 1) * (o - 1) / o;
    return -logsafe(o) - 2 * logsafe(s[1]) - logsafe(s[2]) - 3;
  }
  // coneops_expcone.jl:530-577
  __device__ static void higher_correction(const M3 &Hd, const double *z,
                                           const double *u, const double *v,
                                           double *eta, double) {
    eta[1] = 1.0;
    eta[2] = -z[0] / z[2];
    eta[0] = logsafe(eta[2]);
    double psi = z[0] * eta[0] - z[0] + z[1];
    double dotpu = eta[0] * u[0] + eta[1] * u[1] + eta[2] * u[2];
    double dotpv = eta[0] * v[0] + eta[1] * v[1] + eta[2] * v[2];
    double coef = ((u[0] * (v[0] / z[0] - v[2] / z[2]) +
                    u[2] * (z[0] * v[2] / z[2] - v[0]) / z[2]) * psi -
                   2 * dotpu * dotpv) / (psi * psi * psi);
    for (int i = 0; i < 3; ++i) eta[i] *= coef;
    double ip2 = 1.0 / psi / psi;
    eta[0] += (1 / psi - 2 / z[0]) * u[0] * v[0] / (z[0] * z[0]) -
              u[2] * v[2] / (z[2] * z[2]) / psi +
              dotpu * ip2 * (v[0] / z[0] - v[2] / z[2]) +
              dotpv * ip2 * (u[0] / z[0] - u[2] / z[2]);
    eta[2] += 2 * (z[0] / psi - 1) * u[2] * v[2] / (z[2] * z[2] * z[2]) -
              (u[2] * v[0] + u[0] * v[2]) / (z[2] * z[2]) / psi +
              dotpu * ip2 * (z[0] * v[2] / (z[2] * z[2]) - v[0] / z[2]) +
              dotpv * ip2 * (z[0] * u[2] / (z[2] * z[2]) - u[0] / z[2]);
    for (int i = 0; i < 3; ++i) eta[i] /= 2;
    (void)Hd;
  }
  __device__ static void unit_init(double *s, double) {
    s[0] = -1.051383945322714;
    s[1] = 0.556409619469370;
    s[2] = 1.258967884768947;
  }
};

// coneops_powcone.jl:449-478 restated (Newton-Raphson from the left)
__device__ double pow_nr(double s3, double phi, double a) {
  double x0 = -1.0 / s3 + (2 * s3 + sqrt(phi * phi / s3 / s3 + 3 * phi)) / (phi - s3 * s3);
  double t0 = -2 * a * logsafe(a) - 2 * (1 - a) * logsafe(1 - a);
  double x = x0;
  for (int iter = 0; iter < 100; ++iter) {
    double t1 = x * x, t2 = x * 2 / s3;
    double dfdx = 2 * a * a / (a * x + (1 + a) / s3) +
                  2 * (1 - a) * (1 - a) / ((1 - a) * x + (2 - a) / s3) -
                  2 * (x + 1 / s3) / (t1 + t2);
    t2 = 2 * x / s3;
    double f0 = 2 * a * logsafe(2 * a * t1 + (1 + a) * t2) +
                2 * (1 - a) * logsafe(2 * (1 - a) * t1 + (2 - a) * t2) -
                logsafe(phi) - logsafe(t1 + t2) - 2 * logsafe(t2) + t0;
    double dx = -f0 / dfdx;
    if (dx < kDEps || fabs(dx / x) < sqrt(kDEps) || fabs(dfdx) < kDEps) break;
    x += dx;
  }
  return x;
}

struct PowOps {
  __device__ static void grad_primal(const double *s, double *g, double a) {
    double phi = pow(s[0], 2 * a) * pow(s[1], 2 - 2 * a);
    double abs_s = fabs(s[2]);
    if (abs_s > kDEps) {
      g[2] = pow_nr(abs_s, phi, a);
      if (s[2] < 0) g[2] = -g[2];
      g[0] = -(a * g[2] * s[2] + 1 + a) / s[0];
      g[1] = -((1 - a) * g[2] * s[2] + 2 - a) / s[1];
    } else {
      g[2] = 0;
      g[0] = -(1 + a) / s[0];
      g[1] = -(2 - a) / s[1];
    }
  }
  // coneops_powcone.jl:408-440
  __device__ static void dual_grad_H(const double *z, double *grad, M3 &H, double a) {
    double phi = pow(z[0] / a, 2 * a) * pow(z[1] / (1 - a), 2 - 2 * a);
    double psi = phi - z[2] * z[2];
    double g0 = 2 * a * phi / (z[0] * psi);
    double g1 = 2 * (1 - a) * phi / (z[1] * psi);
    double g2 = -2 * z[2] / psi;
    H(0, 0) = g0 * g0 - 2 * a * (2 * a - 1) * phi / (z[0] * z[0] * psi) + (1 - a) / (z[0] * z[0]);
    H(0, 1) = g0 * g1 - 4 * a * (1 - a) * phi / (z[0] * z[1] * psi);
    H(1, 0) = H(0, 1);
    H(1, 1) = g1 * g1 - 2 * (1 - a) * (1 - 2 * a) * phi / (z[1] * z[1] * psi) + a / (z[1] * z[1]);
    H(0, 2) = g0 * g2;
    H(2, 0) = H(0, 2);
    H(1, 2) = g1 * g2;
    H(2, 1) = H(1, 2);
    H(2, 2) = g2 * g2 + 2 / psi;
    grad[0] = -2 * a * phi / (z[0] * psi) - (1 - a) / z[0];
    grad[1] = -2 * (1 - a) * phi / (z[1] * psi) - a / z[1];
    grad[2] = 2 * z[2] / psi;
  }
  __device__ static bool primal_feasible(const double *s, double a) {
    if (s[0] > 0 && s[1] > 0) {
      double res = exp(2 * a * logsafe(s[0]) + 2 * (1 - a) * logsafe(s[1])) - s[2] * s[2];
      if (res > 0) return true;
    }
    return false;
  }
  __device__ static bool dual_feasible(const double *z, double a) {
    if (z[0] > 0 && z[1] > 0) {
      double res = exp(2 * a * logsafe(z[0] / a) + 2 * (1 - a) * logsafe(z[1] / (1 - a))) -
                   z[2] * z[2];
      if (res > 0) return true;
    }
    return false;
  }
  __device__ static double barrier_dual(const double *z, double a) {
    return -logsafe(pow(z[0] / a, 2 * a) * pow(z[1] / (1 - a), 2 - 2 * a) - z[2] * z[2]) -
           (1 - a) * logsafe(z[0]) - a * logsafe(z[1]);
  }
  __device__ static double barrier_primal(const double *s, double a) {
    double g[3];
    grad_primal(s, g, a);
    return logsafe(pow(-g[0] / a, 2 * a) * pow(-g[1] / (1 - a), 2 - 2 * a) - g[2] * g[2]) +
           (1 - a) * logsafe(-g[0]) + a * logsafe(-g[1]) - 3;
  }
  // coneops_powcone.jl:329-404
  __device__ static void higher_correction(const M3 &Hd, const double *z,
                                           const double *u, const double *v,
                                           double *eta, double a) {
    double phi = pow(z[0] / a, 2 * a) * pow(z[1] / (1 - a), 2 - 2 * a);
    double psi = phi - z[2] * z[2];
    eta[0] = 2 * a * phi / z[0];
    eta[1] = 2 * (1 - a) * phi / z[1];
    eta[2] = -2 * z[2];
    double H11 = 2 * a * (2 * a - 1) * phi / (z[0] * z[0]);
    double H12 = 4 * a * (1 - a) * phi / (z[0] * z[1]);
    double H22 = 2 * (1 - a) * (1 - 2 * a) * phi / (z[1] * z[1]);
    double dotpu = eta[0] * u[0] + eta[1] * u[1] + eta[2] * u[2];
    double dotpv = eta[0] * v[0] + eta[1] * v[1] + eta[2] * v[2];
    double Hv0 = H11 * v[0] + H12 * v[1], Hv1 = H12 * v[0] + H22 * v[1], Hv2 = -2 * v[2];
    double coef = ((u[0] * Hv0 + u[1] * Hv1 + u[2] * Hv2) * psi - 2 * dotpu * dotpv) /
                  (psi * psi * psi);
    double coef2 = 4 * a * (2 * a - 1) * (1 - a) * phi * (u[0] / z[0] - u[1] / z[1]) *
                   (v[0] / z[0] - v[1] / z[1]) / psi;
    double ip2 = 1 / psi / psi;
    eta[0] = coef * eta[0] - 2 * (1 - a) * u[0] * v[0] / (z[0] * z[0] * z[0]) +
             coef2 / z[0] + Hv0 * dotpu * ip2;
    eta[1] = coef * eta[1] - 2 * a * u[1] * v[1] / (z[1] * z[1] * z[1]) -
             coef2 / z[1] + Hv1 * dotpu * ip2;
    eta[2] = coef * eta[2] + Hv2 * dotpu * ip2;
    double Hu0 = H11 * u[0] + H12 * u[1], Hu1 = H12 * u[0] + H22 * u[1], Hu2 = -2 * u[2];
    eta[0] = (eta[0] + Hu0 * dotpv * ip2) / 2;
    eta[1] = (eta[1] + Hu1 * dotpv * ip2) / 2;
    eta[2] = (eta[2] + Hu2 * dotpv * ip2) / 2;
    (void)Hd;
  }
  __device__ static void unit_init(double *s, double a) {
    s[0] = sqrt(1.0 + a);
    s[1] = sqrt(1.0 + (1.0 - a));
    s[2] = 0.0;
  }
};

// mathutils.jl:381-420
__device__ bool chol3(const M3 &A, M3 &L) {
  for (int i = 0; i < 9; ++i) L.a[i] = 0;
  double t = A(0, 0);
  if (t <= 0) return false;
  L(0, 0) = sqrt(t);
  L(1, 0) = A(1, 0) / L(0, 0);
  t = A(1, 1) - L(1, 0) * L(1, 0);
  if (t <= 0) return false;
  L(1, 1) = sqrt(t);
  L(2, 0) = A(2, 0) / L(0, 0);
  L(2, 1) = (A(2, 1) - L(1, 0) * L(2, 0)) / L(1, 1);
  t = A(2, 2) - L(2, 0) * L(2, 0) - L(2, 1) * L(2, 1);
  if (t <= 0) return false;
  L(2, 2) = sqrt(t);
  return true;
}
__device__ void chol3_solve(const M3 &L, const double *b, double *x) {
  double L11 = L(0, 0), L21 = L(1, 0), L31 = L(2, 0), L22 = L(1, 1), L32 = L(2, 1), L33 = L(2, 2);
  double c1 = b[0] / L11;
  double c2 = (b[1] * L11 - b[0] * L21) / (L11 * L22);
  double c3 = (b[2] * L11 * L22 - b[1] * L11 * L32 + b[0] * L21 * L32 - b[0] * L22 * L31) /
              (L11 * L22 * L33);
  x[0] = (c1 * L22 * L33 - c2 * L21 * L33 + c3 * L21 * L32 - c3 * L22 * L31) / (L11 * L22 * L33);
  x[1] = (c2 * L33 - c3 * L32) / (L22 * L33);
  x[2] = c3 / L33;
}

template <class Ops>
struct NonsymArgs {
  int n, begin;
  const int *inst;
  const double *alpha;  // pow only
  double *Hd, *Hs, *grad, *zs;
};

// coneops_nonsymmetric_common.jl:50-164 (dual and primal-dual scalings)
// Register caps (7 and 8 resident blocks of 128 threads) for the two
// register-heavy exp/pow kernels: more warps in flight hide their FP64
// latency better than the spill-free allocation did (measured on 4 M exp and
// 4 M pow cones: update_scaling 520 -> 425 us and 676 -> 576 us, pow
// combined_ds_shift 280 -> 228 us; exp combined_ds_shift unchanged at 8).
// The block's 128 cones are staged through shared memory on both sides:
// their s and z (3 doubles each, 24-byte stride in global memory) are read
// with coalesced loads, and their 24 outputs per cone (Hd, Hs, grad, z) are
// written back as contiguous runs, instead of one 8-byte access per cone
// and lane at a 24- or 72-byte stride.
template <class Ops>
__global__ void __launch_bounds__(128, 7) k_nonsym_update_scaling(ConeSet cs, NonsymArgs<Ops> a,
                                        const double *__restrict__ s_,
                                        const double *__restrict__ z_,
                                        const double *mu_, const int *scaling) {
  __shared__ double ss[3 * 128], sz[3 * 128], sHd[9 * 128], sHs[9 * 128], sg[3 * 128];
  __shared__ unsigned char on[128];
  const int c0 = blockIdx.x * 128, nb = min(128, a.n - c0), tid = threadIdx.x;
  for (int i = tid; i < 3 * nb; i += 128) {
    ss[i] = s_[a.begin + 3 * c0 + i];
    sz[i] = z_[a.begin + 3 * c0 + i];
  }
  __syncthreads();
  const int c = c0 + tid;
  const int inst = tid < nb ? a.inst[c] : -1;
  const bool act = tid < nb && active_inst(cs, inst);
  on[tid] = act ? 1 : 0;
  if (act) {
    double pa = a.alpha ? a.alpha[c] : 0.0;
    double sv[3] = {ss[3 * tid], ss[3 * tid + 1], ss[3 * tid + 2]};
    double zv[3] = {sz[3 * tid], sz[3 * tid + 1], sz[3 * tid + 2]};
    double grad[3];
    M3 Hd, Hs;
    Ops::dual_grad_H(zv, grad, Hd, pa);
    double mu = mu_[inst];
    bool dual = scaling[inst] == 1;
    bool used_pd = false;
    if (!dual) {
      const double *st = grad;
      double zt[3];
      Ops::grad_primal(sv, zt, pa);
      double dot_sz = zv[0] * sv[0] + zv[1] * sv[1] + zv[2] * sv[2];
      double mu_l = dot_sz / 3;
      double mut = (zt[0] * st[0] + zt[1] * st[1] + zt[2] * st[2]) / 3;
      double ds[3], dz[3];
      for (int i = 0; i < 3; ++i) {
        ds[i] = sv[i] + mu_l * st[i];
        dz[i] = zv[i] + mu_l * zt[i];
      }
      double dot_dsz = ds[0] * dz[0] + ds[1] * dz[1] + ds[2] * dz[2];
      double de1 = mu_l * mut - 1;
      double Hz[3];
      for (int i = 0; i < 3; ++i) Hz[i] = Hd(i, 0) * zt[0] + Hd(i, 1) * zt[1] + Hd(i, 2) * zt[2];
      double de2 = zt[0] * Hz[0] + zt[1] * Hz[1] + zt[2] * Hz[2] - 3 * mut * mut;
      if (fabs(de1) > sqrt(kDEps) && fabs(de2) > kDEps && dot_sz > 0 && dot_dsz > 0) {
        double tmp[3];
        for (int i = 0; i < 3; ++i) tmp[i] = mut * st[i] - Hz[i];
        for (int i = 0; i < 9; ++i) Hs.a[i] = Hd.a[i];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) Hs(i, j) -= st[i] * st[j] / 3 + tmp[i] * tmp[j] / de2;
        double fro = 0;
        for (int i = 0; i < 9; ++i) fro += Hs.a[i] * Hs.a[i];
        double t = mu_l * sqrt(fro);
        double ax[3] = {zv[1] * zt[2] - zv[2] * zt[1], zv[2] * zt[0] - zv[0] * zt[2],
                        zv[0] * zt[1] - zv[1] * zt[0]};
        double an = sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]);
        for (int i = 0; i < 3; ++i) ax[i] /= an;
        for (int i = 0; i < 3; ++i)
          for (int j = i; j < 3; ++j)
            Hs(i, j) = sv[i] * sv[j] / dot_sz + ds[i] * ds[j] / dot_dsz + t * ax[i] * ax[j];
        Hs(1, 0) = Hs(0, 1);
        Hs(2, 0) = Hs(0, 2);
        Hs(2, 1) = Hs(1, 2);
        used_pd = true;
      } else {
        mu = mu_l;  // central-path fallback uses the local mu
      }
    }
    if (!used_pd)
      for (int i = 0; i < 9; ++i) Hs.a[i] = mu * Hd.a[i];
    for (int i = 0; i < 9; ++i) {
      sHd[9 * tid + i] = Hd.a[i];
      sHs[9 * tid + i] = Hs.a[i];
    }
    for (int i = 0; i < 3; ++i) sg[3 * tid + i] = grad[i];
  }
  __syncthreads();
  for (int i = tid; i < 9 * nb; i += 128)
    if (on[i / 9]) {
      a.Hd[9 * c0 + i] = sHd[i];
      a.Hs[9 * c0 + i] = sHs[i];
    }
  for (int i = tid; i < 3 * nb; i += 128)
    if (on[i / 3]) {
      a.grad[3 * c0 + i] = sg[i];
      a.zs[3 * c0 + i] = sz[i];
    }
}

// =================================================================== PSD
// Group-per-cone helpers on column-major n x n matrices in shared memory.
// A cone is handled by a group of G lanes of one warp: G = 16 when every
// PSD side of the set is at most 16 (two cones per warp), else G = 32.
// Groups of one warp run independently (their own loop trip counts), so
// every barrier and shuffle names the group's lanes only.
struct PsdGrp {
  int lane, G;
  unsigned mask;  // this group's lanes
  unsigned warp;  // lanes of the warp's groups still working (for votes)
  __device__ __forceinline__ void sync() const { __syncwarp(mask); }
  __device__ __forceinline__ double sum(double v) const {
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
    return v;
  }
  __device__ __forceinline__ double min(double v) const {
    for (int o = G / 2; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(mask, v, o));
    return v;
  }
};
__host__ __device__ __forceinline__ int psd_group(int nmax) { return nmax <= 16 ? 16 : 32; }
struct PsdCtx {
  int c, lane, n, t, off, inst;
  PsdGrp g;
  bool valid;
};

__device__ __forceinline__ void svec_to_mat(int n, const double *x, double *M, const PsdGrp &g) {
  const double is2 = 0.70710678118654752440;  // 1/sqrt(2)
  int t = n * (n + 1) / 2;
  for (int k = g.lane; k < t; k += g.G) {
    int col = (int)((sqrt(8.0 * k + 1.0) - 1.0) * 0.5);
    while ((col + 1) * (col + 2) / 2 <= k) ++col;
    while (col * (col + 1) / 2 > k) --col;
    int row = k - col * (col + 1) / 2;
    double v = x[k];
    if (row == col)
      M[row + n * col] = v;
    else {
      M[row + n * col] = v * is2;
      M[col + n * row] = v * is2;
    }
  }
}
__device__ __forceinline__ void mat_to_svec(int n, const double *M, double *x, const PsdGrp &g) {
  const double is2 = 0.70710678118654752440;
  int t = n * (n + 1) / 2;
  for (int k = g.lane; k < t; k += g.G) {
    int col = (int)((sqrt(8.0 * k + 1.0) - 1.0) * 0.5);
    while ((col + 1) * (col + 2) / 2 <= k) ++col;
    while (col * (col + 1) / 2 > k) --col;
    int row = k - col * (col + 1) / 2;
    x[k] = row == col ? M[row + n * col] : (M[row + n * col] + M[col + n * row]) * is2;
  }
}
// C = op(A) * op(B)   (n x n), ta/tb: transpose flags
__device__ void mm(int n, const double *A, bool ta, const double *B, bool tb, double *C,
                   const PsdGrp &g) {
  for (int e = g.lane; e < n * n; e += g.G) {
    int i = e % n, j = e / n;
    double t = 0;
    for (int k = 0; k < n; ++k) {
      double a = ta ? A[k + n * i] : A[i + n * k];
      double b = tb ? B[j + n * k] : B[k + n * j];
      t += a * b;
    }
    C[e] = t;
  }
  g.sync();
}
// in-place lower Cholesky; returns false if not positive definite
__device__ bool warp_chol(int n, double *A, const PsdGrp &g) {
  bool ok = true;
  for (int j = 0; j < n; ++j) {
    double d = A[j + n * j];
    for (int k = 0; k < j; ++k) d -= A[j + n * k] * A[j + n * k];
    if (!(d > 0)) ok = false;
    d = ok ? sqrt(d) : 1.0;
    g.sync();
    for (int i = j + 1 + g.lane; i < n; i += g.G) {
      double t = A[i + n * j];
      for (int k = 0; k < j; ++k) t -= A[i + n * k] * A[j + n * k];
      A[i + n * j] = t / d;
    }
    if (g.lane == 0) A[j + n * j] = d;
    for (int i = g.lane; i < j; i += g.G) A[i + n * j] = 0;
    g.sync();
  }
  return ok;
}
// one-sided Jacobi SVD: M = U diag(S) V^T; S descending.  M overwritten by U.
__device__ void warp_svd(int n, double *M, double *V, double *S, double *tmp, const PsdGrp &g) {
  for (int e = g.lane; e < n * n; e += g.G) V[e] = (e % n == e / n) ? 1.0 : 0.0;
  g.sync();
  for (int sweep = 0; sweep < 60; ++sweep) {
    int rotated = 0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        double a = 0, b = 0, gd = 0;
        for (int r = g.lane; r < n; r += g.G) {
          double mp = M[r + n * p], mq = M[r + n * q];
          a += mp * mp;
          b += mq * mq;
          gd += mp * mq;
        }
        a = g.sum(a);
        b = g.sum(b);
        gd = g.sum(gd);
        // columns orthogonal to 1e-14 of their norms: the rounding noise of
        // the dot products of n <= 48 rows sits near n^(1/2) eps, so a
        // tighter bound keeps rotating at noise level until the sweep cap.
        // A skipped pair applies the identity rotation (bit for bit no
        // change), so both groups of a warp follow the same path.
        const bool skip = fabs(gd) <= 1e-14 * sqrt(a * b) || gd == 0;
        double cs = 1.0, sn = 0.0;
        if (!skip) {
          rotated = 1;
          double zeta = (b - a) / (2 * gd);
          double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1 + zeta * zeta));
          cs = 1 / sqrt(1 + t * t);
          sn = cs * t;
        }
        for (int r = g.lane; r < n; r += g.G) {
          double mp = M[r + n * p], mq = M[r + n * q];
          M[r + n * p] = cs * mp - sn * mq;
          M[r + n * q] = sn * mp + cs * mq;
          double vp = V[r + n * p], vq = V[r + n * q];
          V[r + n * p] = cs * vp - sn * vq;
          V[r + n * q] = sn * vp + cs * vq;
        }
        g.sync();
      }
    if (!__any_sync(g.warp, rotated)) break;  // every group of the warp converged
  }
  // column norms, sort descending (selection on the group's lane 0 into tmp perm)
  for (int c = g.lane; c < n; c += g.G) {
    double t = 0;
    for (int k = 0; k < n; ++k) t += M[k + n * c] * M[k + n * c];
    S[c] = sqrt(t);
  }
  g.sync();
  int *perm = reinterpret_cast<int *>(tmp + n * n);
  if (g.lane == 0) {
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j)
        if (S[perm[j]] > S[perm[i]]) {
          int x = perm[i];
          perm[i] = perm[j];
          perm[j] = x;
        }
  }
  g.sync();
  // tmp <- U (sorted), M <- V (sorted) via copies
  for (int e = g.lane; e < n * n; e += g.G) {
    int i = e % n, j = e / n, pj = perm[j];
    double sj = S[pj];
    tmp[e] = sj > 0 ? M[i + n * pj] / sj : 0.0;
  }
  g.sync();
  for (int e = g.lane; e < n * n; e += g.G) M[e] = tmp[e];
  g.sync();
  for (int e = g.lane; e < n * n; e += g.G) {
    int i = e % n, j = e / n;
    tmp[e] = V[i + n * perm[j]];
  }
  constexpr int kRows = (kPsdMaxSide + 15) / 16;  // rows per lane (G >= 16)
  double sl[kRows];
#pragma unroll
  for (int r = 0; r < kRows; ++r)
    sl[r] = g.lane + g.G * r < n ? S[perm[g.lane + g.G * r]] : 0.0;
  g.sync();
  for (int e = g.lane; e < n * n; e += g.G) V[e] = tmp[e];
#pragma unroll
  for (int r = 0; r < kRows; ++r)
    if (g.lane + g.G * r < n) S[g.lane + g.G * r] = sl[r];
  g.sync();
}
// cyclic Jacobi eigenvalues of symmetric A (destroyed); returns min eigenvalue,
// and if ev != null writes all eigenvalues.
__device__ double warp_eig_min(int n, double *A, double *ev, const PsdGrp &g) {
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0, tot = 0;
    for (int e = g.lane; e < n * n; e += g.G) {
      double a = A[e] * A[e];
      tot += a;
      if (e % n != e / n) off += a;
    }
    off = g.sum(off);
    tot = g.sum(tot);
    // converged when the off-diagonal part is below 1e-13 of the matrix
    // (Frobenius norms): every eigenvalue is then within 1e-13 |A|_F of a
    // diagonal entry.  (A tighter relative bound sits at the rounding
    // noise of the rotations and is never reached, so the sweeps ran to
    // their cap.)
    const bool conv = off <= 1e-26 * tot || off == 0;
    if (__all_sync(g.warp, conv)) break;  // every group of the warp converged
    // threshold Jacobi: a rotation whose effect on the diagonal is below
    // the rounding of its entries (apq^2 <= 2^-106 |app aqq|) or of the
    // matrix (apq^2 <= 1e-30 |A|_F^2 / n^2) is skipped; a sweep without a
    // rotation ends the iteration.  A skipped pair (and every pair of a
    // converged group) applies the identity rotation, bit for bit no
    // change, so both groups of a warp follow the same path.
    const double tiny = 1e-30 * tot / (double(n) * n);
    bool rotated = false;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = A[p + n * q];
        double app = A[p + n * p], aqq = A[q + n * q];
        const double a2 = apq * apq;
        const bool skip = conv || apq == 0 ||
                          a2 <= 1.2325951644078310e-32 * fabs(app * aqq) || a2 <= tiny;
        double c = 1.0, s = 0.0;
        if (!skip) {
          rotated = true;
          double theta = (aqq - app) / (2 * apq);
          double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
          c = 1 / sqrt(t * t + 1);
          s = t * c;
        }
        g.sync();
        for (int r = g.lane; r < n; r += g.G) {
          double akp = A[r + n * p], akq = A[r + n * q];
          A[r + n * p] = c * akp - s * akq;
          A[r + n * q] = s * akp + c * akq;
        }
        g.sync();
        for (int r = g.lane; r < n; r += g.G) {
          double apk = A[p + n * r], aqk = A[q + n * r];
          A[p + n * r] = c * apk - s * aqk;
          A[q + n * r] = s * apk + c * aqk;
        }
        g.sync();
      }
    if (!__any_sync(g.warp, rotated)) break;
  }
  double v = CUDART_INF;
  for (int r = g.lane; r < n; r += g.G) {
    const double a = A[r + n * r];
    v = fmin(v, a);
    if (ev) ev[r] = a;
  }
  g.sync();
  return g.min(v);
}

__device__ __forceinline__ PsdCtx psd_ctx(const ConeSet &cs) {
  PsdCtx p;
  const int G = psd_group(cs.psd_nmax);
  int w = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  p.lane = threadIdx.x % G;
  p.g.lane = p.lane;
  p.g.G = G;
  p.g.mask = G == 32 ? 0xffffffffu : (0xffffu << (threadIdx.x & 16));
  p.valid = w < cs.n_psd;
  p.c = p.valid ? w : cs.n_psd - 1;
  p.n = cs.psd_n[p.c];
  p.t = p.n * (p.n + 1) / 2;
  p.off = cs.psd_off[p.c];
  p.inst = cs.psd_inst[p.c];
  if (p.valid && !active_inst(cs, p.inst)) p.valid = false;
  p.g.warp = __ballot_sync(0xffffffffu, p.valid);
  return p;
}
__device__ __forceinline__ double *psd_smem(int nmax, int nmats) {
  extern __shared__ double smem[];
  int wib = threadIdx.x / psd_group(nmax);  // the group's slice
  return smem + (size_t)wib * nmats * nmax * nmax;
}

// coneops_psdtrianglecone.jl:79-142
__global__ void k_psd_update_scaling(ConeSet cs, const double *__restrict__ s,
                                     const double *__restrict__ z, int *scale_ok) {
  PsdCtx p = psd_ctx(cs);
  if (!p.valid) return;  // the whole group shares p.valid
  int n = p.n, nm = cs.psd_nmax, nn = nm * nm;
  double *L1 = psd_smem(nm, 7), *L2 = L1 + nn, *M = L2 + nn, *V = M + nn,
         *T = V + nn, *S = T + 2 * nn;
  for (int e = p.lane; e < n * n; e += p.g.G) L1[e] = L2[e] = 0;
  p.g.sync();
  svec_to_mat(n, s + p.off, L1, p.g);
  svec_to_mat(n, z + p.off, L2, p.g);
  p.g.sync();
  bool ok1 = warp_chol(n, L1, p.g);
  bool ok2 = warp_chol(n, L2, p.g);
  p.g.warp = __ballot_sync(p.g.warp, ok1 && ok2);  // groups going on to the SVD
  if (!(ok1 && ok2)) {
    if (p.lane == 0) scale_ok[p.inst] = 0;
    return;
  }
  mm(n, L2, true, L1, false, M, p.g);  // M = L2' L1
  warp_svd(n, M, V, S, T, p.g);        // M <- U
  double *R = cs.psd_R + (size_t)p.c * nn, *Ri = cs.psd_Rinv + (size_t)p.c * nn;
  double *lam = cs.psd_lam + (size_t)p.c * nm;
  // R = L1 V Lis ; Rinv = Lis U' L2'
  for (int e = p.lane; e < n * n; e += p.g.G) {
    int i = e % n, j = e / n;
    double t = 0, u = 0;
    for (int k = 0; k < n; ++k) {
      t += L1[i + n * k] * V[k + n * j];
      u += M[k + n * i] * L2[j + n * k];
    }
    R[e] = t * (1.0 / sqrt(S[j]));
    Ri[e] = (1.0 / sqrt(S[i])) * u;
  }
  for (int r = p.lane; r < n; r += p.g.G) lam[r] = S[r];
}

// y = a*op(Rx)... helper: Y = Rx' X Rx (trans=false) or Rx X Rx' (trans=true)
__device__ void psd_wmul(int n, const double *Rx, bool trans, const double *X, double *Y,
                         double *T, const PsdGrp &g) {
  if (trans) {
    mm(n, X, false, Rx, true, T, g);   // T = X Rx'
    mm(n, Rx, false, T, false, Y, g);  // Y = Rx T
  } else {
    mm(n, Rx, true, X, false, T, g);   // T = Rx' X
    mm(n, T, false, Rx, false, Y, g);  // Y = T Rx
  }
}

// ================================================================ refresh
// SOC dense Hs entry (row r <= col c), coneops_socone.jl:453-490
__device__ __forceinline__ double soc_dense_hs(const double *w, int r, int c, double e2) {
  double v;
  if (r == 0 && c == 0) {
    const double s2 = 1.4142135623730951;
    v = (s2 * w[0] - 1.0) * (s2 * w[0] + 1.0);
  } else {
    v = 2 * w[r] * w[c];
    if (r == c) v += 1.0;
  }
  return v * e2;
}
// symmetric Kronecker entry of A (x)_s A at svec (row=(i,j), col=(k,l)),
// coneops_psdtrianglecone.jl:509-547
__device__ __forceinline__ double skron_entry(const double *A, int n, int i, int j, int k,
                                              int l) {
  const double sqrt2 = 1.4142135623730951;
  bool ij = (i == j), kl = (k == l);
  double Ajl = A[j + n * l], Ajk = A[j + n * k];
  if (!ij && !kl) return A[i + n * k] * Ajl + A[i + n * l] * Ajk;
  if (ij && !kl) return sqrt2 * Ajl * Ajk;
  if (!ij && kl) return sqrt2 * A[i + n * l] * Ajk;
  return Ajl * Ajl;
}
__device__ __forceinline__ void tri_coord(int k, int &row, int &col) {
  col = (int)((sqrt(8.0 * k + 1.0) - 1.0) * 0.5);
  while ((col + 1) * (col + 2) / 2 <= k) ++col;
  while (col * (col + 1) / 2 > k) --col;
  row = k - col * (col + 1) / 2;
}

__global__ void k_nn_refresh(ConeSet cs, const int *__restrict__ pos, double *kv) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= cs.n_nn) return;
  if (!active_row(cs, cs.nn_begin + e)) return;
  double w = cs.nn_w[e];
  kv[pos[e]] = -(w * w);
}

template <int G>
__global__ void k_soc_refresh(ConeSet cs, KKTMapDev map, double *kv) {
  SocCtx<G> ctx(cs);
  if (!ctx.valid) return;
  int r = ctx.off - cs.soc_begin;
  const double *w = cs.soc_w + r;
  double eta = cs.soc_eta[ctx.c], e2 = eta * eta;
  if (cs.soc_sparse[ctx.c]) {
    double d = cs.soc_d[ctx.c];
    SOC_FOR(i) {
      double hd = (i == 0) ? e2 * d : e2;
      kv[map.socs_diag[r + i]] = -hd;
      const int *uv = map.socs_uv + 4 * (size_t)(r + i);
      double vv = -e2 * cs.soc_v[r + i], uu = -e2 * cs.soc_u[r + i];
      kv[uv[0]] = vv;
      kv[uv[1]] = vv;
      kv[uv[2]] = uu;
      kv[uv[3]] = uu;
    }
    if (ctx.lane == 0) {
      kv[map.socs_D[2 * ctx.c]] = -e2;
      kv[map.socs_D[2 * ctx.c + 1]] = e2;
    }
  } else {
    int t = ctx.dim * (ctx.dim + 1) / 2;
    const int *pp = map.socd_pos + 2 * (size_t)map.socd_off[ctx.c];
    for (int k = ctx.lane; k < t; k += G) {
      int row, col;
      tri_coord(k, row, col);
      double v = -soc_dense_hs(w, row, col, e2);
      kv[pp[2 * k]] = v;
      if (pp[2 * k + 1] >= 0) kv[pp[2 * k + 1]] = v;
    }
  }
}

__global__ void k_nonsym_refresh(ConeSet cs, int nc, const int *inst, const double *Hs,
                                 const int *pos, double *kv) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  if (!active_inst(cs, inst[c])) return;
  const double *H = Hs + 9 * c;
  // triu entries in pack order: (0,0),(0,1),(1,1),(0,2),(1,2),(2,2)
  const int ri[6] = {0, 0, 1, 0, 1, 2}, ci[6] = {0, 1, 1, 2, 2, 2};
  for (int k = 0; k < 6; ++k) {
    double v = -H[ri[k] + 3 * ci[k]];
    kv[pos[12 * c + 2 * k]] = v;
    int q = pos[12 * c + 2 * k + 1];
    if (q >= 0) kv[q] = v;
  }
}

__global__ void k_psd_refresh(ConeSet cs, KKTMapDev map, double *kv) {
  PsdCtx p = psd_ctx(cs);
  if (!p.valid) return;
  int n = p.n, nm = cs.psd_nmax, nn = nm * nm;
  double *A = psd_smem(nm, 1);
  const double *R = cs.psd_R + (size_t)p.c * nn;
  mm(n, R, false, R, true, A, p.g);  // A = R R'
  int tt = p.t * (p.t + 1) / 2;
  const int *pp = map.psd_pos + 2 * (size_t)map.psd_off[p.c];
  for (int e = p.lane; e < tt; e += p.g.G) {
    int row, col;
    tri_coord(e, row, col);  // svec indices (row <= col)
    int i, j, k, l;
    tri_coord(row, i, j);
    tri_coord(col, k, l);
    double v = -skron_entry(A, n, i, j, k, l);
    kv[pp[2 * e]] = v;
    if (pp[2 * e + 1] >= 0) kv[pp[2 * e + 1]] = v;
  }
}

// get_Hs! into reference-layout blocks (used by the cone-level ABI only)
__global__ void k_nn_get_hs(ConeSet cs, const int *blk, double *Hs) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= cs.n_nn) return;
  double w = cs.nn_w[e];
  Hs[blk[e]] = w * w;
}
template <int G>
__global__ void k_soc_get_hs(ConeSet cs, const int *blk, double *Hs) {
  SocCtx<G> ctx(cs);
  if (!ctx.valid) return;
  int r = ctx.off - cs.soc_begin;
  const double *w = cs.soc_w + r;
  double eta = cs.soc_eta[ctx.c], e2 = eta * eta;
  double *out = Hs + blk[ctx.c];
  if (cs.soc_sparse[ctx.c]) {
    SOC_FOR(i) out[i] = (i == 0) ? e2 * cs.soc_d[ctx.c] : e2;
  } else {
    int t = ctx.dim * (ctx.dim + 1) / 2;
    for (int k = ctx.lane; k < t; k += G) {
      int row, col;
      tri_coord(k, row, col);
      out[k] = soc_dense_hs(w, row, col, e2);
    }
  }
}
__global__ void k_nonsym_get_hs(int nc, const double *Hsd, const int *blk, double *Hs) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const double *H = Hsd + 9 * c;
  double *o = Hs + blk[c];
  o[0] = H[0];
  o[1] = H[3];
  o[2] = H[4];
  o[3] = H[6];
  o[4] = H[7];
  o[5] = H[8];
}
__global__ void k_psd_get_hs(ConeSet cs, const int *blk, double *Hs) {
  PsdCtx p = psd_ctx(cs);
  if (!p.valid) return;
  int n = p.n, nm = cs.psd_nmax, nn = nm * nm;
  double *A = psd_smem(nm, 1);
  const double *R = cs.psd_R + (size_t)p.c * nn;
  mm(n, R, false, R, true, A, p.g);
  int tt = p.t * (p.t + 1) / 2;
  double *o = Hs + blk[p.c];
  for (int e = p.lane; e < tt; e += p.g.G) {
    int row, col, i, j, k, l;
    tri_coord(e, row, col);
    tri_coord(row, i, j);
    tri_coord(col, k, l);
    o[e] = skron_entry(A, n, i, j, k, l);
  }
}

// ================================================================= mul_Hs
__global__ void k_zero_fill(ConeSet cs, double *y) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= cs.n_zero) return;
  int g = cs.zero_begin + e;
  if (!active_row(cs, g)) return;
  y[g] = 0.0;
}
__global__ void k_nn_mul_hs(ConeSet cs, double *y, const double *__restrict__ x) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= cs.n_nn) return;
  int g = cs.nn_begin + e;
  if (!active_row(cs, g)) return;
  double w = cs.nn_w[e];
  y[g] = w * (w * x[g]);
}
template <int G>
__global__ void k_soc_mul_hs(ConeSet cs, double *y_, const double *__restrict__ x_) {
  SocCtx<G> ctx(cs);
  int r = ctx.off - cs.soc_begin;
  const double *w = cs.soc_w + r, *x = x_ + ctx.off;
  double t = 0;
  SOC_FOR(i) t += w[i] * x[i];
  double c = 2 * group_sum<G>(t);
  if (!ctx.valid) return;
  double eta = cs.soc_eta[ctx.c], e2 = eta * eta;
  double *y = y_ + ctx.off;
  SOC_FOR(i) {
    double v = (i == 0) ? -x[0] : x[i];
    y[i] = (v + c * w[i]) * e2;
  }
}
__global__ void k_nonsym_mul_hs(ConeSet cs, int nc, int begin, const int *inst,
                                const double *Hs, double *y, const double *x) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  if (!active_inst(cs, inst[c])) return;
  const double *H = Hs + 9 * c;
  const double *xv = x + begin + 3 * c;
  double x0 = xv[0], x1 = xv[1], x2 = xv[2];
  double *yv = y + begin + 3 * c;
  for (int i = 0; i < 3; ++i) yv[i] = H[i] * x0 + H[i + 3] * x1 + H[i + 6] * x2;
}
__global__ void k_psd_mul_hs(ConeSet cs, double *y, const double *__restrict__ x) {
  PsdCtx p = psd_ctx(cs);
  if (!p.valid) return;
  int n = p.n, nm = cs.psd_nmax, nn = nm * nm;
  double *X = psd_smem(nm, 3), *Y = X + nn, *T = Y + nn;
  const double *R = cs.psd_R + (size_t)p.c * nn;
  svec_to_mat(n, x + p.off, X, p.g);
  p.g.sync();
  psd_wmul(n, R, false, X, Y, T, p.g);  // Y = R' X R   (W x)
  mat_to_svec(n, Y, T, p.g);            // svec round trip of W x
  p.g.sync();
  svec_to_mat(n, T, Y, p.g);
  p.g.sync();
  psd_wmul(n, R, true, Y, X, T, p.g);   // X = R Y R'   (W^T W x)
  mat_to_svec(n, X, y + p.off, p.g);
}

// ============================================================== affine_ds
// kNNRows rows per thread (a block covers kNNRows * blockDim consecutive
// rows, row k * blockDim + threadIdx of its range): the loads of all of a
// thread's rows are issued before the first store.
__global__ void k_nn_affine_ds(ConeSet cs, double *ds) {
  const int base = blockIdx.x * blockDim.x * kNNRows + threadIdx.x;
  double l[kNNRows];
  bool on[kNNRows];
#pragma unroll
  for (int k = 0; k < kNNRows; ++k) {
    const int e = base + k * blockDim.x;
    on[k] = e < cs.n_nn && active_row(cs, cs.nn_begin + e);
    l[k] = on[k] ? cs.nn_lambda[e] : 0.0;
  }
#pragma unroll
  for (int k = 0; k < kNNRows; ++k)
    if (on[k]) ds[cs.nn_begin + base + k * blockDim.x] = l[k] * l[k];
}
template <int G>
__global__ void k_soc_affine_ds(ConeSet cs, double *ds_) {
  SocCtx<G> ctx(cs);
  int r = ctx.off - cs.soc_begin;
  const double *l = cs.soc_lambda + r;
  double t = 0;
  SOC_FOR(i) t += l[i] * l[i];
  t = group_sum<G>(t);
  if (!ctx.valid) return;
  double *ds = ds_ + ctx.off;
  double l0 = l[0];
  SOC_FOR(i) ds[i] = (i == 0) ? t : (l0 * l[i] + l0 * l[i]);
}
__global__ void k_nonsym_copy(ConeSet cs, int nc, int begin, const int *inst, double *dst,
                              const double *src) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 3 * nc) return;
  if (!active_inst(cs, inst[e / 3])) return;
  dst[begin + e] = src[begin + e];
}
__global__ void k_psd_affine_ds(ConeSet cs, double *ds) {
  PsdCtx p = psd_ctx(cs);
  if (!p.valid) return;
  const double *lam = cs.psd_lam + (size_t)p.c * cs.psd_nmax;
  for (int k = p.lane; k < p.t; k += p.g.G) {
    int row, col;
    tri_coord(k, row, col);
    ds[p.off + k] = (row == col) ? lam[row] * lam[row] : 0.0;
  }
}

// ======================================================= combined_ds_shift
// symmetric cones: shift = (W^{-T} ds) o (W dz) - sigma*mu*e
// (coneops_defaults.jl:335-368); step_z/step_s are not written back.
__global__ void k_nn_combined(ConeSet cs, double *shift, const double *__restrict__ dz,
                              const double *__restrict__ ds, const double *sm) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= cs.n_nn) return;
  int g = cs.nn_begin + e;
  int inst = row_instance(cs, g);
  if (!active_inst(cs, inst)) return;
  double w = cs.nn_w[e];
  double wz = dz[g] * w, ws = ds[g] / w;
  shift[g] = ws * wz - sm[inst];
}
template <int G>
__global__ void k_soc_combined(ConeSet cs, double *shift_, const double *__restrict__ dz_,
                               const double *__restrict__ ds_, const double *sm) {
  SocCtx<G> ctx(cs);
  int r = ctx.off - cs.soc_begin;
  const double *w = cs.soc_w + r, *dz = dz_ + ctx.off, *ds = ds_ + ctx.off;
  double eta = cs.soc_eta[ctx.c], w0 = w[0];
  double zz = soc_tail_dot<G>(w, dz, ctx);
  double zs = soc_tail_dot<G>(w, ds, ctx);
  double cz = dz[0] + zz / (1 + w0);
  double csn = -ds[0] + zs / (1 + w0);
  // Wz and Ws elements, then circ
  double wz0 = eta * (w0 * dz[0] + zz);
  double ws0 = (1 / eta) * (w0 * ds[0] - zs);
  double dot = 0;
  SOC_FOR(i) {
    double a = (i == 0) ? wz0 : eta * (dz[i] + cz * w[i]);
    double b = (i == 0) ? ws0 : (1 / eta) * (ds[i] + csn * w[i]);
    dot += a * b;
  }
  dot = group_sum<G>(dot);
  if (!ctx.valid) return;
  double *sh = shift_ + ctx.off;
  double smv = sm[ctx.inst];
  SOC_FOR(i) {
    if (i == 0) {
      sh[0] = dot - smv;
    } else {
      double a = eta * (dz[i] + cz * w[i]);
      double b = (1 / eta) * (ds[i] + csn * w[i]);
      sh[i] = ws0 * a + wz0 * b;
    }
  }
}
// asymmetric: shift = grad*sigma*mu - eta(3rd order correction)
template <class Ops>
__global__ void __launch_bounds__(128, 8) k_nonsym_combined(ConeSet cs, NonsymArgs<Ops> a, double *shift,
                                  const double *__restrict__ dz,
                                  const double *__restrict__ ds, const double *sm) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.n) return;
  int inst = a.inst[c];
  if (!active_inst(cs, inst)) return;
  double pa = a.alpha ? a.alpha[c] : 0.0;
  M3 Hd, L;
  for (int i = 0; i < 9; ++i) Hd.a[i] = a.Hd[9 * c + i];
  const double *zs = a.zs + 3 * c;
  double z[3] = {zs[0], zs[1], zs[2]};
  int b = a.begin + 3 * c;
  double v[3] = {dz[b], dz[b + 1], dz[b + 2]};
  double dsv[3] = {ds[b], ds[b + 1], ds[b + 2]};
  double eta[3] = {0, 0, 0};
  if (chol3(Hd, L)) {
    double u[3];
    chol3_solve(L, dsv, u);
    Ops::higher_correction(Hd, z, u, v, eta, pa);
  }
  double smv = sm[inst];
  for (int i = 0; i < 3; ++i) shift[b + i] = a.grad[3 * c + i] * smv - eta[i];
}
__global__ void k_psd_combined(ConeSet cs, double *shift, const double *__restrict__ dz,
                               const double *__restrict__ ds, const double *sm) {
  PsdCtx p = psd_ctx(cs);
  if (!p.valid) return;
  int n = p.n, nm = cs.psd_nmax, nn = nm * nm;
  double *X = psd_smem(nm, 5), *Z = X + nn, *S = Z + nn, *T = S + nn, *Y = T + nn;
  const double *R = cs.psd_R + (size_t)p.c * nn, *Ri = cs.psd_Rinv + (size_t)p.c * nn;
  for (int e = p.lane; e < n * n; e += p.g.G) X[e] = 0;
  p.g.sync();
  svec_to_mat(n, dz + p.off, X, p.g);
  p.g.sync();
  psd_wmul(n, R, false, X, Z, T, p.g);  // Z = R' dZ R   (W dz)
  svec_to_mat(n, ds + p.off, X, p.g);
  p.g.sync();
  psd_wmul(n, Ri, true, X, S, T, p.g);  // S = Ri dS Ri'  (W^{-T} ds)
  // svec round trip (the reference stores W dz and W^{-T} ds as svec)
  mat_to_svec(n, Z, Y, p.g);
  p.g.sync();
  svec_to_mat(n, Y, Z, p.g);
  mat_to_svec(n, S, Y, p.g);
  p.g.sync();
  svec_to_mat(n, Y, S, p.g);
  p.g.sync();
  // X = (S Z + Z S)/2
  for (int e = p.lane; e < n * n; e += p.g.G) {
    int i = e % n, j = e / n;
    double t = 0;
    for (int k = 0; k < n; ++k) t += S[i + n * k] * Z[k + n * j] + Z[i + n * k] * S[k + n * j];
    X[e] = 0.5 * t;
  }
  p.g.sync();
  double smv = sm[p.inst];
  double *out = shift + p.off;
  mat_to_svec(n, X, out, p.g);
  p.g.sync();
  for (int k = p.lane; k < n; k += p.g.G) out[(k + 1) * (k + 2) / 2 - 1] -= smv;
}

// ===================================================== ds_from_dz_offset
__global__ void k_nn_ds_offset(ConeSet cs, double *out, const double *__restrict__ ds,
                               const double *__restrict__ z) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= cs.n_nn) return;
  int g = cs.nn_begin + e;
  if (!active_row(cs, g)) return;
  out[g] = ds[g] / z[g];
}
// coneops_socone.jl:539-566
template <int G>
__global__ void k_soc_ds_offset(ConeSet cs, double *out_, const double *__restrict__ ds_,
                                const double *__restrict__ z_) {
  SocCtx<G> ctx(cs);
  int r = ctx.off - cs.soc_begin;
  const double *w = cs.soc_w + r, *l = cs.soc_lambda + r, *ds = ds_ + ctx.off,
               *z = z_ + ctx.off;
  double resz = soc_res(z[0], soc_tail_sq<G>(z, ctx));
  double l1ds1 = soc_tail_dot<G>(l, ds, ctx);
  double w1ds1 = soc_tail_dot<G>(w, ds, ctx);
  if (!ctx.valid) return;
  double eta = cs.soc_eta[ctx.c];
  double c = l[0] * ds[0] - l1ds1;
  double il = 1 / l[0];
  double *out = out_ + ctx.off;
  SOC_FOR(i) {
    double o;
    if (i == 0) {
      o = z[0] * (c / resz);
      o += eta * w1ds1;
    } else {
      o = -z[i] * (c / resz);
      o += eta * (ds[i] + w1ds1 / (1 + w[0]) * w[i]);
    }
    out[i] = o * il;
  }
}
__global__ void k_psd_ds_offset(ConeSet cs, double *out, const double *__restrict__ ds) {
  PsdCtx p = psd_ctx(cs);
  if (!p.valid) return;
  int n = p.n, nm = cs.psd_nmax, nn = nm * nm;
  double *X = psd_smem(nm, 4), *Z = X + nn, *T = Z + nn, *Y = T + nn;
  const double *R = cs.psd_R + (size_t)p.c * nn;
  const double *lam = cs.psd_lam + (size_t)p.c * nm;
  svec_to_mat(n, ds + p.off, Z, p.g);
  p.g.sync();
  for (int e = p.lane; e < n * n; e += p.g.G) {
    int i = e % n, j = e / n;
    X[e] = 2 * Z[e] / (lam[i] + lam[j]);
  }
  p.g.sync();
  // work stored as svec then re-expanded (as the reference does)
  mat_to_svec(n, X, Y, p.g);
  p.g.sync();
  svec_to_mat(n, Y, X, p.g);
  p.g.sync();
  psd_wmul(n, R, true, X, Z, T, p.g);  // Z = R X R'
  mat_to_svec(n, Z, out + p.off, p.g);
}

// ============================================================ step length
__global__ void k_nn_step(ConeSet cs, const double *__restrict__ dz,
                          const double *__restrict__ ds, const double *__restrict__ z,
                          const double *__restrict__ s, double *alpha) {
  if (cs.B == 1) {
    // one problem: kNNRows rows per thread (as k_nn_affine_ds), one
    // block-level reduction per kNNRows * blockDim rows
    const int base = blockIdx.x * blockDim.x * kNNRows + threadIdx.x;
    double a = CUDART_INF;
    if (active_inst(cs, 0)) {
      // all four vectors loaded in one round; the smallest ratio -x / dx
      // (dx < 0, x > 0) is selected by cross-multiplication, n / d < bn / bd
      // <=> n bd < bn d for positive denominators, and divided once
      double dzv[kNNRows], dsv[kNNRows], zv[kNNRows], sv[kNNRows];
#pragma unroll
      for (int k = 0; k < kNNRows; ++k) {
        const int e = base + k * blockDim.x;
        const bool in = e < cs.n_nn;
        dzv[k] = in ? dz[cs.nn_begin + e] : 0.0;
        dsv[k] = in ? ds[cs.nn_begin + e] : 0.0;
        zv[k] = in ? z[cs.nn_begin + e] : 0.0;
        sv[k] = in ? s[cs.nn_begin + e] : 0.0;
      }
      double bn = 1.0, bd = 0.0;  // best ratio bn / bd (bd = 0: none)
#pragma unroll
      for (int k = 0; k < kNNRows; ++k) {
        if (dzv[k] < 0 && (bd == 0.0 || zv[k] * bd < bn * -dzv[k])) {
          bn = zv[k];
          bd = -dzv[k];
        }
        if (dsv[k] < 0 && (bd == 0.0 || sv[k] * bd < bn * -dsv[k])) {
          bn = sv[k];
          bd = -dsv[k];
        }
      }
      if (bd != 0.0) a = bn / bd;
    }
    block_seg_min_nonneg(alpha, a == CUDART_INF ? -1 : 0, a);
    return;
  }
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  int inst = -1;
  double a = CUDART_INF;
  if (e < cs.n_nn) {
    int g = cs.nn_begin + e;
    inst = row_instance(cs, g);
    if (active_inst(cs, inst)) {
      double dzi = dz[g], dsi = ds[g];
      if (dzi < 0) a = fmin(a, -z[g] / dzi);
      if (dsi < 0) a = fmin(a, -s[g] / dsi);
      if (a == CUDART_INF) inst = -1;
    } else {
      inst = -1;
    }
  }
  seg_atomic_min_nonneg(alpha, inst, a);  // short per-instance segments
}

// coneops_socone.jl:745-814 with group reductions
template <int G>
__device__ double soc_step_component(const double *x, const double *y, double amax,
                                     const SocCtx<G> &ctx) {
  double x0 = x[0], y0 = y[0];
  double ysq = soc_tail_sq<G>(y, ctx);
  double xsq = soc_tail_sq<G>(x, ctx);
  double xy = soc_tail_dot<G>(x, y, ctx);
  if (x0 >= 0 && y0 < 0) amax = fmin(amax, -x0 / y0);
  double a = soc_res(y0, ysq);
  double b = 2 * (x0 * y0 - xy);
  double c = fmax(0.0, soc_res(x0, xsq));
  double d = b * b - 4 * a * c;
  if ((a > 0 && b > 0) || d < 0) return amax;
  if (a == 0) return amax;
  if (c == 0) return a >= 0 ? amax : 0.0;
  double t = (b >= 0) ? (-b - sqrt(d)) : (-b + sqrt(d));
  double r1 = (2 * c) / t, r2 = t / (2 * a);
  r1 = r1 < 0 ? kDMax : r1;
  r2 = r2 < 0 ? kDMax : r2;
  return fmin(amax, fmin(r1, r2));
}
template <int G>
__global__ void k_soc_step(ConeSet cs, const double *__restrict__ dz,
                           const double *__restrict__ ds, const double *__restrict__ z,
                           const double *__restrict__ s, double *alpha) {
  SocCtx<G> ctx(cs);
  double amax = alpha[ctx.inst];  // upper bound already there (atomic min target)
  double az = soc_step_component<G>(z + ctx.off, dz + ctx.off, amax, ctx);
  double as = soc_step_component<G>(s + ctx.off, ds + ctx.off, amax, ctx);
  if (cs.B == 1)
    block_seg_min_nonneg(alpha, (ctx.valid && ctx.lane == 0) ? ctx.inst : -1, fmin(az, as));
  else if (ctx.valid && ctx.lane == 0)
    atomic_min_nonneg(alpha + ctx.inst, fmin(az, as));
}
__global__ void k_psd_step(ConeSet cs, const double *__restrict__ dz,
                           const double *__restrict__ ds, double *alpha) {
  PsdCtx p = psd_ctx(cs);
  if (!p.valid) return;
  int n = p.n, nm = cs.psd_nmax, nn = nm * nm;
  double *X = psd_smem(nm, 4), *Y = X + nn, *T = Y + nn, *V = T + nn;
  const double *R = cs.psd_R + (size_t)p.c * nn, *Ri = cs.psd_Rinv + (size_t)p.c * nn;
  const double *lam = cs.psd_lam + (size_t)p.c * nm;
  double amax = alpha[p.inst];
  double res = amax;
  for (int side = 0; side < 2; ++side) {
    svec_to_mat(n, (side == 0 ? dz : ds) + p.off, X, p.g);
    p.g.sync();
    if (side == 0)
      psd_wmul(n, R, false, X, Y, T, p.g);  // W dz = R' dZ R
    else
      psd_wmul(n, Ri, true, X, Y, T, p.g);  // W^{-T} ds = Ri dS Ri'
    // svec round trip then scale by Lis both sides
    mat_to_svec(n, Y, V, p.g);
    p.g.sync();
    svec_to_mat(n, V, Y, p.g);
    p.g.sync();
    for (int e = p.lane; e < n * n; e += p.g.G) {
      int i = e % n, j = e / n;
      Y[e] *= (1.0 / sqrt(lam[i])) * (1.0 / sqrt(lam[j]));
    }
    p.g.sync();
    double gmin = warp_eig_min(n, Y, nullptr, p.g);
    double a = gmin < 0 ? fmin(1.0 / (-gmin), amax) : amax;
    res = fmin(res, a);
  }
  if (p.lane == 0) atomic_min_nonneg_filtered(alpha + p.inst, res);
}
// coneops_nonsymmetric_common.jl:5-34 backtracking, per cone
template <class Ops>
__global__ void k_nonsym_step(ConeSet cs, NonsymArgs<Ops> a, const double *__restrict__ dz,
                              const double *__restrict__ ds, const double *__restrict__ z,
                              const double *__restrict__ s, const double *astart,
                              double *alpha, double step, double amin) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  int inst = c < a.n ? a.inst[c] : -1;
  if (inst >= 0 && !active_inst(cs, inst)) inst = -1;
  double res = CUDART_INF;
  if (inst >= 0) {
    double pa = a.alpha ? a.alpha[c] : 0.0;
    int b = a.begin + 3 * c;
    double a0 = astart[inst];
    res = a0;
    for (int side = 0; side < 2; ++side) {
      const double *q = side == 0 ? z : s;
      const double *dq = side == 0 ? dz : ds;
      double al = a0, wq[3];
      while (true) {
        for (int i = 0; i < 3; ++i) wq[i] = q[b + i] + al * dq[b + i];
        bool ok = side == 0 ? Ops::dual_feasible(wq, pa) : Ops::primal_feasible(wq, pa);
        if (ok) break;
        if ((al *= step) < amin) {
          al = 0;
          break;
        }
      }
      res = fmin(res, al);
    }
  }
  if (cs.B == 1)
    block_seg_min_nonneg(alpha, inst, res);
  else if (inst >= 0)
    atomic_min_nonneg(alpha + inst, res);
}

// ================================================================ barrier
// Per-cone values go to cs.cone_tmp (soc | exp | pow | psd) and one block per
// instance sums them, with the nonnegative rows, in a fixed order, so the
// barrier of an instance does not depend on the rest of the batch.
template <int G>
__global__ void k_soc_barrier(ConeSet cs, const double *__restrict__ z_,
                              const double *__restrict__ s_, const double *__restrict__ dz_,
                              const double *__restrict__ ds_, const double *alpha,
                              const int *bt) {
  SocCtx<G> ctx(cs);
  double a = alpha[ctx.inst];
  const double *z = z_ + ctx.off, *s = s_ + ctx.off, *dz = dz_ + ctx.off,
               *ds = ds_ + ctx.off;
  double sq = 0, zq = 0;
  SOC_FOR(i) if (i > 0) {
    double si = s[i] + a * ds[i], zi = z[i] + a * dz[i];
    sq += si * si;
    zq += zi * zi;
  }
  sq = group_sum<G>(sq);
  zq = group_sum<G>(zq);
  if (!ctx.valid || !bt[ctx.inst] || ctx.lane != 0) return;
  double rs = soc_res(s[0] + a * ds[0], sq), rz = soc_res(z[0] + a * dz[0], zq);
  cs.cone_tmp[ctx.c] = (rs > 0 && rz > 0) ? -logsafe(rs * rz) / 2 : CUDART_INF;
}
template <class Ops>
__global__ void k_nonsym_barrier(ConeSet cs, NonsymArgs<Ops> a, int slot0,
                                 const double *__restrict__ z, const double *__restrict__ s,
                                 const double *__restrict__ dz, const double *__restrict__ ds,
                                 const double *alpha, const int *bt) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.n) return;
  int inst = a.inst[c];
  if (!active_inst(cs, inst) || !bt[inst]) return;
  double pa = a.alpha ? a.alpha[c] : 0.0;
  double al = alpha[inst];
  int b = a.begin + 3 * c;
  double cz[3], csv[3];
  for (int i = 0; i < 3; ++i) {
    cz[i] = z[b + i] + al * dz[b + i];
    csv[i] = s[b + i] + al * ds[b + i];
  }
  cs.cone_tmp[slot0 + c] = Ops::barrier_dual(cz, pa) + Ops::barrier_primal(csv, pa);
}
__global__ void k_psd_barrier(ConeSet cs, const double *__restrict__ z,
                              const double *__restrict__ s, const double *__restrict__ dz,
                              const double *__restrict__ ds, const double *alpha,
                              const int *bt) {
  PsdCtx p = psd_ctx(cs);
  if (!p.valid || !bt[p.inst]) return;
  int n = p.n, nm = cs.psd_nmax;
  double *Q = psd_smem(nm, 2), *q = Q + nm * nm;
  double a = alpha[p.inst];
  double total = 0;
  for (int side = 0; side < 2; ++side) {
    const double *x = side == 0 ? z : s, *dx = side == 0 ? dz : ds;
    for (int k = p.lane; k < p.t; k += p.g.G) q[k] = x[p.off + k] + a * dx[p.off + k];
    p.g.sync();
    svec_to_mat(n, q, Q, p.g);
    p.g.sync();
    bool ok = warp_chol(n, Q, p.g);
    double ld;
    if (ok) {
      double t = 0.0;
      for (int r = p.lane; r < n; r += p.g.G) t += log(Q[r + n * r]);
      ld = 2 * p.g.sum(t);
    } else {
      ld = CUDART_INF;
    }
    total -= ld;
    p.g.sync();
  }
  if (p.lane == 0) cs.cone_tmp[cs.n_soc + cs.n_exp + cs.n_pow + p.c] = total;
}
// bar[i] += nonneg rows + sum of the instance's per-cone values (fixed order)
__global__ void k_barrier_inst(ConeSet cs, const double *__restrict__ z,
                               const double *__restrict__ s, const double *__restrict__ dz,
                               const double *__restrict__ ds, const double *alpha,
                               const int *bt, double *bar) {
  const int i = blockIdx.x;
  if (!active_inst(cs, i) || !bt[i]) return;
  __shared__ double red[32];
  const double a = alpha[i];
  double t = 0;
  const int e0 = cs.rng_nn[2 * i], en = cs.rng_nn[2 * i + 1];
  for (int e = threadIdx.x; e < en; e += blockDim.x) {
    const int g = cs.nn_begin + e0 + e;
    const double si = s[g] + a * ds[g], zi = z[g] + a * dz[g];
    t -= logsafe(si * zi);
  }
  t = warp_sum(t);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
    const int o_exp = cs.n_soc, o_pow = o_exp + cs.n_exp, o_psd = o_pow + cs.n_pow;
    for (int c = 0; c < cs.rng_soc[2 * i + 1]; ++c) tot += cs.cone_tmp[cs.rng_soc[2 * i] + c];
    for (int c = 0; c < cs.rng_exp[2 * i + 1]; ++c)
      tot += cs.cone_tmp[o_exp + cs.rng_exp[2 * i] + c];
    for (int c = 0; c < cs.rng_pow[2 * i + 1]; ++c)
      tot += cs.cone_tmp[o_pow + cs.rng_pow[2 * i] + c];
    for (int c = 0; c < cs.rng_psd[2 * i + 1]; ++c)
      tot += cs.cone_tmp[o_psd + cs.rng_psd[2 * i] + c];
    bar[i] += tot;
  }
}

// ================================================================ margins
template <int G>
__global__ void k_soc_margins(ConeSet cs, const double *__restrict__ z_) {
  SocCtx<G> ctx(cs);
  const double *z = z_ + ctx.off;
  double t = soc_tail_sq<G>(z, ctx);
  if (!ctx.valid || ctx.lane != 0) return;
  cs.cone_tmp[ctx.c] = z[0] - sqrt(t);
}
__global__ void k_psd_margins(ConeSet cs, const double *__restrict__ z) {
  PsdCtx p = psd_ctx(cs);
  if (!p.valid) return;
  int n = p.n, nm = cs.psd_nmax;
  double *Z = psd_smem(nm, 2), *ev = Z + nm * nm;
  const int slot = cs.n_soc + cs.n_exp + cs.n_pow + p.c;
  p.g.warp = __ballot_sync(p.g.warp, n != 0);  // groups going on to the eigenvalues
  if (n == 0) {
    // an empty cone: (floatmax, 0), coneops_psdtrianglecone.jl:16-19
    if (p.lane == 0) {
      cs.cone_tmp[slot] = kDMax;
      cs.cone_tmp2[slot] = 0.0;
    }
    return;
  }
  svec_to_mat(n, z + p.off, Z, p.g);
  p.g.sync();
  double mn = warp_eig_min(n, Z, ev, p.g);
  double pos = 0.0;
  for (int r = p.lane; r < n; r += p.g.G) pos += ev[r] > 0 ? ev[r] : 0.0;
  pos = p.g.sum(pos);
  if (p.lane == 0) {
    cs.cone_tmp[slot] = mn;
    cs.cone_tmp2[slot] = pos;
  }
}
// margins of each instance: minimum over its cones, sum of the positive
// parts (coneops_nncone.jl:19-39, coneops_socone.jl:310-319,
// coneops_psdtrianglecone.jl:10-28), fixed summation order
__global__ void k_margins_inst(ConeSet cs, const double *__restrict__ z, double *amin,
                               double *asum) {
  const int i = blockIdx.x;
  if (!active_inst(cs, i)) return;
  __shared__ double rmin[32], rsum[32];
  double mn = kDMax, sm = 0;
  const int e0 = cs.rng_nn[2 * i], en = cs.rng_nn[2 * i + 1];
  for (int e = threadIdx.x; e < en; e += blockDim.x) {
    const double v = z[cs.nn_begin + e0 + e];
    mn = fmin(mn, v);
    sm += v > 0 ? v : 0.0;
  }
  mn = warp_min(mn);
  sm = warp_sum(sm);
  if ((threadIdx.x & 31) == 0) {
    rmin[threadIdx.x >> 5] = mn;
    rsum[threadIdx.x >> 5] = sm;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = kDMax, t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      m = fmin(m, rmin[w]);
      t += rsum[w];
    }
    for (int c = 0; c < cs.rng_soc[2 * i + 1]; ++c) {
      const double a = cs.cone_tmp[cs.rng_soc[2 * i] + c];
      m = fmin(m, a);
      t += fmax(0.0, a);
    }
    const int o_psd = cs.n_soc + cs.n_exp + cs.n_pow;
    for (int c = 0; c < cs.rng_psd[2 * i + 1]; ++c) {
      const int slot = o_psd + cs.rng_psd[2 * i] + c;
      m = fmin(m, cs.cone_tmp[slot]);
      t += cs.cone_tmp2[slot];
    }
    amin[i] = m;
    asum[i] = t;
  }
}

// ============================================ shifts, unit init, identity
__global__ void k_zero_shift(ConeSet cs, double *z, int pd) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= cs.n_zero) return;
  int g = cs.zero_begin + e;
  if (!active_row(cs, g)) return;
  if (pd == 0) z[g] = 0.0;
}
__global__ void k_nn_shift(ConeSet cs, double *z, const double *alpha) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= cs.n_nn) return;
  int g = cs.nn_begin + e;
  int inst = row_instance(cs, g);
  if (!active_inst(cs, inst)) return;
  z[g] += alpha[inst];
}
__global__ void k_soc_shift(ConeSet cs, double *z, const double *alpha) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cs.n_soc) return;
  int inst = cs.soc_inst[c];
  if (!active_inst(cs, inst)) return;
  z[cs.soc_off[c]] += alpha[inst];
}
__global__ void k_psd_shift(ConeSet cs, double *z, const double *alpha) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cs.n_psd) return;
  int inst = cs.psd_inst[c];
  if (!active_inst(cs, inst)) return;
  int n = cs.psd_n[c];
  for (int k = 1; k <= n; ++k) z[cs.psd_off[c] + k * (k + 1) / 2 - 1] += alpha[inst];
}
__global__ void k_unit_init(ConeSet cs, double *z, double *s) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= cs.m_total) return;
  if (!active_row(cs, g)) return;
  double v = 0.0;
  if (g >= cs.nn_begin && g < cs.nn_begin + cs.n_nn) v = 1.0;
  s[g] = v;
  z[g] = v;
}
__global__ void k_unit_init_cones(ConeSet cs, double *z, double *s) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  int total = cs.n_soc + cs.n_exp + cs.n_pow + cs.n_psd;
  if (c >= total) return;
  if (c < cs.n_soc) {
    if (!active_inst(cs, cs.soc_inst[c])) return;
    int o = cs.soc_off[c];
    s[o] += 1.0;
    z[o] += 1.0;
    return;
  }
  c -= cs.n_soc;
  if (c < cs.n_exp) {
    if (!active_inst(cs, cs.exp_inst[c])) return;
    double v[3];
    ExpOps::unit_init(v, 0);
    int b = cs.exp_begin + 3 * c;
    for (int i = 0; i < 3; ++i) s[b + i] = z[b + i] = v[i];
    return;
  }
  c -= cs.n_exp;
  if (c < cs.n_pow) {
    if (!active_inst(cs, cs.pow_inst[c])) return;
    double v[3];
    PowOps::unit_init(v, cs.pow_alpha[c]);
    int b = cs.pow_begin + 3 * c;
    for (int i = 0; i < 3; ++i) s[b + i] = z[b + i] = v[i];
    return;
  }
  c -= cs.n_pow;
  if (!active_inst(cs, cs.psd_inst[c])) return;
  int n = cs.psd_n[c];
  for (int k = 1; k <= n; ++k) {
    int idx = cs.psd_off[c] + k * (k + 1) / 2 - 1;
    s[idx] += 1.0;
    z[idx] += 1.0;
  }
}
__global__ void k_identity(ConeSet cs) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < cs.n_nn) {
    if (active_row(cs, cs.nn_begin + t)) cs.nn_w[t] = 1.0;
  }
  if (t < cs.soc_rows) {
    int g = cs.soc_begin + t;
    if (active_row(cs, g)) {
      // first element of its cone?  soc rows are contiguous per cone; a row is
      // a head iff it equals the cone's offset -- found by the cone loop below
      cs.soc_w[t] = 0.0;
      cs.soc_u[t] = 0.0;
      cs.soc_v[t] = 0.0;
    }
  }
}
__global__ void k_identity_cones(ConeSet cs) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < cs.n_soc) {
    if (!active_inst(cs, cs.soc_inst[c])) return;
    int r = cs.soc_off[c] - cs.soc_begin;
    cs.soc_w[r] = 1.0;
    cs.soc_eta[c] = 1.0;
    if (cs.soc_sparse[c]) {
      cs.soc_d[c] = 0.5;
      cs.soc_u[r] = sqrt(0.5);
    }
    return;
  }
  c -= cs.n_soc;
  if (c < cs.n_psd) {
    if (!active_inst(cs, cs.psd_inst[c])) return;
    int nm = cs.psd_nmax, n = cs.psd_n[c];
    double *R = cs.psd_R + (size_t)c * nm * nm, *Ri = cs.psd_Rinv + (size_t)c * nm * nm;
    for (int e = 0; e < n * n; ++e) {
      double v = (e % n == e / n) ? 1.0 : 0.0;
      R[e] = v;
      Ri[e] = v;
    }
  }
}

// ======================================================== SOC tile kernels
// One block per tile of consecutive small cones (dim <= kSocTileMaxDim), one
// thread per cone.  The tile's rows are staged in shared memory by coalesced
// loads, each thread runs its cone's formulas over its own rows (the
// formulas of the lane-group kernels above, with their sums in the same
// butterfly order, tree16), and results leave through coalesced stores of
// the rows whose cone is active.
// Shared rows keep their global order (tsk is the identity): with the mixed
// cone dimensions of real tiles the threads' strides are irregular and no
// fixed skew spreads the banks better (about 2.2 wavefronts per access
// either way), while one word per 16 rows made uniform dim-10 tiles 5-way
// conflicted.
__device__ __forceinline__ int tsk(int i) { return i; }
// words of one staged array for a tile of `rows` rows
__host__ __device__ __forceinline__ int tile_words(int rows) { return rows; }
// Sum of a cone's per-element terms in the order of the lane-group kernels'
// butterfly reduction (pairs at distance 8, 4, 2, 1 over 16 leaves, leaves
// from the cone's dimension on are +0): for dim <= 16 this is the same
// result, bit for bit, as group_sum<G> for every G >= dim.  leaf(l) is the
// partial a group lane l would hold (0.0 + its term).
template <class F>
__device__ __forceinline__ double tree16(int d, F leaf) {
  double p[8];
#pragma unroll
  for (int l = 0; l < 8; ++l) {
    double a = l < d ? leaf(l) : 0.0;
    double b = l + 8 < d ? leaf(l + 8) : 0.0;
    p[l] = a + b;
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1)
#pragma unroll
    for (int l = 0; l < o; ++l) p[l] = p[l] + p[l + o];
  return p[0];
}
struct SocTileCtx {
  int c0, nc, r0, nrows;  // tile: cones [c0, c0+nc), global rows [r0, r0+nrows)
  int k, c, off, dim, inst;  // this thread's cone (k < nc) and its rows in the tile
  bool valid;
  int words;              // words of one staged array
  unsigned short *rcone;  // [rows per tile] local cone of each tile row
  unsigned char *ok;      // [cones per tile] cone's rows are written back
};

// Shared layout: `narr` staged arrays of tile_words(rows) doubles, then
// rcone, ok.
__device__ __forceinline__ double *tile_arr(int a, int words) {
  extern __shared__ __align__(16) double tile_smem[];
  return tile_smem + (size_t)a * words;
}
__device__ __forceinline__ SocTileCtx soc_tile_ctx(const ConeSet &cs, const int *tiles,
                                                   int trows, int narr) {
  SocTileCtx t;
  t.words = tile_words(trows);
  int b = blockIdx.x;
  t.c0 = tiles[2 * b];
  int c1 = tiles[2 * b + 1];
  t.nc = c1 - t.c0;
  t.r0 = cs.soc_off[t.c0];
  t.nrows = cs.soc_off[c1 - 1] + cs.soc_dim[c1 - 1] - t.r0;
  t.rcone = reinterpret_cast<unsigned short *>(tile_arr(narr, t.words));
  t.ok = reinterpret_cast<unsigned char *>(t.rcone + trows);
  t.k = threadIdx.x;
  t.valid = t.k < t.nc;
  t.c = t.valid ? t.c0 + t.k : t.c0;
  t.off = cs.soc_off[t.c] - t.r0;
  t.dim = cs.soc_dim[t.c];
  t.inst = cs.soc_inst[t.c];
  if (t.valid) {
    for (int i = 0; i < t.dim; ++i) t.rcone[t.off + i] = (unsigned short)t.k;
    t.ok[t.k] = 0;
    if (!active_inst(cs, t.inst)) t.valid = false;
  }
  return t;
}
// Staging copies go global -> shared with cp.async (no register round trip),
// so every thread has all of its copies in flight at once; tile_loaded()
// waits for this thread's copies and the block barrier that follows makes
// them visible to the block.
__device__ __forceinline__ void tile_load(double *dst, const double *__restrict__ src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst + tsk(i)));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src + i)
                 : "memory");
  }
}
__device__ __forceinline__ void tile_loaded() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}
__device__ __forceinline__ void tile_store(double *dst, const double *src, int n,
                                           const SocTileCtx &t) {
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    if (t.ok[t.rcone[i]]) dst[i] = src[tsk(i)];
}

// update_scaling! for tiled cones (coneops_socone.jl:372-451; sparse d/u/v of
// coneops_socone_gpu.jl:338-470).  w and lambda overwrite the staged s and z
// rows in place (each thread only reads its own rows).
__global__ void k_soc_tile_update_scaling(ConeSet cs, const int *tiles, int trows, const double *__restrict__ s_,
                                          const double *__restrict__ z_, int *scale_ok) {
  SocTileCtx t = soc_tile_ctx(cs, tiles, trows, 4);
  double *S = tile_arr(0, t.words), *Z = tile_arr(1, t.words), *U = tile_arr(2, t.words), *V = tile_arr(3, t.words);
  tile_load(S, s_ + t.r0, t.nrows);
  tile_load(Z, z_ + t.r0, t.nrows);
  tile_loaded();
  __syncthreads();
  bool sparse_tile = false;
  if (t.valid) {
    const int o = t.off, d = t.dim;
    double s0 = S[tsk(o)], z0 = Z[tsk(o)];
    double z1sq = tree16(d, [&](int l) {
      double zl = Z[tsk(o + l)];
      return l > 0 ? 0.0 + zl * zl : 0.0;
    });
    double s1sq = tree16(d, [&](int l) {
      double sl = S[tsk(o + l)];
      return l > 0 ? 0.0 + sl * sl : 0.0;
    });
    double zs = soc_res(z0, z1sq), ss = soc_res(s0, s1sq);
    double zscale = zs > 0.0 ? sqrt(zs) : 0.0;
    double sscale = ss > 0.0 ? sqrt(ss) : 0.0;
    bool fail = (zscale == 0.0 || sscale == 0.0);
    if (fail) zscale = sscale = 1.0;
    double eta = sqrt(sscale / zscale);
    const double isc = 1.0 / sscale, izc = 1.0 / zscale;
    double w1sq_a = tree16(d, [&](int l) {
      double wl = __dadd_rn(__dmul_rn(S[tsk(o + l)], isc), __dmul_rn(-Z[tsk(o + l)], izc));
      return l > 0 ? 0.0 + wl * wl : 0.0;
    });
    double w0pre = __dadd_rn(__dmul_rn(s0, isc), __dmul_rn(z0, izc));
    double wres = soc_res(w0pre, w1sq_a);
    double wscale = wres > 0.0 ? sqrt(wres) : 0.0;
    if (wscale == 0.0) {
      fail = true;
      wscale = 1.0;
    }
    const double iwc = 1.0 / wscale;
    double w1sq = tree16(d, [&](int l) {
      double wl = __dmul_rn(
          __dadd_rn(__dmul_rn(S[tsk(o + l)], isc), __dmul_rn(-Z[tsk(o + l)], izc)), iwc);
      return l > 0 ? 0.0 + wl * wl : 0.0;
    });
    double w0 = sqrt(1 + w1sq);
    double gamma = 0.5 * wscale;
    double c1 = __dmul_rn(__dadd_rn(gamma, __dmul_rn(z0, izc)), isc);
    double c2 = __dmul_rn(__dadd_rn(gamma, __dmul_rn(s0, isc)), izc);
    double inv = 1.0 / __dadd_rn(w0pre, 2 * gamma);
    double sc = sqrt(sscale * zscale);
    bool sparse = cs.soc_sparse[t.c] != 0;
    double u0 = 0, u1 = 0, v1 = 0, dd = 0;
    if (sparse) {
      double wsq = w0 * w0 + w1sq;
      double wsqinv = 1 / wsq;
      dd = wsqinv / 2;
      u0 = sqrt(wsq - dd);
      u1 = 2 * w0 / u0;
      v1 = sqrt(2 * (2 + wsqinv) / (2 * wsq - wsqinv));
    }
    if (fail) {
      scale_ok[t.inst] = 0;
    } else {
      for (int i = 1; i < d; ++i) {
        double si = S[tsk(o + i)], zi = Z[tsk(o + i)];
        double wi = __dmul_rn(__dadd_rn(__dmul_rn(si, isc), __dmul_rn(-zi, izc)), iwc);
        S[tsk(o + i)] = wi;
        Z[tsk(o + i)] = ((c1 * si + c2 * zi) * inv) * sc;
        if (sparse) {
          U[tsk(o + i)] = u1 * wi;
          V[tsk(o + i)] = v1 * wi;
        }
      }
      S[tsk(o)] = w0;
      Z[tsk(o)] = gamma * sc;
      if (sparse) {
        U[tsk(o)] = u0;
        V[tsk(o)] = 0.0;
      }
      cs.soc_eta[t.c] = eta;
      if (sparse) cs.soc_d[t.c] = dd;
      t.ok[t.k] = sparse ? 2 : 1;
    }
    sparse_tile = sparse;
  }
  sparse_tile = __syncthreads_or(sparse_tile);
  const int r = t.r0 - cs.soc_begin;
  tile_store(cs.soc_w + r, S, t.nrows, t);
  tile_store(cs.soc_lambda + r, Z, t.nrows, t);
  if (sparse_tile) {
    for (int i = threadIdx.x; i < t.nrows; i += blockDim.x)
      if (t.ok[t.rcone[i]] == 2) {
        cs.soc_u[r + i] = U[tsk(i)];
        cs.soc_v[r + i] = V[tsk(i)];
      }
  }
}

// mul_Hs for tiled cones: y = eta^2 (J x + 2 (w'x) w), J = diag(-1, 1, ...);
// y overwrites the staged x rows in place.
__global__ void k_soc_tile_mul_hs(ConeSet cs, const int *tiles, int trows, double *y_,
                                  const double *__restrict__ x_) {
  SocTileCtx t = soc_tile_ctx(cs, tiles, trows, 2);
  double *W = tile_arr(0, t.words), *X = tile_arr(1, t.words);
  tile_load(W, cs.soc_w + (t.r0 - cs.soc_begin), t.nrows);
  tile_load(X, x_ + t.r0, t.nrows);
  tile_loaded();
  __syncthreads();
  if (t.valid) {
    const int o = t.off, d = t.dim;
    double tt = tree16(d, [&](int l) { return 0.0 + W[tsk(o + l)] * X[tsk(o + l)]; });
    double c = 2 * tt;
    double eta = cs.soc_eta[t.c], e2 = eta * eta;
    for (int i = 0; i < d; ++i) {
      double xi = X[tsk(o + i)];
      double v = (i == 0) ? -xi : xi;
      X[tsk(o + i)] = (v + c * W[tsk(o + i)]) * e2;
    }
    t.ok[t.k] = 1;
  }
  __syncthreads();
  tile_store(y_ + t.r0, X, t.nrows, t);
}

// affine_ds! for tiled cones: ds = lambda o lambda
__global__ void k_soc_tile_affine_ds(ConeSet cs, const int *tiles, int trows, double *ds_) {
  SocTileCtx t = soc_tile_ctx(cs, tiles, trows, 1);
  double *L = tile_arr(0, t.words);
  tile_load(L, cs.soc_lambda + (t.r0 - cs.soc_begin), t.nrows);
  tile_loaded();
  __syncthreads();
  if (t.valid) {
    const int o = t.off, d = t.dim;
    double tt = tree16(d, [&](int l) {
      double ll = L[tsk(o + l)];
      return 0.0 + ll * ll;
    });
    double l0 = L[tsk(o)];
    for (int i = 1; i < d; ++i) {
      double li = L[tsk(o + i)];
      L[tsk(o + i)] = l0 * li + l0 * li;
    }
    L[tsk(o)] = tt;
    t.ok[t.k] = 1;
  }
  __syncthreads();
  tile_store(ds_ + t.r0, L, t.nrows, t);
}

// combined_ds_shift! for tiled cones (coneops_defaults.jl:335-368): the
// shift overwrites the staged dz rows in place.
__global__ void k_soc_tile_combined(ConeSet cs, const int *tiles, int trows, double *shift_, const double *__restrict__ dz_,
                                    const double *__restrict__ ds_, const double *sm) {
  SocTileCtx t = soc_tile_ctx(cs, tiles, trows, 3);
  double *W = tile_arr(0, t.words), *DZ = tile_arr(1, t.words), *DS = tile_arr(2, t.words);
  tile_load(W, cs.soc_w + (t.r0 - cs.soc_begin), t.nrows);
  tile_load(DZ, dz_ + t.r0, t.nrows);
  tile_load(DS, ds_ + t.r0, t.nrows);
  tile_loaded();
  __syncthreads();
  if (t.valid) {
    const int o = t.off, d = t.dim;
    double eta = cs.soc_eta[t.c], w0 = W[tsk(o)];
    double zz = tree16(d, [&](int l) {
      return l > 0 ? 0.0 + W[tsk(o + l)] * DZ[tsk(o + l)] : 0.0;
    });
    double zs = tree16(d, [&](int l) {
      return l > 0 ? 0.0 + W[tsk(o + l)] * DS[tsk(o + l)] : 0.0;
    });
    double dz0 = DZ[tsk(o)], ds0 = DS[tsk(o)];
    double cz = dz0 + zz / (1 + w0);
    double csn = -ds0 + zs / (1 + w0);
    double wz0 = eta * (w0 * dz0 + zz);
    double ws0 = (1 / eta) * (w0 * ds0 - zs);
    double dot = tree16(d, [&](int l) {
      double wl = W[tsk(o + l)];
      double a = (l == 0) ? wz0 : eta * (DZ[tsk(o + l)] + cz * wl);
      double b = (l == 0) ? ws0 : (1 / eta) * (DS[tsk(o + l)] + csn * wl);
      return 0.0 + a * b;
    });
    for (int i = 1; i < d; ++i) {
      double wi = W[tsk(o + i)];
      double a = eta * (DZ[tsk(o + i)] + cz * wi);
      double b = (1 / eta) * (DS[tsk(o + i)] + csn * wi);
      DZ[tsk(o + i)] = ws0 * a + wz0 * b;
    }
    DZ[tsk(o)] = dot - sm[t.inst];
    t.ok[t.k] = 1;
  }
  __syncthreads();
  tile_store(shift_ + t.r0, DZ, t.nrows, t);
}

// Δs_from_Δz_offset! for tiled cones (coneops_socone.jl:539-566): the output
// overwrites the staged ds rows in place.
__global__ void k_soc_tile_ds_offset(ConeSet cs, const int *tiles, int trows, double *out_, const double *__restrict__ ds_,
                                     const double *__restrict__ z_) {
  SocTileCtx t = soc_tile_ctx(cs, tiles, trows, 4);
  double *W = tile_arr(0, t.words), *L = tile_arr(1, t.words), *DS = tile_arr(2, t.words), *Z = tile_arr(3, t.words);
  const int r = t.r0 - cs.soc_begin;
  tile_load(W, cs.soc_w + r, t.nrows);
  tile_load(L, cs.soc_lambda + r, t.nrows);
  tile_load(DS, ds_ + t.r0, t.nrows);
  tile_load(Z, z_ + t.r0, t.nrows);
  tile_loaded();
  __syncthreads();
  if (t.valid) {
    const int o = t.off, d = t.dim;
    double z1sq = tree16(d, [&](int l) {
      double zl = Z[tsk(o + l)];
      return l > 0 ? 0.0 + zl * zl : 0.0;
    });
    double l1ds1 = tree16(d, [&](int l) {
      return l > 0 ? 0.0 + L[tsk(o + l)] * DS[tsk(o + l)] : 0.0;
    });
    double w1ds1 = tree16(d, [&](int l) {
      return l > 0 ? 0.0 + W[tsk(o + l)] * DS[tsk(o + l)] : 0.0;
    });
    double z0 = Z[tsk(o)], l0 = L[tsk(o)], w0 = W[tsk(o)];
    double resz = soc_res(z0, z1sq);
    double eta = cs.soc_eta[t.c];
    double c = l0 * DS[tsk(o)] - l1ds1;
    double il = 1 / l0;
    for (int i = 1; i < d; ++i) {
      double o_i = -Z[tsk(o + i)] * (c / resz);
      o_i += eta * (DS[tsk(o + i)] + w1ds1 / (1 + w0) * W[tsk(o + i)]);
      DS[tsk(o + i)] = o_i * il;
    }
    double o0 = z0 * (c / resz);
    o0 += eta * w1ds1;
    DS[tsk(o)] = o0 * il;
    t.ok[t.k] = 1;
  }
  __syncthreads();
  tile_store(out_ + t.r0, DS, t.nrows, t);
}

// step_length for tiled cones (coneops_socone.jl:745-814), sequential sums
__device__ double soc_tile_step_component(const double *X, const double *Y, int o, int d,
                                          double amax) {
  double x0 = X[tsk(o)], y0 = Y[tsk(o)];
  double ysq = tree16(d, [&](int l) {
    double yl = Y[tsk(o + l)];
    return l > 0 ? 0.0 + yl * yl : 0.0;
  });
  double xsq = tree16(d, [&](int l) {
    double xl = X[tsk(o + l)];
    return l > 0 ? 0.0 + xl * xl : 0.0;
  });
  double xy = tree16(d, [&](int l) {
    return l > 0 ? 0.0 + X[tsk(o + l)] * Y[tsk(o + l)] : 0.0;
  });
  if (x0 >= 0 && y0 < 0) amax = fmin(amax, -x0 / y0);
  double a = soc_res(y0, ysq);
  double b = 2 * (x0 * y0 - xy);
  double c = fmax(0.0, soc_res(x0, xsq));
  double dd = b * b - 4 * a * c;
  if ((a > 0 && b > 0) || dd < 0) return amax;
  if (a == 0) return amax;
  if (c == 0) return a >= 0 ? amax : 0.0;
  double tq = (b >= 0) ? (-b - sqrt(dd)) : (-b + sqrt(dd));
  double r1 = (2 * c) / tq, r2 = tq / (2 * a);
  r1 = r1 < 0 ? kDMax : r1;
  r2 = r2 < 0 ? kDMax : r2;
  return fmin(amax, fmin(r1, r2));
}
__global__ void k_soc_tile_step(ConeSet cs, const int *tiles, int trows, const double *__restrict__ dz_,
                                const double *__restrict__ ds_, const double *__restrict__ z_,
                                const double *__restrict__ s_, double *alpha) {
  SocTileCtx t = soc_tile_ctx(cs, tiles, trows, 4);
  double *DZ = tile_arr(0, t.words), *DS = tile_arr(1, t.words), *Z = tile_arr(2, t.words), *S = tile_arr(3, t.words);
  tile_load(DZ, dz_ + t.r0, t.nrows);
  tile_load(DS, ds_ + t.r0, t.nrows);
  tile_load(Z, z_ + t.r0, t.nrows);
  tile_load(S, s_ + t.r0, t.nrows);
  tile_loaded();
  __syncthreads();
  double a = CUDART_INF;
  if (t.valid) {
    double amax = alpha[t.inst];
    double az = soc_tile_step_component(Z, DZ, t.off, t.dim, amax);
    double as = soc_tile_step_component(S, DS, t.off, t.dim, amax);
    a = fmin(az, as);
  }
  block_seg_min_nonneg(alpha, t.valid ? t.inst : -1, a);
}

std::vector<int> soc_tiles(const int *off, const int *dim, int n, int max_cones, int max_rows) {
  std::vector<int> t;
  const int lo = 1, hi = kSocTileMaxDim;
  int k = 0;
  while (k < n) {
    if (dim[k] > hi || dim[k] < lo) {
      ++k;
      continue;
    }
    int start = k, rows = 0;
    while (k < n && dim[k] >= lo && dim[k] <= hi && k - start < max_cones &&
           rows + dim[k] <= max_rows && (k == start || off[k] == off[k - 1] + dim[k - 1])) {
      rows += dim[k];
      ++k;
    }
    t.push_back(start);
    t.push_back(k);
  }
  return t;
}

// =============================================================== launchers
static inline int blocks_for(long long n, int b = kBlock) {
  return n <= 0 ? 0 : ceil_div(n, b);
}
#define LAUNCH_SOC(KERNEL, ...)                                                        \
  do {                                                                                 \
    if (cs.n_soc > 0) {                                                                \
      int G = cs.soc_group;                                                            \
      int nb = blocks_for((long long)cs.n_soc * G);                                    \
      switch (G) {                                                                     \
        case 2: KERNEL<2><<<nb, kBlock, 0, st>>>(__VA_ARGS__); break;                  \
        case 4: KERNEL<4><<<nb, kBlock, 0, st>>>(__VA_ARGS__); break;                  \
        case 8: KERNEL<8><<<nb, kBlock, 0, st>>>(__VA_ARGS__); break;                  \
        case 16: KERNEL<16><<<nb, kBlock, 0, st>>>(__VA_ARGS__); break;                \
        default: KERNEL<32><<<nb, kBlock, 0, st>>>(__VA_ARGS__); break;                \
      }                                                                                \
    }                                                                                  \
  } while (0)

// Shared memory of a tile kernel staging `narr` arrays of `rows` rows.
static inline size_t soc_tile_smem(int narr, int rows) {
  return (size_t)narr * tile_words(rows) * sizeof(double) + rows * sizeof(unsigned short) +
         rows / 8;
}
// One SOC operation with the cone set's launch shape: tiles of the chosen
// size over the cones of dim <= 16 and the lane-group kernel for the larger
// ones, or lane groups for every cone.
#define LAUNCH_SOC_SHAPED(OP, TILE_KERNEL, NARR, GROUP_KERNEL, ...)                    \
  do {                                                                                 \
    if (cs.n_soc > 0) {                                                                \
      const int _v = cs.soc_variant[OP];                                               \
      if (_v >= 1 && _v <= kSocTileShapes && cs.soc_ntiles[_v] > 0) {                  \
        const int _rows = soc_tile_rows(_v);                                           \
        TILE_KERNEL<<<cs.soc_ntiles[_v], soc_tile_cones(_v), soc_tile_smem(NARR, _rows), \
                      st>>>(cs, cs.soc_tile[_v], _rows, __VA_ARGS__);                  \
        if (cs.soc_group == 32) {                                                      \
          ConeSet csl = cs;                                                            \
          csl.soc_skip_lo = 1;                                                         \
          csl.soc_skip_hi = kSocTileMaxDim;                                            \
          LAUNCH_SOC(GROUP_KERNEL, csl, __VA_ARGS__);                                  \
        }                                                                              \
      } else {                                                                         \
        LAUNCH_SOC(GROUP_KERNEL, cs, __VA_ARGS__);                                     \
      }                                                                                \
    }                                                                                  \
  } while (0)
static inline int nn_block(const ConeSet &cs) { return cs.nn_block > 0 ? cs.nn_block : kBlock; }

static inline void psd_launch_dims(const ConeSet &cs, int nmats, int &nb, int &nt,
                                   size_t &smem) {
  // groups (cones) per block: 64 threads' worth while their matrices fit
  // 200 KB
  const int G = psd_group(cs.psd_nmax), want = 32 * kPsdWarps / G;
  const size_t per = (size_t)nmats * cs.psd_nmax * cs.psd_nmax * sizeof(double);
  const int groups =
      per == 0 ? want : (int)std::max<size_t>(1, std::min<size_t>(want, (200 * 1024) / per));
  nt = G * groups;
  nb = blocks_for((long long)cs.n_psd * G, nt);
  smem = (size_t)groups * per + 256;
}
#define LAUNCH_PSD(KERNEL, NMATS, ...)                                                 \
  do {                                                                                 \
    if (cs.n_psd > 0) {                                                                \
      static const bool _attr = (cudaFuncSetAttribute(                                  \
                                     KERNEL, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                     210 * 1024) == cudaSuccess);                      \
      (void)_attr;                                                                     \
      int _nb, _nt;                                                                    \
      size_t _smem;                                                                    \
      psd_launch_dims(cs, NMATS, _nb, _nt, _smem);                                     \
      KERNEL<<<_nb, _nt, _smem, st>>>(__VA_ARGS__);                                    \
    }                                                                                  \
  } while (0)

static NonsymArgs<ExpOps> exp_args(const ConeSet &cs) {
  return NonsymArgs<ExpOps>{cs.n_exp, cs.exp_begin, cs.exp_inst, nullptr,
                            cs.exp_Hd, cs.exp_Hs, cs.exp_grad, cs.exp_z};
}
static NonsymArgs<PowOps> pow_args(const ConeSet &cs) {
  return NonsymArgs<PowOps>{cs.n_pow, cs.pow_begin, cs.pow_inst, cs.pow_alpha,
                            cs.pow_Hd, cs.pow_Hs, cs.pow_grad, cs.pow_z};
}

void cones_update_scaling(const ConeSet &cs, const double *s, const double *z,
                          const double *mu, const int *scaling, int *scale_ok,
                          cudaStream_t st) {
  if (cs.n_nn) k_nn_update_scaling<<<blocks_for(cs.n_nn, nn_block(cs)), nn_block(cs), 0, st>>>(cs, s, z);
  LAUNCH_SOC_SHAPED(kSocUpdateScaling, k_soc_tile_update_scaling, 4, k_soc_update_scaling, s, z,
                    scale_ok);
  if (cs.n_exp)
    k_nonsym_update_scaling<ExpOps><<<blocks_for(cs.n_exp, 128), 128, 0, st>>>(
        cs, exp_args(cs), s, z, mu, scaling);
  if (cs.n_pow)
    k_nonsym_update_scaling<PowOps><<<blocks_for(cs.n_pow, 128), 128, 0, st>>>(
        cs, pow_args(cs), s, z, mu, scaling);
  LAUNCH_PSD(k_psd_update_scaling, 7, cs, s, z, scale_ok);
}

void cones_refresh_kkt(const ConeSet &cs, const KKTMapDev &map, double *kv,
                       cudaStream_t st) {
  if (cs.n_nn) k_nn_refresh<<<blocks_for(cs.n_nn), kBlock, 0, st>>>(cs, map.nn_pos, kv);
  LAUNCH_SOC(k_soc_refresh, cs, map, kv);
  if (cs.n_exp)
    k_nonsym_refresh<<<blocks_for(cs.n_exp), kBlock, 0, st>>>(cs, cs.n_exp, cs.exp_inst,
                                                             cs.exp_Hs, map.exp_pos, kv);
  if (cs.n_pow)
    k_nonsym_refresh<<<blocks_for(cs.n_pow), kBlock, 0, st>>>(cs, cs.n_pow, cs.pow_inst,
                                                             cs.pow_Hs, map.pow_pos, kv);
  LAUNCH_PSD(k_psd_refresh, 1, cs, map, kv);
}

void cones_get_Hs(const ConeSet &cs, const int *nn_blk, const int *soc_blk,
                  const int *exp_blk, const int *pow_blk, const int *psd_blk, double *Hs,
                  cudaStream_t st) {
  if (cs.n_nn) k_nn_get_hs<<<blocks_for(cs.n_nn), kBlock, 0, st>>>(cs, nn_blk, Hs);
  LAUNCH_SOC(k_soc_get_hs, cs, soc_blk, Hs);
  if (cs.n_exp)
    k_nonsym_get_hs<<<blocks_for(cs.n_exp), kBlock, 0, st>>>(cs.n_exp, cs.exp_Hs, exp_blk, Hs);
  if (cs.n_pow)
    k_nonsym_get_hs<<<blocks_for(cs.n_pow), kBlock, 0, st>>>(cs.n_pow, cs.pow_Hs, pow_blk, Hs);
  LAUNCH_PSD(k_psd_get_hs, 1, cs, psd_blk, Hs);
}

void cones_mul_Hs(const ConeSet &cs, double *y, const double *x, cudaStream_t st) {
  if (cs.n_zero) k_zero_fill<<<blocks_for(cs.n_zero), kBlock, 0, st>>>(cs, y);
  if (cs.n_nn) k_nn_mul_hs<<<blocks_for(cs.n_nn, nn_block(cs)), nn_block(cs), 0, st>>>(cs, y, x);
  LAUNCH_SOC_SHAPED(kSocMulHs, k_soc_tile_mul_hs, 2, k_soc_mul_hs, y, x);
  if (cs.n_exp)
    k_nonsym_mul_hs<<<blocks_for(cs.n_exp), kBlock, 0, st>>>(cs, cs.n_exp, cs.exp_begin,
                                                            cs.exp_inst, cs.exp_Hs, y, x);
  if (cs.n_pow)
    k_nonsym_mul_hs<<<blocks_for(cs.n_pow), kBlock, 0, st>>>(cs, cs.n_pow, cs.pow_begin,
                                                            cs.pow_inst, cs.pow_Hs, y, x);
  LAUNCH_PSD(k_psd_mul_hs, 3, cs, y, x);
}

void cones_affine_ds(const ConeSet &cs, double *ds, const double *s, cudaStream_t st) {
  if (cs.n_zero) k_zero_fill<<<blocks_for(cs.n_zero), kBlock, 0, st>>>(cs, ds);
  if (cs.n_nn)
    k_nn_affine_ds<<<blocks_for(cs.n_nn, nn_block(cs) * kNNRows), nn_block(cs), 0, st>>>(cs, ds);
  LAUNCH_SOC_SHAPED(kSocAffineDs, k_soc_tile_affine_ds, 1, k_soc_affine_ds, ds);
  if (cs.n_exp)
    k_nonsym_copy<<<blocks_for(3 * cs.n_exp), kBlock, 0, st>>>(cs, cs.n_exp, cs.exp_begin,
                                                              cs.exp_inst, ds, s);
  if (cs.n_pow)
    k_nonsym_copy<<<blocks_for(3 * cs.n_pow), kBlock, 0, st>>>(cs, cs.n_pow, cs.pow_begin,
                                                              cs.pow_inst, ds, s);
  LAUNCH_PSD(k_psd_affine_ds, 0, cs, ds);
}

void cones_combined_ds_shift(const ConeSet &cs, double *shift, const double *dz,
                             const double *ds, const double *sm, cudaStream_t st) {
  if (cs.n_zero) k_zero_fill<<<blocks_for(cs.n_zero), kBlock, 0, st>>>(cs, shift);
  if (cs.n_nn) k_nn_combined<<<blocks_for(cs.n_nn, nn_block(cs)), nn_block(cs), 0, st>>>(cs, shift, dz, ds, sm);
  LAUNCH_SOC_SHAPED(kSocCombined, k_soc_tile_combined, 3, k_soc_combined, shift, dz, ds, sm);
  if (cs.n_exp)
    k_nonsym_combined<ExpOps><<<blocks_for(cs.n_exp, 128), 128, 0, st>>>(
        cs, exp_args(cs), shift, dz, ds, sm);
  if (cs.n_pow)
    k_nonsym_combined<PowOps><<<blocks_for(cs.n_pow, 128), 128, 0, st>>>(
        cs, pow_args(cs), shift, dz, ds, sm);
  LAUNCH_PSD(k_psd_combined, 5, cs, shift, dz, ds, sm);
}

void cones_ds_from_dz_offset(const ConeSet &cs, double *out, const double *ds,
                             const double *z, cudaStream_t st) {
  if (cs.n_zero) k_zero_fill<<<blocks_for(cs.n_zero), kBlock, 0, st>>>(cs, out);
  if (cs.n_nn) k_nn_ds_offset<<<blocks_for(cs.n_nn, nn_block(cs)), nn_block(cs), 0, st>>>(cs, out, ds, z);
  LAUNCH_SOC_SHAPED(kSocDsOffset, k_soc_tile_ds_offset, 4, k_soc_ds_offset, out, ds, z);
  if (cs.n_exp)
    k_nonsym_copy<<<blocks_for(3 * cs.n_exp), kBlock, 0, st>>>(cs, cs.n_exp, cs.exp_begin,
                                                              cs.exp_inst, out, ds);
  if (cs.n_pow)
    k_nonsym_copy<<<blocks_for(3 * cs.n_pow), kBlock, 0, st>>>(cs, cs.n_pow, cs.pow_begin,
                                                              cs.pow_inst, out, ds);
  LAUNCH_PSD(k_psd_ds_offset, 4, cs, out, ds);
}

void cones_step_length_sym(const ConeSet &cs, const double *dz, const double *ds,
                           const double *z, const double *s, double *alpha,
                           cudaStream_t st) {
  if (cs.n_nn)
    k_nn_step<<<blocks_for(cs.n_nn, nn_block(cs) * (cs.B == 1 ? kNNRows : 1)), nn_block(cs), 0,
                st>>>(cs, dz, ds, z, s, alpha);
  LAUNCH_SOC_SHAPED(kSocStep, k_soc_tile_step, 4, k_soc_step, dz, ds, z, s, alpha);
  LAUNCH_PSD(k_psd_step, 4, cs, dz, ds, alpha);
}

void cones_step_length_asym(const ConeSet &cs, const double *dz, const double *ds,
                            const double *z, const double *s, const double *astart,
                            double *alpha, double step, double amin, cudaStream_t st) {
  if (cs.n_exp)
    k_nonsym_step<ExpOps><<<blocks_for(cs.n_exp, 128), 128, 0, st>>>(
        cs, exp_args(cs), dz, ds, z, s, astart, alpha, step, amin);
  if (cs.n_pow)
    k_nonsym_step<PowOps><<<blocks_for(cs.n_pow, 128), 128, 0, st>>>(
        cs, pow_args(cs), dz, ds, z, s, astart, alpha, step, amin);
}

void cones_barrier(const ConeSet &cs, const double *z, const double *s, const double *dz,
                   const double *ds, const double *alpha, const int *bt, double *bar,
                   cudaStream_t st) {
  LAUNCH_SOC(k_soc_barrier, cs, z, s, dz, ds, alpha, bt);
  if (cs.n_exp)
    k_nonsym_barrier<ExpOps><<<blocks_for(cs.n_exp, 128), 128, 0, st>>>(
        cs, exp_args(cs), cs.n_soc, z, s, dz, ds, alpha, bt);
  if (cs.n_pow)
    k_nonsym_barrier<PowOps><<<blocks_for(cs.n_pow, 128), 128, 0, st>>>(
        cs, pow_args(cs), cs.n_soc + cs.n_exp, z, s, dz, ds, alpha, bt);
  LAUNCH_PSD(k_psd_barrier, 2, cs, z, s, dz, ds, alpha, bt);
  k_barrier_inst<<<cs.B, 128, 0, st>>>(cs, z, s, dz, ds, alpha, bt, bar);
}

void cones_margins(const ConeSet &cs, const double *z, int pd, double *amin, double *asum,
                   cudaStream_t st) {
  (void)pd;
  LAUNCH_SOC(k_soc_margins, cs, z);
  LAUNCH_PSD(k_psd_margins, 2, cs, z);
  k_margins_inst<<<cs.B, 128, 0, st>>>(cs, z, amin, asum);
}

void cones_scaled_unit_shift(const ConeSet &cs, double *z, const double *alpha, int pd,
                             cudaStream_t st) {
  if (cs.n_zero) k_zero_shift<<<blocks_for(cs.n_zero), kBlock, 0, st>>>(cs, z, pd);
  if (cs.n_nn) k_nn_shift<<<blocks_for(cs.n_nn), kBlock, 0, st>>>(cs, z, alpha);
  if (cs.n_soc) k_soc_shift<<<blocks_for(cs.n_soc), kBlock, 0, st>>>(cs, z, alpha);
  if (cs.n_psd) k_psd_shift<<<blocks_for(cs.n_psd), kBlock, 0, st>>>(cs, z, alpha);
}

void cones_unit_initialization(const ConeSet &cs, double *z, double *s, cudaStream_t st) {
  if (cs.m_total) k_unit_init<<<blocks_for(cs.m_total), kBlock, 0, st>>>(cs, z, s);
  int total = cs.n_soc + cs.n_exp + cs.n_pow + cs.n_psd;
  if (total) k_unit_init_cones<<<blocks_for(total), kBlock, 0, st>>>(cs, z, s);
}

void cones_set_identity_scaling(const ConeSet &cs, cudaStream_t st) {
  int t = cs.n_nn > cs.soc_rows ? cs.n_nn : cs.soc_rows;
  if (t) k_identity<<<blocks_for(t), kBlock, 0, st>>>(cs);
  int c = cs.n_soc + cs.n_psd;
  if (c) k_identity_cones<<<blocks_for(c), kBlock, 0, st>>>(cs);
}


// ============================================================ autotuning
void cones_default_shapes(ConeSet &cs) {
  cs.nn_block = kBlock;
  cs.soc_variant[kSocUpdateScaling] = kSocTileShapes;
  for (int op = 1; op < kSocOps; ++op) cs.soc_variant[op] = 0;
  cs.soc_skip_lo = 1;  // empty skip range: lane groups take every cone
  cs.soc_skip_hi = 0;
}

int cones_autotune(ConeSet &cs, cudaStream_t st) {
  if (cs.n_nn == 0 && cs.n_soc == 0) return 0;
  const size_t m = std::max(cs.m_total, 1), B = std::max(cs.B, 1), nn = cs.n_nn,
               sr = cs.soc_rows, nsoc = cs.n_soc;
  // scratch: five vectors, the NN / SOC state, per-instance scalars
  const size_t words = 5 * m + 2 * nn + 4 * sr + 2 * nsoc + 4 * B + 8;
  double *buf = nullptr;
  cudaError_t e = cudaMalloc(&buf, words * sizeof(double));
  if (e != cudaSuccess) {  // no room for scratch: keep the default shapes
    cudaGetLastError();
    return 0;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  ConeSet t = cs;
  t.inst_active = nullptr;  // every instance runs while timing
  double *s = buf, *z = s + m, *dz = z + m, *ds = dz + m, *y = ds + m, *p = y + m;
  t.nn_w = p, p += nn;
  t.nn_lambda = p, p += nn;
  t.soc_w = p, p += sr;
  t.soc_lambda = p, p += sr;
  t.soc_u = p, p += sr;
  t.soc_v = p, p += sr;
  t.soc_eta = p, p += nsoc;
  t.soc_d = p, p += nsoc;
  double *mu = p, *sm = p + B, *alpha = p + 2 * B;
  int *scaling = reinterpret_cast<int *>(p + 3 * B), *scale_ok = scaling + B;
  cudaMemsetAsync(buf, 0, words * sizeof(double), st);
  cones_unit_initialization(t, z, s, st);
  {
    std::vector<double> sc(3 * B);
    for (size_t i = 0; i < B; ++i) sc[i] = 1.0, sc[B + i] = 0.1, sc[2 * B + i] = 1.0;
    std::vector<int> ok(B, 1);
    cudaMemcpyAsync(mu, sc.data(), sc.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(scale_ok, ok.data(), B * sizeof(int), cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);  // host vectors leave scope
  }
  // Each candidate: one warm-up launch, then the median of 5 single launches,
  // each after L2 has been overwritten (an IPM step reaches these kernels
  // after the factorisation has streamed far more than L2 holds).
  const size_t flush_bytes = (size_t)160 << 20;
  void *flush = nullptr;
  if (cudaMalloc(&flush, flush_bytes) != cudaSuccess) {
    flush = nullptr;
    cudaGetLastError();
  }
  auto timed = [&](auto launch) {
    launch();
    float t[5];
    for (int r = 0; r < 5; ++r) {
      if (flush) cudaMemsetAsync(flush, r, flush_bytes, st);
      cudaEventRecord(e0, st);
      launch();
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      t[r] = 0.f;
      cudaEventElapsedTime(&t[r], e0, e1);
    }
    std::sort(t, t + 5);
    return t[2];
  };
  // a candidate replaces the default only when it is clearly faster
  auto better = [](float ms, float best_ms) { return ms < 0.95f * best_ms; };
  auto run = [&](const ConeSet &c, int op) {
    switch (op) {
      case kSocUpdateScaling: cones_update_scaling(c, s, z, mu, scaling, scale_ok, st); break;
      case kSocAffineDs: cones_affine_ds(c, y, s, st); break;
      case kSocCombined: cones_combined_ds_shift(c, y, dz, ds, sm, st); break;
      case kSocDsOffset: cones_ds_from_dz_offset(c, y, ds, z, st); break;
      case kSocMulHs: cones_mul_Hs(c, y, dz, st); break;
      case kSocStep: cones_step_length_sym(c, dz, ds, z, s, alpha, st); break;
      default: break;
    }
  };
  // only the cone type being tuned launches
  ConeSet only = t;
  only.n_zero = 0, only.n_exp = 0, only.n_pow = 0, only.n_psd = 0;
  run(only, kSocUpdateScaling);  // fills the scratch state the other operations read
  if (cs.n_nn > 0) {
    ConeSet c = only;
    c.n_soc = 0;
    auto nn_ms = [&](int b) {
      c.nn_block = b;
      return timed([&]() {
        run(c, kSocUpdateScaling);
        run(c, kSocAffineDs);
        run(c, kSocCombined);
        run(c, kSocDsOffset);
        run(c, kSocStep);
      });
    };
    int best = cs.nn_block;
    float best_ms = nn_ms(best);
    for (int b : {128, 256, 512}) {
      if (b == cs.nn_block) continue;
      float ms = nn_ms(b);
      if (better(ms, best_ms)) best_ms = ms, best = b;
    }
    cs.nn_block = best;
  }
  if (cs.n_soc > 0) {
    ConeSet c = only;
    c.n_nn = 0;
    for (int op = 0; op < kSocOps; ++op) {
      auto soc_ms = [&](int v) {
        c.soc_variant[op] = v;
        return timed([&]() { run(c, op); });
      };
      int best = cs.soc_variant[op];
      float best_ms = soc_ms(best);
      for (int v = 0; v <= kSocTileShapes; ++v) {
        if (v == cs.soc_variant[op] || (v > 0 && cs.soc_ntiles[v] == 0)) continue;
        float ms = soc_ms(v);
        if (better(ms, best_ms)) best_ms = ms, best = v;
      }
      c.soc_variant[op] = best;
      cs.soc_variant[op] = best;
    }
  }
  e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (flush) cudaFree(flush);
  cudaFree(buf);
  return e == cudaSuccess ? 0 : -1000 - (int)e;
}

}  // namespace clgpu
