// oracle_cones.cpp -- CPU restatement of Clarabel's cone operations.
// TEST INFRASTRUCTURE ONLY (see clarabel_oracle.h).
//
// Each cone follows the matching file under src/cones/ of the reference:
//   ZeroCone         coneops_zerocone.jl:389-560
//   NonnegativeCone  coneops_nncone.jl:5-298
//   SecondOrderCone  coneops_socone.jl:303-814
//   ExponentialCone  coneops_expcone.jl:193-711
//   PowerCone        coneops_powcone.jl:1-478
//   PSDTriangleCone  coneops_psdtrianglecone.jl:1-547
//   shared           coneops_defaults.jl:335-385, coneops_nonsymmetric_common.jl,
//                    mathutils.jl:381-432 (3x3 Cholesky)
#include <algorithm>
#include <cstring>
#include <numeric>
#include <stdexcept>

#include "oracle_internal.hpp"

namespace orc {

static inline double dotv(const double *a, const double *b, int n) {
  double t = 0;
  for (int i = 0; i < n; ++i) t += a[i] * b[i];
  return t;
}
static inline double norm2(const double *a, int n) {
  return std::sqrt(dotv(a, a, n));
}

bool Cone::rectify_equilibration(double *delta, const double *e) {
  // coneops_defaults.jl:32-44: delta = mean(e)/e
  int n = numel();
  double t = 0;
  for (int i = 0; i < n; ++i) t += e[i];
  t /= n;
  for (int i = 0; i < n; ++i) delta[i] = t / e[i];
  return true;
}

// ------------------------------------------------------------- symmetric
// Generic pieces of coneops_defaults.jl:335-385 for symmetric cones.
struct SymCone : Cone {
  virtual void mul_W(bool trans, double *y, const double *x, double a,
                     double b) = 0;
  virtual void mul_Winv(bool trans, double *y, const double *x, double a,
                        double b) = 0;
  virtual void lambda_inv_circ_op(double *x, const double *z) = 0;
  virtual void circ_op(double *x, const double *y, const double *z) = 0;
  void combined_ds_shift(double *shift, double *step_z, double *step_s,
                         double sm) override {
    int n = numel();
    Vec tmp(shift, shift + 0);
    tmp.assign(step_z, step_z + n);
    mul_W(false, step_z, tmp.data(), 1.0, 0.0);
    tmp.assign(step_s, step_s + n);
    mul_Winv(true, step_s, tmp.data(), 1.0, 0.0);
    circ_op(shift, step_s, step_z);
    scaled_unit_shift(shift, -sm, PrimalCone);
  }
  void ds_from_dz_offset(double *out, const double *ds, double *work,
                         const double *) override {
    lambda_inv_circ_op(work, ds);
    mul_W(true, out, work, 1.0, 0.0);
  }
};

// ------------------------------------------------------------- zero
struct ZeroCone : Cone {
  int dim;
  explicit ZeroCone(int d) : dim(d) {}
  int type() const override { return OR_CONE_ZERO; }
  int numel() const override { return dim; }
  int degree() const override { return 0; }
  bool rectify_equilibration(double *delta, const double *) override {
    for (int i = 0; i < dim; ++i) delta[i] = 1.0;
    return false;
  }
  void margins(const double *, int, double &a, double &b) override {
    a = kMax;
    b = 0;
  }
  void scaled_unit_shift(double *z, double, int pd) override {
    if (pd == PrimalCone)
      for (int i = 0; i < dim; ++i) z[i] = 0;
  }
  void unit_initialization(double *z, double *s) override {
    for (int i = 0; i < dim; ++i) z[i] = s[i] = 0;
  }
  void set_identity_scaling() override {}
  bool update_scaling(const double *, const double *, double, int) override {
    return true;
  }
  void get_Hs(double *Hs) override {
    for (int i = 0; i < dim; ++i) Hs[i] = 0;
  }
  void mul_Hs(double *y, const double *, double *) override {
    for (int i = 0; i < dim; ++i) y[i] = 0;
  }
  void affine_ds(double *ds, const double *) override {
    for (int i = 0; i < dim; ++i) ds[i] = 0;
  }
  void combined_ds_shift(double *shift, double *, double *, double) override {
    for (int i = 0; i < dim; ++i) shift[i] = 0;
  }
  void ds_from_dz_offset(double *out, const double *, double *,
                         const double *) override {
    for (int i = 0; i < dim; ++i) out[i] = 0;
  }
  void step_length(const double *, const double *, const double *,
                   const double *, const oracle_settings &, double amax,
                   double &az, double &as) override {
    az = as = amax;
  }
  double compute_barrier(const double *, const double *, const double *,
                         const double *, double) override {
    return 0;
  }
};

// ------------------------------------------------------------- nonnegative
struct NNCone : SymCone {
  int dim;
  Vec w, lambda;
  explicit NNCone(int d) : dim(d), w(d, 1.0), lambda(d, 0.0) {}
  int type() const override { return OR_CONE_NONNEG; }
  int numel() const override { return dim; }
  int degree() const override { return dim; }
  bool rectify_equilibration(double *delta, const double *) override {
    for (int i = 0; i < dim; ++i) delta[i] = 1.0;
    return false;
  }
  void margins(const double *z, int, double &a, double &b) override {
    a = dim > 0 ? *std::min_element(z, z + dim) : kMax;
    b = 0;
    for (int i = 0; i < dim; ++i) b += z[i] > 0 ? z[i] : 0.0;
  }
  void scaled_unit_shift(double *z, double a, int) override {
    for (int i = 0; i < dim; ++i) z[i] += a;
  }
  void unit_initialization(double *z, double *s) override {
    for (int i = 0; i < dim; ++i) z[i] = s[i] = 1.0;
  }
  void set_identity_scaling() override { std::fill(w.begin(), w.end(), 1.0); }
  bool update_scaling(const double *s, const double *z, double,
                      int) override {
    for (int i = 0; i < dim; ++i) {
      lambda[i] = std::sqrt(s[i] * z[i]);
      w[i] = std::sqrt(s[i] / z[i]);
    }
    return true;
  }
  void get_Hs(double *Hs) override {
    for (int i = 0; i < dim; ++i) Hs[i] = w[i] * w[i];
  }
  void mul_Hs(double *y, const double *x, double *) override {
    for (int i = 0; i < dim; ++i) y[i] = w[i] * (w[i] * x[i]);
  }
  void affine_ds(double *ds, const double *) override {
    for (int i = 0; i < dim; ++i) ds[i] = lambda[i] * lambda[i];
  }
  void ds_from_dz_offset(double *out, const double *ds, double *,
                         const double *z) override {
    for (int i = 0; i < dim; ++i) out[i] = ds[i] / z[i];
  }
  void step_length(const double *dz, const double *ds, const double *z,
                   const double *s, const oracle_settings &, double amax,
                   double &az, double &as) override {
    az = amax;
    as = amax;
    for (int i = 0; i < dim; ++i) {
      if (dz[i] < 0) az = std::min(az, -z[i] / dz[i]);
      if (ds[i] < 0) as = std::min(as, -s[i] / ds[i]);
    }
  }
  double compute_barrier(const double *z, const double *s, const double *dz,
                         const double *ds, double a) override {
    double bar = 0;
    for (int i = 0; i < dim; ++i) {
      double si = s[i] + a * ds[i];
      double zi = z[i] + a * dz[i];
      bar -= logsafe(si * zi);
    }
    return bar;
  }
  void mul_W(bool, double *y, const double *x, double a, double b) override {
    for (int i = 0; i < dim; ++i) y[i] = a * (x[i] * w[i]) + b * y[i];
  }
  void mul_Winv(bool, double *y, const double *x, double a,
                double b) override {
    for (int i = 0; i < dim; ++i) y[i] = a * (x[i] / w[i]) + b * y[i];
  }
  void lambda_inv_circ_op(double *x, const double *z) override {
    for (int i = 0; i < dim; ++i) x[i] = z[i] / lambda[i];
  }
  void circ_op(double *x, const double *y, const double *z) override {
    for (int i = 0; i < dim; ++i) x[i] = y[i] * z[i];
  }
};

// ------------------------------------------------------------- SOC
static inline double soc_residual(const double *z, int n) {
  double z1 = norm2(z + 1, n - 1);
  return (z[0] - z1) * (z[0] + z1);
}
static inline double sqrt_soc_residual(const double *z, int n) {
  double r = soc_residual(z, n);
  return r > 0.0 ? std::sqrt(r) : 0.0;
}
static inline double soc_residual_shifted(const double *z, const double *dz,
                                          double a, int n) {
  double x0 = z[0] + a * dz[0];
  double x1sq = 0;
  for (int i = 1; i < n; ++i) {
    double zi = z[i] + a * dz[i];
    x1sq += zi * zi;
  }
  double x1 = std::sqrt(x1sq);
  return (x0 - x1) * (x0 + x1);
}
// coneops_socone.jl:745-814
static double step_length_soc_component(const double *x, const double *y,
                                        double amax, int n) {
  if (x[0] >= 0 && y[0] < 0) amax = std::min(amax, -x[0] / y[0]);
  double a = soc_residual(y, n);
  double b = 2 * (x[0] * y[0] - dotv(x + 1, y + 1, n - 1));
  double c = std::max(0.0, soc_residual(x, n));
  double d = b * b - 4 * a * c;
  if (c < 0) throw std::domain_error("starting point of line search not in SOC");
  if ((a > 0 && b > 0) || d < 0) return amax;
  if (a == 0) return amax;
  if (c == 0) return a >= 0 ? amax : 0.0;
  double t = (b >= 0) ? (-b - std::sqrt(d)) : (-b + std::sqrt(d));
  double r1 = (2 * c) / t;
  double r2 = t / (2 * a);
  r1 = r1 < 0 ? kMax : r1;
  r2 = r2 < 0 ? kMax : r2;
  return std::min(amax, std::min(r1, r2));
}

struct SOCCone : SymCone {
  int dim;
  SOCState st;
  explicit SOCCone(int d) : dim(d) {
    st.w.assign(d, 0.0);
    st.lambda.assign(d, 0.0);
    st.sparse = d > 5;  // SOC_NO_EXPANSION_MAX_SIZE, src/Clarabel.jl:9
    if (st.sparse) {
      st.u.assign(d, 0.0);
      st.v.assign(d, 0.0);
    }
  }
  int type() const override { return OR_CONE_SOC; }
  int numel() const override { return dim; }
  int degree() const override { return 1; }
  bool is_sparse_expandable() const override { return st.sparse; }
  bool Hs_is_diagonal() const override { return st.sparse; }
  void margins(const double *z, int, double &a, double &b) override {
    a = z[0] - norm2(z + 1, dim - 1);
    b = std::max(0.0, a);
  }
  void scaled_unit_shift(double *z, double a, int) override { z[0] += a; }
  void unit_initialization(double *z, double *s) override {
    for (int i = 0; i < dim; ++i) z[i] = s[i] = 0;
    s[0] += 1.0;
    z[0] += 1.0;
  }
  void set_identity_scaling() override {
    std::fill(st.w.begin(), st.w.end(), 0.0);
    st.w[0] = 1.0;
    st.eta = 1.0;
    if (st.sparse) {
      st.d = 0.5;
      std::fill(st.u.begin(), st.u.end(), 0.0);
      st.u[0] = std::sqrt(0.5);
      std::fill(st.v.begin(), st.v.end(), 0.0);
    }
  }
  // coneops_socone.jl:372-451
  bool update_scaling(const double *s, const double *z, double,
                      int) override {
    double zscale = sqrt_soc_residual(z, dim);
    double sscale = sqrt_soc_residual(s, dim);
    if (zscale == 0.0 || sscale == 0.0) return false;
    st.eta = std::sqrt(sscale / zscale);
    Vec &w = st.w;
    for (int i = 0; i < dim; ++i) w[i] = s[i] / sscale;
    w[0] += z[0] / zscale;
    for (int i = 1; i < dim; ++i) w[i] -= z[i] / zscale;
    double wscale = sqrt_soc_residual(w.data(), dim);
    if (wscale == 0.0) return false;
    for (int i = 0; i < dim; ++i) w[i] /= wscale;
    double w1sq = 0;
    for (int i = 1; i < dim; ++i) w1sq += w[i] * w[i];
    w[0] = std::sqrt(1 + w1sq);
    double gamma = 0.5 * wscale;
    Vec &lam = st.lambda;
    lam[0] = gamma;
    double c1 = (gamma + z[0] / zscale) / sscale;
    double c2 = (gamma + s[0] / sscale) / zscale;
    for (int i = 1; i < dim; ++i) lam[i] = c1 * s[i] + c2 * z[i];
    double inv = 1.0 / (s[0] / sscale + z[0] / zscale + 2 * gamma);
    for (int i = 1; i < dim; ++i) lam[i] *= inv;
    double sc = std::sqrt(sscale * zscale);
    for (int i = 0; i < dim; ++i) lam[i] *= sc;
    if (st.sparse) {
      double alpha = 2 * w[0];
      double wsq = w[0] * w[0] + w1sq;
      double wsqinv = 1 / wsq;
      st.d = wsqinv / 2;
      double u0 = std::sqrt(wsq - st.d);
      double u1 = alpha / u0;
      double v0 = 0;
      double v1 = std::sqrt(2 * (2 + wsqinv) / (2 * wsq - wsqinv));
      st.u[0] = u0;
      for (int i = 1; i < dim; ++i) st.u[i] = u1 * w[i];
      st.v[0] = v0;
      for (int i = 1; i < dim; ++i) st.v[i] = v1 * w[i];
    }
    return true;
  }
  void get_Hs(double *Hs) override {
    double e2 = st.eta * st.eta;
    if (st.sparse) {
      for (int i = 0; i < dim; ++i) Hs[i] = e2;
      Hs[0] *= st.d;
    } else {
      const Vec &w = st.w;
      Hs[0] = (std::sqrt(2.0) * w[0] - 1.0) * (std::sqrt(2.0) * w[0] + 1.0);
      int h = 1;
      for (int col = 1; col < dim; ++col) {
        double wc = w[col];
        for (int row = 0; row <= col; ++row) Hs[h++] = 2 * w[row] * wc;
        Hs[h - 1] += 1.0;
      }
      int len = triangular_number(dim);
      for (int i = 0; i < len; ++i) Hs[i] *= e2;
    }
  }
  void mul_Hs(double *y, const double *x, double *) override {
    double c = 2 * dotv(st.w.data(), x, dim);
    for (int i = 0; i < dim; ++i) y[i] = x[i];
    y[0] = -x[0];
    for (int i = 0; i < dim; ++i) y[i] += c * st.w[i];
    double e2 = st.eta * st.eta;
    for (int i = 0; i < dim; ++i) y[i] *= e2;
  }
  void affine_ds(double *ds, const double *) override {
    circ_op(ds, st.lambda.data(), st.lambda.data());
  }
  // coneops_socone.jl:539-566
  void ds_from_dz_offset(double *out, const double *ds, double *,
                         const double *z) override {
    double resz = soc_residual(z, dim);
    double l1ds1 = dotv(st.lambda.data() + 1, ds + 1, dim - 1);
    double w1ds1 = dotv(st.w.data() + 1, ds + 1, dim - 1);
    for (int i = 0; i < dim; ++i) out[i] = -z[i];
    out[0] = z[0];
    double c = st.lambda[0] * ds[0] - l1ds1;
    for (int i = 0; i < dim; ++i) out[i] *= c / resz;
    out[0] += st.eta * w1ds1;
    for (int i = 1; i < dim; ++i)
      out[i] += st.eta * (ds[i] + w1ds1 / (1 + st.w[0]) * st.w[i]);
    double il = 1 / st.lambda[0];
    for (int i = 0; i < dim; ++i) out[i] *= il;
  }
  void step_length(const double *dz, const double *ds, const double *z,
                   const double *s, const oracle_settings &, double amax,
                   double &az, double &as) override {
    az = step_length_soc_component(z, dz, amax, dim);
    as = step_length_soc_component(s, ds, amax, dim);
  }
  double compute_barrier(const double *z, const double *s, const double *dz,
                         const double *ds, double a) override {
    double rs = soc_residual_shifted(s, ds, a, dim);
    double rz = soc_residual_shifted(z, dz, a, dim);
    if (rs > 0 && rz > 0) return -logsafe(rs * rz) / 2;
    return kInf;
  }
  void mul_W(bool, double *y, const double *x, double a, double b) override {
    const Vec &w = st.w;
    double zeta = dotv(w.data() + 1, x + 1, dim - 1);
    double c = x[0] + zeta / (1 + w[0]);
    y[0] = a * st.eta * (w[0] * x[0] + zeta) + b * y[0];
    for (int i = 1; i < dim; ++i)
      y[i] = a * st.eta * (x[i] + c * w[i]) + b * y[i];
  }
  void mul_Winv(bool, double *y, const double *x, double a,
                double b) override {
    const Vec &w = st.w;
    double zeta = dotv(w.data() + 1, x + 1, dim - 1);
    double c = -x[0] + zeta / (1 + w[0]);
    y[0] = (a / st.eta) * (w[0] * x[0] - zeta) + b * y[0];
    for (int i = 1; i < dim; ++i)
      y[i] = (a / st.eta) * (x[i] + c * w[i]) + b * y[i];
  }
  void lambda_inv_circ_op(double *x, const double *z) override {
    const double *y = st.lambda.data();
    double p = soc_residual(y, dim);
    double pinv = 1 / p;
    double v = dotv(y + 1, z + 1, dim - 1);
    x[0] = (y[0] * z[0] - v) * pinv;
    double c = pinv * (v / y[0] - z[0]);
    for (int i = 1; i < dim; ++i) x[i] = c * y[i] + (1 / y[0]) * z[i];
  }
  void circ_op(double *x, const double *y, const double *z) override {
    double y0 = y[0], z0 = z[0];
    double d = dotv(y, z, dim);
    for (int i = 1; i < dim; ++i) x[i] = y0 * z[i] + z0 * y[i];
    x[0] = d;
  }
};

// ------------------------------------------------------------- nonsymmetric
// 3x3 matrices are column-major m[i + 3*j].
static inline double M3(const double *m, int i, int j) { return m[i + 3 * j]; }

// mathutils.jl:381-405
static bool chol3_factor(double *L, const double *A) {
  std::fill(L, L + 9, 0.0);
  double t = M3(A, 0, 0);
  if (t <= 0) return false;
  L[0] = std::sqrt(t);
  L[1] = M3(A, 1, 0) / L[0];
  t = M3(A, 1, 1) - L[1] * L[1];
  if (t <= 0) return false;
  L[4] = std::sqrt(t);
  L[2] = M3(A, 2, 0) / L[0];
  L[5] = (M3(A, 2, 1) - L[1] * L[2]) / L[4];
  t = M3(A, 2, 2) - L[2] * L[2] - L[5] * L[5];
  if (t <= 0) return false;
  L[8] = std::sqrt(t);
  return true;
}
// mathutils.jl:409-420
static void chol3_solve(const double *L, const double *b, double *x) {
  double L11 = L[0], L21 = L[1], L31 = L[2], L22 = L[4], L32 = L[5],
         L33 = L[8];
  double c1 = b[0] / L11;
  double c2 = (b[1] * L11 - b[0] * L21) / (L11 * L22);
  double c3 = (b[2] * L11 * L22 - b[1] * L11 * L32 + b[0] * L21 * L32 -
               b[0] * L22 * L31) /
              (L11 * L22 * L33);
  x[0] = (c1 * L22 * L33 - c2 * L21 * L33 + c3 * L21 * L32 - c3 * L22 * L31) /
         (L11 * L22 * L33);
  x[1] = (c2 * L33 - c3 * L32) / (L22 * L33);
  x[2] = c3 / L33;
}

// coneops_expcone.jl:655-711 (the third Taylor term keeps the reference's
// unassigned "q * zinv" statement, so q is not divided a third time)
static double wright_omega(double z) {
  if (z < 0) throw std::domain_error("argument not in supported range");
  double w;
  if (z < 1.0 + M_PI) {
    double zm1 = z - 1.0;
    double p = zm1;
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
    double logz = logsafe(z);
    double zinv = 1.0 / z;
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

static double newton_raphson_onesided(double x0,
                                      double (*f0)(double, const double *),
                                      double (*f1)(double, const double *),
                                      const double *prm) {
  // coneops_nonsymmetric_common.jl:170-192
  int iter = 0;
  double x = x0;
  while (iter < 100) {
    ++iter;
    double dfdx = f1(x, prm);
    double dx = -f0(x, prm) / dfdx;
    if (dx < kEps || std::fabs(dx / x) < std::sqrt(kEps) ||
        std::fabs(dfdx) < kEps)
      break;
    x += dx;
  }
  return x;
}

struct NonsymCone : Cone {
  double H_dual[9] = {0}, Hs[9] = {0}, grad[3] = {0}, zsave[3] = {0};
  bool is_symmetric() const override { return false; }
  bool Hs_is_diagonal() const override { return false; }
  int numel() const override { return 3; }
  int degree() const override { return 3; }
  virtual void gradient_primal(const double *s, double *g) const = 0;
  virtual void update_dual_grad_H(const double *z) = 0;
  virtual bool is_primal_feasible(const double *s) const = 0;
  virtual bool is_dual_feasible(const double *z) const = 0;
  virtual double barrier_primal(const double *s) const = 0;
  virtual double barrier_dual(const double *z) const = 0;
  virtual void higher_correction(double *eta, const double *ds,
                                 const double *v) = 0;
  void margins(const double *, int, double &, double &) override {
    throw std::logic_error("This function should never be reached.");
  }
  void scaled_unit_shift(double *, double, int) override {
    throw std::logic_error("This function should never be reached.");
  }
  void set_identity_scaling() override {
    throw std::logic_error("This function should never be reached.");
  }
  void use_dual_scaling(double mu) {
    for (int i = 0; i < 9; ++i) Hs[i] = mu * H_dual[i];
  }
  // coneops_nonsymmetric_common.jl:82-164
  void use_primal_dual_scaling(const double *s, const double *z) {
    const double *st = grad;
    double zt[3];
    gradient_primal(s, zt);
    double dot_sz = dotv(z, s, 3);
    double mu = dot_sz / 3;
    double mut = dotv(zt, st, 3) / 3;
    double ds_[3], dz_[3];
    for (int i = 0; i < 3; ++i) {
      ds_[i] = s[i] + mu * st[i];
      dz_[i] = z[i] + mu * zt[i];
    }
    double dot_dsz = dotv(ds_, dz_, 3);
    double de1 = mu * mut - 1;
    double Hz[3];
    for (int i = 0; i < 3; ++i)
      Hz[i] = M3(H_dual, i, 0) * zt[0] + M3(H_dual, i, 1) * zt[1] +
              M3(H_dual, i, 2) * zt[2];
    double de2 = dotv(zt, Hz, 3) - 3 * mut * mut;
    if (std::fabs(de1) > std::sqrt(kEps) && std::fabs(de2) > kEps &&
        dot_sz > 0 && dot_dsz > 0) {
      double tmp[3];
      for (int i = 0; i < 3; ++i) tmp[i] = mut * st[i] - Hz[i];
      for (int i = 0; i < 9; ++i) Hs[i] = H_dual[i];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          Hs[i + 3 * j] -= st[i] * st[j] / 3 + tmp[i] * tmp[j] / de2;
      double fro = 0;
      for (int i = 0; i < 9; ++i) fro += Hs[i] * Hs[i];
      double t = mu * std::sqrt(fro);
      double ax[3];
      ax[0] = z[1] * zt[2] - z[2] * zt[1];
      ax[1] = z[2] * zt[0] - z[0] * zt[2];
      ax[2] = z[0] * zt[1] - z[1] * zt[0];
      double an = norm2(ax, 3);
      for (int i = 0; i < 3; ++i) ax[i] /= an;
      for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j)
          Hs[i + 3 * j] = s[i] * s[j] / dot_sz + ds_[i] * ds_[j] / dot_dsz +
                          t * ax[i] * ax[j];
      Hs[1] = Hs[3];
      Hs[2] = Hs[6];
      Hs[5] = Hs[7];
    } else {
      use_dual_scaling(mu);
    }
  }
  bool update_scaling(const double *s, const double *z, double mu,
                      int strategy) override {
    update_dual_grad_H(z);
    if (strategy == Dual)
      use_dual_scaling(mu);
    else
      use_primal_dual_scaling(s, z);
    for (int i = 0; i < 3; ++i) zsave[i] = z[i];
    return true;
  }
  void get_Hs(double *out) override {
    // pack_triu, mathutils.jl:344
    out[0] = Hs[0];
    out[1] = Hs[3];
    out[2] = Hs[4];
    out[3] = Hs[6];
    out[4] = Hs[7];
    out[5] = Hs[8];
  }
  void mul_Hs(double *y, const double *x, double *) override {
    for (int i = 0; i < 3; ++i)
      y[i] = M3(Hs, i, 0) * x[0] + M3(Hs, i, 1) * x[1] + M3(Hs, i, 2) * x[2];
  }
  void affine_ds(double *ds, const double *s) override {
    for (int i = 0; i < 3; ++i) ds[i] = s[i];
  }
  void combined_ds_shift(double *shift, double *step_z, double *step_s,
                         double sm) override {
    double eta[3] = {0, 0, 0};
    higher_correction(eta, step_s, step_z);
    for (int i = 0; i < 3; ++i) shift[i] = grad[i] * sm - eta[i];
  }
  void ds_from_dz_offset(double *out, const double *ds, double *,
                         const double *) override {
    for (int i = 0; i < 3; ++i) out[i] = ds[i];
  }
  // coneops_nonsymmetric_common.jl:5-34
  template <class F>
  static double backtrack(const double *dq, const double *q, double a0,
                          double amin, double step, F feas) {
    double a = a0, wq[3];
    while (true) {
      for (int i = 0; i < 3; ++i) wq[i] = q[i] + a * dq[i];
      if (feas(wq)) break;
      if ((a *= step) < amin) {
        a = 0;
        break;
      }
    }
    return a;
  }
  void step_length(const double *dz, const double *ds, const double *z,
                   const double *s, const oracle_settings &st, double amax,
                   double &az, double &as) override {
    double step = st.linesearch_backtrack_step;
    double amin = st.min_terminate_step_length;
    az = backtrack(dz, z, amax, amin, step,
                   [this](const double *q) { return is_dual_feasible(q); });
    as = backtrack(ds, s, amax, amin, step,
                   [this](const double *q) { return is_primal_feasible(q); });
  }
  double compute_barrier(const double *z, const double *s, const double *dz,
                         const double *ds, double a) override {
    double cz[3], cs[3];
    for (int i = 0; i < 3; ++i) {
      cz[i] = z[i] + a * dz[i];
      cs[i] = s[i] + a * ds[i];
    }
    return barrier_dual(cz) + barrier_primal(cs);
  }
};

struct ExpCone : NonsymCone {
  int type() const override { return OR_CONE_EXP; }
  void unit_initialization(double *z, double *s) override {
    s[0] = -1.051383945322714;
    s[1] = 0.556409619469370;
    s[2] = 1.258967884768947;
    for (int i = 0; i < 3; ++i) z[i] = s[i];
  }
  double barrier_dual(const double *z) const override {
    double l = logsafe(-z[2] / z[0]);
    return -logsafe(-z[2] * z[0]) - logsafe(z[1] - z[0] - z[0] * l);
  }
  double barrier_primal(const double *s) const override {
    double o = wright_omega(1 - s[0] / s[1] - logsafe(s[1] / s[2]));
    o = (o - 1) * (o - 1) / o;
    return -logsafe(o) - 2 * logsafe(s[1]) - logsafe(s[2]) - 3;
  }
  bool is_primal_feasible(const double *s) const override {
    if (s[2] > 0 && s[1] > 0) {
      double res = s[1] * logsafe(s[2] / s[1]) - s[0];
      if (res > 0) return true;
    }
    return false;
  }
  bool is_dual_feasible(const double *z) const override {
    if (z[2] > 0 && z[0] < 0) {
      double res = z[1] - z[0] - z[0] * logsafe(-z[2] / z[0]);
      if (res > 0) return true;
    }
    return false;
  }
  void gradient_primal(const double *s, double *g) const override {
    double o = wright_omega(1 - s[0] / s[1] - logsafe(s[1] / s[2]));
    g[0] = 1.0 / ((o - 1.0) * s[1]);
    g[1] = g[0] + g[0] * logsafe(o * s[1] / s[2]) - 1.0 / s[1];
    g[2] = o / ((1.0 - o) * s[2]);
  }
  // coneops_expcone.jl:581-610
  void update_dual_grad_H(const double *z) override {
    double l = logsafe(-z[2] / z[0]);
    double r = -z[0] * l - z[0] + z[1];
    double c2 = 1.0 / r;
    grad[0] = c2 * l - 1 / z[0];
    grad[1] = -c2;
    grad[2] = (c2 * z[0] - 1) / z[2];
    double *H = H_dual;
    H[0] = ((r * r - z[0] * r + l * l * z[0] * z[0]) / (r * z[0] * z[0] * r));
    H[3] = (-l / (r * r));
    H[1] = H[3];
    H[4] = (1 / (r * r));
    H[6] = ((z[1] - z[0]) / (r * r * z[2]));
    H[2] = H[6];
    H[7] = (-z[0] / (r * r * z[2]));
    H[5] = H[7];
    H[8] = ((r * r - z[0] * r + z[0] * z[0]) / (r * r * z[2] * z[2]));
  }
  // coneops_expcone.jl:530-577
  void higher_correction(double *eta, const double *ds,
                         const double *v) override {
    double cholH[9];
    if (!chol3_factor(cholH, H_dual)) return;  // eta stays zero
    double u[3];
    chol3_solve(cholH, ds, u);
    const double *z = zsave;
    eta[1] = 1.0;
    eta[2] = -z[0] / z[2];
    eta[0] = logsafe(eta[2]);
    double psi = z[0] * eta[0] - z[0] + z[1];
    double dotpu = dotv(eta, u, 3);
    double dotpv = dotv(eta, v, 3);
    double coef = ((u[0] * (v[0] / z[0] - v[2] / z[2]) +
                    u[2] * (z[0] * v[2] / z[2] - v[0]) / z[2]) *
                       psi -
                   2 * dotpu * dotpv) /
                  (psi * psi * psi);
    for (int i = 0; i < 3; ++i) eta[i] *= coef;
    double inv_psi2 = 1.0 / psi / psi;
    eta[0] += (1 / psi - 2 / z[0]) * u[0] * v[0] / (z[0] * z[0]) -
              u[2] * v[2] / (z[2] * z[2]) / psi +
              dotpu * inv_psi2 * (v[0] / z[0] - v[2] / z[2]) +
              dotpv * inv_psi2 * (u[0] / z[0] - u[2] / z[2]);
    eta[2] += 2 * (z[0] / psi - 1) * u[2] * v[2] / (z[2] * z[2] * z[2]) -
              (u[2] * v[0] + u[0] * v[2]) / (z[2] * z[2]) / psi +
              dotpu * inv_psi2 * (z[0] * v[2] / (z[2] * z[2]) - v[0] / z[2]) +
              dotpv * inv_psi2 * (z[0] * u[2] / (z[2] * z[2]) - u[0] / z[2]);
    for (int i = 0; i < 3; ++i) eta[i] /= 2;
  }
};

static double pow_f0(double x, const double *p) {
  double s3 = p[0], phi = p[1], a = p[2], t0 = p[3];
  double t1 = x * x, t2 = 2 * x / s3;
  return 2 * a * logsafe(2 * a * t1 + (1 + a) * t2) +
         2 * (1 - a) * logsafe(2 * (1 - a) * t1 + (2 - a) * t2) - logsafe(phi) -
         logsafe(t1 + t2) - 2 * logsafe(t2) + t0;
}
static double pow_f1(double x, const double *p) {
  double s3 = p[0], a = p[2];
  double t1 = x * x, t2 = x * 2 / s3;
  return 2 * a * a / (a * x + (1 + a) / s3) +
         2 * (1 - a) * (1 - a) / ((1 - a) * x + (2 - a) / s3) -
         2 * (x + 1 / s3) / (t1 + t2);
}

struct PowCone : NonsymCone {
  double alpha;
  explicit PowCone(double a) : alpha(a) {}
  int type() const override { return OR_CONE_POW; }
  void unit_initialization(double *z, double *s) override {
    s[0] = std::sqrt(1.0 + alpha);
    s[1] = std::sqrt(1.0 + (1.0 - alpha));
    s[2] = 0.0;
    for (int i = 0; i < 3; ++i) z[i] = s[i];
  }
  double barrier_dual(const double *z) const override {
    double a = alpha;
    return -logsafe(std::pow(z[0] / a, 2 * a) *
                        std::pow(z[1] / (1 - a), 2 - 2 * a) -
                    z[2] * z[2]) -
           (1 - a) * logsafe(z[0]) - a * logsafe(z[1]);
  }
  double barrier_primal(const double *s) const override {
    double a = alpha, g[3];
    gradient_primal(s, g);
    return logsafe(std::pow(-g[0] / a, 2 * a) *
                       std::pow(-g[1] / (1 - a), 2 - 2 * a) -
                   g[2] * g[2]) +
           (1 - a) * logsafe(-g[0]) + a * logsafe(-g[1]) - 3;
  }
  bool is_primal_feasible(const double *s) const override {
    double a = alpha;
    if (s[0] > 0 && s[1] > 0) {
      double res = std::exp(2 * a * logsafe(s[0]) + 2 * (1 - a) * logsafe(s[1])) -
                   s[2] * s[2];
      if (res > 0) return true;
    }
    return false;
  }
  bool is_dual_feasible(const double *z) const override {
    double a = alpha;
    if (z[0] > 0 && z[1] > 0) {
      double res = std::exp(2 * a * logsafe(z[0] / a) +
                            2 * (1 - a) * logsafe(z[1] / (1 - a))) -
                   z[2] * z[2];
      if (res > 0) return true;
    }
    return false;
  }
  // coneops_powcone.jl:288-316 and :449-478
  void gradient_primal(const double *s, double *g) const override {
    double a = alpha;
    double phi = std::pow(s[0], 2 * a) * std::pow(s[1], 2 - 2 * a);
    double abs_s = std::fabs(s[2]);
    if (abs_s > kEps) {
      double s3 = abs_s;
      double x0 = -1.0 / s3 + (2 * s3 + std::sqrt(phi * phi / s3 / s3 + 3 * phi)) /
                                  (phi - s3 * s3);
      double t0 = -2 * a * logsafe(a) - 2 * (1 - a) * logsafe(1 - a);
      double prm[4] = {s3, phi, a, t0};
      g[2] = newton_raphson_onesided(x0, pow_f0, pow_f1, prm);
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
  void update_dual_grad_H(const double *z) override {
    double a = alpha;
    double phi = std::pow(z[0] / a, 2 * a) * std::pow(z[1] / (1 - a), 2 - 2 * a);
    double psi = phi - z[2] * z[2];
    double g0 = 2 * a * phi / (z[0] * psi);
    double g1 = 2 * (1 - a) * phi / (z[1] * psi);
    double g2 = -2 * z[2] / psi;
    double *H = H_dual;
    H[0] = g0 * g0 - 2 * a * (2 * a - 1) * phi / (z[0] * z[0] * psi) +
           (1 - a) / (z[0] * z[0]);
    H[3] = g0 * g1 - 4 * a * (1 - a) * phi / (z[0] * z[1] * psi);
    H[1] = H[3];
    H[4] = g1 * g1 - 2 * (1 - a) * (1 - 2 * a) * phi / (z[1] * z[1] * psi) +
           a / (z[1] * z[1]);
    H[6] = g0 * g2;
    H[2] = H[6];
    H[7] = g1 * g2;
    H[5] = H[7];
    H[8] = g2 * g2 + 2 / psi;
    grad[0] = -2 * a * phi / (z[0] * psi) - (1 - a) / z[0];
    grad[1] = -2 * (1 - a) * phi / (z[1] * psi) - a / z[1];
    grad[2] = 2 * z[2] / psi;
  }
  // coneops_powcone.jl:329-404
  void higher_correction(double *eta, const double *ds,
                         const double *v) override {
    double cholH[9];
    if (!chol3_factor(cholH, H_dual)) return;
    double u[3];
    chol3_solve(cholH, ds, u);
    double a = alpha;
    const double *z = zsave;
    double phi = std::pow(z[0] / a, 2 * a) * std::pow(z[1] / (1 - a), 2 - 2 * a);
    double psi = phi - z[2] * z[2];
    eta[0] = 2 * a * phi / z[0];
    eta[1] = 2 * (1 - a) * phi / z[1];
    eta[2] = -2 * z[2];
    double Hp11 = 2 * a * (2 * a - 1) * phi / (z[0] * z[0]);
    double Hp12 = 4 * a * (1 - a) * phi / (z[0] * z[1]);
    double Hp22 = 2 * (1 - a) * (1 - 2 * a) * phi / (z[1] * z[1]);
    double dotpu = dotv(eta, u, 3);
    double dotpv = dotv(eta, v, 3);
    double Hv[3];
    Hv[0] = Hp11 * v[0] + Hp12 * v[1];
    Hv[1] = Hp12 * v[0] + Hp22 * v[1];
    Hv[2] = -2 * v[2];
    double coef = (dotv(u, Hv, 3) * psi - 2 * dotpu * dotpv) / (psi * psi * psi);
    double coef2 = 4 * a * (2 * a - 1) * (1 - a) * phi *
                   (u[0] / z[0] - u[1] / z[1]) * (v[0] / z[0] - v[1] / z[1]) /
                   psi;
    double inv_psi2 = 1 / psi / psi;
    eta[0] = coef * eta[0] - 2 * (1 - a) * u[0] * v[0] / (z[0] * z[0] * z[0]) +
             coef2 / z[0] + Hv[0] * dotpu * inv_psi2;
    eta[1] = coef * eta[1] - 2 * a * u[1] * v[1] / (z[1] * z[1] * z[1]) -
             coef2 / z[1] + Hv[1] * dotpu * inv_psi2;
    eta[2] = coef * eta[2] + Hv[2] * dotpu * inv_psi2;
    double Hu[3];
    Hu[0] = Hp11 * u[0] + Hp12 * u[1];
    Hu[1] = Hp12 * u[0] + Hp22 * u[1];
    Hu[2] = -2 * u[2];
    for (int i = 0; i < 3; ++i) eta[i] = (eta[i] + Hu[i] * dotpv * inv_psi2) / 2;
  }
};

// ------------------------------------------------------------- PSD
// small dense helpers (column-major n x n)
static bool chol_lower(int n, double *A) {  // A <- L (lower), upper zeroed
  for (int j = 0; j < n; ++j) {
    double d = A[j + n * j];
    for (int k = 0; k < j; ++k) d -= A[j + n * k] * A[j + n * k];
    if (!(d > 0)) return false;
    d = std::sqrt(d);
    A[j + n * j] = d;
    for (int i = j + 1; i < n; ++i) {
      double t = A[i + n * j];
      for (int k = 0; k < j; ++k) t -= A[i + n * k] * A[j + n * k];
      A[i + n * j] = t / d;
    }
    for (int i = 0; i < j; ++i) A[i + n * j] = 0;
  }
  return true;
}
// cyclic Jacobi eigenvalues of symmetric A (destroyed); ascending output
static void sym_eigvals(int n, double *A, double *ev) {
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0, tot = 0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        double a = A[i + n * j] * A[i + n * j];
        tot += a;
        if (i != j) off += a;
      }
    if (off <= 1e-30 * tot || off == 0) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = A[p + n * q];
        if (apq == 0) continue;
        double app = A[p + n * p], aqq = A[q + n * q];
        double theta = (aqq - app) / (2 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) /
                   (std::fabs(theta) + std::sqrt(theta * theta + 1));
        double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < n; ++k) {
          double akp = A[k + n * p], akq = A[k + n * q];
          A[k + n * p] = c * akp - s * akq;
          A[k + n * q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          double apk = A[p + n * k], aqk = A[q + n * k];
          A[p + n * k] = c * apk - s * aqk;
          A[q + n * k] = s * apk + c * aqk;
        }
      }
  }
  for (int i = 0; i < n; ++i) ev[i] = A[i + n * i];
  std::sort(ev, ev + n);
}
// one-sided Jacobi SVD: M = U diag(S) V^T (M destroyed, S descending)
static void svd_jacobi(int n, double *M, double *U, double *S, double *V) {
  for (int i = 0; i < n * n; ++i) V[i] = 0;
  for (int i = 0; i < n; ++i) V[i + n * i] = 1;
  for (int sweep = 0; sweep < 100; ++sweep) {
    bool rotated = false;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        double a = 0, b = 0, g = 0;
        for (int k = 0; k < n; ++k) {
          a += M[k + n * p] * M[k + n * p];
          b += M[k + n * q] * M[k + n * q];
          g += M[k + n * p] * M[k + n * q];
        }
        if (std::fabs(g) <= 1e-15 * std::sqrt(a * b) || g == 0) continue;
        rotated = true;
        double zeta = (b - a) / (2 * g);
        double t = (zeta >= 0 ? 1.0 : -1.0) /
                   (std::fabs(zeta) + std::sqrt(1 + zeta * zeta));
        double c = 1 / std::sqrt(1 + t * t), s = c * t;
        for (int k = 0; k < n; ++k) {
          double mp = M[k + n * p], mq = M[k + n * q];
          M[k + n * p] = c * mp - s * mq;
          M[k + n * q] = s * mp + c * mq;
          double vp = V[k + n * p], vq = V[k + n * q];
          V[k + n * p] = c * vp - s * vq;
          V[k + n * q] = s * vp + c * vq;
        }
      }
    if (!rotated) break;
  }
  std::vector<int> idx(n);
  std::vector<double> nr(n);
  for (int j = 0; j < n; ++j) nr[j] = norm2(M + n * j, n);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(),
                   [&](int x, int y) { return nr[x] > nr[y]; });
  std::vector<double> Vt(V, V + n * n), Mt(M, M + n * n);
  for (int jj = 0; jj < n; ++jj) {
    int j = idx[jj];
    S[jj] = nr[j];
    for (int k = 0; k < n; ++k) {
      V[k + n * jj] = Vt[k + n * j];
      U[k + n * jj] = nr[j] > 0 ? Mt[k + n * j] / nr[j] : 0.0;
    }
  }
}

struct PSDCone : SymCone {
  int n, nel;
  Vec R, Rinv, lam, Lis, Hs, W1, W2, W3;
  explicit PSDCone(int nn)
      : n(nn), nel(triangular_number(nn)), R(nn * nn), Rinv(nn * nn),
        lam(nn), Lis(nn), Hs((size_t)triangular_number(nn) * triangular_number(nn)),
        W1(nn * nn), W2(nn * nn), W3(nn * nn) {}
  int type() const override { return OR_CONE_PSD; }
  int numel() const override { return nel; }
  int degree() const override { return n; }
  bool Hs_is_diagonal() const override { return false; }
  // coneops_psdtrianglecone.jl:476-504
  void svec_to_mat(double *M, const double *x) const {
    const double is2 = 1.0 / std::sqrt(2.0);
    int idx = 0;
    for (int col = 0; col < n; ++col)
      for (int row = 0; row <= col; ++row) {
        if (row == col)
          M[row + n * col] = x[idx];
        else {
          M[row + n * col] = x[idx] * is2;
          M[col + n * row] = x[idx] * is2;
        }
        ++idx;
      }
  }
  void mat_to_svec(double *x, const double *M) const {
    const double is2 = 1 / std::sqrt(2.0);
    int idx = 0;
    for (int col = 0; col < n; ++col)
      for (int row = 0; row <= col; ++row) {
        x[idx] = row == col ? M[row + n * col]
                            : (M[row + n * col] + M[col + n * row]) * is2;
        ++idx;
      }
  }
  void margins(const double *z, int, double &a, double &b) override {
    if (nel == 0) {
      a = kMax;
      b = 0;
      return;
    }
    std::vector<double> Z(n * n), e(n);
    svec_to_mat(Z.data(), z);
    sym_eigvals(n, Z.data(), e.data());
    a = e[0];
    b = 0;
    for (double v : e)
      if (v > 0) b += v;
  }
  void scaled_unit_shift(double *z, double a, int) override {
    for (int k = 1; k <= n; ++k) z[triangular_number(k) - 1] += a;
  }
  void unit_initialization(double *z, double *s) override {
    for (int i = 0; i < nel; ++i) z[i] = s[i] = 0;
    scaled_unit_shift(s, 1.0, PrimalCone);
    scaled_unit_shift(z, 1.0, DualCone);
  }
  void set_identity_scaling() override {
    std::fill(R.begin(), R.end(), 0.0);
    for (int i = 0; i < n; ++i) R[i + n * i] = 1;
    Rinv = R;
    std::fill(Hs.begin(), Hs.end(), 0.0);
    for (int i = 0; i < nel; ++i) Hs[i + (size_t)nel * i] = 1;
  }
  // coneops_psdtrianglecone.jl:79-142
  bool update_scaling(const double *s, const double *z, double,
                      int) override {
    if (nel == 0) return true;
    std::vector<double> L1(n * n), L2(n * n), tmp(n * n), U(n * n), V(n * n);
    svec_to_mat(L1.data(), s);
    svec_to_mat(L2.data(), z);
    if (!chol_lower(n, L1.data()) || !chol_lower(n, L2.data())) return false;
    // tmp = L2' * L1
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        double t = 0;
        for (int k = 0; k < n; ++k) t += L2[k + n * i] * L1[k + n * j];
        tmp[i + n * j] = t;
      }
    svd_jacobi(n, tmp.data(), U.data(), lam.data(), V.data());
    for (int i = 0; i < n; ++i) Lis[i] = 1.0 / std::sqrt(lam[i]);
    // R = L1 * V * Lis
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        double t = 0;
        for (int k = 0; k < n; ++k) t += L1[i + n * k] * V[k + n * j];
        R[i + n * j] = t * Lis[j];
      }
    // Rinv = Lis * U' * L2'
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        double t = 0;
        for (int k = 0; k < n; ++k) t += U[k + n * i] * L2[j + n * k];
        Rinv[i + n * j] = Lis[i] * t;
      }
    // RRt
    std::vector<double> RRt(n * n);
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        double t = 0;
        for (int k = 0; k < n; ++k) t += R[i + n * k] * R[j + n * k];
        RRt[i + n * j] = t;
      }
    skron(RRt.data());
    return true;
  }
  // coneops_psdtrianglecone.jl:509-547 (upper triangle of A (x)_s A)
  void skron(const double *A) {
    const double sqrt2 = std::sqrt(2.0);
    auto a = [&](int i, int j) { return A[i + n * j]; };
    int col = 0;
    for (int l = 0; l < n; ++l)
      for (int k = 0; k <= l; ++k) {
        int row = 0;
        bool kl = (k == l);
        for (int j = 0; j < n; ++j) {
          double Ajl = a(j, l), Ajk = a(j, k);
          for (int i = 0; i <= j; ++i) {
            if (row > col) break;
            bool ij = (i == j);
            double v;
            if (!ij && !kl)
              v = a(i, k) * Ajl + a(i, l) * Ajk;
            else if (ij && !kl)
              v = sqrt2 * Ajl * Ajk;
            else if (!ij && kl)
              v = sqrt2 * a(i, l) * Ajk;
            else
              v = Ajl * Ajl;
            Hs[row + (size_t)nel * col] = v;
            ++row;
          }
        }
        ++col;
      }
  }
  void get_Hs(double *out) override {
    int k = 0;
    for (int col = 0; col < nel; ++col)
      for (int row = 0; row <= col; ++row) out[k++] = Hs[row + (size_t)nel * col];
  }
  void mul_Wx_inner(bool trans, double *y, const double *x, double a,
                    double b, const Vec &Rx) {
    double *X = W1.data(), *Y = W2.data(), *T = W3.data();
    svec_to_mat(X, x);
    svec_to_mat(Y, y);
    if (trans) {
      // T = X * Rx';  Y = a*Rx*T + b*Y
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          double t = 0;
          for (int k = 0; k < n; ++k) t += X[i + n * k] * Rx[j + n * k];
          T[i + n * j] = t;
        }
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          double t = 0;
          for (int k = 0; k < n; ++k) t += Rx[i + n * k] * T[k + n * j];
          Y[i + n * j] = a * t + b * Y[i + n * j];
        }
    } else {
      // T = Rx' * X; Y = a*T*Rx + b*Y
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          double t = 0;
          for (int k = 0; k < n; ++k) t += Rx[k + n * i] * X[k + n * j];
          T[i + n * j] = t;
        }
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          double t = 0;
          for (int k = 0; k < n; ++k) t += T[i + n * k] * Rx[k + n * j];
          Y[i + n * j] = a * t + b * Y[i + n * j];
        }
    }
    mat_to_svec(y, Y);
  }
  void mul_W(bool trans, double *y, const double *x, double a,
             double b) override {
    mul_Wx_inner(trans, y, x, a, b, R);
  }
  void mul_Winv(bool trans, double *y, const double *x, double a,
                double b) override {
    mul_Wx_inner(trans, y, x, a, b, Rinv);
  }
  void mul_Hs(double *y, const double *x, double *work) override {
    mul_W(false, work, x, 1.0, 0.0);
    mul_W(true, y, work, 1.0, 0.0);
  }
  void affine_ds(double *ds, const double *) override {
    for (int i = 0; i < nel; ++i) ds[i] = 0;
    for (int k = 1; k <= n; ++k) ds[triangular_number(k) - 1] = lam[k - 1] * lam[k - 1];
  }
  void lambda_inv_circ_op(double *x, const double *z) override {
    double *X = W1.data(), *Z = W2.data();
    svec_to_mat(X, x);
    svec_to_mat(Z, z);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) X[i + n * j] = 2 * Z[i + n * j] / (lam[i] + lam[j]);
    mat_to_svec(x, X);
  }
  void circ_op(double *x, const double *y, const double *z) override {
    double *Y = W1.data(), *Z = W2.data(), *X = W3.data();
    svec_to_mat(Y, y);
    svec_to_mat(Z, z);
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        double t = 0;
        for (int k = 0; k < n; ++k)
          t += Y[i + n * k] * Z[k + n * j] + Z[i + n * k] * Y[k + n * j];
        X[i + n * j] = 0.5 * t;
      }
    mat_to_svec(x, X);
  }
  double step_component(const double *d, double amax) {
    double gamma;
    if (nel == 0)
      gamma = kMax;
    else {
      std::vector<double> M(n * n), e(n);
      svec_to_mat(M.data(), d);
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) M[i + n * j] *= Lis[i] * Lis[j];
      sym_eigvals(n, M.data(), e.data());
      gamma = e[0];
    }
    if (gamma < 0) return std::min(1.0 / (-gamma), amax);
    return amax;
  }
  void step_length(const double *dz, const double *ds, const double *,
                   const double *, const oracle_settings &, double amax,
                   double &az, double &as) override {
    std::vector<double> d(nel);
    mul_W(false, d.data(), dz, 1.0, 0.0);
    az = step_component(d.data(), amax);
    mul_Winv(true, d.data(), ds, 1.0, 0.0);
    as = step_component(d.data(), amax);
  }
  double logdet_barrier(const double *x, const double *dx, double a) {
    std::vector<double> q(nel), Q(n * n);
    for (int i = 0; i < nel; ++i) q[i] = x[i] + a * dx[i];
    svec_to_mat(Q.data(), q.data());
    if (!chol_lower(n, Q.data())) return kInf;
    double ld = 0;
    for (int i = 0; i < n; ++i) ld += 2 * std::log(Q[i + n * i]);
    return ld;
  }
  double compute_barrier(const double *z, const double *s, const double *dz,
                         const double *ds, double a) override {
    double bar = 0;
    bar -= logdet_barrier(z, dz, a);
    bar -= logdet_barrier(s, ds, a);
    return bar;
  }
};

std::unique_ptr<Cone> make_cone(int type, int dim, double param) {
  switch (type) {
    case OR_CONE_ZERO: return std::make_unique<ZeroCone>(dim);
    case OR_CONE_NONNEG: return std::make_unique<NNCone>(dim);
    case OR_CONE_SOC: return std::make_unique<SOCCone>(dim);
    case OR_CONE_EXP: return std::make_unique<ExpCone>();
    case OR_CONE_POW: return std::make_unique<PowCone>(param);
    case OR_CONE_PSD: return std::make_unique<PSDCone>(dim);
  }
  throw std::invalid_argument("unknown cone type");
}

SOCState *soc_state(Cone *c) {
  auto *s = dynamic_cast<SOCCone *>(c);
  return s ? &s->st : nullptr;
}
NNStateView nn_state(Cone *c) {
  auto *s = dynamic_cast<NNCone *>(c);
  NNStateView v{nullptr, nullptr};
  if (s) {
    v.w = &s->w;
    v.lambda = &s->lambda;
  }
  return v;
}
void psd_lambda(Cone *c, double *out) {
  auto *p = dynamic_cast<PSDCone *>(c);
  if (p)
    for (int i = 0; i < p->n; ++i) out[i] = p->lam[i];
}

// ------------------------------------------------------------- composite
// src/cones/compositecone_type.jl and coneops_compositecone.jl
void CompositeCone::build(int ncones, const int *types, const int *dims,
                          const double *params) {
  cones.clear();
  rng_start.clear();
  rng_len.clear();
  blk_start.clear();
  blk_len.clear();
  numel = degree = hs_len = 0;
  symmetric = true;
  for (int i = 0; i < ncones; ++i) {
    cones.push_back(make_cone(types[i], dims[i], params ? params[i] : 0.0));
    Cone *c = cones.back().get();
    symmetric = symmetric && c->is_symmetric();
    rng_start.push_back(numel);
    rng_len.push_back(c->numel());
    blk_start.push_back(hs_len);
    blk_len.push_back(c->hs_block_len());
    numel += c->numel();
    degree += c->degree();
    hs_len += c->hs_block_len();
  }
}
bool CompositeCone::rectify_equilibration(double *delta, const double *e) {
  bool any = false;
  for (int i = 0; i < numel; ++i) delta[i] = 1;
  for (size_t k = 0; k < cones.size(); ++k)
    any |= cones[k]->rectify_equilibration(delta + rng_start[k], e + rng_start[k]);
  return any;
}
void CompositeCone::margins(const double *z, int pd, double &a, double &b) {
  a = kMax;
  b = 0;
  for (size_t k = 0; k < cones.size(); ++k) {
    double ai, bi;
    cones[k]->margins(z + rng_start[k], pd, ai, bi);
    a = std::min(a, ai);
    b += bi;
  }
}
void CompositeCone::scaled_unit_shift(double *z, double a, int pd) {
  for (size_t k = 0; k < cones.size(); ++k)
    cones[k]->scaled_unit_shift(z + rng_start[k], a, pd);
}
void CompositeCone::unit_initialization(double *z, double *s) {
  for (size_t k = 0; k < cones.size(); ++k)
    cones[k]->unit_initialization(z + rng_start[k], s + rng_start[k]);
}
void CompositeCone::set_identity_scaling() {
  for (auto &c : cones) c->set_identity_scaling();
}
bool CompositeCone::update_scaling(const double *s, const double *z, double mu,
                                   int strategy) {
  for (size_t k = 0; k < cones.size(); ++k)
    if (!cones[k]->update_scaling(s + rng_start[k], z + rng_start[k], mu, strategy))
      return false;
  return true;
}
void CompositeCone::get_Hs(double *Hs) {
  for (size_t k = 0; k < cones.size(); ++k) cones[k]->get_Hs(Hs + blk_start[k]);
}
void CompositeCone::mul_Hs(double *y, const double *x, double *work) {
  for (size_t k = 0; k < cones.size(); ++k)
    cones[k]->mul_Hs(y + rng_start[k], x + rng_start[k], work + rng_start[k]);
}
void CompositeCone::affine_ds(double *ds, const double *s) {
  for (size_t k = 0; k < cones.size(); ++k)
    cones[k]->affine_ds(ds + rng_start[k], s + rng_start[k]);
}
void CompositeCone::combined_ds_shift(double *shift, double *step_z,
                                      double *step_s, double sm) {
  for (size_t k = 0; k < cones.size(); ++k)
    cones[k]->combined_ds_shift(shift + rng_start[k], step_z + rng_start[k],
                                step_s + rng_start[k], sm);
}
void CompositeCone::ds_from_dz_offset(double *out, const double *ds,
                                      double *work, const double *z) {
  for (size_t k = 0; k < cones.size(); ++k)
    cones[k]->ds_from_dz_offset(out + rng_start[k], ds + rng_start[k],
                                work + rng_start[k], z + rng_start[k]);
}
// coneops_compositecone.jl:471-508: symmetric cones first, then cap at
// max_step_fraction if any cone is asymmetric, then the asymmetric cones.
void CompositeCone::step_length(const double *dz, const double *ds,
                                const double *z, const double *s,
                                const oracle_settings &st, double amax,
                                double &az, double &as) {
  double a = amax;
  auto inner = [&](bool want_sym) {
    for (size_t k = 0; k < cones.size(); ++k) {
      if (cones[k]->is_symmetric() != want_sym) continue;
      int o = rng_start[k];
      double nz, ns;
      cones[k]->step_length(dz + o, ds + o, z + o, s + o, st, a, nz, ns);
      a = std::min(a, std::min(nz, ns));
    }
  };
  inner(true);
  if (!symmetric) a = std::min(a, st.max_step_fraction);
  inner(false);
  az = as = a;
}
double CompositeCone::compute_barrier(const double *z, const double *s,
                                      const double *dz, const double *ds,
                                      double a) {
  double b = 0;
  for (size_t k = 0; k < cones.size(); ++k) {
    int o = rng_start[k];
    b += cones[k]->compute_barrier(z + o, s + o, dz + o, ds + o, a);
  }
  return b;
}

}  // namespace orc
