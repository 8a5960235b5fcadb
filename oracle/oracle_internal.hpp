// oracle_internal.hpp -- shared declarations for the CPU oracle.
// TEST INFRASTRUCTURE ONLY (see clarabel_oracle.h).
#pragma once
#include <cmath>
#include <cstdint>
#include <limits>
#include <memory>
#include <vector>

#include "clarabel_oracle.h"

namespace orc {

using Vec = std::vector<double>;
constexpr double kInf = std::numeric_limits<double>::infinity();
constexpr double kMax = std::numeric_limits<double>::max();
constexpr double kEps = 2.220446049250313e-16;

enum ScalingStrategy { PrimalDual = 0, Dual = 1 };
enum PrimalOrDual { PrimalCone = 0, DualCone = 1 };

// src/utils/mathutils.jl:12 logsafe
inline double logsafe(double v) { return v < 0 ? -kMax : std::log(v); }
inline double clip(double s, double lo, double hi) {
  return s < lo ? lo : (s > hi ? hi : s);
}
inline int triangular_number(int k) { return (k * (k + 1)) >> 1; }

struct Settings {
  oracle_settings s;
};

// ---------------------------------------------------------------- cones
// Mirrors the per-cone API of src/cones/coneops_defaults.jl.
struct Cone {
  virtual ~Cone() {}
  virtual int type() const = 0;
  virtual int numel() const = 0;
  virtual int degree() const = 0;
  virtual bool is_symmetric() const { return true; }
  virtual bool is_sparse_expandable() const { return false; }
  virtual bool Hs_is_diagonal() const { return true; }
  // coneops_defaults.jl:32 (default) ; zero/NN override to "no change"
  virtual bool rectify_equilibration(double *delta, const double *e);
  virtual void margins(const double *z, int pd, double &a, double &b) = 0;
  virtual void scaled_unit_shift(double *z, double a, int pd) = 0;
  virtual void unit_initialization(double *z, double *s) = 0;
  virtual void set_identity_scaling() = 0;
  virtual bool update_scaling(const double *s, const double *z, double mu,
                              int strategy) = 0;
  virtual void get_Hs(double *Hs) = 0;
  virtual void mul_Hs(double *y, const double *x, double *work) = 0;
  virtual void affine_ds(double *ds, const double *s) = 0;
  virtual void combined_ds_shift(double *shift, double *step_z,
                                 double *step_s, double sm) = 0;
  virtual void ds_from_dz_offset(double *out, const double *ds, double *work,
                                 const double *z) = 0;
  virtual void step_length(const double *dz, const double *ds,
                           const double *z, const double *s,
                           const oracle_settings &st, double amax,
                           double &az, double &as) = 0;
  virtual double compute_barrier(const double *z, const double *s,
                                 const double *dz, const double *ds,
                                 double a) = 0;
  int hs_block_len() const {
    return Hs_is_diagonal() ? numel() : triangular_number(numel());
  }
};

std::unique_ptr<Cone> make_cone(int type, int dim, double param);

struct CompositeCone {
  std::vector<std::unique_ptr<Cone>> cones;
  std::vector<int> rng_start, rng_len;      // s/z ranges
  std::vector<int> blk_start, blk_len;      // Hs block ranges
  int numel = 0, degree = 0, hs_len = 0;
  bool symmetric = true;
  void build(int ncones, const int *types, const int *dims,
             const double *params);
  bool rectify_equilibration(double *delta, const double *e);
  void margins(const double *z, int pd, double &a, double &b);
  void scaled_unit_shift(double *z, double a, int pd);
  void unit_initialization(double *z, double *s);
  void set_identity_scaling();
  bool update_scaling(const double *s, const double *z, double mu,
                      int strategy);
  void get_Hs(double *Hs);
  void mul_Hs(double *y, const double *x, double *work);
  void affine_ds(double *ds, const double *s);
  void combined_ds_shift(double *shift, double *step_z, double *step_s,
                         double sm);
  void ds_from_dz_offset(double *out, const double *ds, double *work,
                         const double *z);
  void step_length(const double *dz, const double *ds, const double *z,
                   const double *s, const oracle_settings &st, double amax,
                   double &az, double &as);
  double compute_barrier(const double *z, const double *s, const double *dz,
                         const double *ds, double a);
  bool allows_primal_dual_scaling() const { return true; }
};

// SOC state exposed for tests and KKT sparse expansion
struct SOCState {
  Vec w, lambda;
  double eta = 1;
  bool sparse = false;
  double d = 0.5;
  Vec u, v;
};
SOCState *soc_state(Cone *c);
struct NNStateView {
  const Vec *w, *lambda;
};
NNStateView nn_state(Cone *c);
void psd_lambda(Cone *c, double *out);  // n eigen-scalings

// ---------------------------------------------------------------- LDL
// Up-looking LDL^T of a symmetric matrix given by its upper triangle in CSC,
// restating QDLDL's published algorithm (etree + up-looking row solves +
// sign-aware dynamic regularisation).
struct LDL {
  int n = 0;
  std::vector<int> perm, iperm;           // ordering
  std::vector<int> Ap, Ai;                // permuted triu pattern
  std::vector<int> mapK;                  // KKT nz index -> permuted nz index
  std::vector<double> Ax;                 // permuted triu values
  std::vector<int> etree, Lnz, Lp, Li;
  std::vector<double> Lx, D, Dinv;
  std::vector<int> Dsigns;                // permuted signs
  bool reg_enable = true;
  bool round_fp32 = false;
  bool arith_fp32 = false;  // the elimination itself in FP32 arithmetic
  double reg_eps = 1e-13, reg_delta = 2e-7;
  int reg_count = 0;
  // workspaces
  std::vector<int> iwork, bwork, yidx, ebuf, nextcol;
  std::vector<double> fwork;
  void setup(int n, const std::vector<int> &Kp, const std::vector<int> &Ki,
             const std::vector<int> &Dsigns_unperm);
  void update_values(const std::vector<int> &kidx, const double *vals,
                     int count);
  void update_value(int kidx, double v);
  void scale_values(const std::vector<int> &kidx, double scale, int count);
  bool refactor();
  bool refactor_fp32();
  void solve(double *x) const;  // in place
};

// minimum-degree ordering of a symmetric pattern (upper CSC incl diag)
std::vector<int> min_degree_order(int n, const std::vector<int> &Kp,
                                  const std::vector<int> &Ki);

}  // namespace orc
