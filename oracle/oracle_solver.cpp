// oracle_solver.cpp -- CPU restatement of Clarabel's IPM driver and KKT path.
// TEST INFRASTRUCTURE ONLY (see clarabel_oracle.h).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <stdexcept>

#include "oracle_internal.hpp"

namespace orc {

struct CSC {
  int m = 0, n = 0;
  std::vector<int> p, i;
  Vec x;
  int nnz() const { return p.empty() ? 0 : p[n]; }
};

// y = alpha*A*x + beta*y
static void csc_mul(const CSC &A, const double *x, double *y, double alpha,
                    double beta) {
  for (int r = 0; r < A.m; ++r) y[r] *= beta;
  for (int j = 0; j < A.n; ++j)
    for (int k = A.p[j]; k < A.p[j + 1]; ++k) y[A.i[k]] += alpha * A.x[k] * x[j];
}
// y = alpha*A'*x + beta*y
static void csc_mul_t(const CSC &A, const double *x, double *y, double alpha,
                      double beta) {
  for (int j = 0; j < A.n; ++j) {
    double t = 0;
    for (int k = A.p[j]; k < A.p[j + 1]; ++k) t += A.x[k] * x[A.i[k]];
    y[j] = alpha * t + beta * y[j];
  }
}
// y = Sym(triu A) * x
static void csc_symv_triu(const CSC &A, const double *x, double *y) {
  for (int r = 0; r < A.n; ++r) y[r] = 0;
  for (int j = 0; j < A.n; ++j)
    for (int k = A.p[j]; k < A.p[j + 1]; ++k) {
      int i = A.i[k];
      y[i] += A.x[k] * x[j];
      if (i != j) y[j] += A.x[k] * x[i];
    }
}
static double dot(const double *a, const double *b, int n) {
  double t = 0;
  for (int i = 0; i < n; ++i) t += a[i] * b[i];
  return t;
}
static double norm_inf(const double *a, int n) {
  double t = 0;
  for (int i = 0; i < n; ++i) t = std::max(t, std::fabs(a[i]));
  return t;
}
static double norm_scaled(const Vec &m, const double *v, int n) {
  double t = 0;
  for (int i = 0; i < n; ++i) {
    double p = m[i] * v[i];
    t += p * p;
  }
  return std::sqrt(t);
}

struct Variables {
  Vec x, s, z;
  double tau = 1, kappa = 1;
  void init(int n, int m) {
    x.assign(n, 0);
    s.assign(m, 0);
    z.assign(m, 0);
  }
};

struct Residuals {
  Vec rx, rz, rx_inf, rz_inf, Px;
  double rtau = 0, dot_qx = 0, dot_bz = 0, dot_sz = 0, dot_xPx = 0;
};

struct Equil {
  Vec d, dinv, e, einv;
  double c = 1;
};

// --------------------------------------------------------- KKT (triu)
// src/kktsolvers/direct-ldl/directldl_kkt_assembly.jl + directldl_datamaps.jl
struct KKTMaps {
  std::vector<int> P, A, Hsblocks, diag_full;
  struct SOCMap {
    int cone;
    std::vector<int> u, v;
    int D[2];
  };
  std::vector<SOCMap> soc;
};

struct KKTSolver {
  int m, n, p;
  CSC K;  // triu
  KKTMaps map;
  std::vector<int> Dsigns;
  Vec Hsblocks, xsol, b, work1, work2;
  LDL ldl;
  const oracle_settings *st;
  CompositeCone *cones;
  double diag_reg = 0;
  // refinement statistics of the last solve loop: solves, sweeps, solves
  // that ended above the tolerance, and the worst final |e| / tolerance
  int ir_solves = 0, ir_sweeps = 0, ir_unconverged = 0;
  double ir_worst = 0;

  void assemble(const CSC &P, const CSC &A, CompositeCone &C) {
    cones = &C;
    m = A.m;
    n = P.n;
    int nsoc = 0;
    for (auto &c : C.cones)
      if (c->is_sparse_expandable()) ++nsoc;
    p = 2 * nsoc;
    int N = n + m + p;
    // rows of A per row (A^T columns)
    std::vector<std::vector<std::pair<int, int>>> arow(m);
    for (int j = 0; j < A.n; ++j)
      for (int k = A.p[j]; k < A.p[j + 1]; ++k) arow[A.i[k]].push_back({j, k});
    // column lists (row, tag) where tag encodes the source
    // tag >=0 : P nz index; tag = -1-kA : A nz; special codes via vectors
    K.m = K.n = N;
    K.p.assign(N + 1, 0);
    std::vector<std::vector<int>> colrows(N);
    std::vector<std::vector<int>> colsrc(N);  // 0=P,1=A,2=Hs,3=soc u/v,4=diag
    std::vector<std::vector<int>> colidx(N);
    map.P.assign(P.nnz(), -1);
    map.A.assign(A.nnz(), -1);
    map.Hsblocks.assign(C.hs_len, -1);
    for (int j = 0; j < n; ++j) {
      bool hasdiag = false;
      for (int k = P.p[j]; k < P.p[j + 1]; ++k) {
        colrows[j].push_back(P.i[k]);
        colsrc[j].push_back(0);
        colidx[j].push_back(k);
        if (P.i[k] == j) hasdiag = true;
      }
      if (!hasdiag) {
        colrows[j].push_back(j);
        colsrc[j].push_back(4);
        colidx[j].push_back(j);
      }
    }
    for (int r = 0; r < m; ++r)
      for (auto &pr : arow[r]) {
        colrows[n + r].push_back(pr.first);
        colsrc[n + r].push_back(1);
        colidx[n + r].push_back(pr.second);
      }
    int pcol = n + m;
    for (size_t ci = 0; ci < C.cones.size(); ++ci) {
      Cone *c = C.cones[ci].get();
      int row0 = C.rng_start[ci] + n, dim = c->numel(), b0 = C.blk_start[ci];
      if (c->Hs_is_diagonal()) {
        for (int k = 0; k < dim; ++k) {
          colrows[row0 + k].push_back(row0 + k);
          colsrc[row0 + k].push_back(2);
          colidx[row0 + k].push_back(b0 + k);
        }
      } else {
        int h = b0;
        for (int col = 0; col < dim; ++col)
          for (int row = 0; row <= col; ++row) {
            colrows[row0 + col].push_back(row0 + row);
            colsrc[row0 + col].push_back(2);
            colidx[row0 + col].push_back(h++);
          }
      }
      if (c->is_sparse_expandable()) {
        KKTMaps::SOCMap sm;
        sm.cone = (int)ci;
        sm.u.assign(dim, -1);
        sm.v.assign(dim, -1);
        for (int k = 0; k < dim; ++k) {
          colrows[pcol].push_back(row0 + k);  // v column
          colsrc[pcol].push_back(3);
          colidx[pcol].push_back(((int)map.soc.size() << 20) | (k << 1) | 0);
          colrows[pcol + 1].push_back(row0 + k);  // u column
          colsrc[pcol + 1].push_back(3);
          colidx[pcol + 1].push_back(((int)map.soc.size() << 20) | (k << 1) | 1);
        }
        colrows[pcol].push_back(pcol);
        colsrc[pcol].push_back(5);
        colidx[pcol].push_back(((int)map.soc.size() << 1) | 0);
        colrows[pcol + 1].push_back(pcol + 1);
        colsrc[pcol + 1].push_back(5);
        colidx[pcol + 1].push_back(((int)map.soc.size() << 1) | 1);
        map.soc.push_back(sm);
        pcol += 2;
      }
    }
    for (int j = 0; j < N; ++j) K.p[j + 1] = K.p[j] + (int)colrows[j].size();
    K.i.assign(K.p[N], 0);
    K.x.assign(K.p[N], 0.0);
    map.diag_full.assign(N, -1);
    for (int j = 0; j < N; ++j) {
      int q = K.p[j];
      for (size_t t = 0; t < colrows[j].size(); ++t, ++q) {
        int r = colrows[j][t];
        K.i[q] = r;
        int src = colsrc[j][t], id = colidx[j][t];
        if (src == 0) {
          map.P[id] = q;
          K.x[q] = P.x[id];
        } else if (src == 1) {
          map.A[id] = q;
          K.x[q] = A.x[id];
        } else if (src == 2) {
          map.Hsblocks[id] = q;
        } else if (src == 3) {
          int s = id >> 20, k = (id >> 1) & 0x7ffff, uv = id & 1;
          if (uv) map.soc[s].u[k] = q;
          else map.soc[s].v[k] = q;
        } else if (src == 5) {
          map.soc[id >> 1].D[id & 1] = q;
        }
        if (r == j) map.diag_full[j] = q;
      }
    }
    Dsigns.assign(N, 1);
    for (int i = n; i < n + m; ++i) Dsigns[i] = -1;
    for (int k = 0; k < nsoc; ++k) {
      Dsigns[n + m + 2 * k] = -1;
      Dsigns[n + m + 2 * k + 1] = 1;
    }
    Hsblocks.assign(C.hs_len, 0.0);
    xsol.assign(N, 0.0);
    b.assign(N, 0.0);
    work1.assign(N, 0.0);
    work2.assign(N, 0.0);
    ldl.reg_enable = st->dynamic_regularization_enable != 0;
    ldl.reg_eps = st->dynamic_regularization_eps;
    ldl.reg_delta = st->dynamic_regularization_delta;
    ldl.round_fp32 = st->factor_fp32 != 0;
    ldl.arith_fp32 = st->factor_fp32 == 2;
    ldl.setup(N, K.p, K.i, Dsigns);
    for (int q = 0; q < K.p[N]; ++q) ldl.Ax[ldl.mapK[q]] = K.x[q];
  }

  void set_values(const std::vector<int> &idx, const double *v, int cnt) {
    for (int i = 0; i < cnt; ++i) K.x[idx[i]] = v[i];
    ldl.update_values(idx, v, cnt);
  }

  // kktsolver_directldl.jl:213-296
  bool update() {
    cones->get_Hs(Hsblocks.data());
    for (double &h : Hsblocks) h *= -1.0;
    set_values(map.Hsblocks, Hsblocks.data(), (int)Hsblocks.size());
    for (auto &sm : map.soc) {
      SOCState *ss = soc_state(cones->cones[sm.cone].get());
      double e2 = ss->eta * ss->eta;
      int dim = (int)sm.u.size();
      set_values(sm.u, ss->u.data(), dim);
      set_values(sm.v, ss->v.data(), dim);
      for (int k = 0; k < dim; ++k) {
        K.x[sm.u[k]] *= -e2;
        K.x[sm.v[k]] *= -e2;
      }
      ldl.scale_values(sm.u, -e2, dim);
      ldl.scale_values(sm.v, -e2, dim);
      double dv[2] = {-e2, e2};
      std::vector<int> di = {sm.D[0], sm.D[1]};
      set_values(di, dv, 2);
    }
    return regularize_and_refactor();
  }

  bool regularize_and_refactor() {
    int N = n + m + p;
    Vec diag_kkt(N), diag_shift(N);
    if (st->static_regularization_enable) {
      for (int i = 0; i < N; ++i) diag_kkt[i] = K.x[map.diag_full[i]];
      double maxdiag = norm_inf(diag_kkt.data(), N);
      double eps = st->static_regularization_constant +
                   st->static_regularization_proportional * maxdiag;
      for (int i = 0; i < N; ++i)
        diag_shift[i] = diag_kkt[i] + (Dsigns[i] == 1 ? eps : -eps);
      set_values(map.diag_full, diag_shift.data(), N);
      diag_reg = eps;
    }
    bool ok = ldl.refactor();
    if (st->static_regularization_enable)
      for (int i = 0; i < N; ++i) K.x[map.diag_full[i]] = diag_kkt[i];
    return ok;
  }

  void setrhs(const double *rx, const double *rz) {
    for (int i = 0; i < n; ++i) b[i] = rx[i];
    for (int i = 0; i < m; ++i) b[n + i] = rz[i];
    for (int i = n + m; i < n + m + p; ++i) b[i] = 0;
  }

  double refine_error(Vec &e, const Vec &xi) {
    int N = n + m + p;
    csc_symv_triu(K, xi.data(), e.data());
    for (int i = 0; i < N; ++i) e[i] = b[i] - e[i];
    return norm_inf(e.data(), N);
  }

  // kktsolver_directldl.jl:348-451
  bool solve(double *lhsx, double *lhsz) {
    int N = n + m + p;
    xsol = b;
    ldl.solve(xsol.data());
    bool ok;
    if (st->iterative_refinement_enable) {
      Vec &e = work1, &dx = work2;
      double normb = norm_inf(b.data(), N);
      double norme = refine_error(e, xsol);
      if (!std::isfinite(norme)) return false;
      const double tol = st->iterative_refinement_abstol +
                         st->iterative_refinement_reltol * normb;
      double final_e = norme;
      for (int it = 0; it < st->iterative_refinement_max_iter; ++it) {
        if (norme <= tol) break;
        double last = norme;
        dx = e;
        ldl.solve(dx.data());
        ++ir_sweeps;
        for (int i = 0; i < N; ++i) dx[i] += xsol[i];
        norme = refine_error(e, dx);
        if (!std::isfinite(norme)) return false;
        double ratio = last / norme;
        if (ratio < st->iterative_refinement_stop_ratio) {
          if (ratio > 1.0) std::swap(xsol, dx);
          final_e = ratio > 1.0 ? norme : last;
          norme = final_e;
          break;
        }
        std::swap(xsol, dx);
        final_e = norme;
      }
      ++ir_solves;
      if (final_e > tol) {
        ++ir_unconverged;
        ir_worst = std::max(ir_worst, final_e / tol);
      }
      ok = true;
    } else {
      ok = true;
      for (int i = 0; i < N; ++i)
        if (!std::isfinite(xsol[i])) ok = false;
    }
    if (ok) {
      if (lhsx) std::copy(xsol.begin(), xsol.begin() + n, lhsx);
      if (lhsz) std::copy(xsol.begin() + n, xsol.begin() + n + m, lhsz);
    }
    return ok;
  }
};

// --------------------------------------------------------- solver
struct Solver {
  oracle_settings st;
  int n = 0, m = 0;
  CSC P, A;  // P triu, equilibrated in place
  Vec q, b;
  double normq = 0, normb = 0;
  Equil eq;
  CompositeCone cones;
  Variables vars, step_rhs, step_lhs, prev_vars;
  Residuals res;
  KKTSolver kkt;
  Vec x1, z1, x2, z2, workx, workz, work_conic;
  oracle_info info{};
  double prev_cost_primal = kInf, prev_cost_dual = kInf, prev_res_primal = kInf,
         prev_res_dual = kInf, prev_gap_abs = kInf, prev_gap_rel = kInf;
  std::chrono::steady_clock::time_point t0;

  // problemdata.jl:196-284 (Ruiz, CPU semantics)
  void equilibrate() {
    eq.d.assign(n, 1.0);
    eq.dinv.assign(n, 1.0);
    eq.e.assign(m, 1.0);
    eq.einv.assign(m, 1.0);
    eq.c = 1.0;
    if (!st.equilibrate_enable) return;
    Vec &dwork = eq.dinv, &ework = eq.einv;
    double smin = st.equilibrate_min_scaling, smax = st.equilibrate_max_scaling;
    for (int it = 0; it < st.equilibrate_max_iter; ++it) {
      // kkt_col_norms!: col_norms_sym(P), then A col norms, A row norms
      std::fill(dwork.begin(), dwork.end(), 0.0);
      for (int j = 0; j < n; ++j)
        for (int k = P.p[j]; k < P.p[j + 1]; ++k) {
          double t = std::fabs(P.x[k]);
          int r = P.i[k];
          dwork[j] = std::max(dwork[j], t);
          dwork[r] = std::max(dwork[r], t);
        }
      for (int j = 0; j < n; ++j)
        for (int k = A.p[j]; k < A.p[j + 1]; ++k)
          dwork[j] = std::max(dwork[j], std::fabs(A.x[k]));
      std::fill(ework.begin(), ework.end(), 0.0);
      for (int k = 0; k < A.nnz(); ++k)
        ework[A.i[k]] = std::max(ework[A.i[k]], std::fabs(A.x[k]));
      for (auto &v : dwork) v = (v == 0.0) ? 1.0 : v;
      for (auto &v : ework) v = (v == 0.0) ? 1.0 : v;
      for (auto &v : dwork) v = 1.0 / std::sqrt(v);
      for (auto &v : ework) v = 1.0 / std::sqrt(v);
      for (int i = 0; i < n; ++i) dwork[i] = clip(dwork[i], smin / eq.d[i], smax / eq.d[i]);
      for (int i = 0; i < m; ++i) ework[i] = clip(ework[i], smin / eq.e[i], smax / eq.e[i]);
      scale_data(&dwork, ework);
      for (int i = 0; i < n; ++i) eq.d[i] *= dwork[i];
      for (int i = 0; i < m; ++i) eq.e[i] *= ework[i];
      // col_norms!(dwork, P): triu column norms (CPU path), or the row norms
      // of the full symmetric P (GPU path, row_norms_gpu!)
      std::fill(dwork.begin(), dwork.end(), 0.0);
      for (int j = 0; j < n; ++j)
        for (int k = P.p[j]; k < P.p[j + 1]; ++k) {
          dwork[j] = std::max(dwork[j], std::fabs(P.x[k]));
          if (st.gpu_equilibration) dwork[P.i[k]] = std::max(dwork[P.i[k]], std::fabs(P.x[k]));
        }
      double mean = 0;
      for (double v : dwork) mean += v;
      mean /= n;
      double inf_q = norm_inf(q.data(), n);
      if (mean != 0.0 && inf_q != 0.0) {
        double sc = std::max(inf_q, mean);
        double ct = clip(1.0 / sc, smin / eq.c, smax / eq.c);
        for (auto &v : P.x) v *= ct;
        for (auto &v : q) v *= ct;
        eq.c *= ct;
      }
    }
    if (cones.rectify_equilibration(ework.data(), eq.e.data())) {
      scale_data(nullptr, ework);
      for (int i = 0; i < m; ++i) eq.e[i] *= ework[i];
    }
    for (int i = 0; i < n; ++i) eq.dinv[i] = 1.0 / eq.d[i];
    for (int i = 0; i < m; ++i) eq.einv[i] = 1.0 / eq.e[i];
  }
  void scale_data(const Vec *d, const Vec &e) {
    if (d) {
      for (int j = 0; j < n; ++j)
        for (int k = P.p[j]; k < P.p[j + 1]; ++k)
          P.x[k] *= (*d)[P.i[k]] * (*d)[j];
      for (int j = 0; j < n; ++j)
        for (int k = A.p[j]; k < A.p[j + 1]; ++k)
          A.x[k] *= e[A.i[k]] * (*d)[j];
      for (int i = 0; i < n; ++i) q[i] *= (*d)[i];
    } else {
      for (int k = 0; k < A.nnz(); ++k) A.x[k] *= e[A.i[k]];
    }
    for (int i = 0; i < m; ++i) b[i] *= e[i];
  }

  // residuals.jl:1-37
  void residuals_update() {
    const Variables &v = vars;
    res.dot_qx = dot(q.data(), v.x.data(), n);
    res.dot_bz = dot(b.data(), v.z.data(), m);
    res.dot_sz = dot(v.s.data(), v.z.data(), m);
    csc_symv_triu(P, v.x.data(), res.Px.data());
    res.dot_xPx = dot(v.x.data(), res.Px.data(), n);
    csc_mul_t(A, v.z.data(), res.rx_inf.data(), -1.0, 0.0);
    for (int i = 0; i < m; ++i) res.rz_inf[i] = v.s[i];
    csc_mul(A, v.x.data(), res.rz_inf.data(), 1.0, 1.0);
    for (int i = 0; i < n; ++i)
      res.rx[i] = res.rx_inf[i] - res.Px[i] - q[i] * v.tau;
    for (int i = 0; i < m; ++i) res.rz[i] = res.rz_inf[i] - b[i] * v.tau;
    res.rtau = res.dot_qx + res.dot_bz + v.kappa + res.dot_xPx / v.tau;
  }

  // info.jl:1-64
  void info_update() {
    double tinv = 1.0 / vars.tau;
    double cinv = 1.0 / eq.c;
    double xPx = res.dot_xPx * tinv * tinv / 2;
    info.cost_primal = (res.dot_qx * tinv + xPx) * cinv;
    info.cost_dual = (-res.dot_bz * tinv - xPx) * cinv;
    double normx = norm_scaled(eq.d, vars.x.data(), n);
    double normz = norm_scaled(eq.e, vars.z.data(), m) * cinv;
    double norms = norm_scaled(eq.einv, vars.s.data(), m);
    info.res_primal_inf =
        (norm_scaled(eq.dinv, res.rx_inf.data(), n) * cinv) / std::max(1.0, normz);
    info.res_dual_inf =
        std::max(norm_scaled(eq.dinv, res.Px.data(), n) / std::max(1.0, normx),
                 norm_scaled(eq.einv, res.rz_inf.data(), m) /
                     std::max(1.0, normx + norms));
    normx *= tinv;
    normz *= tinv;
    norms *= tinv;
    info.res_primal = norm_scaled(eq.einv, res.rz.data(), m) * tinv /
                      std::max(1.0, normb + normx + norms);
    info.res_dual = norm_scaled(eq.dinv, res.rx.data(), n) * tinv * cinv /
                    std::max(1.0, normq + normx + normz);
    info.gap_abs = std::fabs(info.cost_primal - info.cost_dual);
    info.gap_rel = info.gap_abs / std::max(1.0, std::min(std::fabs(info.cost_primal),
                                                         std::fabs(info.cost_dual)));
    info.ktratio = vars.kappa * tinv;
    info.solve_time =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  void check_convergence(double tga, double tgr, double tf, double tia,
                         double tir, double tkt, int ss, int ps, int ds) {
    if (info.ktratio <= 1.0 && ((info.gap_abs < tga || info.gap_rel < tgr) &&
                                info.res_primal < tf && info.res_dual < tf)) {
      info.status = ss;
    } else if (info.ktratio > 1000. / tkt) {
      if (res.dot_bz < -tia && info.res_primal_inf < -tir * res.dot_bz)
        info.status = ps;
      else if (res.dot_qx < -tia && info.res_dual_inf < -tir * res.dot_qx)
        info.status = ds;
    }
  }

  // info.jl:135-190
  bool check_termination(int iter) {
    info.status = 0;
    check_convergence(st.tol_gap_abs, st.tol_gap_rel, st.tol_feas,
                      st.tol_infeas_abs, st.tol_infeas_rel, st.tol_ktratio, 1, 2, 3);
    if (info.status == 0 && iter > 1 &&
        (info.res_dual > prev_res_dual || info.res_primal > prev_res_primal)) {
      if (info.ktratio < 100 * kEps &&
          (prev_gap_abs < st.tol_gap_abs || prev_gap_rel < st.tol_gap_rel))
        info.status = 10;
      if (info.ktratio < 1.0) {
        if ((info.res_dual > 100 * st.tol_feas && info.res_dual > 100 * prev_res_dual) ||
            (info.res_primal > 100 * st.tol_feas &&
             info.res_primal > 100 * prev_res_primal))
          info.status = 10;
      }
    }
    if (info.status == 0) {
      if (st.max_iter == info.iterations)
        info.status = 7;
      else if (info.solve_time > st.time_limit)
        info.status = 8;
    }
    return info.status != 0;
  }

  void save_prev() {
    prev_cost_primal = info.cost_primal;
    prev_cost_dual = info.cost_dual;
    prev_res_primal = info.res_primal;
    prev_res_dual = info.res_dual;
    prev_gap_abs = info.gap_abs;
    prev_gap_rel = info.gap_rel;
    prev_vars = vars;
  }
  void reset_to_prev() {
    info.cost_primal = prev_cost_primal;
    info.cost_dual = prev_cost_dual;
    info.res_primal = prev_res_primal;
    info.res_dual = prev_res_dual;
    info.gap_abs = prev_gap_abs;
    info.gap_rel = prev_gap_rel;
    vars = prev_vars;
  }

  // kktsystem.jl:57-87
  bool kkt_update() {
    if (!kkt.update()) return false;
    for (int i = 0; i < n; ++i) workx[i] = -q[i];
    kkt.setrhs(workx.data(), b.data());
    return kkt.solve(x2.data(), z2.data());
  }

  // kktsystem.jl:90-127
  bool kkt_solve_initial_point() {
    if (P.nnz() == 0) {
      std::fill(workx.begin(), workx.end(), 0.0);
      kkt.setrhs(workx.data(), b.data());
      bool ok = kkt.solve(vars.x.data(), vars.s.data());
      for (auto &v : vars.s) v = -v;
      if (!ok) return ok;
      for (int i = 0; i < n; ++i) workx[i] = -q[i];
      std::fill(workz.begin(), workz.end(), 0.0);
      kkt.setrhs(workx.data(), workz.data());
      return kkt.solve(nullptr, vars.z.data());
    }
    for (int i = 0; i < n; ++i) workx[i] = -q[i];
    kkt.setrhs(workx.data(), b.data());
    bool ok = kkt.solve(vars.x.data(), vars.z.data());
    for (int i = 0; i < m; ++i) vars.s[i] = -vars.z[i];
    return ok;
  }

  // kktsystem.jl:130-210
  bool kkt_solve(Variables &lhs, Variables &rhs, bool affine) {
    for (int i = 0; i < n; ++i) workx[i] = rhs.x[i];
    Vec &dsc = work_conic;
    if (affine)
      dsc = vars.s;
    else
      cones.ds_from_dz_offset(dsc.data(), rhs.s.data(), lhs.z.data(), vars.z.data());
    for (int i = 0; i < m; ++i) workz[i] = dsc[i] - rhs.z[i];
    kkt.setrhs(workx.data(), workz.data());
    if (!kkt.solve(x1.data(), z1.data())) return false;
    Vec &xi = workx;
    for (int i = 0; i < n; ++i) xi[i] = vars.x[i] / vars.tau;
    Vec Pw(n);
    csc_symv_triu(P, x1.data(), Pw.data());
    double tau_num = rhs.tau - rhs.kappa / vars.tau + dot(q.data(), x1.data(), n) +
                     dot(b.data(), z1.data(), m) + 2 * dot(xi.data(), Pw.data(), n);
    for (int i = 0; i < n; ++i) xi[i] -= x2[i];
    double tau_den = vars.kappa / vars.tau - dot(q.data(), x2.data(), n) -
                     dot(b.data(), z2.data(), m);
    csc_symv_triu(P, xi.data(), Pw.data());
    double t1 = dot(xi.data(), Pw.data(), n);
    csc_symv_triu(P, x2.data(), Pw.data());
    double t2 = dot(x2.data(), Pw.data(), n);
    tau_den += t1 - t2;
    lhs.tau = tau_num / tau_den;
    for (int i = 0; i < n; ++i) lhs.x[i] = x1[i] + lhs.tau * x2[i];
    for (int i = 0; i < m; ++i) lhs.z[i] = z1[i] + lhs.tau * z2[i];
    cones.mul_Hs(lhs.s.data(), lhs.z.data(), workz.data());
    for (int i = 0; i < m; ++i) lhs.s[i] = -(lhs.s[i] + dsc[i]);
    lhs.kappa = -(rhs.kappa + vars.kappa * lhs.tau) / vars.tau;
    return true;
  }

  // variables.jl:276-304
  void shift_to_cone_interior(Vec &z, int pd) {
    double mm, pm;
    cones.margins(z.data(), pd, mm, pm);
    double target = std::max(1.0, 0.1 * pm / cones.degree);
    if (mm <= 0) {
      cones.scaled_unit_shift(z.data(), -mm, pd);
      cones.scaled_unit_shift(z.data(), target, pd);
    } else if (mm < target) {
      cones.scaled_unit_shift(z.data(), target - mm, pd);
    } else {
      cones.scaled_unit_shift(z.data(), 0.0, pd);
    }
  }

  void default_start() {
    if (cones.symmetric) {
      cones.set_identity_scaling();
      kkt_update();
      kkt_solve_initial_point();
      shift_to_cone_interior(vars.s, PrimalCone);
      shift_to_cone_interior(vars.z, DualCone);
      vars.tau = 1;
      vars.kappa = 1;
    } else {
      cones.unit_initialization(vars.z.data(), vars.s.data());
      std::fill(vars.x.begin(), vars.x.end(), 0.0);
      vars.tau = 1;
      vars.kappa = 1;
    }
  }

  double calc_step_length(bool combined) {
    double at = step_lhs.tau < 0 ? -vars.tau / step_lhs.tau : kMax;
    double ak = step_lhs.kappa < 0 ? -vars.kappa / step_lhs.kappa : kMax;
    double a = std::min(std::min(at, ak), 1.0);
    double az, as;
    cones.step_length(step_lhs.z.data(), step_lhs.s.data(), vars.z.data(),
                      vars.s.data(), st, a, az, as);
    a = std::min(az, as);
    if (combined) a *= st.max_step_fraction;
    return a;
  }

  double barrier(double a) {
    double cc = cones.degree + 1;
    double ct = vars.tau + a * step_lhs.tau;
    double ck = vars.kappa + a * step_lhs.kappa;
    double sz = 0;
    for (int i = 0; i < m; ++i)
      sz += (vars.z[i] + a * step_lhs.z[i]) * (vars.s[i] + a * step_lhs.s[i]);
    double mu = (sz + ct * ck) / cc;
    double bar = cc * logsafe(mu) - logsafe(ct) - logsafe(ck);
    bar += cones.compute_barrier(vars.z.data(), vars.s.data(), step_lhs.z.data(),
                                 step_lhs.s.data(), a);
    return bar;
  }

  double get_step_length(bool combined, int scaling) {
    double a = calc_step_length(combined);
    if (!cones.symmetric && combined && scaling == Dual) {
      double step = st.linesearch_backtrack_step;
      for (int j = 0; j < 50; ++j) {
        if (barrier(a) < 1.0) return a;
        a = step * a;
      }
    }
    return a;
  }

  void solve_loop() {
    kkt.ir_solves = kkt.ir_sweeps = kkt.ir_unconverged = 0;
    kkt.ir_worst = 0;
    int iter = 0;
    double sigma = 1.0, alpha = 0.0, mu = kMax;
    t0 = std::chrono::steady_clock::now();
    // a solver object may be solved repeatedly (solve! after setup!): every
    // piece of per-solve state starts afresh
    info = oracle_info{};
    prev_cost_primal = prev_cost_dual = prev_res_primal = prev_res_dual = kInf;
    prev_gap_abs = prev_gap_rel = kInf;
    info.status = 0;
    default_start();
    int scaling = cones.allows_primal_dual_scaling() ? PrimalDual : Dual;
    while (true) {
      residuals_update();
      mu = (res.dot_sz + vars.tau * vars.kappa) / (cones.degree + 1);
      info.mu = mu;
      info.step_length = alpha;
      info.sigma = sigma;
      info.iterations = iter;
      info_update();
      if (st.verbose)
        std::printf("%3d  %+.8e  %+.8e  %.2e %.2e %.2e %.2e %.2e\n", iter,
                    info.cost_primal, info.cost_dual, info.gap_rel,
                    info.res_primal, info.res_dual, info.ktratio, mu);
      bool isdone = check_termination(iter);
      if (isdone) {
        // _strategy_checkpoint_insufficient_progress
        if (info.status != 10) break;
        reset_to_prev();
        if (!cones.symmetric && scaling == PrimalDual) {
          info.status = 0;
          scaling = Dual;
          continue;
        }
        break;
      }
      bool sc_ok = cones.update_scaling(vars.s.data(), vars.z.data(), mu, scaling);
      if (!sc_ok) {
        info.status = 9;
        break;
      }
      iter += 1;
      bool ok = kkt_update();
      // affine step rhs (variables.jl:161-175)
      step_rhs.x = res.rx;
      step_rhs.z = res.rz;
      cones.affine_ds(step_rhs.s.data(), vars.s.data());
      step_rhs.tau = res.rtau;
      step_rhs.kappa = vars.tau * vars.kappa;
      ok = ok && kkt_solve(step_lhs, step_rhs, true);
      if (ok) {
        alpha = get_step_length(false, scaling);
        sigma = std::pow(1 - alpha, 3);
        double mfac = iter > 1 ? 1.0 : alpha;
        // combined step rhs (variables.jl:178-216)
        double sm = sigma * mu;
        for (int i = 0; i < n; ++i) step_rhs.x[i] = (1 - sigma) * res.rx[i];
        step_rhs.tau = (1 - sigma) * res.rtau;
        step_rhs.kappa = -sm + mfac * step_lhs.tau * step_lhs.kappa +
                         vars.tau * vars.kappa;
        if (mfac != 1.0)
          for (auto &v : step_lhs.z) v *= mfac;
        cones.combined_ds_shift(step_rhs.z.data(), step_lhs.z.data(),
                                step_lhs.s.data(), sm);
        for (int i = 0; i < m; ++i) step_rhs.s[i] += step_rhs.z[i];
        for (int i = 0; i < m; ++i) step_rhs.z[i] = (1 - sigma) * res.rz[i];
        ok = kkt_solve(step_lhs, step_rhs, false);
      }
      // _strategy_checkpoint_numerical_error
      if (!ok) {
        if (!cones.symmetric && scaling == PrimalDual) {
          scaling = Dual;
          alpha = 0;
          continue;
        }
        info.status = 9;
        alpha = 0;
        break;
      }
      alpha = get_step_length(true, scaling);
      // _strategy_checkpoint_small_step
      if (!cones.symmetric && scaling == PrimalDual && alpha < st.min_switch_step_length) {
        scaling = Dual;
        alpha = 0;
        continue;
      } else if (alpha <= std::max(0.0, st.min_terminate_step_length)) {
        info.status = 10;
        alpha = 0;
        break;
      }
      save_prev();
      for (int i = 0; i < n; ++i) vars.x[i] += alpha * step_lhs.x[i];
      for (int i = 0; i < m; ++i) vars.s[i] += alpha * step_lhs.s[i];
      for (int i = 0; i < m; ++i) vars.z[i] += alpha * step_lhs.z[i];
      vars.tau += alpha * step_lhs.tau;
      vars.kappa += alpha * step_lhs.kappa;
    }
    if (alpha == 0.0) {
      info.mu = mu;
      info.step_length = alpha;
      info.sigma = sigma;
      info.iterations = iter;
    }
    // info_post_process!
    if (info.status == 9 || info.status == 10 || info.status == 7 || info.status == 8)
      check_convergence(st.reduced_tol_gap_abs, st.reduced_tol_gap_rel,
                        st.reduced_tol_feas, st.reduced_tol_infeas_abs,
                        st.reduced_tol_infeas_rel, st.reduced_tol_ktratio, 4, 5, 6);
    info.solve_time =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  void setup(int n_, int m_, const int *Pp, const int *Pi, const double *Px,
             const double *q_, const int *Ap, const int *Ai, const double *Ax,
             const double *b_, int ncones, const int *types, const int *dims,
             const double *params) {
    n = n_;
    m = m_;
    // triu copy of P
    P.m = P.n = n;
    P.p.assign(n + 1, 0);
    for (int j = 0; j < n; ++j) {
      for (int k = Pp[j]; k < Pp[j + 1]; ++k)
        if (Pi[k] <= j) {
          P.i.push_back(Pi[k]);
          P.x.push_back(Px[k]);
        }
      P.p[j + 1] = (int)P.i.size();
    }
    A.m = m;
    A.n = n;
    A.p.assign(Ap, Ap + n + 1);
    A.i.assign(Ai, Ai + Ap[n]);
    A.x.assign(Ax, Ax + Ap[n]);
    q.assign(q_, q_ + n);
    b.assign(b_, b_ + m);
    for (auto &v : b) v = std::min(v, 1e20);
    normq = norm_inf(q.data(), n);
    normb = norm_inf(b.data(), m);
    cones.build(ncones, types, dims, params);
    if (cones.numel != m) throw std::invalid_argument("cone dims != m");
    vars.init(n, m);
    step_rhs.init(n, m);
    step_lhs.init(n, m);
    prev_vars.init(n, m);
    res.rx.assign(n, 0);
    res.rx_inf.assign(n, 0);
    res.Px.assign(n, 0);
    res.rz.assign(m, 0);
    res.rz_inf.assign(m, 0);
    equilibrate();
    kkt.st = &st;
    kkt.assemble(P, A, cones);
    x1.assign(n, 0);
    x2.assign(n, 0);
    workx.assign(n, 0);
    z1.assign(m, 0);
    z2.assign(m, 0);
    workz.assign(m, 0);
    work_conic.assign(m, 0);
  }

  void finish(double *x, double *s, double *z) {
    bool infeas = info.status == 2 || info.status == 3 || info.status == 5 ||
                  info.status == 6;
    if (infeas) {
      info.obj_val = NAN;
      info.obj_val_dual = NAN;
    } else {
      info.obj_val = info.cost_primal;
      info.obj_val_dual = info.cost_dual;
    }
    double sinv = infeas ? 1.0 / vars.kappa : 1.0 / vars.tau;
    double cinv = 1.0 / eq.c;
    for (int i = 0; i < n; ++i) x[i] = vars.x[i] * eq.d[i] * sinv;
    for (int i = 0; i < m; ++i) z[i] = vars.z[i] * eq.e[i] * (sinv * cinv);
    for (int i = 0; i < m; ++i) s[i] = vars.s[i] * eq.einv[i] * sinv;
  }
};

}  // namespace orc

using namespace orc;

extern "C" {

void oracle_default_settings(oracle_settings *s) {
  // src/settings.jl:70-148
  s->max_iter = 200;
  s->time_limit = kInf;
  s->max_step_fraction = 0.99;
  s->tol_gap_abs = 1e-8;
  s->tol_gap_rel = 1e-8;
  s->tol_feas = 1e-8;
  s->tol_infeas_abs = 1e-8;
  s->tol_infeas_rel = 1e-8;
  s->tol_ktratio = 1e-6;
  s->reduced_tol_gap_abs = 5e-5;
  s->reduced_tol_gap_rel = 5e-5;
  s->reduced_tol_feas = 1e-4;
  s->reduced_tol_infeas_abs = 5e-12;
  s->reduced_tol_infeas_rel = 5e-5;
  s->reduced_tol_ktratio = 1e-4;
  s->equilibrate_enable = 1;
  s->equilibrate_max_iter = 10;
  s->equilibrate_min_scaling = 1e-4;
  s->equilibrate_max_scaling = 1e4;
  s->linesearch_backtrack_step = 0.8;
  s->min_switch_step_length = 1e-2;
  s->min_terminate_step_length = 1e-4;
  s->static_regularization_enable = 1;
  s->static_regularization_constant = 1e-8;
  s->static_regularization_proportional = kEps * kEps;
  s->dynamic_regularization_enable = 1;
  s->dynamic_regularization_eps = 1e-13;
  s->dynamic_regularization_delta = 2e-7;
  s->iterative_refinement_enable = 1;
  s->iterative_refinement_reltol = 1e-12;
  s->iterative_refinement_abstol = 1e-12;
  s->iterative_refinement_max_iter = 10;
  s->iterative_refinement_stop_ratio = 5;
  s->verbose = 0;
  s->gpu_equilibration = 0;
  s->factor_fp32 = 0;
}

int oracle_solve(int n, int m, const int *Pp, const int *Pi, const double *Px,
                 const double *q, const int *Ap, const int *Ai,
                 const double *Ax, const double *b, int ncones,
                 const int *cone_types, const int *cone_dims,
                 const double *cone_params, const oracle_settings *settings,
                 double *x, double *s, double *z, oracle_info *info) {
  if (n < 0 || m < 0) return -1;
  try {
    Solver S;
    if (settings)
      S.st = *settings;
    else
      oracle_default_settings(&S.st);
    S.setup(n, m, Pp, Pi, Px, q, Ap, Ai, Ax, b, ncones, cone_types, cone_dims,
            cone_params);
    S.solve_loop();
    S.finish(x, s, z);
    *info = S.info;
    info->ir_solves = S.kkt.ir_solves;
    info->ir_sweeps = S.kkt.ir_sweeps;
    info->ir_unconverged = S.kkt.ir_unconverged;
    info->ir_worst_ratio = S.kkt.ir_worst;
  } catch (std::exception &e) {
    std::fprintf(stderr, "oracle_solve: %s\n", e.what());
    return -2;
  }
  return 0;
}

// Solver(P,q,A,b,cones,settings) once, then solve! any number of times
// (src/solver.jl:5-17 and :231-422): setup work (equilibration, KKT
// assembly, ordering, symbolic factorisation) stays outside the solves.
struct oracle_solver {
  Solver S;
};

oracle_solver *oracle_solver_create(int n, int m, const int *Pp, const int *Pi,
                                    const double *Px, const double *q, const int *Ap,
                                    const int *Ai, const double *Ax, const double *b,
                                    int ncones, const int *cone_types, const int *cone_dims,
                                    const double *cone_params,
                                    const oracle_settings *settings) {
  if (n < 0 || m < 0) return nullptr;
  auto *h = new oracle_solver;
  try {
    if (settings)
      h->S.st = *settings;
    else
      oracle_default_settings(&h->S.st);
    h->S.setup(n, m, Pp, Pi, Px, q, Ap, Ai, Ax, b, ncones, cone_types, cone_dims,
               cone_params);
  } catch (std::exception &e) {
    std::fprintf(stderr, "oracle_solver_create: %s\n", e.what());
    delete h;
    return nullptr;
  }
  return h;
}
int oracle_solver_run(oracle_solver *h, double *x, double *s, double *z, oracle_info *info) {
  if (!h) return -1;
  try {
    h->S.solve_loop();
    h->S.finish(x, s, z);
    *info = h->S.info;
    info->ir_solves = h->S.kkt.ir_solves;
    info->ir_sweeps = h->S.kkt.ir_sweeps;
    info->ir_unconverged = h->S.kkt.ir_unconverged;
    info->ir_worst_ratio = h->S.kkt.ir_worst;
  } catch (std::exception &e) {
    std::fprintf(stderr, "oracle_solver_run: %s\n", e.what());
    return -2;
  }
  return 0;
}
void oracle_solver_destroy(oracle_solver *h) { delete h; }

struct oracle_cones {
  CompositeCone C;
  oracle_settings st;
};

oracle_cones *oracle_cones_create(int ncones, const int *types,
                                  const int *dims, const double *params) {
  auto *c = new oracle_cones;
  c->C.build(ncones, types, dims, params);
  oracle_default_settings(&c->st);
  return c;
}
void oracle_cones_destroy(oracle_cones *c) { delete c; }
int oracle_cones_numel(const oracle_cones *c) { return c->C.numel; }
int oracle_cones_degree(const oracle_cones *c) { return c->C.degree; }
int oracle_cones_hs_len(const oracle_cones *c) { return c->C.hs_len; }
int oracle_update_scaling(oracle_cones *c, const double *s, const double *z,
                          double mu, int strategy) {
  return c->C.update_scaling(s, z, mu, strategy) ? 0 : 1;
}
void oracle_set_identity_scaling(oracle_cones *c) { c->C.set_identity_scaling(); }
void oracle_get_Hs(oracle_cones *c, double *Hs) { c->C.get_Hs(Hs); }
void oracle_mul_Hs(oracle_cones *c, double *y, const double *x) {
  std::vector<double> w(c->C.numel);
  c->C.mul_Hs(y, x, w.data());
}
void oracle_affine_ds(oracle_cones *c, double *ds, const double *s) {
  c->C.affine_ds(ds, s);
}
void oracle_combined_ds_shift(oracle_cones *c, double *shift, double *step_z,
                              double *step_s, const double *, double sm) {
  c->C.combined_ds_shift(shift, step_z, step_s, sm);
}
void oracle_ds_from_dz_offset(oracle_cones *c, double *out, const double *ds,
                              const double *z) {
  std::vector<double> w(c->C.numel);
  c->C.ds_from_dz_offset(out, ds, w.data(), z);
}
double oracle_step_length(oracle_cones *c, const double *dz, const double *ds,
                          const double *z, const double *s, double amax,
                          double msf, double bt, double amin) {
  c->st.max_step_fraction = msf;
  c->st.linesearch_backtrack_step = bt;
  c->st.min_terminate_step_length = amin;
  double az, as;
  c->C.step_length(dz, ds, z, s, c->st, amax, az, as);
  return std::min(az, as);
}
double oracle_compute_barrier(oracle_cones *c, const double *z, const double *s,
                              const double *dz, const double *ds, double a) {
  return c->C.compute_barrier(z, s, dz, ds, a);
}
void oracle_margins(oracle_cones *c, const double *z, int pd, double *a,
                    double *b) {
  c->C.margins(z, pd, *a, *b);
}
void oracle_scaled_unit_shift(oracle_cones *c, double *z, double a, int pd) {
  c->C.scaled_unit_shift(z, a, pd);
}
void oracle_unit_initialization(oracle_cones *c, double *z, double *s) {
  c->C.unit_initialization(z, s);
}
int oracle_get_state(oracle_cones *c, int which, double *out) {
  int k = 0;
  for (size_t ci = 0; ci < c->C.cones.size(); ++ci) {
    Cone *cn = c->C.cones[ci].get();
    int o = c->C.rng_start[ci], d = cn->numel();
    if (which == 0 || which == 1) {
      if (auto *ss = soc_state(cn)) {
        const Vec &v = which == 0 ? ss->w : ss->lambda;
        for (int i = 0; i < d; ++i) out[o + i] = v[i];
      } else {
        NNStateView nv = nn_state(cn);
        if (nv.w) {
          const Vec &v = which == 0 ? *nv.w : *nv.lambda;
          for (int i = 0; i < d; ++i) out[o + i] = v[i];
        } else if (which == 1 && cn->type() == OR_CONE_PSD) {
          for (int i = 0; i < d; ++i) out[o + i] = 0;
          psd_lambda(cn, out + o);
        } else {
          for (int i = 0; i < d; ++i) out[o + i] = 0;
        }
      }
      k = c->C.numel;
    } else if (which == 2) {
      SOCState *ss = soc_state(cn);
      out[ci] = ss ? ss->eta : 0.0;
      k = (int)c->C.cones.size();
    } else if (which == 3) {
      SOCState *ss = soc_state(cn);
      if (ss && ss->sparse) {
        out[k++] = ss->d;
        for (int i = 0; i < d; ++i) out[k++] = ss->u[i];
        for (int i = 0; i < d; ++i) out[k++] = ss->v[i];
      }
    }
  }
  return k;
}

}  // extern "C"
