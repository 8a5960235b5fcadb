// oracle_ldl.cpp -- CPU sparse LDL^T for the oracle.
// TEST INFRASTRUCTURE ONLY (see clarabel_oracle.h).
//
// The reference's CPU path factors the triu KKT with QDLDL.jl 0.4.1
// (src/kktsolvers/direct-ldl/directldl_qdldl.jl:18-25 passes Dsigns,
// dynamic_regularization_eps/delta, logical=true).  QDLDL's published
// algorithm is restated here: elimination tree + nonzero counts, then an
// up-looking factorisation that builds row k of L by a sparse triangular
// solve over the etree reach, with D[k] replaced by delta*sign whenever
// sign*D[k] <= eps.  The fill-reducing ordering is a minimum-degree
// ordering written for this file (the reference uses AMD.jl); ordering only
// changes rounding, not results.
#include <algorithm>
#include <numeric>
#include <set>

#include "oracle_internal.hpp"

namespace orc {

std::vector<int> min_degree_order(int n, const std::vector<int> &Kp,
                                  const std::vector<int> &Ki) {
  std::vector<std::vector<int>> adj(n);
  for (int j = 0; j < n; ++j)
    for (int p = Kp[j]; p < Kp[j + 1]; ++p) {
      int i = Ki[p];
      if (i == j) continue;
      adj[i].push_back(j);
      adj[j].push_back(i);
    }
  for (auto &a : adj) {
    std::sort(a.begin(), a.end());
    a.erase(std::unique(a.begin(), a.end()), a.end());
  }
  // rows that are dense in the original pattern are ordered last
  double dense_thr = std::max(16.0, 10.0 * std::sqrt((double)n));
  std::vector<char> dense(n, 0), done(n, 0);
  std::set<std::pair<int, int>> pq;
  for (int i = 0; i < n; ++i) {
    if (adj[i].size() > dense_thr)
      dense[i] = 1;
    else
      pq.insert({(int)adj[i].size(), i});
  }
  std::vector<int> order;
  order.reserve(n);
  std::vector<int> tmp;
  while (!pq.empty()) {
    int v = pq.begin()->second;
    pq.erase(pq.begin());
    done[v] = 1;
    order.push_back(v);
    // neighbours that are still live
    std::vector<int> nb;
    for (int u : adj[v])
      if (!done[u]) nb.push_back(u);
    for (int u : nb) {
      if (dense[u]) continue;
      pq.erase({(int)adj[u].size(), u});
      // adj[u] <- (adj[u] U nb) \ {u, v, eliminated}
      tmp.clear();
      std::set_union(adj[u].begin(), adj[u].end(), nb.begin(), nb.end(),
                     std::back_inserter(tmp));
      adj[u].clear();
      for (int w : tmp)
        if (w != u && !done[w]) adj[u].push_back(w);
      pq.insert({(int)adj[u].size(), u});
    }
    adj[v].clear();
    adj[v].shrink_to_fit();
  }
  for (int i = 0; i < n; ++i)
    if (dense[i]) order.push_back(i);
  return order;
}

void LDL::setup(int n_, const std::vector<int> &Kp, const std::vector<int> &Ki,
                const std::vector<int> &Dsigns_unperm) {
  n = n_;
  perm = min_degree_order(n, Kp, Ki);
  iperm.assign(n, 0);
  for (int k = 0; k < n; ++k) iperm[perm[k]] = k;
  // permuted upper triangle with map from original nz positions
  int nnz = Kp[n];
  std::vector<int> cnt(n + 1, 0);
  for (int j = 0; j < n; ++j)
    for (int p = Kp[j]; p < Kp[j + 1]; ++p) {
      int a = iperm[Ki[p]], b = iperm[j];
      cnt[std::max(a, b) + 1]++;
    }
  Ap.assign(n + 1, 0);
  for (int j = 0; j < n; ++j) Ap[j + 1] = Ap[j] + cnt[j + 1];
  std::vector<int> next(Ap.begin(), Ap.end() - 1);
  Ai.assign(nnz, 0);
  mapK.assign(nnz, 0);
  for (int j = 0; j < n; ++j)
    for (int p = Kp[j]; p < Kp[j + 1]; ++p) {
      int a = iperm[Ki[p]], b = iperm[j];
      int col = std::max(a, b), row = std::min(a, b);
      int q = next[col]++;
      Ai[q] = row;
      mapK[p] = q;
    }
  Ax.assign(nnz, 0.0);
  Dsigns.assign(n, 1);
  for (int k = 0; k < n; ++k) Dsigns[k] = Dsigns_unperm[perm[k]];
  // elimination tree and column counts (QDLDL_etree)
  etree.assign(n, -1);
  Lnz.assign(n, 0);
  std::vector<int> work(n, -1);
  for (int j = 0; j < n; ++j) {
    work[j] = j;
    for (int p = Ap[j]; p < Ap[j + 1]; ++p) {
      int i = Ai[p];
      while (work[i] != j) {
        if (etree[i] == -1) etree[i] = j;
        Lnz[i]++;
        work[i] = j;
        i = etree[i];
      }
    }
  }
  Lp.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) Lp[i + 1] = Lp[i] + Lnz[i];
  Li.assign(Lp[n], 0);
  Lx.assign(Lp[n], 0.0);
  D.assign(n, 0.0);
  Dinv.assign(n, 0.0);
  iwork.assign(n, 0);
  bwork.assign(n, 0);
  yidx.assign(n, 0);
  ebuf.assign(n, 0);
  nextcol.assign(n, 0);
  fwork.assign(n, 0.0);
}

void LDL::update_values(const std::vector<int> &kidx, const double *vals,
                        int count) {
  for (int i = 0; i < count; ++i) Ax[mapK[kidx[i]]] = vals[i];
}
void LDL::update_value(int kidx, double v) { Ax[mapK[kidx]] = v; }
void LDL::scale_values(const std::vector<int> &kidx, double scale, int count) {
  for (int i = 0; i < count; ++i) Ax[mapK[kidx[i]]] *= scale;
}

// QDLDL_factor restated: up-looking, row k of L by sparse triangular solve.
// With arith_fp32 every value is an FP32 one and every operation an FP32
// operation (refactor_fp32).
bool LDL::refactor() {
  if (arith_fp32) return refactor_fp32();
  const int UNUSED = 0, USED = 1;
  reg_count = 0;
  std::fill(bwork.begin(), bwork.end(), UNUSED);
  std::fill(fwork.begin(), fwork.end(), 0.0);
  for (int i = 0; i < n; ++i) nextcol[i] = Lp[i];
  for (int k = 0; k < n; ++k) {
    int nnzY = 0;
    D[k] = 0;
    for (int p = Ap[k]; p < Ap[k + 1]; ++p) {
      int b = Ai[p];
      if (b == k) {
        D[k] += Ax[p];
        continue;
      }
      fwork[b] = Ax[p];
      int nx = b;
      if (bwork[nx] == UNUSED) {
        bwork[nx] = USED;
        ebuf[0] = nx;
        int nnzE = 1;
        nx = etree[b];
        while (nx != -1 && nx < k) {
          if (bwork[nx] == USED) break;
          bwork[nx] = USED;
          ebuf[nnzE++] = nx;
          nx = etree[nx];
        }
        while (nnzE) yidx[nnzY++] = ebuf[--nnzE];
      }
    }
    for (int i = nnzY - 1; i >= 0; --i) {
      int c = yidx[i];
      int t = nextcol[c];
      double yc = fwork[c];
      for (int j = Lp[c]; j < t; ++j) fwork[Li[j]] -= Lx[j] * yc;
      Li[t] = k;
      Lx[t] = yc * Dinv[c];
      D[k] -= yc * Lx[t];
      nextcol[c]++;
      fwork[c] = 0;
      bwork[c] = UNUSED;
    }
    if (reg_enable && D[k] * Dsigns[k] <= reg_eps) {
      D[k] = reg_delta * Dsigns[k];
      ++reg_count;
    }
    Dinv[k] = 1.0 / D[k];
  }
  if (round_fp32) {
    for (auto &v : Lx) v = (double)(float)v;
    for (int k = 0; k < n; ++k) {
      D[k] = (double)(float)D[k];
      Dinv[k] = (double)(float)(1.0 / D[k]);
    }
  }
  for (int k = 0; k < n; ++k)
    if (!std::isfinite(Dinv[k])) return false;
  return true;
}

// The same elimination in FP32 arithmetic: values rounded to FP32 as they
// enter, each product and difference an FP32 operation, the pivot inverse
// the FP32 rounding of 1 / d.  L, D and D^-1 hold the FP32 values.
bool LDL::refactor_fp32() {
  const int UNUSED = 0, USED = 1;
  reg_count = 0;
  std::vector<float> fw(n, 0.f), Lf(Lx.size(), 0.f), Df(n, 0.f), Dif(n, 0.f);
  std::fill(bwork.begin(), bwork.end(), UNUSED);
  for (int i = 0; i < n; ++i) nextcol[i] = Lp[i];
  for (int k = 0; k < n; ++k) {
    int nnzY = 0;
    float dk = 0.f;
    for (int p = Ap[k]; p < Ap[k + 1]; ++p) {
      int b = Ai[p];
      if (b == k) {
        dk += (float)Ax[p];
        continue;
      }
      fw[b] = (float)Ax[p];
      int nx = b;
      if (bwork[nx] == UNUSED) {
        bwork[nx] = USED;
        ebuf[0] = nx;
        int nnzE = 1;
        nx = etree[b];
        while (nx != -1 && nx < k) {
          if (bwork[nx] == USED) break;
          bwork[nx] = USED;
          ebuf[nnzE++] = nx;
          nx = etree[nx];
        }
        while (nnzE) yidx[nnzY++] = ebuf[--nnzE];
      }
    }
    for (int i = nnzY - 1; i >= 0; --i) {
      int c = yidx[i];
      int t = nextcol[c];
      const float yc = fw[c];
      for (int j = Lp[c]; j < t; ++j) {
        const volatile float prod = Lf[j] * yc;  // no contraction into an FMA
        fw[Li[j]] -= prod;
      }
      Li[t] = k;
      Lf[t] = yc * Dif[c];
      const volatile float prod = yc * Lf[t];
      dk -= prod;
      nextcol[c]++;
      fw[c] = 0.f;
      bwork[c] = UNUSED;
    }
    if (reg_enable && (double)dk * Dsigns[k] <= reg_eps) {
      dk = (float)(reg_delta * Dsigns[k]);
      ++reg_count;
    }
    Df[k] = dk;
    Dif[k] = (float)(1.0 / (double)dk);
  }
  for (size_t q = 0; q < Lx.size(); ++q) Lx[q] = Lf[q];
  for (int k = 0; k < n; ++k) {
    D[k] = Df[k];
    Dinv[k] = Dif[k];
  }
  for (int k = 0; k < n; ++k)
    if (!std::isfinite(Dinv[k])) return false;
  return true;
}

void LDL::solve(double *x) const {
  std::vector<double> y(n);
  for (int k = 0; k < n; ++k) y[k] = x[perm[k]];
  for (int j = 0; j < n; ++j)
    for (int p = Lp[j]; p < Lp[j + 1]; ++p) y[Li[p]] -= Lx[p] * y[j];
  for (int j = 0; j < n; ++j) y[j] *= Dinv[j];
  for (int j = n - 1; j >= 0; --j)
    for (int p = Lp[j]; p < Lp[j + 1]; ++p) y[j] -= Lx[p] * y[Li[p]];
  for (int k = 0; k < n; ++k) x[perm[k]] = y[k];
}

}  // namespace orc
