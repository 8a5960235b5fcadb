// amd.cpp -- approximate minimum degree ordering on the quotient graph.
//
// The fill-reducing ordering of the large single problems.  cuDSS's
// analysis phase orders the KKT matrix in the reference
// (src/kktsolvers/gpu/directldl_cudss.jl:20-23); the reference CPU path uses
// AMD.jl (src/kktsolvers/direct-ldl/directldl_qdldl.jl:18-25).  This is an
// implementation of the published approximate minimum degree algorithm
// (P. Amestoy, T. Davis, I. Duff, "An approximate minimum degree ordering
// algorithm", SIAM J. Matrix Anal. Appl. 17(4), 1996):
//
//  * the elimination graph is kept implicitly as a quotient graph: every
//    eliminated pivot becomes an element holding the list of variables it
//    couples, so the memory stays O(nnz) however large the fill;
//  * a variable's degree is the approximate external degree
//        min(n - k, d_old + |Lp \ i|, |A_i \ i| + |Lp \ i| + sum |Le \ Lp|),
//    where |Le \ Lp| is computed for every element touching the new element
//    Lp in one pass;
//  * elements entirely inside Lp are absorbed (element and aggressive
//    absorption), variables with identical adjacency are merged into
//    supervariables (hash + exact comparison), and variables adjacent only
//    to the new element are eliminated with the pivot (mass elimination);
//  * rows denser than max(16, 10 sqrt(n)) are ordered last.
//
// The layout (one std::vector per list rather than AMD's single workspace
// with garbage collection) is this project's own.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "setup.hpp"

namespace clgpu {

namespace {

enum : signed char { kVar = 0, kElem = 1, kDead = 2 };

struct DegreeLists {
  std::vector<int> head, next, prev;
  int mindeg = 0;
  explicit DegreeLists(int n) : head(n + 1, -1), next(n, -1), prev(n, -1) {}
  void insert(int i, int d) {
    next[i] = head[d];
    prev[i] = -1;
    if (head[d] >= 0) prev[head[d]] = i;
    head[d] = i;
    if (d < mindeg) mindeg = d;
  }
  void remove(int i, int d) {
    if (prev[i] >= 0)
      next[prev[i]] = next[i];
    else
      head[d] = next[i];
    if (next[i] >= 0) prev[next[i]] = prev[i];
    next[i] = prev[i] = -1;
  }
  int pop(int n) {
    while (mindeg <= n && head[mindeg] < 0) ++mindeg;
    if (mindeg > n) return -1;
    const int i = head[mindeg];
    remove(i, mindeg);
    return i;
  }
};

}  // namespace

std::vector<int> amd_order_qg(int n, const std::vector<int> &xadj, const std::vector<int> &adj) {
  std::vector<int> order;
  order.reserve(n);
  if (n == 0) return order;
  std::vector<std::vector<int>> vlist(n), elist(n), lelem(n);
  std::vector<signed char> status(n, kVar);
  std::vector<int> nv(n, 1), degree(n, 0), esize(n, 0);
  // members[i]: nodes merged into principal variable i (supervariables and
  // mass elimination), output right after i
  std::vector<std::vector<int>> members(n);
  for (int i = 0; i < n; ++i) {
    auto &v = vlist[i];
    for (int p = xadj[i]; p < xadj[i + 1]; ++p)
      if (adj[p] != i) v.push_back(adj[p]);
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
  }
  const double dense_thr = std::max(16.0, 10.0 * std::sqrt((double)n));
  std::vector<int> dense;
  for (int i = 0; i < n; ++i)
    if ((double)vlist[i].size() > dense_thr) {
      status[i] = kDead;
      dense.push_back(i);
    }
  if (!dense.empty())
    for (int i = 0; i < n; ++i) {
      if (status[i] != kVar) continue;
      auto &v = vlist[i];
      v.erase(std::remove_if(v.begin(), v.end(), [&](int j) { return status[j] != kVar; }),
              v.end());
    }
  DegreeLists dl(n);
  int live = 0;
  for (int i = 0; i < n; ++i)
    if (status[i] == kVar) {
      degree[i] = (int)vlist[i].size();
      dl.insert(i, degree[i]);
      ++live;
    }
  // w[e] - wflg = |Le \ Lp| for elements touched in the current step
  std::vector<long long> w(n, 0);
  long long wflg = 1;
  std::vector<int> mark(n, -1);  // mark[i] == p: i is in the current Lp
  std::vector<int> Lp;
  std::vector<uint64_t> hashv(n, 0);
  int k = 0;  // weighted number of eliminated nodes
  const int nlive = live;
  while (k < nlive) {
    const int p = dl.pop(n);
    if (p < 0) break;
    // ---- new element Lp = (union of Le over e in E_p) + A_p - p
    Lp.clear();
    mark[p] = p;
    for (int e : elist[p]) {
      if (status[e] != kElem) continue;
      for (int i : lelem[e])
        if (status[i] == kVar && mark[i] != p) {
          mark[i] = p;
          Lp.push_back(i);
        }
      status[e] = kDead;  // absorbed into p
      std::vector<int>().swap(lelem[e]);
    }
    for (int i : vlist[p])
      if (status[i] == kVar && mark[i] != p) {
        mark[i] = p;
        Lp.push_back(i);
      }
    std::vector<int>().swap(elist[p]);
    std::vector<int>().swap(vlist[p]);
    status[p] = kElem;
    k += nv[p];
    int degme = 0;
    for (int i : Lp) {
      degme += nv[i];
      dl.remove(i, degree[i]);
    }
    // ---- |Le \ Lp| for every element adjacent to Lp
    if (wflg > (1LL << 60)) {
      std::fill(w.begin(), w.end(), 0);
      wflg = 1;
    }
    for (int i : Lp)
      for (int e : elist[i]) {
        if (status[e] != kElem) continue;
        if (w[e] < wflg) w[e] = wflg + esize[e];
        w[e] -= nv[i];
      }
    // ---- prune the lists of every i in Lp and recompute its degree
    for (int i : Lp) {
      auto &E = elist[i];
      long long deg_e = 0;
      uint64_t h = 0;
      size_t we = 0;
      for (size_t r = 0; r < E.size(); ++r) {
        const int e = E[r];
        if (status[e] != kElem) continue;
        const long long ext = w[e] - wflg;
        if (ext <= 0) {  // Le inside Lp: aggressive absorption into p
          status[e] = kDead;
          std::vector<int>().swap(lelem[e]);
          continue;
        }
        deg_e += ext;
        E[we++] = e;
        h += (uint64_t)e;
      }
      E.resize(we);
      E.push_back(p);
      h += (uint64_t)p;
      auto &V = vlist[i];
      long long deg_v = 0;
      size_t wv = 0;
      for (size_t r = 0; r < V.size(); ++r) {
        const int j = V[r];
        if (status[j] != kVar || mark[j] == p || nv[j] == 0) continue;
        deg_v += nv[j];
        V[wv++] = j;
        h += (uint64_t)j;
      }
      V.resize(wv);
      long long d = std::min<long long>((long long)degree[i] + degme - nv[i],
                                        deg_v + deg_e + degme - nv[i]);
      d = std::min<long long>(d, (long long)(nlive - k - nv[i]));
      if (d < 0) d = 0;
      degree[i] = (int)d;
      hashv[i] = h;
    }
    // ---- mass elimination: variables adjacent to nothing but p
    {
      size_t wl = 0;
      for (size_t r = 0; r < Lp.size(); ++r) {
        const int i = Lp[r];
        if (elist[i].size() == 1 && vlist[i].empty()) {
          nv[p] += nv[i];
          k += nv[i];
          members[p].push_back(i);
          status[i] = kDead;
          nv[i] = 0;
          std::vector<int>().swap(elist[i]);
          continue;
        }
        Lp[wl++] = Lp[r];
      }
      Lp.resize(wl);
    }
    // ---- supervariables: equal hash, then exact list comparison
    if (Lp.size() > 1) {
      std::vector<std::pair<uint64_t, int>> hs;
      hs.reserve(Lp.size());
      for (int i : Lp) hs.push_back({hashv[i] % (uint64_t)(n > 1 ? n - 1 : 1), i});
      std::sort(hs.begin(), hs.end());
      for (size_t a = 0; a < hs.size();) {
        size_t b = a + 1;
        while (b < hs.size() && hs[b].first == hs[a].first) ++b;
        if (b - a > 1) {
          for (size_t x = a; x < b; ++x) {
            const int i = hs[x].second;
            if (nv[i] == 0) continue;
            auto Ei = elist[i], Vi = vlist[i];
            std::sort(Ei.begin(), Ei.end());
            std::sort(Vi.begin(), Vi.end());
            for (size_t y = x + 1; y < b; ++y) {
              const int j = hs[y].second;
              if (nv[j] == 0) continue;
              if (elist[j].size() != Ei.size() || vlist[j].size() != Vi.size()) continue;
              auto Ej = elist[j], Vj = vlist[j];
              std::sort(Ej.begin(), Ej.end());
              std::sort(Vj.begin(), Vj.end());
              if (Ej != Ei || Vj != Vi) continue;
              // j is indistinguishable from i: merge j into i
              nv[i] += nv[j];
              degree[i] -= nv[j];
              if (degree[i] < 0) degree[i] = 0;
              members[i].push_back(j);
              nv[j] = 0;
              status[j] = kDead;
              std::vector<int>().swap(elist[j]);
              std::vector<int>().swap(vlist[j]);
            }
          }
        }
        a = b;
      }
      size_t wl = 0;
      for (size_t r = 0; r < Lp.size(); ++r)
        if (nv[Lp[r]] > 0) Lp[wl++] = Lp[r];
      Lp.resize(wl);
    }
    // ---- the new element and the degree lists
    int es = 0;
    for (int i : Lp) {
      es += nv[i];
      dl.insert(i, std::min(degree[i], n));
    }
    esize[p] = es;
    lelem[p] = Lp;
    if (Lp.empty()) status[p] = kDead;
    order.push_back(p);
    long long maxw = 0;
    for (int i : Lp) maxw += nv[i];
    wflg += std::max<long long>(maxw, 1) + n + 1;
  }
  // expand the pivots: each principal pivot, then what was merged into it
  std::vector<int> out;
  out.reserve(n);
  std::vector<int> stack;
  for (int p : order) {
    stack.assign(1, p);
    while (!stack.empty()) {
      const int v = stack.back();
      stack.pop_back();
      out.push_back(v);
      for (auto it = members[v].rbegin(); it != members[v].rend(); ++it) stack.push_back(*it);
    }
  }
  for (int i : dense) out.push_back(i);
  return out;
}

}  // namespace clgpu
