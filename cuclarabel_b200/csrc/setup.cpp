// setup.cpp -- host-side preparation of one problem instance.
//
// Follows the reference's GPU setup chain (src/solver.jl:129-195):
//   gpu_data_copy!           P upper triangle symmetrised to full (:618-630)
//   DefaultProblemDataGPU    b capped at 1e20, norms of q and b
//                            (src/problemdata.jl:73-136)
//   data_equilibrate! (GPU)  Ruiz scaling with full-P row norms
//                            (src/problemdata.jl:286-374, mathutils_gpu.jl)
//   CompositeConeGPU         cones ordered zero, nonneg, soc, exp, pow, psd
//                            (compositecone_type_gpu.jl:72-216).  Unlike the
//                            reference, unsorted cone lists are accepted and
//                            placed type-major; the solution is returned in
//                            the caller's row order.
//   _assemble_full_kkt_matrix  full KKT [P A'; A -Hs] with two extra rows and
//                            columns per second-order cone above the
//                            threshold (directgpu_kkt_assembly.jl:69-170)
// plus the ordering and symbolic factorisation that cuDSS's analysis phase
// performs in the reference (directldl_cudss.jl:20-23).
#include <algorithm>
#include <cmath>
#include <numeric>
#include <cstdint>
#include <set>

#include "pinned.hpp"
#include "setup.hpp"

namespace clgpu {

static inline int tri(int k) { return k * (k + 1) / 2; }
static inline double clip(double s, double lo, double hi) {
  return s < lo ? lo : (s > hi ? hi : s);
}

// ---------------------------------------------------------------- ordering
// Minimum-degree ordering on the explicit elimination graph.  Each step
// eliminates a vertex of smallest current degree and turns its neighbourhood
// into a clique.  Vertices whose initial degree exceeds 10*sqrt(n) are
// treated as dense and ordered last (as AMD does).
std::vector<int> amd_order(int n, std::vector<std::vector<int>> &adj) {
  for (auto &a : adj) {
    std::sort(a.begin(), a.end());
    a.erase(std::unique(a.begin(), a.end()), a.end());
  }
  double dense_thr = std::max(16.0, 10.0 * std::sqrt((double)n));
  std::vector<char> dense(n, 0), done(n, 0);
  std::set<std::pair<int, int>> pq;
  for (int i = 0; i < n; ++i) {
    if ((double)adj[i].size() > dense_thr)
      dense[i] = 1;
    else
      pq.insert({(int)adj[i].size(), i});
  }
  // dense vertices are dropped from the graph during the elimination
  if (std::any_of(dense.begin(), dense.end(), [](char c) { return c != 0; }))
    for (int i = 0; i < n; ++i) {
      if (dense[i]) continue;
      auto &a = adj[i];
      size_t w = 0;
      for (size_t r = 0; r < a.size(); ++r)
        if (!dense[a[r]]) a[w++] = a[r];
      if (w != a.size()) {
        pq.erase({(int)a.size(), i});
        a.resize(w);
        pq.insert({(int)a.size(), i});
      }
    }
  std::vector<int> order;
  order.reserve(n);
  std::vector<int> nb, tmp;
  while (!pq.empty()) {
    int v = pq.begin()->second;
    pq.erase(pq.begin());
    done[v] = 1;
    order.push_back(v);
    nb.clear();
    for (int u : adj[v])
      if (!done[u]) nb.push_back(u);
    for (int u : nb) {
      pq.erase({(int)adj[u].size(), u});
      tmp.clear();
      std::set_union(adj[u].begin(), adj[u].end(), nb.begin(), nb.end(),
                     std::back_inserter(tmp));
      auto &a = adj[u];
      a.clear();
      for (int w : tmp)
        if (w != u && !done[w]) a.push_back(w);
      pq.insert({(int)a.size(), u});
    }
    std::vector<int>().swap(adj[v]);
  }
  for (int i = 0; i < n; ++i)
    if (dense[i]) order.push_back(i);
  return order;
}

// Minimum degree on at most 32 vertices (adjacency as bit masks); ties go
// to the lower local index, as in amd_order.  Appends to order[no..].
static void md_small(const int *S, int k, const uint32_t *mask_in, int *order, int &no) {
  uint32_t m[32];
  for (int a = 0; a < k; ++a) m[a] = mask_in[a];
  uint32_t alive = k == 32 ? 0xffffffffu : ((1u << k) - 1u);
  for (int step = 0; step < k; ++step) {
    int best = -1, bd = 64;
    for (uint32_t w = alive; w; w &= w - 1) {
      const int a = __builtin_ctz(w);
      const int d = __builtin_popcount(m[a] & alive);
      if (d < bd) {
        bd = d;
        best = a;
      }
    }
    alive &= ~(1u << best);
    const uint32_t nb = m[best] & alive;
    for (uint32_t w = nb; w; w &= w - 1) {
      const int u = __builtin_ctz(w);
      m[u] |= nb;
      m[u] &= ~(1u << u);
    }
    order[no++] = S[best];
  }
}

std::vector<int> nd_order(int n, std::vector<std::vector<int>> &adj) {
  std::vector<int> xadj(n + 1, 0), adjncy;
  for (int i = 0; i < n; ++i) xadj[i + 1] = xadj[i] + (int)adj[i].size();
  adjncy.reserve(xadj[n]);
  for (auto &a : adj) adjncy.insert(adjncy.end(), a.begin(), a.end());
  return nd_order_csr(n, xadj, adjncy);
}

// Nested dissection (George's level-structure bisection).  A connected
// vertex set larger than kNdLeaf is split by a middle level of a breadth-first
// level structure rooted at a pseudo-peripheral vertex; only the vertices of
// that level with a neighbour in the next level form the separator.  The two
// halves are ordered first (recursively), the separator last, so the halves
// become independent subtrees of the elimination tree.  Small sets are
// ordered by minimum degree.  The KKT graphs of stage-structured problems
// are long and thin: minimum degree eliminates them from both ends inward
// and leaves an elimination tree of height ~N/2, while dissection keeps the
// height near (separator size) x log2(N), which is what bounds the
// level-scheduled factorisation and substitutions.  Dense vertices (degree
// above max(16, 10 sqrt(n))) are ordered last, as in amd_order.  The input
// CSR may hold repeated neighbours; it is deduplicated in place.
//
// The pending vertex sets form a stack whose lists live in one array: the
// set being split is always on top, its parts (which partition it) are
// written back over it, so the array never holds more than n vertices and
// the recursion allocates nothing.
std::vector<int> nd_order_csr(int n, std::vector<int> &xadj0, std::vector<int> &adj0) {
  constexpr int kNdLeaf = 8;
  // sort + deduplicate every row in place (rows are short: insertion sort)
  {
    int w = 0;
    for (int i = 0; i < n; ++i) {
      const int b0 = xadj0[i], len = xadj0[i + 1] - b0;
      int *r = adj0.data() + b0;
      for (int a = 1; a < len; ++a) {
        const int x = r[a];
        int c = a - 1;
        while (c >= 0 && r[c] > x) {
          r[c + 1] = r[c];
          --c;
        }
        r[c + 1] = x;
      }
      const int start = w;
      for (int q = 0; q < len; ++q)
        if (q == 0 || r[q] != r[q - 1]) adj0[w++] = r[q];
      xadj0[i] = start;
    }
    xadj0[n] = w;
  }
  const double dense_thr = std::max(16.0, 10.0 * std::sqrt((double)n));
  std::vector<char> dense(n, 0);
  bool any_dense = false;
  for (int i = 0; i < n; ++i) {
    dense[i] = (double)(xadj0[i + 1] - xadj0[i]) > dense_thr;
    any_dense |= dense[i] != 0;
  }
  // the graph without the dense vertices (a copy only when there are some:
  // the caller reads the deduplicated CSR afterwards)
  std::vector<int> xadj_nd, adj_nd;
  const int *xa = xadj0.data(), *ad = adj0.data();
  if (any_dense) {
    xadj_nd.assign(n + 1, 0);
    adj_nd.reserve(xadj0[n]);
    for (int i = 0; i < n; ++i) {
      if (!dense[i])
        for (int q = xadj0[i]; q < xadj0[i + 1]; ++q)
          if (!dense[adj0[q]]) adj_nd.push_back(adj0[q]);
      xadj_nd[i + 1] = (int)adj_nd.size();
    }
    xa = xadj_nd.data();
    ad = adj_nd.data();
  }
  std::vector<int> order(n);
  int no = 0;
  std::vector<int> work((size_t)n * 10 + 2);
  int *mark = work.data(), *lidx = mark + n, *indeg = lidx + n;
  // two level structures (the current best and a candidate); queue[s] lists
  // structure s's vertices in visiting order
  int *level[2] = {indeg + n, indeg + 2 * n};
  int *queue[2] = {indeg + 3 * n, indeg + 4 * n};
  int *arena = indeg + 5 * n;    // the pending sets' vertex lists
  int *scratch = indeg + 6 * n;  // a split's parts before they are written back
  int *lcount = indeg + 7 * n;   // vertices per level (depth <= n)
  for (int i = 0; i < n; ++i) {
    mark[i] = -1;
    level[0][i] = level[1][i] = -1;
  }
  int cnt[2] = {0, 0};
  int stamp = 0;
  struct Task {
    int off, len;
    bool emit;  // a separator: emitted as it is
  };
  std::vector<Task> stack;
  stack.reserve(64);
  {
    int top = 0;
    for (int i = 0; i < n; ++i)
      if (!dense[i]) arena[top++] = i;
    if (top) stack.push_back({0, top, false});
  }
  std::vector<int> cstart;
  // breadth-first levels of the set marked sid from src into structure b
  // (clearing b's previous visit); also records every visited vertex's
  // degree inside the set.  Returns the depth.
  auto bfs = [&](int src, int sid, int b) {
    int *lv = level[b], *qu = queue[b];
    for (int i = 0; i < cnt[b]; ++i) lv[qu[i]] = -1;
    int head = 0, tail = 0, depth = 0;
    qu[tail++] = src;
    lv[src] = 0;
    while (head < tail) {
      const int v = qu[head++];
      const int lnext = lv[v] + 1;
      depth = std::max(depth, lnext);
      int d = 0;
      for (int q = xa[v]; q < xa[v + 1]; ++q) {
        const int u = ad[q];
        if (mark[u] != sid) continue;
        ++d;
        if (lv[u] < 0) {
          lv[u] = lnext;
          qu[tail++] = u;
        }
      }
      indeg[v] = d;
    }
    cnt[b] = tail;
    return depth;
  };
  auto clear_levels = [&](int b) {
    for (int i = 0; i < cnt[b]; ++i) level[b][queue[b][i]] = -1;
    cnt[b] = 0;
  };
  std::vector<std::vector<int>> la;
  auto md_leaf = [&](const int *S, int k) {
    const int sid = ++stamp;
    for (int a = 0; a < k; ++a) {
      mark[S[a]] = sid;
      lidx[S[a]] = a;
    }
    if (k <= 32) {
      uint32_t masks[32];
      for (int a = 0; a < k; ++a) {
        uint32_t mk = 0;
        for (int q = xa[S[a]]; q < xa[S[a] + 1]; ++q)
          if (mark[ad[q]] == sid) mk |= 1u << lidx[ad[q]];
        masks[a] = mk;
      }
      md_small(S, k, masks, order.data(), no);
    } else {
      la.assign(k, {});
      for (int a = 0; a < k; ++a)
        for (int q = xa[S[a]]; q < xa[S[a] + 1]; ++q)
          if (mark[ad[q]] == sid) la[a].push_back(lidx[ad[q]]);
      for (int a : amd_order(k, la)) order[no++] = S[a];
    }
  };
  while (!stack.empty()) {
    const Task t = stack.back();
    stack.pop_back();
    int *S = arena + t.off;
    const int ns = t.len;
    if (t.emit) {
      for (int i = 0; i < ns; ++i) order[no++] = S[i];
      continue;
    }
    if (ns <= kNdLeaf) {
      md_leaf(S, ns);
      continue;
    }
    const int sid = ++stamp;
    for (int i = 0; i < ns; ++i) mark[S[i]] = sid;
    clear_levels(0);
    clear_levels(1);
    // connected components (dissect each on its own); the first search also
    // gives every vertex's degree inside the set
    bfs(S[0], sid, 0);
    if (cnt[0] < ns) {
      // components in discovery order, each in its search order, written
      // back so that the first one is on top
      const int comp_id = ++stamp;  // vertices already assigned get mark comp_id
      int nsc = 0;
      cstart.clear();
      for (int i = 0; i < ns; ++i) {
        const int v = S[i];
        if (mark[v] == comp_id) continue;
        bfs(v, sid, 1);
        cstart.push_back(nsc);
        for (int j = 0; j < cnt[1]; ++j) {
          scratch[nsc++] = queue[1][j];
          mark[queue[1][j]] = comp_id;
        }
      }
      cstart.push_back(nsc);
      clear_levels(0);
      clear_levels(1);
      int w = t.off;
      for (int c = (int)cstart.size() - 2; c >= 0; --c) {
        const int len = cstart[c + 1] - cstart[c];
        std::copy(scratch + cstart[c], scratch + cstart[c + 1], arena + w);
        stack.push_back({w, len, false});
        w += len;
      }
      continue;
    }
    // pseudo-peripheral root: a vertex of least degree in the set, then a
    // least-degree vertex of the deepest level while that deepens the
    // structure (three moves at most)
    int root = S[0];
    for (int i = 0; i < ns; ++i)
      if (indeg[S[i]] < indeg[root]) root = S[i];
    int cur = 0;
    int depth = bfs(root, sid, cur);
    for (int it = 0; it < 3; ++it) {
      const int *lv = level[cur], *qu = queue[cur];
      int cand = -1;
      for (int i = cnt[cur] - 1; i >= 0 && lv[qu[i]] == depth - 1; --i)
        if (cand < 0 || indeg[qu[i]] < indeg[cand]) cand = qu[i];
      const int d2 = bfs(cand, sid, 1 - cur);
      if (d2 <= depth) break;
      depth = d2;
      cur = 1 - cur;
    }
    const int *lev = level[cur];
    if (depth < 3) {
      md_leaf(S, ns);
      continue;
    }
    for (int l = 0; l < depth; ++l) lcount[l] = 0;
    for (int i = 0; i < ns; ++i) lcount[lev[S[i]]]++;
    int ell = 1, cum = 0;
    for (int l = 0; l < depth; ++l) {
      cum += lcount[l];
      if (2 * cum >= ns) {
        ell = std::max(1, std::min(depth - 2, l));
        break;
      }
    }
    // parts A (levels below ell, and the vertices of level ell without a
    // neighbour in level ell + 1), B (levels above ell) and the separator,
    // each in the set's order; written back as separator, B, A (A on top)
    int na = 0, nb = 0, nsep = 0;
    for (int i = 0; i < ns; ++i) {
      const int v = S[i];
      const int lv = lev[v];
      int part = 0;
      if (lv > ell) {
        part = 1;
      } else if (lv == ell) {
        for (int q = xa[v]; q < xa[v + 1]; ++q) {
          const int u = ad[q];
          if (mark[u] == sid && lev[u] == ell + 1) {
            part = 2;
            break;
          }
        }
      }
      lidx[v] = part;
      na += part == 0;
      nb += part == 1;
      nsep += part == 2;
    }
    std::copy(S, S + ns, scratch);
    int pa = t.off + nsep + nb, pb = t.off + nsep, ps = t.off;
    for (int i = 0; i < ns; ++i) {
      const int v = scratch[i];
      const int part = lidx[v];
      arena[part == 0 ? pa++ : (part == 1 ? pb++ : ps++)] = v;
    }
    stack.push_back({t.off, nsep, true});
    if (nb) stack.push_back({t.off + nsep, nb, false});
    if (na) stack.push_back({t.off + nsep + nb, na, false});
  }
  for (int i = 0; i < n; ++i)
    if (dense[i]) order[no++] = i;
  order.resize(no);
  return order;
}

// ---------------------------------------------------------------- helpers
static void csc_transpose(const HostCSC &A, HostCSC &T) {
  T.m = A.n;
  T.n = A.m;
  T.p.assign(A.m + 1, 0);
  for (int k = 0; k < A.p[A.n]; ++k) T.p[A.i[k] + 1]++;
  for (int r = 0; r < A.m; ++r) T.p[r + 1] += T.p[r];
  std::vector<int> next(T.p.begin(), T.p.end() - 1);
  T.i.assign(A.p[A.n], 0);
  T.x.assign(A.p[A.n], 0.0);
  for (int j = 0; j < A.n; ++j)
    for (int k = A.p[j]; k < A.p[j + 1]; ++k) {
      int q = next[A.i[k]]++;
      T.i[q] = j;
      T.x[q] = A.x[k];
    }
}

// entries of the single-warp kernels' encoded streams addressable by a
// chunk word (ldl.cuh kStartMask)
constexpr long long kStreamMaxEntries = (1LL << 22) - 1;

// dense columns: a factor column longer than this belongs to a dense front
// (the supernodal path factors it with tensor-core tiles; the single-warp
// kernels are built for sparse columns)
constexpr int kScalarMaxColumn = 512;

// true when the scalar factor of the pattern (CSR graph, repeats allowed,
// no self loops needed) under perm has more than `limit` entries below the
// diagonal, or a column longer than kScalarMaxColumn; elimination-tree
// path walk (Liu), stopping early
// When it returns false, parent and cnt hold the elimination tree and the
// column counts of L under perm (the symbolic factorisation reuses them).
static bool scalar_fill_exceeds(int N, const std::vector<int> &xadj,
                                const std::vector<int> &adj, const std::vector<int> &perm,
                                long long limit, std::vector<int> &parent,
                                std::vector<int> &cnt) {
  std::vector<int> iperm(N), mark(N, -1);
  parent.assign(N, -1);
  cnt.assign(N, 0);
  for (int k = 0; k < N; ++k) iperm[perm[k]] = k;
  long long lnz = 0;
  for (int k = 0; k < N; ++k) {
    mark[k] = k;
    const int o = perm[k];
    for (int p = xadj[o]; p < xadj[o + 1]; ++p) {
      int i = iperm[adj[p]];
      if (i >= k) continue;
      while (mark[i] != k) {
        if (parent[i] == -1) parent[i] = k;
        ++lnz;
        if (++cnt[i] > kScalarMaxColumn) return true;
        mark[i] = k;
        i = parent[i];
      }
    }
    if (lnz > limit) return true;
  }
  return false;
}

bool prepare_instance(const clgpu_problem &pb, const SetupOptions &opt, Prepared &out) {
  const int n = pb.n, m = pb.m;
  out = Prepared();
  out.n = n;
  out.m = m;
  if (n < 0 || m < 0) {
    out.error = "negative dimensions";
    return false;
  }
  // ---- cones: sizes and type-major order
  int rows = 0;
  std::vector<int> user_start(pb.ncones);
  for (int c = 0; c < pb.ncones; ++c) {
    int t = pb.cone_types[c], d = pb.cone_dims[c];
    int nv;
    if (t == CLGPU_CONE_EXP || t == CLGPU_CONE_POW)
      nv = 3;
    else if (t == CLGPU_CONE_PSD)
      nv = tri(d);
    else if (t >= 0 && t <= 5)
      nv = d;
    else {
      out.error = "unknown cone type";
      return false;
    }
    if (d < 0) {
      out.error = "negative cone dimension";
      return false;
    }
    if (t == CLGPU_CONE_POW) {
      double a = pb.cone_params ? pb.cone_params[c] : 0.0;
      if (!(a > 0 && a < 1)) {
        out.error = "power cone alpha must lie in (0,1)";
        return false;
      }
    }
    user_start[c] = rows;
    rows += nv;
  }
  if (rows != m) {
    out.error = "Constraint dimensions inconsistent with size of cones.";
    return false;
  }
  out.type_rows.assign(6, 0);
  out.type_cones.assign(6, 0);
  out.user_row_of.assign(m, 0);
  {
    int lr = 0;
    for (int t = 0; t < 6; ++t) {
      for (int c = 0; c < pb.ncones; ++c) {
        if (pb.cone_types[c] != t) continue;
        int d = pb.cone_dims[c];
        int nv = (t == 3 || t == 4) ? 3 : (t == 5 ? tri(d) : d);
        if (t == CLGPU_CONE_PSD && d == 0) continue;  // empty PSD cone: no rows
        out.ctype.push_back(t);
        out.cdim.push_back(t == 3 || t == 4 ? 3 : d);
        out.cparam.push_back(pb.cone_params ? pb.cone_params[c] : 0.0);
        out.cstart.push_back(lr);
        for (int k = 0; k < nv; ++k) out.user_row_of[lr + k] = user_start[c] + k;
        out.type_rows[t] += nv;
        out.type_cones[t] += 1;
        lr += nv;
        if (t == 3 || t == 4) out.symmetric = false;
        out.degree += (t == 0) ? 0 : (t == 2 ? 1 : (t == 3 || t == 4 ? 3 : d));
      }
    }
  }
  // ---- data: triu P -> full; A; q; b (capped)
  HostCSC Pu;
  Pu.m = Pu.n = n;
  Pu.p.assign(n + 1, 0);
  for (int j = 0; j < n; ++j) {
    for (int k = pb.Pp[j]; k < pb.Pp[j + 1]; ++k)
      if (pb.Pi[k] <= j) {
        Pu.i.push_back(pb.Pi[k]);
        Pu.x.push_back(pb.Px[k]);
      }
    Pu.p[j + 1] = (int)Pu.i.size();
  }
  out.p_nnz = Pu.p[n];
  bool pu_sorted = true;  // every triu column strictly increasing
  for (int j = 0; j < n && pu_sorted; ++j)
    for (int k = Pu.p[j] + 1; k < Pu.p[j + 1]; ++k)
      if (Pu.i[k] <= Pu.i[k - 1]) {
        pu_sorted = false;
        break;
      }
  if (pu_sorted) {
    // full = triu + strict triu transposed, built in place: column j gets
    // its own triu rows (<= j, ascending) when column j is visited, then the
    // rows i > j from the later columns i, in increasing i -- sorted, as the
    // general form's per-column sort leaves them
    HostCSC &F = out.Pfull;
    F.m = F.n = n;
    F.p.assign(n + 1, 0);
    for (int j = 0; j < n; ++j)
      for (int k = Pu.p[j]; k < Pu.p[j + 1]; ++k) {
        F.p[j + 1]++;
        if (Pu.i[k] != j) F.p[Pu.i[k] + 1]++;
      }
    for (int j = 0; j < n; ++j) F.p[j + 1] += F.p[j];
    F.i.resize(F.p[n]);
    F.x.resize(F.p[n]);
    std::vector<int> pos(F.p.begin(), F.p.end() - 1);
    for (int j = 0; j < n; ++j)
      for (int k = Pu.p[j]; k < Pu.p[j + 1]; ++k) {
        const int i = Pu.i[k];
        F.i[pos[j]] = i;
        F.x[pos[j]++] = Pu.x[k];
        if (i != j) {
          F.i[pos[i]] = j;
          F.x[pos[i]++] = Pu.x[k];
        }
      }
  } else {
    // full = triu + strict triu transposed
    std::vector<std::vector<std::pair<int, double>>> cols(n);
    for (int j = 0; j < n; ++j)
      for (int k = Pu.p[j]; k < Pu.p[j + 1]; ++k) {
        int i = Pu.i[k];
        cols[j].push_back({i, Pu.x[k]});
        if (i != j) cols[i].push_back({j, Pu.x[k]});
      }
    HostCSC &F = out.Pfull;
    F.m = F.n = n;
    F.p.assign(n + 1, 0);
    for (int j = 0; j < n; ++j) {
      std::sort(cols[j].begin(), cols[j].end());
      for (auto &pr : cols[j]) {
        F.i.push_back(pr.first);
        F.x.push_back(pr.second);
      }
      F.p[j + 1] = (int)F.i.size();
    }
  }
  out.A.m = m;
  out.A.n = n;
  out.A.p.assign(pb.Ap, pb.Ap + n + 1);
  out.A.i.assign(pb.Ai, pb.Ai + pb.Ap[n]);
  out.A.x.assign(pb.Ax, pb.Ax + pb.Ap[n]);
  for (int k = 0; k < out.A.p[n]; ++k)
    if (out.A.i[k] < 0 || out.A.i[k] >= m) {
      out.error = "A row index out of range";
      return false;
    }
  out.q.assign(pb.q, pb.q + n);
  out.b.assign(pb.b, pb.b + m);
  for (auto &v : out.b) v = std::min(v, 1e20);
  out.normq = 0;
  for (double v : out.q) out.normq = std::max(out.normq, std::fabs(v));
  out.normb = 0;
  for (double v : out.b) out.normb = std::max(out.normb, std::fabs(v));
  // ---- Ruiz equilibration (GPU path semantics)
  std::vector<double> &d = out.d, &e = out.e;
  d.assign(n, 1.0);
  e.assign(m, 1.0);
  out.c = 1.0;
  HostCSC &P = out.Pfull, &A = out.A;
  auto scale_data = [&](const std::vector<double> *dw, const std::vector<double> &ew) {
    if (dw) {
      for (int j = 0; j < n; ++j)
        for (int k = P.p[j]; k < P.p[j + 1]; ++k) P.x[k] *= (*dw)[P.i[k]] * (*dw)[j];
      for (int j = 0; j < n; ++j)
        for (int k = A.p[j]; k < A.p[j + 1]; ++k) A.x[k] *= ew[A.i[k]] * (*dw)[j];
      for (int i = 0; i < n; ++i) out.q[i] *= (*dw)[i];
    } else {
      for (int k = 0; k < A.p[n]; ++k) A.x[k] *= ew[A.i[k]];
    }
    for (int i = 0; i < m; ++i) out.b[i] *= ew[i];
  };
  // the device can take the numeric part of setup when every value has one
  // KKT position: P's upper entries and A's entries sorted, none repeated
  if (opt.defer_equilibration) {
    bool sorted = true;
    for (int j = 0; j < n && sorted; ++j)
      for (int k = pb.Pp[j] + 1; k < pb.Pp[j + 1]; ++k)
        if (pb.Pi[k] <= j && pb.Pi[k - 1] >= pb.Pi[k]) sorted = false;
    for (int j = 0; j < n && sorted; ++j)
      for (int k = pb.Ap[j] + 1; k < pb.Ap[j + 1]; ++k)
        if (pb.Ai[k - 1] >= pb.Ai[k]) sorted = false;
    out.eq_deferred = sorted;
  }
  if (opt.equilibrate_enable && !out.eq_deferred) {
    double smin = opt.equilibrate_min_scaling, smax = opt.equilibrate_max_scaling;
    std::vector<double> dw(n), ew(m);
    for (int it = 0; it < opt.equilibrate_max_iter; ++it) {
      std::fill(dw.begin(), dw.end(), 0.0);
      std::fill(ew.begin(), ew.end(), 0.0);
      for (int j = 0; j < n; ++j)
        for (int k = P.p[j]; k < P.p[j + 1]; ++k)
          dw[j] = std::max(dw[j], std::fabs(P.x[k]));
      for (int j = 0; j < n; ++j)
        for (int k = A.p[j]; k < A.p[j + 1]; ++k) {
          double t = std::fabs(A.x[k]);
          dw[j] = std::max(dw[j], t);
          ew[A.i[k]] = std::max(ew[A.i[k]], t);
        }
      for (auto &v : dw) v = (v == 0.0) ? 1.0 : v;
      for (auto &v : ew) v = (v == 0.0) ? 1.0 : v;
      for (auto &v : dw) v = 1.0 / std::sqrt(v);
      for (auto &v : ew) v = 1.0 / std::sqrt(v);
      for (int i = 0; i < n; ++i) dw[i] = clip(dw[i], smin / d[i], smax / d[i]);
      for (int i = 0; i < m; ++i) ew[i] = clip(ew[i], smin / e[i], smax / e[i]);
      scale_data(&dw, ew);
      for (int i = 0; i < n; ++i) d[i] *= dw[i];
      for (int i = 0; i < m; ++i) e[i] *= ew[i];
      // mean of the row norms of the (full) scaled P
      std::fill(dw.begin(), dw.end(), 0.0);
      for (int j = 0; j < n; ++j)
        for (int k = P.p[j]; k < P.p[j + 1]; ++k)
          dw[j] = std::max(dw[j], std::fabs(P.x[k]));
      double mean = 0;
      for (double v : dw) mean += v;
      mean = n > 0 ? mean / n : 0.0;
      double inf_q = 0;
      for (double v : out.q) inf_q = std::max(inf_q, std::fabs(v));
      if (mean != 0.0 && inf_q != 0.0) {
        double sc = std::max(inf_q, mean);
        double ct = clip(1.0 / sc, smin / out.c, smax / out.c);
        for (auto &v : P.x) v *= ct;
        for (auto &v : out.q) v *= ct;
        out.c *= ct;
      }
    }
    // rectify_equilibration!: cones without elementwise scaling get
    // delta = mean(e)/e over the cone (coneops_defaults.jl:32-44)
    bool any = false;
    std::vector<double> delta(m, 1.0);
    for (size_t c = 0; c < out.ctype.size(); ++c) {
      int t = out.ctype[c];
      if (t == CLGPU_CONE_ZERO || t == CLGPU_CONE_NONNEG) continue;
      int nv = (t == 3 || t == 4) ? 3 : (t == 5 ? tri(out.cdim[c]) : out.cdim[c]);
      if (nv == 0) continue;
      any = true;
      double mu = 0;
      for (int k = 0; k < nv; ++k) mu += e[out.user_row_of[out.cstart[c] + k]];
      mu /= nv;
      for (int k = 0; k < nv; ++k) {
        int r = out.user_row_of[out.cstart[c] + k];
        delta[r] = mu / e[r];
      }
    }
    if (any) {
      scale_data(nullptr, delta);
      for (int i = 0; i < m; ++i) e[i] *= delta[i];
    }
  }

  // ---- KKT pattern (local): x 0..n-1, z rows n..n+m-1 in type-major local
  // order, 2 extra per sparse SOC after that.
  std::vector<int> local_of_user(m);
  for (int lr = 0; lr < m; ++lr) local_of_user[out.user_row_of[lr]] = lr;
  int nsparse = 0;
  std::vector<int> sparse_idx(out.ctype.size(), -1);
  for (size_t c = 0; c < out.ctype.size(); ++c)
    if (out.ctype[c] == CLGPU_CONE_SOC && out.cdim[c] > opt.soc_threshold)
      sparse_idx[c] = nsparse++;
  const int N = n + m + 2 * nsparse;
  out.N = N;
  // entries (r <= c); source tags resolved later by position lookups
  struct Ent {
    int r, c;
    double v;
  };
  std::vector<Ent> ents;
  ents.reserve(P.p[n] + A.p[n] + N + 16);
  for (int j = 0; j < n; ++j) {
    bool hasdiag = false;
    for (int k = P.p[j]; k < P.p[j + 1]; ++k) {
      int i = P.i[k];
      if (i <= j) ents.push_back({i, j, P.x[k]});
      if (i == j) hasdiag = true;
    }
    if (!hasdiag) ents.push_back({j, j, 0.0});
  }
  for (int j = 0; j < n; ++j)
    for (int k = A.p[j]; k < A.p[j + 1]; ++k)
      ents.push_back({j, n + local_of_user[A.i[k]], A.x[k]});
  for (size_t c = 0; c < out.ctype.size(); ++c) {
    int t = out.ctype[c], st = n + out.cstart[c];
    int nv = (t == 3 || t == 4) ? 3 : (t == 5 ? tri(out.cdim[c]) : out.cdim[c]);
    bool diag = (t == CLGPU_CONE_ZERO || t == CLGPU_CONE_NONNEG || sparse_idx[c] >= 0);
    if (diag) {
      for (int k = 0; k < nv; ++k) ents.push_back({st + k, st + k, 0.0});
    } else {
      for (int col = 0; col < nv; ++col)
        for (int row = 0; row <= col; ++row) ents.push_back({st + row, st + col, 0.0});
    }
    if (sparse_idx[c] >= 0) {
      int pc = n + m + 2 * sparse_idx[c];
      for (int k = 0; k < nv; ++k) {
        ents.push_back({st + k, pc, 0.0});
        ents.push_back({st + k, pc + 1, 0.0});
      }
      ents.push_back({pc, pc, 0.0});
      ents.push_back({pc + 1, pc + 1, 0.0});
    }
  }
  // ---- ordering (graph of the off-diagonal pattern, CSR with repeats)
  std::vector<int> etree, colcnt;  // from the fill check (scalar path)
  {
    std::vector<int> xadj(N + 1, 0);
    for (auto &en : ents)
      if (en.r != en.c) {
        xadj[en.r + 1]++;
        xadj[en.c + 1]++;
      }
    for (int i = 0; i < N; ++i) xadj[i + 1] += xadj[i];
    std::vector<int> adjncy(xadj[N]), cur(xadj.begin(), xadj.end() - 1);
    for (auto &en : ents)
      if (en.r != en.c) {
        adjncy[cur[en.r]++] = en.c;
        adjncy[cur[en.c]++] = en.r;
      }
    // instances whose work vector exceeds the single-warp kernels' budget
    // (48 KB of FP64), whose factor or matrix exceeds the range of their
    // stream chunk words, or whose factor has dense columns (> 512 entries)
    // take the supernodal factorisation
    out.supernodal = (long long)N * 8 > 48 * 1024 || (long long)xadj[N] + N > kStreamMaxEntries;
    if (!out.supernodal) {
      out.perm = nd_order_csr(N, xadj, adjncy);
      out.supernodal = scalar_fill_exceeds(N, xadj, adjncy, out.perm, kStreamMaxEntries,
                                           etree, colcnt);
    }
    if (out.supernodal) {
      if (!sn_analyse(N, xadj, adjncy, out.perm, out.sym, &out.error)) return false;
    }
  }
  out.iperm.assign(N, 0);
  for (int k = 0; k < N; ++k) out.iperm[out.perm[k]] = k;
  // ---- permuted full CSR (sorted columns, duplicates summed)
  {
    std::vector<int> rs(N + 1, 0);
    for (auto &en : ents) {
      const int a = out.iperm[en.r], bb = out.iperm[en.c];
      rs[a + 1]++;
      if (a != bb) rs[bb + 1]++;
    }
    for (int r = 0; r < N; ++r) rs[r + 1] += rs[r];
    std::vector<std::pair<int, double>> rv(rs[N]);
    {
      std::vector<int> cur(rs.begin(), rs.end() - 1);
      for (auto &en : ents) {
        const int a = out.iperm[en.r], bb = out.iperm[en.c];
        rv[cur[a]++] = {bb, en.v};
        if (a != bb) rv[cur[bb]++] = {a, en.v};
      }
    }
    out.Kp.assign(N + 1, 0);
    out.Kdiag.assign(N, -1);
    out.Kj.reserve(rs[N]);
    out.Kx.reserve(rs[N]);
    for (int r = 0; r < N; ++r) {
      auto *b0 = rv.data() + rs[r], *b1 = rv.data() + rs[r + 1];
      // rows are short: insertion sort by column (stable)
      for (auto *x = b0 + 1; x < b1; ++x) {
        auto v = *x;
        auto *y = x;
        while (y > b0 && (y - 1)->first > v.first) {
          *y = *(y - 1);
          --y;
        }
        *y = v;
      }
      const int start = (int)out.Kj.size();
      for (auto *x = b0; x < b1; ++x) {
        if ((int)out.Kj.size() > start && out.Kj.back() == x->first) {
          out.Kx.back() += x->second;
          continue;
        }
        out.Kj.push_back(x->first);
        out.Kx.push_back(x->second);
        if (x->first == r) out.Kdiag[r] = (int)out.Kj.size() - 1;
      }
      out.Kp[r + 1] = (int)out.Kj.size();
    }
  }
  auto pos_of = [&](int lr, int lc) -> int {  // local unpermuted (lr, lc)
    int a = out.iperm[lr], bb = out.iperm[lc];
    auto beg = out.Kj.begin() + out.Kp[a], end = out.Kj.begin() + out.Kp[a + 1];
    auto it = std::lower_bound(beg, end, bb);
    return (it != end && *it == bb) ? (int)(it - out.Kj.begin()) : -1;
  };
  // Dsigns: +1 x, -1 z, (-1,+1) per sparse SOC pair
  out.Dsign.assign(N, 1);
  for (int o = 0; o < N; ++o) {
    signed char sgn = 1;
    if (o >= n && o < n + m) sgn = -1;
    if (o >= n + m) sgn = ((o - n - m) % 2 == 0) ? -1 : 1;
    out.Dsign[out.iperm[o]] = sgn;
  }
  // ---- symbolic LDL^T on the permuted matrix (scalar structures; the
  // supernodal instances have theirs from sn_analyse)
  if (out.supernodal) {
    out.Lp.assign(N + 1, 0);
    out.Rp.assign(N + 1, 0);
    out.lvl_ptr.assign(1, 0);
  } else {
    // elimination tree and column counts: those of the fill check (the same
    // pattern and ordering), else from the permuted matrix
    std::vector<int> parent, Lnz, work(N, -1);
    if ((int)etree.size() == N && (int)colcnt.size() == N) {
      parent.swap(etree);
      Lnz.swap(colcnt);
    } else {
      parent.assign(N, -1);
      Lnz.assign(N, 0);
      for (int k = 0; k < N; ++k) {
        work[k] = k;
        for (int p = out.Kp[k]; p < out.Kp[k + 1]; ++p) {
          int i = out.Kj[p];
          if (i >= k) break;
          while (work[i] != k) {
            if (parent[i] == -1) parent[i] = k;
            Lnz[i]++;
            work[i] = k;
            i = parent[i];
          }
        }
      }
    }
    out.Lp.assign(N + 1, 0);
    for (int i = 0; i < N; ++i) out.Lp[i + 1] = out.Lp[i] + Lnz[i];
    long long lnz = out.Lp[N];
    if (lnz > 1500000000LL) {
      out.error = "factor too large";
      return false;
    }
    out.Li.assign(lnz, 0);
    out.Rp.assign(N + 1, 0);
    out.Rk.reserve(lnz);
    out.Rpos.reserve(lnz);
    std::vector<int> next(out.Lp.begin(), out.Lp.end() - 1);
    std::fill(work.begin(), work.end(), -1);
    for (int k = 0; k < N; ++k) {
      work[k] = k;
      for (int p = out.Kp[k]; p < out.Kp[k + 1]; ++p) {
        int i = out.Kj[p];
        if (i >= k) break;
        while (work[i] != k) {
          int q = next[i]++;
          out.Li[q] = k;
          out.Rk.push_back(i);
          out.Rpos.push_back(q);
          work[i] = k;
          i = parent[i];
        }
      }
      out.Rp[k + 1] = (int)out.Rk.size();
    }
    // elimination-tree levels (longest path from a leaf): every node of a
    // level depends only on nodes of lower levels, so a level's columns can
    // be factored and substituted concurrently
    std::vector<int> lev(N, 0);
    int nlev = 0;
    for (int j = 0; j < N; ++j) {
      if (parent[j] >= 0) lev[parent[j]] = std::max(lev[parent[j]], lev[j] + 1);
      nlev = std::max(nlev, lev[j] + 1);
    }
    out.lvl_ptr.assign(nlev + 1, 0);
    for (int j = 0; j < N; ++j) out.lvl_ptr[lev[j] + 1]++;
    for (int l = 0; l < nlev; ++l) out.lvl_ptr[l + 1] += out.lvl_ptr[l];
    out.lvl_nodes.assign(N, 0);
    std::vector<int> cur(out.lvl_ptr.begin(), out.lvl_ptr.end() - 1);
    for (int j = 0; j < N; ++j) out.lvl_nodes[cur[lev[j]]++] = j;
  }
  // ---- value-update maps
  {
    const int pnz = pb.Pp[n];
    out.p_user_nnz = pnz;
    out.pmap.assign(4 * (size_t)pnz, -1);
    out.pxy.assign(2 * (size_t)pnz, -1);
    const HostCSC &F = out.Pfull;
    auto fpos = [&](int r, int c) -> int {  // position of (r, c) in the full CSC
      auto beg = F.i.begin() + F.p[c], end = F.i.begin() + F.p[c + 1];
      auto it = std::lower_bound(beg, end, r);
      return (it != end && *it == r) ? (int)(it - F.i.begin()) : -1;
    };
    // KKT positions by row scatter: every lookup of a column j below is in
    // KKT row iperm[j] (scattered into kcol, stamped by row), and the
    // transposed entry's position comes from ktr: rows of the symmetric
    // pattern are sorted, so walking the rows in order meets the entries
    // (c, r) of each row c in increasing r (one cursor per row)
    const int KN = (int)out.Kp.size() - 1, knz = (int)out.Kj.size();
    std::vector<int> ktr(knz), kcur(out.Kp.begin(), out.Kp.end() - 1), kcol(KN, -1),
        kstamp(KN, -1);
    for (int r = 0; r < KN; ++r)
      for (int q = out.Kp[r]; q < out.Kp[r + 1]; ++q) ktr[q] = kcur[out.Kj[q]]++;
    auto scatter_row = [&](int lr) {  // row of local (unpermuted) index lr
      const int a = out.iperm[lr];
      for (int q = out.Kp[a]; q < out.Kp[a + 1]; ++q) {
        kcol[out.Kj[q]] = q;
        kstamp[out.Kj[q]] = a;
      }
      return a;
    };
    auto in_row = [&](int a, int lc) {  // position of (row a, local column lc), or -1
      const int bb = out.iperm[lc];
      return kstamp[bb] == a ? kcol[bb] : -1;
    };
    for (int j = 0; j < n; ++j) {
      const int a = scatter_row(j);
      for (int k = pb.Pp[j]; k < pb.Pp[j + 1]; ++k) {
        const int i = pb.Pi[k];
        if (i > j) continue;
        if (k > pb.Pp[j] && pb.Pi[k - 1] >= i) out.updatable = false;  // repeats / unsorted
        out.pmap[4 * (size_t)k] = fpos(i, j);
        out.pmap[4 * (size_t)k + 1] = i != j ? fpos(j, i) : -1;
        const int pji = in_row(a, i);  // (j, i); its transpose is (i, j)
        out.pmap[4 * (size_t)k + 2] = pji >= 0 ? ktr[pji] : -1;
        out.pmap[4 * (size_t)k + 3] = i != j ? pji : -1;
        out.pxy[2 * (size_t)k] = i;
        out.pxy[2 * (size_t)k + 1] = j;
      }
    }
    const int anz = A.p[n];
    out.amapk.assign(2 * (size_t)anz, -1);
    for (int j = 0; j < n; ++j) {
      const int a = scatter_row(j);
      for (int k = A.p[j]; k < A.p[j + 1]; ++k) {
        if (k > A.p[j] && A.i[k - 1] >= A.i[k]) out.updatable = false;
        const int zr = n + local_of_user[A.i[k]];
        const int pjz = in_row(a, zr);
        out.amapk[2 * (size_t)k] = pjz;
        out.amapk[2 * (size_t)k + 1] = pjz >= 0 ? ktr[pjz] : -1;
      }
    }
  }
  // ---- refresh positions
  for (size_t c = 0; c < out.ctype.size(); ++c) {
    int t = out.ctype[c], st = n + out.cstart[c];
    int nv = (t == 3 || t == 4) ? 3 : (t == 5 ? tri(out.cdim[c]) : out.cdim[c]);
    if (t == CLGPU_CONE_NONNEG) {
      for (int k = 0; k < nv; ++k) out.nn_pos.push_back(pos_of(st + k, st + k));
    } else if (t == CLGPU_CONE_SOC) {
      if (sparse_idx[c] >= 0) {
        int pc = n + m + 2 * sparse_idx[c];
        out.socd_start.push_back(-1);
        for (int k = 0; k < nv; ++k) {
          out.socs_diag.push_back(pos_of(st + k, st + k));
          out.socs_uv.push_back(pos_of(st + k, pc));
          out.socs_uv.push_back(pos_of(pc, st + k));
          out.socs_uv.push_back(pos_of(st + k, pc + 1));
          out.socs_uv.push_back(pos_of(pc + 1, st + k));
        }
        out.socs_D.push_back(pos_of(pc, pc));
        out.socs_D.push_back(pos_of(pc + 1, pc + 1));
      } else {
        out.socd_start.push_back((int)out.socd_pos.size() / 2);
        for (int col = 0; col < nv; ++col)
          for (int row = 0; row <= col; ++row) {
            out.socd_pos.push_back(pos_of(st + row, st + col));
            out.socd_pos.push_back(row == col ? -1 : pos_of(st + col, st + row));
          }
        for (int k = 0; k < nv; ++k) {
          out.socs_diag.push_back(-1);
          for (int q = 0; q < 4; ++q) out.socs_uv.push_back(-1);
        }
        out.socs_D.push_back(-1);
        out.socs_D.push_back(-1);
      }
    } else if (t == CLGPU_CONE_EXP || t == CLGPU_CONE_POW) {
      std::vector<int> &pp = (t == CLGPU_CONE_EXP) ? out.exp_pos : out.pow_pos;
      const int ri[6] = {0, 0, 1, 0, 1, 2}, ci[6] = {0, 1, 1, 2, 2, 2};
      for (int k = 0; k < 6; ++k) {
        pp.push_back(pos_of(st + ri[k], st + ci[k]));
        pp.push_back(ri[k] == ci[k] ? -1 : pos_of(st + ci[k], st + ri[k]));
      }
    } else if (t == CLGPU_CONE_PSD) {
      out.psd_start.push_back((int)out.psd_pos.size() / 2);
      for (int col = 0; col < nv; ++col)
        for (int row = 0; row <= col; ++row) {
          out.psd_pos.push_back(pos_of(st + row, st + col));
          out.psd_pos.push_back(row == col ? -1 : pos_of(st + col, st + row));
        }
    }
  }
  for (int v : out.nn_pos)
    if (v < 0) {
      out.error = "internal: missing KKT position";
      return false;
    }
  return true;
}

}  // namespace clgpu

// ------------------------------------------------------------------ check
// Host replay of the device factorisation/solve on the prepared structures.
// Used by tests (no GPU needed) to validate the ordering, symbolic
// factorisation and every refresh map before any kernel reads them.
extern "C" int clgpu_debug_pinned_stats(long long *out) {
  if (!out) return -1;
  clgpu::PinnedPool::get().stats(out);
  return 0;
}

extern "C" int clgpu_debug_instance_path(const clgpu_problem *pb, const clgpu_settings *st,
                                         int *supernodal, long long *factor_entries) {
  using namespace clgpu;
  SetupOptions opt;
  if (st) {
    opt.soc_threshold = st->soc_threshold;
    opt.equilibrate_enable = st->equilibrate_enable;
    opt.equilibrate_max_iter = st->equilibrate_max_iter;
  }
  Prepared p;
  if (!prepare_instance(*pb, opt, p)) return -2;
  if (supernodal) *supernodal = p.supernodal ? 1 : 0;
  if (factor_entries) {
    long long e = 0;
    if (p.supernodal) {
      for (int t = 0; t < p.sym.ns(); ++t) {
        const long long nc = p.sym.col0[t + 1] - p.sym.col0[t], nr = p.sym.rptr[t + 1] - p.sym.rptr[t];
        e += nc * (nc - 1) / 2 + nc * nr;
      }
    } else {
      e = (long long)p.Li.size();
    }
    *factor_entries = e;
  }
  return 0;
}

extern "C" int clgpu_debug_check_instance(const clgpu_problem *pb, const clgpu_settings *st,
                                          double *resid) {
  using namespace clgpu;
  SetupOptions opt;
  if (st) {
    opt.soc_threshold = st->soc_threshold;
    opt.equilibrate_enable = st->equilibrate_enable;
    opt.equilibrate_max_iter = st->equilibrate_max_iter;
  }
  Prepared p;
  if (!prepare_instance(*pb, opt, p)) return -2;
  const int N = p.N;
  const int knz = (int)p.Kj.size(), lnz = (int)p.Li.size();
  // bounds of every index structure the kernels use
  if ((int)p.Kp.size() != N + 1 || p.Kp[N] != knz) return -10;
  for (int r = 0; r < N; ++r) {
    if (p.Kdiag[r] < p.Kp[r] || p.Kdiag[r] >= p.Kp[r + 1]) return -11;
    for (int q = p.Kp[r]; q < p.Kp[r + 1]; ++q)
      if (p.Kj[q] < 0 || p.Kj[q] >= N || (q > p.Kp[r] && p.Kj[q] <= p.Kj[q - 1])) return -12;
  }
  if (p.supernodal) {
    // supernodal instance: build its device plan and replay the multifrontal
    // factorisation and solve on a quasi-definite test matrix
    auto inK0 = [&](int v) { return v == -1 || (v >= 0 && v < knz); };
    for (int v : p.nn_pos) if (!inK0(v) || v < 0) return -16;
    for (int v : p.socd_pos) if (!inK0(v)) return -17;
    for (int v : p.socs_uv) if (!inK0(v)) return -19;
    SnPlan plan;
    std::string err;
    std::vector<SnInstance> in{{&p.sym, p.Kp.data(), p.Kj.data(), 0, 0, 0}};
    if (!sn_build_plan(in, plan, &err)) return -30;
    for (size_t q = 0; q < plan.amap.size(); ++q) {
      const SnPair a = plan.amap[q];
      if (a.x < 0 || a.x >= knz) return -31;
    }
    for (int s = 0; s < plan.ns; ++s) {
      const long long ld = plan.ld[s];
      for (int q = plan.acol[plan.cbase[s]]; q < plan.acol[plan.cbase[s] + plan.ncol[s]]; ++q) {
        const int off = plan.amap[q].y, r = off % (int)ld, c = off / (int)ld;
        if (c >= plan.ncol[s] || r < c || r >= ld) return -32;
      }
      for (int k = 0; k < plan.nrow[s]; ++k) {
        const int* fi = plan.fidx.data() + plan.fix_off[s];
        if (fi[plan.u0[s] + k] < 0 || fi[plan.u0[s] + k] >= N) return -33;
      }
    }
    // children: relative indices strictly increasing, inside the parent's
    // front and never on its dummy or padding positions
    for (int s = 0; s < plan.ns; ++s)
      for (int a = plan.ch_ptr[s]; a < plan.ch_ptr[s + 1]; ++a) {
        const int c = plan.ch[a];
        const int *rel = plan.rel.data() + plan.rel_off[c];
        const int *fi = plan.fidx.data() + plan.fix_off[s];
        for (int k = 0; k < plan.nrow[c]; ++k) {
          if (rel[k] < 0 || rel[k] >= plan.ld[s] || fi[rel[k]] < 0) return -34;
          if (k > 0 && rel[k] <= rel[k - 1]) return -35;
        }
      }
    // every launch's tasks inside the task list, tiles inside their fronts
    for (auto *sched : {&plan.fact, &plan.fwd, &plan.bwd})
      for (const SnLaunch &L : *sched) {
        if (L.begin < 0 || L.count <= 0 || (size_t)L.begin + L.count > plan.tasks.size()) return -36;
        for (int q = L.begin; q < L.begin + L.count; ++q) {
          const SnQuad t = plan.tasks[q];
          if (t.x < 0 || t.x >= plan.ns) return -37;
          const int ld = plan.ld[t.x], k0 = t.y & 0xffff, K = t.y >> 16;
          if (L.kind == SN_DIAG || L.kind == SN_TRSM || L.kind == SN_UPDATE ||
              L.kind == SN_FWD_DIAG || L.kind == SN_FWD_GEMV || L.kind == SN_BWD_PARTIAL ||
              L.kind == SN_BWD_DIAG) {
            if (!plan.large[t.x] || K <= 0 || K > kSnNB || K % kSnKPad || k0 + K > plan.u0[t.x])
              return -38;
            if ((L.kind == SN_TRSM || L.kind == SN_UPDATE || L.kind == SN_FWD_GEMV ||
                 L.kind == SN_BWD_PARTIAL) &&
                (t.z < k0 + K || t.z + kSnNB > ld || (t.z - k0 - K) % kSnNB))
              return -39;
            if (L.kind == SN_UPDATE &&
                (t.w < k0 + K || t.w + 64 > ld || (t.w - k0 - K) % 64 || t.z + kSnNB <= t.w))
              return -40;
          }
          if ((L.kind == SN_ASSEMBLE || L.kind == SN_FWD_GATHER) &&
              (t.y < 0 || t.z > ld || t.y >= t.z))
            return -41;
          if (L.kind == SN_ASSEMBLE || L.kind == SN_FWD_GATHER) {
            // the chunk's children: entries q of each map inside [t.y, t.z)
            if (t.w < plan.chunk_off[t.x] || t.w >= plan.chunk_off[t.x + 1] ||
                (t.w - plan.chunk_off[t.x]) * kSnAsmCols != t.y)
              return -44;
            for (int e = plan.cl_ptr[t.w]; e < plan.cl_ptr[t.w + 1]; ++e) {
              const SnQuad c = plan.clist[e];
              bool child = false;
              for (int a = plan.ch_ptr[t.x]; a < plan.ch_ptr[t.x + 1]; ++a) child |= plan.ch[a] == c.x;
              if (!child || c.y < 0 || c.y >= c.z || c.z > plan.nrow[c.x]) return -45;
              const int *rel = plan.rel.data() + plan.rel_off[c.x];
              if (rel[c.y] < t.y || rel[c.z - 1] >= t.z) return -46;
            }
          }
          if ((L.kind == SN_SMALL_FACTOR || L.kind == SN_FWD_SMALL || L.kind == SN_BWD_SMALL) &&
              (plan.large[t.x] || ld > kSnSmallMax))
            return -42;
        }
      }
    std::vector<double> Kx(knz, 0.0);
    for (int r = 0; r < N; ++r)
      for (int q = p.Kp[r]; q < p.Kp[r + 1]; ++q) {
        int c = p.Kj[q];
        if (c != r) Kx[q] = 0.01 * std::sin(1.0 + r + 7.0 * c) * std::sin(1.0 + c + 7.0 * r);
      }
    for (int r = 0; r < N; ++r) Kx[p.Kdiag[r]] = p.Dsign[r] * 2.0;
    std::vector<int> voff{0, N};
    const double res = sn_host_check(plan, p.Kp, p.Kj, Kx, p.Dsign, voff, 1e-7);
    if (resid) *resid = res;
    return 0;
  }
  if ((int)p.Lp.size() != N + 1 || p.Lp[N] != lnz || (int)p.Rp.size() != N + 1) return -13;
  for (int j = 0; j < N; ++j)
    for (int q = p.Lp[j]; q < p.Lp[j + 1]; ++q)
      if (p.Li[q] <= j || p.Li[q] >= N || (q > p.Lp[j] && p.Li[q] <= p.Li[q - 1])) return -14;
  for (int j = 0; j < N; ++j)
    for (int q = p.Rp[j]; q < p.Rp[j + 1]; ++q) {
      int k = p.Rk[q], pos = p.Rpos[q];
      if (k < 0 || k >= j || pos < p.Lp[k] || pos >= p.Lp[k + 1] || p.Li[pos] != j) return -15;
    }
  auto inK = [&](int v, bool allow_neg) { return (allow_neg && v == -1) || (v >= 0 && v < knz); };
  for (int v : p.nn_pos) if (!inK(v, false)) return -16;
  for (int v : p.socd_pos) if (!inK(v, true)) return -17;
  for (int v : p.socs_diag) if (!inK(v, true)) return -18;
  for (int v : p.socs_uv) if (!inK(v, true)) return -19;
  for (int v : p.socs_D) if (!inK(v, true)) return -20;
  for (int v : p.exp_pos) if (!inK(v, true)) return -21;
  for (int v : p.pow_pos) if (!inK(v, true)) return -22;
  for (int v : p.psd_pos) if (!inK(v, true)) return -23;
  // a quasi-definite test matrix on the KKT pattern: +/-(1 + 1e-3*rowsum)
  std::vector<double> Kx(knz, 0.0);
  for (int r = 0; r < N; ++r)
    for (int q = p.Kp[r]; q < p.Kp[r + 1]; ++q) {
      int c = p.Kj[q];
      if (c != r) Kx[q] = 0.01 * std::sin(1.0 + r + 7.0 * c) * std::sin(1.0 + c + 7.0 * r);
    }
  for (int r = 0; r < N; ++r) Kx[p.Kdiag[r]] = p.Dsign[r] * 2.0;
  // level-scheduled left-looking factorisation, same loops as the kernel:
  // wide levels merge every update into the column's own sorted row list
  // (a row that is not found is a structure error), narrow levels use the
  // dense accumulator
  const int nlev = (int)p.lvl_ptr.size() - 1;
  if (nlev < 1 || p.lvl_ptr[nlev] != N) return -24;
  {
    std::vector<int> seen(N, 0), lvl(N, -1);
    for (int l = 0; l < nlev; ++l)
      for (int t = p.lvl_ptr[l]; t < p.lvl_ptr[l + 1]; ++t) {
        int j = p.lvl_nodes[t];
        if (j < 0 || j >= N || seen[j]) return -25;
        seen[j] = 1;
        lvl[j] = l;
      }
    for (int j = 0; j < N; ++j)
      for (int r = p.Rp[j]; r < p.Rp[j + 1]; ++r)
        if (lvl[p.Rk[r]] >= lvl[j]) return -26;  // dependency must be on a lower level
  }
  std::vector<double> w(N, 0.0), Lx(lnz, 0.0), D(N, 0.0);
  const int narrow_below = 16;  // NT/2 for the single-warp kernel
  for (int l = 0; l < nlev; ++l) {
    const int a = p.lvl_ptr[l], bnd = p.lvl_ptr[l + 1];
    for (int t = a; t < bnd; ++t) {
      const int j = p.lvl_nodes[t];
      const int q0 = p.Lp[j], q1 = p.Lp[j + 1];
      if (bnd - a >= narrow_below) {
        for (int q = q0; q < q1; ++q) Lx[q] = 0.0;
        double dj = 0;
        int q = q0;
        for (int pp = p.Kp[j]; pp < p.Kp[j + 1]; ++pp) {
          int c = p.Kj[pp];
          if (c < j) continue;
          if (c == j) {
            dj = Kx[pp];
            continue;
          }
          while (q < q1 && p.Li[q] != c) ++q;
          if (q >= q1) return -27;
          Lx[q] = Kx[pp];
        }
        for (int r = p.Rp[j]; r < p.Rp[j + 1]; ++r) {
          int k = p.Rk[r], pos = p.Rpos[r];
          double f = Lx[pos] * D[k];
          dj -= Lx[pos] * f;
          q = q0;
          for (int tt = pos + 1; tt < p.Lp[k + 1]; ++tt) {
            while (q < q1 && p.Li[q] != p.Li[tt]) ++q;
            if (q >= q1) return -28;
            Lx[q] -= Lx[tt] * f;
          }
        }
        D[j] = dj;
        for (int qq = q0; qq < q1; ++qq) Lx[qq] /= dj;
      } else {
        for (int pp = p.Kp[j]; pp < p.Kp[j + 1]; ++pp)
          if (p.Kj[pp] >= j) w[p.Kj[pp]] = Kx[pp];
        for (int r = p.Rp[j]; r < p.Rp[j + 1]; ++r) {
          int k = p.Rk[r], pos = p.Rpos[r];
          double f = Lx[pos] * D[k];
          w[j] -= Lx[pos] * f;
          for (int tt = pos + 1; tt < p.Lp[k + 1]; ++tt) w[p.Li[tt]] -= Lx[tt] * f;
        }
        D[j] = w[j];
        for (int qq = q0; qq < q1; ++qq) {
          Lx[qq] = w[p.Li[qq]] / D[j];
          w[p.Li[qq]] = 0;
        }
        w[j] = 0;
      }
    }
  }
  std::vector<double> b(N), y(N);
  for (int i = 0; i < N; ++i) b[i] = std::cos(0.3 * i);
  y = b;
  for (int l = 0; l < nlev; ++l)
    for (int t = p.lvl_ptr[l]; t < p.lvl_ptr[l + 1]; ++t) {
      int i = p.lvl_nodes[t];
      for (int r = p.Rp[i]; r < p.Rp[i + 1]; ++r) y[i] -= Lx[p.Rpos[r]] * y[p.Rk[r]];
    }
  for (int j = 0; j < N; ++j) y[j] /= D[j];
  for (int l = nlev - 1; l >= 0; --l)
    for (int t = p.lvl_ptr[l]; t < p.lvl_ptr[l + 1]; ++t) {
      int j = p.lvl_nodes[t];
      for (int tt = p.Lp[j]; tt < p.Lp[j + 1]; ++tt) y[j] -= Lx[tt] * y[p.Li[tt]];
    }
  double mx = 0;
  for (int r = 0; r < N; ++r) {
    double t = 0;
    for (int q = p.Kp[r]; q < p.Kp[r + 1]; ++q) t += Kx[q] * y[p.Kj[q]];
    mx = std::max(mx, std::fabs(t - b[r]));
  }
  if (resid) *resid = mx;
  return 0;
}
