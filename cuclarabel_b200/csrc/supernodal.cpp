// supernodal.cpp -- host-side analysis of the supernodal LDL^T.
//
// The analysis cuDSS performs once per sparsity pattern in the reference
// (src/kktsolvers/gpu/directldl_cudss.jl:20-23): ordering, elimination
// tree, supernode detection and symbolic factorisation.  Each step is a
// textbook algorithm, written for this project:
//   ordering         approximate minimum degree (amd.cpp)
//   elimination tree Liu's algorithm with path compression
//   postorder        depth-first, children in increasing order
//   column counts    row-subtree traversal (each row of L marks the path
//                    from its entries up the tree), O(nnz(L)) time, O(N)
//                    memory
//   supernodes       fundamental supernodes (a chain j -> j+1 where j+1 has
//                    one child and one entry fewer), then relaxed
//                    amalgamation: a supernode absorbs its last child when
//                    the merged front adds few explicit zeros
//   row structure    bottom-up union of the original entries and the
//                    children's structures
#include "supernodal.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>

#include "setup.hpp"

namespace clgpu {

namespace {

// relaxed amalgamation: merge when the merged supernode has at most 16
// columns, or when the explicit zeros stay below the fraction allowed for
// its width
bool relax_ok(long long ncol, double zeros, double total) {
  if (ncol <= 16) return true;
  const double frac = total > 0 ? zeros / total : 0.0;
  if (ncol <= 48) return frac < 0.30;
  if (ncol <= 128) return frac < 0.10;
  return frac < 0.03;
}

}  // namespace

bool sn_analyse(int N, const std::vector<int> &xadj, const std::vector<int> &adj,
                std::vector<int> &perm, SnSymbolic &sym, std::string *err) {
  sym = SnSymbolic();
  sym.N = N;
  perm = amd_order_qg(N, xadj, adj);
  std::vector<int> ip(N);
  for (int k = 0; k < N; ++k) ip[perm[k]] = k;
  // lower pattern of the permuted matrix by rows: for row k, columns j < k
  auto build_rows = [&](const std::vector<int> &iperm, std::vector<int> &rp, std::vector<int> &rc) {
    rp.assign(N + 1, 0);
    for (int v = 0; v < N; ++v)
      for (int q = xadj[v]; q < xadj[v + 1]; ++q) {
        const int a = iperm[v], b = iperm[adj[q]];
        if (b < a) rp[a + 1]++;
      }
    for (int k = 0; k < N; ++k) rp[k + 1] += rp[k];
    rc.assign(rp[N], 0);
    std::vector<int> cur(rp.begin(), rp.end() - 1);
    for (int v = 0; v < N; ++v)
      for (int q = xadj[v]; q < xadj[v + 1]; ++q) {
        const int a = iperm[v], b = iperm[adj[q]];
        if (b < a) rc[cur[a]++] = b;
      }
    for (int k = 0; k < N; ++k) {
      std::sort(rc.begin() + rp[k], rc.begin() + rp[k + 1]);
      auto e = std::unique(rc.begin() + rp[k], rc.begin() + rp[k + 1]);
      // keep the pointer layout: pad duplicates with the last valid value
      for (auto it = e; it != rc.begin() + rp[k + 1]; ++it) *it = -1;
    }
  };
  std::vector<int> rp, rc;
  build_rows(ip, rp, rc);
  // elimination tree
  std::vector<int> parent(N, -1), anc(N, -1);
  for (int k = 0; k < N; ++k)
    for (int q = rp[k]; q < rp[k + 1]; ++q) {
      int i = rc[q];
      while (i != -1 && i < k) {
        const int nx = anc[i];
        anc[i] = k;
        if (nx == -1) parent[i] = k;
        i = nx;
      }
    }
  // postorder (children in increasing order)
  std::vector<int> head(N, -1), next(N, -1);
  for (int j = N - 1; j >= 0; --j)
    if (parent[j] >= 0) {
      next[j] = head[parent[j]];
      head[parent[j]] = j;
    }
  std::vector<int> post;
  post.reserve(N);
  {
    std::vector<int> stack;
    for (int r = 0; r < N; ++r) {
      if (parent[r] != -1) continue;
      stack.push_back(r);
      while (!stack.empty()) {
        const int v = stack.back();
        if (head[v] >= 0) {
          const int c = head[v];
          head[v] = next[c];
          stack.push_back(c);
        } else {
          stack.pop_back();
          post.push_back(v);
        }
      }
    }
  }
  if ((int)post.size() != N) {
    if (err) *err = "internal: elimination tree postorder";
    return false;
  }
  // relabel: new index of old permuted column post[t] is t
  {
    std::vector<int> perm2(N);
    for (int t = 0; t < N; ++t) perm2[t] = perm[post[t]];
    perm.swap(perm2);
    for (int k = 0; k < N; ++k) ip[perm[k]] = k;
    std::vector<int> inv(N);
    for (int t = 0; t < N; ++t) inv[post[t]] = t;
    std::vector<int> par2(N, -1);
    for (int j = 0; j < N; ++j) par2[inv[j]] = parent[j] >= 0 ? inv[parent[j]] : -1;
    parent.swap(par2);
  }
  build_rows(ip, rp, rc);
  // column counts (entries below the diagonal) by row subtrees
  std::vector<long long> cnt(N, 0);
  {
    std::vector<int> mark(N, -1);
    for (int k = 0; k < N; ++k) {
      mark[k] = k;
      for (int q = rp[k]; q < rp[k + 1]; ++q) {
        int i = rc[q];
        if (i < 0) continue;
        while (mark[i] != k) {
          cnt[i]++;
          mark[i] = k;
          i = parent[i];
        }
      }
    }
  }
  // fundamental supernodes
  std::vector<int> nchild(N, 0);
  for (int j = 0; j < N; ++j)
    if (parent[j] >= 0) nchild[parent[j]]++;
  std::vector<int> fstart;
  for (int j = 0; j < N; ++j) {
    const bool cont = j > 0 && parent[j - 1] == j && nchild[j] == 1 && cnt[j] == cnt[j - 1] - 1;
    if (!cont) fstart.push_back(j);
  }
  const int nf = (int)fstart.size();
  fstart.push_back(N);
  std::vector<int> fof(N);
  for (int s = 0; s < nf; ++s)
    for (int j = fstart[s]; j < fstart[s + 1]; ++j) fof[j] = s;
  // relaxed amalgamation over the supernodal tree (postorder: children first)
  std::vector<int> fpar(nf, -1);
  for (int s = 0; s < nf; ++s) {
    const int last = fstart[s + 1] - 1;
    fpar[s] = parent[last] >= 0 ? fof[parent[last]] : -1;
  }
  std::vector<long long> ncol(nf), nrow(nf);
  std::vector<double> real(nf);
  for (int s = 0; s < nf; ++s) {
    ncol[s] = fstart[s + 1] - fstart[s];
    nrow[s] = cnt[fstart[s + 1] - 1];
    real[s] = 0;
    for (int j = fstart[s]; j < fstart[s + 1]; ++j) real[s] += (double)cnt[j];
  }
  std::vector<int> start(fstart.begin(), fstart.end() - 1), into(nf, -1);
  auto find = [&](int s) {
    while (into[s] >= 0) s = into[s];
    return s;
  };
  for (int s = 0; s < nf; ++s) {
    if (into[s] >= 0 || fpar[s] < 0) continue;
    const int p = find(fpar[s]);
    if (start[s] + ncol[s] != start[p]) continue;  // not the last child
    const long long nc = ncol[s] + ncol[p];
    const double total = (double)nc * (nc - 1) / 2.0 + (double)nc * nrow[p];
    const double rl = real[s] + real[p];
    if (!relax_ok(nc, total - rl, total)) continue;
    into[s] = p;
    start[p] = start[s];
    ncol[p] = nc;
    real[p] = rl;
  }
  // surviving supernodes in column order
  std::vector<int> keep;
  for (int s = 0; s < nf; ++s)
    if (into[s] < 0) keep.push_back(s);
  std::sort(keep.begin(), keep.end(), [&](int a, int b) { return start[a] < start[b]; });
  const int ns = (int)keep.size();
  std::vector<int> newid(nf, -1);
  for (int t = 0; t < ns; ++t) newid[keep[t]] = t;
  sym.col0.assign(ns + 1, N);
  sym.parent.assign(ns, -1);
  for (int t = 0; t < ns; ++t) {
    const int s = keep[t];
    sym.col0[t] = start[s];
    sym.parent[t] = fpar[s] >= 0 ? newid[find(fpar[s])] : -1;
  }
  // row structures, bottom-up (supernodes are numbered in postorder)
  std::vector<std::vector<int>> kids(ns);
  for (int t = 0; t < ns; ++t)
    if (sym.parent[t] >= 0) {
      if (sym.parent[t] <= t) {
        if (err) *err = "internal: supernode order";
        return false;
      }
      kids[sym.parent[t]].push_back(t);
    }
  std::vector<int> mark(N, -1);
  std::vector<std::vector<int>> st(ns);
  double nnz = 0, flops = 0;
  long long tot = 0;
  for (int t = 0; t < ns; ++t) {
    const int c0 = sym.col0[t], c1 = sym.col0[t + 1];
    std::vector<int> &R = st[t];
    auto add = [&](int r) {
      if (r >= c1 && mark[r] != t) {
        mark[r] = t;
        R.push_back(r);
      }
    };
    // original entries of the pivot columns (the graph is symmetric), then
    // the children's structures
    for (int j = c0; j < c1; ++j) {
      const int v = perm[j];
      for (int q = xadj[v]; q < xadj[v + 1]; ++q) add(ip[adj[q]]);
    }
    for (int c : kids[t])
      for (int r : st[c]) add(r);
    std::sort(R.begin(), R.end());
    const double nc = c1 - c0, nr = (double)R.size();
    nnz += nc * (nc - 1) / 2 + nc * nr;
    for (int j = 0; j < (int)nc; ++j) {
      const double below = (nc - 1 - j) + nr;
      flops += below * below;
    }
    tot += (long long)R.size();
  }
  if (tot > 2000000000LL) {
    if (err) *err = "factor too large";
    return false;
  }
  sym.rptr.assign(ns + 1, 0);
  sym.rows.reserve(tot);
  for (int t = 0; t < ns; ++t) {
    sym.rows.insert(sym.rows.end(), st[t].begin(), st[t].end());
    sym.rptr[t + 1] = (int)sym.rows.size();
  }
  sym.nnz_l = nnz;
  sym.flops = flops;
  return true;
}


// ------------------------------------------------------------ device plan
namespace {

inline long long align32(long long v) { return (v + 31) & ~31LL; }
inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

// panels of a blocked front: [k, k + K) for each, the first one taking
// u0 mod kSnNB columns when that is nonzero
void panels_of(int u0, std::vector<std::pair<int, int>> &out) {
  out.clear();
  int k = 0;
  const int first = u0 % kSnNB;
  if (first) {
    out.push_back({0, first});
    k = first;
  }
  for (; k < u0; k += kSnNB) out.push_back({k, kSnNB});
}

}  // namespace

bool sn_build_plan(const std::vector<SnInstance> &in, SnPlan &P, std::string *err) {
  P = SnPlan();
  auto fail = [&](const char *m) {
    if (err) *err = m;
    return false;
  };
  int ns = 0;
  for (auto &x : in) ns += x.sym->ns();
  P.ns = ns;
  P.inst.resize(ns);
  P.col0g.resize(ns);
  P.ncol.resize(ns);
  P.nrow.resize(ns);
  P.u0.resize(ns);
  P.ld.resize(ns);
  P.large.resize(ns);
  P.cbase.resize(ns + 1);
  P.fix_off.resize(ns + 1);
  P.rel_off.resize(ns + 1);
  P.ch_ptr.assign(ns + 1, 0);
  P.uoff.resize(ns + 1);
  P.foff.resize(ns + 1);
  P.woff.assign(ns + 1, 0);
  P.soff.assign(ns + 1, 0);
  std::vector<int> level(ns, 0), gpar(ns, -1);
  long long fo = 0, wo = 0, so = 0, uo = 0, fx = 0, ro = 0;
  int cb = 0, sbase = 0;
  for (auto &x : in) {
    const SnSymbolic &S = *x.sym;
    for (int t = 0; t < S.ns(); ++t) {
      const int s = sbase + t;
      const int nc = S.col0[t + 1] - S.col0[t], nr = S.rptr[t + 1] - S.rptr[t];
      P.inst[s] = x.inst;
      P.col0g[s] = x.vbase + S.col0[t];
      P.ncol[s] = nc;
      P.nrow[s] = nr;
      const bool lg = nc + nr > kSnSmallMax;
      P.large[s] = lg ? 1 : 0;
      P.u0[s] = lg ? round_up(nc, kSnKPad) : nc;
      P.ld[s] = lg ? P.u0[s] + round_up(nr, kSnNB) : nc + nr;
      if ((long long)P.ld[s] * P.ld[s] >= (1LL << 31)) return fail("front too large");
      P.cbase[s] = cb;
      cb += nc;
      P.fix_off[s] = (int)fx;
      fx += P.ld[s];
      P.rel_off[s] = (int)ro;
      ro += nr;
      P.uoff[s] = (int)uo;
      uo += nr;
      P.foff[s] = fo;
      fo += align32((long long)P.ld[s] * P.ld[s]);
      if (lg) {
        P.woff[s] = wo;
        wo += align32(kSnNB + (long long)P.ld[s] * kSnNB);
        P.soff[s] = so;
        so += align32(2LL * P.ld[s]);
      }
      gpar[s] = S.parent[t] >= 0 ? sbase + S.parent[t] : -1;
    }
    sbase += S.ns();
  }
  if (fx > 2000000000LL || ro > 2000000000LL || uo > 2000000000LL) return fail("plan too large");
  P.cbase[ns] = cb;
  P.fix_off[ns] = (int)fx;
  P.rel_off[ns] = (int)ro;
  P.uoff[ns] = (int)uo;
  P.foff[ns] = fo;
  P.woff[ns] = wo;
  P.soff[ns] = so;
  P.f_elems = fo;
  P.w_elems = wo;
  P.s_elems = so;
  P.u_elems = uo;
  // children lists (postorder: children have smaller numbers than parents)
  for (int s = 0; s < ns; ++s)
    if (gpar[s] >= 0) P.ch_ptr[gpar[s] + 1]++;
  for (int s = 0; s < ns; ++s) P.ch_ptr[s + 1] += P.ch_ptr[s];
  P.ch.assign(P.ch_ptr[ns], 0);
  {
    std::vector<int> cur(P.ch_ptr.begin(), P.ch_ptr.end() - 1);
    for (int s = 0; s < ns; ++s)
      if (gpar[s] >= 0) P.ch[cur[gpar[s]]++] = s;
  }
  for (int s = 0; s < ns; ++s)
    if (gpar[s] >= 0) level[gpar[s]] = std::max(level[gpar[s]], level[s] + 1);
  // front index lists, relative indices, assembly maps
  P.fidx.assign(fx, -1);
  P.rel.assign(ro, 0);
  P.acol.assign(cb + 1, 0);
  sbase = 0;
  for (auto &x : in) {
    const SnSymbolic &S = *x.sym;
    for (int t = 0; t < S.ns(); ++t) {
      const int s = sbase + t, c0 = S.col0[t];
      int *fi = P.fidx.data() + P.fix_off[s];
      for (int c = 0; c < P.ncol[s]; ++c) fi[c] = x.vbase + c0 + c;
      for (int k = 0; k < P.nrow[s]; ++k) fi[P.u0[s] + k] = x.vbase + S.rows[S.rptr[t] + k];
      // relative indices into the parent's front
      const int pt = S.parent[t];
      if (pt >= 0) {
        const int p = sbase + pt;
        const int pc0 = S.col0[pt], pc1 = S.col0[pt + 1];
        const int *pr = S.rows.data() + S.rptr[pt], *pre = S.rows.data() + S.rptr[pt + 1];
        for (int k = 0; k < P.nrow[s]; ++k) {
          const int r = S.rows[S.rptr[t] + k];
          int pos;
          if (r >= pc0 && r < pc1) {
            pos = r - pc0;
          } else {
            const int *it = std::lower_bound(pr, pre, r);
            if (it == pre || *it != r) return fail("internal: child row outside the parent's front");
            pos = P.u0[p] + (int)(it - pr);
          }
          P.rel[P.rel_off[s] + k] = pos;
        }
      } else if (P.nrow[s] != 0) {
        return fail("internal: root with a row structure");
      }
      // original entries of the pivot columns: row j's entries at columns >= j
      const int *rb = S.rows.data() + S.rptr[t], *re = S.rows.data() + S.rptr[t + 1];
      for (int c = 0; c < P.ncol[s]; ++c) {
        const int j = c0 + c;
        for (int q = x.Kp[j]; q < x.Kp[j + 1]; ++q) {
          const int i = x.Kj[q];
          if (i < j) continue;
          int rp;
          if (i < c0 + P.ncol[s]) {
            rp = i - c0;
          } else {
            const int *it = std::lower_bound(rb, re, i);
            if (it == re || *it != i) return fail("internal: entry outside the front");
            rp = P.u0[s] + (int)(it - rb);
          }
          const long long kp = x.kbase + q;
          if (kp > 2000000000LL) return fail("KKT too large");
          P.amap.push_back({(int)kp, c * P.ld[s] + rp});
        }
        P.acol[P.cbase[s] + c + 1] = (int)P.amap.size();
      }
    }
    sbase += S.ns();
  }
  // ---- children per chunk of the blocked fronts (assembly, forward gather)
  P.chunk_off.assign(ns + 1, 0);
  for (int s = 0; s < ns; ++s)
    P.chunk_off[s + 1] = P.chunk_off[s] + (P.large[s] ? (P.ld[s] + kSnAsmCols - 1) / kSnAsmCols : 0);
  {
    std::vector<std::vector<SnQuad>> lists(P.chunk_off[ns]);
    for (int s = 0; s < ns; ++s) {
      if (!P.large[s]) continue;
      for (int a = P.ch_ptr[s]; a < P.ch_ptr[s + 1]; ++a) {
        const int c = P.ch[a], cn = P.nrow[c];
        const int *rel = P.rel.data() + P.rel_off[c];
        for (int q = 0; q < cn;) {
          const int chunk = rel[q] / kSnAsmCols;
          int qe = q + 1;
          while (qe < cn && rel[qe] / kSnAsmCols == chunk) ++qe;
          lists[P.chunk_off[s] + chunk].push_back({c, q, qe, 0});
          q = qe;
        }
      }
    }
    P.cl_ptr.assign(P.chunk_off[ns] + 1, 0);
    for (size_t g = 0; g < lists.size(); ++g) P.cl_ptr[g + 1] = P.cl_ptr[g] + (int)lists[g].size();
    P.clist.reserve(P.cl_ptr.back());
    for (auto &l : lists) P.clist.insert(P.clist.end(), l.begin(), l.end());
  }
  // ---- schedules, level by level
  int H = 0;
  for (int s = 0; s < ns; ++s) H = std::max(H, level[s] + 1);
  std::vector<std::vector<int>> small(H), big(H);
  for (int s = 0; s < ns; ++s) (P.large[s] ? big : small)[level[s]].push_back(s);
  auto launch = [&](std::vector<SnLaunch> &sched, int kind, int begin, int smem = 0,
                    double fl = 0.0) {
    const int count = (int)P.tasks.size() - begin;
    if (count > 0) sched.push_back({kind, begin, count, smem, fl});
  };
  auto kK = [](int k, int K) { return k | (K << 16); };
  std::vector<std::pair<int, int>> pan;
  double flops = 0;
  for (int L = 0; L < H; ++L) {
    // factorisation
    int b0 = (int)P.tasks.size(), smem = 0;
    double fl = 0;
    for (int s : small[L]) {
      P.tasks.push_back({s, 0, 0, 0});
      smem = std::max(smem, P.ld[s] * P.ld[s]);
      for (int c = 0; c < P.ncol[s]; ++c) {
        const double below = P.ld[s] - 1 - c;
        fl += below * below;
      }
    }
    flops += fl;
    P.small_smem_max = std::max(P.small_smem_max, smem);
    launch(P.fact, SN_SMALL_FACTOR, b0, smem, fl);
    if (big[L].empty()) continue;
    b0 = (int)P.tasks.size();
    for (int s : big[L])
      for (int c = 0; c < P.ld[s]; c += kSnAsmCols)
        P.tasks.push_back({s, c, std::min(P.ld[s], c + kSnAsmCols),
                           P.chunk_off[s] + c / kSnAsmCols});
    launch(P.fact, SN_ASSEMBLE, b0);
    std::vector<std::vector<std::pair<int, int>>> pl(big[L].size());
    size_t maxp = 0;
    for (size_t a = 0; a < big[L].size(); ++a) {
      panels_of(P.u0[big[L][a]], pl[a]);
      maxp = std::max(maxp, pl[a].size());
    }
    for (size_t p = 0; p < maxp; ++p) {
      // flops: 2 K^3 / 3 per diagonal block; K^2 per TRSM row; 2 K per
      // lower-triangle entry of the update
      b0 = (int)P.tasks.size();
      fl = 0;
      for (size_t a = 0; a < big[L].size(); ++a)
        if (p < pl[a].size()) {
          const int K = pl[a][p].second;
          P.tasks.push_back({big[L][a], kK(pl[a][p].first, K), 0, 0});
          fl += 2.0 * K * K * K / 3.0;
        }
      flops += fl;
      launch(P.fact, SN_DIAG, b0, 0, fl);
      b0 = (int)P.tasks.size();
      fl = 0;
      for (size_t a = 0; a < big[L].size(); ++a) {
        if (p >= pl[a].size()) continue;
        const int s = big[L][a], k = pl[a][p].first, K = pl[a][p].second, e = k + K;
        for (int r0 = e; r0 < P.ld[s]; r0 += kSnNB) {
          P.tasks.push_back({s, kK(k, K), r0, 0});
          fl += 1.0 * K * K * kSnNB;
        }
      }
      flops += fl;
      launch(P.fact, SN_TRSM, b0, 0, fl);
      b0 = (int)P.tasks.size();
      fl = 0;
      for (size_t a = 0; a < big[L].size(); ++a) {
        if (p >= pl[a].size()) continue;
        const int s = big[L][a], k = pl[a][p].first, K = pl[a][p].second, e = k + K;
        // 128 x 64 tiles: for every 64-column block, the 128-row tiles from
        // the one holding its diagonal down
        for (int c0 = e; c0 < P.ld[s]; c0 += 64)
          for (int r0 = e + (c0 - e) / kSnNB * kSnNB; r0 < P.ld[s]; r0 += kSnNB) {
            P.tasks.push_back({s, kK(k, K), r0, c0});
            double below = 0;  // entries on or below the diagonal
            for (int n = 0; n < 64; ++n) below += std::max(0, std::min(kSnNB, r0 + kSnNB - c0 - n));
            fl += 2.0 * below * K;
          }
      }
      flops += fl;
      launch(P.fact, SN_UPDATE, b0, 0, fl);
    }
  }
  P.flops = flops;
  // forward substitution, leaves first
  for (int L = 0; L < H; ++L) {
    int b0 = (int)P.tasks.size();
    for (int s : small[L]) P.tasks.push_back({s, 0, 0, 0});
    launch(P.fwd, SN_FWD_SMALL, b0);
    if (big[L].empty()) continue;
    b0 = (int)P.tasks.size();
    for (int s : big[L])
      for (int c = 0; c < P.ld[s]; c += kSnAsmCols)
        P.tasks.push_back({s, c, std::min(P.ld[s], c + kSnAsmCols),
                           P.chunk_off[s] + c / kSnAsmCols});
    launch(P.fwd, SN_FWD_GATHER, b0);
    std::vector<std::vector<std::pair<int, int>>> pl(big[L].size());
    size_t maxp = 0;
    for (size_t a = 0; a < big[L].size(); ++a) {
      panels_of(P.u0[big[L][a]], pl[a]);
      maxp = std::max(maxp, pl[a].size());
    }
    for (size_t p = 0; p < maxp; ++p) {
      b0 = (int)P.tasks.size();
      for (size_t a = 0; a < big[L].size(); ++a)
        if (p < pl[a].size()) P.tasks.push_back({big[L][a], kK(pl[a][p].first, pl[a][p].second), 0, 0});
      launch(P.fwd, SN_FWD_DIAG, b0);
      b0 = (int)P.tasks.size();
      for (size_t a = 0; a < big[L].size(); ++a) {
        if (p >= pl[a].size()) continue;
        const int s = big[L][a], k = pl[a][p].first, K = pl[a][p].second;
        for (int r0 = k + K; r0 < P.ld[s]; r0 += kSnNB) P.tasks.push_back({s, kK(k, K), r0, 0});
      }
      launch(P.fwd, SN_FWD_GEMV, b0);
    }
    b0 = (int)P.tasks.size();
    for (int s : big[L]) P.tasks.push_back({s, 0, 0, 0});
    launch(P.fwd, SN_FWD_SCATTER, b0);
  }
  // backward substitution, roots first
  for (int L = H - 1; L >= 0; --L) {
    int b0;
    if (!big[L].empty()) {
      b0 = (int)P.tasks.size();
      for (int s : big[L]) P.tasks.push_back({s, 0, 0, 0});
      launch(P.bwd, SN_BWD_GATHER, b0);
      std::vector<std::vector<std::pair<int, int>>> pl(big[L].size());
      size_t maxp = 0;
      for (size_t a = 0; a < big[L].size(); ++a) {
        panels_of(P.u0[big[L][a]], pl[a]);
        maxp = std::max(maxp, pl[a].size());
      }
      for (size_t pp = 0; pp < maxp; ++pp) {
        b0 = (int)P.tasks.size();
        for (size_t a = 0; a < big[L].size(); ++a) {
          if (pp >= pl[a].size()) continue;
          const size_t p = pl[a].size() - 1 - pp;
          const int s = big[L][a], k = pl[a][p].first, K = pl[a][p].second;
          for (int r0 = k + K; r0 < P.ld[s]; r0 += kSnNB) P.tasks.push_back({s, kK(k, K), r0, 0});
        }
        launch(P.bwd, SN_BWD_PARTIAL, b0);
        b0 = (int)P.tasks.size();
        for (size_t a = 0; a < big[L].size(); ++a) {
          if (pp >= pl[a].size()) continue;
          const size_t p = pl[a].size() - 1 - pp;
          P.tasks.push_back({big[L][a], kK(pl[a][p].first, pl[a][p].second), 0, 0});
        }
        launch(P.bwd, SN_BWD_DIAG, b0);
      }
      b0 = (int)P.tasks.size();
      for (int s : big[L]) P.tasks.push_back({s, 0, 0, 0});
      launch(P.bwd, SN_BWD_SCATTER, b0);
    }
    b0 = (int)P.tasks.size();
    for (int s : small[L]) P.tasks.push_back({s, 0, 0, 0});
    launch(P.bwd, SN_BWD_SMALL, b0);
  }
  if (P.tasks.size() > 2000000000ULL) return fail("schedule too large");
  for (auto &x : in) P.insts.push_back(x.inst);
  return true;
}

// ------------------------------------------------------------ host replay
double sn_host_check(const SnPlan &P, const std::vector<int> &Kp, const std::vector<int> &Kj,
                     const std::vector<double> &Kx, const std::vector<signed char> &Dsign,
                     const std::vector<int> &voff, double eps) {
  const int ns = P.ns;
  std::vector<double> F(P.f_elems, 0.0), Dv(voff.back(), 0.0), U(P.u_elems, 0.0);
  // factorisation, supernodes in postorder (children first)
  for (int s = 0; s < ns; ++s) {
    const int ld = P.ld[s], u0 = P.u0[s], nc = P.ncol[s];
    double *f = F.data() + P.foff[s];
    std::fill(f, f + (long long)ld * ld, 0.0);
    for (int c = 0; c < nc; ++c)
      for (int q = P.acol[P.cbase[s] + c]; q < P.acol[P.cbase[s] + c + 1]; ++q)
        f[P.amap[q].y] += Kx[P.amap[q].x];
    for (int c = 0; c < nc; ++c) f[(long long)c * ld + c] += Dsign[P.col0g[s] + c] > 0 ? eps : -eps;
    for (int c = nc; c < u0; ++c) f[(long long)c * ld + c] = 1.0;
    for (int a = P.ch_ptr[s]; a < P.ch_ptr[s + 1]; ++a) {
      const int cs = P.ch[a];
      const int cld = P.ld[cs], cu = P.u0[cs], cn = P.nrow[cs];
      const double *cf = F.data() + P.foff[cs];
      const int *rel = P.rel.data() + P.rel_off[cs];
      for (int q = 0; q < cn; ++q)
        for (int r = q; r < cn; ++r)
          f[(long long)rel[q] * ld + rel[r]] += cf[(long long)(cu + q) * cld + cu + r];
    }
    for (int j = 0; j < u0; ++j) {
      const double d = f[(long long)j * ld + j];
      for (int i = j + 1; i < ld; ++i) {
        const double a = f[(long long)j * ld + i];
        if (a == 0.0) continue;
        const double l = a / d;
        for (int r = i; r < ld; ++r) f[(long long)i * ld + r] -= l * f[(long long)j * ld + r];
      }
      for (int i = j + 1; i < ld; ++i) f[(long long)j * ld + i] /= d;
      if (j < nc) Dv[P.col0g[s] + j] = d;
    }
  }
  // test right-hand side and solve
  const int NT = voff.back();
  std::vector<double> b(NT), y(NT);
  for (int i = 0; i < NT; ++i) b[i] = std::cos(0.3 * i);
  y = b;
  std::vector<double> v;
  for (int s = 0; s < ns; ++s) {
    const int ld = P.ld[s], u0 = P.u0[s], nc = P.ncol[s], nr = P.nrow[s];
    const double *f = F.data() + P.foff[s];
    v.assign(ld, 0.0);
    for (int c = 0; c < nc; ++c) v[c] = y[P.col0g[s] + c];
    for (int a = P.ch_ptr[s]; a < P.ch_ptr[s + 1]; ++a) {
      const int cs = P.ch[a];
      const int *rel = P.rel.data() + P.rel_off[cs];
      for (int k = 0; k < P.nrow[cs]; ++k) v[rel[k]] += U[P.uoff[cs] + k];
    }
    for (int j = 0; j < u0; ++j)
      for (int i = j + 1; i < ld; ++i) v[i] -= f[(long long)j * ld + i] * v[j];
    for (int c = 0; c < nc; ++c) y[P.col0g[s] + c] = v[c];
    for (int k = 0; k < nr; ++k) U[P.uoff[s] + k] = v[u0 + k];
  }
  for (int s = 0; s < ns; ++s)
    for (int c = 0; c < P.ncol[s]; ++c) y[P.col0g[s] + c] /= Dv[P.col0g[s] + c];
  for (int s = ns - 1; s >= 0; --s) {
    const int ld = P.ld[s], u0 = P.u0[s], nc = P.ncol[s], nr = P.nrow[s];
    const double *f = F.data() + P.foff[s];
    const int *fi = P.fidx.data() + P.fix_off[s];
    v.assign(ld, 0.0);
    for (int c = 0; c < nc; ++c) v[c] = y[P.col0g[s] + c];
    for (int k = 0; k < nr; ++k) v[u0 + k] = y[fi[u0 + k]];
    for (int j = u0 - 1; j >= 0; --j) {
      double t = v[j];
      for (int i = j + 1; i < ld; ++i) t -= f[(long long)j * ld + i] * v[i];
      v[j] = t;
    }
    for (int c = 0; c < nc; ++c) y[P.col0g[s] + c] = v[c];
  }
  // residual against the shifted matrix, over the plan's instances
  double mx = 0, nb = 0;
  // (Kp holds N + 1 pointers per instance, Kj local column indices)
  for (int inst : P.insts) {
    const int vb = voff[inst], n = voff[inst + 1] - vb;
    const int *kp = Kp.data() + vb + inst;
    for (int r = 0; r < n; ++r) {
      double t = 0;
      for (int q = kp[r]; q < kp[r + 1]; ++q) {
        const int c = Kj[q];
        t += Kx[q] * y[vb + c] + (c == r ? (Dsign[vb + r] > 0 ? eps : -eps) * y[vb + c] : 0.0);
      }
      mx = std::max(mx, std::fabs(t - b[vb + r]));
      nb = std::max(nb, std::fabs(b[vb + r]));
    }
  }
  return nb > 0 ? mx / nb : mx;
}
}  // namespace clgpu
