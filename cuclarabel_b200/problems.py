"""Seeded synthetic problem generators for the benchmark configurations.

All draws use numpy's PCG64 generator.  The reference's README example uses
Julia's MersenneTwister, which cannot be reproduced here, so the problems have
the reference's shapes and value distributions, not its exact draws.

Problems are returned as (P, q, A, b, cones) with P upper triangular CSC,
A CSC and cones as a list of cone objects (cuclarabel_b200.api).

  portfolio(seed=1)         factor-model portfolio QP, 50 assets, 5 factors
  mixed_socp(scale, seed)   large mixed-cone QP/SOCP (n=20000, m=60000 at
                            scale 1): 2000 zero, 28000 nonneg, 3000 SOC(10)
  exp_pow_psd(scale, seed)  conic LP with exp/pow/PSD cones (n=30000 at
                            scale 1): 20000 exp, 5000 pow, 200 PSD(10),
                            10000 nonneg
  psd_lp(side, ncones, ...) linear SDP over PSD blocks of one side
  mpc_qp(seed)              one MPC-style QP/SOCP, n ~ U{20..400}, m ~ 2n
  mpc_batch(count, seed0)   `count` MPC-style instances, instance i seeded i

The mixed/exp/MPC families are feasible and bounded by construction: draw
x0, a strictly interior slack s0 and dual z0, then set b = A x0 + s0 and
q = -P x0 - A' z0.
"""
import numpy as np
import scipy.sparse as sp

from .api import (ExponentialConeT, NonnegativeConeT, PowerConeT, PSDTriangleConeT,
                  SecondOrderConeT, ZeroConeT)

EXP_UNIT = np.array([-1.051383945322714, 0.556409619469370, 1.258967884768947])


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def _finish(P, A, x0, s0, z0, cones):
    P = sp.csc_matrix(P)
    A = sp.csc_matrix(A)
    b = A @ x0 + s0
    q = -(P @ x0) - A.T @ z0
    return sp.triu(P, format="csc"), np.asarray(q).ravel(), A, np.asarray(b).ravel(), cones


def portfolio(seed=1, n_assets=50, k=5):
    """Factor-model portfolio QP (README.md:60-96 of the reference)."""
    r = _rng(seed)
    n = n_assets
    D = r.uniform(0, 1, n) * np.sqrt(k)
    F = sp.random(n, k, density=0.5, random_state=r, data_rvs=r.standard_normal, format="csc")
    mu = (3 + 9 * r.uniform(0, 1, n)) / 100.0
    gamma, a, d = 1.0, 1e-3, 1.0
    x0 = np.zeros(n)
    # variables: x (n), y (k), s (n), t (n)
    nv = 3 * n + k
    ix, iy, is_, it = 0, n, n + k, 2 * n + k
    P = sp.diags(np.concatenate([2 * D, 2 * np.ones(k), np.zeros(2 * n)]), format="csc")
    q = np.concatenate([-mu / gamma, np.zeros(k + 2 * n)])
    rows, cols, vals, b = [], [], [], []
    r0 = 0
    # zero: F' x - y = 0
    Ft = F.T.tocoo()
    for i, j, v in zip(Ft.row, Ft.col, Ft.data):
        rows.append(r0 + i); cols.append(ix + j); vals.append(v)
    for i in range(k):
        rows.append(r0 + i); cols.append(iy + i); vals.append(-1.0)
    b += [0.0] * k
    r0 += k
    # zero: sum(x) + a sum(s) = d + sum(x0)
    for j in range(n):
        rows.append(r0); cols.append(ix + j); vals.append(1.0)
        rows.append(r0); cols.append(is_ + j); vals.append(a)
    b.append(d + x0.sum())
    r0 += 1
    # zero: x + t = x0
    for j in range(n):
        rows.append(r0 + j); cols.append(ix + j); vals.append(1.0)
        rows.append(r0 + j); cols.append(it + j); vals.append(1.0)
    b += list(x0)
    r0 += n
    # nonneg: -x <= 0
    for j in range(n):
        rows.append(r0 + j); cols.append(ix + j); vals.append(-1.0)
    b += [0.0] * n
    r0 += n
    # SOC(2): (s_i, t_i)
    for j in range(n):
        rows.append(r0); cols.append(is_ + j); vals.append(-1.0)
        rows.append(r0 + 1); cols.append(it + j); vals.append(-1.0)
        b += [0.0, 0.0]
        r0 += 2
    A = sp.csc_matrix((vals, (rows, cols)), shape=(r0, nv))
    cones = [ZeroConeT(k + 1 + n), NonnegativeConeT(n)] + [SecondOrderConeT(2)] * n
    return sp.triu(P, format="csc"), q, A, np.array(b), cones


def _soc_interior(r, dims):
    out = []
    for d in dims:
        tail = r.standard_normal(d - 1)
        out.append(np.concatenate([[1.0 + np.linalg.norm(tail)], tail]))
    return np.concatenate(out) if out else np.zeros(0)


def mixed_socp(scale=1.0, seed=2):
    """Single large mixed-cone QP/SOCP (n=20000, m=60000 at scale 1)."""
    r = _rng(seed)
    n = max(10, int(round(20000 * scale)))
    nz, nnn, nsoc = [max(1, int(round(v * scale))) for v in (2000, 28000, 3000)]
    m = nz + nnn + 10 * nsoc
    per_col = 8
    rows = np.concatenate([r.choice(m, size=per_col, replace=False) for _ in range(n)])
    cols = np.repeat(np.arange(n), per_col)
    A = sp.csc_matrix((r.standard_normal(n * per_col), (rows, cols)), shape=(m, n))
    G = sp.random(n, 10, density=1e-3, random_state=r, data_rvs=r.standard_normal,
                  format="csc")
    P = sp.diags(r.uniform(0.1, 1, n)) + G @ G.T
    x0 = r.standard_normal(n)
    s0 = np.concatenate([np.zeros(nz), r.uniform(0.5, 2, nnn), _soc_interior(r, [10] * nsoc)])
    z0 = np.concatenate([r.standard_normal(nz), r.uniform(0.5, 2, nnn),
                         _soc_interior(r, [10] * nsoc)])
    cones = [ZeroConeT(nz), NonnegativeConeT(nnn)] + [SecondOrderConeT(10)] * nsoc
    return _finish(P, A, x0, s0, z0, cones)


def _svec_sym(M):
    n = M.shape[0]
    out = []
    for j in range(n):
        for i in range(j + 1):
            out.append(M[i, j] if i == j else M[i, j] * np.sqrt(2))
    return np.array(out)


def exp_pow_psd(scale=1.0, seed=3, psd_n=10):
    """Conic LP with exp/pow/PSD/nonneg cones (n=30000 at scale 1)."""
    r = _rng(seed)
    n = max(12, int(round(30000 * scale)))
    nexp = max(1, int(round(20000 * scale)))
    npow = max(1, int(round(5000 * scale)))
    npsd = max(1, int(round(200 * scale)))
    nnn = max(1, int(round(10000 * scale)))
    t = psd_n * (psd_n + 1) // 2
    m_lin = nnn + 3 * nexp + 3 * npow
    per_row = 4
    rows = np.repeat(np.arange(m_lin), per_row)
    cols = np.concatenate([r.choice(n, size=per_row, replace=False) for _ in range(m_lin)])
    vals = r.standard_normal(m_lin * per_row)
    # PSD blocks: each cone couples 4 variables through sparse symmetric matrices
    prow, pcol, pval = [], [], []
    for c in range(npsd):
        for j in r.choice(n, size=4, replace=False):
            M = sp.random(psd_n, psd_n, density=0.3, random_state=r,
                          data_rvs=r.standard_normal).toarray()
            M = M + M.T
            v = _svec_sym(M)
            nzv = np.nonzero(v)[0]
            prow += list(m_lin + c * t + nzv)
            pcol += [j] * len(nzv)
            pval += list(v[nzv])
    m = m_lin + npsd * t
    A = sp.csc_matrix((np.concatenate([vals, pval]),
                       (np.concatenate([rows, prow]), np.concatenate([cols, pcol]))),
                      shape=(m, n))
    alphas = r.uniform(0.2, 0.8, npow)
    x0 = r.standard_normal(n)

    def interior():
        parts = [r.uniform(0.5, 2, nnn)]
        parts.append(np.concatenate([EXP_UNIT * r.uniform(0.5, 2) for _ in range(nexp)]))
        parts.append(np.concatenate([np.array([np.sqrt(1 + a), np.sqrt(2 - a), 0.0])
                                     * r.uniform(0.5, 2) for a in alphas]))
        for _ in range(npsd):
            E = r.standard_normal((psd_n, psd_n)) * 0.1
            parts.append(_svec_sym(np.eye(psd_n) + (E + E.T) / 2))
        return np.concatenate(parts)
    s0, z0 = interior(), interior()
    cones = ([NonnegativeConeT(nnn)] + [ExponentialConeT()] * nexp
             + [PowerConeT(float(a)) for a in alphas] + [PSDTriangleConeT(psd_n)] * npsd)
    return _finish(sp.csc_matrix((n, n)), A, x0, s0, z0, cones)


def psd_lp(side=24, ncones=3, m_eq=None, seed=0):
    """Linear SDP: ncones PSD blocks of the given side (svec variables x),
    m_eq random equality rows coupling them, x + b_psd in the PSD cone,
    cost from an interior dual (same interior-point construction as the
    other families)."""
    r = _rng(seed)
    t = side * (side + 1) // 2
    n = ncones * t
    m_eq = m_eq if m_eq is not None else max(1, n // 4)
    Aeq = sp.random(m_eq, n, density=min(1.0, 8.0 / n), random_state=r,
                    data_rvs=r.standard_normal, format="csc")
    A = sp.vstack([Aeq, -sp.identity(n, format="csc")], format="csc")

    def interior():
        parts = []
        for _ in range(ncones):
            E = r.standard_normal((side, side)) * (0.6 / np.sqrt(side))
            parts.append(_svec_sym(np.eye(side) + (E + E.T) / 2))
        return np.concatenate(parts)
    x0 = r.standard_normal(n)
    s0 = np.concatenate([np.zeros(m_eq), interior()])
    z0 = np.concatenate([r.standard_normal(m_eq), interior()])
    cones = [ZeroConeT(m_eq)] + [PSDTriangleConeT(side)] * ncones
    return _finish(sp.csc_matrix((n, n)), A, x0, s0, z0, cones)


def mpc_qp(seed, n=None):
    """One MPC-style QP/SOCP instance (instance id == seed)."""
    r = _rng(seed)
    if n is None:
        n = int(r.integers(20, 401))
    # P: diag U(0.1,1) + band-2 N(0,0.1) symmetrised, shifted to PSD (a
    # Gershgorin shift: every diagonal entry is raised until it dominates its
    # row by 1e-3)
    dg = r.uniform(0.1, 1, n)
    b1, b2 = r.normal(0, 0.1, n - 1), r.normal(0, 0.1, n - 2)
    rowsum = np.zeros(n)
    rowsum[:-1] += np.abs(b1)
    rowsum[1:] += np.abs(b1)
    rowsum[:-2] += np.abs(b2)
    rowsum[2:] += np.abs(b2)
    dg = np.maximum(dg, rowsum + 1e-3)
    P = sp.diags([dg, b1, b1, b2, b2], [0, 1, -1, 2, -2], shape=(n, n), format="csc")
    # banded equality rows (dynamics-like), bandwidth 4; the windows start at
    # distinct, evenly spaced columns so the rows are independent
    neq = n // 4
    erow, ecol, eval_ = [], [], []
    for i in range(neq):
        j0 = (i * (n - 4)) // max(1, neq - 1) if neq > 1 else 0
        for j in range(j0, min(n, j0 + 4)):
            erow.append(i); ecol.append(j); eval_.append(r.standard_normal())
    # SOC cones
    ksoc = int(r.integers(5, 21))
    sdims = [int(v) for v in r.integers(3, 9, ksoc)]
    nsoc_rows = sum(sdims)
    # box constraints as nonnegative rows: +/- x_j <= u_j on the first variables
    nbox_vars = max(1, (2 * n - neq - nsoc_rows) // 2)
    nbox_vars = min(nbox_vars, n)
    rows, cols, vals = list(erow), list(ecol), list(eval_)
    r0 = neq
    for j in range(nbox_vars):
        rows += [r0, r0 + 1]; cols += [j, j]; vals += [1.0, -1.0]
        r0 += 2
    # each SOC acts on one stage: a window of consecutive variables, two
    # N(0,1) coefficients per row
    for d in sdims:
        w0 = int(r.integers(0, max(1, n - d - 1)))
        for k in range(d):
            for j in (w0 + k, min(n - 1, w0 + k + 1)):
                rows.append(r0 + k); cols.append(int(j)); vals.append(r.standard_normal())
        r0 += d
    m = r0
    A = sp.csc_matrix((vals, (rows, cols)), shape=(m, n))
    x0 = r.standard_normal(n)
    s0 = np.concatenate([np.zeros(neq), r.uniform(0.5, 2, 2 * nbox_vars), _soc_interior(r, sdims)])
    z0 = np.concatenate([r.standard_normal(neq), r.uniform(0.5, 2, 2 * nbox_vars),
                         _soc_interior(r, sdims)])
    cones = ([ZeroConeT(neq)] if neq else []) + [NonnegativeConeT(2 * nbox_vars)] \
        + [SecondOrderConeT(d) for d in sdims]
    return _finish(P, A, x0, s0, z0, cones)


def mpc_batch(count=4096, seed0=0):
    return [mpc_qp(seed0 + i) for i in range(count)]
