"""The seeded synthetic workloads follow the shapes their configurations
name (host only): the portfolio QP, the mixed QP/SOCP and the exp/pow/PSD
LP at reduced scale, and the MPC family of the batched benchmark."""
import numpy as np
import pytest
import scipy.sparse as sp

from cuclarabel_b200 import problems
from cuclarabel_b200.api import (ExponentialConeT, NonnegativeConeT, PowerConeT,
                                 PSDTriangleConeT, SecondOrderConeT, ZeroConeT)


def counts(cones):
    out = {}
    for c in cones:
        out.setdefault(type(c).__name__, []).append(c)
    return out


def rows(cones):
    return sum(c.nvars() for c in cones)


def test_portfolio_shape():
    P, q, A, b, cones = problems.portfolio(seed=1)
    n_assets, k = 50, 5
    assert P.shape == (3 * n_assets + k,) * 2 and A.shape == (206, 155)
    c = counts(cones)
    assert [z.dim for z in c["ZeroConeT"]] == [k + 1 + n_assets]
    assert [z.dim for z in c["NonnegativeConeT"]] == [n_assets]
    assert len(c["SecondOrderConeT"]) == n_assets and {s.dim for s in c["SecondOrderConeT"]} == {2}
    assert rows(cones) == A.shape[0] == len(b)


def test_mixed_socp_shape_at_scale():
    s = 0.05
    P, q, A, b, cones = problems.mixed_socp(scale=s, seed=2)
    n = int(round(20000 * s))
    c = counts(cones)
    assert A.shape[1] == n and P.shape == (n, n)
    assert c["ZeroConeT"][0].dim == int(round(2000 * s))
    assert c["NonnegativeConeT"][0].dim == int(round(28000 * s))
    assert len(c["SecondOrderConeT"]) == int(round(3000 * s))
    assert {x.dim for x in c["SecondOrderConeT"]} == {10}
    assert np.all(np.diff(sp.csc_matrix(A).indptr) == 8)  # 8 nonzeros per column
    Pf = (P + sp.triu(P, 1).T).toarray()
    assert np.linalg.eigvalsh(Pf).min() > 0.05  # diag U(0.1, 1) + G G'


def test_exp_pow_psd_shape_at_scale():
    s = 0.01
    P, q, A, b, cones = problems.exp_pow_psd(scale=s, seed=3)
    c = counts(cones)
    assert P.nnz == 0  # conic LP
    assert len(c["ExponentialConeT"]) == int(round(20000 * s))
    assert len(c["PowerConeT"]) == int(round(5000 * s))
    assert all(0.2 <= p.alpha <= 0.8 for p in c["PowerConeT"])
    assert len(c["PSDTriangleConeT"]) == max(1, int(round(200 * s)))
    assert {x.dim for x in c["PSDTriangleConeT"]} == {10}
    assert rows(cones) == A.shape[0] == len(b)


@pytest.mark.parametrize("seed", range(0, 40, 3))
def test_mpc_instance_shape(seed):
    P, q, A, b, cones = problems.mpc_qp(seed)
    n, m = A.shape[1], A.shape[0]
    assert 20 <= n <= 400
    c = counts(cones)
    socs = c["SecondOrderConeT"]
    assert 5 <= len(socs) <= 20 and all(3 <= s.dim <= 8 for s in socs)
    # m ~ 2n: box rows fill up to 2n around the equality and SOC rows; on the
    # smallest instances 5-20 SOCs of dim 3-8 alone exceed 2n rows
    neq0 = c["ZeroConeT"][0].dim if "ZeroConeT" in c else 0
    fixed = neq0 + sum(x.dim for x in socs)
    if fixed + 2 <= 2 * n:
        assert abs(m - 2 * n) <= 2
    else:
        assert m == fixed + 2
    assert isinstance(cones[0], (ZeroConeT, NonnegativeConeT))
    assert rows(cones) == m == len(b)
    Pf = (P + sp.triu(P, 1).T).toarray()
    assert np.linalg.eigvalsh(Pf).min() > 0  # diagonally dominant by construction
    # banded equality rows: at most 4 nonzeros in a window of 4 columns
    neq = c["ZeroConeT"][0].dim if "ZeroConeT" in c else 0
    Ar = sp.csr_matrix(A)
    for i in range(neq):
        cols = Ar.indices[Ar.indptr[i]:Ar.indptr[i + 1]]
        assert len(cols) <= 4 and cols.max() - cols.min() <= 3


def test_mpc_batch_is_seeded_by_instance_id():
    a = problems.mpc_batch(3, seed0=10)
    b = [problems.mpc_qp(10 + i) for i in range(3)]
    for x, y in zip(a, b):
        assert np.array_equal(x[1], y[1]) and np.array_equal(x[3], y[3])
        assert (x[2] != y[2]).nnz == 0
