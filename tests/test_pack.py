"""The batch packer (no GPU): the compiled packer (csrc/pack.c) points the
clgpu_problem structs at the problems' own arrays; the general path
concatenates them.  Both must describe the same data, and inputs the
compiled packer does not take must fall through to the general path."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

from cuclarabel_b200 import api, problems
from cuclarabel_b200.api import NonnegativeConeT, PowerConeT, ZeroConeT

FIELDS = (("Pp", ctypes.c_int), ("Pi", ctypes.c_int), ("Px", ctypes.c_double),
          ("q", ctypes.c_double), ("Ap", ctypes.c_int), ("Ai", ctypes.c_int),
          ("Ax", ctypes.c_double), ("b", ctypes.c_double), ("cone_types", ctypes.c_int),
          ("cone_dims", ctypes.c_int), ("cone_params", ctypes.c_double))


def _read(addr, n, ct):
    if n == 0:
        return np.zeros(0)
    return np.ctypeslib.as_array(ctypes.cast(int(addr), ctypes.POINTER(ct)), shape=(n,)).copy()


def _contents(arr):
    out = []
    for x in arr:
        n, m, nc = int(x["n"]), int(x["m"]), int(x["ncones"])
        pn = int(_read(x["Pp"], n + 1, ctypes.c_int)[-1])
        an = int(_read(x["Ap"], n + 1, ctypes.c_int)[-1])
        lens = {"Pp": n + 1, "Pi": pn, "Px": pn, "q": n, "Ap": n + 1, "Ai": an, "Ax": an,
                "b": m, "cone_types": nc, "cone_dims": nc, "cone_params": nc}
        out.append((n, m, nc, [_read(x[f], lens[f], ct) for f, ct in FIELDS]))
    return out


def _general(pbs):
    saved = api._pack
    api._pack = None
    try:
        return api._pack_batch(pbs)
    finally:
        api._pack = saved


def _same(a, b):
    assert a[2] == b[2] and a[3] == b[3]
    for (n1, m1, c1, f1), (n2, m2, c2, f2) in zip(_contents(a[0]), _contents(b[0])):
        assert (n1, m1, c1) == (n2, m2, c2)
        for x, y in zip(f1, f2):
            assert np.array_equal(x, y)


@pytest.mark.skipif(api._pack is None, reason="compiled packer not built")
def test_compiled_packer_matches_general_path():
    pbs = problems.mpc_batch(48, seed0=7) + [problems.portfolio(seed=1)]
    fast = api._pack_batch(pbs)
    assert "problems" in fast[1]  # the compiled path was taken
    _same(fast, _general(pbs))


@pytest.mark.skipif(api._pack is None, reason="compiled packer not built")
def test_compiled_packer_falls_through():
    P = sp.csc_matrix(np.eye(2))
    A = sp.csc_matrix(np.array([[1.0, 1.0], [1.0, 0.0], [0.0, 1.0], [1.0, 0.0], [0.0, 1.0],
                                [-1.0, 0.0]]))
    q = np.array([1.0, 1.0])
    b = np.array([1.0, 0.7, 0.7, 1.0, 1.0, 0.0])
    cones = [ZeroConeT(1), NonnegativeConeT(2), PowerConeT(0.3)]
    base = (P, q, A, b, cones)
    _same(api._pack_batch([base]), _general([base]))
    P64 = P.copy()
    P64.indices = P64.indices.astype(np.int64)
    P64.indptr = P64.indptr.astype(np.int64)
    for variant in (
            [P, q, A, b, cones],                                       # not a tuple
            (P, list(q), A, b, cones),                                 # q not an ndarray
            (P.tocsr(), q, A, b, cones),                               # P not CSC
            (P, q, A, b, {"f": 1, "l": 2, "p": [0.3]}),                # dict cones
            (P64, q, A, b, cones)):                                    # int64 indices
        r = api._pack_batch([variant])
        assert "problems" not in r[1]
        _same(r, _general([base]))
    with pytest.raises(Exception):
        api._pack_batch([(P, q, A, b[:-1], cones)])  # shape mismatch: the reference's error
