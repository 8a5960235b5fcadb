"""Shared helpers for the parity tests (CPU oracle vs the B200 library)."""
import json
import os

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))

# parity bar for full solves: same status, objective within 1e-7 relative,
# iterations within +-2 (primal/dual residuals are checked against tol_feas)
OBJ_RTOL = 1e-7
ITER_TOL = 2


def golden_cases():
    with open(os.path.join(HERE, "golden", "reference_tests.json")) as f:
        cases = json.load(f)
    out = []
    for c in cases:
        n, m = len(c["q"]), len(c["b"])
        P = sp.csc_matrix(np.array(c["P"], dtype=float).reshape(n, n))
        A = sp.csc_matrix(np.array(c["A"], dtype=float).reshape(m, n)) if m else sp.csc_matrix((0, n))
        out.append((c["name"], P, np.array(c["q"], float), A, np.array(c["b"], float),
                    [tuple(k) for k in c["cones"]], c["expect"]))
    return out


def to_cone_objects(specs):
    from cuclarabel_b200 import (ExponentialConeT, NonnegativeConeT, PowerConeT,
                                 PSDTriangleConeT, SecondOrderConeT, ZeroConeT)
    out = []
    for t, d, p in specs:
        out.append([ZeroConeT(d), NonnegativeConeT(d), SecondOrderConeT(d), ExponentialConeT(),
                    PowerConeT(p), PSDTriangleConeT(d)][t])
    return out


def rel_err(a, b):
    return abs(a - b) / max(1.0, abs(b))
