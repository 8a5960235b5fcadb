"""Problem files in the reference's JSON layout (src/json.jl), host side."""
import json
import math

import numpy as np
import pytest
import scipy.sparse as sp

from cuclarabel_b200 import (ExponentialConeT, NonnegativeConeT, PowerConeT,
                             PSDTriangleConeT, SecondOrderConeT, Settings, ZeroConeT, problems)
from cuclarabel_b200.json_io import problem_from_json, problem_to_json


def test_round_trip_mixed_cones(tmp_path):
    P, q, A, b, cones = problems.exp_pow_psd(scale=0.002, seed=5)
    st = Settings(max_iter=77, tol_gap_abs=1e-9)
    obj = problem_to_json(P, q, A, b, cones, st)
    f = tmp_path / "p.json"
    f.write_text(json.dumps(obj))
    P2, q2, A2, b2, c2, st2 = problem_from_json(json.loads(f.read_text()))
    assert (P2 != sp.triu(sp.csc_matrix(P))).nnz == 0
    assert (A2 != sp.csc_matrix(A)).nnz == 0
    assert np.array_equal(q2, q) and np.array_equal(b2, b)
    assert c2 == list(cones)
    assert st2.max_iter == 77 and st2.tol_gap_abs == 1e-9
    assert math.isinf(st2.time_limit) and st2.time_limit > 0   # written as floatmax


def test_reads_reference_layout():
    """The object write_to_file produces for test/UnitTests/test_json.jl's
    problem (0-based CSC, triangular P, one-key cones, floatmax for Inf,
    a CPU direct_solve_method)."""
    obj = {
        "settings": {"max_iter": 200, "time_limit": np.finfo(float).max,
                     "direct_solve_method": "qdldl", "static_regularization_constant": 1e-8,
                     "some_cpu_only_setting": True},
        "P": {"m": 2, "n": 2, "colptr": [0, 1, 3], "rowval": [0, 0, 1], "nzval": [4.0, 1.0, 2.0]},
        "q": [1.0, 1.0],
        "A": {"m": 3, "n": 2, "colptr": [0, 2, 4], "rowval": [0, 1, 0, 2],
              "nzval": [1.0, 1.0, 1.0, 1.0]},
        "b": [1.0, 1.0, 1.0],
        "cones": [{"NonnegativeConeT": 1}, {"ZeroConeT": 1}, {"NonnegativeConeT": 1}],
    }
    P, q, A, b, cones, st = problem_from_json(obj)
    assert np.array_equal(P.toarray(), [[4.0, 1.0], [0.0, 2.0]])
    assert np.array_equal(A.toarray(), [[1.0, 1.0], [1.0, 0.0], [0.0, 1.0]])
    assert cones == [NonnegativeConeT(1), ZeroConeT(1), NonnegativeConeT(1)]
    assert math.isinf(st.time_limit) and st.direct_solve_method == "cudss"


def test_cone_encodings():
    cones = [ZeroConeT(2), NonnegativeConeT(3), SecondOrderConeT(4), ExponentialConeT(),
             PowerConeT(0.3), PSDTriangleConeT(3)]
    n = 1
    m = 2 + 3 + 4 + 3 + 3 + 6
    obj = problem_to_json(sp.csc_matrix((n, n)), np.zeros(n), sp.csc_matrix((m, n)), np.zeros(m),
                          cones)
    assert obj["cones"] == [{"ZeroConeT": 2}, {"NonnegativeConeT": 3}, {"SecondOrderConeT": 4},
                            {"ExponentialConeT": []}, {"PowerConeT": 0.3},
                            {"PSDTriangleConeT": 3}]
    assert problem_from_json(obj)[4] == cones
    obj["cones"].append({"GenPowerConeT": [[0.5, 0.5], 1]})
    with pytest.raises(ValueError):
        problem_from_json(obj)
