"""Problem files: write_to_file / read_from_file (src/json.jl:17-85).

The file is one JSON object {"settings", "P", "q", "A", "b", "cones"} in the
reference's layout: sparse matrices as {"m", "n", "colptr", "rowval",
"nzval"} with 0-based indices (json.jl:131-139), P as its upper triangle (the
solver's stored form), cones as one-key objects {"ZeroConeT": dim},
{"PowerConeT": alpha}, {"ExponentialConeT": []} (json.jl:141-156), and
settings with infinite values written as +-floatmax and restored on reading
(json.jl:88-108).  The data is the user's, unscaled; this solver path has no
presolve or chordal decomposition, so it is also the solver's internal form.
"""
import json
import math

import numpy as np
import scipy.sparse as sp

from .api import (ExponentialConeT, NonnegativeConeT, PowerConeT, PSDTriangleConeT,
                  SecondOrderConeT, Settings, Solver, ZeroConeT, settings_from)

_FLOATMAX = np.finfo(np.float64).max
_CONES = {"ZeroConeT": ZeroConeT, "NonnegativeConeT": NonnegativeConeT,
          "SecondOrderConeT": SecondOrderConeT, "PSDTriangleConeT": PSDTriangleConeT,
          "PowerConeT": PowerConeT, "ExponentialConeT": ExponentialConeT}
# CPU direct solvers of the reference; this library runs its own FP64 LDL^T
_CPU_METHODS = ("qdldl", "faer", "mkl", "panua", "cholmod")


def _lower_csc(M):
    M = sp.csc_matrix(M)
    M.sum_duplicates()
    M.sort_indices()
    return {"m": int(M.shape[0]), "n": int(M.shape[1]),
            "colptr": M.indptr.astype(np.int64).tolist(),
            "rowval": M.indices.astype(np.int64).tolist(),
            "nzval": M.data.astype(np.float64).tolist()}


def _parse_csc(d):
    return sp.csc_matrix((np.asarray(d["nzval"], np.float64),
                          np.asarray(d["rowval"], np.int64),
                          np.asarray(d["colptr"], np.int64)),
                         shape=(int(d["m"]), int(d["n"])))


def _lower_cone(c):
    name = type(c).__name__
    if isinstance(c, PowerConeT):
        return {name: float(c.alpha)}
    if isinstance(c, ExponentialConeT):
        return {name: []}
    return {name: int(c.dim)}


def _parse_cone(d):
    if len(d) != 1:
        raise ValueError("a cone entry has exactly one key")
    (key, val), = d.items()
    if key not in _CONES:
        raise ValueError("unsupported cone type %s" % key)
    if key == "ExponentialConeT":
        return ExponentialConeT()
    if key == "PowerConeT":
        return PowerConeT(float(val))
    return _CONES[key](int(val))


def _lower_settings(st):
    out = {}
    for f in Settings.__dataclass_fields__:
        v = getattr(st, f)
        if isinstance(v, float) and math.isinf(v):  # sanitize_settings! (json.jl:88-96)
            v = math.copysign(_FLOATMAX, v)
        out[f] = v.item() if isinstance(v, np.generic) else v
    return out


def _parse_settings(d):
    st = Settings()
    for key, v in d.items():
        if key not in Settings.__dataclass_fields__:
            continue  # reference settings this path has no use for
        cur = getattr(st, key)
        if isinstance(cur, bool):
            v = bool(v)
        elif isinstance(cur, int):
            v = int(v)
        elif isinstance(cur, float):
            v = float(v)
            if abs(v) == _FLOATMAX:  # desanitize_settings! (json.jl:99-108)
                v = math.copysign(math.inf, v)
        elif key == "direct_solve_method":
            v = str(v)
            if v in _CPU_METHODS:
                v = "cudss"
        setattr(st, key, v)
    return st


def problem_to_json(P, q, A, b, cones, settings=None):
    """The file's JSON object for one problem."""
    st = settings_from(settings)
    return {"settings": _lower_settings(st), "P": _lower_csc(sp.triu(sp.csc_matrix(P))),
            "q": np.asarray(q, np.float64).ravel().tolist(), "A": _lower_csc(A),
            "b": np.asarray(b, np.float64).ravel().tolist(),
            "cones": [_lower_cone(c) for c in cones]}


def problem_from_json(obj):
    """(P, q, A, b, cones, settings) from the file's JSON object."""
    return (_parse_csc(obj["P"]), np.asarray(obj["q"], np.float64), _parse_csc(obj["A"]),
            np.asarray(obj["b"], np.float64), [_parse_cone(c) for c in obj["cones"]],
            _parse_settings(obj.get("settings", {})))


def write_to_file(solver, filename):
    """write_to_file(solver, filename) (json.jl:17-54): the solver's problem
    data and settings, unscaled.  Solving first is not needed."""
    P, q, A, b, cones = solver.problem
    with open(filename, "w") as f:
        json.dump(problem_to_json(P, q, A, b, cones, solver.settings), f)


def read_from_file(filename, settings=None):
    """read_from_file(filename[, settings]) (json.jl:63-85): a Solver for the
    problem in `filename`, with its stored settings unless `settings` is
    given."""
    with open(filename) as f:
        P, q, A, b, cones, st = problem_from_json(json.load(f))
    return Solver(P, q, A, b, cones, st if settings is None else settings)
