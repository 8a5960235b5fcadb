"""Python mirror of Clarabel's user API on top of libclgpu.

``Solver(P, q, A, b, cones, settings)`` + ``solve()`` follow
src/solver.jl:5-70 (constructor, dict cones) and :231-422 (solve!) of the
CuClarabel tree; ``Settings`` carries the fields of src/settings.jl:70-148;
statuses follow src/statuscodes.jl:24-36.  ``BatchSolver`` solves many
independent problems in one lock-step device loop.
"""
import ctypes
import enum
from dataclasses import dataclass, field, fields

import numpy as np
import scipy.sparse as sp

from . import _lib

try:
    from . import _pack  # compiled problem packer (csrc/pack.c)
except ImportError:  # not built: the general packing path below
    _pack = None


# ---------------------------------------------------------------- cones
class SupportedCone:
    code = -1

    def spec(self):
        raise NotImplementedError

    def nvars(self):
        raise NotImplementedError


@dataclass(frozen=True)
class ZeroConeT(SupportedCone):
    dim: int
    code = 0

    def spec(self):
        return (0, int(self.dim), 0.0)

    def nvars(self):
        return int(self.dim)


@dataclass(frozen=True)
class NonnegativeConeT(SupportedCone):
    dim: int
    code = 1

    def spec(self):
        return (1, int(self.dim), 0.0)

    def nvars(self):
        return int(self.dim)


@dataclass(frozen=True)
class SecondOrderConeT(SupportedCone):
    dim: int
    code = 2

    def spec(self):
        return (2, int(self.dim), 0.0)

    def nvars(self):
        return int(self.dim)


@dataclass(frozen=True)
class ExponentialConeT(SupportedCone):
    code = 3

    def spec(self):
        return (3, 3, 0.0)

    def nvars(self):
        return 3


@dataclass(frozen=True)
class PowerConeT(SupportedCone):
    alpha: float
    code = 4

    def spec(self):
        return (4, 3, float(self.alpha))

    def nvars(self):
        return 3


@dataclass(frozen=True)
class PSDTriangleConeT(SupportedCone):
    dim: int
    code = 5

    def spec(self):
        return (5, int(self.dim), 0.0)

    def nvars(self):
        d = int(self.dim)
        return d * (d + 1) // 2


def cones_from_dict(cone):
    """SCS-style dict -> cone list (src/solver.jl:35-70)."""
    out = []
    if "f" in cone:
        out.append(ZeroConeT(cone["f"]))
    if "l" in cone:
        out.append(NonnegativeConeT(cone["l"]))
    for d in cone.get("q", []):
        out.append(SecondOrderConeT(d))
    for d in cone.get("s", []):
        out.append(PSDTriangleConeT(d))
    for _ in range(cone.get("ep", 0)):
        out.append(ExponentialConeT())
    for a in cone.get("p", []):
        out.append(PowerConeT(a))
    return out


class SolverStatus(enum.IntEnum):
    UNSOLVED = 0
    SOLVED = 1
    PRIMAL_INFEASIBLE = 2
    DUAL_INFEASIBLE = 3
    ALMOST_SOLVED = 4
    ALMOST_PRIMAL_INFEASIBLE = 5
    ALMOST_DUAL_INFEASIBLE = 6
    MAX_ITERATIONS = 7
    MAX_TIME = 8
    NUMERICAL_ERROR = 9
    INSUFFICIENT_PROGRESS = 10


_METHODS = {"cudss": 0, "gpu": 0, "fp64": 0, "cudssmixed": 1, "gpumixed": 1, "mixed": 1,
            "mixed_f64elim": 2}


@dataclass
class Settings:
    """Solver settings (src/settings.jl:70-148).  ``direct_solve_method``
    accepts the reference names "cudss" (FP64 factorisation) and
    "cudssmixed" (FP32 factorisation + FP64 iterative refinement); both run
    this library's batched LDL^T.  "mixed_f64elim" is this library's variant
    of the mixed form: FP64 elimination, the factor stored and applied in
    FP32, FP64 refinement."""
    max_iter: int = 200
    time_limit: float = float("inf")
    verbose: bool = False
    max_step_fraction: float = 0.99
    tol_gap_abs: float = 1e-8
    tol_gap_rel: float = 1e-8
    tol_feas: float = 1e-8
    tol_infeas_abs: float = 1e-8
    tol_infeas_rel: float = 1e-8
    tol_ktratio: float = 1e-6
    reduced_tol_gap_abs: float = 5e-5
    reduced_tol_gap_rel: float = 5e-5
    reduced_tol_feas: float = 1e-4
    reduced_tol_infeas_abs: float = 5e-12
    reduced_tol_infeas_rel: float = 5e-5
    reduced_tol_ktratio: float = 1e-4
    equilibrate_enable: bool = True
    equilibrate_max_iter: int = 10
    equilibrate_min_scaling: float = 1e-4
    equilibrate_max_scaling: float = 1e4
    linesearch_backtrack_step: float = 0.8
    min_switch_step_length: float = 1e-2
    min_terminate_step_length: float = 1e-4
    direct_kkt_solver: bool = True
    direct_solve_method: str = "cudss"
    static_regularization_enable: bool = True
    static_regularization_constant: float = 1e-8
    static_regularization_proportional: float = np.finfo(float).eps ** 2
    dynamic_regularization_enable: bool = True
    dynamic_regularization_eps: float = 1e-13
    dynamic_regularization_delta: float = 2e-7
    iterative_refinement_enable: bool = True
    iterative_refinement_reltol: float = 1e-12
    iterative_refinement_abstol: float = 1e-12
    iterative_refinement_max_iter: int = 10
    iterative_refinement_stop_ratio: float = 5.0
    presolve_enable: bool = True
    chordal_decomposition_enable: bool = True
    soc_threshold: int = 5
    setup_threads: int = 0
    fused_solves: bool = True
    device_setup: bool = True
    autotune: bool = True

    def to_c(self):
        if self.direct_solve_method not in _METHODS:
            raise ValueError("Unsupported direct LDL linear solver :%s" % self.direct_solve_method)
        c = _lib.ClgpuSettings()
        _lib.load().clgpu_default_settings(ctypes.byref(c))
        for f, _ in _lib.ClgpuSettings._fields_:
            if f == "direct_solve_method":
                c.direct_solve_method = _METHODS[self.direct_solve_method]
            elif hasattr(self, f):
                v = getattr(self, f)
                setattr(c, f, int(v) if isinstance(v, (bool, np.bool_)) else v)
        return c


def settings_from(settings=None, **kwargs):
    s = Settings() if settings is None else settings
    if isinstance(s, dict):
        kwargs = {**s, **kwargs}
        s = Settings()
    names = {f.name for f in fields(Settings)}
    for k, v in kwargs.items():
        if k not in names:
            raise TypeError("unknown setting %r" % k)
        setattr(s, k, v)
    return s


@dataclass
class DefaultSolution:
    """src/types.jl DefaultSolution."""
    x: np.ndarray
    z: np.ndarray
    s: np.ndarray
    status: SolverStatus
    obj_val: float
    obj_val_dual: float
    solve_time: float
    iterations: int
    r_prim: float
    r_dual: float
    info: dict = field(default_factory=dict)


def _as_csc(M, shape):
    """CSC view of M without a copy when it already is CSC with canonical
    (sorted, duplicate-free) indices."""
    if M is None:
        return sp.csc_matrix(shape)
    if not (sp.issparse(M) and M.format == "csc"):
        M = sp.csc_matrix(M)
    if not M.has_canonical_format:
        M = M.copy()
        M.sum_duplicates()
    return M


def _i32(a):
    return a if (a.dtype == np.int32 and a.flags.c_contiguous) else np.ascontiguousarray(a, np.int32)


def _f64(a):
    return a if (a.dtype == np.float64 and a.flags.c_contiguous) else np.ascontiguousarray(a, np.float64)


def _prep_problem(P, q, A, b, cones):
    """Host arrays of one problem for clgpu_problem.  P may be full or upper
    triangular: the library reads its upper triangle (src/solver.jl:618-630
    applies triu on the same path)."""
    q = _f64(np.asarray(q, dtype=np.float64).ravel())
    b = _f64(np.asarray(b, dtype=np.float64).ravel())
    n, m = len(q), len(b)
    if isinstance(cones, dict):
        cones = cones_from_dict(cones)
    specs = [c.spec() for c in cones]
    P = _as_csc(P, (n, n))
    A = _as_csc(A, (m, n))
    # _check_dimensions (src/solver.jl:199-211)
    if A.shape[0] != m:
        raise ValueError("A and b incompatible dimensions.")
    if sum(_nvars(s) for s in specs) != m:
        raise ValueError("Constraint dimensions inconsistent with size of cones.")
    if A.shape[1] != n:
        raise ValueError("A and q incompatible dimensions.")
    if P.shape[0] != n:
        raise ValueError("P and q incompatible dimensions.")
    if P.shape[0] != P.shape[1]:
        raise ValueError("P not square.")
    keep = (_i32(P.indptr), _i32(P.indices), _f64(P.data), q,
            _i32(A.indptr), _i32(A.indices), _f64(A.data), b,
            np.array([s[0] for s in specs] or [0], np.int32),
            np.array([s[1] for s in specs] or [0], np.int32),
            np.array([s[2] for s in specs] or [0.0], np.float64))
    cp = _lib.ClgpuProblem(
        n, m, *(a.ctypes.data_as(_lib.dp if a.dtype == np.float64 else _lib.ip)
                for a in keep[:8]),
        len(specs), *(a.ctypes.data_as(_lib.dp if a.dtype == np.float64 else _lib.ip)
                      for a in keep[8:]))
    return cp, keep, n, m


_PROBLEM_DTYPE = np.dtype([
    ("n", np.int32), ("m", np.int32),
    ("Pp", np.uint64), ("Pi", np.uint64), ("Px", np.uint64), ("q", np.uint64),
    ("Ap", np.uint64), ("Ai", np.uint64), ("Ax", np.uint64), ("b", np.uint64),
    ("ncones", np.int32), ("pad", np.int32),
    ("cone_types", np.uint64), ("cone_dims", np.uint64), ("cone_params", np.uint64)])


def _pack_batch(problems):
    """clgpu_problem array for a batch.  The compiled packer (csrc/pack.c)
    points the structs straight at the problems' own arrays when every
    problem is a (P, q, A, b, cones) tuple of canonical CSC matrices and
    float64 vectors; otherwise each field's arrays are concatenated once and
    every instance's pointers are computed from offsets."""
    if _pack is not None:
        arr = np.zeros(len(problems), _PROBLEM_DTYPE)
        r = _pack.pack(problems, arr)
        if r is not None:
            ct, cd, cp, dims, pn, an = r
            d = np.frombuffer(dims, np.int32)[:2 * len(problems)].reshape(-1, 2)
            keep = {"arr": arr, "ct": ct, "cd": cd, "cp": cp, "problems": problems}
            return arr, keep, list(map(tuple, d.tolist())), (int(pn), int(an))
    parts = {k: [] for k in ("Pp", "Pi", "Px", "q", "Ap", "Ai", "Ax", "b")}
    ct, cd, cp = [], [], []
    nm = np.zeros((len(problems), 3), np.int64)
    for k, (P, q, A, b, cones) in enumerate(problems):
        q = np.asarray(q, dtype=np.float64).ravel()
        b = np.asarray(b, dtype=np.float64).ravel()
        n, m = len(q), len(b)
        if isinstance(cones, dict):
            cones = cones_from_dict(cones)
        specs = [c.spec() for c in cones]
        nc = len(specs)
        if nc:
            t_, d_, a_ = zip(*specs)
            ct.extend(t_)
            cd.extend(d_)
            cp.extend(a_)
            nv = sum(d if t < 3 else (3 if t < 5 else d * (d + 1) // 2) for t, d in zip(t_, d_))
        else:
            nv = 0
        P = _as_csc(P, (n, n))
        A = _as_csc(A, (m, n))
        if A.shape != (m, n) or P.shape != (n, n) or nv != m:
            _prep_problem(P, q, A, b, cones)  # raises the reference's message
        parts["Pp"].append(P.indptr); parts["Pi"].append(P.indices); parts["Px"].append(P.data)
        parts["q"].append(q)
        parts["Ap"].append(A.indptr); parts["Ai"].append(A.indices); parts["Ax"].append(A.data)
        parts["b"].append(b)
        nm[k] = (n, m, nc)
    keep = {}
    arr = np.zeros(len(problems), _PROBLEM_DTYPE)
    arr["n"], arr["m"], arr["ncones"] = nm[:, 0], nm[:, 1], nm[:, 2]
    n_, m_, c_ = nm[:, 0], nm[:, 1], nm[:, 2]
    cone_lists = {"ct": np.asarray(ct + [0], np.int32), "cd": np.asarray(cd + [0], np.int32),
                  "cp": np.asarray(cp + [0.0], np.float64)}
    for f, dt in (("Pp", np.int32), ("Pi", np.int32), ("Px", np.float64), ("q", np.float64),
                  ("Ap", np.int32), ("Ai", np.int32), ("Ax", np.float64), ("b", np.float64),
                  ("ct", np.int32), ("cd", np.int32), ("cp", np.float64)):
        if f in cone_lists:
            flat, lens = cone_lists[f], c_
        else:
            flat = np.concatenate([a if a.dtype == dt else np.asarray(a, dt) for a in parts[f]]
                                  + [np.zeros(1, dt)])
            lens = np.fromiter((len(a) for a in parts[f]), np.int64, len(problems))
        keep[f] = flat
        offs = np.concatenate([[0], np.cumsum(lens)[:-1]]) * flat.itemsize
        field = {"ct": "cone_types", "cd": "cone_dims", "cp": "cone_params"}.get(f, f)
        arr[field] = np.uint64(flat.ctypes.data) + offs.astype(np.uint64)
    keep["arr"] = arr
    counts = (len(keep["Px"]) - 1, len(keep["Ax"]) - 1)
    return arr, keep, [(int(n), int(m)) for n, m, _ in nm], counts


def _nvars(spec):
    t, d, _ = spec
    return 3 if t in (3, 4) else (d * (d + 1) // 2 if t == 5 else d)


# launch kinds of the supernodal factorisation (CLGPU_SN_KINDS, clgpu.h)
SN_KIND_NAMES = ["small_fronts", "assemble", "diag", "trsm", "update", "fwd_small",
                 "fwd_gather", "fwd_diag", "fwd_gemv", "fwd_scatter", "bwd_small", "bwd_gather",
                 "bwd_partial", "bwd_diag", "bwd_scatter"]
SN_KINDS = len(SN_KIND_NAMES)


class _StagingView:
    """Read-only array interface over n doubles of a solver's pinned result
    staging.  numpy keeps this object as the array's base, and it keeps the
    solver: the staging (freed by clgpu_solver_destroy) outlives every view."""

    def __init__(self, addr, n, owner):
        self._owner = owner
        self.__array_interface__ = {"shape": (n,), "typestr": "<f8", "version": 3,
                                    "data": (addr, True)}


class BatchSolver:
    """Many independent problems solved in one lock-step device loop."""

    def __init__(self, problems, settings=None, **kwargs):
        self.settings = settings_from(settings, **kwargs)
        L = _lib.load()
        arr, keep, self.dims, (self._np, self._na) = _pack_batch(problems)
        cs = self.settings.to_c()
        h = ctypes.c_void_p()
        rc = L.clgpu_solver_create(arr.ctypes.data_as(ctypes.POINTER(_lib.ClgpuProblem)),
                                   len(problems), ctypes.byref(cs), ctypes.byref(h))
        del keep
        if rc != 0:
            raise RuntimeError("clgpu_solver_create failed with code %d" % rc)
        self._h = h  # host arrays were copied by the library
        self._destroy = L.clgpu_solver_destroy  # held for interpreter shutdown
        self.nx = sum(d[0] for d in self.dims)
        self.mz = sum(d[1] for d in self.dims)

    def __del__(self):
        h = getattr(self, "_h", None)
        destroy = getattr(self, "_destroy", None)
        if h and destroy is not None:
            destroy(h)
            self._h = None

    def update_data(self, P=None, q=None, A=None, b=None, stream=0):
        """update_data!(solver, P, q, A, b) for every instance
        (src/data_updating.jl).  Each argument is a concatenated 1-D array of
        new values -- for P and A the nonzeros in the CSC order given at setup,
        instance by instance -- or a list with one entry per instance (sparse
        matrices with the setup sparsity, or value arrays); None leaves that
        part unchanged.  The equilibration computed at setup is reused, as in
        the reference."""
        def cat(v, kind):
            if v is None:
                return None
            if isinstance(v, (list, tuple)):
                parts = []
                for k, x in enumerate(v):
                    if kind in ("P", "A") and sp.issparse(x):
                        x = _as_csc(x, x.shape).data
                    parts.append(np.asarray(x, np.float64).ravel())
                v = np.concatenate(parts) if parts else np.zeros(0)
            return _f64(np.asarray(v, np.float64).ravel())
        Pv, qv, Av, bv = cat(P, "P"), cat(q, "q"), cat(A, "A"), cat(b, "b")
        for v, n, name in ((Pv, self._np, "P"), (qv, self.nx, "q"), (Av, self._na, "A"),
                           (bv, self.mz, "b")):
            if v is not None and len(v) != n:
                raise ValueError("%s: expected %d values, got %d" % (name, n, len(v)))
        ptr = lambda v: None if v is None else v.ctypes.data_as(_lib.dp)  # noqa: E731
        rc = _lib.load().clgpu_solver_update_data(self._h, ptr(Pv), ptr(qv), ptr(Av), ptr(bv),
                                                   ctypes.c_void_p(stream))
        if rc != 0:
            raise RuntimeError("clgpu_solver_update_data failed with code %d" % rc)

    def solve_only(self, stream=0):
        """solve! without building per-instance solution objects (read the
        results with results() or solutions())."""
        rc = _lib.load().clgpu_solver_solve(self._h, ctypes.c_void_p(stream))
        if rc != 0:
            raise RuntimeError("clgpu_solver_solve failed with code %d" % rc)

    def solve(self, stream=0):
        L = _lib.load()
        rc = L.clgpu_solver_solve(self._h, ctypes.c_void_p(stream))
        if rc != 0:
            raise RuntimeError("clgpu_solver_solve failed with code %d" % rc)
        return self.solutions()

    def results(self, out=None, view=False):
        """The last solve's results as arrays (no per-instance objects): x, s,
        z concatenated over instances (offsets xoff / moff) and a structured
        array of the DefaultInfo fields, one row per instance.  `out` may be
        a previous return value of results(): its arrays are filled in place
        (no new host allocation for repeated solves).  view=True returns x,
        s, z as read-only arrays over the library's pinned result staging,
        without a copy; the next solve overwrites them, and each array keeps
        the solver (and so the staging) alive while it exists."""
        L = _lib.load()
        B = len(self.dims)
        if view:
            px, ps, pz = _lib.dp(), _lib.dp(), _lib.dp()
            rc = L.clgpu_solver_get_solution_views(self._h, ctypes.byref(px), ctypes.byref(ps),
                                                   ctypes.byref(pz))
            if rc != 0:
                raise RuntimeError("clgpu_solver_get_solution_views failed with code %d" % rc)
            infos = out["_infos"] if out is not None else (_lib.ClgpuInfo * B)()
            rc = L.clgpu_solver_get_solutions(self._h, None, None, None, infos)
            if rc != 0:
                raise RuntimeError("clgpu_solver_get_solutions failed with code %d" % rc)
            arrs = []
            for p, n in ((px, self.nx), (ps, self.mz), (pz, self.mz)):
                if n == 0:
                    a = np.empty(0)
                    a.flags.writeable = False
                    arrs.append(a)
                    continue
                addr = ctypes.cast(p, ctypes.c_void_p).value
                arrs.append(np.asarray(_StagingView(addr, n, self)))
            info = np.ctypeslib.as_array(infos)
            return {"x": arrs[0], "s": arrs[1], "z": arrs[2], "info": info,
                    "status": info["status"].copy(), "_infos": infos}
        if out is not None:
            x, s, z = out["x"], out["s"], out["z"]
            for a, n in ((x, self.nx), (s, self.mz), (z, self.mz)):
                if a.dtype != np.float64 or not a.flags.c_contiguous or len(a) < n:
                    raise ValueError("results(out=...): arrays of the last results() needed")
            infos = out["_infos"]
        else:
            x = np.empty(max(self.nx, 1))
            s = np.empty(max(self.mz, 1))
            z = np.empty(max(self.mz, 1))
            infos = (_lib.ClgpuInfo * B)()
        rc = L.clgpu_solver_get_solutions(self._h, x.ctypes.data_as(_lib.dp),
                                          s.ctypes.data_as(_lib.dp), z.ctypes.data_as(_lib.dp),
                                          infos)
        if rc != 0:
            raise RuntimeError("clgpu_solver_get_solutions failed with code %d" % rc)
        info = np.ctypeslib.as_array(infos)
        return {"x": x[:self.nx], "s": s[:self.mz], "z": z[:self.mz], "info": info,
                "status": info["status"].copy(), "_infos": infos}

    def solutions(self):
        L = _lib.load()
        B = len(self.dims)
        x = np.zeros(max(self.nx, 1))
        s = np.zeros(max(self.mz, 1))
        z = np.zeros(max(self.mz, 1))
        infos = (_lib.ClgpuInfo * B)()
        rc = L.clgpu_solver_get_solutions(self._h, x.ctypes.data_as(_lib.dp),
                                          s.ctypes.data_as(_lib.dp), z.ctypes.data_as(_lib.dp),
                                          infos)
        if rc != 0:
            raise RuntimeError("clgpu_solver_get_solutions failed with code %d" % rc)
        out = []
        xo = mo = 0
        for k, (n, m) in enumerate(self.dims):
            inf = infos[k]
            d = {f: getattr(inf, f) for f, _ in _lib.ClgpuInfo._fields_}
            out.append(DefaultSolution(
                x=x[xo:xo + n].copy(), z=z[mo:mo + m].copy(), s=s[mo:mo + m].copy(),
                status=SolverStatus(inf.status), obj_val=inf.obj_val,
                obj_val_dual=inf.obj_val_dual, solve_time=inf.solve_time,
                iterations=inf.iterations, r_prim=inf.res_primal, r_dual=inf.res_dual,
                info=d))
            xo += n
            mo += m
        return out

    # ------------------------------------------------------------ serving
    # Continuous batching: the instances are slots.  serve_admit starts new
    # solves in idle slots (optionally with new q / b, one array per slot)
    # while others are mid-solve; serve_step runs one IPM iteration of every
    # running slot and returns the slots that finished in it; serve_collect
    # returns their solutions and frees the slots.

    def serve_admit(self, slots, q=None, b=None, stream=0):
        slots = np.ascontiguousarray(np.asarray(slots, dtype=np.int32))
        if slots.size == 0:
            return
        def packed(vals, which):
            if vals is None:
                return None
            if len(vals) != slots.size:
                raise ValueError("one %s array per admitted slot" % which)
            parts = []
            for k, v in zip(slots, vals):
                v = np.asarray(v, np.float64).ravel()
                want = self.dims[k][0] if which == "q" else self.dims[k][1]
                if v.size != want:
                    raise ValueError("slot %d: %s needs %d values" % (k, which, want))
                parts.append(v)
            return _f64(np.concatenate(parts))
        qv, bv = packed(q, "q"), packed(b, "b")
        ptr = lambda v: None if v is None else v.ctypes.data_as(_lib.dp)  # noqa: E731
        rc = _lib.load().clgpu_serve_admit(self._h, slots.ctypes.data_as(_lib.ip), slots.size,
                                           ptr(qv), ptr(bv), ctypes.c_void_p(stream))
        if rc != 0:
            raise RuntimeError("clgpu_serve_admit failed with code %d" % rc)

    def serve_step(self, stream=0):
        """One IPM iteration of every running slot: (finished slots, running)."""
        fin = np.empty(len(self.dims), np.int32)
        nf, nr = ctypes.c_int(), ctypes.c_int()
        rc = _lib.load().clgpu_serve_step(self._h, ctypes.c_void_p(stream),
                                          fin.ctypes.data_as(_lib.ip), ctypes.byref(nf),
                                          ctypes.byref(nr))
        if rc != 0:
            raise RuntimeError("clgpu_serve_step failed with code %d" % rc)
        return fin[:nf.value].tolist(), nr.value

    def serve_collect(self, slots, stream=0):
        slots = np.ascontiguousarray(np.asarray(slots, dtype=np.int32))
        n = slots.size
        if n == 0:
            return []
        nx = sum(self.dims[k][0] for k in slots)
        mz = sum(self.dims[k][1] for k in slots)
        x, s, z = np.empty(max(nx, 1)), np.empty(max(mz, 1)), np.empty(max(mz, 1))
        infos = (_lib.ClgpuInfo * n)()
        rc = _lib.load().clgpu_serve_collect(self._h, slots.ctypes.data_as(_lib.ip), n,
                                             x.ctypes.data_as(_lib.dp), s.ctypes.data_as(_lib.dp),
                                             z.ctypes.data_as(_lib.dp), infos,
                                             ctypes.c_void_p(stream))
        if rc != 0:
            raise RuntimeError("clgpu_serve_collect failed with code %d" % rc)
        out, xo, mo = [], 0, 0
        for k, slot in enumerate(slots):
            n_i, m_i = self.dims[slot]
            inf = infos[k]
            d = {f: getattr(inf, f) for f, _ in _lib.ClgpuInfo._fields_}
            out.append(DefaultSolution(
                x=x[xo:xo + n_i].copy(), z=z[mo:mo + m_i].copy(), s=s[mo:mo + m_i].copy(),
                status=SolverStatus(inf.status), obj_val=inf.obj_val,
                obj_val_dual=inf.obj_val_dual, solve_time=inf.solve_time,
                iterations=inf.iterations, r_prim=inf.res_primal, r_dual=inf.res_dual, info=d))
            xo += n_i
            mo += m_i
        return out

    def device_bytes(self):
        return _lib.load().clgpu_solver_device_bytes(self._h)

    def launch_count(self):
        return _lib.load().clgpu_solver_launch_count(self._h)

    SOC_OPS = ("update_scaling", "affine_ds", "combined_ds_shift", "ds_from_dz_offset",
               "step_length", "mul_Hs")

    def launch_shapes(self):
        """Launch shapes the setup autotuner chose for this batch: threads per
        block of the nonnegative kernels, and per SOC operation "groups" (one
        lane group per cone) or "tiles<C>" (shared-memory tiles of C cones)."""
        nb, v = ctypes.c_int(), (ctypes.c_int * len(self.SOC_OPS))()
        rc = _lib.load().clgpu_solver_get_launch_shapes(self._h, ctypes.byref(nb), v)
        if rc != 0:
            raise RuntimeError("clgpu_solver_get_launch_shapes failed with code %d" % rc)
        return {"nn_block": nb.value,
                "soc": {op: ("groups" if x == 0 else "tiles%d" % (32 << (x - 1)))
                        for op, x in zip(self.SOC_OPS, v)}}

    def set_profiling(self, enable=True):
        _lib.load().clgpu_solver_set_profiling(self._h, 1 if enable else 0)

    def profile(self):
        """Device time of the last solve: total and per phase (ms)."""
        L = _lib.load()
        vals = [ctypes.c_double() for _ in range(5)]
        passes = ctypes.c_int()
        L.clgpu_solver_get_profile(self._h, *[ctypes.byref(v) for v in vals],
                                   ctypes.byref(passes))
        ms = (ctypes.c_double * 6)()
        calls = (ctypes.c_longlong * 6)()
        L.clgpu_solver_get_phase_times(self._h, ms, calls)
        names = ["ldl_factor", "ldl_solve", "kkt_refresh", "residual", "update_scaling",
                 "ldl_solve2"]
        by = (ctypes.c_double * 3)()
        L.clgpu_solver_get_phase_bytes(self._h, by)
        out = dict(ms_total=vals[0].value, passes=passes.value,
                   phases={n: (ms[i], calls[i]) for i, n in enumerate(names)},
                   bytes={"ldl_factor": by[0], "ldl_solve": by[1], "ldl_solve2": by[2]})
        sms = (ctypes.c_double * SN_KINDS)()
        sfl = (ctypes.c_double * SN_KINDS)()
        scl = (ctypes.c_longlong * SN_KINDS)()
        if L.clgpu_solver_get_sn_profile(self._h, sms, sfl, scl) == 0:
            out["supernodal"] = {n: {"ms": sms[i], "flops": sfl[i], "launches": scl[i]}
                                 for i, n in enumerate(SN_KIND_NAMES)}
            cnt = (ctypes.c_longlong * 3)()
            worst = ctypes.c_double()
            L.clgpu_solver_get_sn_refinement(self._h, cnt, ctypes.byref(worst))
            out["refinement"] = {"solves": cnt[0], "sweeps": cnt[1], "unconverged": cnt[2],
                                 "worst_ratio": worst.value}
        return out


class Solver(BatchSolver):
    """Clarabel.Solver(P, q, A, b, cones, settings) for one problem."""

    def __init__(self, P, q, A, b, cones, settings=None, **kwargs):
        super().__init__([(P, q, A, b, cones)], settings, **kwargs)
        self.solution = None
        # the problem as given (for write_to_file), kept current by update_*
        n, m = len(np.ravel(q)), len(np.ravel(b))
        if isinstance(cones, dict):
            cones = cones_from_dict(cones)
        self.problem = (_as_csc(P, (n, n)).copy(), np.array(q, np.float64).ravel(),
                        _as_csc(A, (m, n)).copy(), np.array(b, np.float64).ravel(), list(cones))

    def solve(self, stream=0):
        self.solution = super().solve(stream)[0]
        return self.solution

    # update_P! / update_q! / update_A! / update_b! (src/data_updating.jl)
    def update_P(self, P):
        self.update_data(P=[P])
        P0, q, A, b, c = self.problem
        P1 = P0.copy()
        P1.data = (_as_csc(P, P0.shape).data if sp.issparse(P)
                   else np.asarray(P, np.float64).ravel()).copy()
        self.problem = (P1, q, A, b, c)

    def update_q(self, q):
        self.update_data(q=q)
        P, _, A, b, c = self.problem
        self.problem = (P, np.array(q, np.float64).ravel(), A, b, c)

    def update_A(self, A):
        self.update_data(A=[A])
        P, q, A0, b, c = self.problem
        A1 = A0.copy()
        A1.data = (_as_csc(A, A0.shape).data if sp.issparse(A)
                   else np.asarray(A, np.float64).ravel()).copy()
        self.problem = (P, q, A1, b, c)

    def update_b(self, b):
        self.update_data(b=b)
        P, q, A, _, c = self.problem
        self.problem = (P, q, A, np.array(b, np.float64).ravel(), c)

    @property
    def info(self):
        return None if self.solution is None else self.solution.info
