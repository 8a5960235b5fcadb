"""CPU oracle for the Clarabel interior-point path (TEST INFRASTRUCTURE ONLY).

This package wraps ``liboracle.so`` (a C++ restatement of the reference's CPU
Clarabel path; see ``clarabel_oracle.h`` for the file-by-file citations).  It
is the checker for the B200 library: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline legs may use it.
The product package ``cuclarabel_b200`` never imports it.

Cones are passed as ``(type_code, dim, param)`` tuples, or as objects with a
``spec()`` method returning such a tuple.  Type codes: 0 zero, 1 nonnegative,
2 second-order, 3 exponential, 4 power (param = alpha), 5 PSD triangle
(dim = matrix side).
"""
import ctypes
import os
import subprocess

import numpy as np
import scipy.sparse as sp

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

STATUS_NAMES = {
    0: "UNSOLVED", 1: "SOLVED", 2: "PRIMAL_INFEASIBLE", 3: "DUAL_INFEASIBLE",
    4: "ALMOST_SOLVED", 5: "ALMOST_PRIMAL_INFEASIBLE",
    6: "ALMOST_DUAL_INFEASIBLE", 7: "MAX_ITERATIONS", 8: "MAX_TIME",
    9: "NUMERICAL_ERROR", 10: "INSUFFICIENT_PROGRESS",
}


class OracleSettings(ctypes.Structure):
    _fields_ = [
        ("max_iter", ctypes.c_int), ("time_limit", ctypes.c_double),
        ("max_step_fraction", ctypes.c_double),
        ("tol_gap_abs", ctypes.c_double), ("tol_gap_rel", ctypes.c_double),
        ("tol_feas", ctypes.c_double), ("tol_infeas_abs", ctypes.c_double),
        ("tol_infeas_rel", ctypes.c_double), ("tol_ktratio", ctypes.c_double),
        ("reduced_tol_gap_abs", ctypes.c_double),
        ("reduced_tol_gap_rel", ctypes.c_double),
        ("reduced_tol_feas", ctypes.c_double),
        ("reduced_tol_infeas_abs", ctypes.c_double),
        ("reduced_tol_infeas_rel", ctypes.c_double),
        ("reduced_tol_ktratio", ctypes.c_double),
        ("equilibrate_enable", ctypes.c_int),
        ("equilibrate_max_iter", ctypes.c_int),
        ("equilibrate_min_scaling", ctypes.c_double),
        ("equilibrate_max_scaling", ctypes.c_double),
        ("linesearch_backtrack_step", ctypes.c_double),
        ("min_switch_step_length", ctypes.c_double),
        ("min_terminate_step_length", ctypes.c_double),
        ("static_regularization_enable", ctypes.c_int),
        ("static_regularization_constant", ctypes.c_double),
        ("static_regularization_proportional", ctypes.c_double),
        ("dynamic_regularization_enable", ctypes.c_int),
        ("dynamic_regularization_eps", ctypes.c_double),
        ("dynamic_regularization_delta", ctypes.c_double),
        ("iterative_refinement_enable", ctypes.c_int),
        ("iterative_refinement_reltol", ctypes.c_double),
        ("iterative_refinement_abstol", ctypes.c_double),
        ("iterative_refinement_max_iter", ctypes.c_int),
        ("iterative_refinement_stop_ratio", ctypes.c_double),
        ("verbose", ctypes.c_int),
        ("gpu_equilibration", ctypes.c_int),
        ("factor_fp32", ctypes.c_int),
    ]


class OracleInfo(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int), ("iterations", ctypes.c_int),
        ("obj_val", ctypes.c_double), ("obj_val_dual", ctypes.c_double),
        ("cost_primal", ctypes.c_double), ("cost_dual", ctypes.c_double),
        ("res_primal", ctypes.c_double), ("res_dual", ctypes.c_double),
        ("res_primal_inf", ctypes.c_double), ("res_dual_inf", ctypes.c_double),
        ("gap_abs", ctypes.c_double), ("gap_rel", ctypes.c_double),
        ("ktratio", ctypes.c_double), ("mu", ctypes.c_double),
        ("sigma", ctypes.c_double), ("step_length", ctypes.c_double),
        ("solve_time", ctypes.c_double),
        ("ir_solves", ctypes.c_int), ("ir_sweeps", ctypes.c_int),
        ("ir_unconverged", ctypes.c_int), ("ir_worst_ratio", ctypes.c_double),
    ]


def build():
    """Compile liboracle.so in place (g++ only)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        vp = ctypes.c_void_p
        L.oracle_default_settings.argtypes = [ctypes.POINTER(OracleSettings)]
        L.oracle_solve.argtypes = [
            ctypes.c_int, ctypes.c_int, ip, ip, dp, dp, ip, ip, dp, dp,
            ctypes.c_int, ip, ip, dp, ctypes.POINTER(OracleSettings), dp, dp,
            dp, ctypes.POINTER(OracleInfo)]
        L.oracle_solve.restype = ctypes.c_int
        L.oracle_solver_create.argtypes = [
            ctypes.c_int, ctypes.c_int, ip, ip, dp, dp, ip, ip, dp, dp,
            ctypes.c_int, ip, ip, dp, ctypes.POINTER(OracleSettings)]
        L.oracle_solver_create.restype = vp
        L.oracle_solver_run.argtypes = [vp, dp, dp, dp, ctypes.POINTER(OracleInfo)]
        L.oracle_solver_run.restype = ctypes.c_int
        L.oracle_solver_destroy.argtypes = [vp]
        L.oracle_cones_create.argtypes = [ctypes.c_int, ip, ip, dp]
        L.oracle_cones_create.restype = vp
        L.oracle_cones_destroy.argtypes = [vp]
        for f in ("oracle_cones_numel", "oracle_cones_degree", "oracle_cones_hs_len"):
            getattr(L, f).argtypes = [vp]
            getattr(L, f).restype = ctypes.c_int
        L.oracle_update_scaling.argtypes = [vp, dp, dp, ctypes.c_double, ctypes.c_int]
        L.oracle_update_scaling.restype = ctypes.c_int
        L.oracle_set_identity_scaling.argtypes = [vp]
        L.oracle_get_Hs.argtypes = [vp, dp]
        L.oracle_mul_Hs.argtypes = [vp, dp, dp]
        L.oracle_affine_ds.argtypes = [vp, dp, dp]
        L.oracle_combined_ds_shift.argtypes = [vp, dp, dp, dp, dp, ctypes.c_double]
        L.oracle_ds_from_dz_offset.argtypes = [vp, dp, dp, dp]
        L.oracle_step_length.argtypes = [vp, dp, dp, dp, dp] + [ctypes.c_double] * 4
        L.oracle_step_length.restype = ctypes.c_double
        L.oracle_compute_barrier.argtypes = [vp, dp, dp, dp, dp, ctypes.c_double]
        L.oracle_compute_barrier.restype = ctypes.c_double
        L.oracle_margins.argtypes = [vp, dp, ctypes.c_int, dp, dp]
        L.oracle_scaled_unit_shift.argtypes = [vp, dp, ctypes.c_double, ctypes.c_int]
        L.oracle_unit_initialization.argtypes = [vp, dp, dp]
        L.oracle_get_state.argtypes = [vp, ctypes.c_int, dp]
        L.oracle_get_state.restype = ctypes.c_int
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def cone_arrays(cones):
    specs = [c.spec() if hasattr(c, "spec") else tuple(c) for c in cones]
    t = np.array([s[0] for s in specs], dtype=np.int32)
    d = np.array([s[1] for s in specs], dtype=np.int32)
    p = np.array([float(s[2]) if len(s) > 2 else 0.0 for s in specs], dtype=np.float64)
    return t, d, p


def default_settings(**kw):
    st = OracleSettings()
    lib().oracle_default_settings(ctypes.byref(st))
    for k, v in kw.items():
        setattr(st, k, v)
    return st


def _arrays(P, q, A, b, cones):
    n = len(q)
    m = len(b)
    P = sp.csc_matrix(P, shape=(n, n))
    P = sp.triu(P, format="csc")
    P.sort_indices()
    A = sp.csc_matrix(A, shape=(m, n))
    A.sort_indices()
    t, d, p = cone_arrays(cones)
    return (n, m, np.ascontiguousarray(P.indptr, np.int32),
            np.ascontiguousarray(P.indices, np.int32), np.ascontiguousarray(P.data, np.float64),
            np.ascontiguousarray(q, np.float64), np.ascontiguousarray(A.indptr, np.int32),
            np.ascontiguousarray(A.indices, np.int32), np.ascontiguousarray(A.data, np.float64),
            np.ascontiguousarray(b, np.float64), t, d, p)


class SolverObject:
    """Setup once, solve repeatedly (Solver(...) then solve!, the CPU path of
    src/solver.jl); each run starts from the default initial point."""

    def __init__(self, P, q, A, b, cones, **settings):
        self._a = _arrays(P, q, A, b, cones)
        n, m, Pp, Pi, Px, q, Ap, Ai, Ax, b, t, d, p = self._a
        self.n, self.m = n, m
        st = default_settings(**settings)
        self.h = lib().oracle_solver_create(n, m, _ip(Pp), _ip(Pi), _dp(Px), _dp(q), _ip(Ap),
                                            _ip(Ai), _dp(Ax), _dp(b), len(t), _ip(t), _ip(d),
                                            _dp(p), ctypes.byref(st))
        if not self.h:
            raise RuntimeError("oracle_solver_create failed")
        self._x, self._s, self._z = np.zeros(n), np.zeros(m), np.zeros(m)

    def run(self):
        info = OracleInfo()
        rc = lib().oracle_solver_run(self.h, _dp(self._x), _dp(self._s), _dp(self._z),
                                     ctypes.byref(info))
        if rc != 0:
            raise RuntimeError("oracle_solver_run failed with code %d" % rc)
        out = {f: getattr(info, f) for f, _ in OracleInfo._fields_}
        out.update(x=self._x.copy(), s=self._s.copy(), z=self._z.copy(),
                   status_name=STATUS_NAMES[info.status])
        return out

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().oracle_solver_destroy(h)
            self.h = None


def solve(P, q, A, b, cones, **settings):
    """Solve with the CPU oracle.  Returns dict(x, s, z, info-fields...)."""
    n = len(q)
    m = len(b)
    P = sp.csc_matrix(P, shape=(n, n))
    P = sp.triu(P, format="csc")
    P.sort_indices()
    A = sp.csc_matrix(A, shape=(m, n))
    A.sort_indices()
    Pp, Pi, Px = (np.ascontiguousarray(P.indptr, np.int32),
                  np.ascontiguousarray(P.indices, np.int32),
                  np.ascontiguousarray(P.data, np.float64))
    Ap, Ai, Ax = (np.ascontiguousarray(A.indptr, np.int32),
                  np.ascontiguousarray(A.indices, np.int32),
                  np.ascontiguousarray(A.data, np.float64))
    q = np.ascontiguousarray(q, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    t, d, p = cone_arrays(cones)
    st = default_settings(**settings)
    x = np.zeros(n)
    s = np.zeros(m)
    z = np.zeros(m)
    info = OracleInfo()
    rc = lib().oracle_solve(n, m, _ip(Pp), _ip(Pi), _dp(Px), _dp(q), _ip(Ap),
                            _ip(Ai), _dp(Ax), _dp(b), len(t), _ip(t), _ip(d),
                            _dp(p), ctypes.byref(st), _dp(x), _dp(s), _dp(z),
                            ctypes.byref(info))
    if rc != 0:
        raise RuntimeError("oracle_solve failed with code %d" % rc)
    out = {f: getattr(info, f) for f, _ in OracleInfo._fields_}
    out.update(x=x, s=s, z=z, status_name=STATUS_NAMES[info.status])
    return out


class Cones:
    """Composite cone handle for per-operation parity checks."""

    def __init__(self, cones):
        t, d, p = cone_arrays(cones)
        self._keep = (t, d, p)
        self.h = lib().oracle_cones_create(len(t), _ip(t), _ip(d), _dp(p))
        self.numel = lib().oracle_cones_numel(self.h)
        self.degree = lib().oracle_cones_degree(self.h)
        self.hs_len = lib().oracle_cones_hs_len(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_cones_destroy(self.h)
            self.h = None

    def update_scaling(self, s, z, mu, strategy=0):
        s = np.ascontiguousarray(s, np.float64)
        z = np.ascontiguousarray(z, np.float64)
        return lib().oracle_update_scaling(self.h, _dp(s), _dp(z), mu, strategy)

    def set_identity_scaling(self):
        lib().oracle_set_identity_scaling(self.h)

    def get_Hs(self):
        out = np.zeros(self.hs_len)
        lib().oracle_get_Hs(self.h, _dp(out))
        return out

    def mul_Hs(self, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.numel)
        lib().oracle_mul_Hs(self.h, _dp(y), _dp(x))
        return y

    def affine_ds(self, s):
        s = np.ascontiguousarray(s, np.float64)
        ds = np.zeros(self.numel)
        lib().oracle_affine_ds(self.h, _dp(ds), _dp(s))
        return ds

    def combined_ds_shift(self, step_z, step_s, z, sigma_mu):
        step_z = np.array(step_z, np.float64)
        step_s = np.array(step_s, np.float64)
        z = np.ascontiguousarray(z, np.float64)
        shift = np.zeros(self.numel)
        lib().oracle_combined_ds_shift(self.h, _dp(shift), _dp(step_z), _dp(step_s),
                                       _dp(z), sigma_mu)
        return shift

    def ds_from_dz_offset(self, ds, z):
        ds = np.ascontiguousarray(ds, np.float64)
        z = np.ascontiguousarray(z, np.float64)
        out = np.zeros(self.numel)
        lib().oracle_ds_from_dz_offset(self.h, _dp(out), _dp(ds), _dp(z))
        return out

    def step_length(self, dz, ds, z, s, alpha_max, max_step_fraction=0.99,
                    backtrack=0.8, alpha_min=1e-4):
        a = [np.ascontiguousarray(v, np.float64) for v in (dz, ds, z, s)]
        return lib().oracle_step_length(self.h, *[_dp(v) for v in a], alpha_max,
                                        max_step_fraction, backtrack, alpha_min)

    def compute_barrier(self, z, s, dz, ds, alpha):
        a = [np.ascontiguousarray(v, np.float64) for v in (z, s, dz, ds)]
        return lib().oracle_compute_barrier(self.h, *[_dp(v) for v in a], alpha)

    def margins(self, z, pd):
        z = np.ascontiguousarray(z, np.float64)
        a = np.zeros(1)
        b = np.zeros(1)
        lib().oracle_margins(self.h, _dp(z), pd, _dp(a), _dp(b))
        return a[0], b[0]

    def scaled_unit_shift(self, z, alpha, pd):
        z = np.array(z, np.float64)
        lib().oracle_scaled_unit_shift(self.h, _dp(z), alpha, pd)
        return z

    def unit_initialization(self):
        z = np.zeros(self.numel)
        s = np.zeros(self.numel)
        lib().oracle_unit_initialization(self.h, _dp(z), _dp(s))
        return z, s

    def state(self, which, size):
        out = np.zeros(size)
        k = lib().oracle_get_state(self.h, which, _dp(out))
        return out[:k]
