"""Numeric setup on the device (data_equilibrate!, GPU form,
src/problemdata.jl:286-374, and the KKT value assembly of
directgpu_kkt_assembly.jl:69-170): with device_setup = 1 the Ruiz
equilibration, cost scaling, rectification and the KKT values are computed
by kernels; they must equal the host setup's (device_setup = 0) bit for bit,
and so must every solve."""
import ctypes

import numpy as np
import pytest

from cuclarabel_b200 import BatchSolver, Solver, _lib, problems

pytestmark = pytest.mark.gpu


def _setup_arrays(solver):
    L = _lib.load()
    B = len(solver.dims)
    nnz = ctypes.c_longlong()
    assert L.clgpu_solver_debug_setup(solver._h, None, None, None, None, None, None,
                                      ctypes.byref(nnz)) == 0
    out = {k: np.zeros(n) for k, n in (("d", solver.nx), ("e", solver.mz), ("c", B),
                                       ("q", solver.nx), ("b", solver.mz),
                                       ("Kx", nnz.value))}
    dp = lambda a: a.ctypes.data_as(_lib.dp)
    assert L.clgpu_solver_debug_setup(solver._h, dp(out["d"]), dp(out["e"]), dp(out["c"]),
                                      dp(out["q"]), dp(out["b"]), dp(out["Kx"]), None) == 0
    return out


FAMILIES = {
    "mpc_batch": lambda: problems.mpc_batch(64, seed0=70),
    "portfolio": lambda: [problems.portfolio(seed=1)],
    "exp_pow_psd": lambda: [problems.exp_pow_psd(scale=0.004, seed=3)],
    "mixed_socp_supernodal": lambda: [problems.mixed_socp(scale=0.08, seed=4)],
}


@pytest.mark.parametrize("family", list(FAMILIES))
def test_device_setup_equals_host_setup_bitwise(cuda_device, family):
    pbs = FAMILIES[family]()
    dev = BatchSolver(pbs, device_setup=True)
    host = BatchSolver(pbs, device_setup=False)
    a, b = _setup_arrays(dev), _setup_arrays(host)
    for k in a:
        assert np.array_equal(a[k], b[k]), (family, k, np.abs(a[k] - b[k]).max())
    ra, rb = dev.solve(), host.solve()
    for x, y in zip(ra, rb):
        assert x.status == y.status and x.iterations == y.iterations
        assert np.array_equal(x.x, y.x) and np.array_equal(x.z, y.z)


def test_device_setup_with_equilibration_off(cuda_device):
    pbs = problems.mpc_batch(8, seed0=3)
    a = _setup_arrays(BatchSolver(pbs, device_setup=True, equilibrate_enable=False))
    b = _setup_arrays(BatchSolver(pbs, device_setup=False, equilibrate_enable=False))
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert np.all(a["d"] == 1.0) and np.all(a["e"] == 1.0) and np.all(a["c"] == 1.0)
