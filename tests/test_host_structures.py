"""Host-side validation of the per-instance structures the device kernels
read (ordering, symbolic LDL^T, refresh maps): the library replays the
left-looking factorisation on the CPU and solves a test system.  No GPU."""
import ctypes

import numpy as np
import pytest

from cuclarabel_b200 import _lib, problems
from cuclarabel_b200.api import Settings, _prep_problem
from helpers import golden_cases, to_cone_objects


def check(pb, **kw):
    cp, keep, n, m = _prep_problem(*pb)
    st = Settings(**kw).to_c()
    r = ctypes.c_double()
    rc = _lib.load().clgpu_debug_check_instance(ctypes.byref(cp), ctypes.byref(st),
                                                ctypes.byref(r))
    return rc, r.value


@pytest.mark.parametrize("case", golden_cases(), ids=[c[0] for c in golden_cases()])
def test_golden_structures(case):
    name, P, q, A, b, cones, e = case
    rc, res = check((P, q, A, b, to_cone_objects(cones)))
    assert rc == 0 and res < 1e-10


@pytest.mark.parametrize("seed", range(12))
def test_mpc_structures(seed):
    rc, res = check(problems.mpc_qp(seed))
    assert rc == 0 and res < 1e-9


def test_config_families():
    for pb in (problems.portfolio(), problems.mixed_socp(0.01), problems.exp_pow_psd(0.003)):
        rc, res = check(pb)
        assert rc == 0 and res < 1e-9
    # dense SOC path (threshold above every cone)
    rc, res = check(problems.mpc_qp(3), soc_threshold=100)
    assert rc == 0 and res < 1e-9


@pytest.mark.parametrize("side,ncones", [(24, 3), (40, 2)])
def test_psd_block_structures(side, ncones):
    """Dense PSD blocks: side 40 fills the factor beyond the single-warp
    streams' range and is prepared for the supernodal factorisation."""
    rc, res = check(problems.psd_lp(side, ncones, seed=0))
    assert rc == 0 and res < 1e-9


def _path(pb):
    cp, keep, n, m = _prep_problem(*pb)
    st = Settings().to_c()
    sn, ent = ctypes.c_int(), ctypes.c_longlong()
    rc = _lib.load().clgpu_debug_instance_path(ctypes.byref(cp), ctypes.byref(st),
                                               ctypes.byref(sn), ctypes.byref(ent))
    assert rc == 0
    return sn.value, ent.value


def test_factorisation_paths():
    """Sparse factors stay on the single-warp kernels (the bench batch's
    instances, every 64th of the 4096 here), dense fronts take the
    supernodal path: linear SDPs whose PSD blocks reach side 24 to 40 with
    three or fewer blocks coupled by equality rows (factor columns of 500+
    entries) and the large configurations."""
    for seed in range(0, 4096, 64):
        sn, ent = _path(problems.mpc_qp(seed))
        assert sn == 0, seed
    assert _path(problems.psd_lp(20, 3, seed=0))[0] == 0
    assert _path(problems.psd_lp(24, 3, seed=0))[0] == 1
    assert _path(problems.psd_lp(32, 3, seed=0))[0] == 1
    assert _path(problems.psd_lp(36, 2, seed=0))[0] == 1
    assert _path(problems.psd_lp(40, 1, seed=0))[0] == 1
    assert _path(problems.mixed_socp(0.1))[0] == 1


def replay(pb, **kw):
    cp, keep, n, m = _prep_problem(*pb)
    st = Settings(**kw).to_c()
    r = ctypes.c_double()
    rc = _lib.load().clgpu_debug_factor_stream(ctypes.byref(cp), ctypes.byref(st),
                                               ctypes.byref(r))
    return rc, r.value


@pytest.mark.parametrize("seed", range(8))
def test_factor_op_stream_replays_to_the_dense_factor(seed):
    """The streamed factorisation's op stream (8-byte records: four 14-bit
    work-vector positions, segment position, last bit), replayed on the host
    in the kernel's schedule, gives the L and D of a dense LDL^T of the same
    permuted matrix."""
    rc, res = replay(problems.mpc_qp(seed))
    assert rc == 0 and res < 1e-12, (rc, res)


def test_factor_op_stream_other_families():
    pbs = [problems.portfolio()]
    for name, P, q, A, b, cones, e in golden_cases()[:6]:
        pbs.append((P, q, A, b, to_cone_objects(cones)))
    for pb in pbs:
        rc, res = replay(pb)
        assert rc == 0 and res < 1e-12, (rc, res)
