"""clgpu_margins_static: the handle-free margins entry point whose scratch is
a static device array.  It must return exactly what clgpu_margins returns on
a handle built from the same cones, on consecutive calls (no state carried
from one call to the next), and reject layouts above its fixed capacity.

The file name sorts last so the entry point is also exercised after every
other GPU test has run in the same process."""
import ctypes

import numpy as np
import pytest

from cuclarabel_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_CONES = 32768        # CLGPU_MARGINS_STATIC_MAX_CONES
ERR_TOO_LARGE = -20      # CLGPU_ERR_STATIC_TOO_LARGE

LAYOUTS = {
    "mixed": [(0, 2, 0.0), (1, 5, 0.0), (2, 3, 0.0), (2, 8, 0.0), (3, 3, 0.0), (4, 3, 0.4),
              (5, 4, 0.0), (5, 0, 0.0), (5, 3, 0.0)],
    "many_soc": [(1, 40, 0.0)] + [(2, 3 + (k % 9), 0.0) for k in range(300)],
    "psd_only": [(5, 10, 0.0), (5, 2, 0.0), (5, 16, 0.0)],
    "nn_only": [(1, 1000, 0.0)],
}


def _rows(spec):
    t, d, _ = spec
    return 3 if t in (3, 4) else (d * (d + 1) // 2 if t == 5 else d)


def _arrays(specs):
    t = np.array([s[0] for s in specs], np.int32)
    d = np.array([s[1] for s in specs], np.int32)
    p = np.array([s[2] for s in specs], np.float64)
    return t, d, p


def _handle_margins(L, specs, zt, pd):
    t, d, p = _arrays(specs)
    h = ctypes.c_void_p()
    assert L.clgpu_cones_create(len(t), t.ctypes.data_as(_lib.ip), d.ctypes.data_as(_lib.ip),
                                p.ctypes.data_as(_lib.dp), 5, ctypes.byref(h)) == 0
    a, b = ctypes.c_double(), ctypes.c_double()
    try:
        assert L.clgpu_margins(h, zt.data_ptr(), pd, ctypes.byref(a), ctypes.byref(b),
                               None) == 0
    finally:
        L.clgpu_cones_destroy(h)
    return a.value, b.value


def _static_margins(L, specs, zt, pd, stream):
    t, d, _ = _arrays(specs)
    a, b = ctypes.c_double(), ctypes.c_double()
    rc = L.clgpu_margins_static(len(t), t.ctypes.data_as(_lib.ip), d.ctypes.data_as(_lib.ip),
                                zt.data_ptr(), pd, ctypes.byref(a), ctypes.byref(b), stream)
    assert rc == 0, rc
    return a.value, b.value


@pytest.mark.parametrize("name", list(LAYOUTS))
def test_static_margins_match_handle_margins(cuda_device, name):
    import torch
    L = _lib.load()
    specs = LAYOUTS[name]
    m = sum(_rows(s) for s in specs)
    rng = np.random.default_rng(11)
    stream = torch.cuda.current_stream().cuda_stream
    # two different vectors, each checked on two calls in a row
    for trial in range(2):
        z = rng.standard_normal(m) * (1.0 + trial)
        zt = torch.tensor(z, dtype=torch.float64, device="cuda")
        for pd in (0, 1):
            ref = _handle_margins(L, specs, zt, pd)
            first = _static_margins(L, specs, zt, pd, stream)
            second = _static_margins(L, specs, zt, pd, stream)
            assert first == ref, (name, trial, pd, first, ref)
            assert second == ref, (name, trial, pd, second, ref)


def test_static_margins_layout_change_between_calls(cuda_device):
    """A larger layout followed by a smaller one: the second call must not
    see the first call's cones."""
    import torch
    L = _lib.load()
    big, small = LAYOUTS["many_soc"], LAYOUTS["mixed"]
    rng = np.random.default_rng(5)
    zb = torch.tensor(rng.standard_normal(sum(_rows(s) for s in big)), dtype=torch.float64,
                      device="cuda")
    zs = torch.tensor(rng.standard_normal(sum(_rows(s) for s in small)), dtype=torch.float64,
                      device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert _static_margins(L, big, zb, 0, stream) == _handle_margins(L, big, zb, 0)
    assert _static_margins(L, small, zs, 0, stream) == _handle_margins(L, small, zs, 0)
    assert _static_margins(L, big, zb, 1, stream) == _handle_margins(L, big, zb, 1)


def test_static_margins_rejects_oversize_layout(cuda_device):
    import torch
    L = _lib.load()
    n = MAX_CONES + 1
    t = np.full(n, 2, np.int32)
    d = np.full(n, 3, np.int32)
    zt = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    a, b = ctypes.c_double(-7.0), ctypes.c_double(-7.0)
    rc = L.clgpu_margins_static(n, t.ctypes.data_as(_lib.ip), d.ctypes.data_as(_lib.ip),
                                zt.data_ptr(), 0, ctypes.byref(a), ctypes.byref(b), None)
    assert rc == ERR_TOO_LARGE
    assert a.value == -7.0 and b.value == -7.0  # outputs untouched on rejection
    # exactly at the limit is accepted
    t, d = t[:MAX_CONES], d[:MAX_CONES]
    rc = L.clgpu_margins_static(MAX_CONES, t.ctypes.data_as(_lib.ip), d.ctypes.data_as(_lib.ip),
                                zt.data_ptr(), 0, ctypes.byref(a), ctypes.byref(b), None)
    assert rc == 0
    assert a.value == 0.0 and b.value == 0.0  # z = 0: every SOC margin is 0


def test_empty_psd_cone_leaves_margins_unchanged(cuda_device):
    """An empty PSD cone contributes (floatmax, 0) (the reference's
    coneops_psdtrianglecone.jl:16-19), so inserting one changes neither
    margin -- also right after a call that left other values in the shared
    scratch slot the empty cone occupies."""
    import torch
    L = _lib.load()
    with_empty = [(1, 3, 0.0), (5, 3, 0.0), (5, 0, 0.0), (5, 2, 0.0)]
    without = [(1, 3, 0.0), (5, 3, 0.0), (5, 2, 0.0)]
    rng = np.random.default_rng(9)
    z = torch.tensor(rng.standard_normal(sum(_rows(s) for s in without)), dtype=torch.float64,
                     device="cuda")
    zp = torch.tensor(rng.standard_normal(sum(_rows(s) for s in LAYOUTS["psd_only"])),
                      dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for pd in (0, 1):
        _static_margins(L, LAYOUTS["psd_only"], zp, pd, stream)  # leaves PSD values behind
        ref = _handle_margins(L, without, z, pd)
        assert _static_margins(L, with_empty, z, pd, stream) == ref
        assert _handle_margins(L, with_empty, z, pd) == ref
