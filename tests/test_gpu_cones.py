"""Per-operation parity of the cone kernels (cone-level C ABI, device
pointers) against the CPU oracle's restatement of src/cones/*.jl."""
import ctypes

import numpy as np
import pytest

import oracle
from cuclarabel_b200 import _lib

pytestmark = pytest.mark.gpu
TOL = 1e-12  # relative, FP64 cone arithmetic


def interior(rng, spec, scale=1.0):
    t, d, p = spec
    if t == 0:
        return rng.standard_normal(d) * scale
    if t == 1:
        return rng.uniform(0.5, 2, d)
    if t == 2:
        tail = rng.standard_normal(d - 1)
        return np.concatenate([[1.0 + np.linalg.norm(tail) * rng.uniform(1.05, 2)], tail])
    if t == 3:
        return np.array([-1.051383945322714, 0.556409619469370, 1.258967884768947]) * \
            rng.uniform(0.5, 2) + rng.normal(0, 0.02, 3)
    if t == 4:
        return np.array([np.sqrt(1 + p), np.sqrt(2 - p), 0.0]) * rng.uniform(0.5, 2) + \
            np.array([0, 0, rng.normal(0, 0.1)])
    # off-diagonal noise shrinks with the side so the matrix stays positive
    # definite (semicircle radius about 0.6 at every side)
    E = rng.standard_normal((d, d)) * (0.2 if d <= 10 else 0.6 / np.sqrt(d))
    M = np.eye(d) + (E + E.T) / 2
    out = []
    for j in range(d):
        for i in range(j + 1):
            out.append(M[i, j] if i == j else M[i, j] * np.sqrt(2))
    return np.array(out)


SPECS = {
    "nn": [(1, 7, 0.0)],
    "soc_dense": [(2, 3, 0.0), (2, 5, 0.0), (2, 4, 0.0)],
    "soc_sparse": [(2, 10, 0.0), (2, 6, 0.0), (2, 40, 0.0)],
    "exp": [(3, 3, 0.0)] * 5,
    "pow": [(4, 3, 0.3), (4, 3, 0.7), (4, 3, 0.55)],
    "psd": [(5, 3, 0.0), (5, 10, 0.0)],
    # sides above one warp's 32 lanes (row loops in the warp kernels) and
    # mixed sides in one launch
    "psd_large": [(5, 20, 0.0), (5, 33, 0.0), (5, 40, 0.0), (5, 7, 0.0)],
    "mixed": [(0, 2, 0.0), (1, 4, 0.0), (2, 3, 0.0), (2, 8, 0.0), (3, 3, 0.0), (4, 3, 0.4),
              (5, 4, 0.0)],
    # several shared-memory tiles of small cones (at most 128 cones or 1024
    # rows each), broken by cones above the tile limit (dim > 16)
    "soc_tiles": [(2, int(d), 0.0) for d in
                  np.random.default_rng(42).choice([2, 3, 5, 8, 10, 13, 16, 17, 24, 33],
                                                   size=300,
                                                   p=[.1, .15, .15, .15, .1, .1, .1, .05,
                                                      .05, .05])],
}


class GPUCones:
    def __init__(self, specs):
        import torch
        self.torch = torch
        self.L = _lib.load()
        t = np.array([s[0] for s in specs], np.int32)
        d = np.array([s[1] for s in specs], np.int32)
        p = np.array([s[2] for s in specs], np.float64)
        h = ctypes.c_void_p()
        rc = self.L.clgpu_cones_create(len(t), t.ctypes.data_as(_lib.ip),
                                       d.ctypes.data_as(_lib.ip), p.ctypes.data_as(_lib.dp), 5,
                                       ctypes.byref(h))
        assert rc == 0
        self.h = h
        self.numel = self.L.clgpu_cones_numel(h)
        self.hs_len = self.L.clgpu_cones_hs_len(h)

    def dev(self, a):
        return self.torch.tensor(np.asarray(a, np.float64), device="cuda")

    def empty(self, n):
        return self.torch.zeros(max(n, 1), dtype=self.torch.float64, device="cuda")

    def __del__(self):
        self.L.clgpu_cones_destroy(self.h)


def setup(name, seed=0):
    specs = SPECS[name]
    rng = np.random.default_rng(seed)
    s = np.concatenate([interior(rng, sp) for sp in specs])
    z = np.concatenate([interior(rng, sp) for sp in specs])
    return specs, rng, s, z


def close(a, b, tol=TOL):
    a, b = np.asarray(a), np.asarray(b)
    return np.allclose(a, b, rtol=tol, atol=tol * max(1.0, np.abs(b).max(initial=0)))


@pytest.mark.parametrize("name", list(SPECS))
@pytest.mark.parametrize("strategy", [0, 1])
def test_update_scaling_hs_and_products(cuda_device, name, strategy):
    specs, rng, s, z = setup(name)
    mu = float(s @ z / 10)
    C = oracle.Cones(specs)
    G = GPUCones(specs)
    assert C.update_scaling(s, z, mu, strategy) == 0
    ds_, dz_ = G.dev(s), G.dev(z)
    assert G.L.clgpu_update_scaling(G.h, ds_.data_ptr(), dz_.data_ptr(), mu, strategy, None) == 0
    # Hs blocks (invariant to the SVD sign choices of the PSD scaling)
    hs = G.empty(G.hs_len)
    assert G.L.clgpu_get_Hs(G.h, hs.data_ptr(), None) == 0
    assert close(hs.cpu().numpy()[:C.hs_len], C.get_Hs(), 1e-11)
    # mul_Hs
    x = rng.standard_normal(C.numel)
    y = G.empty(C.numel)
    d_x = G.dev(x)
    assert G.L.clgpu_mul_Hs(G.h, y.data_ptr(), d_x.data_ptr(), None) == 0
    assert close(y.cpu().numpy(), C.mul_Hs(x), 1e-11)
    # affine_ds
    out = G.empty(C.numel)
    assert G.L.clgpu_affine_ds(G.h, out.data_ptr(), ds_.data_ptr(), None) == 0
    assert close(out.cpu().numpy(), C.affine_ds(s), 1e-11)
    # combined_ds_shift
    stz, sts = rng.standard_normal(C.numel) * 0.1, rng.standard_normal(C.numel) * 0.1
    sm = 0.37 * mu
    sh = G.empty(C.numel)
    d_stz, d_sts = G.dev(stz), G.dev(sts)
    assert G.L.clgpu_combined_ds_shift(G.h, sh.data_ptr(), d_stz.data_ptr(),
                                       d_sts.data_ptr(), dz_.data_ptr(), sm, None) == 0
    assert close(sh.cpu().numpy(), C.combined_ds_shift(stz, sts, z, sm), 1e-10)
    # ds_from_dz_offset
    dsv = rng.standard_normal(C.numel)
    o = G.empty(C.numel)
    d_dsv = G.dev(dsv)
    assert G.L.clgpu_ds_from_dz_offset(G.h, o.data_ptr(), d_dsv.data_ptr(),
                                       dz_.data_ptr(), None) == 0
    assert close(o.cpu().numpy(), C.ds_from_dz_offset(dsv, z), 1e-10)


@pytest.mark.parametrize("name", list(SPECS))
def test_step_length_and_barrier(cuda_device, name):
    specs, rng, s, z = setup(name, seed=3)
    C = oracle.Cones(specs)
    G = GPUCones(specs)
    C.update_scaling(s, z, 1.0, 0)
    d_s, d_z = G.dev(s), G.dev(z)
    G.L.clgpu_update_scaling(G.h, d_s.data_ptr(), d_z.data_ptr(), 1.0, 0, None)
    for trial in range(4):
        dz = rng.standard_normal(C.numel) * (0.5 + trial)
        ds = rng.standard_normal(C.numel) * (0.5 + trial)
        ref = C.step_length(dz, ds, z, s, 1.0)
        a = ctypes.c_double()
        d_dz, d_ds = G.dev(dz), G.dev(ds)
        assert G.L.clgpu_step_length(G.h, d_dz.data_ptr(), d_ds.data_ptr(),
                                     d_z.data_ptr(), d_s.data_ptr(), 1.0, 0.99, 0.8,
                                     1e-4, ctypes.byref(a), None) == 0
        assert abs(a.value - ref) <= 1e-10 * max(1.0, ref), (a.value, ref)
        alpha = 0.5 * ref
        bref = C.compute_barrier(z, s, dz, ds, alpha)
        bar = ctypes.c_double()
        assert G.L.clgpu_compute_barrier(G.h, d_z.data_ptr(), d_s.data_ptr(),
                                         d_dz.data_ptr(), d_ds.data_ptr(), alpha,
                                         ctypes.byref(bar), None) == 0
        assert abs(bar.value - bref) <= 1e-9 * max(1.0, abs(bref))


@pytest.mark.parametrize("name", ["nn", "soc_dense", "soc_sparse", "psd", "psd_large"])
def test_margins_shift_and_init(cuda_device, name):
    specs, rng, s, z = setup(name, seed=5)
    C = oracle.Cones(specs)
    G = GPUCones(specs)
    v = rng.standard_normal(C.numel)
    for pd in (0, 1):
        a, b = ctypes.c_double(), ctypes.c_double()
        d_v = G.dev(v)
        assert G.L.clgpu_margins(G.h, d_v.data_ptr(), pd, ctypes.byref(a), ctypes.byref(b),
                                 None) == 0
        ra, rb = C.margins(v, pd)
        assert abs(a.value - ra) < 1e-11 and abs(b.value - rb) < 1e-10
        t = G.dev(v)
        assert G.L.clgpu_scaled_unit_shift(G.h, t.data_ptr(), 0.75, pd, None) == 0
        assert close(t.cpu().numpy(), C.scaled_unit_shift(v, 0.75, pd), 1e-14)
    zz, ss = G.empty(C.numel), G.empty(C.numel)
    assert G.L.clgpu_unit_initialization(G.h, zz.data_ptr(), ss.data_ptr(), None) == 0
    rz, rs = C.unit_initialization()
    assert close(zz.cpu().numpy(), rz, 1e-15) and close(ss.cpu().numpy(), rs, 1e-15)


def test_scaling_failure_reported(cuda_device):
    """A point outside the cone is reported as a numerical failure (return 1),
    as the CPU path's update_scaling! does (coneops_socone.jl:385-387)."""
    specs = [(2, 4, 0.0)]
    G = GPUCones(specs)
    s = np.array([0.1, 1.0, 0.0, 0.0])  # not interior
    z = np.array([2.0, 0.1, 0.1, 0.1])
    d_s, d_z = G.dev(s), G.dev(z)
    assert G.L.clgpu_update_scaling(G.h, d_s.data_ptr(), d_z.data_ptr(), 1.0, 0, None) == 1


def test_kernel_time_profiling_leaves_results_unchanged(cuda_device):
    """With profiling on, an operation reports a positive kernel time and
    writes the same values as without profiling."""
    specs, rng, s, z = setup("mixed", seed=11)
    G = GPUCones(specs)
    d_s, d_z = G.dev(s), G.dev(z)
    x = G.dev(rng.standard_normal(G.numel))
    outs = []
    for prof in (0, 1):
        assert G.L.clgpu_cones_set_profiling(G.h, prof) == 0
        assert G.L.clgpu_update_scaling(G.h, d_s.data_ptr(), d_z.data_ptr(), 1.0, 0, None) == 0
        y = G.empty(G.numel)
        assert G.L.clgpu_mul_Hs(G.h, y.data_ptr(), x.data_ptr(), None) == 0
        ms = ctypes.c_double(-1.0)
        assert G.L.clgpu_cones_last_kernel_ms(G.h, ctypes.byref(ms)) == 0
        assert (ms.value > 0) if prof else (ms.value == 0.0)
        outs.append(y.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("name", ["soc_tiles", "soc_sparse", "mixed", "nn"])
def test_launch_shapes_give_identical_results(cuda_device, name):
    """Every launch shape the autotuner may pick (lane groups or tiles of
    32 / 64 / 128 cones for the SOC operations, 64..512 threads per block for
    the nonnegative kernels) returns the same bits."""
    specs, rng, s, z = setup(name, seed=7)
    G = GPUCones(specs)
    m = G.numel
    d_s, d_z = G.dev(s), G.dev(z)
    dz, ds = G.dev(rng.standard_normal(m) * 0.3), G.dev(rng.standard_normal(m) * 0.3)
    x = G.dev(rng.standard_normal(m))
    runs = []
    for v, nb in [(0, 128), (1, 256), (2, 512), (3, 64)]:
        assert G.L.clgpu_cones_set_launch_shapes(G.h, nb, (ctypes.c_int * 6)(*[v] * 6)) == 0
        nbo, vo = ctypes.c_int(), (ctypes.c_int * 6)()
        assert G.L.clgpu_cones_get_launch_shapes(G.h, ctypes.byref(nbo), vo) == 0
        assert nbo.value == nb and list(vo) == [v] * 6
        out = {}
        assert G.L.clgpu_update_scaling(G.h, d_s.data_ptr(), d_z.data_ptr(), 1.0, 0, None) == 0
        hs = G.empty(G.hs_len)
        assert G.L.clgpu_get_Hs(G.h, hs.data_ptr(), None) == 0
        out["Hs"] = hs.cpu().numpy()
        for key, call in (
                ("mul_Hs", lambda y: G.L.clgpu_mul_Hs(G.h, y.data_ptr(), x.data_ptr(), None)),
                ("affine_ds", lambda y: G.L.clgpu_affine_ds(G.h, y.data_ptr(), d_s.data_ptr(),
                                                            None)),
                ("combined", lambda y: G.L.clgpu_combined_ds_shift(
                    G.h, y.data_ptr(), dz.data_ptr(), ds.data_ptr(), d_z.data_ptr(), 0.05, None)),
                ("ds_offset", lambda y: G.L.clgpu_ds_from_dz_offset(
                    G.h, y.data_ptr(), ds.data_ptr(), d_z.data_ptr(), None))):
            y = G.empty(m)
            assert call(y) == 0
            out[key] = y.cpu().numpy()
        a = ctypes.c_double()
        assert G.L.clgpu_step_length(G.h, dz.data_ptr(), ds.data_ptr(), d_z.data_ptr(),
                                     d_s.data_ptr(), 1.0, 0.99, 0.8, 1e-4, ctypes.byref(a),
                                     None) == 0
        out["alpha"] = np.array([a.value])
        runs.append(out)
    for r in runs[1:]:
        for k, v in r.items():
            assert np.array_equal(v.view(np.uint64), runs[0][k].view(np.uint64)), k
    assert G.L.clgpu_cones_set_launch_shapes(G.h, 48, None) == -1
    assert G.L.clgpu_cones_set_launch_shapes(G.h, 0, (ctypes.c_int * 6)(0, 0, 4, 0, 0, 0)) == -1
