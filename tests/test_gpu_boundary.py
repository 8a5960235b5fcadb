"""The KKT- and variable-level C ABI a Julia solve! keeps its own loop
around: mul_Hs_diag!, rectify_equilibration!, the Hs -> KKT refresh, a
step_length that leaves alpha on the device, the LDL solver protocol
(regularise + refactor, refined solve), residuals_update! and
variables_add_step!.

The cone-level additions are checked against the library's own mul_Hs,
get_Hs and step_length (each checked against the oracle in
test_gpu_cones.py); residuals, add_step and rectify against numpy
restatements of the reference's formulas; the LDL solver by its residual
on KKT systems with the problem families' patterns."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

from cuclarabel_b200 import _lib, problems
from cuclarabel_b200.api import Settings
from test_gpu_cones import GPUCones, interior

pytestmark = pytest.mark.gpu

SPECS = [(0, 2, 0.0), (1, 5, 0.0), (2, 3, 0.0), (2, 10, 0.0), (2, 4, 0.0), (2, 7, 0.0),
         (3, 3, 0.0), (4, 3, 0.45), (5, 3, 0.0)]


def _scaled_cones(seed=0, specs=SPECS):
    rng = np.random.default_rng(seed)
    s = np.concatenate([interior(rng, p) for p in specs])
    z = np.concatenate([interior(rng, p) for p in specs])
    G = GPUCones(specs)
    ds_, dz_ = G.dev(s), G.dev(z)
    assert G.L.clgpu_update_scaling(G.h, ds_.data_ptr(), dz_.data_ptr(), float(s @ z / 10), 0,
                                    None) == 0
    return G, rng, s, z, (ds_, dz_)


def _rows(p):
    t, d, _ = p
    return 3 if t in (3, 4) else (d * (d + 1) // 2 if t == 5 else d)


def test_mul_Hs_diag_skips_only_the_sparse_soc_rows(cuda_device):
    G, rng, s, z, keep = _scaled_cones(1)
    x = G.dev(rng.standard_normal(G.numel))
    full = G.empty(G.numel)
    assert G.L.clgpu_mul_Hs(G.h, full.data_ptr(), x.data_ptr(), None) == 0
    sentinel = rng.standard_normal(G.numel)
    y = G.dev(sentinel)
    assert G.L.clgpu_mul_Hs_diag(G.h, y.data_ptr(), x.data_ptr(), None) == 0
    yd, yf = y.cpu().numpy(), full.cpu().numpy()
    r = 0
    for p in SPECS:
        n = _rows(p)
        sparse = p[0] == 2 and p[1] > 5
        if sparse:
            assert np.array_equal(yd[r:r + n], sentinel[r:r + n])
        else:
            assert np.array_equal(yd[r:r + n], yf[r:r + n])
        r += n


def test_rectify_equilibration(cuda_device):
    G, rng, _, _, _ = _scaled_cones(2)
    e = rng.uniform(0.3, 3.0, G.numel)
    de, dd = G.dev(e), G.empty(G.numel)
    changed = ctypes.c_int(-1)
    assert G.L.clgpu_rectify_equilibration(G.h, dd.data_ptr(), de.data_ptr(),
                                           ctypes.byref(changed), None) == 0
    assert changed.value == 1
    # coneops_default.jl / mathutils_gpu.jl: delta = mean(e_cone) / e on
    # every non-elementwise cone, 1 elsewhere
    expect = np.ones(G.numel)
    r = 0
    for p in SPECS:
        n = _rows(p)
        if p[0] >= 2:
            expect[r:r + n] = e[r:r + n].mean() / e[r:r + n]
        r += n
    assert np.allclose(dd.cpu().numpy(), expect, rtol=1e-14, atol=0)


def test_refresh_kkt_blocks_and_sparse_expansion(cuda_device):
    """-Hs lands at the Hs map; for every sparse SOC the expansion entries
    reproduce the full block: eliminating the two extra rows from
    [-eta^2 D, -eta^2 v, -eta^2 u; . , -eta^2, 0; ., 0, eta^2] gives -W'W."""
    import torch
    G, rng, _, _, _ = _scaled_cones(3)
    hs = G.empty(G.hs_len)
    assert G.L.clgpu_get_Hs(G.h, hs.data_ptr(), None) == 0
    hs = hs.cpu().numpy()[:G.hs_len]
    sparse = [p for p in SPECS if p[0] == 2 and p[1] > 5]
    nvu = 2 * sum(p[1] for p in sparse)
    total = G.hs_len + 2 * nvu + 2 * len(sparse)
    perm = rng.permutation(total).astype(np.int32)
    hs_map = perm[:G.hs_len]
    vu = perm[G.hs_len:G.hs_len + nvu]
    vut = perm[G.hs_len + nvu:G.hs_len + 2 * nvu]
    D = perm[G.hs_len + 2 * nvu:]
    dev = lambda a: torch.tensor(a, dtype=torch.int32, device="cuda")
    d_hs, d_vu, d_vut, d_D = dev(hs_map), dev(vu), dev(vut), dev(D)
    kv = G.empty(total)
    kv32 = torch.zeros(total, dtype=torch.float32, device="cuda")
    assert G.L.clgpu_refresh_kkt(G.h, kv.data_ptr(), d_hs.data_ptr(), d_vu.data_ptr(),
                                 d_vut.data_ptr(), d_D.data_ptr(), kv32.data_ptr(), None) == 0
    k = kv.cpu().numpy()
    assert np.array_equal(k[hs_map], -hs)
    assert np.array_equal(kv32.cpu().numpy(), k.astype(np.float32))
    assert np.array_equal(k[vu], k[vut])
    # full W'W blocks from mul_Hs on unit vectors
    r = blk = j = si = 0
    for p in SPECS:
        n = _rows(p)
        t, d = p[0], p[1]
        if t == 2 and d > 5:
            H = np.zeros((d, d))
            for c in range(d):
                e = np.zeros(G.numel)
                e[r + c] = 1.0
                y = G.empty(G.numel)
                de = G.dev(e)
                assert G.L.clgpu_mul_Hs(G.h, y.data_ptr(), de.data_ptr(), None) == 0
                H[:, c] = y.cpu().numpy()[r:r + d]
            kcc = np.diag(k[hs_map[blk:blk + d]])
            v, u = k[vu[j:j + d]], k[vu[j + d:j + 2 * d]]
            d1, d2 = k[D[2 * si]], k[D[2 * si + 1]]
            schur = kcc - np.outer(v, v) / d1 - np.outer(u, u) / d2
            assert np.allclose(schur, -H, rtol=1e-11, atol=1e-11 * np.abs(H).max())
            j += 2 * d
            si += 1
        blk += n if (t <= 1 or (t == 2 and d > 5)) else n * (n + 1) // 2
        r += n


@pytest.mark.parametrize("asym", [False, True])
def test_step_length_device_matches_host_form(cuda_device, asym):
    import torch
    specs = SPECS if asym else [p for p in SPECS if p[0] not in (3, 4)]
    G, rng, s, z, (ds_, dz_) = _scaled_cones(4, specs)
    dz, dsv = rng.standard_normal(G.numel), rng.standard_normal(G.numel)
    ddz, dds = G.dev(dz), G.dev(dsv)
    a_host = ctypes.c_double()
    assert G.L.clgpu_step_length(G.h, ddz.data_ptr(), dds.data_ptr(), dz_.data_ptr(),
                                 ds_.data_ptr(), 1.0, 0.99, 0.8, 1e-4,
                                 ctypes.byref(a_host), None) == 0
    amax = torch.tensor([1.0], dtype=torch.float64, device="cuda")
    a_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert G.L.clgpu_step_length_device(G.h, ddz.data_ptr(), dds.data_ptr(), dz_.data_ptr(),
                                        ds_.data_ptr(), amax.data_ptr(), 0.99, 0.8, 1e-4,
                                        a_dev.data_ptr(), None) == 0
    assert a_dev.item() == a_host.value


# ------------------------------------------------------------------ LDL
def _kkt(pb, rng, delta=1.0):
    """[P + I, A'; A, -H] with H a positive diagonal: quasi-definite, the
    pattern of the problem's KKT matrix without the cone blocks."""
    P, _, A, _, _ = pb
    n, m = A.shape[1], A.shape[0]
    Pf = (P + sp.triu(P, 1).T).tocsr()
    K = sp.bmat([[Pf + delta * sp.eye(n), A.T], [A, -sp.diags(rng.uniform(0.5, 2, m))]],
                format="csr")
    K.sort_indices()
    dsig = np.concatenate([np.ones(n), -np.ones(m)]).astype(np.int8)
    return K, dsig


def _ldl(K, dsig, method="cudss"):
    L = _lib.load()
    st = Settings(direct_solve_method=method).to_c()
    h = ctypes.c_void_p()
    Kp, Kj = K.indptr.astype(np.int32), K.indices.astype(np.int32)
    rc = L.clgpu_ldl_create(K.shape[0], Kp.ctypes.data_as(_lib.ip), Kj.ctypes.data_as(_lib.ip),
                            dsig.ctypes.data_as(ctypes.POINTER(ctypes.c_byte)), ctypes.byref(st),
                            ctypes.byref(h))
    assert rc == 0, rc
    return L, h


@pytest.mark.parametrize("family,scale,method", [
    ("mpc", 0, "cudss"),
    ("mixed_socp", 0.3, "cudss"),       # N = 24000: several blocked fronts of many panels
    ("exp_pow_psd", 0.05, "cudss"),
    ("mixed_socp", 0.3, "cudssmixed"),  # FP32 factor, FP64 refinement
])
def test_ldl_refactor_and_refined_solve(cuda_device, family, scale, method):
    import torch
    rng = np.random.default_rng(7)
    pb = (problems.mpc_qp(11) if family == "mpc" else
          getattr(problems, family)(scale=scale))
    K, dsig = _kkt(pb, rng)
    L, h = _ldl(K, dsig, method)
    try:
        kx = torch.tensor(K.data, dtype=torch.float64, device="cuda")
        eps = ctypes.c_double()
        assert L.clgpu_ldl_refactor(h, kx.data_ptr(), ctypes.byref(eps), None) == 0
        expect_eps = 1e-8 + np.finfo(float).eps ** 2 * np.abs(K.diagonal()).max()
        assert eps.value == pytest.approx(expect_eps, rel=1e-12)
        for trial in range(2):
            b = rng.standard_normal(K.shape[0])
            db = torch.tensor(b, dtype=torch.float64, device="cuda")
            dx = torch.zeros_like(db)
            assert L.clgpu_ldl_solve(h, db.data_ptr(), dx.data_ptr(), None) == 0
            x = dx.cpu().numpy()
            res = np.abs(K @ x - b).max() / np.abs(b).max()
            assert res < 1e-11, (family, method, res)  # refinement stops at 1e-12 (1 + |b|)
        # a second refactor with new values (same pattern)
        K2 = K.copy()
        K2.data = K.data * rng.uniform(0.9, 1.1, K.nnz)
        K2 = (K2 + K2.T) / 2
        K2 = K2.tocsr()
        K2.sort_indices()
        assert np.array_equal(K2.indices, K.indices)
        kx2 = torch.tensor(K2.data, dtype=torch.float64, device="cuda")
        assert L.clgpu_ldl_refactor(h, kx2.data_ptr(), None, None) == 0
        b = rng.standard_normal(K.shape[0])
        db = torch.tensor(b, dtype=torch.float64, device="cuda")
        dx = torch.zeros_like(db)
        assert L.clgpu_ldl_solve(h, db.data_ptr(), dx.data_ptr(), None) == 0
        assert np.abs(K2 @ dx.cpu().numpy() - b).max() / np.abs(b).max() < 1e-11
    finally:
        L.clgpu_ldl_destroy(h)


def test_ldl_rejects_a_missing_diagonal(cuda_device):
    K = sp.csr_matrix(np.array([[0.0, 1.0], [1.0, 2.0]]))
    K.eliminate_zeros()
    L = _lib.load()
    h = ctypes.c_void_p()
    dsig = np.array([1, -1], np.int8)
    Kp, Kj = K.indptr.astype(np.int32), K.indices.astype(np.int32)
    assert L.clgpu_ldl_create(2, Kp.ctypes.data_as(_lib.ip), Kj.ctypes.data_as(_lib.ip),
                              dsig.ctypes.data_as(ctypes.POINTER(ctypes.c_byte)), None,
                              ctypes.byref(h)) == -2


# ------------------------------------------------------- residuals, add_step
def _dev(a, dtype=None):
    import torch
    a = np.asarray(a)
    return torch.tensor(a, dtype=dtype or (torch.int32 if a.dtype.kind == "i" else torch.float64),
                        device="cuda")


def test_residuals_and_add_step(cuda_device):
    import torch
    rng = np.random.default_rng(5)
    P, q, A, b, _ = problems.mpc_qp(21)
    n, m = A.shape[1], A.shape[0]
    Pf = (P + sp.triu(P, 1).T).tocsr()
    Ac, At = A.tocsr(), A.T.tocsr()
    x, s, z = rng.standard_normal(n), rng.uniform(0.1, 1, m), rng.uniform(0.1, 1, m)
    tau, kappa = 0.8, 0.3
    d = {k: _dev(v) for k, v in dict(Pp=Pf.indptr.astype(np.int32), Pj=Pf.indices.astype(np.int32),
                                     Px=Pf.data, Ap=Ac.indptr.astype(np.int32),
                                     Aj=Ac.indices.astype(np.int32), Ax=Ac.data,
                                     Atp=At.indptr.astype(np.int32),
                                     Atj=At.indices.astype(np.int32), Atx=At.data, q=q, b=b,
                                     x=x, s=s, z=z, tau=[tau], kappa=[kappa]).items()}
    out = {k: torch.zeros(nn, dtype=torch.float64, device="cuda")
           for k, nn in (("rx", n), ("rz", m), ("rxi", n), ("rzi", m), ("px", n), ("dots", 5))}
    L = _lib.load()
    work = torch.zeros(L.clgpu_residuals_work_len(), dtype=torch.float64, device="cuda")
    args = [d[k].data_ptr() for k in ("Pp", "Pj", "Px", "Ap", "Aj", "Ax", "Atp", "Atj", "Atx",
                                      "q", "b", "x", "s", "z", "tau", "kappa")]
    args += [out[k].data_ptr() for k in ("rx", "rz", "rxi", "rzi", "px", "dots")]
    assert L.clgpu_residuals(n, m, *args, work.data_ptr(), None) == 0
    torch.cuda.synchronize()
    # residuals.jl:39-75
    Px = Pf @ x
    rxi, rzi = -(At @ z), Ac @ x + s
    ok = lambda a, e: np.allclose(a.cpu().numpy(), e, rtol=1e-13, atol=1e-13 * np.abs(e).max())
    assert ok(out["px"], Px) and ok(out["rxi"], rxi) and ok(out["rzi"], rzi)
    assert ok(out["rx"], rxi - Px - q * tau) and ok(out["rz"], rzi - b * tau)
    qx, bz, sz, xPx = q @ x, b @ z, s @ z, x @ Px
    assert ok(out["dots"], np.array([qx, bz, sz, xPx, qx + bz + kappa + xPx / tau]))
    # variables_add_step! (variables.jl:146-158)
    dx, dsv, dz = rng.standard_normal(n), rng.standard_normal(m), rng.standard_normal(m)
    dd = {k: _dev(v) for k, v in dict(dx=dx, ds=dsv, dz=dz, dt=[0.5], dk=[-0.2],
                                      al=[0.37]).items()}
    assert L.clgpu_add_step(n, m, d["x"].data_ptr(), d["s"].data_ptr(), d["z"].data_ptr(),
                            d["tau"].data_ptr(), d["kappa"].data_ptr(), dd["dx"].data_ptr(),
                            dd["ds"].data_ptr(), dd["dz"].data_ptr(), dd["dt"].data_ptr(),
                            dd["dk"].data_ptr(), dd["al"].data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert ok(d["x"], x + 0.37 * dx) and ok(d["s"], s + 0.37 * dsv) and ok(d["z"], z + 0.37 * dz)
    assert d["tau"].item() == tau + 0.37 * 0.5 and d["kappa"].item() == kappa + 0.37 * -0.2
