"""The reference's own cone identities, run on the device kernels' numbers.

Restates test/UnitTests/test_coneops_secondordercone.jl:31-91 and
test_coneops_psdtrianglecone.jl:112-251 of the reference: the scaling state
update_scaling leaves on the GPU (read back with clgpu_cones_debug_scaling)
must satisfy the Nesterov-Todd identities, with the reference's
tolerances.  These identities hold for any correct implementation, so they
pin the device's second-order and PSD arithmetic independently of the
oracle.  Matrices are drawn with randn as the reference's testing_utils.jl
draws them (randsym = A + A', randpsd = A A')."""
import ctypes

import numpy as np
import pytest

from cuclarabel_b200 import _lib

pytestmark = pytest.mark.gpu
SQRT_EPS = np.sqrt(np.finfo(float).eps)


def randsym(rng, n):
    A = rng.standard_normal((n, n))
    return A + A.T


def randpsd(rng, n):
    A = rng.standard_normal((n, n))
    return A @ A.T


def svec(M):
    n = M.shape[0]
    return np.array([M[i, j] if i == j else M[i, j] * np.sqrt(2)
                     for j in range(n) for i in range(j + 1)])


def smat(v, n):
    M = np.zeros((n, n))
    k = 0
    for j in range(n):
        for i in range(j + 1):
            M[i, j] = M[j, i] = v[k] if i == j else v[k] / np.sqrt(2)
            k += 1
    return M


class Handle:
    def __init__(self, specs, soc_threshold):
        import torch
        self.torch = torch
        self.L = _lib.load()
        t = np.array([s[0] for s in specs], np.int32)
        d = np.array([s[1] for s in specs], np.int32)
        p = np.zeros(len(specs))
        h = ctypes.c_void_p()
        assert self.L.clgpu_cones_create(len(t), t.ctypes.data_as(_lib.ip),
                                         d.ctypes.data_as(_lib.ip), p.ctypes.data_as(_lib.dp),
                                         soc_threshold, ctypes.byref(h)) == 0
        self.h = h
        self.numel = self.L.clgpu_cones_numel(h)

    def dev(self, a):
        return self.torch.tensor(np.asarray(a, np.float64), device="cuda")

    def shift_interior(self, v, pd):
        """margins + scaled_unit_shift, as the reference test does"""
        dv = self.dev(v)
        a, b = ctypes.c_double(), ctypes.c_double()
        assert self.L.clgpu_margins(self.h, dv.data_ptr(), pd, ctypes.byref(a), ctypes.byref(b),
                                    None) == 0
        cor = 0.0 if a.value > 0 else 1.0 - a.value
        assert self.L.clgpu_scaled_unit_shift(self.h, dv.data_ptr(), cor, pd, None) == 0
        return dv.cpu().numpy()

    def update_scaling(self, s, z, mu):
        ds, dz = self.dev(s), self.dev(z)
        assert self.L.clgpu_update_scaling(self.h, ds.data_ptr(), dz.data_ptr(), mu, 0,
                                           None) == 0

    def mul_Hs_matrix(self):
        """W'W (Hs) column by column through mul_Hs"""
        H = np.zeros((self.numel, self.numel))
        for c in range(self.numel):
            e = np.zeros(self.numel)
            e[c] = 1.0
            de, y = self.dev(e), self.dev(np.zeros(self.numel))
            assert self.L.clgpu_mul_Hs(self.h, y.data_ptr(), de.data_ptr(), None) == 0
            H[:, c] = y.cpu().numpy()
        return H

    def __del__(self):
        self.L.clgpu_cones_destroy(self.h)


def soc_state(H, n):
    w, lam, u, v = (np.zeros(n) for _ in range(4))
    eta, d = np.zeros(1), np.zeros(1)
    dp = lambda a: a.ctypes.data_as(_lib.dp)
    assert H.L.clgpu_cones_debug_scaling(H.h, dp(w), dp(lam), dp(u), dp(v), dp(eta), dp(d),
                                         None, None, None, None) == 0
    return w, lam, u, v, eta[0], d[0]


def soc_W(w, eta):
    """W and W^-1 of the SOC NT scaling (the products of mul_W! /
    mul_Winv!, coneops_socone.jl:314-360, as matrices)"""
    n = len(w)
    w1 = w[1:]
    W = np.zeros((n, n))
    W[0, 0] = w[0]
    W[0, 1:] = W[1:, 0] = w1
    W[1:, 1:] = np.eye(n - 1) + np.outer(w1, w1) / (1 + w[0])
    Wi = W.copy()
    Wi[0, 1:] = Wi[1:, 0] = -w1
    return eta * W, Wi / eta


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_soc_W_construction(cuda_device, seed):
    """test_coneops_secondordercone.jl:31-88 (n = 5 > threshold 4: the
    sparse expansion)."""
    n = 5
    rng = np.random.default_rng(242713 + seed)
    H = Handle([(2, n, 0.0)], soc_threshold=4)
    s, z = rng.standard_normal(n), rng.standard_normal(n)
    z = H.shift_interior(z, 1)
    s = H.shift_interior(s, 0)
    H.update_scaling(s, z, float(s @ z))
    w, lam, u, v, eta, d = soc_state(H, n)
    D = np.eye(n)
    D[0, 0] = d
    W2_A = eta ** 2 * (D + np.outer(u, u) - np.outer(v, v))
    J = -np.eye(n)
    J[0, 0] = 1.0
    Hinv = eta ** 2 * (2 * np.outer(w, w) - J)
    scale = max(1.0, np.linalg.norm(Hinv))
    assert np.linalg.norm(W2_A - Hinv) <= 1e-14 * scale
    W_B, W_Binv = soc_W(w, eta)
    assert np.linalg.norm(W_B - W_B.T) <= 1e-14
    assert np.linalg.norm(W_B @ W_Binv - np.eye(n)) <= \
        1e-14 * max(1.0, np.linalg.norm(W_B) * np.linalg.norm(W_Binv))
    assert np.linalg.norm(W_B @ W_B - W2_A) <= 1e-12 * scale
    # the device's own W'W product agrees, and the NT point: W z = W^-1 s = lambda
    assert np.linalg.norm(H.mul_Hs_matrix() - W2_A) <= 1e-12 * scale
    assert np.linalg.norm(W_B @ z - lam) <= 1e-12 * max(1.0, np.linalg.norm(lam))
    assert np.linalg.norm(W_Binv @ s - lam) <= 1e-12 * max(1.0, np.linalg.norm(lam))


def test_soc_dense_scaling_identities(cuda_device):
    """The dense form (n = 4 <= threshold): W'W from mul_Hs is the
    eta^2 (2 w w' - J) of the reference, and W z = W^-1 s = lambda."""
    n = 4
    rng = np.random.default_rng(11)
    H = Handle([(2, n, 0.0)], soc_threshold=4)
    z = H.shift_interior(rng.standard_normal(n), 1)
    s = H.shift_interior(rng.standard_normal(n), 0)
    H.update_scaling(s, z, float(s @ z))
    w, lam, _, _, eta, _ = soc_state(H, n)
    J = -np.eye(n)
    J[0, 0] = 1.0
    Hinv = eta ** 2 * (2 * np.outer(w, w) - J)
    assert np.linalg.norm(H.mul_Hs_matrix() - Hinv) <= 1e-12 * max(1.0, np.linalg.norm(Hinv))
    W, Wi = soc_W(w, eta)
    assert np.linalg.norm(W @ z - lam) <= 1e-12 * max(1.0, np.linalg.norm(lam))
    assert np.linalg.norm(Wi @ s - lam) <= 1e-12 * max(1.0, np.linalg.norm(lam))


def psd_state(H, n):
    R, Ri = np.zeros(n * n), np.zeros(n * n)
    lam = np.zeros(n)
    nmax = ctypes.c_int()
    dp = lambda a: a.ctypes.data_as(_lib.dp)
    assert H.L.clgpu_cones_debug_scaling(H.h, None, None, None, None, None, None, dp(R), dp(Ri),
                                         dp(lam), ctypes.byref(nmax)) == 0
    assert nmax.value == n
    return R.reshape(n, n, order="F"), Ri.reshape(n, n, order="F"), lam


@pytest.mark.parametrize("seed", [0, 1])
def test_psd_update_scaling_identities(cuda_device, seed):
    """test_coneops_psdtrianglecone.jl:112-139 and the NT identities of
    :180-211: W = R R', W Z W' = S, R' Z R = Lambda = Rinv S Rinv', and
    W' lambda = R Lambda R' = S."""
    n = 5
    rng = np.random.default_rng(100 + seed)
    H = Handle([(5, n, 0.0)], soc_threshold=5)
    S, Z = randpsd(rng, n), randpsd(rng, n)
    H.update_scaling(svec(S), svec(Z), 0.0)
    R, Rinv, lam = psd_state(H, n)
    Lam = np.diag(lam)
    W = R @ R.T
    assert np.linalg.norm(W @ Z @ W.T - S) <= SQRT_EPS
    assert np.linalg.norm(R.T @ Z @ R - Lam) <= SQRT_EPS
    assert np.linalg.norm(Rinv @ S @ Rinv.T - Lam) <= SQRT_EPS
    assert np.linalg.norm(R @ Lam @ R.T - S) <= 1e-10 * max(1.0, np.linalg.norm(S))


def test_psd_step_length_hits_the_boundary(cuda_device):
    """test_coneops_psdtrianglecone.jl:141-178: the step along dZ alone
    (dS = 0) stops where Z + alpha dZ becomes singular; along PSD directions
    the full step is taken."""
    n = 10
    rng = np.random.default_rng(242713)
    H = Handle([(5, n, 0.0)], soc_threshold=5)
    Z, dZ = randpsd(rng, n), randsym(rng, n)
    S, dS = randpsd(rng, n), randsym(rng, n)
    H.update_scaling(svec(S), svec(Z), 0.0)
    dev = H.dev

    def step(dz, ds):
        a = ctypes.c_double()
        z_, s_, dz_, ds_ = dev(svec(Z)), dev(svec(S)), dev(svec(dz)), dev(svec(ds))
        assert H.L.clgpu_step_length(H.h, dz_.data_ptr(), ds_.data_ptr(), z_.data_ptr(),
                                     s_.data_ptr(), 1.0, 0.99, 0.8, 1e-4, ctypes.byref(a),
                                     None) == 0
        return a.value
    a = step(dZ, 0 * dS)
    assert a < 1.0
    assert abs(np.linalg.eigvalsh(Z + a * dZ).min()) <= SQRT_EPS * np.abs(Z).max()
    a = step(0 * dZ, dS)
    assert a < 1.0
    assert abs(np.linalg.eigvalsh(S + a * dS).min()) <= SQRT_EPS * np.abs(S).max()
    a = step(dZ, dS)
    m = min(np.linalg.eigvalsh(Z + a * dZ).min(), np.linalg.eigvalsh(S + a * dS).min())
    assert abs(m) <= SQRT_EPS * max(np.abs(Z).max(), np.abs(S).max())
    # PSD directions: the maximum step
    assert step(randpsd(rng, n), randpsd(rng, n)) == pytest.approx(1.0, rel=10 * np.finfo(float).eps)


def test_psd_Hs_operations(cuda_device):
    """test_coneops_psdtrianglecone.jl:213-251: the packed Hs of get_Hs
    (upper triangle, column by column) times v equals the device's W'W v."""
    n = 5
    rng = np.random.default_rng(7)
    H = Handle([(5, n, 0.0)], soc_threshold=5)
    S, Z, V1 = randpsd(rng, n), randpsd(rng, n), randpsd(rng, n)
    H.update_scaling(svec(S), svec(Z), 0.0)
    t = n * (n + 1) // 2
    hs = H.dev(np.zeros(t * (t + 1) // 2))
    assert H.L.clgpu_get_Hs(H.h, hs.data_ptr(), None) == 0
    vec = hs.cpu().numpy()
    Hs = np.zeros((t, t))
    k = 0
    for j in range(t):
        for i in range(j + 1):
            Hs[i, j] = Hs[j, i] = vec[k]
            k += 1
    v1 = svec(V1)
    dv1, v3 = H.dev(v1), H.dev(np.zeros(t))
    assert H.L.clgpu_mul_Hs(H.h, v3.data_ptr(), dv1.data_ptr(), None) == 0
    assert np.linalg.norm(Hs @ v1 - v3.cpu().numpy()) <= 1e-8 * max(1.0, np.linalg.norm(v1))
    # W'W v from R directly: W (svec v) = svec(R' V R), W' (svec u) = svec(R U R')
    R, _, _ = psd_state(H, n)
    WtWv = svec(R @ (R.T @ V1 @ R) @ R.T)
    assert np.linalg.norm(Hs @ v1 - WtWv) <= 1e-8 * max(1.0, np.linalg.norm(v1))
