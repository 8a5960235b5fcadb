"""The SOC tile kernels sum a cone's terms with a zero-padded 16-leaf tree
(pairs at distance 8, 4, 2, 1) to reproduce the lane-group kernels'
butterfly reduction over G lanes (xor distances G/2 .. 1, lanes past the
cone's dimension holding +0).  This checks the identity in IEEE double on
the host, for every dimension up to 16 and every group width G >= dim, with
values that make the summation order visible."""
import numpy as np
import pytest


def butterfly(leaves, G):
    v = np.zeros(32)
    v[:len(leaves)] = leaves
    v = v[:G].copy()
    o = G // 2
    while o > 0:
        v = np.array([v[l] + v[l ^ o] for l in range(G)])
        o //= 2
    assert np.all(v.view(np.uint64) == v[0].view(np.uint64))  # every lane agrees
    return v[0]


def tree16(leaves):
    d = len(leaves)
    p = [(leaves[l] if l < d else 0.0) + (leaves[l + 8] if l + 8 < d else 0.0)
         for l in range(8)]
    for o in (4, 2, 1):
        for l in range(o):
            p[l] = p[l] + p[l + o]
    return p[0]


@pytest.mark.parametrize("dim", range(1, 17))
def test_tree16_equals_group_butterfly_bitwise(dim):
    rng = np.random.default_rng(dim)
    for trial in range(200):
        # wide dynamic range and mixed signs: reordering changes the rounding
        leaves = rng.standard_normal(dim) * 10.0 ** rng.integers(-8, 9, dim)
        if trial % 7 == 0:
            leaves[rng.integers(0, dim)] = -0.0
        ref = tree16(list(leaves))
        G = 2
        while G < dim:
            G *= 2
        while G <= 32:
            assert np.float64(butterfly(leaves, G)).view(np.uint64) == \
                np.float64(ref).view(np.uint64), (dim, G, trial)
            G *= 2


def test_order_matters_for_these_values():
    """The check above is not vacuous: a left-to-right sum of the same
    leaves differs from the tree in the last bits for some inputs."""
    rng = np.random.default_rng(0)
    differ = 0
    for _ in range(500):
        leaves = rng.standard_normal(10) * 10.0 ** rng.integers(-8, 9, 10)
        seq = 0.0
        for x in leaves:
            seq += x
        differ += seq != tree16(list(leaves))
    assert differ > 0
