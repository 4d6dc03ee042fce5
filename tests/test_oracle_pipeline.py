"""Properties of the standard-mode tree, lists and FMM that the device pipeline implements."""
import numpy as np
import pytest

from bachelors_b200 import geometry as G
from oracle import oracle as O


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("cap", [4, 16])
def test_every_pair_counted_once(cap):
    xyz, w, J = G.torus(24, 12, 6, 2.0, 0.5)
    tgt = np.r_[G.uniform_points(300, -3, 3, 7), xyz[::11]]
    c, H = G.root_cube(xyz, tgt)
    cnt = O.coverage(cap, xyz, tgt, c, H)
    assert cnt.min() == 1 and cnt.max() == 1


def test_tree_invariants():
    xyz, w, J = G.torus(32, 16, 8, 2.0, 0.5)
    tgt = G.uniform_points(2000, -3, 3, 3)
    c, H = G.root_cube(xyz, tgt)
    info, lists, so, to = O.tree(16, xyz, tgt, c, H)
    assert sorted(so.tolist()) == list(range(len(xyz)))
    assert sorted(to.tolist()) == list(range(len(tgt)))
    leaf = info[:, 9] == 0
    # a leaf holds at most `cap` points of each kind unless it is at the maximum depth
    ok = ((info[:, 5] - info[:, 4] <= 16) & (info[:, 7] - info[:, 6] <= 16)) | (info[:, 0] == 21)
    assert ok[leaf].all()
    assert lists[:, 0].max() <= 189


@pytest.mark.parametrize("p,tol", [(6, 5e-3), (10, 1e-3)])
def test_fmm_converges_to_direct(p, tol):
    xyz, w, J = G.torus(32, 16, 8, 2.0, 0.5)
    tgt = G.uniform_points(200, -3, 3, 5)
    c, H = G.root_cube(xyz, tgt)
    B, A, _ = O.fmm(p, 16, xyz, w, J, tgt, c, H, want_A=True)
    Bd, Ad = O.direct(xyz, w, J, tgt, want_A=True)
    assert rel(B, Bd) < tol
    assert rel(A, Ad) < tol


def test_curl_matches_dual_gradient():
    # analytic curl of an expansion (dual numbers) against central differences
    p = 8
    rng = np.random.default_rng(0)
    coef = rng.normal(size=((p + 1) ** 2, 3))
    x = np.array([0.2, -0.1, 0.3])
    _, curl = O.eval_expansion(p, coef, x)
    h = 1e-6
    g = np.zeros((3, 3))
    for j in range(3):
        e = np.zeros(3)
        e[j] = h
        g[:, j] = (O.eval_expansion(p, coef, x + e)[0] - O.eval_expansion(p, coef, x - e)[0]) / (2 * h)
    fd = np.array([g[2, 1] - g[1, 2], g[0, 2] - g[2, 0], g[1, 0] - g[0, 1]])
    assert rel(curl, fd) < 1e-7
