"""The BEM problem (the reference's Problem::BEM): the oracle's restatement of its direct integral and of
its P2M against vectors the reference produced (tests/golden/reference_bem.npz, made by
tests/golden/make_golden.py bem), and the multipole form of the kernel: the BEM multipole evaluated with
irregular harmonics reproduces the direct integral at well-separated targets."""
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "reference_bem.npz"))


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def test_bem_direct_matches_reference():
    out = O.bem_direct(G["src"], G["w"], G["B"], G["nrm"], G["tgt"])
    assert rel(out, G["direct"]) < 1e-13


@pytest.mark.parametrize("p", [4, 10])
def test_bem_p2m_matches_reference(p):
    c = G[f"p2m_p{p}_center"]
    # the reference differentiates the regular harmonics by central differences (step 1e-3)
    fd = O.bem_p2m(p, G["src"], G["w"], G["B"], G["nrm"], c, compat=True, fd_eps=1e-3)
    assert rel(fd, G[f"p2m_p{p}"]) < 1e-12
    # the analytic gradient differs from that by the differences' own error only
    an = O.bem_p2m(p, G["src"], G["w"], G["B"], G["nrm"], c, compat=True)
    assert rel(an, G[f"p2m_p{p}"]) < 1e-5


@pytest.mark.parametrize("p,tol", [(4, 2e-2), (10, 2e-7)])
def test_bem_multipole_reproduces_direct_integral(p, tol):
    c = G[f"p2m_p{p}_center"]
    M = O.bem_p2m(p, G["src"], G["w"], G["B"], G["nrm"], c, compat=True)
    far = np.array([O.eval_expansion(p, M, x - c, regular=False, compat=True)[0] for x in G["tgt"]])
    far /= 4 * O.REF_PI
    assert rel(far, G["direct"]) < tol


def test_bem_kernel_is_a_dipole_potential():
    """Each component of the BEM kernel is grad_x(1/|x - q|) . D_c(q) with D = (B . n) I + [B x n]_x^T:
    the restatement's direct sum equals that form (so the P2M of point dipoles is the right expansion)."""
    rng = np.random.default_rng(5)
    src = rng.normal(size=(7, 3))
    w = rng.uniform(0.5, 1, 7)
    B = rng.normal(size=(7, 3))
    nrm = rng.normal(size=(7, 3))
    x = np.array([[4.0, -1.0, 2.0]])
    out = O.bem_direct(src, w, B, nrm, x)[0]
    ref = np.zeros(3)
    for q, wq, b, nq in zip(src, w, B, nrm):
        g = (q - x[0]) / np.linalg.norm(q - x[0]) ** 3          # grad_x 1/|x - q|
        v = np.cross(b, nq)
        D = np.dot(b, nq) * np.eye(3) + np.array([[0, v[2], -v[1]], [-v[2], 0, v[0]], [v[1], -v[0], 0]])
        ref += wq * D @ g
    assert rel(out, ref / (4 * O.REF_PI)) < 1e-14
