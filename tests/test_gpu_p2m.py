"""P2M variants: the warp-per-leaf kernel (lanes own harmonic orders m and p - m) and the
block-per-leaf kernels (16 or 32 recurrence steps per shared tile) give the same multipoles, so
the same field, at every order from 1 to the largest, even and odd (the pairing of orders differs
between them), with leaves of more than 32 points (the warp kernel takes 32 at a time)."""
import numpy as np
import pytest

from bachelors_b200 import FastMultipoleSolver, Plan, geometry as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("p", [1, 2, 5, 8, 13, 15, 16])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
def test_p2m_variants_agree(p, precision, tol):
    dt = np.float32 if precision == "fp32" else np.float64
    xyz, w, J = G.torus(40, 12, 8, 2.0, 0.5)
    plan = Plan(order=p, leaf_capacity=64, precision=precision, m2l="simt")
    plan.set_sources(xyz.astype(dt), w.astype(dt), J.astype(dt))
    plan.set_targets(xyz.astype(dt))
    out = {}
    for cv in (0, 16, 32):
        plan.set_tuning(64, 256, cv)
        B, _ = plan.solve(1.0, 1)
        out[cv] = B.astype(np.float64)
        assert np.isfinite(out[cv]).all(), (cv, np.where(~np.isfinite(out[cv]).all(axis=1))[0][:8])
    plan.close()
    assert rel(out[0], out[16]) < tol
    assert rel(out[32], out[16]) < tol


@pytest.mark.parametrize("p,cap", [(3, 40), (9, 48), (15, 64)])
def test_odd_order_fp64_pipeline_matches_oracle(p, cap):
    """The default (warp-per-leaf) P2M in the whole FP64 solve, odd orders, against the oracle."""
    xyz, w, J = G.torus(32, 16, 8, 2.0, 0.5)
    tgt = G.uniform_points(1000, -3, 3, 5)
    s = FastMultipoleSolver((xyz, w, J), tgt, quadratureOctreeLeafCapacity=cap,
                            calculationPointOctreeLeafCapacity=cap, order=p, precision="fp64")
    assert s.plan.tuning()["p2m_chunk"] == 0
    B, A = s.solve(1.0, "AB")
    s.plan.close()
    c, H = G.root_cube(xyz, tgt)
    Bo, Ao, _ = O.fmm(p, cap, xyz, w, J, tgt, c, H, want_A=True)
    assert rel(B, Bo) < 1e-12
    assert rel(A, Ao) < 1e-12
