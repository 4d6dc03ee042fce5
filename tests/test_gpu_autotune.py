"""The autotuner (fmm_autotune) and the tile choices it picks between: every choice gives the same
field within rounding, the tuned plan still solves correctly, and plans created later with the same
parameters start with the tuned choice."""
import numpy as np
import pytest

from bachelors_b200 import Plan, geometry as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("precision,m2l,tol", [("fp32", "bf16x3", 1e-5), ("fp32", "simt", 1e-6), ("fp64", "simt", 1e-13)])
def test_every_tile_choice_gives_the_same_field(precision, m2l, tol):
    dt = np.float32 if precision == "fp32" else np.float64
    xyz, w, J = G.torus(48, 16, 8, 2.0, 0.5)
    plan = Plan(order=12, leaf_capacity=48, precision=precision, m2l=m2l)
    plan.set_sources(xyz.astype(dt), w.astype(dt), J.astype(dt))
    plan.set_targets(xyz.astype(dt))
    ref = None
    for kc in (64, 32):
        for ts in (256, 128):
            for cv in (0, 16, 32):
                plan.set_tuning(kc, ts, cv)
                assert plan.tuning() == {"m2l_k_chunk": kc, "near_tile": ts, "p2m_chunk": cv}
                B, _ = plan.solve(1.0, 1)
                if ref is None:
                    ref = B.astype(np.float64)
                else:
                    assert rel(B, ref) < tol
    plan.close()


def test_autotune_picks_and_remembers():
    xyz, w, J = G.torus(64, 16, 16, 2.0, 0.5)
    x32, w32, J32 = xyz.astype(np.float32), w.astype(np.float32), J.astype(np.float32)
    plan = Plan(order=10, leaf_capacity=40, precision="fp32", m2l="bf16x3")
    plan.set_sources(x32, w32, J32)
    plan.set_targets(x32)
    from bachelors_b200._lib import FmmError
    with pytest.raises(FmmError):
        plan.autotune()                      # needs a solve first
    B0, _ = plan.solve(1.0, 1)
    t = plan.autotune()
    assert t["m2l_k_chunk"] in (32, 64) and t["near_tile"] in (128, 256) and t["p2m_chunk"] in (0, 16, 32)
    assert t["ms_upward"] > 0 and t["ms_downward"] > 0 and t["ms_near"] > 0
    B1, _ = plan.solve(1.0, 1)
    assert rel(B1, B0) < 1e-5
    idx = np.arange(0, len(xyz), 97)
    D = O.direct(x32.astype(np.float64), w32.astype(np.float64), J32.astype(np.float64), x32[idx].astype(np.float64))
    assert rel(B1[idx], D) < 1e-4
    other = Plan(order=10, leaf_capacity=40, precision="fp32", m2l="bf16x3")
    assert other.tuning() == {k: t[k] for k in ("m2l_k_chunk", "near_tile", "p2m_chunk")}
    with pytest.raises(FmmError):
        other.set_tuning(48, 256, 16)
    other.close()
    plan.close()
