"""Bounded device waits of the tensor-core pipelines (tcgen05 M2L, M2M): when a wait runs out, the
solve returns FMM_E_TIMEOUT instead of hanging, the CTAs wait for their own copies and MMAs before
they free tensor memory, and the plan and its GPU context stay usable - the next solve with the normal
limit matches the CPU restatement.

The failure is made by a wait limit of one nanosecond (fmm_set_wait_limit): no hardware fault, no
trap, no endless loop is involved; every wait still ends."""
import numpy as np
import pytest

from bachelors_b200 import Plan, geometry as G
from bachelors_b200._lib import FMM_E_TIMEOUT, FmmError
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b)


def test_pipeline_wait_limit_runs_out_and_plan_recovers():
    xyz, w, J = G.torus(64, 16, 16, 2.0, 0.5)
    tgt = G.uniform_points(3000, -3, 3, 17)
    x32, w32, J32, t32 = (a.astype(np.float32) for a in (xyz, w, J, tgt))
    plan = Plan(order=8, leaf_capacity=16, precision="fp32", m2l="bf16x3")
    plan.set_sources(x32, w32, J32)
    plan.set_targets(t32)
    B0, _ = plan.solve(1.0, 1)
    plan.set_wait_limit(1e-9)
    statuses = []
    for _ in range(3):
        try:
            plan.solve(1.0, 1)
            statuses.append(0)
        except FmmError as e:
            statuses.append(e.status)
    # every failure is a timeout, and a one-nanosecond limit makes some wait run out
    assert set(statuses) <= {0, FMM_E_TIMEOUT} and FMM_E_TIMEOUT in statuses
    plan.set_wait_limit(2.0)
    B, _ = plan.solve(1.0, 1)
    np.testing.assert_array_equal(B, B0)
    c, H = G.root_cube(x32.astype(np.float64), t32.astype(np.float64))
    Bo, _, _ = O.fmm(8, 16, x32, w32, J32, t32, c, H)
    assert rel(B, Bo) < 2e-5
    plan.close()


def test_wait_limit_is_validated():
    plan = Plan(order=4, precision="fp32", m2l="bf16x3")
    for bad in (0.0, -1.0, 61.0):
        with pytest.raises(FmmError):
            plan.set_wait_limit(bad)
    plan.close()
