"""fmm_set_sources_async: sources copied from page-locked host memory on the plan's copy stream, the tree
build starting once the points are in and taking the strengths at its end. Every result equals the one
after the synchronous fmm_set_sources bit for bit (the same kernels on the same data); pageable memory is
refused; calls that read the sources without a tree build (direct sums, targets = sources) wait for the
copies."""
import numpy as np
import pytest
import torch

from bachelors_b200 import Plan, geometry as G
from bachelors_b200._lib import FmmError

pytestmark = pytest.mark.gpu


def _pinned(*arrays):
    return [torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy() for a in arrays]


def _case(dt):
    xyz, w, J = (a.astype(dt) for a in G.torus(64, 16, 16, 2.0, 0.5))
    tgt = G.uniform_points(3000, -3, 3, 5).astype(dt)
    return xyz, w, J, tgt


@pytest.mark.parametrize("precision,m2l", [("fp32", "bf16x3"), ("fp32", "simt"), ("fp64", "simt")])
def test_async_sources_equal_sync(precision, m2l):
    dt = np.float32 if precision == "fp32" else np.float64
    xyz, w, J, tgt = _case(dt)
    hx, hw, hw2, hJ = _pinned(xyz, w, 2 * w, J)

    def run(asynchronous, same):
        plan = Plan(order=10, leaf_capacity=32, precision=precision, m2l=m2l)
        out = []
        for weights in (hw, hw2):   # twice on one plan: the second copy follows the first solve
            plan.set_sources(hx, weights, hJ, asynchronous=asynchronous)
            if same:
                plan.set_targets_to_sources()
            else:
                plan.set_targets(tgt)
            B, _ = plan.solve(1.0, 1)
            out.append(np.array(B, copy=True))
        D, _ = plan.direct(1.0, 1)
        out.append(np.array(D, copy=True))
        plan.close()
        return out

    for same in (True, False):
        for a, s in zip(run(True, same), run(False, same)):
            np.testing.assert_array_equal(a, s)


def test_async_sources_without_a_solve_in_between():
    """Two asynchronous source sets in a row, then a direct sum and a solve: the second set's data."""
    xyz, w, J, tgt = _case(np.float32)
    hx, hw, hJ = _pinned(xyz, w, J)
    hw2 = _pinned(w * 3)[0]
    plan = Plan(order=8, leaf_capacity=32, precision="fp32", m2l="bf16x3")
    plan.set_sources(hx, hw, hJ, asynchronous=True)
    plan.set_sources(hx, hw2, hJ, asynchronous=True)
    plan.set_targets(tgt)
    Da, _ = plan.direct(1.0, 1)
    Ba, _ = plan.solve(1.0, 1)
    ref = Plan(order=8, leaf_capacity=32, precision="fp32", m2l="bf16x3")
    ref.set_sources(xyz, w * 3, J)
    ref.set_targets(tgt)
    Db, _ = ref.direct(1.0, 1)
    Bb, _ = ref.solve(1.0, 1)
    np.testing.assert_array_equal(Da, Db)
    np.testing.assert_array_equal(Ba, Bb)
    plan.close()
    ref.close()


def test_async_sources_batch_and_azimuthal():
    xyz, w, J, tgt, so, to = G.torus_batch(6, seed=3, count_range=(2 ** 8, 2 ** 11), targets_per_coil=128)
    f32 = lambda a: a.astype(np.float32)
    hx, hw = _pinned(f32(xyz), f32(w))
    out = []
    for asynchronous in (True, False):
        plan = Plan(order=6, leaf_capacity=16, precision="fp32", m2l="bf16x3")
        plan.set_sources(hx, hw, None, asynchronous=asynchronous)   # the azimuthal current direction
        plan.set_targets(f32(tgt))
        plan.set_coils(so, to)
        B, _ = plan.solve(1.0, 1)
        out.append(np.array(B, copy=True))
        plan.close()
    np.testing.assert_array_equal(out[0], out[1])


def test_async_sources_refuse_pageable_memory():
    xyz, w, J, _ = _case(np.float32)
    plan = Plan(order=6, leaf_capacity=32, precision="fp32")
    with pytest.raises(FmmError):
        plan.set_sources(xyz, w, J, asynchronous=True)
    # the plan is still usable with the synchronous call
    plan.set_sources(xyz, w, J)
    plan.set_targets_to_sources()
    B, _ = plan.solve(1.0, 1)
    assert np.all(np.isfinite(B))
    plan.close()
