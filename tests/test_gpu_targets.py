"""fmm_set_targets_to_sources: the targets taken from the device copy of the source points give the
same field as passing the same points again through fmm_set_targets, and results written to host
memory (page-locked by the wrapper) match the device-resident path."""
import numpy as np
import pytest
import torch

from bachelors_b200 import FastMultipoleSolver, Plan, geometry as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_targets_to_sources_equals_explicit_targets(precision):
    dt = np.float32 if precision == "fp32" else np.float64
    xyz, w, J = (a.astype(dt) for a in G.torus(48, 16, 8, 2.0, 0.5))
    a = Plan(order=8, leaf_capacity=32, precision=precision)
    a.set_sources(xyz, w, J)
    a.set_targets(xyz)
    Ba, _ = a.solve(1.0, 1)
    b = Plan(order=8, leaf_capacity=32, precision=precision)
    b.set_sources(xyz, w, J)
    b.set_targets_to_sources()
    Bb, _ = b.solve(1.0, 1)
    np.testing.assert_array_equal(Ba, Bb)
    # twice in a row on one plan, with new strengths in between
    b.set_sources(xyz, 2 * w, J)
    b.set_targets_to_sources()
    Bc, _ = b.solve(1.0, 1)
    np.testing.assert_allclose(Bc, 2 * Bb, rtol=1e-5 if precision == "fp32" else 1e-12, atol=0)
    a.close()
    b.close()


def test_solver_with_points_is_quadratures_and_device_path():
    xyz, w, J = (a.astype(np.float32) for a in G.torus(48, 16, 8, 2.0, 0.5))
    s = FastMultipoleSolver((xyz, w, J), xyz, quadratureOctreeLeafCapacity=32, calculationPointOctreeLeafCapacity=32,
                            order=8, precision="fp32")
    Bh = s.solve(1.0, "B")
    s.plan.close()
    d = lambda x: torch.from_numpy(x).cuda()
    s2 = FastMultipoleSolver((d(xyz), d(w), d(J)), d(xyz), quadratureOctreeLeafCapacity=32,
                             calculationPointOctreeLeafCapacity=32, order=8, precision="fp32")
    Bd = s2.solve(1.0, "B").cpu().numpy()
    s2.plan.close()
    np.testing.assert_array_equal(Bh, Bd)


@pytest.mark.parametrize("m2l", ["bf16x3", "simt"])
def test_targets_stay_the_copy_after_new_sources(m2l):
    """The plan reuses the sources' sorted order for targets set by fmm_set_targets_to_sources; new sources set
    afterwards leave the targets at the earlier points (the copy), as with explicit targets."""
    xyz, w, J = (a.astype(np.float32) for a in G.torus(48, 16, 8, 2.0, 0.5))
    xyz2 = (xyz * np.float32(1.1) + np.float32(0.05)).astype(np.float32)
    a = Plan(order=8, leaf_capacity=32, precision="fp32", m2l=m2l)
    a.set_sources(xyz, w, J)
    a.set_targets_to_sources()
    a.solve(1.0, 1)
    a.set_sources(xyz2, w, J)
    Ba, _ = a.solve(1.0, 1)
    b = Plan(order=8, leaf_capacity=32, precision="fp32", m2l=m2l)
    b.set_sources(xyz2, w, J)
    b.set_targets(xyz)
    Bb, _ = b.solve(1.0, 1)
    np.testing.assert_array_equal(Ba, Bb)
    a.close()
    b.close()
