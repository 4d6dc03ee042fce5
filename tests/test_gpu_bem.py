"""The BEM problem on the device (fmm_set_bem_sources; the reference's Problem::BEM,
FastMultipoleSolver::calcBEM, fast_multipole_solver.cpp:233-250) through the C ABI:

* the direct BEM integral against the CPU restatement of math::calcBEMIntegral (integration.cpp:191-215) on
  the reference's own inputs (tests/golden/reference_bem.npz): FP64 <= 1e-13, FP32 <= 1e-5;
* the device P2M (dipole multipoles from the analytic gradient of the regular harmonics) against the
  restatement of math::calcBEMIntegralContribution (integration.cpp:295-353): a one-box tree evaluated by
  the treecode at well-separated points equals sum_k M_k I_k(x - c) / (4 pi) of the restatement's
  multipole to 1e-12 in FP64;
* the FMM (tree, translations, L2P of the potential, direct near field) against the direct sum.
"""
import os

import numpy as np
import pytest

from bachelors_b200 import FastMultipoleSolver, Plan, Problem, geometry as G
from bachelors_b200._lib import FmmError
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_bem.npz"))


def rel(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b)


def cylinder_surface(n_phi=48, n_z=24, radius=0.8, height=2.0, seed=3):
    """Midpoint quadrature of a closed cylinder's side, outward normals, a smooth field B on it."""
    f = 2 * np.pi * (np.arange(n_phi) + 0.5) / n_phi
    z = height * ((np.arange(n_z) + 0.5) / n_z - 0.5)
    F, Z = np.meshgrid(f, z, indexing="ij")
    xyz = np.stack([radius * np.cos(F), radius * np.sin(F), Z], axis=-1).reshape(-1, 3)
    nrm = np.stack([np.cos(F), np.sin(F), np.zeros_like(F)], axis=-1).reshape(-1, 3)
    w = np.full(len(xyz), 2 * np.pi * radius / n_phi * height / n_z)
    rng = np.random.default_rng(seed)
    B = np.stack([np.sin(F) + 0.3 * Z, np.cos(2 * F), 1.0 + 0.1 * Z ** 2], axis=-1).reshape(-1, 3)
    B += 0.01 * rng.normal(size=B.shape)
    return xyz, w, B, nrm


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("fp32", 1e-5)])
def test_direct_bem_integral_matches_restatement(precision, tol):
    dt = np.float64 if precision == "fp64" else np.float32
    plan = Plan(order=4, precision=precision)
    plan.set_bem_sources(*(GOLD[k].astype(dt) for k in ("src", "w", "B", "nrm")))
    plan.set_targets(GOLD["tgt"].astype(dt))
    _, F = plan.direct(1.0, 2)
    assert rel(F, GOLD["direct"]) < tol
    assert rel(F, O.bem_direct(GOLD["src"], GOLD["w"], GOLD["B"], GOLD["nrm"], GOLD["tgt"])) < tol
    with pytest.raises(FmmError):
        plan.direct(1.0, 1)          # B has no meaning for BEM sources
    plan.close()


@pytest.mark.parametrize("p", [4, 10])
def test_device_p2m_matches_restatement(p):
    src, w, B, nrm = (GOLD[k] for k in ("src", "w", "B", "nrm"))
    c, H = G.root_cube(src)
    plan = Plan(order=p, leaf_capacity=1 << 20, precision="fp64", root=(c, H))   # one box: the root
    plan.set_bem_sources(src, w, B, nrm)
    plan.build_tree()
    plan.upward()
    rng = np.random.default_rng(p)
    far = rng.normal(size=(40, 3))
    far = c + far / np.linalg.norm(far, axis=1, keepdims=True) * (6 * H)
    _, F = plan.treecode(far, 1.0, 2)
    M = O.bem_p2m(p, src, w, B, nrm, c, compat=False)
    Fo = np.array([O.eval_expansion(p, M, x - c, regular=False)[0] for x in far]) / (4 * O.REF_PI)
    assert rel(F, Fo) < 1e-12
    plan.close()


@pytest.mark.parametrize("precision,m2l,tol", [("fp64", "simt", 2e-6), ("fp32", "simt", 2e-5), ("fp32", "bf16x3", 3e-5)])
def test_bem_fmm_matches_direct_sum(precision, m2l, tol):
    xyz, w, B, nrm = cylinder_surface()
    rng = np.random.default_rng(8)
    tgt = np.r_[rng.uniform(-1.5, 1.5, size=(1500, 3)), xyz[::7] + 0.01 * nrm[::7]]
    dt = np.float64 if precision == "fp64" else np.float32
    s = FastMultipoleSolver(tuple(a.astype(dt) for a in (xyz, w, B, nrm)), tgt.astype(dt), Problem.BEM,
                            quadratureOctreeLeafCapacity=32, calculationPointOctreeLeafCapacity=32, order=12,
                            precision=precision, m2l=m2l)
    s.calcMultipoleExpansionsAtLeaves()
    s.calclMultipoleExpansions()
    s.calcLocalMultipoleExpansions()
    F = s.calcBEM(1.0)
    Fd = O.bem_direct(xyz, w, B, nrm, tgt)
    assert np.isfinite(F).all()
    assert rel(F, Fd) < tol
    # the full solve gives the same, and the treecode agrees with the direct sum as well
    _, F2 = s.plan.solve(1.0, 2)
    np.testing.assert_array_equal(F2, F)
    _, Ft = s.plan.treecode(tgt.astype(dt), 1.0, 2)
    assert rel(Ft, Fd) < 5 * tol
    s.plan.close()


def test_bem_plan_rules_and_return_to_biot_savart():
    xyz, w, B, nrm = cylinder_surface(16, 8)
    plan = Plan(order=6, leaf_capacity=16, precision="fp64")
    plan.set_bem_sources(xyz, w, B, nrm)
    plan.set_targets(xyz[:50] * 1.3)
    with pytest.raises(FmmError):
        plan.solve(1.0, 1)
    with pytest.raises(FmmError):
        plan.adjoint(np.zeros((50, 3)))
    _, F = plan.solve(1.0, 2)
    assert rel(F, O.bem_direct(xyz, w, B, nrm, xyz[:50] * 1.3)) < 1e-4
    # plain sources make it a Biot-Savart plan again
    J = np.cross(B, nrm)
    plan.set_sources(xyz, w, J)
    Bf, _ = plan.solve(1.0, 1)
    assert rel(Bf, O.direct(xyz, w, J, xyz[:50] * 1.3)) < 1e-4
    plan.close()
