"""The GPU direct sum and FMM on the reference's Keast torus at the Telma points (see
tests/test_oracle_telma.py), against the reference's own FP64 direct sum: the direct sums to
rounding, the FMM (p = 12) to its truncation error."""
import os

import numpy as np
import pytest

from bachelors_b200 import Plan, geometry as G

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_telma.npz")


@pytest.mark.parametrize("precision,kind,tol", [("fp64", "direct", 1e-13), ("fp64", "fmm", 2e-6),
                                                ("fp32", "direct", 1e-5), ("fp32", "fmm", 1e-5)])
def test_telma_points(precision, kind, tol):
    g = dict(np.load(GOLDEN))
    xyz, w = G.tetra_quadratures(G.hex_torus_tetrahedra(2.0, 0.2, 20, 4, 4), g["rule_x"], g["rule_w"])
    dt = np.float64 if precision == "fp64" else np.float32
    plan = Plan(order=12, leaf_capacity=32, precision=precision, m2l="bf16x3" if precision == "fp32" else "simt")
    plan.set_sources(xyz.astype(dt), w.astype(dt), None)       # J = NULL: the reference's azimuthal current
    plan.set_targets(g["telma_points"].astype(dt))
    B, _ = plan.direct(5.0, 1) if kind == "direct" else plan.solve(5.0, 1)
    ref = g["direct_B_current5"]
    assert np.linalg.norm(B - ref) / np.linalg.norm(ref) < tol
    plan.close()
