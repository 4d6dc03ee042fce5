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


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-14), ("fp32", 1e-6)])
def test_device_generated_torus_matches_host_generator(precision, tol):
    """fmm_torus_quadratures builds the same Keast torus on the GPU as the host generator (itself equal to
    the reference's quadratures, tests/test_oracle_telma.py), and the solver takes it straight from device
    memory: the Telma-point field equals the solve from host inputs."""
    g = dict(np.load(GOLDEN))
    hx, hw = G.tetra_quadratures(G.hex_torus_tetrahedra(2.0, 0.2, 20, 4, 4), g["rule_x"], g["rule_w"])
    dx, dw = G.tetra_torus_quadratures_device(2.0, 0.2, 20, 4, 4, g["rule_x"], g["rule_w"], precision)
    assert dx.shape == hx.shape and dw.shape == hw.shape
    ex = np.abs(dx.cpu().numpy() - hx).max() / np.abs(hx).max()
    ew = np.abs(dw.cpu().numpy() - hw).max() / np.abs(hw).max()
    assert ex < tol and ew < tol
    import torch
    dt = np.float64 if precision == "fp64" else np.float32
    plan = Plan(order=12, leaf_capacity=32, precision=precision)
    plan.set_sources(dx, dw, None)
    plan.set_targets(torch.tensor(g["telma_points"].astype(dt), device="cuda"))
    B, _ = plan.direct(5.0, 1)
    ref = g["direct_B_current5"]
    assert np.linalg.norm(B.cpu().numpy() - ref) / np.linalg.norm(ref) < (1e-13 if precision == "fp64" else 1e-5)
    plan.close()
    # a finer mesh than the reference's (20 x 4 x 4): 16 times the tetrahedra, all on the device
    fx, fw = G.tetra_torus_quadratures_device(2.0, 0.2, 80, 8, 8, g["rule_x"], g["rule_w"], precision)
    assert fx.shape[0] == 80 * 8 * 8 * 5 * len(g["rule_w"])
    vol = 2 * np.pi * 2.0 * 0.2 * 0.2   # the square-section torus's volume; the polygonal mesh is slightly smaller
    assert abs(fw.sum().item() / vol - 1) < 2e-3
    with pytest.raises(Exception):
        G.tetra_torus_quadratures_device(2.0, 0.2, 20, 4, 4, np.zeros((65, 3)), np.zeros(65), precision)
