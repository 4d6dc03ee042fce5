"""Parity at the benchmark's own problem sizes (not only at small test sizes).

* The plain FP64 workload in full: a 128 x 32 x 16 = 65,536-point torus (R = 2, a = 0.5) carrying the
  reference's azimuthal current (J = NULL, FMM/FMMGPU/integration.cpp:155), targets on the 32^3 grid on
  [-3, 3]^3, p = 10, leaf 32, FP64 on the GPU against the CPU restatement on the same tree and lists:
  relative L2 <= 1e-12 for B and A, and the same tree.
* The plain FP32 workload's pipeline (2^20-point torus, 256 x 64 x 64, poloidal current, p = 12, leaf 64)
  on a seeded 2^16-target subset of its uniform targets in [-3, 3]^3, against the restatement of the same
  FP32 inputs: relative L2 <= 1e-5, for the CUDA-core and the split-BF16 tensor-core M2L.
"""
import numpy as np
import pytest

from bachelors_b200 import Plan, geometry as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-5


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_fp64_grid_workload_full_size_matches_oracle():
    xyz, w, _ = G.torus(128, 32, 16, 2.0, 0.5, current="azimuthal")
    tgt = G.cube_grid(32, -3.0, 3.0)
    assert len(xyz) == 65536 and len(tgt) == 32768
    plan = Plan(order=10, leaf_capacity=32, precision="fp64")
    plan.set_sources(xyz, w, None)
    plan.set_targets(tgt)
    B, A = plan.solve(1.0, 3)
    st = plan.stats()
    plan.close()
    c, H = G.root_cube(xyz, tgt)
    Bo, Ao, so = O.fmm(10, 32, xyz, w, None, tgt, c, H, want_A=True)
    assert st["nodes"] == so["nodes"] and st["levels"] == so["levels"] and st["leaves"] == so["leaves"]
    assert st["p2p_interactions"] == so["direct_pairs"]
    assert 0 < st["v_pairs"] <= so["V"]    # the oracle also lists pairs whose boxes hold no points
    assert rel(B, Bo) < FP64_TOL
    assert rel(A, Ao) < FP64_TOL


@pytest.fixture(scope="module")
def fp32_2e20_case():
    """The 2^20-source FP32 inputs, a seeded 2^16-target subset, and the restatement's B there (the
    oracle's FP64 FMM of the FP32 inputs, tens of seconds on the host: computed once)."""
    xyz, w, J = G.torus(256, 64, 64, 2.0, 0.5, current="poloidal")
    x32, w32, J32 = (a.astype(np.float32) for a in (xyz, w, J))
    tgt = G.uniform_points(1 << 20, -3.0, 3.0, 20260002).astype(np.float32)
    sub = np.sort(np.random.default_rng(20260002).choice(len(tgt), size=1 << 16, replace=False))
    t32 = tgt[sub]
    c, H = G.root_cube(x32.astype(np.float64), t32.astype(np.float64))
    Bo, _, so = O.fmm(12, 64, x32, w32, J32, t32, c, H)
    return x32, w32, J32, t32, Bo, so


@pytest.mark.parametrize("m2l", ["simt", "bf16x3"])
def test_fp32_2e20_workload_subset_matches_oracle(fp32_2e20_case, m2l):
    x32, w32, J32, t32, Bo, so = fp32_2e20_case
    plan = Plan(order=12, leaf_capacity=64, precision="fp32", m2l=m2l)
    plan.set_sources(x32, w32, J32)
    plan.set_targets(t32)
    B, _ = plan.solve(1.0, 1)
    st = plan.stats()
    plan.close()
    assert st["nodes"] == so["nodes"] and st["leaves"] == so["leaves"]
    assert st["p2p_interactions"] == so["direct_pairs"]
    assert np.isfinite(B).all()
    assert rel(B, Bo) < FP32_TOL
