"""Parity of the device pipeline (through the C ABI) with the CPU restatement on the same
inputs, tree and lists. FP64: relative L2 <= 1e-12; FP32: <= 1e-5."""
import numpy as np
import pytest

from bachelors_b200 import FastMultipoleSolver, Plan, geometry as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-5


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def lam_of(L):
    return np.floor(np.sqrt(np.arange(L))).astype(int)


@pytest.mark.parametrize("p", [4, 10, 16])
def test_operator_tables(p):
    plan = Plan(order=p, precision="fp64")
    L = (p + 1) ** 2
    lam = lam_of(L)
    rng = np.random.default_rng(p)
    e = rng.normal(size=(L, 3))
    O._load().orc_set_m2l_extra(p)  # full operator
    for oct_ in (0, 5, 7):
        t = np.array([((oct_ & 1) - 0.5) * 0.5, (((oct_ >> 1) & 1) - 0.5) * 0.5, (((oct_ >> 2) & 1) - 0.5) * 0.5])
        T = plan.operator(0, oct_)
        assert rel(T @ e, O.m2m(p, e * (2.0 ** -lam)[:, None], t)) < FP64_TOL
        T = plan.operator(1, oct_)
        assert rel(T @ e, O.l2l(p, e, -t) * (2.0 ** -(lam + 1))[:, None]) < FP64_TOL
    for o in [(2, 0, 0), (-3, 1, 2), (3, 3, -3), (0, -2, 1)]:
        T = plan.operator(2, (o[0] + 3) + 7 * (o[1] + 3) + 49 * (o[2] + 3))
        assert rel(T @ e, O.m2l(p, e, np.array(o, float))) < FP64_TOL
    plan.close()


def _case(n=(32, 16, 8), m=1500, seed=11, current="poloidal"):
    xyz, w, J = G.torus(*n, 2.0, 0.5, current=current)
    tgt = G.uniform_points(m, -3, 3, seed)
    return xyz, w, J, tgt


def _gpu(xyz, w, J, tgt, p, cap, precision, truncate=False, capT=0):
    s = FastMultipoleSolver((xyz, w, J), tgt, quadratureOctreeLeafCapacity=cap,
                            calculationPointOctreeLeafCapacity=capT or cap, order=p, precision=precision,
                            m2l_truncate=truncate)
    B, A = s.solve(1.0, "AB")
    st = s.stats()
    s.plan.close()
    return np.asarray(B, np.float64), np.asarray(A, np.float64), st


@pytest.mark.parametrize("p,cap", [(4, 8), (8, 16), (12, 32)])
def test_fp64_pipeline_matches_oracle(p, cap):
    xyz, w, J, tgt = _case()
    B, A, st = _gpu(xyz, w, J, tgt, p, cap, "fp64")
    c, H = G.root_cube(xyz, tgt)
    Bo, Ao, so = O.fmm(p, cap, xyz, w, J, tgt, c, H, want_A=True)
    assert st["nodes"] == so["nodes"]
    assert rel(B, Bo) < FP64_TOL
    assert rel(A, Ao) < FP64_TOL


def test_fp64_reference_truncation_matches_oracle():
    xyz, w, J, tgt = _case(m=800)
    B, A, _ = _gpu(xyz, w, J, tgt, 10, 16, "fp64", truncate=True)
    c, H = G.root_cube(xyz, tgt)
    Bo, Ao, _ = O.fmm(10, 16, xyz, w, J, tgt, c, H, want_A=True, truncate=True)
    assert rel(B, Bo) < FP64_TOL
    assert rel(A, Ao) < FP64_TOL


@pytest.mark.parametrize("p,cap", [(8, 16), (12, 64)])
def test_fp32_pipeline_matches_oracle(p, cap):
    xyz, w, J, tgt = _case(n=(64, 16, 16), m=3000)
    x32, w32, J32, t32 = (a.astype(np.float32) for a in (xyz, w, J, tgt))
    B, A, _ = _gpu(x32, w32, J32, t32, p, cap, "fp32")
    c, H = G.root_cube(x32.astype(np.float64), t32.astype(np.float64))
    Bo, Ao, _ = O.fmm(p, cap, x32, w32, J32, t32, c, H, want_A=True)
    assert rel(B, Bo) < FP32_TOL
    assert rel(A, Ao) < FP32_TOL


def test_separate_target_capacity_and_azimuthal_current():
    xyz, w, _, tgt = _case(m=1000, current="azimuthal")
    B, A, _ = _gpu(xyz, w, None, tgt, 6, 24, "fp64", capT=8)
    c, H = G.root_cube(xyz, tgt)
    Bo, Ao, _ = O.fmm(6, 24, xyz, w, None, tgt, c, H, want_A=True, cap_tgt=8)
    assert rel(B, Bo) < FP64_TOL
    assert rel(A, Ao) < FP64_TOL


def test_targets_equal_sources_excludes_self():
    xyz, w, J = G.torus(24, 12, 8, 2.0, 0.5)
    B, A, _ = _gpu(xyz, w, J, xyz, 8, 16, "fp64")
    c, H = G.root_cube(xyz, xyz)
    Bo, Ao, _ = O.fmm(8, 16, xyz, w, J, xyz, c, H, want_A=True)
    assert np.isfinite(B).all()
    assert rel(B, Bo) < FP64_TOL
    Bd = O.direct(xyz, w, J, xyz)
    assert rel(B, Bd) < 1e-4


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("fp32", 1e-5)])
def test_direct_matches_oracle(precision, tol):
    xyz, w, J, tgt = _case(n=(16, 8, 4), m=300)
    dt = np.float64 if precision == "fp64" else np.float32
    x, ww, JJ, t = (a.astype(dt) for a in (xyz, w, J, tgt))
    plan = Plan(order=2, precision=precision)
    plan.set_sources(x, ww, JJ)
    plan.set_targets(t)
    B, A = plan.direct(2.5, 3)
    Bo, Ao = O.direct(x, ww, JJ, t, current=2.5, want_A=True)
    assert rel(B, Bo) < tol and rel(A, Ao) < tol
    B64 = plan.direct_fp64(t[:50].astype(np.float64), current=2.5)
    assert rel(B64, Bo[:50]) < (1e-13 if precision == "fp64" else 1e-6)
    plan.close()


def test_tiny_and_ragged_inputs():
    rng = np.random.default_rng(3)
    # one source, one target
    B, A, _ = _gpu(np.array([[0.1, 0.2, 0.3]]), np.array([0.5]), np.array([[0.0, 0.0, 1.0]]),
                   np.array([[1.0, -1.0, 0.5]]), 4, 8, "fp64")
    Bo = O.direct(np.array([[0.1, 0.2, 0.3]]), np.array([0.5]), np.array([[0.0, 0.0, 1.0]]), np.array([[1.0, -1.0, 0.5]]))
    assert rel(B, Bo) < FP64_TOL
    # everything in one leaf
    xyz = rng.normal(size=(20, 3))
    tgt = rng.normal(size=(7, 3))
    w = rng.uniform(0.1, 1, 20)
    J = rng.normal(size=(20, 3))
    B, A, _ = _gpu(xyz, w, J, tgt, 6, 64, "fp64")
    assert rel(B, O.direct(xyz, w, J, tgt)) < 1e-13
    # clustered sources (deep tree) next to a coarse region
    xyz = np.r_[rng.normal(size=(3000, 3)) * 1e-4, rng.uniform(-1, 1, size=(500, 3))]
    w = rng.uniform(0.1, 1, len(xyz))
    J = rng.normal(size=(len(xyz), 3))
    tgt = np.r_[rng.normal(size=(400, 3)) * 1e-4, rng.uniform(-1, 1, size=(400, 3))]
    B, A, st = _gpu(xyz, w, J, tgt, 6, 16, "fp64")
    c, H = G.root_cube(xyz, tgt)
    Bo, Ao, so = O.fmm(6, 16, xyz, w, J, tgt, c, H, want_A=True)
    assert st["levels"] > 8
    assert rel(B, Bo) < FP64_TOL and rel(A, Ao) < FP64_TOL


def test_device_resident_inputs_match_host_inputs():
    import torch
    xyz, w, J, tgt = _case(m=1000)
    x32, w32, J32, t32 = (a.astype(np.float32) for a in (xyz, w, J, tgt))
    Bh, _, _ = _gpu(x32, w32, J32, t32, 8, 32, "fp32")
    dev = [torch.from_numpy(a).cuda() for a in (x32, w32, J32, t32)]
    s = FastMultipoleSolver(tuple(dev[:3]), dev[3], quadratureOctreeLeafCapacity=32,
                            calculationPointOctreeLeafCapacity=32, order=8, precision="fp32")
    Bd = s.solve(1.0, "B")
    assert isinstance(Bd, torch.Tensor) and Bd.is_cuda
    np.testing.assert_array_equal(Bd.cpu().numpy(), Bh.astype(np.float32))


def test_reference_call_sequence():
    xyz, w, J, tgt = _case(m=500)
    s = FastMultipoleSolver((xyz, w, J), tgt, quadratureOctreeLeafCapacity=16, calculationPointOctreeLeafCapacity=16,
                            order=8, precision="fp64")
    with pytest.raises(RuntimeError):
        s.calcLocalMultipoleExpansions()
    s.calcMultipoleExpansionsAtLeaves()
    s.calclMultipoleExpansions()
    s.calcLocalMultipoleExpansions()
    B = s.calcB(3.0)
    A = s.calcA(3.0)
    c, H = G.root_cube(xyz, tgt)
    Bo, Ao, _ = O.fmm(8, 16, xyz, w, J, tgt, c, H, current=3.0, want_A=True)
    assert rel(B, Bo) < FP64_TOL and rel(A, Ao) < FP64_TOL
