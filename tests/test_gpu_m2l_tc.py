"""The tensor-core (tcgen05) M2L against the CUDA-core FP32 M2L and the FP64 oracle on the same
tree. BF16X3 (hi + lo, three products) keeps ~16 bits per product: rel L2 <= 2e-5 against the
oracle. BF16X6 (hi + mid + lo, six products) keeps FP32-level products: rel L2 <= 1e-5, the
FP32 pipeline tolerance. TF32 (one pass on operands rounded to 11 significant bits) is the fast,
coarse mode: rel L2 <= 2e-3."""
import numpy as np
import pytest

from bachelors_b200 import FastMultipoleSolver, geometry as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TC_TOL = {"bf16x3": 2e-5, "bf16x6": 1e-5, "tf32": 2e-3}


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def solve(x, w, J, t, p, cap, m2l):
    s = FastMultipoleSolver((x, w, J), t, quadratureOctreeLeafCapacity=cap, calculationPointOctreeLeafCapacity=cap,
                            order=p, precision="fp32", m2l=m2l)
    B, A = s.solve(1.0, "AB")
    s.plan.close()
    return np.asarray(B, np.float64), np.asarray(A, np.float64)


@pytest.mark.parametrize("mode", ["bf16x3", "bf16x6", "tf32"])
@pytest.mark.parametrize("p,cap", [(4, 16), (8, 16), (12, 32), (16, 32)])
def test_split_bf16_matches_fp32_and_oracle(p, cap, mode):
    xyz, w, J = G.torus(64, 16, 16, 2.0, 0.5)
    tgt = G.uniform_points(3000, -3, 3, 17)
    x, ww, JJ, t = (a.astype(np.float32) for a in (xyz, w, J, tgt))
    Btc, Atc = solve(x, ww, JJ, t, p, cap, mode)
    Bs, As = solve(x, ww, JJ, t, p, cap, "simt")
    c, H = G.root_cube(x.astype(np.float64), t.astype(np.float64))
    Bo, Ao, _ = O.fmm(p, cap, x, ww, JJ, t, c, H, want_A=True)
    assert np.isfinite(Btc).all()
    assert rel(Btc, Bo) < TC_TOL[mode] and rel(Atc, Ao) < TC_TOL[mode]
    assert rel(Btc, Bs) < TC_TOL[mode]


@pytest.mark.parametrize("mode", ["bf16x3", "bf16x6", "tf32"])
def test_split_bf16_repeatable(mode):
    xyz, w, J = G.torus(32, 16, 8, 2.0, 0.5)
    x, ww, JJ = (a.astype(np.float32) for a in (xyz, w, J))
    B1, _ = solve(x, ww, JJ, x, 10, 32, mode)
    B2, _ = solve(x, ww, JJ, x, 10, 32, mode)
    np.testing.assert_array_equal(B1, B2)


@pytest.mark.parametrize("translate", ["0", "1", "3"])
@pytest.mark.parametrize("mode", ["bf16x3", "bf16x6", "tf32"])
def test_translation_forms_match_oracle(monkeypatch, translate, mode):
    """M2M / L2L forms (read when a plan is created): 0 both on the CUDA cores, 1 M2M on the tensor
    cores (the default), 3 both on the tensor cores."""
    monkeypatch.setenv("FMM_TC_TRANSLATE", translate)
    xyz, w, J = G.torus(64, 16, 16, 2.0, 0.5)
    tgt = G.uniform_points(2000, -3, 3, 23)
    x, ww, JJ, t = (a.astype(np.float32) for a in (xyz, w, J, tgt))
    B, A = solve(x, ww, JJ, t, 12, 32, mode)
    c, H = G.root_cube(x.astype(np.float64), t.astype(np.float64))
    Bo, Ao, _ = O.fmm(12, 32, x, ww, JJ, t, c, H, want_A=True)
    assert rel(B, Bo) < TC_TOL[mode] and rel(A, Ao) < TC_TOL[mode]
