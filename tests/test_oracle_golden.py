"""The CPU restatement (oracle) against golden vectors produced by the reference itself
(tests/golden/make_golden.py). Compat mode reproduces the reference's arithmetic quirks, so
agreement is at rounding level."""
import numpy as np
import pytest

from oracle import oracle as O

ORDERS = (4, 10, 16)


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("p", ORDERS)
def test_harmonics(golden, p):
    for x, r, i in zip(golden[f"harm_p{p}_x"], golden[f"harm_p{p}_regular"], golden[f"harm_p{p}_irregular"]):
        assert rel(O.solid_harmonics(p, x, True, compat=True), r) < 1e-13
        assert rel(O.solid_harmonics(p, x, False, compat=True), i) < 1e-13


@pytest.mark.parametrize("p", ORDERS)
@pytest.mark.parametrize("op", ["m2m", "m2l", "l2l"])
def test_translations(golden, p, op):
    fn = getattr(O, op)
    for e, t, ref in zip(golden[f"{op}_p{p}_in"], golden[f"{op}_p{p}_t"], golden[f"{op}_p{p}_out"]):
        assert rel(fn(p, e, t, compat=True), ref) < 1e-12


@pytest.mark.parametrize("p", ORDERS)
def test_p2m(golden, p):
    xyzw = golden[f"p2m_p{p}_xyzw"]
    got = O.p2m(p, xyzw[:, :3], xyzw[:, 3], None, golden[f"p2m_p{p}_center"], compat=True)
    assert rel(got, golden[f"p2m_p{p}_out"]) < 1e-12


@pytest.mark.parametrize("p", ORDERS)
def test_eval_local(golden, p):
    A, _ = O.eval_expansion(p, golden[f"eval_p{p}_local"], golden[f"eval_p{p}_d"], regular=True, compat=True)
    assert rel(A, golden[f"eval_p{p}_out"]) < 1e-12


def test_direct(golden):
    xyzw = golden["direct_xyzw"]
    B = O.direct(xyzw[:, :3], xyzw[:, 3], None, golden["direct_tgt"], current=5.0)
    assert rel(B, golden["direct_B"]) < 1e-13


def test_standard_mode_differs_only_in_reference_quirks(golden):
    # standard mode keeps the complex phase at m = p (the reference skips it, harmonics.cpp:189)
    p = 10
    x = golden[f"harm_p{p}_x"][0]
    std = O.solid_harmonics(p, x, True, compat=False)
    ref = golden[f"harm_p{p}_regular"][0]
    top = [p * p + p + p, p * p]  # (p, p) and (p, -p)
    mask = np.ones(len(std), bool)
    mask[top] = False
    assert rel(std[mask], ref[mask]) < 1e-12
    assert rel(std[top], ref[top]) > 1e-3


def test_reference_fmm_accuracy_recorded(golden):
    # The reference's own FMM (p = 10, FP64) on targets at radius 5 around the torus, against
    # its own direct sum. Its dual-tree MAC and near-field handling make it inaccurate here
    # (about 15 %); the value is recorded by the fixture. The standard-mode pipeline (full M2L
    # operator, direct near field) on the same inputs is far more accurate.
    err_ref = rel(golden["fmm_B"], golden["fmm_direct_B"])
    xyzw = golden["fmm_xyzw"]
    tgt = golden["fmm_tgt"]
    from bachelors_b200 import geometry
    c, H = geometry.root_cube(xyzw[:, :3], tgt)
    B, _, _ = O.fmm(10, 32, xyzw[:, :3], xyzw[:, 3], None, tgt, c, H)
    err = rel(B, golden["fmm_direct_B"])
    assert err < 1e-4
    assert err < err_ref / 100
