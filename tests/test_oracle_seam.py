"""The oracle's restatement of the reference's translation seam (kernels::translateAllCPU,
translateAllCPUMatrixBLAS; FMM/FMMGPU/translation_algorithms_cpu.cpp:9-135) against golden vectors
produced by the reference itself (tests/golden/make_golden.py seam)."""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_seam.npz")


@pytest.fixture(scope="module")
def seam():
    return dict(np.load(GOLDEN))


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("p", (1, 4, 10, 16))
def test_translate_all(seam, p):
    got = O.translate_all(p, seam[f"ta_p{p}_a"], seam[f"ta_p{p}_b"])
    assert rel(got, seam[f"ta_p{p}_out"]) < 1e-14


@pytest.mark.parametrize("p", (1, 4, 10))
def test_translate_all_matrix(seam, p):
    got = O.translate_all_matrix(seam[f"tam_p{p}_a"], seam[f"tam_p{p}_b"])
    assert rel(got, seam[f"tam_p{p}_out"]) < 1e-14


@pytest.mark.parametrize("p", (4, 10, 16))
def test_translate_all_is_m2m_up_to_the_short_literal(seam, p):
    # the real-form seam and the complex-form M2M agree except for the reference's
    # R_SQRT_2 = 0.70710678118 literal (relative 1e-11)
    a, b = seam[f"ta_p{p}_a"], seam[f"ta_p{p}_b"]
    out = seam[f"ta_p{p}_out"]
    # recover the translation vector from the degree-1 regular harmonics: R_1^0 = -z, and the
    # real-form (1, +-1) entries carry x and y up to the convention's factors
    for i in range(len(a)):
        t = _translation_from_regular(p, a[i])
        assert rel(O.m2m(p, b[i], t, compat=True), out[i]) < 1e-10


def _translation_from_regular(p, a):
    """Translation vector whose regular harmonics are `a` (found by matching degree 1)."""
    base = O.solid_harmonics(p, np.array([1.0, 0, 0]), True, compat=True)[1:4]
    basey = O.solid_harmonics(p, np.array([0, 1.0, 0]), True, compat=True)[1:4]
    basez = O.solid_harmonics(p, np.array([0, 0, 1.0]), True, compat=True)[1:4]
    M = np.stack([base, basey, basez], axis=1)   # degree-1 harmonics are linear in (x, y, z)
    t = np.linalg.lstsq(M, a[1:4], rcond=None)[0]
    assert rel(O.solid_harmonics(p, t, True, compat=True), a) < 1e-9
    return t
