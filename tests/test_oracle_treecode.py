"""The reference's treecode (MultipoleSolver::calcB: one source octree, multipoles only, close leaves
dropped) restated in the oracle, against vectors the reference produced
(tests/golden/reference_treecode.npz, made by tests/golden/make_golden.py treecode). Far from the
sources nothing is dropped, and the treecode meets the direct sum there to the expansion's truncation."""
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "reference_treecode.npz"))


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("p,cap", [(10, 16), (12, 32)])
def test_treecode_matches_reference(p, cap):
    xyzw = G["xyzw"]
    B = O.treecode_B(p, cap, xyzw[:, :3], xyzw[:, 3], G["pts"], 1.0)
    assert rel(B, G[f"B_p{p}_cap{cap}"]) < 1e-12


def test_treecode_far_points_meet_direct_sum():
    xyzw = G["xyzw"]
    far = G["pts"][16:]
    B = O.treecode_B(10, 16, xyzw[:, :3], xyzw[:, 3], far, 1.0)
    Bd = O.direct(xyzw[:, :3], xyzw[:, 3], None, far)
    assert rel(B, Bd) < 1e-5
