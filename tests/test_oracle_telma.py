"""The reference's known-answer case (FMM/FMMGPU/main.cpp:50-134): the tetrahedral torus of
createTorus() with the 24-point Keast rule, its direct Biot-Savart field (current 5) at the 100 points
of results/telma_results.txt, and Telma's own H there (tests/golden/make_golden.py telma).

* bachelors_b200.geometry rebuilds the reference's quadratures (hexahedra -> tetrahedra -> rule points)
  to rounding;
* the oracle's direct sum on them equals the reference's direct sum to 1e-14;
* against Telma's field (H x MU0) the agreement is what the reference reports, percent-level: Telma
  integrates its own way (1.4 % mean, 2.6 % worst point here)."""
import os

import numpy as np
import pytest

from bachelors_b200 import geometry as G
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_telma.npz")
MU0 = 1.2566370614e-6


@pytest.fixture(scope="module")
def telma():
    return dict(np.load(GOLDEN))


@pytest.fixture(scope="module")
def quads(telma):
    return G.tetra_quadratures(G.hex_torus_tetrahedra(2.0, 0.2, 20, 4, 4), telma["rule_x"], telma["rule_w"])


def test_generator_reproduces_reference_quadratures(telma, quads):
    xyz, w = quads
    assert len(w) == int(telma["quad_count"]) == 20 * 4 * 4 * 5 * 24
    mine = np.c_[xyz, w]
    ref = telma["quad_sample"]
    np.testing.assert_allclose(mine[telma["quad_sample_index"]], ref, rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(mine.sum(axis=0), telma["quad_sums"], rtol=1e-12, atol=1e-12)


def test_oracle_direct_equals_reference_direct(telma, quads):
    xyz, w = quads
    B = O.direct(xyz, w, None, telma["telma_points"], current=5.0)
    ref = telma["direct_B_current5"]
    assert np.linalg.norm(B - ref) / np.linalg.norm(ref) < 1e-14


def test_agreement_with_telma_is_the_references(telma, quads):
    xyz, w = quads
    B = O.direct(xyz, w, None, telma["telma_points"], current=5.0)
    T = telma["telma_H"] * MU0
    pct = 100 * np.linalg.norm(B - T, axis=1) / np.linalg.norm(T, axis=1)
    assert pct.mean() < 2.0 and pct.max() < 3.0
