"""Tree statistics reported by fmm_get_stats against the oracle's count of the same tree: boxes,
leaves and the direct (target, source) pairs that the near field evaluates."""
import numpy as np
import pytest

from bachelors_b200 import FastMultipoleSolver, geometry as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("p,cap", [(4, 8), (8, 32)])
def test_stats_match_oracle_counts(p, cap):
    xyz, w, J = G.torus(32, 16, 8, 2.0, 0.5)
    tgt = G.uniform_points(1500, -3, 3, 11)
    s = FastMultipoleSolver((xyz, w, J), tgt, quadratureOctreeLeafCapacity=cap,
                            calculationPointOctreeLeafCapacity=cap, order=p, precision="fp64")
    s.solve(1.0, "B")
    st = s.stats()
    s.plan.close()
    c, H = G.root_cube(xyz, tgt)
    _, _, so = O.fmm(p, cap, xyz, w, J, tgt, c, H)
    assert st["nodes"] == so["nodes"]
    assert st["leaves"] == so["leaves"]
    assert 0 < st["v_pairs"] <= so["V"]    # the oracle also lists pairs whose boxes hold no points
    assert st["p2p_interactions"] == so["direct_pairs"]
    assert len(tgt) <= st["p2p_interactions"] <= len(tgt) * len(xyz)


def test_single_leaf_counts():
    xyz, w, J = G.torus(6, 4, 2, 2.0, 0.5)           # 48 points, one leaf of capacity 64
    s = FastMultipoleSolver((xyz, w, J), xyz, quadratureOctreeLeafCapacity=64,
                            calculationPointOctreeLeafCapacity=64, order=4, precision="fp64")
    s.solve(1.0, "B")
    st = s.stats()
    s.plan.close()
    assert st["leaves"] == 1 and st["p2p_pairs"] == 1
    assert st["p2p_interactions"] == 48 * 48
