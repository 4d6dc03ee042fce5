"""The tree levels built in one cooperative launch (kBuildLevels: work queues per level, a decoupled look-back
for the child numbering, one grid barrier per level) against the level-by-level build (three launches and a
host wait per level): the same forest, so the same statistics and bit-identical fields. The batch's first
build outgrows the node capacity guessed from the point counts, so it also runs the overflow-and-rebuild
path; the second build on the same plan starts from the grown capacity."""
import os

import numpy as np
import pytest

from bachelors_b200 import Plan, geometry as G

pytestmark = pytest.mark.gpu

KEYS = ("nodes", "leaves", "levels", "v_pairs", "p2p_pairs", "p2p_interactions")


def _solve(persistent, build, var="FMM_TREE_PERSISTENT", on="1"):
    old = os.environ.get(var)
    os.environ[var] = on if persistent else "0"
    try:
        plan, load = build()
    finally:
        if old is None:
            del os.environ[var]
        else:
            os.environ[var] = old
    out = []
    for _ in range(2):
        load(plan)   # new inputs: the next solve builds the forest again
        B, _ = plan.solve(1.0, 1)
        st = plan.stats()
        out.append((np.array(B, copy=True), {k: st[k] for k in KEYS}))
    plan.close()
    return out


def _single():
    xyz, w, J = G.torus(64, 16, 16, 2.0, 0.5)
    tgt = G.uniform_points(3000, -3, 3, 5)

    def load(plan):
        plan.set_sources(xyz, w, J)
        plan.set_targets(tgt)
    return Plan(order=8, leaf_capacity=16, precision="fp64"), load


def _batch():
    xyz, w, J, tgt, so, to = G.torus_batch(12, seed=7, count_range=(2 ** 8, 2 ** 12), targets_per_coil=256)
    f32 = lambda a: a.astype(np.float32)

    def load(plan):
        plan.set_sources(f32(xyz), f32(w), f32(J))
        plan.set_targets(f32(tgt))
        plan.set_coils(so, to)
    return Plan(order=6, leaf_capacity=8, precision="fp32", m2l="bf16x3"), load


@pytest.mark.parametrize("build", [_single, _batch], ids=["fp64-single", "fp32-batch"])
def test_persistent_levels_equal_level_by_level(build):
    per_level = _solve(False, build)
    persistent = _solve(True, build)
    for (Bp, sp), (Bl, sl) in zip(persistent, per_level):
        assert sp == sl
        assert sp["levels"] > 3
        assert np.all(np.isfinite(Bp))
        assert np.array_equal(Bp, Bl)


@pytest.mark.parametrize("build", [_single, _batch], ids=["fp64-single", "fp32-batch"])
def test_warp_lists_equal_thread_lists(build):
    """The interaction lists built with one warp per box (ballot appends in candidate order) equal the lists
    built with one thread per box: the same statistics and bit-identical fields."""
    per_thread = _solve(False, build, "FMM_LISTS_WARP")
    per_warp = _solve(True, build, "FMM_LISTS_WARP", on="2")   # (2: a warp per box for batches as well)
    for (Bw, sw), (Bt, st) in zip(per_warp, per_thread):
        assert sw == st
        assert np.array_equal(Bw, Bt)
