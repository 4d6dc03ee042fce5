"""The header-only C++ facade (include/fmm_facade.hpp) that keeps the reference's C++ names:
it compiles and links against libfmmcuda.so in both `real` builds (CPU), and on the GPU it gives
the same numbers as the Python mirror of the same calls."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "bachelors_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "facade_check.cpp")


def _compile(out, double):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    if not os.path.exists(os.path.join(LIB_DIR, "libfmmcuda.so")):
        pytest.skip("libfmmcuda.so not built")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", LIB_DIR, "-lfmmcuda", f"-Wl,-rpath,{LIB_DIR}", "-o", out]
    if double:
        cmd.insert(1, "-DFMM_REAL_IS_DOUBLE")
    subprocess.run(cmd, check=True, capture_output=True, text=True)


@pytest.mark.parametrize("double", [False, True])
def test_facade_compiles_and_links(tmp_path, double):
    _compile(str(tmp_path / "facade_check"), double)
    assert os.path.exists(tmp_path / "facade_check")


@pytest.mark.gpu
@pytest.mark.parametrize("double", [False, True])
def test_facade_matches_python_mirror(tmp_path, double):
    import torch  # noqa: F401  (CUDA context in this process for the Python side)
    from bachelors_b200 import Plan, geometry as G, kernels as K
    from oracle import oracle as O
    exe = str(tmp_path / "facade_check")
    _compile(exe, double)
    dt = np.float64 if double else np.float32
    xyz, w, _ = G.torus(48, 12, 6, 2.0, 0.5)
    pts = G.uniform_points(1500, -3, 3, 11)
    np.c_[xyz, w].astype(dt).tofile(tmp_path / "quads.bin")
    pts.astype(dt).tofile(tmp_path / "points.bin")
    p, count = 6, 40
    L = (p + 1) ** 2
    rng = np.random.default_rng(3)
    harm = np.stack([O.solid_harmonics(p, t, True, compat=True) for t in rng.normal(size=(count, 3)) * 0.3])
    expn = rng.normal(size=(count, L, 3))
    np.concatenate([[count, p], harm.ravel(), expn.ravel()]).astype(dt).tofile(tmp_path / "seam.bin")
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    B = np.fromfile(tmp_path / "fmm_B.bin", dtype=dt).reshape(-1, 3)
    # the same phases through the Python mirror: leaf capacity 33 in the reference's sense = 32 here
    plan = Plan(order=10, leaf_capacity=32, target_leaf_capacity=32, precision="fp64" if double else "fp32")
    plan.set_sources(xyz.astype(dt), w.astype(dt), None)
    plan.set_targets(pts.astype(dt))
    Bp, _ = plan.solve(1.0, 1)
    assert np.array_equal(B, Bp)
    D = np.fromfile(tmp_path / "direct_B.bin", dtype=dt).reshape(-1, 3)
    Dref = O.direct(xyz, w, None, pts[:4])
    assert np.linalg.norm(D - Dref) / np.linalg.norm(Dref) < (1e-12 if double else 1e-5)
    seam = np.fromfile(tmp_path / "seam_out.bin", dtype=dt).reshape(count, L, 3)
    assert np.array_equal(seam, K.translateAllGPU(harm.astype(dt), expn.astype(dt)))
    bmat = np.eye(L) + np.eye(L, k=1)
    mat = np.fromfile(tmp_path / "matrix_out.bin", dtype=dt).reshape(3, count, L)
    ref = np.stack([O.translate_all_matrix(expn[:, :, c], bmat) for c in range(3)])
    assert np.linalg.norm(mat - ref) / np.linalg.norm(ref) < (1e-14 if double else 1e-6)
    plan.close()
    # MultipoleSolver::calcB(current, point): the treecode on the source tree (standard mode), current 2
    TB = np.fromfile(tmp_path / "tree_B.bin", dtype=dt).reshape(-1, 3)
    tp = Plan(order=10, leaf_capacity=32, precision="fp64" if double else "fp32")
    tp.set_sources(xyz.astype(dt), w.astype(dt), None)
    tp.build_tree()
    tp.upward()
    Tref, _ = tp.treecode(pts[:8].astype(dt), 2.0, 1)
    assert np.array_equal(TB, Tref)
    Td = O.direct(xyz, w, None, pts[:8], current=2.0)
    assert np.linalg.norm(TB - Td) / np.linalg.norm(Td) < 1e-4
    tp.close()
    # calcBEM: sources = the quadratures with B = (1, 2, 3) and normal = z
    BF = np.fromfile(tmp_path / "bem.bin", dtype=dt).reshape(-1, 3)
    Bq = np.tile([1.0, 2.0, 3.0], (len(w), 1))
    Nq = np.tile([0.0, 0.0, 1.0], (len(w), 1))
    Fd = O.bem_direct(xyz, w, Bq, Nq, pts)
    assert np.linalg.norm(BF - Fd) / np.linalg.norm(Fd) < (1e-5 if double else 3e-5)
