"""Generates the golden vectors in tests/golden/ from the reference itself.

Runs the patched reference build (oracle/_ref/libref_fmm_*.so, made by oracle/ref/build_ref.sh
from the reference sources) on seeded inputs and stores inputs and outputs as .npz. The
reference is not needed afterwards: the tests read only the .npz files.

Usage: python tests/golden/make_golden.py [main] [seam] [telma] [bem] [treecode]   (default: all)
The reference sources are read from REFERENCE_ROOT (default /root/reference).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("REFERENCE_ROOT", "/root/reference")
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from oracle.oracle import Reference  # noqa: E402
from bachelors_b200 import geometry  # noqa: E402


def main():
    rng = np.random.default_rng(20260001)
    ref = Reference("f64", 10)
    out = {}
    for p in (4, 10, 16):
        pts = rng.normal(size=(6, 3)) * rng.uniform(0.2, 3.0, size=(6, 1))
        out[f"harm_p{p}_x"] = pts
        out[f"harm_p{p}_regular"] = np.stack([ref.regular(p, x) for x in pts])
        out[f"harm_p{p}_irregular"] = np.stack([ref.irregular(p, x) for x in pts])
        L = (p + 1) ** 2
        for name, scale in (("m2m", 0.3), ("m2l", 3.0), ("l2l", 0.3)):
            e = rng.normal(size=(2, L, 3))
            t = rng.normal(size=(2, 3)) * scale
            out[f"{name}_p{p}_in"] = e
            out[f"{name}_p{p}_t"] = t
            out[f"{name}_p{p}_out"] = np.stack([getattr(ref, name)(p, e[i], t[i]) for i in range(2)])
        q = rng.normal(size=(24, 3)) * 0.2
        w = rng.uniform(0.1, 1.0, size=24)
        c = rng.normal(size=3) * 0.05
        out[f"p2m_p{p}_xyzw"] = np.c_[q, w]
        out[f"p2m_p{p}_center"] = c
        out[f"p2m_p{p}_out"] = ref.p2m(p, np.c_[q, w], c)
        loc = rng.normal(size=(L, 3))
        d = rng.normal(size=3) * 0.2
        out[f"eval_p{p}_local"] = loc
        out[f"eval_p{p}_d"] = d
        out[f"eval_p{p}_out"] = ref.eval_local(p, loc, d)
    # direct Biot-Savart with the reference's azimuthal current
    src = np.c_[rng.normal(size=(256, 3)), rng.uniform(0.1, 1.0, 256)]
    tgt = rng.normal(size=(32, 3)) * 2
    out["direct_xyzw"] = src
    out["direct_tgt"] = tgt
    out["direct_B"] = ref.direct_B(src, tgt, 5.0)
    # the reference's full FMM pipeline (p = 10, FP64) on a small torus, targets away from it
    xyz, w, _ = geometry.torus(32, 8, 4, 2.0, 0.5)
    far = rng.uniform(-1, 1, size=(64, 3))
    far = far / np.linalg.norm(far, axis=1, keepdims=True) * 5.0
    B, found, _ = ref.fmm(np.c_[xyz, w], far, 64, 32, 1.0)
    assert found == len(far)
    out["fmm_xyzw"] = np.c_[xyz, w]
    out["fmm_tgt"] = far
    out["fmm_B"] = B
    out["fmm_direct_B"] = ref.direct_B(np.c_[xyz, w], far, 1.0)
    np.savez_compressed(os.path.join(HERE, "reference_p4_p10_p16.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_p4_p10_p16.npz"), len(out), "arrays")


def seam():
    """kernels::translateAllCPU and translateAllCPUMatrixBLAS (translation_algorithms_cpu.cpp:9-135)."""
    rng = np.random.default_rng(20260002)
    ref = Reference("f64", 10)
    out = {}
    for p in (1, 4, 10, 16):
        L = (p + 1) ** 2
        t = rng.normal(size=(4, 3)) * 0.4
        a = np.stack([ref.regular(p, x) for x in t])
        b = rng.normal(size=(4, L, 3))
        out[f"ta_p{p}_a"] = a
        out[f"ta_p{p}_b"] = b
        out[f"ta_p{p}_out"] = ref.translate_all(p, a, b)
        if p > 10:
            continue
        A = rng.normal(size=(5, L))
        Bm = rng.normal(size=(L, L))
        out[f"tam_p{p}_a"] = A
        out[f"tam_p{p}_b"] = Bm
        out[f"tam_p{p}_out"] = ref.translate_all_matrix(p, A, Bm)
    path = os.path.join(HERE, "reference_seam.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, len(out), "arrays")


def read_telma(path):
    """FMM/FMMGPU/results/telma_results.txt: a header line, the point count, then per point an
    index, x, y, z and the external H field computed by the Telma program (read as in
    FMM/FMMGPU/main.cpp:28-48)."""
    with open(path) as f:
        tok = f.read().split()
    n = int(float(tok[3]))
    vals = np.array([float(v) for v in tok[4:4 + 7 * n]]).reshape(n, 7)
    return vals[:, 1:4], vals[:, 4:7]


def telma():
    """The reference's known-answer case (FMM/FMMGPU/main.cpp:50-134): the field of createTorus()
    (R 2, section 0.2, 20 x 4 x 4 hexahedra, 5 tetrahedra each, the 24-point Keast rule of
    basis_quadratures/keast 7 *.txt) at the 100 points of results/telma_results.txt, where Telma's
    H (times MU0) is the comparison value, with current 5."""
    ref_dir = os.path.join(REF_ROOT, "FMM", "FMMGPU")
    rule_x = os.path.join(ref_dir, "basis_quadratures", "keast 7 x.txt")
    rule_w = os.path.join(ref_dir, "basis_quadratures", "keast 7 w.txt")
    pts, H = read_telma(os.path.join(ref_dir, "results", "telma_results.txt"))
    ref = Reference("f64", 10)
    q = ref.torus_quadratures(2.0, 0.2, 20, 4, 4, rule_x, rule_w)
    out = {
        "rule_x": np.loadtxt(rule_x), "rule_w": np.loadtxt(rule_w),
        "telma_points": pts, "telma_H": H,
        "quad_sample_index": np.arange(0, len(q), 37), "quad_sample": q[::37],
        "quad_count": np.array(len(q)), "quad_sums": q.sum(axis=0),
        "direct_B_current5": ref.direct_B(q, pts, 5.0),
    }
    path = os.path.join(HERE, "reference_telma.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, len(out), "arrays")


def bem_case(rng, n=48, m=24):
    """Seeded BEM quadratures on a cylinder surface (radius 0.3, height 0.6, outward normals, smooth B),
    targets on a sphere of radius 3 around it."""
    phi = rng.uniform(0, 2 * np.pi, n)
    zz = rng.uniform(-0.3, 0.3, n)
    src = np.stack([0.3 * np.cos(phi), 0.3 * np.sin(phi), zz], axis=1)
    nrm = np.stack([np.cos(phi), np.sin(phi), np.zeros(n)], axis=1)
    B = np.stack([0.2 * zz, 1.0 + 0.1 * np.sin(phi), 0.5 * np.cos(phi)], axis=1) + rng.normal(size=(n, 3)) * 0.05
    w = rng.uniform(0.5, 1.5, n) * (2 * np.pi * 0.3 * 0.6 / n)
    u = rng.normal(size=(m, 3))
    tgt = 3.0 * u / np.linalg.norm(u, axis=1)[:, None]
    return src, w, B, nrm, tgt


def bem():
    """The reference's BEM kernels (integration.cpp:191-215, 295-353): direct integral and P2M."""
    rng = np.random.default_rng(20260006)
    ref = Reference("f64", 10)
    src, w, B, nrm, tgt = bem_case(rng)
    out = {"src": src, "w": w, "B": B, "nrm": nrm, "tgt": tgt, "direct": ref.bem_direct(src, w, B, nrm, tgt)}
    for p in (4, 10):
        c = rng.normal(size=3) * 0.05
        out[f"p2m_p{p}_center"] = c
        out[f"p2m_p{p}"] = ref.bem_p2m(p, src, w, B, nrm, c)
    path = os.path.join(HERE, "reference_bem.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, len(out), "arrays")


def treecode():
    """The reference's treecode B (MultipoleSolver::calcB) on a small torus, near and far points."""
    rng = np.random.default_rng(20260007)
    xyz, w, J = geometry.torus(24, 8, 4, 2.0, 0.5)
    near = rng.uniform(-2.9, 2.9, size=(16, 3))
    u = rng.normal(size=(8, 3))
    far = u / np.linalg.norm(u, axis=1)[:, None] * rng.uniform(6.0, 8.0, size=(8, 1))
    pts = np.concatenate([near, far])
    xyzw = np.concatenate([xyz, w[:, None]], axis=1)
    out = {"xyzw": xyzw, "pts": pts}
    # the solver's order is the build's compile-time FMM_ORDER: one build per order
    for p, cap in ((10, 16), (12, 32)):
        out[f"B_p{p}_cap{cap}"] = Reference("f64", p).treecode_B(xyzw, pts, cap, 1.0)
    path = os.path.join(HERE, "reference_treecode.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, len(out), "arrays")


if __name__ == "__main__":
    what = sys.argv[1:] or ["main", "seam", "telma", "bem", "treecode"]
    if "treecode" in what:
        treecode()
    if "bem" in what:
        bem()
    if "telma" in what:
        telma()
    if "main" in what:
        main()
    if "seam" in what:
        seam()
