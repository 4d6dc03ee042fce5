"""ctypes bindings for the CPU restatement (oracle/liboracle.so) and the reference build
(oracle/_ref/libref_fmm_*.so).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg, always as the checker. The product library never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_lib = None


def build() -> None:
    """Compile liboracle.so (and nothing else)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def nharm(p: int) -> int:
    return (p + 1) * (p + 1)


def solid_harmonics(p, xyz, regular=True, compat=False):
    out = np.zeros(nharm(p))
    _load().orc_solid_harmonics(p, int(regular), int(compat), _d(_c64(xyz)), _d(out))
    return out


def solid_harmonics_grad(p, xyz, regular=True):
    out = np.zeros((nharm(p), 3))
    _load().orc_solid_harmonics_grad(p, int(regular), _d(_c64(xyz)), _d(out))
    return out


def solid_harmonics_grad2(p, xyz, regular=True, compat=False):
    """Gradient of the real solid harmonics in either convention: out[(p+1)^2][3]."""
    out = np.zeros((nharm(p), 3))
    _load().orc_solid_harmonics_grad2(p, int(regular), int(compat), _d(_c64(xyz)), _d(out))
    return out


# ----------------------------------------------------------------------------------------------
# BEM problem (the reference's Problem::BEM; FMM/FMMGPU/integration.cpp:191-215, 295-353). A BEM
# quadrature carries a point q, a weight w, a field value B and a surface normal n; its kernel at x is
#   K(x) = w [d (B . n) + d x (B x n)] / |d|^3,   d = q - x,
# and the integral is sum_q K(x) / (4 pi). Each component c is the potential of point dipoles
# (d / |d|^3 = grad_x 1/|x - q|), so its multipole about a centre c0 is
#   M_k = -sum_q w [g_k (B . n) + g_k x (B x n)],   g_k = grad R_k(q - c0),
# evaluated as sum_k M_k I_k(x - c0) / (4 pi) (calcBEM: the potential path, no current factor).
# ----------------------------------------------------------------------------------------------
REF_PI = 3.14159265359   # the reference's math::PI


def bem_direct(src, w, B, nrm, tgt):
    """Direct BEM integral at tgt (math::calcBEMIntegral, integration.cpp:191-215), FP64; a quadrature
    that coincides with a target contributes nothing."""
    src = _c64(src).reshape(-1, 3)
    tgt = _c64(tgt).reshape(-1, 3)
    w = _c64(w)
    Bn = np.einsum("ij,ij->i", _c64(B).reshape(-1, 3), _c64(nrm).reshape(-1, 3))
    v = np.cross(_c64(B).reshape(-1, 3), _c64(nrm).reshape(-1, 3))
    out = np.zeros((len(tgt), 3))
    for j, x in enumerate(tgt):
        d = src - x
        r = np.sqrt(np.einsum("ij,ij->i", d, d))
        ok = r > 0
        inv3 = np.zeros_like(r)
        inv3[ok] = 1.0 / r[ok] ** 3
        k = (d * Bn[:, None] + np.cross(d, v)) * (w * inv3)[:, None]
        out[j] = k.sum(axis=0) / (4 * REF_PI)
    return out


def bem_p2m(p, src, w, B, nrm, center, compat=True, fd_eps=None):
    """BEM multipole about `center` (calcBEMIntegralContribution, integration.cpp:295-353): out[(p+1)^2][3].
    fd_eps=None takes the analytic gradient of the regular harmonics; a value takes the reference's central
    differences with that step (the reference uses math::eps = 1e-3)."""
    src = _c64(src).reshape(-1, 3)
    w = _c64(w)
    Bv = _c64(B).reshape(-1, 3)
    nv = _c64(nrm).reshape(-1, 3)
    c0 = _c64(center)
    out = np.zeros((nharm(p), 3))
    for i in range(len(src)):
        t = src[i] - c0
        if fd_eps is None:
            g = solid_harmonics_grad2(p, t, True, compat)
        else:
            g = np.zeros((nharm(p), 3))
            for a in range(3):
                e = np.zeros(3)
                e[a] = fd_eps
                g[:, a] = (solid_harmonics(p, t + e, True, compat) - solid_harmonics(p, t - e, True, compat)) / (2 * fd_eps)
        first = g * np.dot(Bv[i], nv[i])
        second = np.cross(g, np.cross(Bv[i], nv[i]))
        out -= (first + second) * w[i]
    return out


# ----------------------------------------------------------------------------------------------
# The reference's treecode (MultipoleSolver::calcB, multipole_solver.cpp:686-700): one source octree,
# leaf P2M and complex-translation M2M, then per point a descent that takes a node's multipole when
# 4 r^2 < d^2 (r the box radius, d the distance to its centre) and otherwise its children; a close
# leaf contributes nothing (quadrature_octree.cpp:196-258). The curl uses central differences of the
# irregular harmonics (step 1e-3), as there.
# ----------------------------------------------------------------------------------------------
REF_MU0 = 1.2566370614e-6   # the reference's math::MU0
_OCTANTS = ((-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1), (-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1))


def _tc_build(xyz, idx, c, h, cap, float_centres=True):
    """Node of the reference's quadrature octree (quadrature_octree.cpp:23-97): a box with cap or more
    points is split into 8 children whose centres and half-widths are computed in float (float_centres;
    exact halving otherwise); points are assigned by the half-open box test (box.cpp:13-24), keeping their
    input order."""
    node = {"c": c, "h": h, "idx": idx, "children": []}
    if len(idx) >= cap:
        if float_centres:
            fc = np.float32(c)
            fh = np.float32(h)
            ch = (fh / np.float32(2)).astype(np.float64)
            centres = [np.array([fc[a] + np.float32(sgn[a]) * (fh[a] / np.float32(2)) for a in range(3)],
                                dtype=np.float32).astype(np.float64) for sgn in _OCTANTS]
        else:
            ch = h / 2
            centres = [c + np.array(sgn, dtype=np.float64) * ch for sgn in _OCTANTS]
        for cc in centres:
            p = xyz[idx]
            inside = np.all((cc - ch <= p) & (p < cc + ch), axis=1)
            node["children"].append(_tc_build(xyz, idx[inside], cc, ch, cap, float_centres))
        node["idx"] = idx[:0]
    return node


def _tc_upward(node, p, xyz, w, J, compat):
    if len(node["idx"]) > 0:   # a leaf with points: P2M (integration.cpp:137-161)
        node["M"] = p2m(p, xyz[node["idx"]], w[node["idx"]], None if J is None else J[node["idx"]], node["c"],
                        compat=compat)
        return
    node["M"] = np.zeros((nharm(p), 3))
    for ch in node["children"]:
        _tc_upward(ch, p, xyz, w, J, compat)
    for ch in node["children"]:   # non-empty leaves and subdivided nodes (quadrature_octree.cpp:116-135)
        if len(ch["idx"]) > 0 or ch["children"]:
            node["M"] += m2m(p, ch["M"], ch["c"] - node["c"], compat=compat)


def _tc_rot(node, p, x, eps, compat):
    d2 = float(np.sum((x - node["c"]) ** 2))
    r2 = float(np.sum(node["h"] ** 2))
    if 4 * r2 < d2:
        v = x - node["c"]
        if eps is None:   # analytic gradient of the irregular harmonics
            g = solid_harmonics_grad2(p, v, False, compat)
            hd = [g[:, a] for a in range(3)]
            scale = 1.0
        else:
            hd = []
            for a in range(3):
                e = np.zeros(3)
                e[a] = eps
                hd.append(solid_harmonics(p, v + e, False, compat) - solid_harmonics(p, v - e, False, compat))
            scale = 1.0 / (2 * eps)
        M = node["M"]
        t = np.array([np.dot(M[:, 2], hd[1]) - np.dot(M[:, 1], hd[2]),
                      np.dot(M[:, 0], hd[2]) - np.dot(M[:, 2], hd[0]),
                      np.dot(M[:, 1], hd[0]) - np.dot(M[:, 0], hd[1])])
        return t * scale
    out = np.zeros(3)
    for ch in node["children"]:
        out += _tc_rot(ch, p, x, eps, compat)
    return out


def treecode_B(p, cap, xyz, w, pts, current=1.0, half=3.0, eps=1e-3, compat=True, J=None):
    """B at pts by the reference's treecode, FP64 (root: centre 0, half-width `half`; points outside it
    are not inserted). Returns [m, 3]. compat=True reproduces the reference (its harmonic conventions and
    float box centres); compat=False keeps its tree rule, acceptance test, dropped close leaves and
    central-difference curl but uses the standard harmonics and exact box centres, the definition the
    device treecode's reference mode implements. J: current directions (None: the azimuthal direction).
    eps=None takes the curl from the analytic gradient of the irregular harmonics instead."""
    xyz = _c64(xyz).reshape(-1, 3)
    w = _c64(w)
    pts = _c64(pts).reshape(-1, 3)
    Jc = None if J is None else _c64(J).reshape(-1, 3)
    c0 = np.zeros(3)
    h0 = np.full(3, float(half))
    inside = np.all((c0 - h0 <= xyz) & (xyz < c0 + h0), axis=1)
    root = _tc_build(xyz, np.nonzero(inside)[0], c0, h0, cap, float_centres=compat)
    _tc_upward(root, p, xyz, w, Jc, compat)
    out = np.stack([_tc_rot(root, p, x, eps, compat) for x in pts])
    return out / (4.0 * REF_PI) * current * REF_MU0


def p2m(p, xyz, w, J=None, center=(0, 0, 0), compat=False):
    xyz = _c64(xyz).reshape(-1, 3)
    w = _c64(w)
    out = np.zeros((nharm(p), 3))
    Jc = _c64(J).reshape(-1, 3) if J is not None else None
    _load().orc_p2m(p, int(compat), ctypes.c_int64(len(w)), _d(xyz), _d(w), _d(Jc), _d(_c64(center)), _d(out))
    return out


def _translate(name, p, expansion, t, compat):
    out = np.zeros((nharm(p), 3))
    getattr(_load(), name)(p, int(compat), _d(_c64(expansion)), _d(_c64(t)), _d(out))
    return out


def m2m(p, expansion, t, compat=False):
    return _translate("orc_m2m", p, expansion, t, compat)


def m2l(p, expansion, t, compat=False):
    return _translate("orc_m2l", p, expansion, t, compat)


def l2l(p, expansion, t, compat=False):
    return _translate("orc_l2l", p, expansion, t, compat)


def translate_all(p, a, b):
    """Batched real-form M2M with given harmonics: a [count, L], b [count, L, 3] -> [count, L, 3]."""
    a = _c64(a).reshape(-1, nharm(p))
    b = _c64(b).reshape(len(a), nharm(p), 3)
    out = np.zeros_like(b)
    _load().orc_translate_all(ctypes.c_int64(len(a)), p, _d(a), _d(b), _d(out))
    return out


def translate_all_matrix(a, b):
    """result [count, L] = a [count, L] @ b [L, L] in FP64 (the matrix forms of the same seam)."""
    b = _c64(b)
    L = b.shape[0]
    a = _c64(a).reshape(-1, L)
    out = np.zeros_like(a)
    _load().orc_translate_all_matrix(ctypes.c_int64(len(a)), L, _d(a), _d(b), _d(out))
    return out


def eval_expansion(p, coef, d, regular=True, compat=False):
    A = np.zeros(3)
    curl = np.zeros(3)
    _load().orc_eval_expansion(p, int(regular), int(compat), _d(_c64(coef)), _d(_c64(d)), _d(A), _d(curl))
    return A, curl


def direct(src, w, J, tgt, current=1.0, want_A=False):
    """FP64 direct Biot-Savart B (and optionally A) at tgt; coincident pairs skipped."""
    src = _c64(src).reshape(-1, 3)
    tgt = _c64(tgt).reshape(-1, 3)
    w = _c64(w)
    Jc = _c64(J).reshape(-1, 3) if J is not None else None
    B = np.zeros((len(tgt), 3))
    A = np.zeros((len(tgt), 3)) if want_A else None
    _load().orc_direct(ctypes.c_int64(len(src)), _d(src), _d(w), _d(Jc), ctypes.c_int64(len(tgt)), _d(tgt),
                       ctypes.c_double(current), _d(B), _d(A))
    return (B, A) if want_A else B


def fmm(p, cap, src, w, J, tgt, center, H, current=1.0, want_A=False, truncate=False, cap_tgt=0):
    """Standard-mode FMM (the definition the device pipeline implements). Returns (B, A, stats).
    truncate=True keeps the reference's l + lambda <= p M2L truncation; False keeps the full
    operator (l + lambda <= 2p). cap_tgt: target leaf capacity (0: same as cap)."""
    _load().orc_set_m2l_extra(0 if truncate else p)
    _load().orc_set_target_cap(int(cap_tgt))
    src = _c64(src).reshape(-1, 3)
    tgt = _c64(tgt).reshape(-1, 3)
    w = _c64(w)
    Jc = _c64(J).reshape(-1, 3) if J is not None else None
    B = np.zeros((len(tgt), 3))
    A = np.zeros((len(tgt), 3)) if want_A else None
    stats = np.zeros(8)
    _load().orc_fmm(p, cap, ctypes.c_int64(len(src)), _d(src), _d(w), _d(Jc), ctypes.c_int64(len(tgt)), _d(tgt),
                    ctypes.c_double(current), _d(_c64(center)), ctypes.c_double(H), _d(B), _d(A), _d(stats))
    keys = ["nodes", "levels", "leaves", "V", "U", "W", "X", "direct_pairs"]
    return B, A, dict(zip(keys, stats.tolist()))


def tree(cap, src, tgt, center, H):
    """Node table (level, ix, iy, iz, s0, s1, t0, t1, parent, nchild), list sizes (V, U, W, X),
    and sorted-position -> input index maps of the standard-mode tree."""
    src = _c64(src).reshape(-1, 3)
    tgt = _c64(tgt).reshape(-1, 3)
    lib = _load()
    args = (ctypes.c_int64(len(src)), _d(src), ctypes.c_int64(len(tgt)), _d(tgt), _d(_c64(center)), ctypes.c_double(H))
    n_nodes = lib.orc_tree(cap, *args, ctypes.c_int64(0), None, None, None, None)
    info = np.zeros((n_nodes, 10), dtype=np.int64)
    lists = np.zeros((n_nodes, 4), dtype=np.int64)
    so = np.zeros(len(src), dtype=np.int64)
    to = np.zeros(len(tgt), dtype=np.int64)
    lib.orc_tree.restype = ctypes.c_int64
    lib.orc_tree(cap, *args, ctypes.c_int64(n_nodes), info.ctypes.data_as(_i64p), lists.ctypes.data_as(_i64p),
                 so.ctypes.data_as(_i64p), to.ctypes.data_as(_i64p))
    return info, lists, so, to


def coverage(cap, src, tgt, center, H):
    src = _c64(src).reshape(-1, 3)
    tgt = _c64(tgt).reshape(-1, 3)
    cnt = np.zeros((len(tgt), len(src)), dtype=np.int32)
    _load().orc_coverage(cap, ctypes.c_int64(len(src)), _d(src), ctypes.c_int64(len(tgt)), _d(tgt),
                         _d(_c64(center)), ctypes.c_double(H), cnt.ctypes.data_as(_i32p))
    return cnt


# --------------------------------------------------------------------------------------
# The reference itself, compiled by oracle/ref/build_ref.sh (present only where that ran).
# --------------------------------------------------------------------------------------
class Reference:
    """The patched reference CPU library for one (real type, order) build."""

    def __init__(self, real="f64", order=10):
        path = os.path.join(REF_DIR, f"libref_fmm_{real}_p{order}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        self.lib.ref_fmm.restype = ctypes.c_int
        self.order = order

    @staticmethod
    def available(real="f64", order=10):
        return os.path.exists(os.path.join(REF_DIR, f"libref_fmm_{real}_p{order}.so"))

    def regular(self, p, xyz):
        out = np.zeros(nharm(p))
        self.lib.ref_regular(p, _d(_c64(xyz)), _d(out))
        return out

    def irregular(self, p, xyz):
        out = np.zeros(nharm(p))
        self.lib.ref_irregular(p, _d(_c64(xyz)), _d(out))
        return out

    @staticmethod
    def _bem_rows(src, w, B, nrm):
        return np.ascontiguousarray(np.concatenate([_c64(src).reshape(-1, 3), _c64(w).reshape(-1, 1),
                                                    _c64(B).reshape(-1, 3), _c64(nrm).reshape(-1, 3)], axis=1))

    def treecode_B(self, xyzw, pts, cap, current=1.0):
        """The reference's MultipoleSolver treecode B at pts (multipole_solver.cpp:686-700)."""
        xyzw = _c64(xyzw).reshape(-1, 4)
        pts = _c64(pts).reshape(-1, 3)
        out = np.zeros((len(pts), 3))
        self.lib.ref_treecode_B(len(xyzw), _d(xyzw), len(pts), _d(pts), int(cap), ctypes.c_double(current), _d(out))
        return out

    def bem_direct(self, src, w, B, nrm, tgt):
        """math::calcBEMIntegral at each target."""
        q = self._bem_rows(src, w, B, nrm)
        tgt = _c64(tgt).reshape(-1, 3)
        out = np.zeros((len(tgt), 3))
        self.lib.ref_bem_direct(len(q), _d(q), len(tgt), _d(tgt), _d(out))
        return out

    def bem_p2m(self, p, src, w, B, nrm, center):
        """math::calcBEMIntegralContribution about `center`."""
        q = self._bem_rows(src, w, B, nrm)
        out = np.zeros((nharm(p), 3))
        self.lib.ref_bem_p2m(p, len(q), _d(q), _d(_c64(center)), _d(out))
        return out

    def p2m(self, p, xyzw, center):
        xyzw = _c64(xyzw).reshape(-1, 4)
        out = np.zeros((nharm(p), 3))
        self.lib.ref_p2m(p, len(xyzw), _d(xyzw), _d(_c64(center)), _d(out))
        return out

    def _tr(self, name, p, e, t):
        out = np.zeros((nharm(p), 3))
        getattr(self.lib, name)(p, _d(_c64(e)), _d(_c64(t)), _d(out))
        return out

    def m2m(self, p, e, t):
        return self._tr("ref_m2m", p, e, t)

    def m2l(self, p, e, t):
        return self._tr("ref_m2l", p, e, t)

    def l2l(self, p, e, t):
        return self._tr("ref_l2l", p, e, t)

    def translate_all(self, p, a, b):
        a = _c64(a).reshape(-1, nharm(p))
        b = _c64(b).reshape(len(a), nharm(p), 3)
        out = np.zeros_like(b)
        self.lib.ref_translate_all(len(a), p, _d(a), _d(b), _d(out))
        return out

    def translate_all_matrix(self, p, a, b):
        L = nharm(p)
        a = _c64(a).reshape(-1, L)
        out = np.zeros_like(a)
        self.lib.ref_translate_all_matrix(len(a), p, _d(a), _d(_c64(b).reshape(L, L)), _d(out))
        return out

    def torus_quadratures(self, radius, width, nL, nW, nH, rule_x, rule_w):
        """Quadratures [K, 4] (x, y, z, weight) of the reference's tetrahedral torus and basis rule files."""
        f = self.lib.ref_torus_quadratures
        f.restype = ctypes.c_int
        args = (ctypes.c_double(radius), ctypes.c_double(width), nL, nW, nH, rule_x.encode(), rule_w.encode())
        k = f(*args, None)
        out = np.zeros((k, 4))
        f(*args, _d(out))
        return out

    def eval_local(self, p, local, d):
        out = np.zeros(3)
        self.lib.ref_eval_local(p, _d(_c64(local)), _d(_c64(d)), _d(out))
        return out

    def direct_B(self, xyzw, pts, current=1.0):
        xyzw = _c64(xyzw).reshape(-1, 4)
        pts = _c64(pts).reshape(-1, 3)
        out = np.zeros((len(pts), 3))
        self.lib.ref_direct_B(len(xyzw), _d(xyzw), len(pts), _d(pts), ctypes.c_double(current), _d(out))
        return out

    def fmm(self, xyzw, pts, cap_src, cap_tgt, current=1.0, want_B=True):
        xyzw = _c64(xyzw).reshape(-1, 4)
        pts = _c64(pts).reshape(-1, 3)
        out = np.zeros((len(pts), 3))
        times = np.zeros(5)
        found = self.lib.ref_fmm(len(xyzw), _d(xyzw), len(pts), _d(pts), cap_src, cap_tgt, ctypes.c_double(current),
                                 int(want_B), _d(out), _d(times))
        return out, found, times


def adjoint_direct(src, w, J, tgt, g, current=1.0):
    """FP64 direct-sum adjoint: (dLoss/dJ [N,3], dLoss/d(source positions) [N,3]) for g = dLoss/dB."""
    src = _c64(src).reshape(-1, 3)
    tgt = _c64(tgt).reshape(-1, 3)
    g = _c64(g).reshape(-1, 3)
    w = _c64(w)
    Jc = _c64(J).reshape(-1, 3) if J is not None else None
    dJ = np.zeros((len(src), 3))
    dx = np.zeros((len(src), 3))
    _load().orc_adjoint_direct(ctypes.c_int64(len(src)), _d(src), _d(w), _d(Jc), ctypes.c_int64(len(tgt)), _d(tgt),
                               _d(g), ctypes.c_double(current), _d(dJ), _d(dx))
    return dJ, dx
