"""Seeded synthetic source and target generators.

The reference builds its sources from a hexahedral torus mesh split into tetrahedra with a
24-point Keast rule (FMM/FMMGPU/torus.cpp:9-117, integration.cpp:163-187) and draws targets
with an unseeded std::rand (testing_helpers.cpp:171). Here every workload is a tensor-product
torus quadrature with explicit seeds:

  x = c + Rot(n) ((R + rho cos t) cos f, (R + rho cos t) sin f, rho sin t)
  f, t: n_f / n_t uniform midpoints on [0, 2 pi)
  rho:  n_rho-point Gauss-Legendre on [0, a]
  w = (2 pi / n_f) (2 pi / n_t) w_rho rho (R + rho cos t)      (the cell volume)

The current direction is the poloidal tangent (d x / d t) or the reference's azimuthal
direction perp(x) / |perp(x)| = (-y, x, 0) / rho_xy (integration.cpp:155).
"""
from __future__ import annotations

import numpy as np


def _rotation_to(axis):
    """Rotation matrix taking e_z to the unit vector `axis`."""
    n = np.asarray(axis, dtype=np.float64)
    n = n / np.linalg.norm(n)
    z = np.array([0.0, 0.0, 1.0])
    v = np.cross(z, n)
    c = float(np.dot(z, n))
    if np.linalg.norm(v) < 1e-15:
        return np.eye(3) if c > 0 else np.diag([1.0, -1.0, -1.0])
    vx = np.array([[0, -v[2], v[1]], [v[2], 0, -v[0]], [-v[1], v[0], 0]])
    return np.eye(3) + vx + vx @ vx * (1.0 / (1.0 + c))


def torus(n_phi, n_theta, n_rho, major=2.0, minor=0.5, center=(0.0, 0.0, 0.0), axis=(0.0, 0.0, 1.0),
          current="poloidal", magnitude=1.0):
    """Tensor-product quadrature of a solid torus. Returns (xyz[N,3], w[N], J[N,3]) in float64,
    ordered with the radial index fastest, then poloidal, then toroidal."""
    f = 2 * np.pi * (np.arange(n_phi) + 0.5) / n_phi
    t = 2 * np.pi * (np.arange(n_theta) + 0.5) / n_theta
    xg, wg = np.polynomial.legendre.leggauss(n_rho)
    rho = 0.5 * minor * (xg + 1.0)
    wr = 0.5 * minor * wg
    F, T, P = np.meshgrid(f, t, rho, indexing="ij")
    _, _, WR = np.meshgrid(f, t, wr, indexing="ij")
    ring = major + P * np.cos(T)
    local = np.stack([ring * np.cos(F), ring * np.sin(F), P * np.sin(T)], axis=-1).reshape(-1, 3)
    w = ((2 * np.pi / n_phi) * (2 * np.pi / n_theta) * WR * P * ring).reshape(-1)
    if current == "poloidal":
        d = np.stack([-np.sin(T) * np.cos(F), -np.sin(T) * np.sin(F), np.cos(T)], axis=-1).reshape(-1, 3)
    elif current == "azimuthal":
        d = np.stack([-np.sin(F), np.cos(F), np.zeros_like(F)], axis=-1).reshape(-1, 3)
    else:
        raise ValueError(f"unknown current direction {current!r}")
    Rm = _rotation_to(axis)
    xyz = local @ Rm.T + np.asarray(center, dtype=np.float64)
    J = magnitude * (d @ Rm.T)
    return xyz, w, J


def uniform_points(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=(n, 3))


def grid_points(n, lo, hi):
    g = (np.arange(n) + 0.5) / n * (hi - lo) + lo if n > 1 else np.array([(lo + hi) / 2])
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    return np.stack([X, Y, Z], axis=-1).reshape(-1, 3)


def cube_grid(n, lo, hi):
    """n^3 grid including both ends of [lo, hi] on each axis (the 32^3 grid on [-3, 3]^3)."""
    g = np.linspace(lo, hi, n)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    return np.stack([X, Y, Z], axis=-1).reshape(-1, 3)


def root_cube(*point_sets):
    """The root cube the solver uses by default: the bounding box of all points, made cubic
    around its midpoint with a relative margin of 2^-20 so no point sits on the upper face."""
    lo = np.min([np.min(p, axis=0) for p in point_sets if len(p)], axis=0)
    hi = np.max([np.max(p, axis=0) for p in point_sets if len(p)], axis=0)
    center = 0.5 * (lo + hi)
    H = 0.5 * float(np.max(hi - lo))
    H = H * (1.0 + 2.0 ** -20) + 1e-300
    return center, H


def random_axis(rng):
    """A direction uniform on the unit sphere."""
    v = rng.normal(size=3)
    return v / np.linalg.norm(v)


def torus_batch(n_coils=256, seed=20260004, count_range=(2 ** 12, 2 ** 18), targets_per_coil=2 ** 14,
                major_range=(1.0, 3.0), minor_range=(0.2, 0.6), center_range=(-10.0, 10.0),
                magnitude_range=(0.5, 2.0), n_theta=16, n_rho=4, params=False):
    """Many independent coils for the batched solver: coil i is a torus with major radius
    R ~ U(major_range), minor radius a ~ U(minor_range), an axis uniform on the sphere, a centre
    uniform in center_range^3, a point count log-uniform in count_range (n_phi x n_theta x n_rho
    with n_phi chosen to come closest), a poloidal current of magnitude ~ U(magnitude_range), and
    `targets_per_coil` targets uniform in the cube of side 3R around its centre.

    Returns (xyz[N,3], w[N], J[N,3], tgt[M,3], src_offsets[K+1], tgt_offsets[K+1]) with each coil's
    points contiguous; with params=True also [K, 3] rows (major radius, minor radius, current magnitude)."""
    rng = np.random.default_rng(seed)
    xs, ws, Js, ts, prm = [], [], [], [], []
    so, to = [0], [0]
    lo, hi = np.log(count_range[0]), np.log(count_range[1])
    for _ in range(n_coils):
        R = rng.uniform(*major_range)
        a = rng.uniform(*minor_range)
        axis = random_axis(rng)
        c = rng.uniform(*center_range, size=3)
        count = float(np.exp(rng.uniform(lo, hi)))
        mag = rng.uniform(*magnitude_range)
        n_phi = max(4, int(round(count / (n_theta * n_rho))))
        x, w, J = torus(n_phi, n_theta, n_rho, R, a, c, axis, "poloidal", mag)
        t = c + rng.uniform(-1.5 * R, 1.5 * R, size=(targets_per_coil, 3))
        xs.append(x); ws.append(w); Js.append(J); ts.append(t)
        so.append(so[-1] + len(w)); to.append(to[-1] + len(t))
        prm.append((R, a, mag))
    out = (np.concatenate(xs), np.concatenate(ws), np.concatenate(Js), np.concatenate(ts),
           np.array(so, dtype=np.int64), np.array(to, dtype=np.int64))
    return out + (np.array(prm),) if params else out


def hex_torus_tetrahedra(radius=2.0, section_width=0.2, n_length=20, n_width=4, n_height=4):
    """The reference's tetrahedral torus (FMM/FMMGPU/torus.cpp:9-117): a torus of square cross-section
    (side `section_width`, centre line of radius `radius`, axis z) cut into n_length x n_width x
    n_height hexahedra - n_length steps around the axis (step angle 360 / n_length degrees with the
    reference's PI literal), n_width radial steps and n_height steps in z - and each hexahedron into
    five tetrahedra. Returns the vertices [T, 4, 3], hexahedra in (length, width, height) order."""
    ref_pi = 3.14159265359
    step = 360.0 / n_length * ref_pi / 180.0
    r_in = radius - section_width / 2.0
    bottom = -section_width / 2.0
    dz = section_width / n_height
    dw = section_width / n_width
    tets = []
    # vertex indices of the five tetrahedra of a hexahedron (torus.cpp:103-117)
    split = ((0, 1, 3, 5), (0, 3, 5, 6), (0, 2, 3, 6), (0, 4, 5, 6), (3, 5, 6, 7))
    for i in range(n_length):
        a0 = np.array([r_in * np.cos(step * i), r_in * np.sin(step * i)])
        a1 = np.array([r_in * np.cos(step * (i + 1)), r_in * np.sin(step * (i + 1))])
        u0, u1 = a0 / np.linalg.norm(a0), a1 / np.linalg.norm(a1)
        for j in range(n_width):
            right, next_right = a0 + u0 * dw * j, a0 + u0 * dw * (j + 1)
            left, next_left = a1 + u1 * dw * j, a1 + u1 * dw * (j + 1)
            for k in range(n_height):
                zb, zt = bottom + dz * k, bottom + dz * (k + 1)
                pts = np.array([[*right, zb], [*next_right, zb], [*left, zb], [*next_left, zb],
                                [*right, zt], [*next_right, zt], [*left, zt], [*next_left, zt]])
                tets.extend(pts[list(s)] for s in split)
    return np.array(tets)


def tetra_quadratures(tets, rule_x, rule_w):
    """Quadrature points and weights of tetrahedra [T, 4, 3] for a basis rule on the unit tetrahedron
    (rule_x [K, 3] local coordinates, rule_w [K] weights summing to 1), as the reference maps them
    (integration.cpp:34-42,163-187): x = a + (b - a) u + (c - a) v + (d - a) w, weight = volume x w_i.
    Returns xyz [T K, 3] and w [T K], tetrahedron-major."""
    tets = np.asarray(tets, dtype=np.float64)
    rx = np.asarray(rule_x, dtype=np.float64)
    rw = np.asarray(rule_w, dtype=np.float64)
    a, b, c, d = tets[:, 0], tets[:, 1], tets[:, 2], tets[:, 3]
    vol = np.abs(np.einsum("ij,ij->i", a - d, np.cross(b - d, c - d))) / 6.0
    xyz = a[:, None, :] + (b - a)[:, None, :] * rx[None, :, 0:1] + (c - a)[:, None, :] * rx[None, :, 1:2] \
        + (d - a)[:, None, :] * rx[None, :, 2:3]
    w = vol[:, None] * rw[None, :]
    return xyz.reshape(-1, 3), w.reshape(-1)


def tetra_torus_quadratures_device(radius, section_width, n_length, n_width, n_height, rule_x, rule_w,
                                   precision="fp64", device=0):
    """hex_torus_tetrahedra + tetra_quadratures generated on the GPU (fmm_torus_quadratures): returns
    (xyz [T K, 3], w [T K]) as CUDA tensors on `device`, tetrahedron-major, ready for Plan.set_sources."""
    import ctypes
    import torch
    from . import _lib
    rx = np.ascontiguousarray(np.asarray(rule_x, dtype=np.float64).reshape(-1, 3))
    rw = np.ascontiguousarray(np.asarray(rule_w, dtype=np.float64).reshape(-1))
    k = len(rw)
    total = 5 * n_length * n_width * n_height * k
    dt = torch.float64 if precision == "fp64" else torch.float32
    xyz = torch.empty((total, 3), dtype=dt, device=f"cuda:{device}")
    w = torch.empty((total,), dtype=dt, device=f"cuda:{device}")
    lib = _lib.load()
    with torch.cuda.device(device):
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.check(lib.fmm_torus_quadratures(ctypes.c_double(radius), ctypes.c_double(section_width), int(n_length),
                                             int(n_width), int(n_height), ctypes.c_void_p(rx.ctypes.data),
                                             ctypes.c_void_p(rw.ctypes.data), k,
                                             _lib.FMM_FP64 if precision == "fp64" else _lib.FMM_FP32,
                                             ctypes.c_void_p(xyz.data_ptr()), ctypes.c_void_p(w.data_ptr()), 1, stream))
    return xyz, w
