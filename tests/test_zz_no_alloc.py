"""fmm_direct_B_noalloc: the direct Biot-Savart sum for callers that cannot let a library
allocate device memory (their GPU memory belongs to another allocator, or their loop cannot
afford an allocation). It must agree with the allocating entry point, fmm_direct, within the
FP32 tolerance of the other GPU tests, on consecutive calls that share its fixed scratch array.
This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from bachelors_b200 import Plan, _lib, geometry as G

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-5
MAX_SOURCES = 1 << 18


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def noalloc_B(lib, xyz, w, J, tgt, current):
    import torch
    dev = [torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda() if a is not None else None
           for a in (xyz, w, J, tgt)]
    out = torch.full((len(tgt), 3), float("nan"), dtype=torch.float32, device="cuda")
    ptr = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(lib.fmm_direct_B_noalloc(ptr(dev[0]), ptr(dev[1]), ptr(dev[2]), len(xyz), ptr(dev[3]), len(tgt),
                                        ctypes.c_double(current), ptr(out), stream))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def allocating_B(xyz, w, J, tgt, current):
    plan = Plan(order=2, precision="fp32")
    plan.set_sources(xyz.astype(np.float32), w.astype(np.float32), None if J is None else J.astype(np.float32))
    plan.set_targets(tgt.astype(np.float32))
    B, _ = plan.direct(current, 1)
    plan.close()
    return B


def test_noalloc_direct_matches_allocating_entry_point_on_consecutive_calls():
    lib = _lib.load()
    # first call: a larger source set with explicit currents
    xyz1, w1, J1 = G.torus(64, 16, 16, 2.0, 0.5)
    t1 = G.uniform_points(3000, -3, 3, 101)
    B1 = noalloc_B(lib, xyz1, w1, J1, t1, 2.0)
    assert rel(B1, allocating_B(xyz1, w1, J1, t1, 2.0)) < FP32_TOL
    # second call: fewer sources and the azimuthal current; stale scratch entries beyond n must not leak in
    xyz2, w2, _ = G.torus(32, 8, 8, 1.5, 0.3, center=(0.2, -0.1, 0.3))
    t2 = np.r_[G.uniform_points(1000, -2, 2, 102), xyz2[:50]]
    B2 = noalloc_B(lib, xyz2, w2, None, t2, 1.0)
    assert np.isfinite(B2).all()
    assert rel(B2, allocating_B(xyz2, w2, None, t2, 1.0)) < FP32_TOL


def test_noalloc_rejects_sizes_beyond_its_limit():
    lib = _lib.load()
    st = lib.fmm_direct_B_noalloc(ctypes.c_void_p(16), ctypes.c_void_p(16), None, MAX_SOURCES + 1,
                                  ctypes.c_void_p(16), 1, ctypes.c_double(1.0), ctypes.c_void_p(16), None)
    assert st == _lib.FMM_E_LIMIT
    assert b"limit" in lib.fmm_last_error_string()
