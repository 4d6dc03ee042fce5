"""Host-side mirror of the reference's solver interface over the C ABI.

Reference interface (FMM/FMMGPU/):
  MultipoleSolver(quadratures, problem, leafCapacity)                multipole_solver.hpp:29-48
    calcMultipoleExpansionsAtLeaves(), calclMultipoleExpansions(M2MAlg, Device)
  FastMultipoleSolver(quadratures, points, problem, capS=1000, capT=100)
                                                                       fast_multipole_solver.hpp:25-49
    calcLocalMultipoleExpansions(M2LAlg, Device), calcA(current), calcB(current)
  math::calcBioSavartLaplace(current, point, quadratures)             integration.hpp:46-49
  enums M2MAlg / Device / M2LAlg / Problem                            multipole_solver_enums.hpp:3-29

Differences a caller sees: quadratures are arrays (xyz[N,3], w[N], optional J[N,3]) instead of
std::vector<Quadrature>; results come back in target input order as an [M,3] array instead of
(point, value) pairs in tree order; the algorithm and device enums are accepted and ignored
(there is one GPU algorithm); errors raise FmmError instead of exiting the process.
Inputs given as CUDA torch tensors stay on the device and results are CUDA tensors; numpy
inputs are copied through host memory and results are numpy arrays.
"""
from __future__ import annotations

import ctypes
import weakref
from enum import IntEnum

import numpy as np

from . import _lib

try:  # torch is plumbing for device buffers and streams; numpy-only use works without it
    import torch
except Exception:  # pragma: no cover
    torch = None


class Problem(IntEnum):
    BioSavartLaplace = 0
    BEM = 1


class M2MAlg(IntEnum):
    NoTranslation = 0
    ComplexTranslation = 1
    RealTranslation = 2
    Layers = 3
    Matrices = 4


class Device(IntEnum):
    CPU = 0
    GPU = 1
    Adaptive = 2


class M2LAlg(IntEnum):
    ComplexTranslation = 0
    Matrices = 1


_PRECISION = {"fp32": _lib.FMM_FP32, "fp64": _lib.FMM_FP64}
_M2L = {"simt": _lib.FMM_M2L_SIMT, "bf16x3": _lib.FMM_M2L_BF16X3, "tf32": _lib.FMM_M2L_TF32,
        "bf16x6": _lib.FMM_M2L_BF16X6}


def _is_cuda_tensor(x):
    return torch is not None and isinstance(x, torch.Tensor) and x.is_cuda


class _Buffer:
    """A host (numpy) or device (torch) array with the plan's element type."""

    def __init__(self, x, dtype_np, torch_dtype, shape_tail):
        if _is_cuda_tensor(x):
            t = x.detach().to(torch_dtype).contiguous()
            self.device = True
            self.obj = t
            self.ptr = t.data_ptr()
            self.n = t.shape[0] if t.dim() else 0
        else:
            a = np.ascontiguousarray(np.asarray(x, dtype=dtype_np))
            self.device = False
            self.obj = a
            self.ptr = a.ctypes.data
            self.n = a.shape[0] if a.ndim else 0
        if shape_tail is not None and tuple(self.obj.shape[1:]) != shape_tail:
            raise ValueError(f"expected shape [N, {shape_tail[0]}], got {tuple(self.obj.shape)}")


class Plan:
    """Owns one fmm_plan (one expansion order, leaf capacity, precision and M2L mode)."""

    def __init__(self, order=10, leaf_capacity=64, target_leaf_capacity=0, precision="fp32", m2l="simt",
                 m2l_truncate=False, device=0, root=None, m2l_degree_cutoff=0):
        self.lib = _lib.load()
        cfg = _lib.FmmConfig()
        self.lib.fmm_default_config(ctypes.byref(cfg))
        cfg.order = int(order)
        cfg.leaf_capacity = int(leaf_capacity)
        cfg.target_leaf_capacity = int(target_leaf_capacity)
        cfg.precision = _PRECISION[precision]
        cfg.m2l_mode = _M2L[m2l]
        cfg.m2l_truncate = int(bool(m2l_truncate))
        cfg.device = int(device)
        cfg.m2l_tc_degree_cutoff = int(m2l_degree_cutoff)
        if root is not None:
            center, H = root
            for d in range(3):
                cfg.root_center[d] = float(center[d])
            cfg.root_half_width = float(H)
        self.cfg = cfg
        self.precision = precision
        self.np_dtype = np.float32 if precision == "fp32" else np.float64
        self.torch_dtype = None if torch is None else (torch.float32 if precision == "fp32" else torch.float64)
        h = ctypes.c_void_p()
        _lib.check(self.lib.fmm_plan_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.handle = h
        self._keep = []
        self._pinned = []   # page-locked result buffers: [torch tensor, weakref to the array handed out]
        self.device_mode = False
        self.m = 0
        # bumped whenever the plan's inputs change (sources, targets, strengths, coils), so a caller
        # holding results of an earlier input set can tell that the plan no longer describes them
        self.generation = 0

    def close(self):
        if getattr(self, "handle", None):
            self.lib.fmm_plan_destroy(self.handle)
            self.handle = None
        self._pinned = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _stream(self):
        if self.device_mode and torch is not None:
            return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        return ctypes.c_void_p(0)

    def set_sources(self, xyz, w, J=None, asynchronous=False):
        """Source points, weights and current directions (J None: the azimuthal direction).

        asynchronous=True (host arrays in page-locked memory, e.g. from torch's pin_memory(), of the plan's
        element type): fmm_set_sources_async, which returns before the copies end and lets the next tree
        build run while the weights and directions cross the bus. The arrays must stay unchanged until the
        next solve has returned; the plan keeps references to them until then."""
        x = _Buffer(xyz, self.np_dtype, self.torch_dtype, (3,))
        wb = _Buffer(w, self.np_dtype, self.torch_dtype, ())
        jb = _Buffer(J, self.np_dtype, self.torch_dtype, (3,)) if J is not None else None
        if asynchronous and x.device:
            raise ValueError("asynchronous=True takes host arrays; device inputs are copied on the stream anyway")
        self.device_mode = x.device
        self.n = x.n
        if asynchronous:
            _lib.check(self.lib.fmm_set_sources_async(self.handle, ctypes.c_void_p(x.ptr), ctypes.c_void_p(wb.ptr),
                                                      ctypes.c_void_p(jb.ptr) if jb else None, x.n, self._stream()))
        else:
            _lib.check(self.lib.fmm_set_sources(self.handle, ctypes.c_void_p(x.ptr), ctypes.c_void_p(wb.ptr),
                                                ctypes.c_void_p(jb.ptr) if jb else None, x.n, int(x.device),
                                                self._stream()))
        self._keep = [x, wb, jb]
        self.generation += 1

    def set_bem_sources(self, xyz, w, B, normal):
        """BEM sources (fmm_set_bem_sources): points, weights, field values and normals; the plan then
        computes the reference's BEM integral (solve / direct / treecode with want=2 return it as A)."""
        x = _Buffer(xyz, self.np_dtype, self.torch_dtype, (3,))
        wb = _Buffer(w, self.np_dtype, self.torch_dtype, ())
        bb = _Buffer(B, self.np_dtype, self.torch_dtype, (3,))
        nb = _Buffer(normal, self.np_dtype, self.torch_dtype, (3,))
        self.device_mode = x.device
        self.n = x.n
        _lib.check(self.lib.fmm_set_bem_sources(self.handle, ctypes.c_void_p(x.ptr), ctypes.c_void_p(wb.ptr),
                                                ctypes.c_void_p(bb.ptr), ctypes.c_void_p(nb.ptr), x.n, int(x.device),
                                                self._stream()))
        self._keep = [x, wb, bb, nb]
        self.generation += 1

    def set_targets(self, xyz):
        t = _Buffer(xyz, self.np_dtype, self.torch_dtype, (3,))
        self.device_mode = t.device
        _lib.check(self.lib.fmm_set_targets(self.handle, ctypes.c_void_p(t.ptr), t.n, int(t.device), self._stream()))
        self.m = t.n
        self._keep.append(t)
        self.generation += 1

    def set_targets_to_sources(self):
        """Targets = the source points just set (fmm_set_targets_to_sources): a device-side copy."""
        _lib.check(self.lib.fmm_set_targets_to_sources(self.handle, self._stream()))
        self.m = self.n
        self.generation += 1

    def _out(self, rows=None):
        rows = self.m if rows is None else rows
        if self.device_mode:
            return torch.empty((rows, 3), dtype=self.torch_dtype, device=f"cuda:{self.cfg.device}")
        if torch is not None and torch.cuda.is_available():
            # page-locked host memory, so that the device-to-host copy runs at full DMA speed. Page-locking a
            # large block costs ~0.1 s (201 MB); torch's host allocator keeps only a freed block, so while the
            # caller still holds the previous result every other solve paid it. The plan keeps its own few
            # buffers and reuses one once the array it handed out (and every view of it) is gone.
            shape = (rows, 3)
            for entry in self._pinned:
                t, ref = entry
                if tuple(t.shape) == shape and t.dtype == self.torch_dtype and (ref is None or ref() is None):
                    arr = t.numpy()
                    entry[1] = weakref.ref(arr)
                    return arr
            t = torch.empty(shape, dtype=self.torch_dtype, pin_memory=True)
            arr = t.numpy()
            if len(self._pinned) < 4:
                self._pinned.append([t, weakref.ref(arr)])
            return arr
        return np.empty((rows, 3), dtype=self.np_dtype)

    @staticmethod
    def _ptr(a):
        if a is None:
            return None
        return ctypes.c_void_p(a.data_ptr() if _is_cuda_tensor(a) else a.ctypes.data)

    def set_coils(self, src_offsets, tgt_offsets):
        """Independent problems in one plan (fmm_batch_set_coils): coil c owns sources
        src_offsets[c]:src_offsets[c+1] and targets tgt_offsets[c]:tgt_offsets[c+1]. Call after
        set_sources / set_targets; set_coils(None, None) returns to a single problem."""
        self.generation += 1
        if src_offsets is None:
            _lib.check(self.lib.fmm_batch_set_coils(self.handle, 0, None, None))
            return
        so = np.ascontiguousarray(np.asarray(src_offsets, dtype=np.int64))
        to = np.ascontiguousarray(np.asarray(tgt_offsets, dtype=np.int64))
        if so.shape != to.shape or so.ndim != 1 or len(so) < 2:
            raise ValueError("src_offsets and tgt_offsets must be 1-D with ncoils + 1 entries")
        _lib.check(self.lib.fmm_batch_set_coils(self.handle, len(so) - 1, ctypes.c_void_p(so.ctypes.data),
                                                ctypes.c_void_p(to.ctypes.data)))

    def build_tree(self):
        _lib.check(self.lib.fmm_build_tree(self.handle, self._stream()))

    def upward(self):
        _lib.check(self.lib.fmm_upward(self.handle, self._stream()))

    def downward(self):
        _lib.check(self.lib.fmm_downward(self.handle, self._stream()))

    def _run(self, fn, current, want):
        B = self._out() if want & 1 else None
        A = self._out() if want & 2 else None
        _lib.check(fn(self.handle, ctypes.c_double(current), int(want), self._ptr(B), self._ptr(A),
                      int(self.device_mode), self._stream()))
        return B, A

    def evaluate(self, current=1.0, want=1):
        return self._run(self.lib.fmm_evaluate, current, want)

    def solve(self, current=1.0, want=1):
        return self._run(self.lib.fmm_solve, current, want)

    def direct(self, current=1.0, want=1):
        return self._run(self.lib.fmm_direct, current, want)

    def treecode(self, points, current=1.0, want=1, reference_near=False, fd_curl=False):
        """Treecode point queries on this plan's source tree and multipoles (fmm_treecode; call build_tree
        and upward first). reference_near / fd_curl reproduce the reference's dropped close leaves and its
        central-difference curl. Returns (B, A) for `points` [M,3] (None where not wanted)."""
        pb = _Buffer(points, self.np_dtype, self.torch_dtype, (3,))
        if pb.device != self.device_mode:
            raise ValueError("points must live where the plan's inputs live (host numpy or CUDA tensor)")
        B = self._out(pb.n) if want & 1 else None
        A = self._out(pb.n) if want & 2 else None
        flags = (_lib.FMM_TREECODE_REFERENCE_NEAR if reference_near else 0) | (_lib.FMM_TREECODE_FD_CURL if fd_curl else 0)
        _lib.check(self.lib.fmm_treecode(self.handle, ctypes.c_double(current), int(want), ctypes.c_void_p(pb.ptr), pb.n,
                                         self._ptr(B), self._ptr(A), int(flags), int(self.device_mode), self._stream()))
        return B, A

    def adjoint(self, g, current=1.0, want_dJ=True, want_dx=True):
        """Adjoint FMM: for g = dLoss/dB at the targets ([M,3]) returns (dLoss/dJ, dLoss/d(source
        positions)), each [N,3] or None."""
        gb = _Buffer(g, self.np_dtype, self.torch_dtype, (3,))
        if gb.device != self.device_mode:
            raise ValueError("g must live where the plan's inputs live (host numpy or CUDA tensor)")
        dJ = self._out(self.n) if want_dJ else None
        dx = self._out(self.n) if want_dx else None
        _lib.check(self.lib.fmm_adjoint(self.handle, ctypes.c_double(current), ctypes.c_void_p(gb.ptr), self._ptr(dJ),
                                        self._ptr(dx), int(self.device_mode), self._stream()))
        return dJ, dx

    def adjoint_direct(self, g, current=1.0, want_dJ=True, want_dx=True):
        """The same gradients as adjoint() by direct summation (FP64 accumulation); no tree needed."""
        gb = _Buffer(g, self.np_dtype, self.torch_dtype, (3,))
        if gb.device != self.device_mode:
            raise ValueError("g must live where the plan's inputs live (host numpy or CUDA tensor)")
        dJ = self._out(self.n) if want_dJ else None
        dx = self._out(self.n) if want_dx else None
        _lib.check(self.lib.fmm_adjoint_direct(self.handle, ctypes.c_double(current), ctypes.c_void_p(gb.ptr),
                                               self._ptr(dJ), self._ptr(dx), int(self.device_mode), self._stream()))
        return dJ, dx

    def update_sources(self, w, J=None):
        """New weights / currents for the same source positions; keeps the tree."""
        wb = _Buffer(w, self.np_dtype, self.torch_dtype, ())
        jb = _Buffer(J, self.np_dtype, self.torch_dtype, (3,)) if J is not None else None
        _lib.check(self.lib.fmm_update_sources(self.handle, ctypes.c_void_p(wb.ptr),
                                               ctypes.c_void_p(jb.ptr) if jb else None, int(wb.device),
                                               self._stream()))
        self._keep += [wb, jb]
        self.generation += 1

    def graph_capture(self, want=1):
        """Capture P2M .. L2P + near field on the current tree as a CUDA graph."""
        _lib.check(self.lib.fmm_graph_capture(self.handle, int(want), self._stream()))
        self.graph_want = int(want)

    def graph_launch(self, current=1.0):
        B = self._out() if self.graph_want & 1 else None
        A = self._out() if self.graph_want & 2 else None
        _lib.check(self.lib.fmm_graph_launch(self.handle, ctypes.c_double(current), self._ptr(B), self._ptr(A),
                                             int(self.device_mode), self._stream()))
        return B, A

    def direct_fp64(self, targets, current=1.0):
        t = np.ascontiguousarray(np.asarray(targets, dtype=np.float64).reshape(-1, 3))
        out = np.zeros_like(t)
        _lib.check(self.lib.fmm_direct_fp64_subset(self.handle, ctypes.c_double(current), ctypes.c_void_p(t.ctypes.data),
                                                   len(t), ctypes.c_void_p(out.ctypes.data)))
        return out

    def autotune(self):
        """Times the kernels' tile choices on this plan's data (after a solve) and keeps the fastest;
        later plans with the same order, leaf sizes, precision and M2L mode start with it."""
        t = _lib.FmmTuning()
        _lib.check(self.lib.fmm_autotune(self.handle, ctypes.byref(t), self._stream()))
        return {k: getattr(t, k) for k, _ in _lib.FmmTuning._fields_}

    def tuning(self):
        t = _lib.FmmTuning()
        _lib.check(self.lib.fmm_get_tuning(self.handle, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in _lib.FmmTuning._fields_[:3]}

    def set_tuning(self, m2l_k_chunk=64, near_tile=256, p2m_chunk=0):
        t = _lib.FmmTuning(int(m2l_k_chunk), int(near_tile), int(p2m_chunk), 0.0, 0.0, 0.0)
        _lib.check(self.lib.fmm_set_tuning(self.handle, ctypes.byref(t)))

    def set_wait_limit(self, seconds):
        """Limit of one tensor-core pipeline wait (fmm_set_wait_limit); FmmError FMM_E_TIMEOUT when one runs out."""
        _lib.check(self.lib.fmm_set_wait_limit(self.handle, ctypes.c_double(seconds)))

    def stats(self):
        s = _lib.FmmStats()
        _lib.check(self.lib.fmm_get_stats(self.handle, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in _lib.FmmStats._fields_}

    def operator(self, kind, index):
        L = (self.cfg.order + 1) ** 2
        out = np.zeros((L, L))
        _lib.check(self.lib.fmm_get_operator(self.handle, int(kind), int(index), ctypes.c_void_p(out.ctypes.data)))
        return out


def _set_quadratures(plan, quadratures, problem):
    """Biot-Savart sources (xyz, w[, J]) or BEM sources (xyz, w, B, normal)."""
    if problem == Problem.BEM:
        xyz, w, B, normal = quadratures
        plan.set_bem_sources(xyz, w, B, normal)
    else:
        xyz, w, J = (tuple(quadratures) + (None,))[:3]
        plan.set_sources(xyz, w, J)


class MultipoleSolver:
    """Upward pass and treecode point queries (MultipoleSolver in the reference): calcA / calcB(current,
    point) walk the source tree with the reference's acceptance test (fmm_treecode). Close leaves are
    summed directly and B comes from the analytic curl unless reference_near / fd_curl are set, which
    reproduce the reference's choices."""

    def __init__(self, quadratures, problem=Problem.BioSavartLaplace, quadratureOctreeLeafCapacity=1000, *,
                 order=10, precision="fp32", m2l="simt", m2l_truncate=False, device=0, root=None):
        self.plan = Plan(order=order, leaf_capacity=quadratureOctreeLeafCapacity, precision=precision, m2l=m2l,
                         m2l_truncate=m2l_truncate, device=device, root=root)
        self.problem = Problem(problem)
        _set_quadratures(self.plan, quadratures, self.problem)
        self._multipoles = False
        self.harmonicOrder = int(order)
        self.treecode_flags = {"reference_near": False, "fd_curl": False}

    def calcMultipoleExpansionsAtLeaves(self):
        self.plan.build_tree()
        self.plan.upward()
        self._multipoles = True

    def calclMultipoleExpansions(self, algorithm=M2MAlg.Matrices, device=Device.GPU):
        if not self._multipoles:
            self.calcMultipoleExpansionsAtLeaves()

    def _query(self, current, point, want):
        if not self._multipoles:
            raise RuntimeError("Multipoles are not ready!")
        pts = point if _is_cuda_tensor(point) else np.asarray(point, dtype=self.plan.np_dtype).reshape(-1, 3)
        out = self.plan.treecode(pts, current, want, **self.treecode_flags)[0 if want == 1 else 1]
        return out[0] if not _is_cuda_tensor(point) and np.ndim(point) == 1 else out

    def calcB(self, current, point):
        """B at one point ([3]) or many ([M,3]) by the treecode."""
        return self._query(current, point, 1)

    def calcA(self, current, point):
        return self._query(current, point, 2)


class FastMultipoleSolver(MultipoleSolver):
    def __init__(self, quadratures, points, problem=Problem.BioSavartLaplace, quadratureOctreeLeafCapacity=1000,
                 calculationPointOctreeLeafCapacity=100, *, order=10, precision="fp32", m2l="simt",
                 m2l_truncate=False, device=0, root=None):
        self.plan = Plan(order=order, leaf_capacity=quadratureOctreeLeafCapacity,
                         target_leaf_capacity=calculationPointOctreeLeafCapacity, precision=precision, m2l=m2l,
                         m2l_truncate=m2l_truncate, device=device, root=root)
        self.problem = Problem(problem)
        _set_quadratures(self.plan, quadratures, self.problem)
        xyz = quadratures[0]
        if points is xyz:
            self.plan.set_targets_to_sources()   # B at the quadrature points themselves
        else:
            self.plan.set_targets(points)
        self._multipoles = False
        self._locals = False
        self.harmonicOrder = int(order)
        self.treecode_flags = {"reference_near": False, "fd_curl": False}

    def calcLocalMultipoleExpansions(self, algorithm=M2LAlg.ComplexTranslation, device=Device.GPU):
        if not self._multipoles:
            raise RuntimeError("Multipoles are not ready!")
        self.plan.downward()
        self._locals = True

    def _ready(self):
        if not self._locals:
            raise RuntimeError("Local expansions are not ready!")

    def calcB(self, current, point=None):
        """calcB(current): B at the solver's points (FMM); calcB(current, point): the treecode."""
        if point is not None:
            return self._query(current, point, 1)
        self._ready()
        return self.plan.evaluate(current, 1)[0]

    def calcA(self, current, point=None):
        if point is not None:
            return self._query(current, point, 2)
        self._ready()
        return self.plan.evaluate(current, 2)[1]

    def calcBEM(self, current=1.0):
        """The BEM integral at the points (FastMultipoleSolver::calcBEM: no current factor)."""
        if self.problem != Problem.BEM:
            raise ValueError("calcBEM needs Problem.BEM")
        self._ready()
        return self.plan.evaluate(1.0, 2)[1]

    def solve(self, current=1.0, want="B"):
        w = {"B": 1, "A": 2, "AB": 3}[want]
        B, A = self.plan.solve(current, w)
        self._multipoles = self._locals = True
        return {"B": B, "A": A, "AB": (B, A)}[want]

    def adjoint(self, dL_dB, current=1.0):
        """(dLoss/dJ, dLoss/d(source positions)) for dLoss/dB at the points."""
        return self.plan.adjoint(dL_dB, current)

    def stats(self):
        return self.plan.stats()


def calcBioSavartLaplace(current, points, quadratures, precision="fp64", device=0):
    """Direct Biot-Savart B at `points` (math::calcBioSavartLaplace), on the GPU."""
    plan = Plan(order=1, leaf_capacity=1 << 30, precision=precision, device=device)
    xyz, w, J = (tuple(quadratures) + (None,))[:3]
    plan.set_sources(xyz, w, J)
    plan.set_targets(points)
    B, _ = plan.direct(current, 1)
    plan.close()
    return B
