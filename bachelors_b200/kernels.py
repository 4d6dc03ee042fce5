"""Python mirror of the reference's kernel-caller seam, namespace `kernels`
(FMM/FMMGPU/translation_algorithms.hpp:8-61, FMMCUDADLL/kernel_callers.hpp:5-10), over the C ABI
(fmm_translate_all, fmm_translate_all_matrix, fmm_translate_all_matrix_complex, fmm_add_vectors).

The reference passes raw pointers and an output argument; here every function returns its result.
Arrays may be numpy (copied through host memory, result is numpy) or CUDA torch tensors (work is
queued on torch's current stream, result is a CUDA tensor). The element type follows the inputs:
float32 / complex64 or float64 / complex128, the reference's `real` built as float or double.
The CPU names (translateAllCPU, ...) run the same GPU kernels; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .solver import _is_cuda_tensor, torch


def _prec(x):
    dt = x.dtype
    if torch is not None and isinstance(dt, torch.dtype):
        if dt in (torch.float64, torch.complex128):
            return _lib.FMM_FP64
        if dt in (torch.float32, torch.complex64):
            return _lib.FMM_FP32
    elif np.dtype(dt) in (np.float64, np.complex128):
        return _lib.FMM_FP64
    elif np.dtype(dt) in (np.float32, np.complex64):
        return _lib.FMM_FP32
    raise TypeError(f"unsupported element type {dt}")


def _prep(x, like):
    """Contiguous copy of x with like's element type on like's side (host or device)."""
    if _is_cuda_tensor(like):
        t = x if _is_cuda_tensor(x) else torch.as_tensor(np.asarray(x))
        return t.to(device=like.device, dtype=like.dtype).contiguous()
    return np.ascontiguousarray(np.asarray(x, dtype=like.dtype))


def _stream(x):
    return ctypes.c_void_p(torch.cuda.current_stream(x.device).cuda_stream) if _is_cuda_tensor(x) else None


def _ptr(x):
    return x.data_ptr() if _is_cuda_tensor(x) else x.ctypes.data


def _empty_like(x, shape):
    if _is_cuda_tensor(x):
        return torch.empty(shape, dtype=x.dtype, device=x.device)
    return np.empty(shape, dtype=x.dtype)


def _order_of(L):
    p = int(round(L ** 0.5)) - 1
    if (p + 1) ** 2 != L:
        raise ValueError(f"{L} is not a harmonic count (p+1)^2")
    return p


def _real_like(x):
    """x as a float32/float64 array or CUDA tensor (float32 stays float32, the rest becomes float64)."""
    if _is_cuda_tensor(x):
        return x if x.dtype in (torch.float32, torch.float64) else x.to(torch.float64)
    x = np.asarray(x)
    return x if x.dtype in (np.float32, np.float64) else x.astype(np.float64)


def translateAllGPU(a, b, harmonicCount=None, harmonicOrder=None):
    """kernels::translateAllGPU: per item i, M2M of the vector expansion b[i] ((p+1)^2 x 3) by the
    real regular harmonics a[i] ((p+1)^2). a: [count, L]; b: [count, L, 3]. Returns [count, L, 3]."""
    b = _real_like(b)
    if harmonicOrder is None:
        harmonicOrder = _order_of(int(b.shape[-2]))
    L = (harmonicOrder + 1) ** 2
    b = _prep(b, b)
    a = _prep(a, b)
    count = harmonicCount if harmonicCount is not None else a.reshape(-1).shape[0] // L
    if a.reshape(-1).shape[0] < count * L or b.reshape(-1).shape[0] < count * L * 3:
        raise ValueError("translateAllGPU: arrays shorter than harmonicCount items")
    out = _empty_like(b, (count, L, 3))
    lib = _lib.load()
    _lib.check(lib.fmm_translate_all(_ptr(out), _ptr(a), _ptr(b), count, harmonicOrder, _prec(b),
                                     int(_is_cuda_tensor(b)), _stream(b)))
    return out


translateAllCPU = translateAllGPU


def translateAllGPUMatrixCuBLAS(a, b, harmonicCount=None, harmonicOrder=None):
    """kernels::translateAllGPUMatrixCuBLAS: result (count x L) = a (count x L) @ b (L x L), row-major
    (the reference's column-major C = B * A). a may carry a leading batch axis [batch, count, L]
    (the RealMatrix overload: one product per component, b shared). Returns a's shape."""
    a0 = _real_like(a)
    if harmonicOrder is None:
        harmonicOrder = _order_of(int(a0.shape[-1]))
    L = (harmonicOrder + 1) ** 2
    a = _prep(a0, a0)
    b = _prep(b, a)
    if tuple(b.reshape(-1).shape)[0] != L * L:
        raise ValueError("translateAllGPUMatrixCuBLAS: b must be L x L")
    shape = tuple(a.shape)
    batch = shape[0] if len(shape) == 3 else 1
    count = harmonicCount if harmonicCount is not None else a.reshape(-1).shape[0] // (L * batch)
    out = _empty_like(a, (batch, count, L) if len(shape) == 3 else (count, L))
    lib = _lib.load()
    _lib.check(lib.fmm_translate_all_matrix(_ptr(out), _ptr(a), _ptr(b), count, harmonicOrder, batch, _prec(a),
                                            int(_is_cuda_tensor(a)), _stream(a)))
    return out


translateAllCPUMatrixBLAS = translateAllGPUMatrixCuBLAS


def translateAllGPUMatrix(a, b, harmonicCount=None, harmonicOrder=None):
    """kernels::translateAllGPUMatrix / translateAllCPUMatrix: complex result (count x L) = a @ b."""
    if _is_cuda_tensor(a):
        a0 = a if a.dtype in (torch.complex64, torch.complex128) else a.to(torch.complex128)
    else:
        a0 = np.asarray(a)
        a0 = a0 if a0.dtype in (np.complex64, np.complex128) else a0.astype(np.complex128)
    if harmonicOrder is None:
        harmonicOrder = _order_of(int(a0.shape[-1]))
    L = (harmonicOrder + 1) ** 2
    a = _prep(a0, a0)
    b = _prep(b, a)
    count = harmonicCount if harmonicCount is not None else a.reshape(-1).shape[0] // L
    out = _empty_like(a, (count, L))
    lib = _lib.load()
    _lib.check(lib.fmm_translate_all_matrix_complex(_ptr(out), _ptr(a), _ptr(b), count, harmonicOrder, _prec(a),
                                                    int(_is_cuda_tensor(a)), _stream(a)))
    return out


translateAllCPUMatrix = translateAllGPUMatrix


def addVectors(a, b):
    """kernels::addVectors (FMMCUDADLL/kernel_callers.hpp:7-9): a + b on the GPU, float32 host arrays."""
    a = np.ascontiguousarray(np.asarray(a, np.float32))
    b = np.ascontiguousarray(np.asarray(b, np.float32))
    if a.shape != b.shape:
        raise ValueError("addVectors: sizes differ")
    c = np.empty_like(a)
    _lib.check(_lib.load().fmm_add_vectors(a.ctypes.data, b.ctypes.data, c.ctypes.data, a.size))
    return c
