"""The translation seam on the GPU (fmm_translate_all, fmm_translate_all_matrix,
fmm_translate_all_matrix_complex through bachelors_b200.kernels) against the oracle and the
reference's golden vectors: FP64 to 1e-12, FP32 to 1e-5, host and device buffers."""
import os

import numpy as np
import pytest

from bachelors_b200 import kernels as K
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_seam.npz")


def rel(a, b):
    a = a.cpu().numpy() if hasattr(a, "cpu") else np.asarray(a)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def seam():
    return dict(np.load(GOLDEN))


@pytest.mark.parametrize("p", (1, 4, 10, 16))
def test_translate_all_golden(seam, p):
    a, b, ref = seam[f"ta_p{p}_a"], seam[f"ta_p{p}_b"], seam[f"ta_p{p}_out"]
    assert rel(K.translateAllGPU(a, b), ref) < 1e-12
    assert rel(K.translateAllGPU(a.astype(np.float32), b.astype(np.float32)), ref) < 1e-5


@pytest.mark.parametrize("p", (1, 4, 10))
def test_translate_all_matrix_golden(seam, p):
    a, b, ref = seam[f"tam_p{p}_a"], seam[f"tam_p{p}_b"], seam[f"tam_p{p}_out"]
    assert rel(K.translateAllGPUMatrixCuBLAS(a, b), ref) < 1e-12
    assert rel(K.translateAllGPUMatrixCuBLAS(a.astype(np.float32), b.astype(np.float32)), ref) < 1e-5


@pytest.mark.parametrize("p,count", [(8, 1), (8, 2000), (12, 777), (16, 300), (20, 5)])
def test_translate_all_device_many_items(p, count):
    import torch
    rng = np.random.default_rng(p * 1000 + count)
    L = (p + 1) ** 2
    t = rng.normal(size=(count, 3)) * 0.3
    a = np.stack([O.solid_harmonics(p, x, True, compat=True) for x in t[: min(count, 64)]])
    a = np.resize(a, (count, L))
    b = rng.normal(size=(count, L, 3))
    ref = O.translate_all(p, a, b)
    for dt, tol in ((torch.float64, 1e-12), (torch.float32, 1e-5)):
        got = K.translateAllGPU(torch.tensor(a, dtype=dt, device="cuda"), torch.tensor(b, dtype=dt, device="cuda"))
        torch.cuda.synchronize()
        assert got.is_cuda and got.dtype == dt
        assert rel(got, ref) < tol


@pytest.mark.parametrize("L,count,batch", [(1, 1, 1), (81, 1000, 1), (121, 4097, 3), (289, 130, 2), (300, 65, 1)])
def test_translate_all_matrix_shapes(L, count, batch):
    import torch
    rng = np.random.default_rng(L + count)
    p = int(round(L ** 0.5)) - 1
    if (p + 1) ** 2 != L:
        with pytest.raises(ValueError):
            K.translateAllGPUMatrixCuBLAS(rng.normal(size=(count, L)), rng.normal(size=(L, L)))
        return
    a = rng.normal(size=(batch, count, L))
    b = rng.normal(size=(L, L))
    ref = np.stack([O.translate_all_matrix(a[i], b) for i in range(batch)])
    got = K.translateAllGPUMatrixCuBLAS(torch.tensor(a, device="cuda"), torch.tensor(b, device="cuda"))
    assert rel(got, ref) < 1e-12
    got32 = K.translateAllGPUMatrixCuBLAS(a.astype(np.float32), b.astype(np.float32))
    assert got32.shape == a.shape and rel(got32, ref) < 1e-5


@pytest.mark.parametrize("p,count", [(2, 3), (10, 500)])
def test_translate_all_matrix_complex(p, count):
    rng = np.random.default_rng(7)
    L = (p + 1) ** 2
    a = rng.normal(size=(count, L)) + 1j * rng.normal(size=(count, L))
    b = rng.normal(size=(L, L)) + 1j * rng.normal(size=(L, L))
    ref = a @ b
    assert rel(K.translateAllGPUMatrix(a, b), ref) < 1e-12
    assert rel(K.translateAllGPUMatrix(a.astype(np.complex64), b.astype(np.complex64)), ref) < 1e-5


def test_add_vectors():
    a = np.arange(1000, dtype=np.float32)
    assert np.array_equal(K.addVectors(a, 2 * a), 3 * a)


def test_seam_rejects_bad_arguments():
    from bachelors_b200._lib import FmmError
    with pytest.raises(FmmError):
        K.translateAllGPU(np.zeros((1, 34 ** 2)), np.zeros((1, 34 ** 2, 3)))   # order 33 > 32
