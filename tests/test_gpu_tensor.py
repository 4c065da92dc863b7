"""The tcgen05 GEMM building block of the learned closure: D = A B^T with BF16
operands and FP32 accumulation in tensor memory, against numpy on the same
BF16-rounded operands."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even to bfloat16, returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


@pytest.mark.parametrize("K,N", [(16, 16), (16, 64), (64, 64), (32, 48), (64, 16), (80, 64), (80, 16)])
def test_tensor_gemm(K, N):
    import freeshearlayer_b200 as fsl
    fn = fsl.lib().fsl_selftest_tensor_gemm
    fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
    fn.argtypes = [fp, fp, fp, C.c_int, C.c_int]
    fn.restype = C.c_int
    rng = np.random.default_rng(K * 100 + N)
    A = rng.standard_normal((128, K)).astype(np.float32)
    B = rng.standard_normal((N, K)).astype(np.float32)
    D = np.zeros((128, N), np.float32)
    rc = fn(A, B, D, K, N)
    assert rc == 0, rc
    ref = bf16_round(A).astype(np.float64) @ bf16_round(B).astype(np.float64).T
    np.testing.assert_allclose(D, ref, rtol=1e-5, atol=1e-5)
