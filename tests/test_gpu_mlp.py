"""The surrogate network's BF16 tensor-core kernels (tcgen05) on the GPU.

GEMM: C = A B^T with BF16 operands and FP32 accumulation, checked against
the exact product of the same BF16 values (float64 on the host); tolerance
2^-20 of the sum of |a_k b_k| per entry (FP32 accumulation of at most 8192
terms)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def to_bf16_bits(x):
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    return ((b + 0x7FFF + ((b >> 16) & 1)) >> 16).astype(np.uint16)


def from_bf16_bits(h):
    return (h.astype(np.uint32) << 16).view(np.float32)


@pytest.fixture(scope="module")
def lib():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    from unicorn_b200 import unichem
    L = unichem.load_library()
    U16 = ctypes.POINTER(ctypes.c_uint16)
    L.uc_gemm_bf16.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, U16, U16,
                               ctypes.POINTER(ctypes.c_float)]
    return L


@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (300, 256, 64), (128, 64, 256), (1000, 48, 128),
                                   (256, 512, 64), (200, 16, 8192)])
def test_gemm_matches_host(lib, M, N, K):
    rng = np.random.default_rng(M * 7 + N + K)
    a = to_bf16_bits(rng.standard_normal((M, K)))
    b = to_bf16_bits(rng.standard_normal((N, K)))
    c = np.zeros((M, N), dtype=np.float32)
    U16 = ctypes.POINTER(ctypes.c_uint16)
    rc = lib.uc_gemm_bf16(0, M, N, K, a.ctypes.data_as(U16), b.ctypes.data_as(U16),
                          c.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    assert rc == 0
    A, B = from_bf16_bits(a).astype(np.float64), from_bf16_bits(b).astype(np.float64)
    ref = A @ B.T
    scale = np.abs(A) @ np.abs(B).T
    assert (np.abs(c - ref) <= 2.0 ** -20 * scale + 1e-30).all(), np.max(np.abs(c - ref) / scale)


def test_gemm_rejects_bad_shapes(lib):
    U16 = ctypes.POINTER(ctypes.c_uint16)
    a = np.zeros(64 * 64, np.uint16)
    c = np.zeros(64 * 64, np.float32)
    P = lambda x: x.ctypes.data_as(U16)
    F = c.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    assert lib.uc_gemm_bf16(0, 64, 20, 64, P(a), P(a), F) == -1      # N not a multiple of 16
    assert lib.uc_gemm_bf16(0, 64, 16, 40, P(a), P(a), F) == -1      # K not a multiple of 64
