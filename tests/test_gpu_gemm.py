"""Tensor-core dense products of the surrogate network against numpy FP64.

bf16 mode: the products of bf16-rounded operands are exact in FP32, so the
only error is FP32 accumulation: |C - C_exact| <= 1e-6 * sum_k |a_k b_k|.
split mode (BF16x3): |C - C_exact| <= 3e-5 * sum_k |a_k| |b_k| against the
FP32 operands.  The fused epilogue (scale, bias, GELU with the erf form, the
pre-activation, bf16 and transposed bf16 copies) is checked element-wise.
"""
import math

import numpy as np
import pytest

from suguru_b200.coupling import from_bf16_bits, to_bf16_bits
from suguru_b200.coupling import test_gemm as run_gemm

pytestmark = pytest.mark.gpu

SHAPES = [(128, 128, 64), (300, 200, 192), (4096, 1024, 832), (77, 768, 1024), (1, 16, 64)]


def _bf(x):
    return from_bf16_bits(to_bf16_bits(x)).astype(np.float64)


@pytest.mark.parametrize("splitk", [False, True])
@pytest.mark.parametrize("shape", SHAPES)
def test_gemm_bf16(cuda, shape, splitk):
    M, N, K = shape
    rng = np.random.default_rng(M + N + K)
    A = rng.normal(size=(M, K)).astype(np.float32)
    B = rng.normal(size=(N, K)).astype(np.float32)
    C, _, _, _ = run_gemm(A, B, split=False, splitk=splitk)
    Ab, Bb = _bf(A), _bf(B)
    exact = Ab @ Bb.T
    scale = np.abs(Ab) @ np.abs(Bb).T
    assert (np.abs(C - exact) / scale).max() <= 1e-6


@pytest.mark.parametrize("splitk", [False, True])
@pytest.mark.parametrize("shape", SHAPES[:4])
def test_gemm_split(cuda, shape, splitk):
    M, N, K = shape
    rng = np.random.default_rng(1 + M + N + K)
    A = (rng.normal(size=(M, K)) * np.exp(rng.uniform(-2, 2, size=(M, 1)))).astype(np.float32)
    B = rng.normal(size=(N, K)).astype(np.float32)
    C, _, _, _ = run_gemm(A, B, split=True, splitk=splitk)
    A64, B64 = A.astype(np.float64), B.astype(np.float64)
    exact = A64 @ B64.T
    scale = np.abs(A64) @ np.abs(B64).T
    err = np.abs(C - exact) / scale
    assert err.max() <= 3e-5
    assert np.median(err) <= 2e-6


@pytest.mark.parametrize("splitk", [False, True])
def test_gemm_epilogue(cuda, splitk):
    M, N, K = 260, 136, 512
    rng = np.random.default_rng(9)
    A = rng.normal(size=(M, K)).astype(np.float32)
    B = (0.2 * rng.normal(size=(N, K))).astype(np.float32)
    bias = rng.normal(size=N).astype(np.float32)
    C, P, Cb, CbT = run_gemm(A, B, split=False, bias=bias, gelu=True, alpha=0.5, splitk=splitk)
    pre = 0.5 * (_bf(A) @ _bf(B).T) + bias
    gel = 0.5 * pre * (1.0 + np.vectorize(math.erf)(pre / math.sqrt(2.0)))
    assert np.abs(P - pre).max() <= 1e-5 * (1 + np.abs(pre).max())
    assert np.abs(C - gel).max() <= 1e-5 * (1 + np.abs(gel).max())
    assert np.array_equal(Cb, _bf(C.astype(np.float32)).astype(np.float32))
    assert np.array_equal(CbT, Cb.T)

