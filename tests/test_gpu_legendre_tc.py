"""Tensor-core (tcgen05, BF16x3) Legendre contraction against numpy FP64.

The split-precision product A B^T ~ A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T
keeps about 16 significant bits per operand, so every element must satisfy
|D - D_exact| <= 3e-5 * sum_k |A_k| |B_k|  (BF16x3 bound, FP32 accumulation);
the FP32 CUDA-core kernel must satisfy the same with 1e-6.  Shapes cover the
coupling step's stages (J = N, 3 nD, 2 nO, nD; K = N, nD, nO) and ragged
sizes that exercise the padding of J, K to multiples of 16 and partial
128-row tiles.
"""
import numpy as np
import pytest

from suguru_b200.coupling import test_legendre as run_legendre

pytestmark = pytest.mark.gpu

SHAPES = [  # (M, Q, J, K)
    (16, 1536, 16, 32),   # analysis on the force grid, L = 15
    (16, 1536, 96, 16),   # synthesis with derivatives, L = 15
    (16, 1536, 32, 16),   # synthesis on the SH grid / force grid
    (24, 300, 144, 48),   # L = 23: J = 3 nD = 144, K = nD = 48
    (9, 77, 27, 9),       # L = 8: odd sizes, one partial tile
    (3, 130, 40, 20),     # ragged
]


def _case(M, Q, J, K, seed):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(M, Q, K)).astype(np.float32)
    B = rng.normal(size=(M, J, K)) * np.exp(rng.uniform(-3, 3, size=(M, J, 1)))
    exact = np.einsum("mqk,mjk->mqj", A.astype(np.float64), B)
    scale = np.einsum("mqk,mjk->mqj", np.abs(A.astype(np.float64)), np.abs(B))
    return A, B, exact, scale


@pytest.mark.parametrize("shape", SHAPES)
def test_tensor_core_contraction(cuda, shape):
    A, B, exact, scale = _case(*shape, seed=sum(shape))
    D = run_legendre(A, B, tensor_cores=True)
    assert np.isfinite(D).all()
    err = np.abs(D - exact) / scale
    assert err.max() <= 3e-5, err.max()
    # it is not just FP32 rounding of a BF16 product: the split recovers ~16 bits
    assert np.median(err) <= 2e-6


@pytest.mark.parametrize("shape", SHAPES[:3])
def test_cuda_core_contraction(cuda, shape):
    A, B, exact, scale = _case(*shape, seed=7 + sum(shape))
    D = run_legendre(A, B, tensor_cores=False)
    assert (np.abs(D - exact) / scale).max() <= 1e-6


def test_triangular_synthesis(cuda):
    # synthesis tables vanish for n < m; the tensor-core kernel skips K steps
    # wholly below m, which must not change the result
    M, Q, J, K = 40, 256, 32, 40
    A, B, _, _ = _case(M, Q, J, K, seed=3)
    for m in range(M):
        B[m, :, :m] = 0.0
    exact = np.einsum("mqk,mjk->mqj", A.astype(np.float64), B)
    scale = np.einsum("mqk,mjk->mqj", np.abs(A.astype(np.float64)), np.abs(B)) + 1e-300
    D = run_legendre(A, B, tensor_cores=True, tri=True)
    assert (np.abs(D - exact) / scale).max() <= 3e-5
