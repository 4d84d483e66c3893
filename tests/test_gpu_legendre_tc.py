"""Tensor-core (tcgen05, BF16x3 and BF16x6) Legendre contraction against numpy FP64.

The split-precision product A B^T ~ A0 B0^T + A0 B1^T + A1 B0^T (BF16x3)
keeps about 16 significant bits per operand, so every element must satisfy
|D - D_exact| <= 3e-5 * sum_k |A_k| |B_k|  (BF16x3 bound, FP32 accumulation).
BF16x6 adds A0 B2^T + A2 B0^T + A1 B1^T (the operands are split exactly into
three bf16 parts), so it must meet the FP32 CUDA-core kernel's bound, 1e-6.  Shapes cover the
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


@pytest.mark.parametrize("tile_rows", [128, 64])
@pytest.mark.parametrize("shape", SHAPES)
def test_tensor_core_contraction(cuda, shape, tile_rows):
    A, B, exact, scale = _case(*shape, seed=sum(shape))
    D = run_legendre(A, B, tensor_cores=True, tile_rows=tile_rows)
    assert np.isfinite(D).all()
    err = np.abs(D - exact) / scale
    assert err.max() <= 3e-5, err.max()
    # it is not just FP32 rounding of a BF16 product: the split recovers ~16 bits
    assert np.median(err) <= 2e-6


@pytest.mark.parametrize("tile_rows", [128, 64])
@pytest.mark.parametrize("shape", SHAPES)
def test_tensor_core_six_products(cuda, shape, tile_rows):
    A, B, exact, scale = _case(*shape, seed=11 + sum(shape))
    D6 = run_legendre(A, B, tensor_cores=True, terms=6, tile_rows=tile_rows)
    D3 = run_legendre(A, B, tensor_cores=True, terms=3, tile_rows=tile_rows)
    e6 = np.abs(D6 - exact) / scale
    e3 = np.abs(D3 - exact) / scale
    assert e6.max() <= 1e-6, e6.max()
    # the three extra products are not a no-op: the median error drops by >= 8x
    assert np.median(e6) * 8 <= np.median(e3)


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
    for terms, tol in ((3, 3e-5), (6, 1e-6)):
        D = run_legendre(A, B, tensor_cores=True, tri=True, terms=terms)
        assert (np.abs(D - exact) / scale).max() <= tol
