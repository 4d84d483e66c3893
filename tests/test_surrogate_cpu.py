"""CPU tests of the surrogate's host logic: bf16 rounding used for the
weights and operand images."""
import numpy as np

from suguru_b200.coupling import from_bf16_bits, to_bf16_bits


def test_bf16_rounding_matches_torch():
    import torch
    x = np.random.default_rng(0).normal(size=10000).astype(np.float32) * 1e3
    ref = torch.from_numpy(x).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    assert np.array_equal(to_bf16_bits(x), ref)
    back = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(from_bf16_bits(to_bf16_bits(x)), back)


def _params(rng, din, dh, dout, scale=0.5):
    n = dh * din + dh + dh * dh + dh + dout * dh + dout
    return rng.normal(size=n) * scale


def test_mlp_oracle_gradient_matches_finite_differences():
    """The float64 oracle's backward pass is the derivative of its loss."""
    import mlp_oracle as M
    rng = np.random.default_rng(3)
    din, dh, dout, B = 6, 5, 4, 3
    p = _params(rng, din, dh, dout)
    X = rng.normal(size=(B, din))
    T = rng.normal(size=(B, dout))
    loss, g = M.forward_backward(p, X, T, din, dh, dout, emulate_bf16=False)
    h = 1e-6
    fd = np.zeros_like(p)
    for i in range(p.size):
        e = np.zeros_like(p)
        e[i] = h
        fd[i] = (M.forward_backward(p + e, X, T, din, dh, dout, False)[0]
                 - M.forward_backward(p - e, X, T, din, dh, dout, False)[0]) / (2 * h)
    assert np.abs(g - fd).max() <= 1e-8 * max(1.0, np.abs(fd).max())


def test_mlp_oracle_bf16_emulation_is_close_to_exact():
    import mlp_oracle as M
    rng = np.random.default_rng(4)
    din, dh, dout, B = 64, 64, 64, 64
    p = _params(rng, din, dh, dout, scale=0.1)
    X = rng.normal(size=(B, din))
    T = rng.normal(size=(B, dout))
    l0, g0 = M.forward_backward(p, X, T, din, dh, dout, emulate_bf16=False)
    l1, g1 = M.forward_backward(p, X, T, din, dh, dout, emulate_bf16=True)
    assert abs(l1 - l0) <= 1e-2 * l0
    assert np.linalg.norm(g1 - g0) <= 2e-2 * np.linalg.norm(g0)
