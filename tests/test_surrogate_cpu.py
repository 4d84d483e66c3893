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
