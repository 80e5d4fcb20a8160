"""The MLP oracle itself (oracle/mlp.py), on the CPU: its backward pass
against central differences of its loss, and its BF16 rounding against
torch's."""

import numpy as np


def test_mlp_oracle_gradients_finite_differences():
    from oracle.mlp import finite_difference_check

    assert finite_difference_check(seed=0) < 1e-6
    assert finite_difference_check(seed=1, M=11, K=9, H=5, N=3) < 1e-6
    assert finite_difference_check(seed=2, M=9, K=6, H=5, N=3, layers=3) < 1e-6


def test_bf16_rounding_matches_torch():
    import torch

    from oracle.mlp import bf16

    x = np.random.default_rng(0).standard_normal(4096) * np.logspace(-6, 6, 4096)
    want = torch.as_tensor(x, dtype=torch.float32).to(torch.bfloat16).double().numpy()
    np.testing.assert_array_equal(bf16(x), want)
