"""CPU checks of the learned-correction oracle (oracle/cnn_oracle.py): its backpropagation
formulas are the adjoints of its forward pass, GELU's derivative is right, and its bfloat16
rounding is round-to-nearest-even.  The GPU gradients are compared against this oracle in
tests/test_gpu_learned.py."""
import numpy as np
import pytest
import torch

from oracle import cnn_oracle as co


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(4000) * 10.0 ** rng.integers(-8, 8, 4000),
                        np.array([1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, -0.0, 0.0])]).astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(co.bf16(x), ref)


def test_gelu_grad_finite_difference():
    x = np.linspace(-6.0, 6.0, 241)
    h = 1e-6
    fd = (co.gelu(x + h) - co.gelu(x - h)) / (2 * h)
    assert np.max(np.abs(fd - co.gelu_grad(x))) < 1e-8


@pytest.mark.parametrize("cin,cout", [(16, 32), (32, 8)])
def test_conv_adjoints(cin, cout):
    rng = np.random.default_rng(cin + cout)
    x = rng.standard_normal((2, 64, 64, cin))
    w = rng.standard_normal((cout, 9, cin))
    dz = rng.standard_normal((2, 64, 64, cout))
    lhs = np.sum(co.conv(x, w) * dz)
    assert np.isclose(lhs, np.sum(x * co.conv_input_grad(dz, w)), rtol=1e-12)
    assert np.isclose(lhs, np.sum(w * co.conv_weight_grad(x, dz)), rtol=1e-12)


def test_conv_taps_and_padding():
    """A single unit weight at tap t shifts the image by off(t) = (t // 3 - 1, t % 3 - 1) with zero fill."""
    rng = np.random.default_rng(5)
    x = rng.standard_normal((1, 64, 64, 16))
    for t in range(9):
        w = np.zeros((32, 9, 16))
        w[3, t, 7] = 1.0
        out = co.conv(x, w)[0, :, :, 3]
        dy, dx = t // 3 - 1, t % 3 - 1
        ref = np.zeros((64, 64))
        for r in range(64):
            for c in range(64):
                if 0 <= r + dy < 64 and 0 <= c + dx < 64:
                    ref[r, c] = x[0, r + dy, c + dx, 7]
        assert np.array_equal(out, ref)
