"""The CPU restatement of the warm-start MLP (oracle/mlp_oracle.py): BF16 rounding, and its analytic
gradient against finite differences of its own loss (straight-through BF16 rounding switched off by
using parameters and inputs that are exactly representable in BF16)."""
import numpy as np

from oracle import mlp_oracle as MO


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.0078125, 3.0e-3, 65504.0], np.float32)
    y = MO.bf16(x)
    assert y[0] == 1.0 and y[1] == 1.0  # halfway rounds to even
    assert y[2] == np.float32(1.0078125)
    assert np.all(np.abs(y - x) <= np.abs(x) * 2.0 ** -8)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = MO.bf16(rng.normal(0, 0.2, MO.N_PARAMS).astype(np.float32)).astype(np.float64)
    X = MO.bf16(rng.normal(size=(40, 16)).astype(np.float32)).astype(np.float64)
    X[:, 15] = 0.0
    T = rng.normal(size=(40, 3))
    # FD on the last layer and the biases (no BF16 rounding downstream of them)
    loss, g = MO.loss_and_grad(p, X, T)
    for name in ("W4", "b4"):
        o, shape = MO.OFF[name]
        for j in [0, 1, 2, 5]:
            idx = o + j
            if name == "W4":
                idx = o + j * 7  # entries of rows 0..2
            # weights are rounded to BF16 in the forward: step by exactly one BF16 ulp of the entry
            h = 2.0 ** (np.floor(np.log2(abs(p[idx]))) - 7) if name == "W4" else 1e-4
            pp, pm = p.copy(), p.copy()
            pp[idx] += h
            pm[idx] -= h
            fd = (MO.loss_and_grad(pp, X, T)[0] - MO.loss_and_grad(pm, X, T)[0]) / (2 * h)
            assert abs(fd - g[idx]) <= 1e-5 + 1e-4 * abs(g[idx])
