"""The CPU oracle of the learned-guess network (CPU test): its gradients
against central finite differences of its own loss in float64, and its
bfloat16 rounding against known values."""
import numpy as np

from oracle import mlp_ref


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.140625, 1e-3, 65504.0], dtype=np.float32)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to even (1.0);
    # 1 + 1.5 * 2^-8 rounds up to 1 + 2^-7
    want = np.array([1.0, 1.0, 1.0078125, -3.140625, 0.00099945068359375, 65536.0])
    assert np.array_equal(mlp_ref.bf16(x), want)


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    dims = [16, 24, 8]
    nparam = sum(a * b + b for a, b in zip(dims[:-1], dims[1:]))
    p = rng.normal(scale=0.3, size=nparam)
    X = rng.normal(size=(5, dims[0]))
    T = rng.normal(size=(5, dims[-1]))
    g, _ = mlp_ref.gradients(dims, p, X, T, rounding=False)
    h = 1e-6
    idx = rng.choice(nparam, 40, replace=False)
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp = mlp_ref.gradients(dims, pp, X, T, rounding=False)[1]
        lm = mlp_ref.gradients(dims, pm, X, T, rounding=False)[1]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) < 1e-7 * max(1.0, abs(fd))
