"""The CPU FP64 MLP reference used to check the GPU proxy's gradients is
itself checked against central finite differences (no GPU)."""
import numpy as np

from tests import mlp_ref


def _params(rng, I, H, O):
    return dict(W1=rng.normal(0, 0.3, (H, I)), b1=rng.normal(0, 0.1, H),
                W2=rng.normal(0, 0.3, (H, H)), b2=rng.normal(0, 0.1, H),
                W3=rng.normal(0, 0.3, (O, H)), b3=rng.normal(0, 0.1, O))


def test_fp64_gradients_match_finite_differences():
    rng = np.random.default_rng(7)
    I, H, O, B = 12, 8, 3, 5
    P = _params(rng, I, H, O)
    X = (rng.random((B, I)) < 0.4).astype(np.float64)
    T = rng.normal(size=(B, O))
    _, g, _ = mlp_ref.forward_backward(P, X, T, bf16=False)
    h = 1e-6
    for name in ("W1", "b1", "W2", "b2", "W3", "b3"):
        flat = P[name].reshape(-1)
        for idx in rng.choice(flat.size, size=min(flat.size, 6), replace=False):
            old = flat[idx]
            flat[idx] = old + h
            lp, _, _ = mlp_ref.forward_backward(P, X, T, bf16=False)
            flat[idx] = old - h
            lm, _, _ = mlp_ref.forward_backward(P, X, T, bf16=False)
            flat[idx] = old
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[name].reshape(-1)[idx]) <= 1e-6 + 1e-5 * abs(fd), (name, idx)


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-3], np.float64)
    r = mlp_ref.to_bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                   # tie -> even mantissa
    assert r[2] == 1.0 + 2 ** -6         # tie -> even (rounds up)
    assert r[3] == -2.5
    assert abs(r[4] - 3.0e-3) / 3.0e-3 < 2 ** -8


def test_adam_reference_first_step_is_sign_step():
    p = np.array([0.5, -0.25, 1.0], np.float32)
    g = np.array([0.1, -0.2, 0.0], np.float32)
    p1, m, v = mlp_ref.adam_update(p, g, np.zeros(3), np.zeros(3), 1, 1e-3, 0.9, 0.999, 1e-8)
    assert np.allclose(p1, p - 1e-3 * np.sign(g), atol=1e-7)
