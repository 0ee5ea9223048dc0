"""The surrogate's CPU oracle: its analytic gradients against central finite
differences of the exact (float64, no BF16 rounding) network."""
import numpy as np

from oracle import mlp_oracle as M


def small_params(rng, n_in=16, hidden=12, depth=2, modes=6, F=40):
    dims = [n_in] + [hidden] * depth
    return {"W": [rng.normal(0, 0.5, (dims[l], hidden)) for l in range(depth)],
            "b": [rng.normal(0, 0.1, hidden) for _ in range(depth)],
            "Wout": rng.normal(0, 0.3, (hidden, modes)), "bout": rng.normal(0, 0.1, modes),
            "B": rng.normal(0, 0.3, (modes, F)), "mean": rng.normal(0, 0.1, F)}


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    p = small_params(rng)
    x = rng.normal(0, 1, (5, 16))
    t = rng.normal(0, 1, (5, 40))
    t[0, :7] = np.nan
    loss, g, _ = M.loss_and_grads(p, x, t, bf16_points=False)
    eps = 1e-6

    def num(get, set_, shape):
        out = np.zeros(shape)
        for idx in np.ndindex(*shape):
            v = get()[idx]
            a = get().copy(); a[idx] = v + eps; set_(a); lp = M.loss_and_grads(p, x, t, False)[0]
            a = get().copy(); a[idx] = v - eps; set_(a); lm = M.loss_and_grads(p, x, t, False)[0]
            a = get().copy(); a[idx] = v; set_(a)
            out[idx] = (lp - lm) / (2 * eps) / t.size
        return out

    # the oracle's loss is the plain sum; its gradients carry the 1/n scale
    for key in ("Wout", "bout", "mean"):
        n = num(lambda: p[key], lambda a: p.__setitem__(key, a), p[key].shape)
        assert np.allclose(g[key], n, rtol=1e-5, atol=1e-9), key
    sub = (slice(0, 3), slice(0, 4))
    nB = num(lambda: p["B"], lambda a: p.__setitem__("B", a), p["B"].shape)
    assert np.allclose(g["B"], nB, rtol=1e-5, atol=1e-9)
    for l in range(2):
        nW = num(lambda: p["W"][l], lambda a: p["W"].__setitem__(l, a), p["W"][l].shape)
        assert np.allclose(g["W"][l], nW, rtol=1e-5, atol=1e-9), l
        nb = num(lambda: p["b"][l], lambda a: p["b"].__setitem__(l, a), p["b"][l].shape)
        assert np.allclose(g["b"][l], nb, rtol=1e-5, atol=1e-9), l
    del sub


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.01171875, -3.14159265, 65504.0, np.nan, 1e-40], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0            # halfway: ties to even (mantissa 0)
    assert r[2] == 1.015625       # halfway: ties to even (mantissa 2)
    assert r[3] == -3.140625
    assert np.isnan(r[5])
