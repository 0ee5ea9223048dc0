"""Host-side pieces of the warm-start study: the block state from sampling
sums and from per-cell fields agree, and the half-window noise estimate
removes the statistical part of the error."""
import math

import numpy as np

from cudadsmc_b200 import warmstart as W


def synthetic_sums(rng, cond, ns, scale=1.0):
    """Per-cell sums of ns samples drawn around a smooth field."""
    n_inf, U = W.free_stream(cond)
    st = W.settings_of(cond, 0)
    cell_v = (W.DOM[0] / W.DIM[0]) * (W.DOM[1] / W.DIM[1]) * (W.DOM[2] / W.DIM[2])
    ppc = n_inf * cell_v / st["fnum"]
    x = np.linspace(0, 1, W.CELLS)
    N = rng.poisson(ppc * ns * (1 + 0.5 * np.sin(6 * x)) * scale).astype(np.float64)
    N[:500] = 0  # a body
    vstd = np.sqrt(W.KB * W.T_INF * (1 + x) / W.ARGON["gas_mass"])
    u = np.stack([U * (1 - 0.3 * x), 0.05 * U * np.cos(9 * x), 0 * x], axis=1)
    su = N[:, None] * u + rng.normal(0, 1, (W.CELLS, 3)) * vstd[:, None] * np.sqrt(np.maximum(N, 0))[:, None]
    e = N * (np.sum(u * u, axis=1) + 3 * vstd ** 2)
    return np.column_stack([N, su, e])


def test_block_state_from_fields_matches_sums():
    rng = np.random.default_rng(1)
    cond = (5.0, 0.1, 2.0, 0.1)
    ns = 50
    sums = synthetic_sums(rng, cond, ns)
    n_inf, U = W.free_stream(cond)
    st = W.settings_of(cond, 0)
    cell_v = (W.DOM[0] / W.DIM[0]) * (W.DOM[1] / W.DIM[1]) * (W.DOM[2] / W.DIM[2])
    N = sums[:, 0]
    f = np.full((W.CELLS, 5), np.nan)
    ok = N > 0
    f[ok, 0] = N[ok] * st["fnum"] / (cell_v * ns) / n_inf
    uu = sums[ok, 1:4] / N[ok, None]
    f[ok, 1:4] = uu / U
    f[ok, 4] = W.ARGON["gas_mass"] * (sums[ok, 4] / N[ok] - np.sum(uu * uu, axis=1)) / (3 * W.KB) / W.T_INF
    a = W.block_state_from_sums(sums, ns, cond)
    b = W.block_state_from_fields(f, cond, ~ok)
    good = np.all(np.isfinite(a), axis=1)
    assert good.sum() > 0.9 * len(a)
    assert np.allclose(a[good], b[good], rtol=1e-9, atol=1e-9)


def test_noise_subtraction_recovers_the_systematic_error():
    rng = np.random.default_rng(2)
    cond = (6.0, 0.3, 1.5, 0.08)
    ref_sums = [synthetic_sums(rng, cond, 400) for _ in range(2)]
    run_sums = [synthetic_sums(rng, cond, 20) for _ in range(2)]
    ref = W.block_state_from_sums(ref_sums[0] + ref_sums[1], 800, cond)
    ref_noise = W.half_noise(W.block_state_from_sums(ref_sums[0], 400, cond),
                             W.block_state_from_sums(ref_sums[1], 400, cond))
    b1 = W.block_state_from_sums(run_sums[0], 20, cond)
    b2 = W.block_state_from_sums(run_sums[1], 20, cond)
    mid = W.block_state_from_sums(run_sums[0] + run_sums[1], 40, cond)
    raw = W.field_error(mid, ref)
    corrected = W.field_error(mid, ref, noise2=W.half_noise(b1, b2) + ref_noise)
    assert raw > 0.003
    assert corrected < 0.5 * raw  # same underlying field: what remains is mostly noise residue


def test_inputs_and_free_stream():
    c = W.sample_conditions(1000, 3)
    assert np.all((c[:, 0] >= 2) & (c[:, 0] <= 10))
    assert np.all((c[:, 1] >= 0.01) & (c[:, 1] <= 1))
    x = W.normalize_inputs(c)
    assert np.all(np.abs(x) <= 1.0 + 1e-6)
    n_inf, U = W.free_stream((2.0, 0.01, 1.0, 0.1))
    assert 5e20 < n_inf < 8e20 and 500 < U < 540


def test_two_stream_weight_ramps_with_log_kn():
    assert W.two_stream_weight((5.0, 0.01, 2.0, 0.1)) == 0.0
    assert W.two_stream_weight((5.0, 0.005, 2.0, 0.1)) == 0.0
    assert abs(W.two_stream_weight((5.0, 0.1, 2.0, 0.1)) - 2.0 / 3.0) < 1e-12
    assert W.two_stream_weight((5.0, 0.5, 2.0, 0.1)) == 1.0
