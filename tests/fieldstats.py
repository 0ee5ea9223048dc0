"""Comparison of two runs' sampled fields within their sampling noise.

Each side is B independent runs (replicas) sampled over the same window of
steps.  Per cell and replica the sums (N, sum u, sum v, sum w, sum |v|^2) give
an estimate of the number per step, the stream velocity ux and the
temperature.  A side's estimate is the mean over its replicas and its noise
the standard error of that mean; replicas see the same transient, so a flow
that is still developing is compared fairly.  Two sides agree when the
per-cell differences, in units of the combined standard error, behave as
noise: few cells beyond 3 sigma and a mean square near one.  With B
replicas a side the z-scores follow a Student-t law of about 2(B - 1) degrees
of freedom: for B = 8, about 1 % of the cells beyond 3 and a mean square of
about 1.17.
"""
import numpy as np

KB = 1.3806e-23


def block_fields(sums, steps_per_block, mass):
    """(B, cells, 5) sums over steps_per_block steps -> (B, cells, 3):
    particles per step, ux, T."""
    N = sums[..., 0]
    with np.errstate(divide="ignore", invalid="ignore"):
        u = sums[..., 1:4] / N[..., None]
        T = mass * (sums[..., 4] / N - np.sum(u * u, axis=-1)) / (3.0 * KB)
    return np.stack([N / steps_per_block, u[..., 0], T], axis=-1)


def compare(sums_a, sums_b, steps_per_block, mass, min_count):
    """z-scores of side a against side b ((B, cells, 5) sums each) over the
    cells where every replica of both sides holds at least min_count
    samples."""
    fa = block_fields(sums_a, steps_per_block, mass)
    fb = block_fields(sums_b, steps_per_block, mass)
    valid = (sums_a[..., 0].min(axis=0) >= min_count) & (sums_b[..., 0].min(axis=0) >= min_count)
    ma, mb = fa.mean(axis=0)[valid], fb.mean(axis=0)[valid]
    sa = fa.std(axis=0, ddof=1)[valid] / np.sqrt(fa.shape[0])
    sb = fb.std(axis=0, ddof=1)[valid] / np.sqrt(fb.shape[0])
    z = (ma - mb) / np.sqrt(sa * sa + sb * sb)
    return {"cells": int(valid.sum()), "z": z,
            "frac_beyond_3": float(np.mean(np.abs(z) > 3.0)),
            "mean_z2": float(np.mean(z * z)),
            "mean_z2_per_field": [float(np.mean(z[:, k] ** 2)) for k in range(z.shape[1])]}


def agree(res, max_frac=0.03, z2_range=(0.6, 1.6)):
    """The acceptance rule of the comparisons: at most max_frac of the
    (cell, field) z-scores beyond 3, and each field's mean square z inside
    z2_range (about 1.2 for 8 against 8 independent estimates)."""
    return res["frac_beyond_3"] <= max_frac and all(
        z2_range[0] <= v <= z2_range[1] for v in res["mean_z2_per_field"])
