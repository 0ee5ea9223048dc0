"""Learned warm start of the sphere flow: generate steady fields with this
DSMC, train the surrogate on them, and compare the time to steady state of
warm-started runs (particles seeded from the predicted fields) with the
plain cold start (free-stream fill) on held-out conditions.  The warm runs
use the two-stream fill, each cell a mixture of the free stream and
molecules at the wall temperature weighted by the condition's Kn
(`--seeding two-stream`, the default), and also, for comparison, a local
Maxwellian per cell (`--seeding maxwell` runs that one alone).

The flow: argon VHS (omega 0.81) at T_inf = 200 K over a diffuse sphere of
radius r in a 1.2 x 0.6 x 0.6 m box of 64 x 32 x 32 cells, inflow at -x and
outflow elsewhere, about `ppc` particles per cell.  A condition is (Mach,
Kn, T_wall / T_inf, r); Kn is based on the sphere diameter.

    python -m cudadsmc_b200.warmstart --train 2000 --test 100 --out result.json
"""
import argparse
import json
import math
import time

import numpy as np

KB = 1.3806e-23
ARGON = dict(gas_mass=6.63e-26, gas_diam=4.17e-10, gas_tref=273.0, gas_omega=0.81)
T_INF = 200.0
DOM, DIM = (1.2, 0.6, 0.6), (64, 32, 32)
CELLS = DIM[0] * DIM[1] * DIM[2]
CENTER = (0.4, 0.3, 0.3)
CHANNELS = 5  # n, u, v, w, T


def sample_conditions(n, seed):
    """Mach U[2, 10], Kn log-U[0.01, 1], T_wall/T_inf U[1, 3], r U[0.05, 0.15] m."""
    g = np.random.default_rng(seed)
    return np.stack([g.uniform(2, 10, n), np.exp(g.uniform(math.log(0.01), 0.0, n)),
                     g.uniform(1, 3, n), g.uniform(0.05, 0.15, n)], axis=1)


def normalize_inputs(cond):
    c = np.asarray(cond, np.float64)
    return np.stack([(c[:, 0] - 6.0) / 4.0, (np.log10(c[:, 1]) + 1.0), c[:, 2] - 2.0,
                     (c[:, 3] - 0.1) / 0.05], axis=1).astype(np.float32)


def free_stream(cond):
    """(n_inf [m^-3], U [m/s]) of a condition."""
    mach, kn, _, r = cond
    m, d = ARGON["gas_mass"], ARGON["gas_diam"]
    n_inf = 1.0 / (math.sqrt(2.0) * math.pi * d * d * kn * 2.0 * r)
    u = mach * math.sqrt(5.0 / 3.0 * KB * T_INF / m)
    return n_inf, u


def settings_of(cond, seed, ppc=7.6, sample_every=2):
    mach, kn, tw, r = cond
    n_inf, u = free_stream(cond)
    cell = [DOM[k] / DIM[k] for k in range(3)]
    cell_v = cell[0] * cell[1] * cell[2]
    m = ARGON["gas_mass"]
    cmp = math.sqrt(2 * KB * T_INF / m)
    cbar = math.sqrt(8 * KB * T_INF / (math.pi * m))
    lam = kn * 2.0 * r
    dt = min(0.2 * min(cell) / (u + 3 * cmp), 0.2 * lam / cbar)
    return dict(grid_min=(0, 0, 0), grid_max=DOM, grid_dim=DIM, density=n_inf,
                fnum=n_inf * cell_v / ppc, temp=T_INF, stream_vel=(u, 0.0, 0.0), dt=dt, rng="philox",
                ntc_local=1, sample_every=sample_every, init_kind="maxwell", wall_diffuse=1,
                wall_temp=tw * T_INF, capacity_factor=2.0, seed=seed, geom_nearest=1,
                face_kind={"-x": "inflow", "+x": "outflow", "-y": "outflow", "+y": "outflow",
                           "-z": "outflow", "+z": "outflow"}, **ARGON)


def make_solver(cond, seed):
    import cudadsmc_b200 as cb
    sol = cb.DSMCSolver().Init(cb.settings_t().set(**settings_of(cond, seed)))
    v, t = cb.mesh_icosphere(3, float(cond[3]), CENTER)
    sol.SetModel(v, t, (16, 16, 16))
    return sol


def two_stream_weight(cond):
    """Weight of the two-stream seeding (InitFromFieldsTwoStream) of a
    condition: 0 at Kn 0.01, where the cells are near equilibrium, rising
    with log Kn to 1 from Kn 0.32 on, where free-stream molecules and
    molecules re-emitted by the wall share the cells."""
    return float(np.clip((math.log10(cond[1]) + 2.0) / 1.5, 0.0, 1.0))


def seed_from(sol, norm, cond, seeding):
    """Seeds sol from normalized per-cell fields: a local Maxwellian per cell
    ("maxwell") or the two-stream mixture weighted by the condition's Kn."""
    f = physical_fields(norm, cond)
    if seeding == "two-stream":
        return sol.InitFromFieldsTwoStream(f, two_stream_weight(cond))
    return sol.InitFromFields(f)


def normalized_fields(sol, cond):
    """The sampled fields divided by the free stream (n_inf, U, U, U, T_inf);
    NaN in cells that received no particle."""
    n_inf, u = free_stream(cond)
    f = sol.Fields().astype(np.float64)
    out = f / np.array([n_inf, u, u, u, T_INF])
    out[f[:, 0] <= 0] = np.nan
    return out.astype(np.float32)


def physical_fields(norm, cond):
    n_inf, u = free_stream(cond)
    return (np.asarray(norm, np.float64) * np.array([n_inf, u, u, u, T_INF])).astype(np.float32)


BLOCK = 4  # the error is measured on blocks of BLOCK^3 cells


def _block_sums(a):
    """Sums over blocks of BLOCK^3 cells of a [cells, k] array."""
    k = a.shape[-1]
    b = np.asarray(a, np.float64).reshape(DIM[2] // BLOCK, BLOCK, DIM[1] // BLOCK, BLOCK,
                                          DIM[0] // BLOCK, BLOCK, k)
    return b.sum(axis=(1, 3, 5)).reshape(-1, k)


def block_state_from_sums(sums, ns, cond):
    """Normalized block state (n/n_inf, u/U, v/U, w/U, T/T_inf) from the
    per-cell sampling sums (N, sum u, sum v, sum w, sum |v|^2) of ns samples:
    moments added over each block first, so that sparse cells bias nothing;
    NaN for blocks without samples."""
    n_inf, U = free_stream(cond)
    st = settings_of(cond, 0)
    cell_v = (DOM[0] / DIM[0]) * (DOM[1] / DIM[1]) * (DOM[2] / DIM[2])
    S = _block_sums(sums)
    N = S[:, 0]
    out = np.full((len(S), CHANNELS), np.nan)
    ok = N > 0
    out[ok, 0] = N[ok] * st["fnum"] / (cell_v * BLOCK ** 3 * ns) / n_inf
    u = S[ok, 1:4] / N[ok, None]
    out[ok, 1:4] = u / U
    e = S[ok, 4] / N[ok]
    out[ok, 4] = ARGON["gas_mass"] * (e - np.sum(u * u, axis=1)) / (3 * KB) / T_INF
    return out


def cell_fields_from_sums(sums, ns, cond):
    """Normalized per-cell fields (as normalized_fields gives them) from
    sampling sums."""
    n_inf, U = free_stream(cond)
    st = settings_of(cond, 0)
    cell_v = (DOM[0] / DIM[0]) * (DOM[1] / DIM[1]) * (DOM[2] / DIM[2])
    N = sums[:, 0]
    out = np.full((len(N), CHANNELS), np.nan)
    ok = N > 0
    out[ok, 0] = N[ok] * st["fnum"] / (cell_v * ns) / n_inf
    u = sums[ok, 1:4] / N[ok, None]
    out[ok, 1:4] = u / U
    out[ok, 4] = ARGON["gas_mass"] * (sums[ok, 4] / N[ok] - np.sum(u * u, axis=1)) / (3 * KB) / T_INF
    return out.astype(np.float32)


def block_state_from_fields(norm, cond, empty):
    """The same block state from per-cell normalized fields (a prediction),
    weighting each cell by its density; cells in `empty` (no particles in
    the reference run, e.g. inside the body) count as vacuum."""
    n_inf, U = free_stream(cond)
    f = np.asarray(norm, np.float64)
    w = np.where(empty | ~np.isfinite(f[:, 0]), 0.0, np.maximum(f[:, 0], 0.0))
    u = np.where(np.isfinite(f[:, 1:4]), f[:, 1:4], 0.0)
    T = np.where(np.isfinite(f[:, 4]), f[:, 4], 1.0)
    k_u2 = 3 * KB * T_INF / (ARGON["gas_mass"] * U * U)
    e = np.sum(u * u, axis=1) + k_u2 * T
    S = _block_sums(np.column_stack([w, w[:, None] * u, w * e]))
    W = S[:, 0]
    out = np.full((len(S), CHANNELS), np.nan)
    ok = W > 0
    out[ok, 0] = W[ok] / BLOCK ** 3
    ub = S[ok, 1:4] / W[ok, None]
    out[ok, 1:4] = ub
    out[ok, 4] = (S[ok, 4] / W[ok] - np.sum(ub * ub, axis=1)) / k_u2
    return out


def field_error(a, ref, noise2=0.0):
    """Relative L2 difference of two block states (blocks undefined in either
    are left out).  noise2, the expected squared norm of the statistical
    noise in the difference, is subtracted, so that what remains is the
    systematic part."""
    ok = np.all(np.isfinite(a), axis=-1) & np.all(np.isfinite(ref), axis=-1)
    d2 = float(np.sum((a[ok] - ref[ok]) ** 2))
    return math.sqrt(max(0.0, d2 - noise2)) / float(np.linalg.norm(ref[ok]))


def half_noise(b1, b2):
    """Squared noise norm of the state of two pooled independent half-window
    samples, from their difference: E|b1 - b2|^2 / 4."""
    ok = np.all(np.isfinite(b1), axis=-1) & np.all(np.isfinite(b2), axis=-1)
    return float(np.sum((b1[ok] - b2[ok]) ** 2)) / 4.0


def run_group(conds, seeds, settle, sample, halves=False):
    """Runs the conditions together (one graph launch per step) from the
    free-stream fill.  Returns their normalized per-cell fields sampled over
    `sample` steps after `settle`, or with halves the per-cell sampling sums
    and sample counts of the two half-windows."""
    import cudadsmc_b200 as cb
    sols = [make_solver(c, s) for c, s in zip(conds, seeds)]
    for sol in sols:
        sol.InitSystemState()
    batch = cb.DSMCBatch(sols)
    batch.Step(settle)
    batch.Sync()
    parts = []
    for w in ((sample // 2, sample - sample // 2) if halves else (sample,)):
        for sol in sols:
            sol.ResetSamples()
        batch.Step(w)
        batch.Sync()
        if halves:
            parts.append([sol.SampleStatistics()[::2] for sol in sols])
        else:
            parts.append(np.stack([normalized_fields(s, c) for s, c in zip(sols, conds)]))
    batch.close()
    for s in sols:
        s.close()
    return parts if halves else parts[0]


def generate(conds, seed, settle, sample, group=64, log=print):
    out = np.empty((len(conds), CELLS, CHANNELS), np.float32)
    t0 = time.time()
    for i in range(0, len(conds), group):
        sl = slice(i, min(len(conds), i + group))
        seeds = [seed + j for j in range(sl.start, sl.stop)]
        out[sl] = run_group(conds[sl], seeds, settle, sample)
        if log:
            log(f"fields {sl.stop}/{len(conds)} ({time.time() - t0:.0f} s)")
    return out


def convergence(conds, seeds, refs, ref_noise, window, max_steps, threshold, warm=None, stride=None,
                seeding="maxwell"):
    """Steps until the systematic block-state error of the trailing window of
    `window` steps (its two halves give the noise, which is subtracted)
    against the reference falls to `threshold`, checked every `stride` steps
    once a whole window has run (None if not within max_steps); the error
    curves (one value per check) and the wall time."""
    import cudadsmc_b200 as cb
    stride = stride or window
    assert window % stride == 0 and (window // stride) % 2 == 0 or stride == window
    t0 = time.time()
    sols = [make_solver(c, s) for c, s in zip(conds, seeds)]
    for i, sol in enumerate(sols):
        if warm is not None:
            seed_from(sol, warm[i], conds[i], seeding)
        else:
            sol.InitSystemState()
    batch = cb.DSMCBatch(sols)
    done = [None] * len(sols)
    curves = [[] for _ in sols]
    segs = []  # per segment of `stride` steps: each member's (sums, samples)
    per = window // stride
    seg_len = [stride] if stride != window else [window // 2, window - window // 2]
    steps = 0
    while steps < max_steps and any(d is None for d in done):
        for w in seg_len:
            for sol in sols:
                sol.ResetSamples()
            batch.Step(w)
            batch.Sync()
            segs.append([sol.SampleStatistics()[::2] for sol in sols])
            steps += w
        need = per if stride != window else 2
        if len(segs) < need:
            continue
        last = segs[-need:]
        segs = last
        h = need // 2
        for i, c in enumerate(conds):
            s1 = sum(seg[i][0] for seg in last[:h])
            n1 = sum(seg[i][1] for seg in last[:h])
            s2 = sum(seg[i][0] for seg in last[h:])
            n2 = sum(seg[i][1] for seg in last[h:])
            b1 = block_state_from_sums(s1, n1, c)
            b2 = block_state_from_sums(s2, n2, c)
            mid = block_state_from_sums(s1 + s2, n1 + n2, c)
            e = field_error(mid, refs[i], noise2=half_noise(b1, b2) + ref_noise[i])
            curves[i].append(e)
            if done[i] is None and e <= threshold:
                done[i] = steps
    wall = time.time() - t0
    batch.close()
    for s in sols:
        s.close()
    return done, curves, wall


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--test", type=int, default=100)
    ap.add_argument("--settle", type=int, default=2500)
    ap.add_argument("--sample", type=int, default=1500)
    ap.add_argument("--ref-sample", type=int, default=3000)
    ap.add_argument("--window", type=int, default=200)
    ap.add_argument("--stride", type=int, default=None,
                    help="check the trailing window every STRIDE steps (default: the window)")
    ap.add_argument("--max-steps", type=int, default=4000)
    ap.add_argument("--threshold", type=float, default=0.02)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--batch", type=int, default=128)
    ap.add_argument("--group", type=int, default=64)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--ideal", action="store_true",
                    help="also seed runs from the converged reference fields")
    ap.add_argument("--seeding", choices=("two-stream", "maxwell"), default="two-stream",
                    help="fill of the warm runs: the two-stream mixture weighted by Kn, or a local "
                         "Maxwellian per cell (also run beside the two-stream fill for comparison)")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()

    import torch
    import cudadsmc_b200 as cb
    from cudadsmc_b200.surrogate import WarmStartMLP
    torch.cuda.set_device(0)
    log = lambda m: print(m, flush=True)  # noqa: E731
    train_c = sample_conditions(args.train, args.seed)
    test_c = sample_conditions(args.test, args.seed + 1)
    t0 = time.time()
    fields = generate(train_c, args.seed + 100000, args.settle, args.sample, args.group, log)
    t_gen = time.time() - t0
    x = normalize_inputs(train_c)
    rng = np.random.default_rng(args.seed)
    order = rng.permutation(len(x))
    x, fields = x[order], fields[order]
    F = CELLS * CHANNELS
    flat = fields.reshape(len(x), F)
    mean = np.nanmean(flat, axis=0)
    mean = np.where(np.isfinite(mean), mean, 0.0).astype(np.float32)
    targets = torch.empty((len(x), F), dtype=torch.bfloat16, device="cuda")
    for i in range(0, len(x), 64):
        chunk = torch.from_numpy(np.ascontiguousarray(flat[i:i + 64])).to("cuda")
        cb.lib().dsmc_to_bf16(chunk.data_ptr(), targets[i:i + 64].data_ptr(), chunk.numel(), None)
    torch.cuda.synchronize()
    net = WarmStartMLP(F, n_in=4, hidden=512, depth=4, modes=256, seed=args.seed)
    net.set_mean(mean)
    t1 = time.time()
    hist = net.train(x, targets, epochs=args.epochs, batch=args.batch, lr=1e-3, lr_final=1e-5, log=log)
    torch.cuda.synchronize()
    t_train = time.time() - t1
    # held-out conditions: converged references, then cold and warm runs
    seeds_ref = [args.seed + 200000 + i for i in range(args.test)]
    seeds_run = [args.seed + 300000 + i for i in range(args.test)]
    refs, ref_noise, empty, ref_cells = [], [], [], []
    for i in range(0, args.test, args.group):
        sl = slice(i, min(args.test, i + args.group))
        h1, h2 = run_group(test_c[sl], seeds_ref[sl], args.settle, args.ref_sample, halves=True)
        for c, (s1, n1), (s2, n2) in zip(test_c[sl], h1, h2):
            refs.append(block_state_from_sums(s1 + s2, n1 + n2, c))
            ref_noise.append(half_noise(block_state_from_sums(s1, n1, c), block_state_from_sums(s2, n2, c)))
            empty.append((s1[:, 0] + s2[:, 0]) <= 0)
            ref_cells.append(cell_fields_from_sums(s1 + s2, n1 + n2, c))
    ref_cells = np.stack(ref_cells)
    t2 = time.time()
    pred = net.predict(normalize_inputs(test_c)).cpu().numpy().reshape(args.test, CELLS, CHANNELS)
    torch.cuda.synchronize()
    t_pred = time.time() - t2
    pred_blocks = [block_state_from_fields(pred[i], test_c[i], empty[i]) for i in range(args.test)]
    pred_err = [field_error(pred_blocks[i], refs[i], noise2=ref_noise[i]) for i in range(args.test)]
    pred_err_raw = [field_error(pred_blocks[i], refs[i]) for i in range(args.test)]
    cold_steps, warm_steps, cold_wall, warm_wall = [], [], 0.0, 0.0
    cold_curves, warm_curves = [], []
    maxwell_steps = []  # warm runs from a local Maxwellian per cell, beside the two-stream fill
    for i in range(0, args.test, args.group):
        sl = slice(i, min(args.test, i + args.group))
        d, cc, w = convergence(test_c[sl], seeds_run[sl], refs[sl], ref_noise[sl], args.window,
                               args.max_steps, args.threshold, stride=args.stride)
        cold_steps += d
        cold_curves += cc
        cold_wall += w
        d, cc, w = convergence(test_c[sl], seeds_run[sl], refs[sl], ref_noise[sl], args.window,
                               args.max_steps, args.threshold, warm=pred[sl], stride=args.stride,
                               seeding=args.seeding)
        warm_steps += d
        warm_curves += cc
        warm_wall += w
        if args.seeding != "maxwell":
            d, _, _ = convergence(test_c[sl], seeds_run[sl], refs[sl], ref_noise[sl], args.window,
                                  args.max_steps, args.threshold, warm=pred[sl], stride=args.stride)
            maxwell_steps += d
    # the seeding itself: runs seeded with the converged reference fields
    ideal_steps, ideal_curves = [], []
    if args.ideal:
        for i in range(0, args.test, args.group):
            sl = slice(i, min(args.test, i + args.group))
            d, cc, _ = convergence(test_c[sl], seeds_run[sl], refs[sl], ref_noise[sl], args.window,
                                   args.max_steps, args.threshold, warm=ref_cells[sl], stride=args.stride,
                                   seeding=args.seeding)
            ideal_steps += d
            ideal_curves += cc
    cs = np.array([s if s is not None else np.nan for s in cold_steps], np.float64)
    ws = np.array([s if s is not None else np.nan for s in warm_steps], np.float64)
    both = np.isfinite(cs) & np.isfinite(ws)
    # what is left at the end of the cold runs (systematic error once steady)
    floor = [c[-1] for c in cold_curves]
    res = {
        "train_conditions": args.train, "test_conditions": args.test,
        "settle_steps": args.settle, "sample_steps": args.sample, "ref_sample_steps": args.ref_sample,
        "window": args.window, "stride": args.stride or args.window, "threshold": args.threshold,
        "error_blocks": f"{BLOCK}^3 cells",
        "generation_s": t_gen, "training_s": t_train, "prediction_s": t_pred,
        "loss_first_epoch": hist[0], "loss_last_epoch": hist[-1],
        "error_definition": "relative L2 over blocks of 4^3 cells of (n/n_inf, u/U, v/U, w/U, T/T_inf) "
                            "from moments pooled per block; statistical noise (from half-window "
                            "differences) subtracted",
        "prediction_error_raw_median": float(np.median(pred_err_raw)),
        "prediction_error": {"median": float(np.median(pred_err)), "mean": float(np.mean(pred_err)),
                             "max": float(np.max(pred_err)),
                             "share_below_threshold": float(np.mean(np.array(pred_err) <= args.threshold))},
        "cold_steps": {"median": float(np.nanmedian(cs)), "mean": float(np.nanmean(cs)),
                       "not_converged": int(np.sum(~np.isfinite(cs)))},
        "warm_steps": {"median": float(np.nanmedian(ws)), "mean": float(np.nanmean(ws)),
                       "not_converged": int(np.sum(~np.isfinite(ws)))},
        "steps_speedup": {"median_ratio": float(np.median(cs[both] / ws[both])) if both.any() else None,
                          "ratio_of_means": float(np.mean(cs[both]) / np.mean(ws[both])) if both.any() else None},
        "seeding": args.seeding,
        "maxwell_warm_steps": {
            "median": float(np.nanmedian([np.nan if d is None else d for d in maxwell_steps])),
            "median_ratio": float(np.median([c / m for c, m in zip(cold_steps, maxwell_steps)
                                             if c is not None and m is not None]))}
        if maxwell_steps else None,
        "wall_s": {"cold": cold_wall, "warm": warm_wall},
        "cold_error_at_end": {"median": float(np.median(floor))},
        "seeded_from_reference": {
            "steps_median": float(np.nanmedian([np.nan if d is None else d for d in ideal_steps]))
            if ideal_steps else None,
            "curve_median": [float(np.median([c[k] for c in ideal_curves if len(c) > k]))
                             for k in range(max(len(c) for c in ideal_curves))] if ideal_curves else None},
        "cold_curve_median": [float(np.median([c[k] for c in cold_curves if len(c) > k]))
                              for k in range(max(len(c) for c in cold_curves))],
        "warm_curve_median": [float(np.median([c[k] for c in warm_curves if len(c) > k]))
                              for k in range(max(len(c) for c in warm_curves))],
        "conditions": [{"mach": float(c[0]), "kn": float(c[1]), "tw_ratio": float(c[2]), "r": float(c[3]),
                        "pred_err": float(pe), "cold": cold_steps[i], "warm": warm_steps[i],
                        "warm_maxwell": maxwell_steps[i] if maxwell_steps else None}
                       for i, (c, pe) in enumerate(zip(test_c, pred_err))],
    }
    js = json.dumps(res)
    print(js, flush=True)
    if args.out:
        with open(args.out, "w") as f:
            f.write(js)


if __name__ == "__main__":
    main()
