"""A small reference-compatible flow with gradients, for full-run field
comparisons: argon hard spheres streaming along x at 600 m/s through a box
that is periodic in x (the reference's PeriodicXBoundaryCondition), past an
icosphere reflected specularly with the reference's first-hit test.  The
body leaves a compressed layer in front and a wake behind it, so the sampled
fields carry gradients that the collisions shape.

run_oracle() runs it with the oracle's restatement of the reference step
(cell ids, stable sort, reorder, HybridTaus NTC, move with the body,
sampling after the move per pre-move cell)."""
import math

import numpy as np

from oracle import oracle as O

MASS, DIAM, TREF = 6.63e-26, 4.17e-10, 273.0
GMIN, GMAX, DIM = (0.0, 0.0, 0.0), (0.6, 0.3, 0.3), (24, 12, 12)
CENTER, RADIUS, LEVEL, GEOM_DIM = (0.3, 0.15, 0.15), 0.06, 2, (8, 8, 8)
DENSITY, TEMP, U, PPC = 1e20, 300.0, 600.0, 16
DT = 5e-6


def icosphere(level, radius, center):
    """Icosphere from the regular icosahedron, edges split at their
    normalised midpoints `level` times (outward triangles)."""
    t = (1.0 + 5 ** 0.5) / 2
    v = [np.array(p, float) / np.linalg.norm(p) for p in
         [[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t],
          [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]]]
    f = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
         [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
         [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]]
    for _ in range(level):
        mid = {}

        def m(a, b):
            k = (min(a, b), max(a, b))
            if k not in mid:
                p = v[a] + v[b]
                v.append(p / np.linalg.norm(p))
                mid[k] = len(v) - 1
            return mid[k]
        g = []
        for a, b, c in f:
            ab, bc, ca = m(a, b), m(b, c), m(c, a)
            g += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        f = g
    verts = (np.asarray(center) + radius * np.asarray(v)).astype(np.float32)
    return verts, np.asarray(f, np.uint32)


def fnum():
    cell_v = np.prod((np.asarray(GMAX) - np.asarray(GMIN)) / np.asarray(DIM))
    return float(DENSITY * cell_v / (PPC + 0.5))


def initial_state(seed, temp_scale=1.0):
    """Particles uniform in the box outside the body, drifting Maxwellian;
    HybridTaus seeds and (sigma g)max / remainders per cell.  Returns
    (sim, geom, pos4, vel4, maxrem, seeds, ppc)."""
    from helpers import maxrem_init, taus_seeds
    sim = O.sim_from(GMIN, GMAX, DIM, fnum(), O.cross_section_of(DIAM), "x")
    ppc = int(np.float32(DENSITY) * np.float32(sim.cell_volume) / np.float32(fnum()))
    n = ppc * sim.cells
    rng = np.random.default_rng(seed)
    pts = np.zeros((0, 3))
    while len(pts) < n:
        p = rng.uniform(np.asarray(GMIN) + 1e-4, np.asarray(GMAX) - 1e-4, (n, 3))
        p = p[np.linalg.norm(p - np.asarray(CENTER), axis=1) > RADIUS * 1.02]
        pts = np.concatenate([pts, p])[:n]
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 4), np.float32)
    pos[:, :3] = pts
    pos[:, 3] = 1.0
    vstd = math.sqrt(1.3806e-23 * TEMP * temp_scale / MASS)
    vel[:, :3] = rng.normal(0.0, vstd, (n, 3)) + np.array([U, 0.0, 0.0])
    verts, tris = icosphere(LEVEL, RADIUS, CENTER)
    nrm = np.cross(verts[tris[:, 1]] - verts[tris[:, 0]], verts[tris[:, 2]] - verts[tris[:, 0]])
    nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
    bbox, cell, count, ids, flags = O.build_grid(verts, tris, GEOM_DIM)
    geom = O.geom_from(bbox, cell, GEOM_DIM, count, ids, flags, verts, tris, nrm)
    seeds = taus_seeds(seed + 1, sim.cells)
    mr = maxrem_init(seed + 2, sim.cells, O.max_rel_vel_of(DIAM, TEMP))
    return sim, geom, pos, vel, mr, seeds, ppc


def run_oracle(seed, settle, steps, temp_scale=1.0, pair_scale=1.0):
    """(cells, 5) FP64 sampling sums of one oracle run: `settle` steps, then
    `steps` sampled steps.  temp_scale and pair_scale plant mistakes for the
    tests of the comparison (initial temperature, number of NTC pairs)."""
    sim, geom, pos, vel, mr, seeds, ppc = initial_state(seed, temp_scale)
    st4 = np.zeros((sim.cells, 4), np.float32)
    conc = float(ppc) * pair_scale
    for _ in range(settle):
        pos, vel, cse = O.step(sim, geom, pos, vel, DT, conc, mr, st4, seeds)
    sums = np.zeros((sim.cells, 5), np.float64)
    for _ in range(steps):
        pos, vel, cse = O.step(sim, geom, pos, vel, DT, conc, mr, st4, seeds)
        sums += O.sample_f64(sim, vel, cse)
    return sums


def oracle_replicas(seed0, replicas, settle, steps, **kw):
    """(replicas, cells, 5): independent runs (initial state and random
    streams from seed0 + 10 k)."""
    return np.stack([run_oracle(seed0 + 10 * k, settle, steps, **kw) for k in range(replicas)])


# --------------------------------------------------------------------------
# The same body in the extension mode the capsule workload runs: argon VHS
# (omega 0.81) streaming at Mach 5.8 from an inflow face at x = 0 (outflow on
# the other faces), Philox streams, nearest wall crossings and a diffuse wall
# at 300 K.  run_oracle_fast() runs it with the oracle's restatement of that
# mode (oracle/fast_oracle.c, composed by oracle.step_fast).

FAST = dict(omega=0.81, temp=200.0, u=1500.0, wall_temp=300.0, ppc=10, dt=4e-6,
            center=(0.2, 0.15, 0.15), level=2)
FACES = {"-x": "inflow", "+x": "outflow", "-y": "outflow", "+y": "outflow", "-z": "outflow",
         "+z": "outflow"}
FACE_KINDS = [4, 2, 2, 2, 2, 2]
KB = 1.3806e-23


def fast_fnum():
    cell_v = np.prod((np.asarray(GMAX) - np.asarray(GMIN)) / np.asarray(DIM))
    return float(DENSITY * cell_v / FAST["ppc"])


def vhs_gref(omega):
    g0 = math.sqrt(2.0 * 1.380649e-23 * TREF / (0.5 * MASS))
    return float(np.float32(g0 * math.gamma(2.5 - omega) ** (-1.0 / (2.0 * omega - 1.0))))


def fast_settings():
    """The extension-mode flow as library settings."""
    from cudadsmc_b200 import settings_t
    return settings_t().set(grid_min=GMIN, grid_max=GMAX, grid_dim=DIM, density=DENSITY,
                            fnum=fast_fnum(), temp=FAST["temp"], stream_vel=(FAST["u"], 0.0, 0.0),
                            dt=FAST["dt"], rng="philox", ntc_local=1, sample_every=1,
                            init_kind="maxwell", wall_diffuse=1, wall_temp=FAST["wall_temp"],
                            capacity_factor=2.5, geom_nearest=1, face_kind=FACES, gas_mass=MASS,
                            gas_diam=DIAM, gas_tref=TREF, gas_omega=FAST["omega"])


def fast_initial_state(seed):
    """Free stream outside the body: (6, n) SoA state and per-cell
    ((sigma g)max, remainder)."""
    sim = O.sim_from(GMIN, GMAX, DIM, fast_fnum(), O.cross_section_of(DIAM))
    rng = np.random.default_rng(seed)
    vol = np.prod(np.asarray(GMAX) - np.asarray(GMIN)) - 4.0 / 3.0 * math.pi * RADIUS ** 3
    n = int(round(DENSITY * vol / fast_fnum()))
    pts = np.zeros((0, 3))
    while len(pts) < n:
        p = rng.uniform(np.asarray(GMIN) + 1e-4, np.asarray(GMAX) - 1e-4, (n, 3))
        p = p[np.linalg.norm(p - np.asarray(FAST["center"]), axis=1) > RADIUS * 1.02]
        pts = np.concatenate([pts, p])[:n]
    vstd = math.sqrt(KB * FAST["temp"] / MASS)
    vel = rng.normal(0.0, vstd, (n, 3)) + np.array([FAST["u"], 0.0, 0.0])
    st6 = np.ascontiguousarray(np.concatenate([pts.T, vel.T]).astype(np.float32))
    k, c1 = O.vhs_fast_coeffs(O.cross_section_of(DIAM), FAST["omega"], vhs_gref(FAST["omega"]))
    mr = np.zeros((sim.cells, 2), np.float32)
    mr[:, 0] = np.float32(k * 4000.0 ** c1)
    mr[:, 1] = rng.uniform(0, 1, sim.cells).astype(np.float32)
    return sim, st6, mr


def fast_mesh():
    return icosphere(FAST["level"], RADIUS, FAST["center"])


def run_oracle_fast(seed, settle, steps, run_seed, wall_temp=None, pair_scale=1.0):
    """(cells, 5) FP64 sampling sums of one oracle run of the extension-mode
    flow (the library's sampling: after the move, per pre-move cell).
    wall_temp and pair_scale plant mistakes for the tests of the comparison
    (the body's wall temperature, the number of NTC pairs)."""
    sim, st, mr = fast_initial_state(seed)
    c = fast_settings().cfg
    verts, tris = fast_mesh()
    tri9 = O.triangles_of(verts, tris)
    gref = vhs_gref(FAST["omega"])
    inflows = O.library_inflows(c)
    tw = FAST["wall_temp"] if wall_temp is None else wall_temp
    wall_vstd = float(np.sqrt(np.float32(np.float32(np.float32(KB) * np.float32(tw)) /
                                         np.float32(MASS)), dtype=np.float32))
    keys = O.keys_of(sim, st, np.all((st[:3] >= np.array(GMIN, np.float32)[:, None]) &
                                      (st[:3] <= np.array(GMAX, np.float32)[:, None]), axis=0))
    rem = {}
    sums = np.zeros((sim.cells, 5), np.float64)
    for s in range(1, settle + steps + 1):
        f = O.fast_params(run_seed, s, c.fnum, c.dt, sim.cell_volume, sim.cross_section,
                          FAST["omega"], gref, ntc_local=1, warp_cap=128)
        f.ntc_coef = float(np.float32(f.ntc_coef * pair_scale))
        m = O.fast_move_params(sim, FACE_KINDS, [0.0] * 6, c.dt, run_seed, s, tri9,
                               wall_diffuse=1, wall_vstd=wall_vstd)
        r = O.step_fast(f, m, sim, st, keys, mr, inflows, rem)
        if s > settle:
            n_alive, start = r["n_alive"], r["start"]
            vel = r["state"][3:, :n_alive].astype(np.float64)
            cnt = np.diff(start.astype(np.int64))
            cell_of = np.repeat(np.arange(sim.cells), cnt)
            sums[:, 0] += cnt
            for q in range(3):
                sums[:, 1 + q] += np.bincount(cell_of, vel[q], minlength=sim.cells)
            sums[:, 4] += np.bincount(cell_of, (vel ** 2).sum(0), minlength=sim.cells)
        st, keys, mr, rem = r["state"], r["keys"], r["maxrem"], r["inj_rem"]
    return sums


def oracle_replicas_fast(seed0, replicas, settle, steps, **kw):
    """(replicas, cells, 5): independent runs (initial state from seed0 + 10 k,
    random streams from the run seed seed0 + 7000 + k)."""
    return np.stack([run_oracle_fast(seed0 + 10 * k, settle, steps, seed0 + 7000 + k, **kw)
                     for k in range(replicas)])
