"""The extension-mode restatement (oracle/fast_oracle.c) on its own, on the
CPU.  It has no counterpart in the reference, so it is pinned by physics:
conservation in every collision, the NTC pair count, equal collision rates on
the lane and warp paths, the diffuse wall's re-emission distribution, the
inflow's number flux and its flux-weighted normal speed, and nearest-hit
flights that never end inside a closed body."""
import math

import numpy as np
import pytest

from oracle import oracle as O

KB = 1.3806e-23
M_AR, D_AR = 6.63e-26, 4.17e-10


def cells(seed, ncells, mean, dense=0):
    rng = np.random.default_rng(seed)
    counts = rng.poisson(mean, ncells).astype(np.int64)
    if dense:
        counts[rng.choice(ncells, dense, replace=False)] = rng.integers(60, 300, dense)
    start = np.zeros(ncells + 1, np.uint32)
    start[1:] = np.cumsum(counts)
    vel = rng.normal(0.0, 300.0, (3, int(start[-1]))).astype(np.float32)
    return counts, start, vel


def params(heavy_min=8, omega=0.5, step=3, warp_cap=256):
    cs = O.cross_section_of(D_AR)
    gref = 0.0
    if omega != 0.5:
        g0 = math.sqrt(2.0 * 1.380649e-23 * 273.0 / (0.5 * M_AR))
        gref = float(np.float32(g0 * math.gamma(2.5 - omega) ** (-1.0 / (2.0 * omega - 1.0))))
    return O.fast_params(77, step, 1e15, 2e-5, 1.0 / 4096, cs, omega, gref, ntc_local=1,
                         heavy_min=heavy_min, warp_cap=warp_cap), cs, gref


@pytest.mark.parametrize("omega", [0.5, 0.81])
def test_collisions_conserve_and_count_pairs(omega):
    counts, start, vel = cells(1, 2048, 9, dense=30)
    f, cs, gref = params(omega=omega)
    mr = np.zeros((2048, 2), np.float32)
    vmax = cs * 2000.0 if omega == 0.5 else f.vhs_k * 2000.0 ** f.vhs_c1
    mr[:, 0] = np.float32(vmax)
    mr[:, 1] = np.float32(0.25)
    v = vel.copy()
    mr1 = mr.copy()
    info, sg = O.collide_fast(f, v[0], v[1], v[2], start, mr1)
    # the pair count: floor(coef n (n - 1) vmax + rem) in FP32 with one fused step
    n = counts.astype(np.float32)
    fpc = (np.float32(f.ntc_coef) * n * (n - 1)).astype(np.float32).astype(np.float64) * \
        np.float64(np.float32(vmax)) + 0.25
    expect = np.where(counts >= 2, np.floor(fpc), 0)
    assert np.max(np.abs(info[:, 0] - expect)) <= 1
    assert info[:, 1].sum() > 1000 and sg > 0
    assert set(np.unique(info[:, 2]).tolist()) >= {1, 2}
    nz = counts > 0
    p0 = np.add.reduceat(vel.astype(np.float64), start[:-1][nz], axis=1)
    p1 = np.add.reduceat(v.astype(np.float64), start[:-1][nz], axis=1)
    assert np.max(np.abs(p1 - p0)) < 1e-6 * 300 * counts.max()
    e0 = np.add.reduceat((vel.astype(np.float64) ** 2).sum(0), start[:-1][nz])
    e1 = np.add.reduceat((v.astype(np.float64) ** 2).sum(0), start[:-1][nz])
    assert np.max(np.abs(e1 - e0) / e0) < 1e-5
    assert np.all(mr1[:, 0] >= mr[:, 0])


def test_warp_and_lane_paths_collide_at_the_same_rate():
    counts, start, vel = cells(2, 512, 0, dense=512)
    rates = []
    for heavy_min in (8, 1 << 30):
        f, cs, _ = params(heavy_min=heavy_min, warp_cap=512)
        mr = np.zeros((512, 2), np.float32)
        mr[:, 0] = np.float32(cs * 2000.0)
        v = vel.copy()
        info, _ = O.collide_fast(f, v[0], v[1], v[2], start, mr)
        assert np.all(info[counts >= 2, 2] == (2 if heavy_min == 8 else 1))
        rates.append(info[:, 1].sum() / info[:, 0].sum())
    assert abs(rates[0] - rates[1]) < 0.01 * rates[1], rates


def sphere(level=3):
    """An icosphere built here (subdivided and projected)."""
    t = (1 + 5 ** 0.5) / 2
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
         (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
         (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, float) / np.linalg.norm(p) for p in v]
    for _ in range(level):
        mid = {}
        nf = []

        def m(a, b):
            k = (min(a, b), max(a, b))
            if k not in mid:
                q = verts[a] + verts[b]
                verts.append(q / np.linalg.norm(q))
                mid[k] = len(verts) - 1
            return mid[k]
        for a, b, c in f:
            ab, bc, ca = m(a, b), m(b, c), m(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    return np.array(verts), np.array(f)


def test_nearest_hit_flights_stay_outside_and_reemit_at_wall_temperature():
    v, t = sphere(3)
    center, r = np.array([0.3, 0.3, 0.3]), 0.1
    verts = (v * r + center).astype(np.float32)
    tri9 = O.triangles_of(verts, t)
    sim = O.sim_from((0, 0, 0), (0.6, 0.6, 0.6), (16, 16, 16), 1e15, O.cross_section_of(D_AR))
    vw = float(np.float32(math.sqrt(KB * 300.0 / M_AR)))
    m = O.fast_move_params(sim, [0] * 6, [0.0] * 6, 4e-5, 9, 1, tri9, wall_diffuse=1, wall_vstd=vw)
    rng = np.random.default_rng(5)
    n = 40000
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pos = center + d * rng.uniform(0.1005, 0.13, n)[:, None]
    vel = -d * rng.uniform(500, 2000, n)[:, None]
    st = np.ascontiguousarray(np.concatenate([pos.T, vel.T]).astype(np.float32))
    live, amb = O.move_fast(m, st)
    assert live.all() and amb.mean() < 1e-3
    rr = np.linalg.norm(st[:3].T - center, axis=1)
    # the level-3 icosphere's inscribed radius is above 0.0995 r/0.1
    assert np.mean(rr < 0.0995) == 0.0
    hit = np.any(st[3:] != vel.T.astype(np.float32), axis=0)
    assert hit.mean() > 0.5
    # re-emitted about the outward normal: normal speed Rayleigh(vw), mean
    # vw sqrt(pi/2); tangential components N(0, vw^2)
    # the paths are radial, so the wall normal at the hit is about d
    nrm = d[hit]
    vn = np.sum(st[3:, hit].T * nrm, axis=1)
    assert np.mean(vn > 0) > 0.99  # facets tilt a few degrees off the radial d
    assert abs(vn.mean() / (vw * math.sqrt(math.pi / 2)) - 1) < 0.03
    vt2 = np.sum(st[3:, hit].T ** 2, axis=1) - vn ** 2
    assert abs(np.mean(vt2) / (2 * vw ** 2) - 1) < 0.05


def test_closed_specular_box_keeps_energy():
    sim = O.sim_from((0, 0, 0), (1, 1, 1), (8, 8, 8), 1e15, O.cross_section_of(D_AR))
    m = O.fast_move_params(sim, [0, 0, 0, 0, 3, 3], [0.0] * 6, 1e-3, 3, 2)
    rng = np.random.default_rng(6)
    st = np.ascontiguousarray(np.concatenate([rng.uniform(0, 1, (3, 20000)),
                                              rng.normal(0, 300, (3, 20000))]).astype(np.float32))
    e0 = np.sum(st[3:].astype(np.float64) ** 2)
    live, _ = O.move_fast(m, st)
    assert live.all()
    assert np.all((st[:3] >= 0) & (st[:3] <= 1))
    assert abs(np.sum(st[3:].astype(np.float64) ** 2) / e0 - 1) < 1e-6


def test_inflow_flux_and_normal_speed():
    sim = O.sim_from((0, 0, 0), (1.0, 0.5, 0.5), (16, 8, 8), 1e15, O.cross_section_of(D_AR))
    vstd = math.sqrt(KB * 200.0 / M_AR)
    U = 600.0
    cmp = math.sqrt(2) * vstd
    s = U / cmp
    flux = 1e20 * cmp / (2 * math.sqrt(math.pi)) * (math.exp(-s * s) + math.sqrt(math.pi) * s *
                                                    (1 + math.erf(s))) / 1e15
    inflow = O.inflow_of(0, flux, 0.25, (U, 0.0, 0.0), vstd)
    dt = 1e-5
    rem, ks = O.inject_plan_chain(inflow, dt, 50)
    assert abs(sum(ks) - flux * 0.25 * dt * 50) <= 1.0
    dt2 = 1e-3  # one long step: a large sample of injected particles
    st, amb, _ = O.inject_fast(inflow, sim, dt2, 11, 4, 0.0, 1 << 22)
    k = st.shape[1]
    assert k == int(np.float32(np.float32(flux) * np.float32(0.25)) * np.float32(dt2))
    assert k > 10000
    assert np.all(st[3] > 0)
    # flux-weighted normal speed of a drifting Maxwellian: mean
    # <u^2>/<u> over the inward half-range
    z = np.linspace(0, 10, 200001)
    f = z * np.exp(-(z - s) ** 2)
    mean_ref = np.trapezoid(z * f, z) / np.trapezoid(f, z) * cmp
    assert abs(st[3].mean() / mean_ref - 1) < 0.02
    assert abs(np.std(st[4]) / vstd - 1) < 0.03 and abs(np.mean(st[4])) < 0.05 * vstd
    assert np.all((st[0] >= 0) & (st[0] <= (U + 10 * vstd) * dt2))
