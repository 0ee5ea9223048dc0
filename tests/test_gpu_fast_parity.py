"""Parity of the mode the capsule workload runs (Philox streams, VHS
omega = 0.81, warp-collided dense cells, nearest wall crossings with diffuse
re-emission, per-face boundaries, inflow injection) with its CPU
restatement, oracle/fast_oracle.c, on identical inputs and random streams.

The device code of this mode writes every rounding step explicitly; the
restatement evaluates the same steps.  What may differ, and why:
  - sigma(g) g uses the hardware base-2 log and exponential (relative error
    about 1e-6): an acceptance test within 4e-6 of its threshold may go
    either way.  The oracle reports such near ties per cell; those cells
    (expected: none or a handful) are excluded by that stated cause;
  - sincospif / logf / sincosf differ from libm by an ulp or two: velocities
    agree within 1e-6 of their scale per collision or wall re-emission (a
    particle of a dense cell that collides k times in a pass: k x 1e-6),
    positions within 1e-6 of the box size;
  - a wall crossing within 1e-5 of another crossing, of a triangle edge or of
    an end of the path, and a position within 1e-5 of a cell face, may be
    resolved either way: the oracle flags those particles.
Integer results are exact: pair counts, collisions per cell, remainders,
cell keys, removals, the injected count and the order of the particles.
"""
import math

import numpy as np
import pytest
import torch

from cudadsmc_b200 import DSMCSolver, settings_t, stages, mesh_icosphere
from oracle import oracle as O

from helpers import sim_for

pytestmark = pytest.mark.gpu

KB = 1.3806e-23
M_AR, D_AR, TREF, OMEGA = 6.63e-26, 4.17e-10, 273.0, 0.81
SEED = 0x5EEDC0FFEE


def T(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def U32(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32)).to(dev)


def vhs_gref(omega=OMEGA, m=M_AR, tref=TREF):
    """The reference speed of sigma = sigma_ref (g_ref/g)^(2 omega - 1), as the
    library derives it."""
    if abs(omega - 0.5) < 1e-9:
        return 0.0
    g0 = math.sqrt(2.0 * 1.380649e-23 * tref / (0.5 * m))
    return float(np.float32(g0 * math.gamma(2.5 - omega) ** (-1.0 / (2.0 * omega - 1.0))))


def f32sqrt_ratio(a, b):
    """sqrtf(a / b) in FP32 (the library's thermal-speed arithmetic)."""
    return float(np.sqrt(np.float32(np.float32(a) / np.float32(b)), dtype=np.float32))


def vstd_of(temp, m=M_AR):
    return f32sqrt_ratio(np.float32(np.float32(KB) * np.float32(temp)), m)


def cells_case(seed, ncells, giant=0):
    """Per-cell counts: mostly light cells (mean 8), a few dense ones (60-400
    particles, collided by a warp) and optionally one cell above 2048."""
    rng = np.random.default_rng(seed)
    counts = rng.poisson(8, ncells).astype(np.int64)
    dense = rng.choice(ncells, ncells // 64, replace=False)
    counts[dense] = rng.integers(60, 400, len(dense))
    counts[rng.choice(ncells, 40, replace=False)] = rng.integers(0, 2, 40)
    if giant:
        counts[ncells // 2] = giant
    start = np.zeros(ncells + 1, np.uint32)
    start[1:] = np.cumsum(counts)
    n = int(start[-1])
    vel = rng.normal(0.0, 350.0, (3, n)).astype(np.float32)
    vel[0] += np.float32(900.0)
    return counts, start, vel


@pytest.mark.parametrize("omega", [0.5, OMEGA])
def test_collide_philox_matches_oracle(cuda, omega):
    ncells = 4096
    counts, start, vel = cells_case(3, ncells, giant=2100)
    cs = O.cross_section_of(D_AR)
    gref = vhs_gref(omega)
    fnum, cell_volume = 1e15, float(np.float32(1.0 / 4096))
    # (sigma g)max from a relative speed of 2500 m/s; dt so that a light cell
    # selects a couple of pairs per pass
    if abs(omega - 0.5) < 1e-9:
        vmax = np.float32(cs * 2500.0)
    else:
        k, c1 = O.vhs_fast_coeffs(cs, omega, gref)
        vmax = np.float32(k * 2500.0 ** c1)
    dt = float(np.float32(0.05 / (0.5 * fnum / cell_volume * float(vmax))))
    rng = np.random.default_rng(4)
    mr = np.zeros((ncells, 2), np.float32)
    mr[:, 0] = vmax
    mr[:, 1] = rng.uniform(0, 1, ncells).astype(np.float32)
    step = 77
    f = O.fast_params(SEED, step, fnum, dt, cell_volume, cs, omega, gref, ntc_local=1,
                      warp_cap=2048)
    vo = vel.copy()
    mr_o = mr.copy()
    info, _ = O.collide_fast(f, vo[0], vo[1], vo[2], start, mr_o)
    u, v, w = (T(vel[k].copy(), cuda) for k in range(3))
    mr_t = T(mr.copy(), cuda)
    st_t = torch.zeros(ncells * 4, dtype=torch.float32, device=cuda)
    p = stages.collide_params(ncells, cell_volume, cs, fnum, 0.0, dt, omega=omega, vhs_gref=gref,
                              ntc_local=1, rng="philox", seed=SEED, step=step)
    stages.collide(p, u, v, w, U32(start, cuda), mr_t, stat4=st_t)
    torch.cuda.synchronize()
    vg = np.stack([t.cpu().numpy() for t in (u, v, w)])
    st = st_t.cpu().numpy().reshape(-1, 4)
    mr_g = mr_t.cpu().numpy()

    paths = np.bincount(info[:, 2], minlength=4)
    assert paths[2] >= 40 and paths[3] == 1 and paths[1] > 3000, paths
    tie = info[:, 3] > 0
    print(f"omega={omega}: cells by path {paths.tolist()}, near ties {int(tie.sum())}, "
          f"pairs {int(info[:, 0].sum())}, collisions {int(info[:, 1].sum())}")
    assert tie.sum() <= max(2, ncells // 1000)
    # pair counts and remainders of every cell: exact
    assert np.array_equal(st[:, 0].astype(np.int64), info[:, 0].astype(np.int64))
    assert np.array_equal(mr_g[:, 1], mr_o[:, 1])
    ok = ~tie
    assert np.array_equal(st[ok, 1].astype(np.int64), info[ok, 1].astype(np.int64))
    # (sigma g)max: the largest sigma g of the pass, from velocities that
    # earlier collisions of the cell left an ulp apart
    assert np.allclose(mr_g[ok, 0], mr_o[ok, 0], rtol=4e-6, atol=0)
    slot_ok = np.repeat(ok, counts)
    # relative to the velocity scale of the particle's cell (the rms speed
    # there before the pass: a collision rounds on that scale, whatever the
    # speed it leaves a particle with)
    sp2 = (vel.astype(np.float64) ** 2).sum(0)
    nz0 = counts > 0
    rms = np.zeros(ncells)
    rms[nz0] = np.sqrt(np.add.reduceat(sp2, start[:-1][nz0]) / counts[nz0])
    scale = np.maximum(np.linalg.norm(vo.astype(np.float64), axis=0), np.repeat(rms, counts))
    err = np.max(np.abs(vg - vo), axis=0) / np.maximum(scale, 1.0)
    # the FP32 bound is per collision: a particle of a dense cell takes part
    # in many collisions of one pass (each rounds sincospi's last bit apart),
    # so the bound scales with the collisions per particle of its cell
    per_particle = np.maximum(1.0, 2.0 * info[:, 1] / np.maximum(counts, 1))
    bound = 1e-6 * np.repeat(per_particle, counts)
    light = np.repeat(per_particle <= 1.0, counts)
    print(f"velocity error / speed: light cells {err[slot_ok & light].max():.2e}, "
          f"all {err[slot_ok].max():.2e} (bound up to {bound.max():.1e})")
    assert err[slot_ok & light].max() <= 1e-6
    assert np.all(err[slot_ok] <= bound[slot_ok])
    changed = np.any(vg != vel, axis=0)
    assert changed.mean() > 0.3
    # momentum and energy of every cell conserved to FP32 rounding
    nz = counts > 0
    p0 = np.add.reduceat(vel.astype(np.float64), start[:-1][nz], axis=1)
    p1 = np.add.reduceat(vg.astype(np.float64), start[:-1][nz], axis=1)
    e0 = np.add.reduceat((vel.astype(np.float64) ** 2).sum(0), start[:-1][nz])
    e1 = np.add.reduceat((vg.astype(np.float64) ** 2).sum(0), start[:-1][nz])
    nc = counts[nz]
    assert np.max(np.abs(p1 - p0) / (nc * 1500.0)) < 1e-6
    assert np.max(np.abs(e1 - e0) / e0) < 1e-5


def test_philox_stream_matches_oracle(cuda):
    """The device's Philox-4x32-10 words (through the stage collide's first
    pair draws of a 2-particle cell from its pair stream: pi = umulhi(r0, 2),
    pj = 1 - pi) and the oracle's known-answer generator give the same pair
    choices."""
    ncells = 1024
    counts = np.full(ncells, 2, np.int64)
    start = np.zeros(ncells + 1, np.uint32)
    start[1:] = np.cumsum(counts)
    n = int(start[-1])
    rng = np.random.default_rng(9)
    # particle 0 at rest, particle 1 fast: a collision (always accepted with
    # (sigma g)max below sigma g) swaps momentum in a way that shows which
    # slot was drawn first
    vel = np.zeros((3, n), np.float32)
    vel[0, 1::2] = 1000.0
    cs = O.cross_section_of(D_AR)
    mr = np.zeros((ncells, 2), np.float32)
    mr[:, 0] = np.float32(cs * 10.0)
    mr[:, 1] = np.float32(0.5)
    fnum, cell_volume = 1e15, float(np.float32(1.0 / 4096))
    dt = float(np.float32(0.6 / (0.5 * fnum / cell_volume * 2 * float(mr[0, 0]))))
    f = O.fast_params(SEED, 5, fnum, dt, cell_volume, cs, 0.5, 0.0, ntc_local=1, warp_cap=2048)
    vo, mr_o = vel.copy(), mr.copy()
    info, _ = O.collide_fast(f, vo[0], vo[1], vo[2], start, mr_o)
    u, v, w = (T(vel[k].copy(), cuda) for k in range(3))
    mr_t = T(mr.copy(), cuda)
    p = stages.collide_params(ncells, cell_volume, cs, fnum, 0.0, dt, ntc_local=1, rng="philox",
                              seed=SEED, step=5)
    stages.collide(p, u, v, w, U32(start, cuda), mr_t)
    torch.cuda.synchronize()
    vg = np.stack([t.cpu().numpy() for t in (u, v, w)])
    assert info[:, 0].min() == 1 and info[:, 1].min() == 1
    # the first word of each cell's pair stream decides the slot order: check
    # it against the known-answer Philox of the oracle directly
    first = np.array([O.philox([0, c, 5, 0x70616972], O.seed_words(SEED))[0] for c in range(ncells)],
                     np.uint64)
    pi = (first * 2) >> 32
    assert set(np.unique(pi).tolist()) == {0, 1}
    # slot order and scattering angles from the same words: velocities agree
    # to the last bits of sincospi
    assert np.max(np.abs(vg - vo)) <= 1e-6 * 1000.0


@pytest.mark.parametrize("count", [2, 3])
def test_light_cell_pairs_sharing_particles(cuda, count):
    """Light cells of 2 or 3 particles with 5 pairs each and a low
    (sigma g)max, so that most pairs collide: consecutive pairs share
    particles, and the next pair's velocities (loaded while the current pair
    is decided) must be replaced by the current pair's results.  Velocities
    match the oracle's sequential selections (cells with a near-tie
    acceptance excluded, as everywhere)."""
    ncells = 2048
    counts = np.full(ncells, count, np.int64)
    start = np.zeros(ncells + 1, np.uint32)
    start[1:] = np.cumsum(counts)
    n = int(start[-1])
    rng = np.random.default_rng(21 + count)
    vel = rng.normal(0.0, 500.0, (3, n)).astype(np.float32)
    cs = O.cross_section_of(D_AR)
    mr = np.zeros((ncells, 2), np.float32)
    mr[:, 0] = np.float32(cs * 1.0)  # below every sigma g: the first pair is accepted
    mr[:, 1] = np.float32(0.5)
    fnum, cell_volume = 1e15, float(np.float32(1.0 / 4096))
    # 5.2 + remainder 0.5 selections per cell: M = 5 (a light cell)
    dt = float(np.float32(5.2 / (0.5 * fnum / cell_volume * count * (count - 1) * float(mr[0, 0]))))
    f = O.fast_params(SEED, 11, fnum, dt, cell_volume, cs, 0.5, 0.0, ntc_local=1, warp_cap=2048)
    vo, mr_o = vel.copy(), mr.copy()
    info, _ = O.collide_fast(f, vo[0], vo[1], vo[2], start, mr_o)
    assert np.all(info[:, 0] == 5) and info[:, 1].min() >= 1 and info[:, 1].mean() > 2.5
    u, v, w = (T(vel[k].copy(), cuda) for k in range(3))
    mr_t = T(mr.copy(), cuda)
    p = stages.collide_params(ncells, cell_volume, cs, fnum, 0.0, dt, ntc_local=1, rng="philox",
                              seed=SEED, step=11)
    stages.collide(p, u, v, w, U32(start, cuda), mr_t)
    torch.cuda.synchronize()
    vg = np.stack([t.cpu().numpy() for t in (u, v, w)])
    ok = np.repeat(info[:, 3] == 0, counts)
    assert ok.mean() > 0.99
    speed = np.maximum(np.linalg.norm(vo.astype(np.float64), axis=0), 1.0)
    # five collisions per particle at most: 5 x 1e-6 of the speed
    assert np.max(np.max(np.abs(vg - vo), axis=0)[ok] / speed[ok]) <= 5e-6
    assert np.array_equal(mr_t.cpu().numpy()[:, 1], mr_o[:, 1])


def sphere_solver(dim=(32, 16, 16), dom=(0.6, 0.3, 0.3), density=1e20, ppc=8.0, radius=0.06,
                  level=3, variant=None, faces=None, temp=200.0, stream=1500.0, dt=4e-6):
    cell_v = (dom[0] / dim[0]) * (dom[1] / dim[1]) * (dom[2] / dim[2])
    fnum = density * cell_v / ppc
    faces = faces or {"-x": "inflow", "+x": "outflow", "-y": "outflow", "+y": "outflow",
                      "-z": "outflow", "+z": "outflow"}
    s = settings_t().set(grid_min=(0, 0, 0), grid_max=dom, grid_dim=dim, density=density, fnum=fnum,
                         temp=temp, stream_vel=(stream, 0.0, 0.0), dt=dt, rng="philox", ntc_local=1,
                         sample_every=0, init_kind="maxwell", wall_diffuse=1, wall_temp=300.0,
                         capacity_factor=2.0, seed=SEED, geom_nearest=1, face_kind=faces,
                         gas_mass=M_AR, gas_diam=D_AR, gas_tref=TREF, gas_omega=OMEGA)
    center = (0.35 * dom[0], 0.5 * dom[1], 0.5 * dom[2])
    verts, tris = mesh_icosphere(level, radius, center)
    sol = DSMCSolver().Init(s)
    sol.SetModel(verts, tris, (12, 12, 12))
    if variant is not None:
        sol.SetKernelVariant(variant)
    return sol, s, verts, tris, center


def test_move_nearest_diffuse_matches_oracle(cuda):
    sol, s, verts, tris, center = sphere_solver()
    c = s.cfg
    dom = tuple(c.grid_max)
    n = 120000
    rng = np.random.default_rng(12)
    pos = rng.uniform([0, 0, 0], dom, (n, 3))
    # half the particles aimed at the sphere from close by
    k = n // 2
    d = rng.normal(size=(k, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pos[:k] = np.asarray(center) + d * rng.uniform(0.0605, 0.08, k)[:, None]
    vel = rng.normal(0.0, 400.0, (n, 3))
    vel[:k] += -d * rng.uniform(500, 3000, k)[:, None]
    vel[k:, 0] += 1500.0
    # a few particles inside the body (left over from a fill): removed when
    # their path reaches a face from behind
    pos[k:k + 200] = np.asarray(center) + rng.normal(0, 0.02, (200, 3))
    st6 = np.ascontiguousarray(np.concatenate([pos.T, vel.T]).astype(np.float32))
    dt = 2e-5
    kinds = [4, 2, 1, 0, 3, 3]  # -x inflow, +x outflow, -y diffuse, +y specular, z periodic
    vstd = [0.0, 0.0, vstd_of(250.0), 0.0, 0.0, 0.0]
    step = 9
    grid = stages.make_grid((0, 0, 0), dom, tuple(c.grid_dim))
    mp = stages.move_params(grid, dt, faces={"-x": "inflow", "+x": "outflow", "-y": "diffuse",
                                             "+y": "specular", "-z": "periodic", "+z": "periodic"},
                            face_vstd={"-y": vstd[2]}, seed=SEED, step=step)
    ts = [T(st6[q].copy(), cuda) for q in range(6)]
    stages.move(mp, *ts, solver=sol)
    torch.cuda.synchronize()
    got = np.stack([t.cpu().numpy() for t in ts])
    sim = sim_for((0, 0, 0), dom, tuple(c.grid_dim), c.fnum, D_AR)
    m = O.fast_move_params(sim, kinds, vstd, dt, SEED, step, O.triangles_of(verts, tris),
                           wall_diffuse=1, wall_vstd=vstd_of(300.0))
    ref = st6.copy()
    live, amb = O.move_fast(m, ref)
    live_g = ~np.isnan(got[0])
    print(f"removed {int((~live).sum())}, ambiguous {int(amb.sum())}, "
          f"body hits {int(np.sum(np.any(ref[3:] != st6[3:], 0)))}")
    assert amb.sum() <= n // 2000
    ok = ~amb
    assert np.array_equal(live_g[ok], live[ok])
    assert (~live).sum() > 1000  # outflow and body removals
    both = ok & live
    size = max(dom)
    assert np.max(np.abs(got[:3, both] - ref[:3, both])) <= 1e-6 * size
    speed = np.maximum(np.linalg.norm(ref[3:, both].astype(np.float64), axis=0), 1.0)
    assert np.max(np.max(np.abs(got[3:, both] - ref[3:, both]), axis=0) / speed) <= 1e-6
    hits = np.any(ref[3:] != st6[3:], axis=0) & both
    assert hits.sum() > 20000
    # most particles are reproduced bit for bit (free flights, specular faces)
    exact = np.all(got[:, both] == ref[:, both], axis=0)
    assert exact.mean() > 0.5
    sol.close()


def test_inflow_injection_matches_oracle(cuda):
    """An empty box with an inflow face: after one step the state holds
    exactly the injected particles, in the oracle's order."""
    sol, s, verts, tris, center = sphere_solver(density=3e20)
    c = s.cfg
    sol.UploadState(np.zeros((6, 0), np.float32), soa=True)
    for _ in range(3):
        sol.RunSimulationStep(c.dt)
    st = sol.DownloadState()
    keys = sol.ReadKeys()
    info = sol.Info()
    inflows = O.library_inflows(c)
    assert len(inflows) == 1
    sim = sim_for((0, 0, 0), tuple(c.grid_max), tuple(c.grid_dim), c.fnum, D_AR)
    rem, ks = O.inject_plan_chain(inflows[0], c.dt, info.step - 1)
    inj, amb, rem2 = O.inject_fast(inflows[0], sim, c.dt, SEED, info.step, rem, 1 << 24)
    kk = inj.shape[1]
    assert kk > 500
    assert st.shape[1] >= kk
    got = st[:, -kk:]
    print(f"injected {kk} at step {info.step}; ambiguous {int(amb.sum())}")
    assert amb.sum() <= kk // 1000
    ok = ~amb
    assert np.max(np.abs(got[:3, ok] - inj[:3, ok])) <= 1e-6 * 0.6
    speed = np.linalg.norm(inj[3:, ok].astype(np.float64), axis=0)
    assert np.max(np.max(np.abs(got[3:, ok] - inj[3:, ok]), axis=0) / speed) <= 1e-6
    inside = np.all((inj[:3] >= 0) & (inj[:3] <= np.array(tuple(c.grid_max), np.float32)[:, None]), 0)
    kref = O.keys_of(sim, inj, inside)
    near = O.near_cell_face(sim, inj)
    assert np.array_equal(keys[-kk:][ok & ~near], kref[ok & ~near])
    # flux-weighted inward normal speeds: mean u of the injected particles
    # above the stream speed
    assert inj[3].mean() > 1500.0
    sol.close()


@pytest.mark.parametrize("variant", [5, 7, 0])
def test_step_matches_oracle(cuda, variant):
    """Whole timesteps of a sphere flow in the capsule workload's mode: the
    GPU steps 12 times to develop the flow, then each of three more steps is
    compared with the oracle's step from the GPU's own state before it."""
    sol, s, verts, tris, center = sphere_solver(variant=variant)
    c = s.cfg
    sol.InitSystemState()
    sol.RunSimulationStep(c.dt, 12)
    chunk = sol.KernelVariant()[1]
    sim = sim_for((0, 0, 0), tuple(c.grid_max), tuple(c.grid_dim), c.fnum, D_AR)
    gref = vhs_gref()
    inflows = O.library_inflows(c)
    tri9 = O.triangles_of(verts, tris)
    totals0 = np.array(sol.Totals())
    for rep in range(3):
        st0 = sol.DownloadState()
        keys0 = sol.ReadKeys()
        mr0, _ = sol.GetCellState()
        step = sol.Info().step + 1
        rem, _ = O.inject_plan_chain(inflows[0], c.dt, step - 1)
        f = O.fast_params(SEED, step, c.fnum, c.dt, sim.cell_volume, sim.cross_section, OMEGA, gref,
                          ntc_local=1, warp_cap=chunk)
        m = O.fast_move_params(sim, list(c.face_kind), [0.0] * 6, c.dt, SEED, step, tri9,
                               wall_diffuse=1, wall_vstd=vstd_of(300.0))
        ref = O.step_fast(f, m, sim, st0, keys0, mr0, inflows, {inflows[0].face: rem})
        sol.RunSimulationStep(c.dt)
        st1 = sol.DownloadState()
        keys1 = sol.ReadKeys()
        mr1, _ = sol.GetCellState()
        totals1 = np.array(sol.Totals())
        assert sol.Info().step == step
        R = ref["state"]
        assert st1.shape == R.shape, (st1.shape, R.shape)
        amb = ref["ambiguous"]
        tie = ref["tie_cell"]
        print(f"variant {variant} step {step}: {R.shape[1]} slots, {ref['n_alive']} sorted, "
              f"tie cells {int(tie.sum())}, ambiguous slots {int(amb.sum())}, "
              f"paths {np.bincount(ref['info'][:, 2], minlength=4).tolist()}")
        assert amb.mean() < 2e-3
        ok = ~amb
        assert np.array_equal(keys1[ok], ref["keys"][ok])
        live = ok & (ref["keys"] != O.DEAD)
        assert np.max(np.abs(st1[:3, live] - R[:3, live])) <= 1e-6 * 0.6
        speed = np.maximum(np.linalg.norm(R[3:, live].astype(np.float64), axis=0), 1.0)
        assert np.max(np.max(np.abs(st1[3:, live] - R[3:, live]), axis=0) / speed) <= 1e-6
        assert np.array_equal(mr1[:, 1], ref["maxrem"][:, 1])
        assert np.allclose(mr1[~tie, 0], ref["maxrem"][~tie, 0], rtol=4e-6, atol=0)
        sel = totals1[0] - totals0[0]
        col = totals1[1] - totals0[1]
        assert sel == ref["info"][:, 0].sum()
        assert abs(col - ref["info"][:, 1].sum()) <= ref["info"][tie, 0].sum()
        totals0 = totals1
    sol.close()
