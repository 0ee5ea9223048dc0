"""Stage-by-stage parity of the CUDA kernels with the CPU oracle.

Integer outputs (cell keys, sort order, cell starts/ends, RNG states, pair and
collision counts) must match bit for bit.  Floating point: the move without a
mesh is bit-exact; post-collision velocities match within 2e-6 of the pair's
speed scale (the oracle uses libm cosf/sinf where the kernels use the
hardware __cosf/__sinf the reference uses); mesh hits within 1e-5 of the path
length.
"""
import numpy as np
import pytest
import torch

from cudadsmc_b200 import stages, mesh_icosphere, build_geometry_grid, settings_t, DSMCSolver
from oracle import oracle as O

from helpers import box_case, soa_from_aos, taus_seeds, maxrem_init, sim_for

pytestmark = pytest.mark.gpu

GMIN, GMAX = (0.0, 0.0, 0.0), (1.0, 0.5, 0.5)
DIM = (32, 16, 16)


def T(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def U32(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32)).to(dev)


def np_u32(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n", [1, 1000, 65537])
def test_cell_index_bit_exact(cuda, n):
    pos, _ = box_case(1, DIM, GMIN, GMAX, n, inside=False)
    # out-of-box, negative and boundary coordinates exercise the saturating
    # float->uint conversion and the clamp of GetCellID3D
    pos[: n // 10, 0] = np.float32(-0.25)
    pos[n // 10: n // 5, 1] = np.float32(0.75)
    pos[-1, :3] = np.float32(GMAX)
    sim = sim_for(GMIN, GMAX, DIM, 1e15, 4.17e-10)
    k_ref, i_ref = O.cell_ids(sim, pos)
    g = stages.make_grid(GMIN, GMAX, DIM)
    x, y, z = (T(pos[:, k].copy(), cuda) for k in range(3))
    keys = torch.zeros(n, dtype=torch.int32, device=cuda)
    idx = torch.zeros(n, dtype=torch.int32, device=cuda)
    stages.cell_index(g, x, y, z, keys, idx)
    torch.cuda.synchronize()
    assert np.array_equal(np_u32(keys), k_ref)
    assert np.array_equal(np_u32(idx), i_ref)


@pytest.mark.parametrize("n,nkeys,mode", [
    (0, 5, "rand"), (1, 1, "rand"), (2, 7, "rand"), (100000, 4096, "rand"), (131072, 65536, "rand"),
    (50000, 2048, "same"), (20000, 300, "nearly"), (70000, 10, "rand")])
def test_sort_stable_bit_exact(cuda, n, nkeys, mode):
    rng = np.random.default_rng(n + nkeys)
    if mode == "same":
        keys = np.full(n, nkeys - 1, np.uint32)  # one key holding every entry
    elif mode == "nearly":
        keys = np.sort(rng.integers(0, nkeys, n)).astype(np.uint32)
        swap = rng.integers(0, n, n // 20)
        keys[swap] = rng.integers(0, nkeys, len(swap)).astype(np.uint32)
    else:
        keys = rng.integers(0, nkeys, n).astype(np.uint32)
    vals = rng.permutation(n).astype(np.uint32)
    k_ref, v_ref = O.sort(keys, vals, nkeys)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(v_ref, vals[order])  # oracle = stable sort
    kt, vt = U32(keys, cuda), U32(vals, cuda)
    st = torch.zeros(nkeys + 1, dtype=torch.int32, device=cuda)
    stages.sort(kt, vt, nkeys, cell_start=st)
    torch.cuda.synchronize()
    assert np.array_equal(np_u32(kt), k_ref)
    assert np.array_equal(np_u32(vt), v_ref)
    counts = np.bincount(keys, minlength=nkeys)
    assert np.array_equal(np_u32(st), np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32))


def test_sort_with_caller_workspace(cuda):
    n, nkeys = 30000, 1000
    rng = np.random.default_rng(3)
    keys = rng.integers(0, nkeys, n).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    wb = stages.sort_workspace_bytes(n, nkeys)
    ws = torch.zeros(wb, dtype=torch.uint8, device=cuda)
    kt, vt = U32(keys, cuda), U32(vals, cuda)
    stages.sort(kt, vt, nkeys, workspace=ws)
    torch.cuda.synchronize()
    k_ref, v_ref = O.sort(keys, vals, nkeys)
    assert np.array_equal(np_u32(kt), k_ref) and np.array_equal(np_u32(vt), v_ref)


def test_bounds_reorder_bit_exact(cuda):
    n = 40000
    pos, vel = box_case(5, DIM, GMIN, GMAX, n)
    sim = sim_for(GMIN, GMAX, DIM, 1e15, 4.17e-10)
    keys, idx = O.cell_ids(sim, pos)
    keys, idx = O.sort(keys, idx, sim.cells)
    cse_ref, sp, sv = O.bounds_reorder(sim, keys, idx, pos, vel)
    src = [T(np.ascontiguousarray(a), cuda) for a in soa_from_aos(pos, vel)]
    dst = [torch.zeros_like(a) for a in src]
    cse = torch.zeros(2 * sim.cells, dtype=torch.int32, device=cuda)
    stages.bounds_reorder(U32(keys, cuda), U32(idx, cuda), sim.cells, cse, src, dst)
    torch.cuda.synchronize()
    assert np.array_equal(np_u32(cse).reshape(-1, 2), cse_ref)
    got = np.stack([d.cpu().numpy() for d in dst])
    assert np.array_equal(got, soa_from_aos(sp, sv))


def _sorted_case(seed, n, dim=DIM, vstd=400.0):
    pos, vel = box_case(seed, dim, GMIN, GMAX, n, vstd=vstd)
    sim = sim_for(GMIN, GMAX, dim, 1e15, 4.17e-10)
    keys, idx = O.cell_ids(sim, pos)
    keys, idx = O.sort(keys, idx, sim.cells)
    cse, sp, sv = O.bounds_reorder(sim, keys, idx, pos, vel)
    return sim, sp, sv, cse


@pytest.mark.parametrize("omega,ppc", [(0.5, 8), (0.5, 40), (0.81, 12)])
def test_collide_taus(cuda, omega, ppc):
    n = ppc * 32 * 16 * 16
    sim, sp, sv, cse = _sorted_case(11 + ppc, n)
    gref = 0.0
    if omega != 0.5:
        import math
        m, tref, w = 6.63e-26, 273.0, omega
        gref = math.sqrt(2 * 1.380649e-23 * tref / (0.5 * m)) * math.gamma(2.5 - w) ** (-1 / (2 * w - 1))
        sim = sim_for(GMIN, GMAX, DIM, 1e15, 4.17e-10, omega=omega, vhs_gref=gref)
    cells = sim.cells
    seeds = taus_seeds(7, cells)
    mr = maxrem_init(8, cells, O.max_rel_vel_of(4.17e-10, 300.0))
    st4 = np.zeros((cells, 4), np.float32)
    dt, avg = 2e-5, float(ppc)
    v_or = sv.copy()
    mr_or, st_or, sd_or = mr.copy(), st4.copy(), seeds.copy()
    O.collide(sim, v_or, cse, mr_or, st_or, sd_or, avg, dt)
    starts = np.concatenate([[0], np.cumsum(cse[:, 1] - cse[:, 0])]).astype(np.uint32)
    u, v, w = (T(sv[:, k].copy(), cuda) for k in range(3))
    mr_t, sd_t, st_t = T(mr.copy(), cuda), U32(seeds, cuda), T(st4.copy(), cuda)
    p = stages.collide_params(cells, sim.cell_volume, sim.cross_section, sim.fnum, avg, dt,
                              omega=omega, vhs_gref=gref)
    stages.collide(p, u, v, w, U32(starts, cuda), mr_t, sd_t, st_t)
    torch.cuda.synchronize()
    sd_g = np_u32(sd_t).reshape(-1, 4)
    same = np.all(sd_g == sd_or, axis=1)
    # The oracle runs on the host: its cosf/sinf (libm) and the GPU's
    # __cosf/__sinf differ in the last bits, so post-collision velocities can
    # differ by an ulp, and a later acceptance test in the same cell (random
    # number against sigma g / (sigma g)max) that close to its threshold can
    # go the other way; that cell's stream then consumes a different number
    # of draws.  Such cells (at most 0.1 %) are left out of the exact
    # comparison; against the reference's own GPU kernels every cell is
    # bit-identical (test_gpu_step.py, test_steps_vs_reference_kernels).
    assert same.mean() >= 0.999, f"RNG streams diverged in {np.sum(~same)} cells"
    st_g = st_t.cpu().numpy()
    assert np.array_equal(st_g[same, 0], st_or[same, 0])  # selections
    assert np.array_equal(st_g[same, 1], st_or[same, 1])  # collisions
    assert st_or[:, 1].sum() > 1000
    vg = np.stack([t.cpu().numpy() for t in (u, v, w)], 1)
    vo = v_or[:, :3]
    mask = np.repeat(same, (cse[:, 1] - cse[:, 0]).astype(np.int64))
    scale = 3 * 400.0
    err = np.max(np.abs(vg[mask] - vo[mask])) / scale
    assert err <= 2e-6, err
    mr_g = mr_t.cpu().numpy()
    assert np.allclose(mr_g[same], mr_or[same], rtol=2e-6, atol=0)
    # momentum and energy of every cell are conserved by the collisions
    p0 = np.add.reduceat(sv[:, :3].astype(np.float64), starts[:-1][cse[:, 1] > cse[:, 0]], axis=0)
    p1 = np.add.reduceat(vg.astype(np.float64), starts[:-1][cse[:, 1] > cse[:, 0]], axis=0)
    assert np.max(np.abs(p1 - p0)) / scale < 1e-4
    e0 = np.sum(sv[:, :3].astype(np.float64) ** 2)
    e1 = np.sum(vg.astype(np.float64) ** 2)
    assert abs(e1 - e0) / e0 < 1e-6


def test_collide_philox_reproducible(cuda):
    n = 8 * 32 * 16 * 16
    sim, sp, sv, cse = _sorted_case(21, n)
    cells = sim.cells
    starts = np.concatenate([[0], np.cumsum(cse[:, 1] - cse[:, 0])]).astype(np.uint32)
    outs = []
    for _ in range(2):
        u, v, w = (T(sv[:, k].copy(), cuda) for k in range(3))
        mr_t = T(maxrem_init(8, cells, O.max_rel_vel_of(4.17e-10, 300.0)), cuda)
        p = stages.collide_params(cells, sim.cell_volume, sim.cross_section, sim.fnum, 8.0, 2e-5,
                                  rng="philox", seed=1234, step=5)
        stages.collide(p, u, v, w, U32(starts, cuda), mr_t)
        torch.cuda.synchronize()
        outs.append(np.stack([t.cpu().numpy() for t in (u, v, w)]))
    assert np.array_equal(outs[0], outs[1])
    assert not np.array_equal(outs[0], soa_from_aos(sp, sv)[3:])


@pytest.mark.parametrize("periodic", ["n", "x", "y", "z"])
def test_move_boundaries_bit_exact(cuda, periodic):
    n = 50000
    pos, vel = box_case(31, DIM, GMIN, GMAX, n, vstd=900.0)
    dt = 1e-4  # many particles cross a face in one step
    sim = sim_for(GMIN, GMAX, DIM, 1e15, 4.17e-10, periodic=periodic)
    po, vo = pos.copy(), vel.copy()
    O.move(sim, None, po, vo, dt)
    a = soa_from_aos(pos, vel)
    ts = [T(a[k].copy(), cuda) for k in range(6)]
    mp = stages.move_params(stages.make_grid(GMIN, GMAX, DIM), dt, periodic=periodic)
    stages.move(mp, *ts)
    torch.cuda.synchronize()
    got = np.stack([t.cpu().numpy() for t in ts])
    assert np.array_equal(got, soa_from_aos(po, vo))
    crossed = np.any((pos[:, :3] + vel[:, :3] * dt < GMIN) | (pos[:, :3] + vel[:, :3] * dt > GMAX), 1)
    assert crossed.sum() > 1000


def test_move_sphere_first_hit(cuda):
    # specular icosphere in the middle of the box; particles aimed at it
    center = (0.5, 0.25, 0.25)
    verts, tris = mesh_icosphere(2, 0.1, center)
    gdim = (5, 5, 5)
    bbox, cell, count, ids, flags = build_geometry_grid(verts, tris, gdim)
    nrm = np.cross(verts[tris[:, 1]] - verts[tris[:, 0]], verts[tris[:, 2]] - verts[tris[:, 0]])
    nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
    n = 40000
    rng = np.random.default_rng(41)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = rng.uniform(0.102, 0.14, n)
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 4), np.float32)
    pos[:, :3] = np.asarray(center) + d * r[:, None]
    vel[:, :3] = -d * rng.uniform(200, 1200, n)[:, None] + rng.normal(0, 100, (n, 3))
    dt = 5e-5
    s = settings_t().set(grid_min=GMIN, grid_max=GMAX, grid_dim=DIM, density=1e20, fnum=1e15,
                         temp=300.0, gas_mass=6.63e-26, gas_diam=4.17e-10, periodic="n")
    solver = DSMCSolver().Init(s)
    solver.SetModel(verts, tris, gdim, normals=nrm)
    sim = sim_for(GMIN, GMAX, DIM, 1e15, 4.17e-10)
    geom = O.geom_from(bbox, cell, gdim, count, ids, flags, verts, tris, nrm)
    po, vo = pos.copy(), vel.copy()
    O.move(sim, geom, po, vo, dt)
    a = soa_from_aos(pos, vel)
    ts = [T(a[k].copy(), cuda) for k in range(6)]
    mp = stages.move_params(stages.make_grid(GMIN, GMAX, DIM), dt)
    stages.move(mp, *ts, solver=solver)
    torch.cuda.synchronize()
    got = np.stack([t.cpu().numpy() for t in ts])
    ref = soa_from_aos(po, vo)
    hit_ref = np.any(vo[:, :3] != vel[:, :3], 1)
    hit_gpu = np.any(got[3:].T != vel[:, :3], 1)
    assert hit_ref.sum() > 5000
    assert np.mean(hit_ref == hit_gpu) > 0.9995
    both = hit_ref & hit_gpu
    path = np.linalg.norm(vel[:, :3], axis=1) * dt
    dpos = np.max(np.abs(got[:3].T - ref[:3].T), axis=1)
    assert np.max(dpos[both] / path[both]) < 1e-5
    speed = np.linalg.norm(vel[:, :3], axis=1)
    dvel = np.max(np.abs(got[3:].T - ref[3:].T), axis=1)
    assert np.max(dvel[both] / speed[both]) < 1e-5
    # the reference reflects off the first listed triangle the path crosses,
    # not the nearest, so some paths end inside the body - in both
    rr = np.linalg.norm(got[:3].T - np.asarray(center), axis=1)
    rr_ref = np.linalg.norm(ref[:3].T - np.asarray(center), axis=1)
    assert abs(np.mean(rr < 0.098) - np.mean(rr_ref < 0.098)) < 5e-4
    solver.close()


@pytest.mark.parametrize("diffuse", [0, 1])
def test_move_sphere_nearest_hit_stays_outside(cuda, diffuse):
    """Nearest-hit mode (extension): no path may end inside the body."""
    center = (0.5, 0.25, 0.25)
    verts, tris = mesh_icosphere(3, 0.1, center)
    n = 60000
    rng = np.random.default_rng(43)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = rng.uniform(0.101, 0.16, n)
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 4), np.float32)
    pos[:, :3] = np.asarray(center) + d * r[:, None]
    vel[:, :3] = -d * rng.uniform(200, 3000, n)[:, None] + rng.normal(0, 300, (n, 3))
    s = settings_t().set(grid_min=GMIN, grid_max=GMAX, grid_dim=DIM, density=1e20, fnum=1e15,
                         temp=300.0, gas_mass=6.63e-26, gas_diam=4.17e-10, periodic="n",
                         geom_nearest=1, wall_diffuse=diffuse, wall_temp=300.0)
    solver = DSMCSolver().Init(s)
    solver.SetModel(verts, tris, (8, 8, 8))
    a = soa_from_aos(pos, vel)
    ts = [T(a[k].copy(), cuda) for k in range(6)]
    mp = stages.move_params(stages.make_grid(GMIN, GMAX, DIM), 1e-4, seed=5)
    for _ in range(3):
        stages.move(mp, *ts, solver=solver)
    torch.cuda.synchronize()
    got = np.stack([t.cpu().numpy() for t in ts])
    # inscribed radius of the level-3 icosphere is above 0.0995
    rr = np.linalg.norm(got[:3].T - np.asarray(center), axis=1)
    assert np.mean(rr < 0.0995) < 2e-4
    if diffuse:
        # re-emitted at 300 K: mean speed of the hit particles near sqrt(8kT/(pi m))
        sp = np.linalg.norm(got[3:].T, axis=1)
        hit = np.any(got[3:].T != vel[:, :3], axis=1)
        mean_ref = np.sqrt(8 * 1.3806e-23 * 300 / (np.pi * 6.63e-26))
        assert hit.mean() > 0.5
        assert 0.8 * mean_ref < sp[hit].mean() < 1.35 * mean_ref
    solver.close()


def test_sample_f64(cuda):
    n = 60000
    sim, sp, sv, cse = _sorted_case(51, n)
    starts = np.concatenate([[0], np.cumsum(cse[:, 1] - cse[:, 0])]).astype(np.uint32)
    ref = O.sample_f64(sim, sv, cse)
    u, v, w = (T(sv[:, k].copy(), cuda) for k in range(3))
    acc = torch.zeros(sim.cells * 5, dtype=torch.float64, device=cuda)
    stages.sample(u, v, w, U32(starts, cuda), sim.cells, acc)
    torch.cuda.synchronize()
    got = acc.cpu().numpy().reshape(-1, 5)
    assert np.array_equal(got[:, 0], ref[:, 0])
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-9)
