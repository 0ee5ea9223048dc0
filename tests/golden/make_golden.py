"""Generates the golden fixtures of tests/golden/ from the reference's own
code: kernels/dsmc_kernel.cu (built headless for sm_100a into
oracle/_ref/libdsmc_ref.so, needs a GPU) and its host geometry code.

Usage (on a machine with a GPU and oracle/_ref built):
    python tests/golden/make_golden.py [OUTDIR]
    python tests/golden/make_golden.py --only collide_mt [OUTDIR]

Every fixture stores its seeded inputs and the reference's outputs; the CPU
tests check the oracle against them (tests/test_cpu_oracle_golden.py).
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import torch  # noqa: E402

from oracle import oracle as O  # noqa: E402
from helpers import box_case, taus_seeds, maxrem_init  # noqa: E402

P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731


def icosphere(level, radius, center):
    t = (1.0 + 5 ** 0.5) / 2
    v = [[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t],
         [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]]
    v = [list(np.asarray(p) / np.linalg.norm(p)) for p in v]
    f = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
         [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
         [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]]
    for _ in range(level):
        mid = {}
        def m(a, b):
            k = (min(a, b), max(a, b))
            if k not in mid:
                p = np.asarray(v[a]) + np.asarray(v[b])
                v.append(list(p / np.linalg.norm(p)))
                mid[k] = len(v) - 1
            return mid[k]
        g = []
        for a, b, c in f:
            ab, bc, ca = m(a, b), m(b, c), m(c, a)
            g += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        f = g
    verts = (np.asarray(center) + radius * np.asarray(v)).astype(np.float32)
    return verts, np.asarray(f, np.uint32)


def ref_init(R, gmin, gmax, dim, density, fnum, temp, mass, diam, tref, periodic):
    cfg = O.RefConfig()
    cfg.gmin[:], cfg.gmax[:], cfg.dim[:] = gmin, gmax, dim
    cfg.density, cfg.fnum, cfg.temp = density, fnum, temp
    cfg.mass, cfg.diam, cfg.tref = mass, diam, tref
    cfg.periodic = periodic.encode()
    assert R.ref_init(ctypes.byref(cfg)) == 0
    ppc = ctypes.c_uint32()
    cv, cs, mrv = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    csz = (ctypes.c_float * 3)()
    R.ref_derived(ctypes.byref(ppc), ctypes.byref(cv), ctypes.byref(cs), ctypes.byref(mrv), csz)
    return dict(ppc=ppc.value, cell_volume=cv.value, cross_section=cs.value, max_rel_vel=mrv.value,
                cell=np.asarray(list(csz), np.float32))


def main(out):
    os.makedirs(out, exist_ok=True)
    R = O.ref()
    dev = torch.device("cuda:0")
    gmin, gmax, dim = (0.0, 0.0, 0.0), (0.8, 0.4, 0.4), (8, 4, 4)
    mass, diam, tref, temp = 6.63e-26, 4.17e-10, 273.0, 300.0

    # HybridTaus draws
    st = taus_seeds(1, 64)
    s_t = torch.from_numpy(st.view(np.int32).copy()).to(dev)
    ints = torch.zeros(64 * 16, dtype=torch.int32, device=dev)
    fl = torch.zeros(64 * 16, dtype=torch.float32, device=dev)
    assert R.ref_taus_draws(P(s_t), 64, 16, P(ints), P(fl)) == 0
    np.savez_compressed(os.path.join(out, "taus.npz"), states=st,
                        ints=ints.cpu().numpy().view(np.uint32).reshape(64, 16),
                        floats=fl.cpu().numpy().reshape(64, 16),
                        after=s_t.cpu().numpy().view(np.uint32).reshape(64, 4))

    # cell ids and the stable sort
    d = ref_init(R, gmin, gmax, dim, 1e20, 1e15, temp, mass, diam, tref, "n")
    pos, vel = box_case(2, dim, gmin, gmax, 4096, inside=False)
    pos[:200, 0] = -0.1
    pos[200:400, 2] = 0.55
    pos[400, :3] = gmax
    p_t = torch.from_numpy(pos).to(dev)
    h = torch.zeros(4096, dtype=torch.int32, device=dev)
    ix = torch.zeros(4096, dtype=torch.int32, device=dev)
    assert R.ref_cell_ids(P(p_t), P(h), P(ix), 4096) == 0
    keys = h.cpu().numpy().view(np.uint32).copy()
    assert R.ref_sort(P(h), P(ix), 4096) == 0
    np.savez_compressed(os.path.join(out, "cellids_sort.npz"), gmin=gmin, gmax=gmax, dim=dim,
                        pos=pos, keys=keys, sorted_keys=h.cpu().numpy().view(np.uint32),
                        sorted_idx=ix.cpu().numpy().view(np.uint32))

    # collisions on a sorted case (10 per cell)
    n = 128 * 10
    pos, vel = box_case(3, dim, gmin, gmax, n, vstd=400.0)
    sim = O.sim_from(gmin, gmax, dim, 1e15, d["cross_section"])
    k, i = O.cell_ids(sim, pos)
    k, i = O.sort(k, i, sim.cells)
    cse, sp, sv = O.bounds_reorder(sim, k, i, pos, vel)
    seeds = taus_seeds(4, 128)
    mr = maxrem_init(5, 128, d["max_rel_vel"])
    assert R.ref_set_cell_state(O.p(mr), O.p(seeds)) == 0
    assert R.ref_clear_stats() == 0
    v_t = torch.from_numpy(sv.copy()).to(dev)
    c_t = torch.from_numpy(cse.view(np.int32).copy()).to(dev)
    dt = 4e-5
    assert R.ref_collide(P(v_t), P(c_t), 10, ctypes.c_float(dt)) == 0
    mr_o = np.zeros_like(mr)
    sd_o = np.zeros_like(seeds)
    st4 = np.zeros((128, 4), np.float32)
    R.ref_get_cell_state(O.p(mr_o), O.p(sd_o), O.p(st4), None)
    np.savez_compressed(os.path.join(out, "collide.npz"), gmin=gmin, gmax=gmax, dim=dim, dt=dt,
                        avg_conc=10.0, fnum=1e15, cross_section=d["cross_section"],
                        cell_volume=d["cell_volume"], vel=sv, cse=cse, maxrem=mr, seeds=seeds,
                        vel_out=v_t.cpu().numpy(), maxrem_out=mr_o, seeds_out=sd_o, stat4=st4)

    # moves: the four boundary functors, then the icosphere
    for per in "nxyz":
        ref_init(R, gmin, gmax, dim, 1e20, 1e15, temp, mass, diam, tref, per)
        pos, vel = box_case(6, dim, gmin, gmax, 4000, vstd=900.0)
        p_t, v_t = torch.from_numpy(pos.copy()).to(dev), torch.from_numpy(vel.copy()).to(dev)
        assert R.ref_move(P(p_t), P(v_t), ctypes.c_float(1e-4), 4000, 0, ctypes.c_char(per.encode())) == 0
        np.savez_compressed(os.path.join(out, f"move_{per}.npz"), gmin=gmin, gmax=gmax, dim=dim,
                            dt=1e-4, pos=pos, vel=vel, pos_out=p_t.cpu().numpy(),
                            vel_out=v_t.cpu().numpy())
    center = (0.4, 0.2, 0.2)
    verts, tris = icosphere(2, 0.1, center)
    gdim = (5, 5, 5)
    bbox, cell, count, ids, flags = O.build_grid(verts, tris, gdim, use_ref=True)
    nrm = np.cross(verts[tris[:, 1]] - verts[tris[:, 0]], verts[tris[:, 2]] - verts[tris[:, 0]])
    nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
    ref_init(R, gmin, gmax, dim, 1e20, 1e15, temp, mass, diam, tref, "n")
    gd = np.asarray(gdim, np.int32)
    assert R.ref_set_geometry(O.p(bbox), O.p(cell), O.p(gd), O.p(count), O.p(ids), O.p(flags),
                              O.p(verts.reshape(-1)), len(verts), O.p(tris.reshape(-1)),
                              O.p(nrm.reshape(-1))) == 0
    rng = np.random.default_rng(7)
    dd = rng.normal(size=(4000, 3))
    dd /= np.linalg.norm(dd, axis=1, keepdims=True)
    pos = np.zeros((4000, 4), np.float32)
    vel = np.zeros((4000, 4), np.float32)
    pos[:, :3] = np.asarray(center) + dd * rng.uniform(0.102, 0.14, 4000)[:, None]
    vel[:, :3] = -dd * rng.uniform(200, 1200, 4000)[:, None] + rng.normal(0, 100, (4000, 3))
    p_t, v_t = torch.from_numpy(pos.copy()).to(dev), torch.from_numpy(vel.copy()).to(dev)
    assert R.ref_move(P(p_t), P(v_t), ctypes.c_float(5e-5), 4000, 1, ctypes.c_char(b"n")) == 0
    np.savez_compressed(os.path.join(out, "move_sphere.npz"), gmin=gmin, gmax=gmax, dim=dim, dt=5e-5,
                        verts=verts, tris=tris, normals=nrm, gdim=gdim, bbox=bbox, cell=cell,
                        count=count, ids=ids, flags=flags, pos=pos, vel=vel,
                        pos_out=p_t.cpu().numpy(), vel_out=v_t.cpu().numpy())

    # three whole steps with sampling on the last
    d = ref_init(R, gmin, gmax, dim, 1.2e20, 1e16, temp, mass, diam, tref, "n")
    n = d["ppc"] * 128
    pos, vel = box_case(8, dim, gmin, gmax, n, vstd=400.0)
    seeds = taus_seeds(9, 128)
    mr = maxrem_init(10, 128, d["max_rel_vel"])
    assert R.ref_set_cell_state(O.p(mr), O.p(seeds)) == 0
    assert R.ref_clear_stats() == 0
    pc, vc = torch.from_numpy(pos.copy()).to(dev), torch.from_numpy(vel.copy()).to(dev)
    po, vo = torch.zeros_like(pc), torch.zeros_like(vc)
    hh = torch.zeros(n, dtype=torch.int32, device=dev)
    ii = torch.zeros(n, dtype=torch.int32, device=dev)
    cs = torch.zeros(256, dtype=torch.int32, device=dev)
    for s in range(3):
        pc, po = po, pc
        vc, vo = vo, vc
        assert R.ref_step(P(pc), P(po), P(vc), P(vo), P(hh), P(ii), P(cs), n, ctypes.c_float(1e-5),
                          1, 0, 1 if s == 2 else 0) == 0
    mr_o = np.zeros_like(mr)
    sd_o = np.zeros_like(seeds)
    st4 = np.zeros((128, 4), np.float32)
    # statistics_t (include/statistics.h:31-37) is 32 bytes: numInSample,
    # xyzSum, velMag, 4 bytes of alignment padding, the float2 padd
    cs8 = np.zeros((128, 8), np.float32)
    R.ref_get_cell_state(O.p(mr_o), O.p(sd_o), O.p(st4), O.p(cs8))
    np.savez_compressed(os.path.join(out, "step3.npz"), gmin=gmin, gmax=gmax, dim=dim, dt=1e-5,
                        ppc=d["ppc"], fnum=1e16, cross_section=d["cross_section"],
                        cell_volume=d["cell_volume"], max_rel_vel=d["max_rel_vel"], pos=pos, vel=vel,
                        maxrem=mr, seeds=seeds, pos_out=pc.cpu().numpy(), vel_out=vc.cpu().numpy(),
                        maxrem_out=mr_o, seeds_out=sd_o, stat4=st4, cell_stats=cs8[:, :5].copy(),
                        cse=cs.cpu().numpy().view(np.uint32).reshape(-1, 2))
    print("golden fixtures written to", out)


def collide_mt(out):
    """The -mt collisions (ComputeBirdCollisionsDev) on the case of
    collide.npz, with the reference's twisters set up as its solver does:
    data/MersenneTwister.dat (copied to oracle/_ref by `make -C oracle ref`)
    and seed 999 (SEED, include/MersenneTwister.h:17)."""
    os.makedirs(out, exist_ok=True)
    R = O.ref()
    dev = torch.device("cuda:0")
    gmin, gmax, dim = (0.0, 0.0, 0.0), (0.8, 0.4, 0.4), (8, 4, 4)
    mass, diam, tref, temp = 6.63e-26, 4.17e-10, 273.0, 300.0
    d = ref_init(R, gmin, gmax, dim, 1e20, 1e15, temp, mass, diam, tref, "n")
    n = 128 * 10
    pos, vel = box_case(3, dim, gmin, gmax, n, vstd=400.0)
    sim = O.sim_from(gmin, gmax, dim, 1e15, d["cross_section"])
    k, i = O.cell_ids(sim, pos)
    k, i = O.sort(k, i, sim.cells)
    cse, sp, sv = O.bounds_reorder(sim, k, i, pos, vel)
    mr = maxrem_init(5, 128, d["max_rel_vel"])
    assert R.ref_mt_init(O.MT_DAT.encode(), 999) == 0
    cfg = np.zeros((128, 4), np.uint32)
    st0 = np.zeros((128, 21), np.uint32)
    assert R.ref_mt_get(128, O.p(cfg), O.p(st0)) == 0
    assert R.ref_set_cell_state(O.p(mr), None) == 0
    assert R.ref_clear_stats() == 0
    v_t = torch.from_numpy(sv.copy()).to(dev)
    c_t = torch.from_numpy(cse.view(np.int32).copy()).to(dev)
    dt = 4e-5
    assert R.ref_collide_mt(P(v_t), P(c_t), 10, ctypes.c_float(dt)) == 0
    st1 = np.zeros_like(st0)
    assert R.ref_mt_get(128, None, O.p(st1)) == 0
    mr_o = np.zeros_like(mr)
    st4 = np.zeros((128, 4), np.float32)
    R.ref_get_cell_state(O.p(mr_o), None, O.p(st4), None)
    np.savez_compressed(os.path.join(out, "collide_mt.npz"), gmin=gmin, gmax=gmax, dim=dim, dt=dt,
                        avg_conc=10.0, fnum=1e15, cross_section=d["cross_section"],
                        cell_volume=d["cell_volume"], vel=sv, cse=cse, maxrem=mr, mt_cfg=cfg,
                        mt_state=st0, vel_out=v_t.cpu().numpy(), maxrem_out=mr_o,
                        mt_state_out=st1, stat4=st4)
    print("collide_mt.npz written to", out)


if __name__ == "__main__":
    # make_golden.py [--only collide_mt] [OUTDIR]
    args = sys.argv[1:]
    only = None
    if args[:1] == ["--only"]:
        only, args = args[1], args[2:]
    outdir = args[0] if args else os.path.dirname(os.path.abspath(__file__))
    if only in (None, "collide_mt"):
        if only is None:
            main(outdir)
        collide_mt(outdir)
    else:
        raise SystemExit(f"unknown fixture {only}")
