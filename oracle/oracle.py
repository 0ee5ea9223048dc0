"""ctypes binding of the CPU oracle (liboracle.so), of the reference's own
kernels built headless (_ref/libdsmc_ref.so) and of the reference's twister
code (_ref/libmt_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product package.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libdsmc_ref.so")

_P = ctypes.c_void_p
c_f3 = ctypes.c_float * 3
c_u3 = ctypes.c_uint32 * 3


class OrcSim(ctypes.Structure):
    _fields_ = [("gmin", c_f3), ("gmax", c_f3), ("cell", c_f3), ("dim", c_u3),
                ("cells", ctypes.c_uint32), ("cell_volume", ctypes.c_float),
                ("cross_section", ctypes.c_float), ("fnum", ctypes.c_float),
                ("periodic", ctypes.c_char), ("omega", ctypes.c_float),
                ("vhs_gref", ctypes.c_float)]


class OrcGeom(ctypes.Structure):
    _fields_ = [("bmin", c_f3), ("bmax", c_f3), ("cell", c_f3), ("dim", c_u3),
                ("flags", _P), ("start_end", _P), ("tri_vidx", _P), ("verts", _P),
                ("normals", _P)]


class RefConfig(ctypes.Structure):
    _fields_ = [("gmin", c_f3), ("gmax", c_f3), ("dim", ctypes.c_int * 3),
                ("density", ctypes.c_float), ("fnum", ctypes.c_float), ("temp", ctypes.c_float),
                ("mass", ctypes.c_float), ("diam", ctypes.c_float), ("tref", ctypes.c_float),
                ("periodic", ctypes.c_char)]


def p(a):
    return None if a is None else a.ctypes.data_as(_P)


_orc = None


def ensure_built():
    srcs = [os.path.join(HERE, f) for f in ("dsmc_oracle.c", "fast_oracle.c", "dsmc_oracle.h")]
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < max(
            os.path.getmtime(f) for f in srcs):
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)


def orc():
    """The CPU oracle library (built on demand from dsmc_oracle.c)."""
    global _orc
    if _orc is None:
        ensure_built()
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_taus_int.restype = ctypes.c_uint32
        L.orc_taus_float.restype = ctypes.c_float
        L.orc_build_grid.restype = ctypes.c_long
        L.orc_tri_box_overlap.restype = ctypes.c_int
        L.orc_get_threads.restype = ctypes.c_int
        L.orc_mt_lcg.restype = ctypes.c_uint32
        L.orc_mt_lcg.argtypes = [ctypes.c_uint32]
        L.orc_mt_int.restype = ctypes.c_uint32
        L.orc_mt_float.restype = ctypes.c_float
        L.orc_inject_fast.restype = ctypes.c_uint32
        L.orc_inject_plan.restype = ctypes.c_uint32
        _orc = L
    return _orc


def ref_available():
    return os.path.exists(REF_SO)


_ref = None


def ref():
    """The reference's kernels/dsmc_kernel.cu, built headless for sm_100a."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(REF_SO)
        L = ctypes.CDLL(REF_SO)
        L.ref_build_grid.restype = ctypes.c_long
        _ref = L
    return _ref


MT_REF_SO = os.path.join(HERE, "_ref", "libmt_ref.so")
MT_DAT = os.path.join(HERE, "_ref", "MersenneTwister.dat")


def mt_ref_available():
    return os.path.exists(MT_REF_SO) and os.path.exists(MT_DAT)


class MtStruct(ctypes.Structure):
    """mt_struct of the reference's include/dci.h (the CPU twister)."""
    _fields_ = [("aaa", ctypes.c_uint32), ("mm", ctypes.c_int), ("nn", ctypes.c_int),
                ("rr", ctypes.c_int), ("ww", ctypes.c_int), ("wmask", ctypes.c_uint32),
                ("umask", ctypes.c_uint32), ("lmask", ctypes.c_uint32), ("shift0", ctypes.c_int),
                ("shift1", ctypes.c_int), ("shiftB", ctypes.c_int), ("shiftC", ctypes.c_int),
                ("maskB", ctypes.c_uint32), ("maskC", ctypes.c_uint32), ("i", ctypes.c_int),
                ("state", ctypes.POINTER(ctypes.c_uint32))]


_mt_ref = None


def mt_ref():
    """The reference's twister code built unchanged (src/genmtrand.c and the
    host function lcg_rand of kernels/mtwister.cu)."""
    global _mt_ref
    if _mt_ref is None:
        if not os.path.exists(MT_REF_SO):
            raise FileNotFoundError(MT_REF_SO)
        L = ctypes.CDLL(MT_REF_SO)
        L.genrand_mt.restype = ctypes.c_uint32
        L.genrand_mt.argtypes = [ctypes.POINTER(MtStruct)]
        L.sgenrand_mt.restype = None
        L.sgenrand_mt.argtypes = [ctypes.c_uint32, ctypes.POINTER(MtStruct)]
        lcg = getattr(L, "_Z8lcg_randm")  # unsigned long lcg_rand(unsigned long)
        lcg.restype = ctypes.c_ulong
        lcg.argtypes = [ctypes.c_ulong]
        L.lcg_rand = lcg
        _mt_ref = L
    return _mt_ref


def mt_records(path=MT_DAT):
    """The twister records of data/MersenneTwister.dat, (count, 4) uint32:
    matrix_a, mask_b, mask_c, seed (include/MersenneTwister.h:22-27)."""
    return np.fromfile(path, dtype=np.uint32).reshape(-1, 4)


def mt_draws(cfg, count):
    """`count` draws of one twister through the oracle (InitTwisterFast, then
    GetRandomIntegerFast); cfg holds its 4 parameter words."""
    L = orc()
    cfg = np.ascontiguousarray(cfg, dtype=np.uint32)
    st = np.zeros(21, np.uint32)
    L.orc_mt_init(p(cfg), p(st))
    out = np.empty(count, np.uint32)
    for k in range(count):
        out[k] = L.orc_mt_int(p(st), p(cfg))
    return out, st


def sim_from(cfg_grid_min, cfg_grid_max, dim, fnum, cross_section, periodic="n", omega=0.5,
             vhs_gref=0.0):
    """orc_sim with the reference's FP32 derivations (cell size, volume)."""
    s = OrcSim()
    s.gmin[:] = [float(x) for x in cfg_grid_min]
    s.gmax[:] = [float(x) for x in cfg_grid_max]
    cell = [np.float32(np.float32(cfg_grid_max[k]) - np.float32(cfg_grid_min[k])) / np.float32(dim[k])
            for k in range(3)]
    cell = [np.float32(c) for c in cell]
    s.cell[:] = [float(c) for c in cell]
    s.dim[:] = [int(d) for d in dim]
    s.cells = int(dim[0]) * int(dim[1]) * int(dim[2])
    s.cell_volume = float(np.float32(np.float32(cell[0] * cell[1]) * cell[2]))
    s.cross_section = float(cross_section)
    s.fnum = float(fnum)
    s.periodic = periodic.encode() if isinstance(periodic, str) else periodic
    s.omega = omega
    s.vhs_gref = vhs_gref
    return s


def cross_section_of(diam):
    pi = np.float32(3.14159265358979)
    return float(np.float32(np.float32(pi * np.float32(diam)) * np.float32(diam)))


def max_rel_vel_of(diam, temp):
    pi = np.float32(3.14159265358979)
    d = np.float32(diam)
    r = np.float32(np.float32(d * d) * pi)
    r = np.float32(r * np.sqrt(np.float32(temp / 300.0), dtype=np.float32))
    return float(np.float32(r * np.float32(300)))


def taus_int(state):
    s = np.ascontiguousarray(state, np.uint32)
    r = orc().orc_taus_int(p(s))
    state[:] = s
    return r


def philox(ctr, key):
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    o = np.zeros(4, np.uint32)
    orc().orc_philox4x32_10(p(c), p(k), p(o))
    return o


def cell_ids(sim, pos4):
    n = pos4.shape[0]
    keys = np.zeros(n, np.uint32)
    idx = np.zeros(n, np.uint32)
    orc().orc_cell_ids(ctypes.byref(sim), p(np.ascontiguousarray(pos4, np.float32)), n, p(keys), p(idx))
    return keys, idx


def sort(keys, vals, nkeys):
    k = np.ascontiguousarray(keys, np.uint32).copy()
    v = np.ascontiguousarray(vals, np.uint32).copy()
    orc().orc_sort(p(k), p(v), len(k), nkeys)
    return k, v


def bounds_reorder(sim, keys, idx, opos4, ovel4):
    n = len(keys)
    cse = np.zeros((sim.cells, 2), np.uint32)
    sp = np.zeros((n, 4), np.float32)
    sv = np.zeros((n, 4), np.float32)
    orc().orc_bounds_reorder(ctypes.byref(sim), n, p(keys), p(idx), p(opos4), p(ovel4), p(sp), p(sv), p(cse))
    return cse, sp, sv


def collide(sim, vel4, cse, maxrem, stat4, seeds, avg_conc, dt):
    """In place on vel4, maxrem, stat4, seeds (numpy arrays)."""
    orc().orc_collide(ctypes.byref(sim), p(vel4), p(cse), p(maxrem), p(stat4), p(seeds),
                      ctypes.c_float(avg_conc), ctypes.c_float(dt))


def collide_mt(sim, vel4, cse, maxrem, stat4, mt_state, mt_cfg, avg_conc, dt):
    """The -mt collisions (ComputeBirdCollisionsDev), in place on vel4,
    maxrem, stat4 and mt_state ((cells, 21) uint32); mt_cfg is (cells, 4)."""
    orc().orc_collide_mt(ctypes.byref(sim), p(vel4), p(cse), p(maxrem), p(stat4), p(mt_state),
                         p(np.ascontiguousarray(mt_cfg, np.uint32)), ctypes.c_float(avg_conc),
                         ctypes.c_float(dt))


def mt_states(mt_cfg):
    """InitTwisterFast for every twister of mt_cfg ((count, 4) uint32)."""
    cfg = np.ascontiguousarray(mt_cfg, np.uint32)
    st = np.zeros((cfg.shape[0], 21), np.uint32)
    L = orc()
    for k in range(cfg.shape[0]):
        L.orc_mt_init(p(cfg[k]), p(st[k]))
    return st


def geom_from(bbox, cell, dim, count, tri_ids, flags, verts, tris, normals):
    """orc_geom for a binned mesh; keeps the backing arrays alive on the object."""
    g = OrcGeom()
    g.bmin[:] = [float(x) for x in bbox[:3]]
    g.bmax[:] = [float(x) for x in bbox[3:]]
    g.cell[:] = [float(x) for x in cell]
    g.dim[:] = [int(x) for x in dim]
    ncell = int(dim[0]) * int(dim[1]) * int(dim[2])
    se = np.full((ncell, 2), 0xFFFFFFFF, np.uint32)
    off = 0
    for c in range(ncell):
        if count[c]:
            se[c] = (off, off + count[c])
        off += int(count[c])
    tris = np.asarray(tris, np.uint32).reshape(-1, 3)
    tv = np.ascontiguousarray(tris[np.asarray(tri_ids, np.int64)], np.uint32)
    nm = np.ascontiguousarray(np.asarray(normals, np.float32).reshape(-1, 3)[np.asarray(tri_ids, np.int64)])
    fl = np.ascontiguousarray(flags, np.uint32)
    vv = np.ascontiguousarray(verts, np.float32)
    g._keep = (se, tv, nm, fl, vv)
    g.flags, g.start_end, g.tri_vidx, g.verts, g.normals = p(fl), p(se), p(tv), p(vv), p(nm)
    return g


def move(sim, geom, pos4, vel4, dt):
    orc().orc_move(ctypes.byref(sim), None if geom is None else ctypes.byref(geom), p(pos4), p(vel4),
                   pos4.shape[0], ctypes.c_float(dt))


def sample_f64(sim, vel4, cse):
    acc = np.zeros((sim.cells, 5), np.float64)
    orc().orc_sample_f64(ctypes.byref(sim), p(vel4), p(cse), p(acc))
    return acc


def sample_f32(sim, vel4, cse, cs7=None):
    if cs7 is None:
        cs7 = np.zeros((sim.cells, 7), np.float32)
    orc().orc_sample(ctypes.byref(sim), p(vel4), p(cse), p(cs7))
    return cs7


def step(sim, geom, pos4, vel4, dt, avg_conc, maxrem, stat4, seeds, collide=True, sample=False,
         cs7=None):
    """One reference timestep.  Returns the new (pos4, vel4, cse)."""
    n = pos4.shape[0]
    npos = np.zeros_like(pos4)
    nvel = np.zeros_like(vel4)
    keys = np.zeros(n, np.uint32)
    idx = np.zeros(n, np.uint32)
    cse = np.zeros((sim.cells, 2), np.uint32)
    if cs7 is None:
        cs7 = np.zeros((sim.cells, 7), np.float32)
    orc().orc_step(ctypes.byref(sim), None if geom is None else ctypes.byref(geom), p(npos), p(pos4),
                   p(nvel), p(vel4), p(keys), p(idx), p(cse), n, ctypes.c_float(dt),
                   ctypes.c_float(avg_conc), p(maxrem), p(stat4), p(seeds), int(collide), int(sample),
                   p(cs7))
    return npos, nvel, cse


def build_grid(verts, tris, dim, use_ref=False):
    """Geometry grid from the oracle (or the reference's own host code)."""
    v = np.ascontiguousarray(verts, np.float32).reshape(-1)
    t = np.ascontiguousarray(tris, np.uint32).reshape(-1)
    d = np.ascontiguousarray(dim, np.int32)
    ncell = int(d[0]) * int(d[1]) * int(d[2])
    bbox = np.zeros(6, np.float32)
    cell = np.zeros(3, np.float32)
    count = np.zeros(ncell, np.uint32)
    flags = np.zeros(ncell, np.uint8)
    cap = len(t) // 3 * 64 + 1024
    ids = np.zeros(cap, np.uint32)
    fn = ref().ref_build_grid if use_ref else orc().orc_build_grid
    total = fn(p(v), len(v) // 3, p(t), len(t) // 3, p(d), p(bbox), p(cell), p(count), p(ids),
               ctypes.c_long(cap), p(flags))
    assert total <= cap
    return bbox, cell, count, ids[:total].copy(), flags


def set_threads(n):
    orc().orc_set_threads(int(n))


def threads():
    return orc().orc_get_threads()


# ---------------------------------------------------------------------------
# The extension mode (fast_oracle.c): Philox streams, VHS, warp-collided dense
# cells, nearest wall crossings with diffuse walls, per-face boundaries and
# inflow.  No counterpart in the reference.

DEAD = 0xFFFFFFFF


class OrcFast(ctypes.Structure):
    _fields_ = [("key", ctypes.c_uint32 * 2), ("step", ctypes.c_uint32),
                ("ntc_coef", ctypes.c_float), ("avg_conc", ctypes.c_float),
                ("ntc_local", ctypes.c_int), ("hard_sphere", ctypes.c_int),
                ("cross_section", ctypes.c_float), ("vhs_k", ctypes.c_float),
                ("vhs_c1", ctypes.c_float), ("heavy_min", ctypes.c_uint32),
                ("warp_cap", ctypes.c_uint32), ("tie_rel", ctypes.c_float)]


class OrcFastMove(ctypes.Structure):
    _fields_ = [("gmin", c_f3), ("gmax", c_f3), ("cell", c_f3), ("dim", c_u3),
                ("face_kind", ctypes.c_int * 6), ("face_vstd", ctypes.c_float * 6),
                ("dt", ctypes.c_float), ("key", ctypes.c_uint32 * 2), ("step", ctypes.c_uint32),
                ("ntris", ctypes.c_uint32), ("tri", _P), ("plane", _P),
                ("wall_diffuse", ctypes.c_int), ("wall_vstd", ctypes.c_float),
                ("amb_rel", ctypes.c_float)]


class OrcInflow(ctypes.Structure):
    _fields_ = [("face", ctypes.c_int), ("number_flux", ctypes.c_float), ("area", ctypes.c_float),
                ("stream", c_f3), ("vstd", ctypes.c_float)]


def seed_words(seed):
    return [int(seed) & 0xFFFFFFFF, (int(seed) >> 32) & 0xFFFFFFFF]


def vhs_fast_coeffs(cross_section, omega, gref):
    """(vhs_k, vhs_c1) of sigma g = vhs_k 2^(vhs_c1 log2 g), from double."""
    e = 2.0 * float(np.float32(omega)) - 1.0
    return (float(np.float32(float(cross_section) * float(gref) ** e)), float(np.float32(1.0 - e)))


def fast_params(seed, step, fnum, dt, cell_volume, cross_section, omega=0.5, vhs_gref=0.0,
                avg_conc=0.0, ntc_local=1, heavy_min=8, warp_cap=128, tie_rel=4e-6):
    f = OrcFast()
    f.key[:] = seed_words(seed)
    f.step = int(step)
    f.ntc_coef = float(np.float32(0.5 * float(np.float32(fnum)) * float(np.float32(dt)) /
                                  float(np.float32(cell_volume))))
    f.avg_conc = float(avg_conc)
    f.ntc_local = int(ntc_local)
    f.hard_sphere = int(abs(float(np.float32(omega)) - 0.5) < 1e-9)
    f.cross_section = float(cross_section)
    if not f.hard_sphere:
        f.vhs_k, f.vhs_c1 = vhs_fast_coeffs(cross_section, omega, vhs_gref)
    f.heavy_min = int(heavy_min)
    f.warp_cap = int(warp_cap)
    f.tie_rel = float(tie_rel)
    return f


def collide_fast(f, u, v, w, start, maxrem):
    """NTC collisions in place on the sorted velocities u, v, w (float32) and
    maxrem ((cells, 2) float32).  Returns (per cell: pairs, collisions, path,
    near ties) and the sum of the colliding pairs' relative speeds."""
    ncells = len(start) - 1
    info = np.zeros((ncells, 4), np.uint32)
    sg = ctypes.c_double(0.0)
    st = np.ascontiguousarray(start, np.uint32)
    orc().orc_collide_fast(ctypes.byref(f), p(u), p(v), p(w), p(st), ncells, p(maxrem), p(info),
                           ctypes.byref(sg))
    return info, sg.value


def tri_planes(tri9):
    t = np.ascontiguousarray(tri9, np.float32).reshape(-1, 9)
    out = np.zeros((t.shape[0], 4), np.float32)
    orc().orc_tri_planes(p(t), t.shape[0], p(out))
    return out


def triangles_of(verts, tris):
    v = np.asarray(verts, np.float32).reshape(-1, 3)
    t = np.asarray(tris, np.int64).reshape(-1, 3)
    return np.ascontiguousarray(v[t].reshape(-1, 9))


def fast_move_params(sim, face_kind, face_vstd, dt, seed, step, tri9=None, wall_diffuse=1,
                     wall_vstd=0.0, amb_rel=1e-5):
    m = OrcFastMove()
    m.gmin[:] = list(sim.gmin)
    m.gmax[:] = list(sim.gmax)
    m.cell[:] = list(sim.cell)
    m.dim[:] = list(sim.dim)
    m.face_kind[:] = [int(k) for k in face_kind]
    m.face_vstd[:] = [float(x) for x in face_vstd]
    m.dt = float(dt)
    m.key[:] = seed_words(seed)
    m.step = int(step)
    m.wall_diffuse = int(wall_diffuse)
    m.wall_vstd = float(wall_vstd)
    m.amb_rel = float(amb_rel)
    if tri9 is not None and len(tri9):
        t = np.ascontiguousarray(tri9, np.float32).reshape(-1, 9)
        pl = tri_planes(t)
        m._keep = (t, pl)
        m.ntris = t.shape[0]
        m.tri, m.plane = p(t), p(pl)
    else:
        m.ntris = 0
    return m


def move_fast(m, st6, gidx0=0):
    """Flights in place on st6 ((6, n) float32, rows x y z u v w).  Returns
    (live, ambiguous) per particle."""
    n = st6.shape[1]
    live = np.zeros(n, np.uint8)
    amb = np.zeros(n, np.uint8)
    rows = [np.ascontiguousarray(st6[k]) for k in range(6)]
    orc().orc_move_fast(ctypes.byref(m), *[p(r) for r in rows], n, int(gidx0), p(live), p(amb))
    for k in range(6):
        st6[k] = rows[k]
    return live.astype(bool), amb.astype(bool)


def inflow_of(face, number_flux, area, stream, vstd):
    i = OrcInflow()
    i.face, i.number_flux, i.area = int(face), float(number_flux), float(area)
    i.stream[:] = [float(x) for x in stream]
    i.vstd = float(vstd)
    return i


def inject_fast(inflow, sim, dt, seed, step, remainder, max_k, tie_rel=1e-5):
    """One step's injection through one face.  Returns ((6, k) state, ambiguous,
    new remainder)."""
    rem = ctypes.c_float(remainder)
    gmin = np.array(list(sim.gmin), np.float32)
    gmax = np.array(list(sim.gmax), np.float32)
    key = np.array(seed_words(seed), np.uint32)
    buf = [np.zeros(max(int(max_k), 1), np.float32) for _ in range(6)]
    amb = np.zeros(max(int(max_k), 1), np.uint8)
    k = orc().orc_inject_fast(ctypes.byref(inflow), p(gmin), p(gmax), ctypes.c_float(dt), p(key),
                              int(step), ctypes.byref(rem), int(max_k), *[p(b) for b in buf],
                              p(amb), ctypes.c_float(tie_rel))
    return np.stack([b[:k] for b in buf]), amb[:k].astype(bool), rem.value


def inject_plan_chain(inflow, dt, steps, remainder=0.0):
    """The injection remainder after `steps` steps from `remainder` (the
    count of each step from k_inject_plan's arithmetic)."""
    rem = ctypes.c_float(remainder)
    ks = []
    for _ in range(int(steps)):
        ks.append(orc().orc_inject_plan(ctypes.byref(inflow), ctypes.c_float(dt), ctypes.byref(rem),
                                        0xFFFFFFFF))
    return rem.value, ks


def library_inflows(settings_cfg):
    """The inflow faces as the library derives them from a configuration
    (number flux of a drifting Maxwellian through each inflow face, in
    simulator particles, evaluated in double and rounded to float)."""
    import math
    c = settings_cfg
    vstd = math.sqrt(1.3806e-23 * float(np.float32(c.temp)) / float(np.float32(c.gas_mass)))
    cmp = math.sqrt(2.0) * vstd
    out = []
    for f in range(6):
        if c.face_kind[f] != 4:
            continue
        ax = f >> 1
        sign = -1.0 if f & 1 else 1.0
        un = sign * float(np.float32(c.stream_vel[ax]))
        s = un / cmp
        flux = float(np.float32(c.density)) * cmp / (2.0 * math.sqrt(math.pi)) * (
            math.exp(-s * s) + math.sqrt(math.pi) * s * (1.0 + math.erf(s)))
        a1, a2 = (ax + 1) % 3, (ax + 2) % 3
        area = (float(np.float32(np.float32(c.grid_max[a1]) - np.float32(c.grid_min[a1]))) *
                float(np.float32(np.float32(c.grid_max[a2]) - np.float32(c.grid_min[a2]))))
        out.append(inflow_of(f, np.float32(flux / float(np.float32(c.fnum))), np.float32(area),
                             [float(np.float32(x)) for x in c.stream_vel], np.float32(vstd)))
    return out


def keys_of(sim, st6, live=None):
    """Cell ids (GetCellID3D) of the positions in st6; DEAD where not live."""
    n = st6.shape[1]
    pos4 = np.zeros((n, 4), np.float32)
    pos4[:, :3] = st6[:3].T
    keys, _ = cell_ids(sim, pos4)
    if live is not None:
        keys = np.where(live, keys, np.uint32(DEAD)).astype(np.uint32)
    return keys


def near_cell_face(sim, st6, rel=1e-5):
    """Particles within rel of a cell size from a cell face (their key may
    flip with a last-bit difference of the position)."""
    pos = st6[:3].astype(np.float64)
    lo = np.array(list(sim.gmin), np.float64)[:, None]
    cs = np.array(list(sim.cell), np.float64)[:, None]
    fr = (pos - lo) / cs
    return np.any(np.abs(fr - np.round(fr)) < rel, axis=0)


def step_fast(f, m, sim, st6, keys, maxrem, inflows=(), inj_rem=None, max_total=None):
    """One timestep of the extension mode, composed from the restated stages
    in the order the library runs them: stable sort by cell (removed
    particles dropped), NTC collisions, flights (gidx = sorted slot), next
    keys, then the inflow faces' particles appended (plan + fill per face).
    Returns a dict with the new state, keys, maxrem, remainders, per-cell info
    and the near-tie / ambiguity masks over the new slots."""
    keys = np.asarray(keys, np.uint32)
    alive = np.nonzero(keys != DEAD)[0]
    order = alive[np.argsort(keys[alive], kind="stable")]
    nk = keys[order]
    counts = np.bincount(nk, minlength=sim.cells)
    start = np.zeros(sim.cells + 1, np.uint32)
    start[1:] = np.cumsum(counts)
    S = np.ascontiguousarray(st6[:, order], np.float32)
    mr = np.ascontiguousarray(maxrem, np.float32).copy()
    u, v, w = (np.ascontiguousarray(S[k]) for k in (3, 4, 5))
    info, sum_g = collide_fast(f, u, v, w, start, mr)
    S[3], S[4], S[5] = u, v, w
    tie_cell = info[:, 3] > 0
    tie_slot = np.repeat(tie_cell, counts)
    live, amb = move_fast(m, S)
    nkeys = keys_of(sim, S, live)
    amb = amb | (live & near_cell_face(sim, S))
    parts, pkeys, pamb = [S], [nkeys], [amb | tie_slot]
    rems = dict(inj_rem or {})
    total = S.shape[1]
    for inflow in inflows:
        cap = (max_total - total) if max_total is not None else 1 << 26
        st, ia, r = inject_fast(inflow, sim, m.dt, f.key[0] | (f.key[1] << 32), f.step,
                                rems.get(inflow.face, 0.0), cap)
        rems[inflow.face] = r
        inside = np.all((st[:3] >= np.array(list(sim.gmin), np.float32)[:, None]) &
                        (st[:3] <= np.array(list(sim.gmax), np.float32)[:, None]), axis=0)
        parts.append(st)
        pkeys.append(keys_of(sim, st, inside))
        pamb.append(ia | near_cell_face(sim, st))
        total += st.shape[1]
    return {"state": np.concatenate(parts, axis=1), "keys": np.concatenate(pkeys),
            "maxrem": mr, "inj_rem": rems, "info": info, "sum_g": sum_g, "start": start,
            "n_alive": int(len(order)), "ambiguous": np.concatenate(pamb), "tie_cell": tie_cell,
            "order": order}
