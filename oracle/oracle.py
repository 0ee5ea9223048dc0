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
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(
            os.path.join(HERE, "dsmc_oracle.c")):
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
