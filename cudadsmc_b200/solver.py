"""Python host interface mirroring the reference's solver API.

Names follow denglide/CudaDsmc: ``settings_t`` (include/sim_settings.h:32-69),
``DSMCSolver`` with Init / SetModel / InitSystemState / RunSimulationStep /
DoBenchmark / DumpStatistics / SampleStatistics (include/dsmc_base.h:40-80)
and ``CreateSolver`` (kernels/dsmc_base.cu:221-233).  Every call goes through
the C ABI of libdsmc_b200.so; errors raise ``DsmcError`` (the reference throws
std::runtime_error).
"""
import ctypes
import sys

import numpy as np

from . import _capi
from ._capi import Config, Info, check, lib

_P = ctypes.c_void_p


def _ptr(a):
    return a.ctypes.data_as(_P) if a is not None else None


class settings_t:
    """Simulation settings: the reference's settings_t plus extensions."""

    def __init__(self):
        self.cfg = Config()
        check(lib().dsmc_config_default(ctypes.byref(self.cfg)), "settings_t")
        self.maxRunTime = -1.0

    def readFromFile(self, path):
        check(lib().dsmc_config_read_xml(str(path).encode(), ctypes.byref(self.cfg)), "readFromFile")
        return self

    def readFromCmdLine(self, argv):
        arr = (ctypes.c_char_p * len(argv))(*[a.encode() for a in argv])
        rf = ctypes.c_float(-1.0)
        check(lib().dsmc_config_from_args(len(argv), arr, ctypes.byref(self.cfg), ctypes.byref(rf)),
              "readFromCmdLine")
        self.maxRunTime = rf.value
        return self

    def set(self, **kw):
        """Sets fields of the underlying dsmc_config (faces by name, e.g.
        face_kind={'-x': 'inflow'})."""
        sides = ["-x", "+x", "-y", "+y", "-z", "+z"]
        for k, v in kw.items():
            if k == "face_kind":
                for side, kind in v.items():
                    self.cfg.face_kind[sides.index(side)] = _capi.FACE[kind]
                self.cfg.face_mode = 1
            elif k == "face_temp":
                for side, t in v.items():
                    self.cfg.face_temp[sides.index(side)] = t
            elif k == "periodic":
                self.cfg.periodic = v.encode() if isinstance(v, str) else v
            elif k == "rng":
                self.cfg.rng = _capi.RNG[v] if isinstance(v, str) else v
            elif k == "init_kind":
                self.cfg.init_kind = _capi.INIT[v] if isinstance(v, str) else v
            elif k in ("grid_min", "grid_max", "grid_dim", "stream_vel"):
                getattr(self.cfg, k)[:] = list(v)
            else:
                setattr(self.cfg, k, v)
        return self

    def getCellsCount(self):
        d = self.cfg.grid_dim
        return int(d[0]) * int(d[1]) * int(d[2])


class DSMCSolver:
    """The GPU solver (GPUDSMCSolver<particles_state_t> in the reference)."""

    def __init__(self):
        self.h = None
        self.settings = None

    def __del__(self):
        self.close()

    def close(self):
        if getattr(self, "h", None):
            if sys.is_finalizing():  # the interpreter is tearing down modules
                return
            lib().dsmc_destroy(self.h)
            self.h = None

    def _check(self, st, where):
        check(st, where, self.h)

    def Init(self, settings):
        self.close()
        self.settings = settings
        h = ctypes.c_void_p()
        check(lib().dsmc_create(ctypes.byref(settings.cfg), ctypes.byref(h)), "Init")
        self.h = h.value
        return self

    def SetModel(self, verts, tris, grid_dim=(5, 5, 20), normals=None):
        v = np.ascontiguousarray(verts, np.float32).reshape(-1)
        t = np.ascontiguousarray(tris, np.uint32).reshape(-1)
        g = np.ascontiguousarray(grid_dim, np.int32)
        n = None if normals is None else np.ascontiguousarray(normals, np.float32).reshape(-1)
        self._check(lib().dsmc_set_mesh(self.h, _ptr(v), len(v) // 3, _ptr(t), len(t) // 3,
                                        _ptr(n), _ptr(g)), "SetModel")

    def InitSystemState(self, stream_vel=None):
        sv = None if stream_vel is None else np.ascontiguousarray(stream_vel, np.float32)
        n = ctypes.c_uint32()
        self._check(lib().dsmc_init_state(self.h, _ptr(sv), ctypes.byref(n)), "InitSystemState")
        return n.value

    def InitFromFields(self, fields):
        """Seeds the particles from per-cell (n, u, v, w, T) fields [cells, 5],
        n averaged over the whole cell volume as Fields() gives it (a cell the
        body cuts receives n V_c / F_N particles outside the body)."""
        f = np.ascontiguousarray(fields, np.float32).reshape(-1, 5)
        if f.shape[0] != self.settings.getCellsCount():
            raise ValueError("fields must hold one (n, u, v, w, T) row per cell")
        n = ctypes.c_uint32()
        self._check(lib().dsmc_init_from_fields(self.h, _ptr(f), ctypes.byref(n)), "InitFromFields")
        return n.value

    def InitFromFieldsTwoStream(self, fields, weight=1.0):
        """InitFromFields with each cell a mixture of the free stream and a
        Maxwellian at the wall temperature that keeps the cell's mean
        velocity and energy (weight in [0, 1] scales the free-stream share)."""
        f = np.ascontiguousarray(fields, np.float32).reshape(-1, 5)
        if f.shape[0] != self.settings.getCellsCount():
            raise ValueError("fields must hold one (n, u, v, w, T) row per cell")
        n = ctypes.c_uint32()
        self._check(lib().dsmc_init_from_fields_two_stream(self.h, _ptr(f), ctypes.c_float(weight),
                                                           ctypes.byref(n)), "InitFromFieldsTwoStream")
        return n.value

    def RunSimulationStep(self, dt, nsteps=1):
        self._check(lib().dsmc_step(self.h, dt, nsteps), "RunSimulationStep")

    def DoBenchmark(self, itn, dt):
        self._check(lib().dsmc_step_graph(self.h, dt, itn), "DoBenchmark")
        self._check(lib().dsmc_sync(self.h), "DoBenchmark")

    def StepGraph(self, dt, nsteps=1):
        self._check(lib().dsmc_step_graph(self.h, dt, nsteps), "StepGraph")

    def SetKernelVariant(self, variant):
        self._check(lib().dsmc_set_kernel_variant(self.h, int(variant)), "SetKernelVariant")

    def KernelVariant(self):
        """(variant, particles per shared-memory chunk) of the cell kernel."""
        v, cap = ctypes.c_int(0), ctypes.c_int(0)
        self._check(lib().dsmc_get_kernel_variant(self.h, ctypes.byref(v), ctypes.byref(cap)),
                    "KernelVariant")
        return v.value, cap.value

    def Autotune(self, dt, steps=10):
        """Times every split cell-kernel variant (4 and up) on real timesteps
        (the run advances by (KernelVariantCount() - 4) * (steps + 2) steps)
        and keeps the fastest; returns (best, ms per step of each variant, 0
        for the fused variants 0-3, which are not timed)."""
        best = ctypes.c_int(0)
        ms = np.zeros(KernelVariantCount(), np.float32)
        self._check(lib().dsmc_autotune(self.h, dt, int(steps), ctypes.byref(best), _ptr(ms)),
                    "Autotune")
        return best.value, [float(x) for x in ms]

    def Sync(self):
        self._check(lib().dsmc_sync(self.h), "Sync")

    def SetStream(self, stream_ptr):
        self._check(lib().dsmc_set_stream(self.h, stream_ptr), "SetStream")

    def Sample(self):
        self._check(lib().dsmc_sample(self.h), "Sample")

    def ResetSamples(self):
        self._check(lib().dsmc_reset_samples(self.h), "ResetSamples")

    def DumpStatistics(self, path):
        self._check(lib().dsmc_dump_statistics(self.h, str(path).encode()), "DumpStatistics")

    def SampleStatistics(self):
        """(per-cell FP64 sums [cells, 5]: N, sum u, sum v, sum w, sum |v|^2;
        totals [selections, collisions, sum g]; number of samples)."""
        cells = self.settings.getCellsCount()
        s = np.zeros((cells, 5), np.float64)
        ns = ctypes.c_uint32()
        self._check(lib().dsmc_read_cell_sums(self.h, _ptr(s), ctypes.byref(ns)), "SampleStatistics")
        return s, self.Totals(), ns.value

    def Fields(self, out=None):
        """Per-cell n, ux, uy, uz, T [cells, 5] from the FP64 samples (into
        `out`, a C-contiguous float64 array of that shape, when given: pinned
        host memory makes the copy faster)."""
        f = out if out is not None else np.zeros((self.settings.getCellsCount(), 5), np.float64)
        if f.dtype != np.float64 or f.size != 5 * self.settings.getCellsCount() or not f.flags.c_contiguous:
            raise ValueError("Fields(out=...) needs a C-contiguous float64 array of cells x 5")
        self._check(lib().dsmc_read_fields(self.h, _ptr(f)), "Fields")
        return f

    def Totals(self):
        t = np.zeros(3, np.float64)
        self._check(lib().dsmc_get_totals(self.h, _ptr(t)), "Totals")
        return t

    def TotalsAsync(self, out_ptr):
        """Enqueues a copy of the running totals (24 bytes: selections and
        collisions as uint64, the sum of relative speeds as float64) into the
        host buffer at out_ptr (pinned memory) without waiting; the values are
        there once the solver's stream has passed this point."""
        self._check(lib().dsmc_totals_async(self.h, ctypes.c_void_p(out_ptr)), "TotalsAsync")

    @staticmethod
    def TotalsFromBytes(buf):
        """(selections, collisions, sum of relative speeds) from the 24 bytes
        TotalsAsync wrote (a uint8 array or anything numpy can view)."""
        b = np.asarray(buf, dtype=np.uint8).reshape(-1)[:24]
        return np.array([float(b[:8].view(np.uint64)[0]), float(b[8:16].view(np.uint64)[0]),
                         float(b[16:24].view(np.float64)[0])])

    def Info(self):
        i = Info()
        self._check(lib().dsmc_get_info(self.h, ctypes.byref(i)), "Info")
        return i

    KERNELS = ("scan", "scatter", "cell", "inject")

    def Profile(self, enable=True):
        """Starts (or stops) per-kernel CUDA-event timing of dsmc_step."""
        self._check(lib().dsmc_profile(self.h, int(enable)), "Profile")

    def ProfileRead(self):
        """{kernel: (total ms, launches)} since Profile(True)."""
        ms = np.zeros(4, np.float64)
        n = np.zeros(4, np.uint32)
        self._check(lib().dsmc_profile_read(self.h, _ptr(ms), _ptr(n)), "ProfileRead")
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(self.KERNELS)}

    KERNEL_SLOTS = ("scan", "scatter", "order", "inject", "flight", "mesh", "sample", "ntc")

    def ProfileOnly(self, kernels):
        """Keeps the open profile window's events to the named kernels."""
        mask = 0
        for k in kernels:
            mask |= 1 << self.KERNEL_SLOTS.index(k)
        self._check(lib().dsmc_profile_mask(self.h, mask), "ProfileOnly")

    def ProfileReadKernels(self):
        """{kernel: (total ms, launches)} since Profile(True), kernel by kernel
        ("order" is the fused cell kernel when a variant below 4 runs)."""
        n = len(self.KERNEL_SLOTS)
        ms = np.zeros(n, np.float64)
        cnt = np.zeros(n, np.uint32)
        self._check(lib().dsmc_profile_read_kernels(self.h, n, _ptr(ms), _ptr(cnt)),
                    "ProfileReadKernels")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(self.KERNEL_SLOTS) if cnt[i]}

    def UploadState(self, pos, vel=None, soa=False):
        """soa=True: pos is a [6, n] float32 array (x,y,z,u,v,w); else pos/vel
        are [n, 4] float4 arrays as the reference's particles_state_t."""
        if soa:
            a = np.ascontiguousarray(pos, np.float32)
            n = a.shape[1]
            self._check(lib().dsmc_upload_state(self.h, _ptr(a), None, n, 1), "UploadState")
        else:
            p = np.ascontiguousarray(pos, np.float32)
            v = np.ascontiguousarray(vel, np.float32)
            self._check(lib().dsmc_upload_state(self.h, _ptr(p), _ptr(v), p.shape[0], 0), "UploadState")

    def DownloadState(self, soa=True):
        n = ctypes.c_uint32(0)
        self._check(lib().dsmc_download_state(self.h, None, None, ctypes.byref(n), 1), "DownloadState")
        cnt = n.value
        if soa:
            a = np.zeros((6, cnt), np.float32)
            n2 = ctypes.c_uint32(cnt)
            self._check(lib().dsmc_download_state(self.h, _ptr(a), None, ctypes.byref(n2), 1),
                        "DownloadState")
            return a
        p = np.zeros((cnt, 4), np.float32)
        v = np.zeros((cnt, 4), np.float32)
        n2 = ctypes.c_uint32(cnt)
        self._check(lib().dsmc_download_state(self.h, _ptr(p), _ptr(v), ctypes.byref(n2), 0),
                    "DownloadState")
        return p, v

    def EntryReach(self):
        """Per geometry-grid entry (tri_ids order), [entries, 2]: the path
        length r and the elevation sine k such that a particle leaving the
        entry's triangle outward along a shorter path, steeper than k,
        crosses no listed triangle (r = 0: none); empty when the table is
        off."""
        ne = ctypes.c_uint64()
        self._check(lib().dsmc_get_entry_reach(self.h, None, 0, ctypes.byref(ne)), "EntryReach")
        out = np.zeros((ne.value, 2), np.float32)
        if ne.value:
            self._check(lib().dsmc_get_entry_reach(self.h, _ptr(out), ne.value, ctypes.byref(ne)),
                        "EntryReach")
        return out

    def CellSlabs(self):
        """Per cell of the geometry grid, [cells, 4]: (m.x, m.y, m.z, e) with
        |m . v - e| <= 1 for every vertex v of the cell's listed triangles
        (zeros: the cell passes every path)."""
        nc = ctypes.c_uint64()
        self._check(lib().dsmc_get_cell_slabs(self.h, None, 0, ctypes.byref(nc)), "CellSlabs")
        out = np.zeros((nc.value, 4), np.float32)
        if nc.value:
            self._check(lib().dsmc_get_cell_slabs(self.h, _ptr(out), nc.value, ctypes.byref(nc)), "CellSlabs")
        return out

    def GeometryGrid(self):
        """The handle's geometry grid (built on the device by SetModel): bbox,
        cell size, dims, per-cell triangle counts, triangle ids in bin order,
        flags, and each entry's plane (unit normal, offset) as the device
        holds it."""
        dim = np.zeros(3, np.int32)
        ne = ctypes.c_uint64()
        self._check(lib().dsmc_get_geometry_grid(self.h, None, None, _ptr(dim), None, None, None, 0,
                                                 None, ctypes.byref(ne)), "get_geometry_grid")
        ncell = int(dim[0]) * int(dim[1]) * int(dim[2])
        bbox = np.zeros(6, np.float32)
        cell = np.zeros(3, np.float32)
        count = np.zeros(ncell, np.uint32)
        flags = np.zeros(ncell, np.uint8)
        ids = np.zeros(max(ne.value, 1), np.uint32)
        planes = np.zeros((max(ne.value, 1), 4), np.float32)
        self._check(lib().dsmc_get_geometry_grid(self.h, _ptr(bbox), _ptr(cell), _ptr(dim), _ptr(count),
                                                 _ptr(ids), _ptr(planes), ne.value, _ptr(flags),
                                                 ctypes.byref(ne)), "get_geometry_grid")
        return bbox, cell, dim, count, ids[: ne.value], flags, planes[: ne.value]

    def ReadKeys(self):
        """Next-step cell key of every particle slot (0xffffffff: left the
        domain), in the order of DownloadState."""
        n = ctypes.c_uint32(0)
        self._check(lib().dsmc_read_keys(self.h, None, ctypes.byref(n)), "ReadKeys")
        k = np.zeros(n.value, np.uint32)
        n2 = ctypes.c_uint32(n.value)
        self._check(lib().dsmc_read_keys(self.h, _ptr(k), ctypes.byref(n2)), "ReadKeys")
        return k

    def SetTwisters(self, cfg4, state21=None, init_maximums=False):
        """The -mt collisions (ComputeBirdCollisionsDev): cfg4 (cells, 4)
        twister records (read_twisters), state21 (cells, 21) twister states or
        None to initialise them from their seeds; init_maximums also sets
        (sigma g)max and draws the remainders from the twisters
        (InitMaximums)."""
        c = np.ascontiguousarray(cfg4, np.uint32)
        st = None if state21 is None else np.ascontiguousarray(state21, np.uint32)
        self._check(lib().dsmc_set_twisters(self.h, _ptr(c), _ptr(st), int(init_maximums)),
                    "SetTwisters")

    def GetTwisters(self):
        st = np.zeros((self.settings.getCellsCount(), 21), np.uint32)
        self._check(lib().dsmc_get_twisters(self.h, _ptr(st)), "GetTwisters")
        return st

    def SetCellState(self, maxrem=None, seeds=None):
        m = None if maxrem is None else np.ascontiguousarray(maxrem, np.float32)
        s = None if seeds is None else np.ascontiguousarray(seeds, np.uint32)
        self._check(lib().dsmc_set_cell_state(self.h, _ptr(m), _ptr(s)), "SetCellState")

    def GetCellState(self):
        cells = self.settings.getCellsCount()
        m = np.zeros((cells, 2), np.float32)
        s = np.zeros((cells, 4), np.uint32)
        self._check(lib().dsmc_get_cell_state(self.h, _ptr(m), _ptr(s)), "GetCellState")
        return m, s

    def Snapshot(self, path):
        self._check(lib().dsmc_snapshot(self.h, str(path).encode()), "Snapshot")

    def Restore(self, path):
        self._check(lib().dsmc_restore(self.h, str(path).encode()), "Restore")


class DSMCBatch:
    """Independent solvers advanced together by one CUDA graph launch per
    timestep (dsmc_batch_*).  The solvers stay owned by the caller; close the
    batch before them."""

    def __init__(self, solvers):
        self.solvers = list(solvers)
        hs = (ctypes.c_void_p * len(self.solvers))(*[s.h for s in self.solvers])
        b = ctypes.c_void_p()
        check(lib().dsmc_batch_create(hs, len(self.solvers), ctypes.byref(b)), "DSMCBatch")
        self.b = b.value

    def __del__(self):
        self.close()

    def close(self):
        if getattr(self, "b", None):
            if sys.is_finalizing():
                return
            lib().dsmc_batch_destroy(self.b)
            self.b = None

    def _check(self, st, where):
        if st != _capi.DSMC_OK:
            detail = lib().dsmc_batch_last_error(self.b)
            raise _capi.DsmcError(st, where, detail.decode() if detail else "")

    def _dt(self, dt):
        if dt is None:
            return None
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, np.float32), (len(self.solvers),)))
        return d

    def SetStream(self, stream):
        self._check(lib().dsmc_batch_set_stream(self.b, ctypes.c_void_p(stream)), "SetStream")

    def Step(self, nsteps=1, dt=None):
        d = self._dt(dt)
        self._check(lib().dsmc_batch_step(self.b, _ptr(d), int(nsteps)), "Step")

    def Sync(self):
        self._check(lib().dsmc_batch_sync(self.b), "Sync")

    def Autotune(self, steps=5, dt=None):
        d = self._dt(dt)
        v = np.zeros(len(self.solvers), np.int32)
        self._check(lib().dsmc_batch_autotune(self.b, _ptr(d), int(steps), _ptr(v)), "Autotune")
        return [int(x) for x in v]


def read_twisters(path, count, seed=999):
    """InitGPUTwisters' host part: the first `count` twister records of a
    parameter file (data/MersenneTwister.dat), seeds from the lcg chain
    started at `seed` (the reference uses SEED = 999).  (count, 4) uint32."""
    cfg = np.zeros((count, 4), np.uint32)
    check(lib().dsmc_read_twisters(str(path).encode(), seed, count, _ptr(cfg)), "read_twisters")
    return cfg


def KernelVariantCount():
    """Number of launch shapes of the cell kernel (dsmc_kernel_variant_count)."""
    return int(lib().dsmc_kernel_variant_count())


def CreateSolver(kind="gpu"):
    """CreateSolver(SolverGPU).  The reference's CPU solver type returns None
    there as well (kernels/dsmc_base.cu:225-226)."""
    return DSMCSolver() if kind in ("gpu", 0) else None


def mesh_icosphere(level, radius, center=(0.0, 0.0, 0.0)):
    c = np.ascontiguousarray(center, np.float32)
    nv, nt = ctypes.c_uint32(), ctypes.c_uint32()
    check(lib().dsmc_mesh_icosphere(level, radius, _ptr(c), None, ctypes.byref(nv), None,
                                    ctypes.byref(nt)), "mesh_icosphere")
    v = np.zeros((nv.value, 3), np.float32)
    t = np.zeros((nt.value, 3), np.uint32)
    check(lib().dsmc_mesh_icosphere(level, radius, _ptr(c), _ptr(v), ctypes.byref(nv), _ptr(t),
                                    ctypes.byref(nt)), "mesh_icosphere")
    return v, t


def mesh_capsule(nose_radius, cone_deg, length, nose_center, ntarget, seed):
    c = np.ascontiguousarray(nose_center, np.float32)
    nv, nt = ctypes.c_uint32(), ctypes.c_uint32()
    args = (nose_radius, cone_deg, length, _ptr(c), ntarget, seed)
    check(lib().dsmc_mesh_capsule(*args, None, ctypes.byref(nv), None, ctypes.byref(nt)), "mesh_capsule")
    v = np.zeros((nv.value, 3), np.float32)
    t = np.zeros((nt.value, 3), np.uint32)
    check(lib().dsmc_mesh_capsule(*args, _ptr(v), ctypes.byref(nv), _ptr(t), ctypes.byref(nt)),
          "mesh_capsule")
    return v, t


def read_raw_mesh(path):
    """Model::LoadRaw (src/model.cpp:348-401): vertices, triangles, face normals."""
    nv, nt = ctypes.c_uint32(), ctypes.c_uint32()
    check(lib().dsmc_read_raw_mesh(str(path).encode(), None, ctypes.byref(nv), None,
                                   ctypes.byref(nt), None), "read_raw_mesh")
    v = np.zeros((nv.value, 3), np.float32)
    t = np.zeros((nt.value, 3), np.uint32)
    n = np.zeros((nt.value, 3), np.float32)
    check(lib().dsmc_read_raw_mesh(str(path).encode(), _ptr(v), ctypes.byref(nv), _ptr(t),
                                   ctypes.byref(nt), _ptr(n)), "read_raw_mesh")
    return v, t, n


def build_geometry_grid(verts, tris, grid_dim):
    """The uniform geometry grid over a mesh (Model::CreateGrid): bbox, cell
    size, per-cell triangle counts, triangle ids in bin order, flags."""
    v = np.ascontiguousarray(verts, np.float32).reshape(-1)
    t = np.ascontiguousarray(tris, np.uint32).reshape(-1)
    g = np.ascontiguousarray(grid_dim, np.int32)
    ncell = int(g[0]) * int(g[1]) * int(g[2])
    bbox = np.zeros(6, np.float32)
    cell = np.zeros(3, np.float32)
    count = np.zeros(ncell, np.uint32)
    flags = np.zeros(ncell, np.uint8)
    ne = ctypes.c_uint64()
    check(lib().dsmc_build_geometry_grid(_ptr(v), len(v) // 3, _ptr(t), len(t) // 3, _ptr(g),
                                         _ptr(bbox), _ptr(cell), _ptr(count), None, 0, _ptr(flags),
                                         ctypes.byref(ne)), "build_geometry_grid")
    ids = np.zeros(max(ne.value, 1), np.uint32)
    check(lib().dsmc_build_geometry_grid(_ptr(v), len(v) // 3, _ptr(t), len(t) // 3, _ptr(g),
                                         _ptr(bbox), _ptr(cell), _ptr(count), _ptr(ids), ne.value,
                                         _ptr(flags), ctypes.byref(ne)), "build_geometry_grid")
    return bbox, cell, count, ids[: ne.value], flags
