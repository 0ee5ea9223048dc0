"""Stage API on device tensors: the individual stages of one timestep, as the
reference's host wrappers expose them (kernels/dsmc_kernel.cuh:29-78).

Tensors are torch CUDA tensors (torch is used for device memory and streams
only); every stage runs the library's kernels on torch's current stream.
"""
import ctypes

from ._capi import CollideParams, Grid, MoveParams, check, lib, FACE, RNG

_P = ctypes.c_void_p


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def make_grid(gmin, gmax, dim, cell=None):
    """dsmc_grid; cell size defaults to (gmax - gmin) / dim in FP32, as
    settings_t computes it (src/sim_settings.cpp:100-103)."""
    import numpy as np
    g = Grid()
    g.gmin[:] = [float(x) for x in gmin]
    g.gmax[:] = [float(x) for x in gmax]
    g.dim[:] = [int(x) for x in dim]
    if cell is None:
        cell = [float(np.float32(np.float32(gmax[k]) - np.float32(gmin[k])) / np.float32(dim[k]))
                for k in range(3)]
        cell = [float(np.float32(c)) for c in cell]
    g.cell[:] = cell
    return g


def cell_index(grid, x, y, z, keys, idx=None):
    """CalculateCellIDs (kernels/dsmc_kernel.cu:1712-1732)."""
    check(lib().dsmc_stage_cell_index(ctypes.byref(grid), _p(x), _p(y), _p(z), x.numel(),
                                      _p(keys), _p(idx), _stream()), "stage_cell_index")


def sort_workspace_bytes(n, nkeys):
    b = ctypes.c_size_t()
    check(lib().dsmc_stage_sort_workspace(n, nkeys, ctypes.byref(b)), "stage_sort_workspace")
    return b.value


def sort(keys, vals, nkeys, cell_start=None, workspace=None):
    """SortParticlesIndices (kernels/dsmc_kernel.cu:2033-2051): stable sort by key."""
    wb = 0 if workspace is None else workspace.numel() * workspace.element_size()
    check(lib().dsmc_stage_sort(_p(keys), _p(vals), keys.numel(), nkeys, _p(cell_start),
                                _p(workspace), wb, _stream()), "stage_sort")


def sort_static(keys, vals, nkeys, cell_start=None):
    """The stable sort of sort() with the library's static scratch: allocates
    nothing; n <= SORT_STATIC_MAX_N, nkeys <= SORT_STATIC_MAX_KEYS.  Calls that
    may overlap on one device race on the shared scratch."""
    check(lib().dsmc_stage_sort_static(_p(keys), _p(vals), keys.numel(), nkeys, _p(cell_start),
                                       _stream()), "stage_sort_static")


SORT_STATIC_MAX_N = 1048576
SORT_STATIC_MAX_KEYS = 131072


def bounds_reorder(keys, idx, ncells, cse, src=None, dst=None):
    """FindCellBoundaries (kernels/dsmc_kernel.cu:1734-1808).  cse: uint2 per
    cell as an int32 tensor of 2*ncells; src/dst: six float tensors each."""
    s = d = None
    if src is not None:
        s = (ctypes.c_void_p * 6)(*[t.data_ptr() for t in src])
        d = (ctypes.c_void_p * 6)(*[t.data_ptr() for t in dst])
    check(lib().dsmc_stage_bounds_reorder(_p(keys), _p(idx), keys.numel(), ncells, _p(cse),
                                          s, d, _stream()), "stage_bounds_reorder")


def collide_params(ncells, cell_volume, cross_section, fnum, avg_conc, dt, omega=0.5,
                   vhs_gref=0.0, ntc_local=0, rng="taus", seed=0, step=1):
    p = CollideParams()
    p.ncells, p.cell_volume, p.cross_section, p.fnum = ncells, cell_volume, cross_section, fnum
    p.avg_conc, p.dt, p.omega, p.vhs_gref, p.ntc_local = avg_conc, dt, omega, vhs_gref, ntc_local
    p.rng = RNG[rng] if isinstance(rng, str) else rng
    p.seed, p.step = seed, step
    return p


def collide(params, u, v, w, cell_start, maxrem, seeds=None, stat4=None):
    """ComputeBird (kernels/dsmc_kernel.cu:912-1102) on sorted velocities."""
    check(lib().dsmc_stage_collide(ctypes.byref(params), _p(u), _p(v), _p(w), _p(cell_start),
                                   _p(maxrem), _p(seeds), _p(stat4), _stream()), "stage_collide")


def move_params(grid, dt, periodic="n", faces=None, face_vstd=None, seed=0, step=1):
    p = MoveParams()
    p.grid = grid
    p.dt = dt
    p.periodic = periodic.encode() if isinstance(periodic, str) else periodic
    if faces:
        p.face_mode = 1
        sides = ["-x", "+x", "-y", "+y", "-z", "+z"]
        for s, k in faces.items():
            p.face_kind[sides.index(s)] = FACE[k]
        if face_vstd:
            for s, v in face_vstd.items():
                p.face_vstd[sides.index(s)] = v
    p.seed, p.step = seed, step
    return p


def move(params, x, y, z, u, v, w, solver=None):
    """IntegrateAndProcessCollisions / Integrate (kernels/dsmc_kernel.cu:1659-1699);
    mesh collisions use the solver's geometry when a solver is given."""
    h = None if solver is None else ctypes.c_void_p(solver.h)
    check(lib().dsmc_stage_move(h, ctypes.byref(params), _p(x), _p(y), _p(z), _p(u), _p(v), _p(w),
                                x.numel(), _stream()), "stage_move")


def sample(u, v, w, cell_start, ncells, sums5):
    """SampleCellStatistics (kernels/dsmc_kernel.cu:856-910), FP64 sums."""
    check(lib().dsmc_stage_sample(_p(u), _p(v), _p(w), _p(cell_start), ncells, _p(sums5),
                                  _stream()), "stage_sample")
