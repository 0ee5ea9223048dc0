"""The reference's own GPU step against this library's on the same B200.

The reference's kernels (kernels/dsmc_kernel.cu, built unchanged for sm_100a
into oracle/_ref) run DoBenchmark's loop of RunBenchmarkSimulationStep
(include/gpu_dsmc.inl:220-274): cell ids, Thrust sort, cell bounds and
reorder, NTC collisions with HybridTaus, move, sampling every 100th step.
This library runs the same physics (hard spheres, closed specular box,
HybridTaus parity mode, sampling every 100th step) from its step graph, and
in its Philox mode.  Both start from the same particles and per-cell state and
are timed with CUDA events after warm-up steps.

Cases: the closed 1 m box of 16^3 cells with 24 particles per cell (98,304
particles), and a box of 64x32x32 cells with 8 per cell (524,288 particles),
the largest grid the reference's per-cell random state admits.  The test
requires this library's step to be faster in both; it prints the figures.
"""
import ctypes
import json

import numpy as np
import pytest
import torch

from cudadsmc_b200 import DSMCSolver, settings_t
from oracle import oracle as O

from helpers import box_case, maxrem_init, taus_seeds

pytestmark = pytest.mark.gpu

DIAM, MASS, TEMP = 4.17e-10, 6.63e-26, 300.0
CASES = {
    "box16_98k": ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (16, 16, 16), 1e15),
    "box64x32x32_524k": ((0.0, 0.0, 0.0), (1.2, 0.6, 0.6), (64, 32, 32), 8.2e13),
}
WARMUP, STEPS, DT = 20, 300, 1e-5


def _ours(case, rng, pos, vel, mr, seeds):
    gmin, gmax, dim, fnum = CASES[case]
    s = settings_t().set(grid_min=gmin, grid_max=gmax, grid_dim=dim, density=1e20, fnum=fnum,
                         temp=TEMP, gas_mass=MASS, gas_diam=DIAM, gas_tref=273.0, periodic="n",
                         sample_every=100, rng=rng)
    sol = DSMCSolver().Init(s)
    stream = torch.cuda.current_stream()
    sol.SetStream(stream.cuda_stream)
    sol.UploadState(pos, vel)
    sol.SetCellState(mr, seeds)
    sol.StepGraph(DT, WARMUP)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream.synchronize()
    t0.record(stream)
    sol.StepGraph(DT, STEPS)
    t1.record(stream)
    t1.synchronize()
    ms = t0.elapsed_time(t1)
    n_end = sol.Info().num_particles
    sol.close()
    return ms / STEPS, n_end


def _reference(case, pos, vel, mr, seeds):
    gmin, gmax, dim, fnum = CASES[case]
    R = O.ref()
    cfg = O.RefConfig()
    cfg.gmin[:], cfg.gmax[:], cfg.dim[:] = gmin, gmax, dim
    cfg.density, cfg.fnum, cfg.temp = 1e20, fnum, TEMP
    cfg.mass, cfg.diam, cfg.tref = MASS, DIAM, 273.0
    cfg.periodic = b"n"
    assert R.ref_init(ctypes.byref(cfg)) == 0
    assert R.ref_set_cell_state(O.p(mr), O.p(seeds)) == 0
    n = pos.shape[0]
    dev = torch.device("cuda:0")
    p = [torch.from_numpy(pos.copy()).to(dev), torch.zeros((n, 4), dtype=torch.float32, device=dev)]
    v = [torch.from_numpy(vel.copy()).to(dev), torch.zeros((n, 4), dtype=torch.float32, device=dev)]
    hashes = torch.zeros(n, dtype=torch.int32, device=dev)
    idx = torch.zeros(n, dtype=torch.int32, device=dev)
    cells = dim[0] * dim[1] * dim[2]
    cse = torch.zeros(2 * cells, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    cur = ctypes.c_int(0)
    ms = ctypes.c_float()
    for steps in (WARMUP, STEPS):
        st = R.ref_run_steps(P(p[0]), P(p[1]), P(v[0]), P(v[1]), P(hashes), P(idx), P(cse),
                             ctypes.c_uint32(n), ctypes.c_float(DT), 1, 0, steps, cur.value,
                             ctypes.byref(cur), ctypes.byref(ms))
        assert st == 0
    return ms.value / STEPS


@pytest.mark.skipif(not O.ref_available(), reason="reference kernels (oracle/_ref) not built")
@pytest.mark.parametrize("case", sorted(CASES))
def test_step_faster_than_reference_kernels(cuda, case):
    gmin, gmax, dim, fnum = CASES[case]
    probe = DSMCSolver().Init(settings_t().set(grid_min=gmin, grid_max=gmax, grid_dim=dim,
                                               density=1e20, fnum=fnum, temp=TEMP, gas_mass=MASS,
                                               gas_diam=DIAM, gas_tref=273.0, periodic="n"))
    info = probe.Info()
    probe.close()
    n = info.part_per_cell * info.cells
    pos, vel = box_case(77, dim, gmin, gmax, n, vstd=400.0)
    seeds = taus_seeds(78, info.cells)
    mr = maxrem_init(79, info.cells, info.max_rel_vel)
    ref_ms = _reference(case, pos, vel, mr.copy(), seeds.copy())
    taus_ms, n_taus = _ours(case, "taus", pos, vel, mr.copy(), seeds.copy())
    philox_ms, n_philox = _ours(case, "philox", pos, vel, mr.copy(), seeds.copy())
    assert n_taus == n and n_philox == n  # closed box: no particle is lost
    line = {"case": case, "particles": n, "cells": info.cells, "steps": STEPS,
            "reference_kernels_ms_per_step": ref_ms, "ours_taus_ms_per_step": taus_ms,
            "ours_philox_ms_per_step": philox_ms,
            "reference_pts_per_s": n / (ref_ms * 1e-3), "ours_taus_pts_per_s": n / (taus_ms * 1e-3),
            "ours_philox_pts_per_s": n / (philox_ms * 1e-3),
            "speedup_taus": ref_ms / taus_ms, "speedup_philox": ref_ms / philox_ms}
    print("REF_SPEED " + json.dumps(line))
    assert taus_ms < ref_ms and philox_ms < ref_ms
