"""Batched stepping: independent solvers of uneven size advanced by one CUDA
graph launch per timestep give exactly what stepping each of them alone
gives."""
import numpy as np
import pytest

from cudadsmc_b200 import DSMCBatch, DSMCSolver, mesh_icosphere, settings_t
from cudadsmc_b200.solver import KernelVariantCount

pytestmark = pytest.mark.gpu

M_AR, D_AR = 6.63e-26, 4.17e-10


def member(i):
    """Four different flows: sizes, RNG modes, walls and a sphere."""
    dims = [(16, 8, 8), (32, 16, 16), (24, 12, 12), (32, 16, 16)][i]
    dens = [1e20, 3e20, 5e19, 1e20][i]
    s = settings_t().set(grid_min=(0, 0, 0), grid_max=(1.2, 0.6, 0.6), grid_dim=dims, density=dens,
                         fnum=dens * (1.2 / dims[0]) * (0.6 / dims[1]) ** 2 / (6 + 3 * i),
                         temp=200.0, stream_vel=(800.0 + 300 * i, 0, 0), gas_mass=M_AR,
                         gas_diam=D_AR, gas_tref=273.0, gas_omega=0.81,
                         rng="taus" if i == 1 else "philox", ntc_local=1, init_kind="maxwell",
                         sample_every=3, seed=100 + i, capacity_factor=1.6, dt=2e-6 * (1 + i),
                         wall_diffuse=1, wall_temp=300.0 + 50 * i, geom_nearest=1,
                         face_kind={"-x": "inflow", "+x": "outflow", "-y": "outflow",
                                    "+y": "outflow", "-z": "outflow", "+z": "outflow"})
    sol = DSMCSolver().Init(s)
    if i in (0, 3):
        v, t = mesh_icosphere(2, 0.1, (0.4, 0.3, 0.3))
        sol.SetModel(v, t, (8, 8, 8))
    sol.InitSystemState()
    return sol


def test_batch_equals_members_stepped_alone(cuda):
    batched = [member(i) for i in range(4)]
    alone = [member(i) for i in range(4)]
    batch = DSMCBatch(batched)
    batch.Step(5)
    batch.Step(2, dt=[3e-6, 1e-6, 2e-6, 4e-6])  # a new dt per member: recaptured graph
    batch.Sync()
    for i, sol in enumerate(alone):
        sol.RunSimulationStep(sol.settings.cfg.dt, 5)
    for sol, dt in zip(alone, [3e-6, 1e-6, 2e-6, 4e-6]):
        sol.RunSimulationStep(dt, 2)
    for a, b in zip(batched, alone):
        b.Sync()
        assert a.Info().step == b.Info().step == 7
        assert np.array_equal(a.DownloadState(), b.DownloadState())
        ma, sa = a.GetCellState()
        mb, sb = b.GetCellState()
        assert np.array_equal(ma, mb) and np.array_equal(sa, sb)
        ta, tb = a.Totals(), b.Totals()
        assert ta[0] == tb[0] and ta[1] == tb[1]  # selections, collisions
        assert np.array_equal(a.Fields(), b.Fields(), equal_nan=True)
    # launch shapes chosen per member; the batch keeps stepping afterwards
    variants = batch.Autotune(steps=1)
    assert len(variants) == 4 and all(0 <= v < KernelVariantCount() for v in variants)
    n0 = [s.Info().step for s in batched]
    batch.Step(3)
    batch.Sync()
    assert [s.Info().step for s in batched] == [n + 3 for n in n0]
    batch.close()
    for s in batched + alone:
        s.close()
