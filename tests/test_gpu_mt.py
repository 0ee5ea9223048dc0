"""The -mt collisions (ComputeBirdCollisionsDev, kernels/dsmc_kernel.cu:1002-1089)
on the GPU against the oracle's restatement: one and twelve timesteps of the
closed 16^3 box with a Mersenne Twister per cell, the twisters initialised on
the device from their parameter records (InitTwisterFast)."""
import numpy as np
import pytest

from cudadsmc_b200 import DSMCSolver, settings_t
from oracle import oracle as O

from helpers import box_case, maxrem_init, sim_for

pytestmark = pytest.mark.gpu

GMIN, GMAX, DIM = (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (16, 16, 16)
DIAM, MASS, TEMP = 4.17e-10, 6.63e-26, 300.0


def _oracle_steps(sim, pos, vel, mr, st4, mts, cfg, ppc, dt, steps):
    for _ in range(steps):
        keys, idx = O.cell_ids(sim, pos)
        keys, idx = O.sort(keys, idx, sim.cells)
        cse, sp, sv = O.bounds_reorder(sim, keys, idx, pos, vel)
        O.collide_mt(sim, sv, cse, mr, st4, mts, cfg, float(ppc), dt)
        O.move(sim, None, sp, sv, dt)
        pos, vel = sp, sv
    return pos, vel


@pytest.mark.parametrize("steps", [1, 12])
def test_mt_steps_vs_oracle(cuda, steps):
    s = settings_t().set(grid_min=GMIN, grid_max=GMAX, grid_dim=DIM, density=1e20, fnum=1e15,
                         temp=TEMP, gas_mass=MASS, gas_diam=DIAM, gas_tref=273.0, periodic="n",
                         sample_every=0, rng="taus")
    sol = DSMCSolver().Init(s)
    info = sol.Info()
    n = info.part_per_cell * info.cells
    pos, vel = box_case(505, DIM, GMIN, GMAX, n, vstd=400.0)
    rng = np.random.default_rng(506)
    cfg = rng.integers(0, 2**32, (info.cells, 4), dtype=np.uint64).astype(np.uint32)
    mr = maxrem_init(507, info.cells, info.max_rel_vel)
    sol.UploadState(pos, vel)
    sol.SetCellState(mr, None)
    sol.SetTwisters(cfg)
    assert np.array_equal(sol.GetTwisters(), O.mt_states(cfg))  # InitTwisterFast
    dt = 1e-5
    sol.RunSimulationStep(dt, nsteps=steps)
    pg, vg = sol.DownloadState(soa=False)
    st_g = sol.GetTwisters()
    mr_g, _ = sol.GetCellState()
    sim = sim_for(GMIN, GMAX, DIM, 1e15, DIAM)
    mts = O.mt_states(cfg)
    st4 = np.zeros((sim.cells, 4), np.float32)
    mr_o = mr.copy()
    po, vo = _oracle_steps(sim, pos.copy(), vel.copy(), mr_o, st4, mts, cfg, info.part_per_cell,
                           dt, steps)
    same_cells = np.all(st_g == mts, axis=1).mean()
    same_part = np.all(pg[:, :3] == po[:, :3], axis=1).mean()
    # the collisions drew exactly the same numbers (identical twister states:
    # the same pairs, acceptances and angles); velocities differ in the last
    # bits where the kernels' __cosf/__sinf and the oracle's libm cosf/sinf
    # round apart, each collision by about an ulp, and positions by that
    # times dt
    scale = 3 * 400.0
    dv = np.max(np.abs(vg[:, :3] - vo[:, :3]), axis=1) / scale
    dp = np.max(np.abs(pg[:, :3] - po[:, :3]), axis=1)
    print(f"-mt, {steps} steps: cells with identical twister state {same_cells:.6f}, "
          f"particles with identical position {same_part:.6f}, max velocity error {dv.max():.2e}, "
          f"max position error {dp.max():.2e} m")
    assert same_cells == 1.0
    assert np.mean(dv <= 2e-6 * steps) >= 0.999
    assert np.mean(dp <= 1e-6 + 2e-6 * steps * scale * dt) >= 0.999
    if steps == 1:
        assert dv.max() <= 2e-6
        assert np.array_equal(mr_g[:, 1], mr_o[:, 1])  # remainders
    assert sol.Totals()[1] > 0
    sol.close()


def test_mt_needs_reference_rng_mode(cuda):
    s = settings_t().set(grid_min=GMIN, grid_max=GMAX, grid_dim=DIM, density=1e20, fnum=1e15,
                         temp=TEMP, gas_mass=MASS, gas_diam=DIAM, gas_tref=273.0, rng="philox")
    sol = DSMCSolver().Init(s)
    cells = sol.Info().cells
    from cudadsmc_b200._capi import DsmcError
    with pytest.raises(DsmcError):
        sol.SetTwisters(np.zeros((cells, 4), np.uint32))
    sol.close()


def test_mt_init_maximums_as_the_reference_start(cuda):
    """InitMaximums runs before the twisters are initialised in the reference
    (include/gpu_dsmc.inl:363-367): it draws from zeroed states, so every
    remainder is (0 + 1) / 2^32; the twisters then start from their seeds."""
    s = settings_t().set(grid_min=GMIN, grid_max=GMAX, grid_dim=DIM, density=1e20, fnum=1e15,
                         temp=TEMP, gas_mass=MASS, gas_diam=DIAM, gas_tref=273.0, rng="taus")
    sol = DSMCSolver().Init(s)
    info = sol.Info()
    sol.InitSystemState()
    cfg = np.random.default_rng(9).integers(0, 2**32, (info.cells, 4), dtype=np.uint64).astype(np.uint32)
    sol.SetTwisters(cfg, init_maximums=True)
    mr, _ = sol.GetCellState()
    assert np.all(mr[:, 0] == np.float32(info.max_rel_vel))
    assert np.all(mr[:, 1] == np.float32(1.0) / np.float32(4294967296.0))
    assert np.array_equal(sol.GetTwisters(), O.mt_states(cfg))
    sol.close()
