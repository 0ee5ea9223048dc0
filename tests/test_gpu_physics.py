"""Physics checks of the whole timestep (both RNG modes, light and dense
cells): energy conservation, relaxation of a bimodal start to a Maxwellian,
the equilibrium collision rate against kinetic theory, and a free stream held
by the inflow/outflow faces."""
import math

import numpy as np
import pytest

from cudadsmc_b200 import DSMCSolver, settings_t

pytestmark = pytest.mark.gpu

KB = 1.3806e-23
M_AR, D_AR = 6.63e-26, 4.17e-10


def box(ppc_density=1e20, fnum=1e15, rng="philox", omega=0.5, init="maxwell", temp=300.0, t2=0.0,
        dim=(16, 16, 16), **kw):
    s = settings_t().set(grid_min=(0, 0, 0), grid_max=(1, 1, 1), grid_dim=dim, density=ppc_density,
                         fnum=fnum, temp=temp, init_temp2=t2, gas_mass=M_AR, gas_diam=D_AR,
                         gas_tref=273.0, gas_omega=omega, periodic="n", rng=rng, init_kind=init,
                         sample_every=0, seed=17, **kw)
    sol = DSMCSolver().Init(s)
    n = sol.InitSystemState()
    return sol, n


@pytest.mark.parametrize("rng,density", [("taus", 1e20), ("philox", 1e20), ("philox", 8e20)])
def test_energy_conserved(cuda, rng, density):
    sol, n = box(density, rng=rng)
    e0 = np.sum(sol.DownloadState()[3:].astype(np.float64) ** 2)
    sol.RunSimulationStep(4e-5, 40)
    a = sol.DownloadState()
    e1 = np.sum(a[3:].astype(np.float64) ** 2)
    assert a.shape[1] == n
    assert abs(e1 - e0) / e0 < 2e-5
    assert sol.Totals()[1] > n  # every particle collided at least once on average
    sol.close()


@pytest.mark.parametrize("rng", ["taus", "philox"])
def test_bimodal_relaxes_to_maxwellian(cuda, rng):
    # the closed-box relaxation case: argon VHS, 200 K + 600 K halves, 16^3 cells, 100k particles
    sol, n = box(1e20, rng=rng, omega=0.81, init="bimodal", temp=200.0, t2=600.0)
    # n V / F_N = 24.41 per cell: the extension starts fill the fraction too
    assert abs(n - 100000) < 300
    u0 = sol.DownloadState()[3:].astype(np.float64)
    k0 = np.mean(u0 ** 4, axis=1) / np.mean(u0 ** 2, axis=1) ** 2
    assert np.all(k0 > 3.5)  # mixture kurtosis 3.75
    sol.RunSimulationStep(1e-5, 300)
    u = sol.DownloadState()[3:].astype(np.float64)
    T = M_AR * np.mean(np.sum(u ** 2, axis=0)) / (3 * KB)
    assert abs(T - 400.0) < 4.0
    kurt = np.mean(u ** 4, axis=1) / np.mean(u ** 2, axis=1) ** 2
    assert np.all(np.abs(kurt - 3.0) < 0.06), kurt
    sol.close()


@pytest.mark.parametrize("rng,density", [("taus", 1e20), ("philox", 1e20), ("philox", 8e20)])
def test_equilibrium_collision_rate(cuda, rng, density):
    """Hard-sphere collision rate per volume 1/2 n^2 sigma <g>, <g> = 4 sqrt(kT/(pi m))."""
    T = 300.0
    sol, n = box(density, rng=rng, temp=T, ntc_local=1)
    dt, steps = 1e-5, 200
    sol.RunSimulationStep(dt, 20)
    c0 = sol.Totals()[1]
    sol.RunSimulationStep(dt, steps)
    c1 = sol.Totals()[1]
    fnum = 1e15
    vol = 1.0
    dens = n * fnum / vol
    sigma = math.pi * D_AR ** 2
    g = 4 * math.sqrt(KB * T / (math.pi * M_AR))
    expect = 0.5 * dens ** 2 * sigma * g * vol * dt * steps / fnum
    if rng == "taus":
        # the reference draws both partners with rand % N, so a selection picks
        # one particle twice (and cannot collide) with probability 1/N
        # (kernels/dsmc_kernel.cu:945-952); the Philox mode draws distinct pairs
        expect *= 1.0 - 1.0 / sol.Info().part_per_cell
    ratio = (c1 - c0) / expect
    assert abs(ratio - 1.0) < 0.03, ratio
    sol.close()


def test_free_stream_inflow_outflow(cuda):
    """No body: inflow at -x, outflow elsewhere; density and mean velocity of
    the free stream are held."""
    U, T, nd = 1500.0, 200.0, 1e20
    dims = (32, 16, 16)
    s = settings_t().set(grid_min=(0, 0, 0), grid_max=(1.2, 0.6, 0.6), grid_dim=dims, density=nd,
                         fnum=nd * (1.2 / 32) * (0.6 / 16) ** 2 / 10, temp=T, stream_vel=(U, 0, 0),
                         gas_mass=M_AR, gas_diam=D_AR, gas_tref=273.0, gas_omega=0.81, rng="philox",
                         ntc_local=1, init_kind="maxwell", sample_every=10, capacity_factor=1.5,
                         face_kind={"-x": "inflow", "+x": "outflow", "-y": "outflow", "+y": "outflow",
                                    "-z": "outflow", "+z": "outflow"}, seed=3)
    sol = DSMCSolver().Init(s)
    n0 = sol.InitSystemState()
    sol.RunSimulationStep(4e-6, 400)
    sol.ResetSamples()
    sol.RunSimulationStep(4e-6, 400)
    f = sol.Fields()
    info = sol.Info()
    assert info.injected > 0 and info.removed > 0
    # upstream half (lateral outflow has not yet thinned it)
    up = f.reshape(dims[2], dims[1], dims[0], 5)[4:12, 4:12, 2:12]
    assert abs(up[..., 0].mean() / nd - 1) < 0.05
    assert abs(up[..., 1].mean() / U - 1) < 0.02
    assert abs(up[..., 4].mean() / T - 1) < 0.05
    assert 0.7 * n0 < info.num_particles < 1.1 * n0
    sol.close()


@pytest.mark.parametrize("rng", ["taus", "philox"])
def test_run_to_run_deterministic(cuda, rng):
    out = []
    for _ in range(2):
        sol, n = box(8e20, rng=rng)
        sol.StepGraph(2e-5, 10)
        sol.Sync()
        out.append(sol.DownloadState())
        sol.close()
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("graph", [False, True])
def test_inflow_branch_matches_serial_injection(cuda, graph):
    """With the split kernels the inflow injection runs on a side stream
    beside the NTC, flight, mesh and sampling kernels; while the injection is
    profiled it runs in line on the handle's stream.  Both orders compute the
    same steps."""
    U, T, nd = 1500.0, 200.0, 1e20
    dims = (32, 16, 16)
    out = []
    for profiled in (False, True):
        s = settings_t().set(grid_min=(0, 0, 0), grid_max=(1.2, 0.6, 0.6), grid_dim=dims,
                             density=nd, fnum=nd * (1.2 / 32) * (0.6 / 16) ** 2 / 10, temp=T,
                             stream_vel=(U, 0, 0), gas_mass=M_AR, gas_diam=D_AR, gas_tref=273.0,
                             gas_omega=0.81, rng="philox", ntc_local=1, init_kind="maxwell",
                             sample_every=5, capacity_factor=1.5,
                             face_kind={"-x": "inflow", "+x": "outflow", "-y": "outflow",
                                        "+y": "outflow", "-z": "outflow", "+z": "outflow"}, seed=5)
        sol = DSMCSolver().Init(s)
        sol.SetKernelVariant(5)
        sol.InitSystemState()
        if profiled:
            sol.Profile(True)
        if graph:
            sol.StepGraph(4e-6, 60)
        else:
            sol.RunSimulationStep(4e-6, 60)
        if profiled:
            k = sol.ProfileReadKernels()
            assert k["inject"][1] == 60, k["inject"]
        sol.Sync()
        info = sol.Info()
        out.append((sol.DownloadState(), sol.Fields(), info.injected, info.removed,
                    info.num_particles))
        sol.close()
    assert out[0][2] > 0 and out[0][3] > 0
    assert out[0][2:] == out[1][2:]
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1], equal_nan=True)
