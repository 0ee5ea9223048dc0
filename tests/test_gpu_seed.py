"""Initial states: the Maxwellian fill and the field-seeded fill keep
particles out of the body, and the seeded fill follows the given per-cell
density, drift and temperature."""
import math

import numpy as np
import pytest

from cudadsmc_b200 import DSMCSolver, DsmcError, mesh_icosphere, settings_t

pytestmark = pytest.mark.gpu

M_AR, D_AR, KB = 6.63e-26, 4.17e-10, 1.3806e-23
C, R = np.array([0.4, 0.3, 0.3]), 0.1


def solver(seed=3):
    s = settings_t().set(grid_min=(0, 0, 0), grid_max=(1.2, 0.6, 0.6), grid_dim=(32, 16, 16),
                         density=1e20, fnum=1e20 * (1.2 / 32) * (0.6 / 16) ** 2 / 10, temp=200.0,
                         stream_vel=(1000.0, 0, 0), gas_mass=M_AR, gas_diam=D_AR, gas_tref=273.0,
                         gas_omega=0.81, rng="philox", ntc_local=1, init_kind="maxwell", seed=seed,
                         capacity_factor=3.0, wall_diffuse=1, wall_temp=300.0, geom_nearest=1)
    sol = DSMCSolver().Init(s)
    v, t = mesh_icosphere(3, R, tuple(C))
    sol.SetModel(v, t, (16, 16, 16))
    return sol


def test_maxwellian_fill_keeps_out_of_the_body(cuda):
    sol = solver()
    n = sol.InitSystemState()
    a = sol.DownloadState()
    assert a.shape[1] == n
    r = np.linalg.norm(a[:3].T - C, axis=1)
    # the icosphere's facets lie within 1 % of the sphere; redrawn positions
    # leave at most a few particles inside cells the body covers almost fully
    assert np.sum(r < R * 0.99) <= 1e-3 * n
    # a particle reaching a face from inside is removed at that step
    sol.RunSimulationStep(2e-6, 80)
    a = sol.DownloadState()
    r = np.linalg.norm(a[:3].T - C, axis=1)
    assert np.sum(r < R * 0.99) == 0
    sol.close()


def test_field_seeding(cuda):
    sol = solver()
    dims = (32, 16, 16)
    cells = dims[0] * dims[1] * dims[2]
    z, y, x = np.meshgrid(np.arange(dims[2]), np.arange(dims[1]), np.arange(dims[0]), indexing="ij")
    x = x.reshape(-1)
    f = np.zeros((cells, 5), np.float32)
    f[:, 0] = 1e20 * (1 + x / 16.0)                     # density rising along x
    f[:, 1] = 500.0 + 20.0 * x                          # drift along x
    f[:, 4] = 300.0                                     # temperature
    n = sol.InitFromFields(f)
    a = sol.DownloadState()
    assert a.shape[1] == n
    info = sol.Info()
    expect = np.sum(f[:, 0]) * info.cell_volume / sol.settings.cfg.fnum
    assert abs(n / expect - 1) < 0.02  # the covered cells are left out
    r = np.linalg.norm(a[:3].T - C, axis=1)
    assert np.sum(r < R * 0.99) <= 1e-3 * n
    cx = np.minimum((a[0] / (1.2 / 32)).astype(int), 31)
    for col in (2, 16, 29):
        sel = cx == col
        assert abs(a[3, sel].mean() - (500 + 20 * col)) < 30
        T = M_AR * np.var(a[4, sel]) / KB
        assert abs(T / 300 - 1) < 0.1
    # the seeded state steps
    sol.RunSimulationStep(2e-6, 5)
    sol.Sync()
    sol.close()


def test_field_seeding_fills_cut_cells_with_their_count(cuda):
    """n is averaged over the whole cell (the convention of Fields()), so a
    cell the body cuts receives all of its n V_c / F_N particles outside the
    body, and sampled fields seed each cell with the count it had."""
    sol = solver(seed=5)
    dims = (32, 16, 16)
    cells = dims[0] * dims[1] * dims[2]
    h = np.array([1.2 / 32, 0.6 / 16, 0.6 / 16])
    idx = np.arange(cells)
    ijk = np.stack([idx % dims[0], (idx // dims[0]) % dims[1], idx // (dims[0] * dims[1])], 1)
    lo = ijk * h
    near = np.linalg.norm(np.clip(C, lo, lo + h) - C, axis=1)
    # cells partly inside the body with a sub-cell centre (4 x 4 x 4 per
    # cell, where the fill looks for the part outside the body) outside the
    # sphere, and so outside its inscribed icosphere
    g = (np.arange(4) + 0.5) / 4
    sub = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    r_sub = np.linalg.norm(lo[:, None, :] + sub[None] * h - C, axis=2)
    cut = (near < 0.97 * R) & (r_sub.max(axis=1) > 1.001 * R)
    f = np.zeros((cells, 5), np.float32)
    f[:, 0] = 1e20
    f[:, 1] = 1000.0
    f[:, 4] = 200.0
    n = sol.InitFromFields(f)
    a = sol.DownloadState()
    assert a.shape[1] == n
    r = np.linalg.norm(a[:3].T - C, axis=1)
    assert np.sum(r < R * 0.99) <= 1e-3 * n
    cx = np.minimum((a[:3].T / h).astype(np.int64), np.array(dims) - 1)
    per = np.bincount(cx[:, 0] + dims[0] * (cx[:, 1] + dims[1] * cx[:, 2]), minlength=cells)
    per_cell = 1e20 * float(np.prod(h)) / sol.settings.cfg.fnum  # 10
    want = per_cell * np.count_nonzero(cut)
    assert np.count_nonzero(cut) > 80
    # every cell receives n V_c / F_N = 10 (the fractional part of the product
    # is rounding); seeding only the part of each cell outside the body would
    # give about half
    assert abs(per[cut].sum() / want - 1) < 0.06
    # cells away from the body hold the same count
    clear = near > 1.2 * R
    assert abs(per[clear].mean() / per_cell - 1) < 0.01
    sol.close()


def two_stream_share(u, T, U, T_inf, T_w):
    """The free-stream share alpha at which the rest of a cell (mean u, x
    only, temperature T) is a Maxwellian at T_w, by bisection."""
    k = KB / M_AR
    e_inf, e_w, rhs = 3 * k * T_inf + U * U, 3 * k * T_w, 3 * k * T + u * u

    def f(a):
        return a * e_inf + (1 - a) * e_w + (u - a * U) ** 2 / (1 - a) - rhs

    lo, hi = 0.0, 0.98
    assert f(lo) < 0 < f(hi)
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        lo, hi = (lo, mid) if f(mid) > 0 else (mid, hi)
    return 0.5 * (lo + hi)


def test_two_stream_seeding(cuda):
    """Each cell a mixture of the free stream (1000 m/s, 200 K) and a
    Maxwellian at the wall temperature (300 K): the cell's mean velocity and
    temperature are kept, and the share of particles in a box around the
    free stream matches the mixture's; weight 0 is the plain seeding."""
    dims = (32, 16, 16)
    cells = dims[0] * dims[1] * dims[2]
    f = np.zeros((cells, 5), np.float32)
    f[:, 0] = 1e20
    f[:, 1] = 500.0
    f[:, 4] = 1600.0
    sol = solver(seed=7)
    n = sol.InitFromFieldsTwoStream(f, 1.0)
    a = sol.DownloadState().astype(np.float64)
    assert a.shape[1] == n
    r = np.linalg.norm(a[:3].T - C, axis=1)
    assert np.sum(r < R * 0.99) <= 1e-3 * n
    u = a[3:6].mean(axis=1)
    # the two streams lie 2200 m/s apart: the mean of about 80k particles
    # scatters by about 3.5 m/s
    assert abs(u[0] - 500.0) < 15 and abs(u[1]) < 5 and abs(u[2]) < 5
    T = M_AR * a[3:6].var(axis=1).sum() / (3 * KB)
    assert abs(T / 1600.0 - 1) < 0.02
    alpha = two_stream_share(500.0, 1600.0, 1000.0, 200.0, 300.0)
    ub = (500.0 - alpha * 1000.0) / (1 - alpha)
    s_inf, s_w = math.sqrt(KB * 200.0 / M_AR), math.sqrt(KB * 300.0 / M_AR)

    def phi(x):
        return 0.5 * (1 + math.erf(x / math.sqrt(2)))

    box = (np.abs(a[3] - 1000.0) < 2 * s_inf) & (np.abs(a[4]) < 2 * s_inf) & (np.abs(a[5]) < 2 * s_inf)
    p_beam = (phi(2) - phi(-2)) ** 3
    p_body = (phi((1000 + 2 * s_inf - ub) / s_w) - phi((1000 - 2 * s_inf - ub) / s_w)) * \
        (phi(2 * s_inf / s_w) - phi(-2 * s_inf / s_w)) ** 2
    assert abs(box.mean() - (alpha * p_beam + (1 - alpha) * p_body)) < 0.01
    sol.close()
    # weight 0: the plain seeding, particle for particle
    s1, s2 = solver(seed=9), solver(seed=9)
    n1 = s1.InitFromFields(f)
    n2 = s2.InitFromFieldsTwoStream(f, 0.0)
    assert n1 == n2
    assert np.array_equal(s1.DownloadState(), s2.DownloadState())
    with pytest.raises(DsmcError):
        s2.InitFromFieldsTwoStream(f, 1.5)
    s1.close()
    s2.close()
