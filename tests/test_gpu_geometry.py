"""The step's mesh acceleration (extension, nearest-hit mode): the clearance
table that decides which flights are tested against the triangles must never
exceed the true distance to the surface, and full timesteps - whose free
flights skip the mesh on the strength of that table - must keep particles out
of the body with every cell-kernel variant."""
import ctypes

import numpy as np
import pytest
import torch

from cudadsmc_b200 import DSMCSolver, mesh_icosphere, settings_t
from cudadsmc_b200._capi import lib

pytestmark = pytest.mark.gpu

GMIN, GMAX, DIM = (0.0, 0.0, 0.0), (1.0, 0.5, 0.5), (20, 10, 10)
CENTER, RADIUS = (0.5, 0.25, 0.25), 0.1


def point_triangle_distance(q, a, b, c):
    """Distances [P, T] from points q [P, 3] to triangles (a, b, c) [T, 3]
    each (float64): inside the prism over a triangle the distance to its
    plane, otherwise the nearest point of its three edges."""
    q = q[:, None, :]
    ab, bc, ca = b - a, c - b, a - c
    n = np.cross(ab, c - a)
    nn = np.sum(n * n, axis=-1)

    def side(e, p0):
        return np.sum(np.cross(e[None], q - p0[None]) * n[None], axis=-1)

    inside = (side(ab, a) >= 0) & (side(bc, b) >= 0) & (side(ca, c) >= 0)
    plane = np.abs(np.sum((q - a[None]) * n[None], axis=-1)) / np.sqrt(nn)[None]

    def seg(p0, e):
        ee = np.sum(e * e, axis=-1)
        t = np.clip(np.sum((q - p0[None]) * e[None], axis=-1) / ee[None], 0.0, 1.0)
        d = q - (p0[None] + t[..., None] * e[None])
        return np.sqrt(np.sum(d * d, axis=-1))

    edges = np.minimum(seg(a, ab), np.minimum(seg(b, bc), seg(c, ca)))
    return np.where(inside, plane, edges)


def make_solver(grid=(16, 16, 16)):
    s = settings_t().set(grid_min=GMIN, grid_max=GMAX, grid_dim=DIM, density=1e20, fnum=1e15,
                         temp=300.0, gas_mass=6.63e-26, gas_diam=4.17e-10, periodic="n",
                         geom_nearest=1, wall_diffuse=1, wall_temp=300.0, rng="philox",
                         sample_every=0, capacity_factor=2.0)
    solver = DSMCSolver().Init(s)
    verts, tris = mesh_icosphere(3, RADIUS, CENTER)
    solver.SetModel(verts, tris, grid)
    return solver, verts, tris


@pytest.mark.parametrize("grid", [(16, 16, 16), (7, 9, 5)])
def test_clearance_never_exceeds_distance(cuda, grid):
    solver, verts, tris = make_solver(grid)
    rng = np.random.default_rng(11)
    n = 20000
    # points from the surface out to 5 cm, in every direction
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = RADIUS + rng.uniform(0.0, 0.05, n) ** 2 / 0.05
    pts = (np.asarray(CENTER) + d * r[:, None]).astype(np.float32)
    xyz = torch.from_numpy(pts.reshape(-1).copy()).to(cuda)
    out = torch.empty(n, dtype=torch.float32, device=cuda)
    st = lib().dsmc_clearance_at(solver.h, ctypes.c_void_p(xyz.data_ptr()), n,
                                 ctypes.c_void_p(out.data_ptr()), None)
    assert st == 0
    torch.cuda.synchronize()
    clr = out.cpu().numpy()
    v = verts.astype(np.float64)
    a, b, c = v[tris[:, 0]], v[tris[:, 1]], v[tris[:, 2]]
    dist = np.concatenate([point_triangle_distance(pts[i:i + 500].astype(np.float64), a, b, c).min(1)
                           for i in range(0, n, 500)])
    inside_grid = clr >= 0  # -1: outside the mesh's bounding box
    assert inside_grid.sum() > 8000
    # a lower bound everywhere (float32 coordinates: a micron of slack)
    assert np.all(clr[inside_grid] <= dist[inside_grid] + 1e-6), \
        (clr - dist)[inside_grid].max()
    # and a useful one: points 2-5 cm out mostly see a positive clearance
    far = inside_grid & (dist > 0.02)
    assert far.sum() > 1000 and np.mean(clr[far] > 0) > 0.9
    solver.close()


@pytest.mark.parametrize("variant", [0, 4, 5, 7])
def test_full_steps_keep_particles_outside(cuda, variant):
    solver, _, _ = make_solver()
    solver.SetKernelVariant(variant)
    rng = np.random.default_rng(43 + variant)
    n = 30000
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = rng.uniform(0.101, 0.16, n)
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 4), np.float32)
    pos[:, :3] = np.asarray(CENTER) + d * r[:, None]
    pos[:, 3] = 1.0
    vel[:, :3] = -d * rng.uniform(200, 3000, n)[:, None] + rng.normal(0, 300, (n, 3))
    solver.UploadState(pos, vel)
    solver.RunSimulationStep(1e-5, 3)
    solver.Sync()
    pg, vg = solver.DownloadState(soa=False)
    assert pg.shape[0] >= n - 5
    rr = np.linalg.norm(pg[:, :3] - np.asarray(CENTER), axis=1)
    # inscribed radius of the level-3 icosphere is above 0.0995
    assert np.mean(rr < 0.0995) < 2e-4
    if variant >= 4:
        # the split kernels listed the flights that may reach the body
        assert solver.Info().mesh_flights > 0
    solver.close()
