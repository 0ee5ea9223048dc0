"""The geometry grid binned on the device (dsmc_set_mesh, dsmc_geomgrid.cu)
against the host builder (dsmc_build_geometry_grid, which the CPU tests pin
to the reference's Model::CreateGrid), and each entry's plane against the
oracle's: bin for bin, entry for entry, bit for bit."""
import numpy as np
import pytest

from cudadsmc_b200 import DSMCSolver, settings_t
from cudadsmc_b200.solver import build_geometry_grid
from oracle import meshes as OM
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _box_mesh(lo, hi):
    """A closed box of 12 large triangles (outward faces)."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], np.float32)
    t = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                  [2, 3, 7], [2, 7, 6], [1, 2, 6], [1, 6, 5], [3, 0, 4], [3, 4, 7]], np.uint32)
    return v, t


def _cases():
    yield "capsule_20k_48x64x64", OM.capsule(0.15, 20.0, 0.26, (0.5, 0.3, 0.3), 20000, 7), (48, 64, 64)
    yield "icosphere3_16", OM.icosphere(3, 0.1, (0.4, 0.3, 0.3)), (16, 16, 16)
    yield "icosphere5_5x5x20", OM.icosphere(5, 0.2, (0.5, 0.5, 0.5)), (5, 5, 20)
    yield "box12_40", _box_mesh((0.2, 0.25, 0.3), (0.7, 0.6, 0.55)), (40, 40, 40)
    yield "box12_7x3x11", _box_mesh((0.0, 0.0, 0.0), (1.0, 0.5, 2.0)), (7, 3, 11)


@pytest.mark.parametrize("name,mesh,dims", list(_cases()), ids=[c[0] for c in _cases()])
def test_device_binning_equals_host_builder(cuda, name, mesh, dims):
    verts, tris = mesh
    verts = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
    tris = np.ascontiguousarray(tris, np.uint32).reshape(-1, 3)
    s = settings_t().set(grid_min=(0, 0, 0), grid_max=(1, 1, 1), grid_dim=(8, 8, 8), density=1e19,
                         fnum=1e15, temp=300.0, gas_mass=6.63e-26, gas_diam=4.17e-10, gas_tref=273.0)
    sol = DSMCSolver().Init(s)
    sol.SetModel(verts, tris, dims)
    bbox, cell, dim, count, ids, flags, planes = sol.GeometryGrid()
    hb, hc, hcount, hids, hflags = build_geometry_grid(verts, tris, dims)
    assert tuple(dim) == tuple(dims)
    assert np.array_equal(bbox, hb) and np.array_equal(cell, hc)
    assert np.array_equal(count, hcount)
    assert np.array_equal(ids, hids)
    assert np.array_equal(flags, hflags)
    assert hids.size > 0 and flags.sum() >= (count > 0).sum()
    # planes in bin order, as the oracle computes them (FP64, rounded once)
    ref = O.tri_planes(O.triangles_of(verts, tris))
    assert np.array_equal(planes, ref[ids])
    sol.close()
