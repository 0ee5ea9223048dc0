"""The reach table of the nearest-hit traversal (extension): per geometry-grid
entry (r, k), a path length and an elevation sine such that a particle
re-emitted or reflected from the entry's triangle along a shorter path whose
direction makes more than k with the normal crosses no listed triangle, so
the flight ends without a second walk of the grid.  Checked against the
mesh: every triangle that rises above an entry's plane is at least r away
(exact triangle-triangle distances) or rises no faster than k times its
distance from the entry's triangle; the table covers a convex sphere, a
capsule whose rings have different vertex counts, and stops at a crater."""
import numpy as np
import pytest

from cudadsmc_b200 import DSMCSolver, mesh_capsule, mesh_icosphere, settings_t

pytestmark = pytest.mark.gpu

TOL, SLACK = 1e-7, 4e-6  # height allowed above the plane; set-off and rounding of the hit point


def solver_with(verts, tris, grid):
    s = settings_t().set(grid_min=(0, 0, 0), grid_max=(1.0, 0.5, 0.5), grid_dim=(20, 10, 10), density=1e20,
                         fnum=1e15, temp=300.0, gas_mass=6.63e-26, gas_diam=4.17e-10, periodic="n",
                         geom_nearest=1, wall_diffuse=1, wall_temp=300.0, rng="philox", sample_every=0,
                         capacity_factor=2.0)
    sol = DSMCSolver().Init(s)
    sol.SetModel(verts, tris, grid)
    return sol


def seg_seg(p0, p1, q0, q1):
    """Distance between segments p0p1 and q0q1 (arrays [..., 3], float64):
    the closest points of the two lines, clamped to the segments."""
    d1, d2, r = p1 - p0, q1 - q0, p0 - q0
    a = np.sum(d1 * d1, -1)
    e = np.sum(d2 * d2, -1)
    f = np.sum(d2 * r, -1)
    c = np.sum(d1 * r, -1)
    b = np.sum(d1 * d2, -1)
    den = a * e - b * b
    s = np.where(den > 1e-30, np.clip((b * f - c * e) / np.where(den > 1e-30, den, 1.0), 0.0, 1.0), 0.0)
    t = (b * s + f) / e
    a_ = np.where(a > 0.0, a, 1.0)
    s0 = np.where(a > 0.0, np.clip(-c / a_, 0.0, 1.0), 0.0)
    s1 = np.where(a > 0.0, np.clip((b - c) / a_, 0.0, 1.0), 0.0)
    s = np.where(t < 0.0, s0, np.where(t > 1.0, s1, s))
    t = np.clip(t, 0.0, 1.0)
    d = (p0 + d1 * s[..., None]) - (q0 + d2 * t[..., None])
    return np.sqrt(np.sum(d * d, -1))


def point_tri(q, a, b, c):
    """Distance from points q to triangles (a, b, c), elementwise [..., 3]."""
    n = np.cross(b - a, c - a)
    nn = np.sum(n * n, -1)

    def side(p0, p1):
        return np.sum(np.cross(p1 - p0, q - p0) * n, -1)

    inside = (side(a, b) >= 0) & (side(b, c) >= 0) & (side(c, a) >= 0)
    plane = np.abs(np.sum((q - a) * n, -1)) / np.sqrt(nn)
    edges = np.minimum(seg_seg(q, q, a, b), np.minimum(seg_seg(q, q, b, c), seg_seg(q, q, c, a)))
    return np.where(inside, plane, edges)


def tri_tri(T, U):
    """Distance between triangles T [k, 3, 3] and U [k, 3, 3] that do not
    cross: the least of the vertex-face and edge-edge distances."""
    best = np.full(T.shape[0], np.inf)
    for i in range(3):
        best = np.minimum(best, point_tri(T[:, i], U[:, 0], U[:, 1], U[:, 2]))
        best = np.minimum(best, point_tri(U[:, i], T[:, 0], T[:, 1], T[:, 2]))
        for j in range(3):
            best = np.minimum(best, seg_seg(T[:, i], T[:, (i + 1) % 3], U[:, j], U[:, (j + 1) % 3]))
    return best


def points_on(U, m=6):
    """Points of triangles U [k, 3, 3] on a barycentric lattice of step 1/m
    (vertices and edges included): [k, P, 3]."""
    w = np.array([(i, j, m - i - j) for i in range(m + 1) for j in range(m + 1 - i)], np.float64) / m
    return np.einsum("pv,kvc->kpc", w, U)


def check_reach(sol, verts, tris):
    """Checks every entry's (r, k) against the mesh: each triangle that
    rises more than TOL above the entry's plane is either at least r away
    (exact triangle distance) or rises no faster than k times the distance
    from the entry's triangle (at a lattice of its points)."""
    _, cell, _, _, ids, _, _ = sol.GeometryGrid()
    rk = sol.EntryReach()
    assert rk.shape == (len(ids), 2)
    r, k = rk[:, 0].astype(np.float64), rk[:, 1].astype(np.float64)
    v = verts.astype(np.float64)
    tri = v[tris]  # [ntris, 3, 3]
    cap = 0.999 * float(np.min(cell)) - SLACK
    assert np.all(r >= 0.0) and np.all(r <= cap * (1 + 1e-6))
    assert np.all((k >= 0.0) & (k < 0.5) | (r == 0.0))
    T = tri[ids]
    n = np.cross(T[:, 1] - T[:, 0], T[:, 2] - T[:, 0])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    checked = 0
    for s in range(0, len(ids), 256):
        e = np.arange(s, min(s + 256, len(ids)))
        h = np.einsum("ek,tvk->etv", n[e], tri) - np.einsum("ek,ek->e", n[e], T[e, 0])[:, None, None]
        ee, tt = np.nonzero((h.max(axis=2) > TOL) & (r[e][:, None] > 0))
        if not len(ee):
            continue
        E = e[ee]
        far = tri_tri(T[E], tri[tt]) >= r[E]
        # the others: height - TOL <= k * distance at every lattice point
        E2, U = E[~far], tri[tt[~far]]
        if len(E2):
            pts = points_on(U)  # [q, P, 3]
            q, P = pts.shape[:2]
            hp = np.einsum("qpc,qc->qp", pts, n[E2]) - np.einsum("qc,qc->q", n[E2], T[E2, 0])[:, None]
            TT = np.repeat(T[E2], P, axis=0)
            d = point_tri(pts.reshape(-1, 3), TT[:, 0], TT[:, 1], TT[:, 2]).reshape(q, P)
            slack = 1e-12 + 1e-9 * np.abs(hp)
            assert np.all(hp - TOL <= k[E2][:, None] * d + slack), "a triangle rises faster than the slope bound"
        checked += len(E)
    return r, k, cap, checked


def test_reach_covers_a_convex_body(cuda):
    verts, tris = mesh_icosphere(3, 0.1, (0.5, 0.25, 0.25))
    sol = solver_with(verts, tris, (16, 16, 16))
    r, k, cap, _ = check_reach(sol, verts, tris)
    assert np.mean(np.abs(r - cap) <= 1e-6 * cap) > 0.99
    sol.close()


def test_reach_of_a_capsule(cuda):
    verts, tris = mesh_capsule(0.15, 20.0, 0.26, (0.4, 0.25, 0.25), 4000, 7)
    sol = solver_with(verts, tris, (24, 32, 32))
    r, k, cap, checked = check_reach(sol, verts, tris)
    # rings of different vertex counts leave the bands between them slightly
    # concave: those rises are bounded by small slopes
    assert np.mean(r > 0) > 0.99 and checked > 0
    assert np.median(k[r > 0]) < 0.05
    sol.close()


def test_reach_stops_at_a_dent(cuda):
    center = np.array([0.5, 0.25, 0.25])
    verts, tris = mesh_icosphere(3, 0.1, tuple(center))
    v = verts.astype(np.float64) - center
    # push the vertices of a cap of the sphere inward: a crater
    u = v / np.linalg.norm(v, axis=1, keepdims=True)
    w = np.clip((u[:, 0] - 0.8) / 0.2, 0.0, 1.0)
    v *= (1.0 - 0.35 * w)[:, None]
    verts = (v + center).astype(np.float32)
    sol = solver_with(verts, tris, (16, 16, 16))
    r, k, cap, checked = check_reach(sol, verts, tris)
    # the crater's faces see its rim; the far side of the sphere is convex
    _, _, _, _, ids, _, _ = sol.GeometryGrid()
    far = u[tris[ids]][:, :, 0].max(axis=1) < -0.2
    near = w[tris[ids]].min(axis=1) > 0.3
    assert np.all(np.abs(r[far] - cap) <= 1e-6 * cap) and np.all(k[far] == 0.0)
    # inside the crater the rim rises steeply: short or steep paths only
    assert np.mean((r[near] < cap) | (k[near] > 0.1)) > 0.5
    assert checked > 0
    sol.close()


@pytest.mark.parametrize("mesh", ["sphere", "capsule", "crater"])
def test_cell_slabs_hold_their_triangles(cuda, mesh):
    """Every vertex of a cell's listed triangles lies inside the cell's slab
    (|m . v - e| <= 1), and the slabs are thin where the surface is smooth."""
    center = np.array([0.5, 0.25, 0.25])
    if mesh == "capsule":
        verts, tris = mesh_capsule(0.15, 20.0, 0.26, (0.4, 0.25, 0.25), 4000, 7)
        grid = (24, 32, 32)
    else:
        verts, tris = mesh_icosphere(3, 0.1, tuple(center))
        grid = (16, 16, 16)
        if mesh == "crater":
            v = verts.astype(np.float64) - center
            u = v / np.linalg.norm(v, axis=1, keepdims=True)
            v *= (1.0 - 0.35 * np.clip((u[:, 0] - 0.8) / 0.2, 0.0, 1.0))[:, None]
            verts = (v + center).astype(np.float32)
    sol = solver_with(verts, tris, grid)
    _, cell, dim, count, ids, _, _ = sol.GeometryGrid()
    slabs = sol.CellSlabs().astype(np.float64)
    assert slabs.shape == (int(np.prod(dim)), 4)
    start = np.concatenate([np.zeros(1, np.int64), np.cumsum(count.astype(np.int64))])
    v = verts.astype(np.float64)
    used = 0
    for c in np.nonzero(count)[0]:
        m, e = slabs[c, :3], slabs[c, 3]
        if not np.any(m):
            continue
        used += 1
        pts = v[tris[ids[start[c]:start[c + 1]]]].reshape(-1, 3)
        assert np.all(np.abs(pts @ m - e) <= 1.0 + 1e-6), c
    # most cells of a smooth body get a slab, a thin one
    assert used > 0.9 * np.count_nonzero(count)
    thick = 1.0 / np.linalg.norm(slabs[:, :3], axis=1)[np.any(slabs[:, :3], axis=1)]
    assert np.median(thick) < 0.25 * float(np.min(cell))
    sol.close()
