"""The test bodies of the workloads, generated in NumPy: an icosphere and a
sphere-cone capsule, restating the library's dsmc_mesh_icosphere and
dsmc_mesh_capsule (cudadsmc_b200/csrc/dsmc_host.cpp) step for step in double
precision, rounded to float at the end as the library rounds them.  A CPU test
checks that both give the same vertices and triangles.

TEST INFRASTRUCTURE ONLY: used by tests/ and by bench.py's CPU arms, so that
the CPU baseline builds its workload without loading the product library.
Neither body has a counterpart in the reference, which loads its model from
data/ares.raw (kernels/dsmc.cu:394-408).
"""
import math

import numpy as np


def _lround(x):
    """std::lround for the non-negative values used here (halves away from 0)."""
    return int(math.floor(x + 0.5))


def icosphere(level, radius, center):
    """Regular icosahedron, every edge split at its normalised midpoint
    `level` times; outward triangles.  Returns (verts (n, 3) float32,
    tris (m, 3) uint32)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    p = [-1, t, 0, 1, t, 0, -1, -t, 0, 1, -t, 0, 0, -1, t, 0, 1, t,
         0, -1, -t, 0, 1, -t, t, 0, -1, t, 0, 1, -t, 0, -1, -t, 0, 1]
    p = [float(x) for x in p]
    for i in range(0, len(p), 3):
        ln = math.sqrt(p[i] * p[i] + p[i + 1] * p[i + 1] + p[i + 2] * p[i + 2])
        p[i] /= ln
        p[i + 1] /= ln
        p[i + 2] /= ln
    f = [0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4, 11, 10, 2, 10, 7, 6,
         7, 1, 8, 3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8, 3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7,
         9, 8, 1]
    for _ in range(level):
        mid = {}

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key in mid:
                return mid[key]
            x, y, z = p[3 * a] + p[3 * b], p[3 * a + 1] + p[3 * b + 1], p[3 * a + 2] + p[3 * b + 2]
            ln = math.sqrt(x * x + y * y + z * z)
            idx = len(p) // 3
            p.extend([x / ln, y / ln, z / ln])
            mid[key] = idx
            return idx
        g = []
        for i in range(0, len(f), 3):
            a, b, c = f[i], f[i + 1], f[i + 2]
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            g += [a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca]
        f = g
    c = [float(np.float32(x)) for x in center]
    r = float(np.float32(radius))
    pa = np.asarray(p, np.float64).reshape(-1, 3)
    verts = (np.asarray(c)[None, :] + r * pa).astype(np.float32)
    return verts, np.asarray(f, np.uint32).reshape(-1, 3)


def _splitmix64_phase(seed):
    m = (1 << 64) - 1
    z = (int(seed) + 0x9E3779B97F4A7C15) & m
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    z ^= z >> 31
    return (z >> 11) / 9007199254740992.0 * 2 * math.pi


def capsule(nose_radius, cone_deg, length, nose_center, ntarget, seed):
    """Sphere-cone capsule around the +x axis: a spherical nose of radius
    nose_radius facing -x, a cone of half-angle cone_deg tangent to it, a
    flat base `length` behind the nose tip; near-equilateral triangles of
    about ntarget in all, rings of vertices along the profile, the azimuthal
    start drawn from the seed (splitmix64).  Returns (verts, tris)."""
    f32 = lambda x: float(np.float32(x))  # noqa: E731
    rn, theta, ln = f32(nose_radius), f32(cone_deg), f32(length)
    c = [f32(x) for x in nose_center]
    th = theta * math.pi / 180.0
    phi_t = math.pi / 2 - th
    x_tip = f32(c[0] - rn)  # a float difference in the library
    x_t, r_t = c[0] - rn * math.cos(phi_t), rn * math.sin(phi_t)
    x_base = x_tip + ln
    r_base = r_t + (x_base - x_t) * math.tan(th)
    L1 = rn * phi_t
    L2 = math.hypot(x_base - x_t, r_base - r_t)
    L3 = r_base
    area = (2 * math.pi * rn * rn * (1 - math.cos(phi_t)) + math.pi * (r_t + r_base) * L2 +
            math.pi * r_base * r_base)
    h = math.sqrt(4.0 * area / (math.sqrt(3.0) * max(int(ntarget), 64)))
    ds = h * math.sqrt(3.0) / 2
    n1 = max(2, _lround(L1 / ds))
    n2 = max(1, _lround(L2 / ds))
    n3 = max(2, _lround(L3 / ds))
    phase = _splitmix64_phase(seed)
    rx, rr = [], []
    for i in range(1, n1 + 1):
        ph = phi_t * i / n1
        rx.append(c[0] - rn * math.cos(ph))
        rr.append(rn * math.sin(ph))
    for i in range(1, n2 + 1):
        x = x_t + (x_base - x_t) * i / n2
        rx.append(x)
        rr.append(r_t + (x - x_t) * math.tan(th))
    for i in range(1, n3):
        rx.append(x_base)
        rr.append(r_base * (1.0 - i / n3))
    verts = [(x_tip, c[1], c[2])]
    first, count = [], []
    for k in range(len(rx)):
        m = max(3, _lround(2 * math.pi * rr[k] / h))
        first.append(len(verts))
        count.append(m)
        for a in range(m):
            ang = phase + 2 * math.pi * a / m
            verts.append((rx[k], c[1] + rr[k] * math.cos(ang), c[2] + rr[k] * math.sin(ang)))
    tail = len(verts)
    verts.append((x_base, c[1], c[2]))

    def rid(k, a):
        return first[k] + a % count[k]
    tris = []
    for a in range(count[0]):
        tris.append((0, rid(0, a + 1), rid(0, a)))
    for k in range(len(rx) - 1):
        ma, mb = count[k], count[k + 1]
        i = j = 0
        while i < ma or j < mb:
            step_a = j == mb or (i < ma and (i + 1) / ma < (j + 1) / mb)
            if step_a:
                tris.append((rid(k, i), rid(k, i + 1), rid(k + 1, j)))
                i += 1
            else:
                tris.append((rid(k, i), rid(k + 1, j + 1), rid(k + 1, j)))
                j += 1
    last = len(rx) - 1
    for a in range(count[last]):
        tris.append((tail, rid(last, a), rid(last, a + 1)))
    return np.asarray(verts, np.float64).astype(np.float32), np.asarray(tris, np.uint32)
