"""Shared helpers of the parity tests: seeded particle states, layout
conversions and the reference's FP32 derived constants."""
import numpy as np

from oracle import oracle as O


def f32(x):
    return np.float32(x)


def box_case(seed, dim, gmin, gmax, n, vstd=300.0, stream=(0.0, 0.0, 0.0), inside=True):
    """n particles uniform in the box (a margin off the faces) with Gaussian
    velocities: float4 AoS pos/vel as the reference's particles_state_t."""
    rng = np.random.default_rng(seed)
    gmin = np.asarray(gmin, np.float64)
    gmax = np.asarray(gmax, np.float64)
    span = gmax - gmin
    lo = gmin + (1e-3 * span if inside else 0)
    hi = gmax - (1e-3 * span if inside else 0)
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(lo, hi, size=(n, 3))
    pos[:, 3] = 1.0
    vel[:, :3] = rng.normal(0.0, vstd, size=(n, 3)) + np.asarray(stream)
    return pos, vel


def soa_from_aos(pos4, vel4):
    return np.ascontiguousarray(np.concatenate([pos4[:, :3].T, vel4[:, :3].T], 0), np.float32)


def aos_from_soa(a):
    n = a.shape[1]
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 4), np.float32)
    pos[:, :3] = a[:3].T
    pos[:, 3] = 1
    vel[:, :3] = a[3:].T
    return pos, vel


def taus_seeds(seed, cells):
    """HybridTaus seeds as CreateRandomSeedsUint4 forms them
    (kernels/dsmc_kernel.cu:1866-1879): each word >= 128."""
    rng = np.random.default_rng(seed)
    s = rng.integers(0, 2**32, size=(cells, 4), dtype=np.uint64)
    return ((s % (2**32 - 129)) + 128).astype(np.uint32)


def maxrem_init(seed, cells, max_rel_vel):
    rng = np.random.default_rng(seed)
    m = np.zeros((cells, 2), np.float32)
    m[:, 0] = max_rel_vel
    m[:, 1] = rng.uniform(0, 1, cells).astype(np.float32)
    return m


def starts_from_cse(cse, n):
    """Exclusive cell starts (cells+1) from the reference's cellStartEnd."""
    cells = cse.shape[0]
    counts = (cse[:, 1] - cse[:, 0]).astype(np.int64)
    st = np.zeros(cells + 1, np.uint32)
    st[1:] = np.cumsum(counts)
    assert st[-1] == n
    return st


def rel_err(a, b, scale):
    return np.max(np.abs(a.astype(np.float64) - b.astype(np.float64)) / scale)


def sim_for(cfg_min, cfg_max, dim, fnum, diam, periodic="n", omega=0.5, vhs_gref=0.0):
    return O.sim_from(cfg_min, cfg_max, dim, fnum, O.cross_section_of(diam), periodic, omega, vhs_gref)
