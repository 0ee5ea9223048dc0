"""The oracle's restatement of the reference's Mersenne Twister variant (the
-mt path and the initial fill: kernels/mtwister.cu:40-117) and of its -mt
collisions (ComputeBirdCollisionsDev, kernels/dsmc_kernel.cu:1002-1089).

Pinned against the reference's own code, built unchanged into
oracle/_ref/libmt_ref.so:
- lcg_rand (kernels/mtwister.cu:40-44), the per-twister seed chain of
  InitGPUTwisters;
- sgenrand_mt / genrand_mt (src/genmtrand.c), the same generator written as a
  block update of the 19-word state, where the GPU advances one word per draw.
The collision restatement shares every arithmetic step with the HybridTaus
one, which the golden vectors pin; here it is checked for conservation and
for drawing exactly what the reference's loop draws.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O

needs_mt_ref = pytest.mark.skipif(not O.mt_ref_available(),
                                  reason="oracle/_ref/libmt_ref.so not built (make -C oracle ref)")


def _ref_stream(cfg, count):
    """genrand_mt of src/genmtrand.c with the generator's parameters
    (include/MersenneTwister.h:31-40) and the twister's record."""
    R = O.mt_ref()
    state = (ctypes.c_uint32 * 19)()
    m = O.MtStruct(aaa=int(cfg[0]), mm=9, nn=19, rr=1, ww=32, wmask=0xFFFFFFFF, umask=0xFFFFFFFE,
                   lmask=0x1, shift0=12, shift1=18, shiftB=7, shiftC=15, maskB=int(cfg[1]),
                   maskC=int(cfg[2]), i=0, state=ctypes.cast(state, ctypes.POINTER(ctypes.c_uint32)))
    R.sgenrand_mt(int(cfg[3]), ctypes.byref(m))
    return np.array([R.genrand_mt(ctypes.byref(m)) for _ in range(count)], np.uint32)


@needs_mt_ref
def test_seed_chain_matches_reference_lcg():
    R = O.mt_ref()
    rng = np.random.default_rng(5)
    for x in [0, 1, 999, 4294967290, 4294967295, *rng.integers(0, 2**32, 200).tolist()]:
        assert O.orc().orc_mt_lcg(int(x)) == R.lcg_rand(int(x))
    cfg = np.zeros((300, 4), np.uint32)
    O.orc().orc_mt_seed_chain(999, O.p(cfg), 300)
    want, s = [], 999
    for _ in range(300):
        s = R.lcg_rand(s) & 0xFFFFFFFF  # InitGPUTwisters stores it in an unsigned int
        want.append(s)
    assert np.array_equal(cfg[:, 3], np.array(want, np.uint32))


@needs_mt_ref
@pytest.mark.parametrize("twister", [0, 1, 2, 100, 4095, 65535])
def test_twister_stream_matches_reference_genrand(twister):
    cfg = O.mt_records()[twister].copy()
    chain = np.zeros((twister + 1, 4), np.uint32)
    O.orc().orc_mt_seed_chain(999, O.p(chain), twister + 1)
    cfg[3] = chain[twister, 3]
    got, _ = O.mt_draws(cfg, 400)  # 21 passes over the 19-word ring
    assert np.array_equal(got, _ref_stream(cfg, 400))


@needs_mt_ref
def test_twister_stream_matches_reference_for_any_parameters():
    rng = np.random.default_rng(11)
    for _ in range(20):
        cfg = rng.integers(0, 2**32, 4, dtype=np.uint64).astype(np.uint32)
        got, _ = O.mt_draws(cfg, 100)
        assert np.array_equal(got, _ref_stream(cfg, 100))


def test_float_draw_is_the_reference_float_arithmetic():
    cfg = np.array([0x9908B0DF, 0x9D2C5680, 0xEFC60000, 4357], np.uint32)
    ints, _ = O.mt_draws(cfg, 64)
    st = np.zeros(21, np.uint32)
    L = O.orc()
    L.orc_mt_init(O.p(cfg), O.p(st))
    for u in ints:
        f = L.orc_mt_float(O.p(st), O.p(cfg))
        want = (np.float32(u) + np.float32(1.0)) / np.float32(4294967296.0)
        assert np.float32(f) == want


def _collide_case():
    from helpers import box_case, maxrem_init
    dim, gmin, gmax = (8, 8, 8), (0.0, 0.0, 0.0), (0.2, 0.2, 0.2)
    fnum = 1.5e13
    sim = O.sim_from(gmin, gmax, dim, fnum, O.cross_section_of(4.17e-10))
    ppc = int(np.float32(1e20) * np.float32(sim.cell_volume) / np.float32(fnum))
    n = ppc * sim.cells
    pos, vel = box_case(21, dim, gmin, gmax, n, vstd=400.0)
    keys, idx = O.cell_ids(sim, pos)
    keys, idx = O.sort(keys, idx, sim.cells)
    cse, _, svel = O.bounds_reorder(sim, keys, idx, pos, vel)
    cfg = O.mt_records()[: sim.cells].copy() if O.mt_ref_available() else \
        np.random.default_rng(3).integers(0, 2**32, (sim.cells, 4), dtype=np.uint64).astype(np.uint32)
    O.orc().orc_mt_seed_chain(999, O.p(cfg), sim.cells)
    mr = maxrem_init(22, sim.cells, O.max_rel_vel_of(4.17e-10, 300.0))
    return sim, ppc, svel, cse, cfg, mr


def test_mt_collisions_conserve_and_draw_as_the_reference_loop():
    sim, ppc, vel, cse, cfg, mr = _collide_case()
    st = O.mt_states(cfg)
    st0 = st.copy()
    v0 = vel.copy()
    st4 = np.zeros((sim.cells, 4), np.float32)
    mr_out = mr.copy()
    O.collide_mt(sim, vel, cse, mr_out, st4, st, cfg, float(ppc), 1e-5)
    assert st4[:, 1].sum() > 100  # collisions happened
    counts = (cse[:, 1] - cse[:, 0]).astype(np.int64)
    for c in range(sim.cells):
        a, b = int(cse[c, 0]), int(cse[c, 1])
        if b - a < 2:
            assert np.array_equal(st[c], st0[c])
            continue
        # momentum and energy of the cell, in double, to FP32 rounding
        p0, p1 = v0[a:b, :3].astype(np.float64).sum(0), vel[a:b, :3].astype(np.float64).sum(0)
        e0 = (v0[a:b, :3].astype(np.float64) ** 2).sum()
        e1 = (vel[a:b, :3].astype(np.float64) ** 2).sum()
        assert np.all(np.abs(p1 - p0) <= 1e-5 * np.sqrt(e0))
        assert abs(e1 - e0) <= 2e-6 * e0
        # the loop draws two indices and one acceptance number per pair and
        # two angles per collision: replaying that many draws from the
        # cell's initial state ends in the same state
        ndraw = 3 * int(st4[c, 0]) + 2 * int(st4[c, 1])
        _, st_replay = O.mt_draws(cfg[c], ndraw)
        assert np.array_equal(st_replay, st[c]), c
    assert counts.sum() == vel.shape[0]


def test_mt_collisions_are_deterministic_and_differ_from_taus():
    sim, ppc, vel, cse, cfg, mr = _collide_case()
    outs = []
    for _ in range(2):
        v = vel.copy()
        O.collide_mt(sim, v, cse, mr.copy(), np.zeros((sim.cells, 4), np.float32), O.mt_states(cfg),
                     cfg, float(ppc), 1e-5)
        outs.append(v)
    assert np.array_equal(outs[0], outs[1])
    vt = vel.copy()
    from helpers import taus_seeds
    O.collide(sim, vt, cse, mr.copy(), np.zeros((sim.cells, 4), np.float32),
              taus_seeds(5, sim.cells), float(ppc), 1e-5)
    assert not np.array_equal(vt, outs[0])


def test_init_maximums_draws_one_float_per_cell():
    cfg = np.random.default_rng(9).integers(0, 2**32, (64, 4), dtype=np.uint64).astype(np.uint32)
    st = O.mt_states(cfg)
    mr = np.zeros((64, 2), np.float32)
    O.orc().orc_init_maximums_mt(64, ctypes.c_float(123.0), O.p(st), O.p(cfg), O.p(mr))
    assert np.all(mr[:, 0] == np.float32(123.0))
    for c in range(64):
        u, s1 = O.mt_draws(cfg[c], 1)
        assert mr[c, 1] == (np.float32(u[0]) + np.float32(1.0)) / np.float32(4294967296.0)
        assert np.array_equal(s1, st[c])


GOLDEN_MT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "collide_mt.npz")


@pytest.mark.skipif(not os.path.exists(GOLDEN_MT),
                    reason="collide_mt.npz is made on a GPU by tests/golden/make_golden.py --only collide_mt")
def test_mt_collide_matches_reference_fixture():
    """The reference's own -mt kernel on the collide.npz case: its twister set-up
    (InitGPUTwisters seed chain, InitTwisterFast), and after ComputeBirdCollisionsDev
    the twister states, counts and remainders bit-exact, velocities within 2e-6 of
    the thermal scale (libm cosf/sinf here, __cosf/__sinf there)."""
    d = np.load(GOLDEN_MT)
    cfg = d["mt_cfg"]
    chain = np.zeros((cfg.shape[0], 4), np.uint32)
    O.orc().orc_mt_seed_chain(999, O.p(chain), cfg.shape[0])
    assert np.array_equal(cfg[:, 3], chain[:, 3])
    if O.mt_ref_available():
        assert np.array_equal(cfg[:, :3], O.mt_records()[: cfg.shape[0], :3])
    assert np.array_equal(O.mt_states(cfg), d["mt_state"])
    sim = O.sim_from(d["gmin"], d["gmax"], d["dim"], float(d["fnum"]), float(d["cross_section"]))
    vel = d["vel"].copy()
    mr = d["maxrem"].copy()
    st = d["mt_state"].copy()
    st4 = np.zeros((sim.cells, 4), np.float32)
    O.collide_mt(sim, vel, d["cse"], mr, st4, st, cfg, float(d["avg_conc"]), float(d["dt"]))
    assert np.array_equal(st, d["mt_state_out"])
    assert np.array_equal(st4[:, :2], d["stat4"][:, :2])
    assert np.array_equal(mr[:, 1], d["maxrem_out"][:, 1])
    assert np.allclose(mr[:, 0], d["maxrem_out"][:, 0], rtol=1e-6)
    assert np.max(np.abs(vel[:, :3] - d["vel_out"][:, :3])) / (3 * 400.0) <= 2e-6


@needs_mt_ref
def test_library_reads_twister_records_as_the_reference():
    """dsmc_read_twisters: InitGPUTwisters' host part (records of the file,
    seeds from the lcg chain of SEED = 999)."""
    import cudadsmc_b200 as cb
    cfg = cb.read_twisters(O.MT_DAT, 3000)
    recs = O.mt_records()[:3000]
    assert np.array_equal(cfg[:, :3], recs[:, :3])
    chain = np.zeros((3000, 4), np.uint32)
    O.orc().orc_mt_seed_chain(999, O.p(chain), 3000)
    assert np.array_equal(cfg[:, 3], chain[:, 3])
    with pytest.raises(cb.DsmcError):
        cb.read_twisters(O.MT_DAT, 70000)  # beyond the file's 65,536 records
