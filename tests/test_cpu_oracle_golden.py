"""The CPU oracle pinned to the reference's own outputs.

tests/golden/*.npz hold seeded inputs and the outputs of the reference's
kernels/dsmc_kernel.cu (built unchanged for sm_100a and run on a B200 by
tests/golden/make_golden.py) and of its host geometry code.  Integer outputs
must match bit for bit; FP32 outputs within the tolerances stated per test
(the oracle uses libm cosf/sinf where the reference uses the hardware
__cosf/__sinf intrinsics).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name))


def sim_of(d, periodic="n"):
    return O.sim_from(d["gmin"], d["gmax"], d["dim"], float(d["fnum"]) if "fnum" in d.files else 1e15,
                      float(d["cross_section"]) if "cross_section" in d.files else O.cross_section_of(4.17e-10),
                      periodic)


def test_hybrid_taus_matches_reference():
    d = load("taus.npz")
    for i in range(d["states"].shape[0]):
        s = d["states"][i].copy()
        ints = [O.taus_int(s) for _ in range(16)]
        assert np.array_equal(np.asarray(ints, np.uint32), d["ints"][i])
        fl = []
        for _ in range(16):
            fl.append(O.orc().orc_taus_float(O.p(s)))
        assert np.array_equal(np.asarray(fl, np.float32), d["floats"][i])
        assert np.array_equal(s, d["after"][i])


def test_philox_known_answers():
    # Random123 known-answer vectors of Philox-4x32-10
    assert list(O.philox([0, 0, 0, 0], [0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(O.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)) == [0x408F276D, 0x41C83B0E,
                                                                  0xA20BC7C6, 0x6D5451FD]
    assert list(O.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                         [0xA4093822, 0x299F31D0])) == [0xD16CFE09, 0x94FDCCEB, 0x5001E420,
                                                        0x24126EA1]


def test_cell_ids_and_stable_sort_match_reference():
    d = load("cellids_sort.npz")
    sim = O.sim_from(d["gmin"], d["gmax"], d["dim"], 1e15, O.cross_section_of(4.17e-10))
    keys, idx = O.cell_ids(sim, d["pos"])
    assert np.array_equal(keys, d["keys"])
    k, v = O.sort(keys, idx, sim.cells)
    assert np.array_equal(k, d["sorted_keys"])
    assert np.array_equal(v, d["sorted_idx"])


def test_collide_matches_reference():
    d = load("collide.npz")
    sim = O.sim_from(d["gmin"], d["gmax"], d["dim"], float(d["fnum"]), float(d["cross_section"]))
    assert np.float32(sim.cell_volume) == np.float32(d["cell_volume"])
    vel = d["vel"].copy()
    mr, sd = d["maxrem"].copy(), d["seeds"].copy()
    st4 = np.zeros((sim.cells, 4), np.float32)
    O.collide(sim, vel, d["cse"], mr, st4, sd, float(d["avg_conc"]), float(d["dt"]))
    same = np.all(sd == d["seeds_out"], axis=1)
    assert same.all()  # same RNG consumption: every accept decision agrees
    assert np.array_equal(st4[:, 0], d["stat4"][:, 0])  # selections
    assert np.array_equal(st4[:, 1], d["stat4"][:, 1])  # collisions
    assert np.allclose(st4[:, 2], d["stat4"][:, 2], rtol=1e-6)
    assert np.array_equal(mr[:, 1], d["maxrem_out"][:, 1])  # remainders
    assert np.allclose(mr[:, 0], d["maxrem_out"][:, 0], rtol=1e-6)
    scale = 3 * 400.0
    err = np.max(np.abs(vel[:, :3] - d["vel_out"][:, :3])) / scale
    assert err <= 2e-6, err
    exact = np.mean(np.all(vel[:, :3] == d["vel_out"][:, :3], axis=1))
    assert exact > 0.5  # uncollided particles and many collided ones are bit-identical


@pytest.mark.parametrize("per", ["n", "x", "y", "z"])
def test_move_boundaries_match_reference_bit_exact(per):
    d = load(f"move_{per}.npz")
    sim = O.sim_from(d["gmin"], d["gmax"], d["dim"], 1e15, O.cross_section_of(4.17e-10), per)
    pos, vel = d["pos"].copy(), d["vel"].copy()
    O.move(sim, None, pos, vel, float(d["dt"]))
    assert np.array_equal(pos[:, :3], d["pos_out"][:, :3])
    assert np.array_equal(vel[:, :3], d["vel_out"][:, :3])


def test_move_sphere_matches_reference():
    d = load("move_sphere.npz")
    bbox, cell, count, ids, flags = O.build_grid(d["verts"], d["tris"], d["gdim"])
    for a, b in zip((bbox, cell, count, ids, flags), (d["bbox"], d["cell"], d["count"], d["ids"], d["flags"])):
        assert np.array_equal(a, b)  # the oracle's grid = the reference's grid
    sim = O.sim_from(d["gmin"], d["gmax"], d["dim"], 1e15, O.cross_section_of(4.17e-10))
    geom = O.geom_from(bbox, cell, d["gdim"], count, ids, flags, d["verts"], d["tris"], d["normals"])
    pos, vel = d["pos"].copy(), d["vel"].copy()
    O.move(sim, geom, pos, vel, float(d["dt"]))
    hit_o = np.any(vel[:, :3] != d["vel"][:, :3], axis=1)
    hit_r = np.any(d["vel_out"][:, :3] != d["vel"][:, :3], axis=1)
    assert hit_r.sum() > 500
    assert np.mean(hit_o == hit_r) >= 0.999
    both = hit_o & hit_r
    path = np.linalg.norm(d["vel"][:, :3], axis=1) * float(d["dt"])
    dp = np.max(np.abs(pos[:, :3] - d["pos_out"][:, :3]), axis=1)
    assert np.max(dp[both] / path[both]) < 1e-5
    assert np.max(dp[~hit_o & ~hit_r]) == 0.0  # free flight is bit-exact


def test_three_steps_match_reference():
    d = load("step3.npz")
    sim = O.sim_from(d["gmin"], d["gmax"], d["dim"], float(d["fnum"]), float(d["cross_section"]))
    pos, vel = d["pos"].copy(), d["vel"].copy()
    mr, sd = d["maxrem"].copy(), d["seeds"].copy()
    st4 = np.zeros((sim.cells, 4), np.float32)
    cs7 = np.zeros((sim.cells, 7), np.float32)
    for s in range(3):
        pos, vel, cse = O.step(sim, None, pos, vel, float(d["dt"]), float(d["ppc"]), mr, st4, sd,
                               sample=(s == 2), cs7=cs7)
    assert np.array_equal(cse, d["cse"])  # cell starts/ends of the last sort
    assert np.array_equal(sd, d["seeds_out"])
    assert np.array_equal(st4[:, 0], d["stat4"][:, 0])
    assert np.array_equal(st4[:, 1], d["stat4"][:, 1])
    scale = 3 * 400.0
    assert np.max(np.abs(vel[:, :3] - d["vel_out"][:, :3])) / scale < 5e-6
    assert np.max(np.abs(pos[:, :3] - d["pos_out"][:, :3])) < 1e-6
    assert np.array_equal(cs7[:, 0], d["cell_stats"][:, 0])
    assert np.allclose(cs7[:, 1:5], d["cell_stats"][:, 1:5], rtol=1e-5, atol=1e-2)
