"""Host-side checks of the C ABI that need no GPU: every declared entry point
is exported and bound, the reference's configuration formats and defaults,
meshes, the geometry grid against the reference's own binning, and the
multi-process reduction of the benchmark (gloo, two ranks)."""
import ctypes
import os
import re

import numpy as np
import pytest

import cudadsmc_b200 as cb
from cudadsmc_b200 import _capi
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# the reference checkout, when the environment names one (tests that read it skip otherwise)
REF = os.environ.get("DSMC_REFERENCE_DIR", "")


def declared_functions():
    text = open(os.path.join(ROOT, "include", "dsmc_b200.h")).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(dsmc_\w+)\(", text, re.M)))


def test_every_declared_symbol_is_exported_and_bound():
    names = declared_functions()
    assert len(names) >= 35
    lib = ctypes.CDLL(_capi.LIB_PATH)
    bound = {s[0] for s in _capi.SIGNATURES}
    for n in names:
        assert hasattr(lib, n), n
        assert n in bound, n


def test_status_strings():
    L = cb.lib()
    assert L.dsmc_status_string(0) == b"ok"
    assert b"capacity" in L.dsmc_status_string(6)


def test_defaults_are_the_reference_settings():
    s = cb.settings_t()
    c = s.cfg
    # settings_t::settings_t, src/sim_settings.cpp:35-44 with include/dsmc.h
    assert list(c.grid_max) == pytest.approx([0.3, 0.18, 0.18])
    assert list(c.grid_dim) == [30, 18, 18]
    assert c.density == pytest.approx(1e20) and c.fnum == pytest.approx(0.2e14)
    assert c.temp == 300.0 and c.periodic == b"n"
    assert c.gas_mass == pytest.approx(5e-26) and c.gas_diam == pytest.approx(3.5e-10)
    assert c.gas_omega == 0.5 and c.sample_every == 100 and c.seed == 999


def write_config(tmp_path, extra=""):
    (tmp_path / "gases.xml").write_text(
        "<gases>\n<gas name=\"argon\"><mass>6.63e-26</mass><diam>4.17e-10</diam><temp>273</temp>"
        "<omega>0.81</omega></gas>\n</gases>\n")
    cfg = tmp_path / "cfg.xml"
    cfg.write_text(f"""<?xml version="1.0"?>
<config>
  <!-- a box -->
  <grid><min>0 0 0</min><max>1.2 0.6 0.6</max><dim>64 32 32</dim></grid>
  <density>1e20</density>
  <fnum>1.5e13</fnum>
  <temp>200</temp>
  <streamvel>1500 0 0</streamvel>
  <periodic>x</periodic>
  <gas file="gases.xml">argon</gas>
  {extra}
</config>
""")
    return cfg


def test_read_xml_config(tmp_path):
    cfg = write_config(tmp_path, extra='<wall kind="diffuse" T="300" hit="nearest"/>'
                                       '<face side="-x" kind="inflow"/><face side="+x" kind="outflow"/>'
                                       '<rng>philox</rng><seed>42</seed><sample every="25"/>')
    s = cb.settings_t().readFromFile(cfg)
    c = s.cfg
    assert list(c.grid_dim) == [64, 32, 32]
    assert list(c.grid_max) == pytest.approx([1.2, 0.6, 0.6])
    assert c.fnum == pytest.approx(1.5e13) and c.temp == 200.0
    assert list(c.stream_vel) == pytest.approx([1500, 0, 0])
    assert c.periodic == b"x"
    assert c.gas_mass == pytest.approx(6.63e-26) and c.gas_omega == pytest.approx(0.81)
    assert c.wall_diffuse == 1 and c.wall_temp == 300.0 and c.geom_nearest == 1
    assert c.face_mode == 1 and c.face_kind[0] == 4 and c.face_kind[1] == 2
    assert c.rng == 1 and c.seed == 42 and c.sample_every == 25


def test_config_errors(tmp_path):
    with pytest.raises(cb.DsmcError) as e:
        cb.settings_t().readFromFile(tmp_path / "missing.xml")
    assert e.value.status == 7
    bad = tmp_path / "bad.xml"
    bad.write_text("<config><grid><min>0 0 0</min></grid>")
    with pytest.raises(cb.DsmcError) as e:
        cb.settings_t().readFromFile(bad)
    assert e.value.status == 2
    cfg = write_config(tmp_path, extra='<face side="-q" kind="inflow"/>')
    with pytest.raises(cb.DsmcError):
        cb.settings_t().readFromFile(cfg)


def test_command_line(tmp_path):
    cfg = write_config(tmp_path)
    s = cb.settings_t().readFromCmdLine(["prog", "-f", str(cfg), "-benchmark", "-dt", "2.5e-6",
                                         "-density", "3e20", "-run-for", "0.01", "-no-geometry"])
    assert s.cfg.dt == pytest.approx(2.5e-6) and s.cfg.density == pytest.approx(3e20)
    assert s.maxRunTime == pytest.approx(0.01) and s.cfg.geometry == 0
    with pytest.raises(cb.DsmcError):
        cb.settings_t().readFromCmdLine(["prog", "-mt"])


@pytest.mark.skipif(not os.path.exists(REF), reason="reference checkout not present")
@pytest.mark.parametrize("name", ["config.xml", "config_500k.xml", "config_mln.xml"])
def test_reads_the_reference_configs(name):
    s = cb.settings_t().readFromFile(os.path.join(REF, "data", name))
    assert s.cfg.gas_mass == pytest.approx(5e-26)
    assert s.getCellsCount() in (9720, 32768)


@pytest.mark.skipif(not (os.path.exists(REF) and O.ref_available()),
                    reason="reference checkout or oracle/_ref not present")
@pytest.mark.parametrize("name", ["config.xml", "config_500k.xml", "config_mln.xml"])
def test_config_parse_matches_reference_parser(name, monkeypatch):
    """Every value the reference's own settings_t::readFromFile
    (src/sim_settings.cpp:46-132, built unchanged into oracle/_ref) reads from
    its configuration and gas files, bit for bit; and the oracle's FP32 cell
    size (InitSimulationProperties) equal to the reference's."""
    s = cb.settings_t().readFromFile(os.path.join(REF, "data", name)).cfg
    f = np.zeros(18, np.float32)
    i = np.zeros(4, np.int32)
    monkeypatch.chdir(REF)  # the reference opens the gas file relative to the working directory
    assert O.ref().ref_read_settings(os.path.join("data", name).encode(), O.p(f), O.p(i)) == 0
    ours = np.array(list(s.grid_min) + list(s.grid_max) + [s.density, s.fnum, s.temp] +
                    list(s.stream_vel) + [s.gas_mass, s.gas_diam, s.gas_tref], np.float32)
    assert np.array_equal(ours, f[:15])
    assert list(s.grid_dim) == list(i[:3])
    assert s.periodic == bytes([i[3]])
    sim = O.sim_from(s.grid_min, s.grid_max, s.grid_dim, s.fnum, O.cross_section_of(s.gas_diam))
    assert np.array_equal(np.array(sim.cell[:], np.float32), f[15:18])


@pytest.mark.skipif(not (os.path.exists(REF) and O.ref_available()),
                    reason="reference checkout or oracle/_ref not present")
@pytest.mark.parametrize("args", [
    [],
    ["-benchmark", "-no-geometry", "-density", "3e20", "-dt", "2.5e-6", "-run-for", "0.01"],
    ["-f", "data/config_500k.xml", "-density", "7.3e19", "-benchmark"],
    ["-density", "1e21", "-f", "data/config.xml", "-dt", "1e-5"],
    ["-cpu", "-run-for", "2.5", "-dt", "3.3e-6"],
])
def test_command_line_matches_reference_parser(args, monkeypatch):
    """settings_t() and settings_t::readFromCmdLine (src/sim_settings.cpp:34-44,
    134-186) of the reference, built unchanged, against this library's
    command-line parse: defaults, flags in order, a -f file read where it
    appears (later flags override it, earlier ones are overwritten)."""
    monkeypatch.chdir(REF)
    argv = ["prog"] + args
    s = cb.settings_t().readFromCmdLine(argv)
    c = s.cfg
    f = np.zeros(20, np.float32)
    i = np.zeros(8, np.int32)
    arr = (ctypes.c_char_p * len(argv))(*[a.encode() for a in argv])
    assert O.ref().ref_read_cmdline(len(argv), arr, O.p(f), O.p(i)) == 0
    ours = np.array(list(c.grid_min) + list(c.grid_max) + [c.density, c.fnum, c.temp] +
                    list(c.stream_vel), np.float32)
    assert np.array_equal(ours, f[:12])
    if any(a == "-f" for a in args):  # the gas is read from the file only
        assert np.array_equal(np.array([c.gas_mass, c.gas_diam, c.gas_tref], np.float32), f[12:15])
    assert list(c.grid_dim) == list(i[:3]) and c.periodic == bytes([i[3]])
    assert np.float32(c.dt) == f[18] and np.float32(s.maxRunTime) == f[19]
    # the flags set the same values; two defaults differ by design: there is
    # no viewer to run instead of the benchmark loop, and mesh collisions are
    # off until a mesh is set (the reference's main loads its built-in model)
    if "-benchmark" in args:
        assert c.benchmark == 1 and i[4] == 1
    else:
        assert c.benchmark == 1 and i[4] == 0
    if "-no-geometry" in args:
        assert c.geometry == 0 and i[5] == 0
    else:
        assert c.geometry == 0 and i[5] == 1
    assert i[6] == 0  # -mt is refused here (no GPU mode), so it is never given
    assert i[7] == int("-cpu" in args)  # parsed and never read by the reference; ignored here


@pytest.mark.parametrize("level", [0, 1, 3])
def test_icosphere(level):
    v, t = cb.mesh_icosphere(level, 0.1, (0.3, 0.3, 0.3))
    assert t.shape == (20 * 4 ** level, 3)
    r = np.linalg.norm(v - 0.3, axis=1)
    assert np.allclose(r, 0.1, rtol=1e-6)
    a, b, c = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    n = np.cross(b - a, c - a)
    assert np.all(np.sum(n * ((a + b + c) / 3 - 0.3), axis=1) > 0)  # outward


def closed_and_outward(v, t, inside):
    edges = {}
    for tri in t:
        for i in range(3):
            e = (int(tri[i]), int(tri[(i + 1) % 3]))
            edges[e] = edges.get(e, 0) + 1
    for (a, b), k in edges.items():
        assert k == 1 and edges.get((b, a), 0) == 1  # every edge shared by two opposite faces
    a, b, c = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    n = np.cross(b - a, c - a)
    vol = np.sum(np.einsum("ij,ij->i", a, np.cross(b, c))) / 6.0
    return vol


def test_capsule_is_closed_and_outward():
    v, t = cb.mesh_capsule(0.15, 20.0, 0.26, (0.5, 0.3, 0.3), 20000, 7)
    assert 17000 < len(t) < 23000
    vol = closed_and_outward(v, t, None)
    assert vol > 0  # outward orientation gives a positive enclosed volume
    # nose tip at the front, base radius from the 20 degree cone
    assert v[:, 0].min() == pytest.approx(0.35, abs=1e-5)
    v2, t2 = cb.mesh_capsule(0.15, 20.0, 0.26, (0.5, 0.3, 0.3), 20000, 8)
    assert not np.array_equal(v, v2)  # the seed turns the azimuthal start


def test_geometry_grid_matches_oracle_and_reference_golden():
    d = np.load(os.path.join(ROOT, "tests", "golden", "move_sphere.npz"))
    g = cb.build_geometry_grid(d["verts"], d["tris"], d["gdim"])
    for a, b in zip(g, (d["bbox"], d["cell"], d["count"], d["ids"], d["flags"])):
        assert np.array_equal(a, b)
    v, t = cb.mesh_capsule(0.15, 20.0, 0.26, (0.5, 0.3, 0.3), 8000, 3)
    g1 = cb.build_geometry_grid(v, t, (12, 16, 16))
    g2 = O.build_grid(v, t, (12, 16, 16))
    for a, b in zip(g1, g2):
        assert np.array_equal(a, b)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "data", "ares.raw")),
                    reason="reference checkout not present")
def test_raw_mesh_and_grid_vs_reference_host_code():
    v, t, n = cb.read_raw_mesh(os.path.join(REF, "data", "ares.raw"))
    assert v.shape == (4148, 3) and t.shape == (7744, 3)
    # half of the asset's faces are zero-area, stored with zero normals
    area = np.linalg.norm(np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]]), axis=1)
    live = area > 1e-12
    assert np.allclose(np.linalg.norm(n[live], axis=1), 1.0, atol=1e-3)
    assert np.all(np.linalg.norm(n[~live], axis=1) == 0)
    if O.ref_available():
        g1 = cb.build_geometry_grid(v, t, (5, 5, 20))
        g2 = O.build_grid(v, t, (5, 5, 20), use_ref=True)
        for a, b in zip(g1, g2):
            assert np.array_equal(a, b)


def test_tri_box_overlap_vs_reference_random():
    if not O.ref_available():
        pytest.skip("reference host code (oracle/_ref) not built")
    R = O.ref()
    rng = np.random.default_rng(9)
    for _ in range(20000):
        c = rng.uniform(-1, 1, 3).astype(np.float32)
        h = rng.uniform(0.05, 0.5, 3).astype(np.float32)
        t = rng.uniform(-1.5, 1.5, 9).astype(np.float32)
        assert O.orc().orc_tri_box_overlap(O.p(c), O.p(h), O.p(t)) == R.ref_tri_box_overlap(O.p(c), O.p(h), O.p(t))


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(cb.DsmcError) as e:
        cb.DSMCSolver().Init(cb.settings_t())
    assert e.value.status in (3, 4)


def _gloo_worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms, tot = bench.reduce_over_ranks(10.0 + rank, 1000 * (rank + 1), world, "cpu")
    out.put((rank, ms, tot))
    dist.destroy_process_group()


def test_replica_reduction_two_ranks_gloo():
    import random
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = random.randint(20000, 40000)
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
    for rank, ms, tot in res:
        assert ms == 11.0  # slowest rank
        assert tot == 3000.0  # all particle-steps


def test_totals_bytes_layout():
    """dsmc_totals_async writes selections and collisions as uint64 and the
    sum of relative speeds as float64, 24 bytes; TotalsFromBytes reads them."""
    b = np.zeros(24, np.uint8)
    b[:8].view(np.uint64)[0] = 2**40 + 3
    b[8:16].view(np.uint64)[0] = 12345
    b[16:24].view(np.float64)[0] = 6.5e9
    t = cb.DSMCSolver.TotalsFromBytes(b)
    assert t.tolist() == [float(2**40 + 3), 12345.0, 6.5e9]
