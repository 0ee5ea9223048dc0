"""Throughput benchmark of the B200 DSMC timestep.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME]

One "step" is one DSMC timestep of the whole workload (scan, scatter, cell
kernel with collisions, move, sampling every 100 steps, inflow injection).
The metric is particle-timesteps per second: the particles in cells summed
over the timed steps (counted on the device) divided by the device time of
the timed region (CUDA events, max over ranks).  With N > 1 every rank runs
an independent replica of the workload (the timestep does not shard; the only
cross-rank traffic is the reduction of the timings).

--impl reference times the CPU restatement of the reference's step (oracle/,
OpenMP over all host cores) on a bounded sample of the same workload.

Both arms also report, under `legacy_dsmc_cpu`, the reference's own legacy
2-D CPU solver (src/dsmc_cpu.cpp on its compile-time 30 x 18 grid, single
thread) when oracle/_ref/dsmc_cpu_legacy is built: the only CPU solver the
reference ships, reported beside the port, not in place of it.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

KB = 1.380649e-23
ARGON = dict(gas_mass=6.63e-26, gas_diam=4.17e-10, gas_tref=273.0, gas_omega=0.81)

# ------------------------------------------------------------- workloads ----


def wl_capsule_4m():
    """Hypersonic argon over a blunt capsule, 128x64x64 cells: 4.26M particles
    at the free-stream fill, about 3.3M once the flow around the body has
    developed (the timed steps)."""
    dom = (1.2, 0.6, 0.6)
    dim = (128, 64, 64)
    cell_v = (dom[0] / dim[0]) * (dom[1] / dim[1]) * (dom[2] / dim[2])
    n_inf, T_inf, mach = 1e20, 200.0, 7.0
    a = math.sqrt(5.0 / 3.0 * KB * T_inf / ARGON["gas_mass"])
    U = mach * a
    fnum = n_inf * cell_v / 8.4
    s = dict(grid_min=(0, 0, 0), grid_max=dom, grid_dim=dim, density=n_inf, fnum=fnum, temp=T_inf,
             stream_vel=(U, 0.0, 0.0), dt=2e-6, rng="philox", ntc_local=1, sample_every=100,
             init_kind="maxwell", wall_diffuse=1, wall_temp=500.0, capacity_factor=1.6, seed=20261203,
             geom_nearest=1,
             face_kind={"-x": "inflow", "+x": "outflow", "-y": "outflow", "+y": "outflow",
                        "-z": "outflow", "+z": "outflow"}, **ARGON)
    mesh = dict(kind="capsule", nose_radius=0.15, cone_deg=20.0, length=0.26,
                nose_center=(0.35 + 0.15, 0.3, 0.3), ntarget=20000, seed=7, grid=(48, 64, 64))
    return dict(name="capsule_mach7_argon_4M_128x64x64", settings=s, mesh=mesh,
                desc=f"argon VHS w=0.81, Mach {mach:.0f} (U={U:.0f} m/s), T=200 K, n=1e20, "
                     "diffuse capsule wall 500 K (nose r=0.15 m, 20 deg cone, ~20k tris), "
                     "inflow -x, outflow elsewhere, 1.2x0.6x0.6 m, 128x64x64 cells, 4.26M particles at the fill, "
                     "about 3.3M in the developed flow")


def wl_sphere_500k():
    dom = (1.2, 0.6, 0.6)
    dim = (64, 32, 32)
    cell_v = (dom[0] / dim[0]) * (dom[1] / dim[1]) * (dom[2] / dim[2])
    fnum = 1e20 * cell_v / 7.63
    s = dict(grid_min=(0, 0, 0), grid_max=dom, grid_dim=dim, density=1e20, fnum=fnum, temp=200.0,
             stream_vel=(1500.0, 0.0, 0.0), dt=4e-6, rng="philox", ntc_local=1, sample_every=100,
             init_kind="maxwell", wall_diffuse=1, wall_temp=300.0, capacity_factor=1.6, seed=20261203,
             geom_nearest=1,
             face_kind={"-x": "inflow", "+x": "outflow", "-y": "outflow", "+y": "outflow",
                        "-z": "outflow", "+z": "outflow"}, **ARGON)
    mesh = dict(kind="icosphere", level=3, radius=0.1, center=(0.4, 0.3, 0.3), grid=(16, 16, 16))
    return dict(name="sphere_argon_500k_64x32x32", settings=s, mesh=mesh,
                desc="argon VHS, U=1500 m/s, T=200 K, diffuse icosphere(3) r=0.1 m at 300 K, "
                     "inflow -x, 64x32x32 cells, ~500k particles")


def wl_box_100k():
    s = dict(grid_min=(0, 0, 0), grid_max=(1, 1, 1), grid_dim=(16, 16, 16), density=1e20, fnum=1e15,
             temp=400.0, init_temp2=600.0, dt=1e-5, rng="philox", periodic="n", sample_every=100,
             init_kind="bimodal", seed=20261203, **ARGON)
    s["temp"] = 200.0
    return dict(name="box_argon_bimodal_100k_16cube", settings=s, mesh=None,
                desc="argon VHS in a closed 1 m specular box, 16^3 cells, 98,304 particles, "
                     "equal mix of 200 K and 600 K Maxwellians")


def batch_members(count=64, seed=20261203):
    """The batched ensemble: `count` sphere flows (icosphere level 3, r=0.1 m,
    1.2x0.6x0.6 m, 64x32x32 cells, inflow -x, outflow elsewhere, diffuse wall)
    with particle counts log-uniform in 50k-2M, Mach uniform in 2-10, Knudsen
    number (sphere diameter) log-uniform in 0.01-1 through the density, and
    T_wall/T_inf uniform in 1-3; seeded."""
    rng = np.random.default_rng(seed)
    dom, dim = (1.2, 0.6, 0.6), (64, 32, 32)
    cells = dim[0] * dim[1] * dim[2]
    cell = [dom[k] / dim[k] for k in range(3)]
    cell_v = cell[0] * cell[1] * cell[2]
    T, L, m, d = 200.0, 0.2, ARGON["gas_mass"], ARGON["gas_diam"]
    a = math.sqrt(5.0 / 3.0 * KB * T / m)
    cmp = math.sqrt(2 * KB * T / m)
    cbar = math.sqrt(8 * KB * T / (math.pi * m))
    out = []
    for i in range(count):
        n_part = math.exp(rng.uniform(math.log(5e4), math.log(2e6)))
        mach = rng.uniform(2.0, 10.0)
        kn = math.exp(rng.uniform(math.log(0.01), math.log(1.0)))
        tw = rng.uniform(1.0, 3.0)
        nd = 1.0 / (math.sqrt(2.0) * math.pi * d * d * kn * L)
        u = mach * a
        fnum = nd * cell_v / (n_part / cells)
        dt = min(0.2 * min(cell) / (u + 3 * cmp), 0.2 * kn * L / cbar)
        st = dict(grid_min=(0, 0, 0), grid_max=dom, grid_dim=dim, density=nd, fnum=fnum, temp=T,
                  stream_vel=(u, 0.0, 0.0), dt=dt, rng="philox", ntc_local=1, sample_every=100,
                  init_kind="maxwell", wall_diffuse=1, wall_temp=tw * T, capacity_factor=1.6,
                  seed=seed + i, geom_nearest=1,
                  face_kind={"-x": "inflow", "+x": "outflow", "-y": "outflow", "+y": "outflow",
                             "-z": "outflow", "+z": "outflow"}, **ARGON)
        out.append(dict(settings=st, particles=n_part, mach=mach, kn=kn, tw_ratio=tw))
    return out


def wl_batch64():
    return dict(name="batch64_sphere_flows", settings=None,
                mesh=dict(kind="icosphere", level=3, radius=0.1, center=(0.4, 0.3, 0.3),
                          grid=(16, 16, 16)),
                members=batch_members(64),
                desc="64 independent sphere flows (64x32x32 cells each) in one graph-launched "
                     "step: particles log-U[50k, 2M], Mach U[2, 10], Kn log-U[0.01, 1], "
                     "T_wall/T_inf U[1, 3]")


WORKLOADS = {"capsule4m": wl_capsule_4m, "sphere500k": wl_sphere_500k, "box100k": wl_box_100k,
             "batch64": wl_batch64}
DEFAULT_WORKLOAD = "capsule4m"


def build_solver(wl, seed_offset=0):
    import cudadsmc_b200 as cb
    st = dict(wl["settings"])
    st["seed"] = st.get("seed", 1) + seed_offset
    s = cb.settings_t().set(**st)
    sol = cb.DSMCSolver().Init(s)
    m = wl["mesh"]
    if m is not None:
        if m["kind"] == "capsule":
            v, t = cb.mesh_capsule(m["nose_radius"], m["cone_deg"], m["length"], m["nose_center"],
                                   m["ntarget"], m["seed"])
        else:
            v, t = cb.mesh_icosphere(m["level"], m["radius"], m["center"])
        sol.SetModel(v, t, m["grid"])
    return sol


# ------------------------------------------------------------------ clocks ---

class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed
    region: NVML polled every millisecond from a thread (the region can be a
    few milliseconds long), nvidia-smi at 100 ms where NVML is not usable.
    Read-only: nothing here changes a setting of the GPU."""
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    BITS = [0x8, 0x40, 0x20, 0x4]  # nvmlClocksEventReason* of the same names

    def __init__(self, gpu_index, period_s=0.001):
        self.idx = gpu_index
        self.period = period_s
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []  # (sm MHz, max MHz, reason bits)
        self.stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(int(self.idx))
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self._poll_once()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nvml = None
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _poll_once(self):
        p = self.nvml
        mhz = p.nvmlDeviceGetClockInfo(self.h, p.NVML_CLOCK_SM)
        try:
            bits = p.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        except AttributeError:
            bits = p.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
        self.samples.append((float(mhz), float(self.max_mhz), int(bits)))

    def _poll(self):
        while not self.stop.is_set():
            try:
                self._poll_once()
            except Exception:
                return
            self.stop.wait(self.period)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        self.stop.set()
        if self.nvml is not None:
            self.t.join(timeout=2)
            try:
                self._poll_once()
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        mhz, mx, reasons = [], None, set()
        if self.samples:
            for m, x, bits in self.samples:
                mhz.append(m)
                mx = x
                for nm, b in zip(self.NAMES, self.BITS):
                    if bits & b:
                        reasons.add(nm)
            src = f"NVML every {self.period * 1e3:.0f} ms"
        else:
            for ln in self.lines:
                f = [x.strip() for x in ln.split(",")]
                if len(f) < 7:
                    continue
                try:
                    mhz.append(float(f[0]))
                    mx = float(f[1])
                except ValueError:
                    continue
                for k, nm in enumerate(self.NAMES):
                    if f[3 + k].lower().startswith("active"):
                        reasons.add(nm)
            src = "nvidia-smi every 100 ms"
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz), "source": src}


# ------------------------------------------------------------- CPU oracle ---

def cpu_oracle_sample(wl, budget_s=12.0, max_threads=None, warmup=1, max_steps=50):
    """The oracle's restatement of the reference step (OpenMP over the host
    cores) on the workload's own grid, particle count and body: the
    reference's free-stream fill (part_per_cell per cell, cells covered by
    the body included), HybridTaus NTC with the workload's VHS exponent, the
    reference's first-hit specular body, and its closed-box boundary functor.
    The reference expresses neither inflow/outflow faces nor diffuse walls
    nor Philox streams; those three are its closest counterparts.  The mesh
    comes from oracle/meshes.py, so the product library is not loaded.
    `warmup` untimed steps, then timed steps until budget_s or max_steps.
    Returns (particle-timesteps/s, threads, description, particles, steps,
    seconds)."""
    from oracle import oracle as O
    from oracle import meshes as OM
    if max_threads:
        O.set_threads(max_threads)
    s = wl["settings"]
    dim = list(s["grid_dim"])
    gmin, gmax = np.asarray(s["grid_min"], np.float64), np.asarray(s["grid_max"], np.float64)
    w = s.get("gas_omega", 0.5)
    gref = 0.0
    if abs(w - 0.5) > 1e-9:
        gref = math.sqrt(2 * KB * s["gas_tref"] / (0.5 * s["gas_mass"])) * math.gamma(2.5 - w) ** (-1 / (2 * w - 1))
    sim = O.sim_from(gmin, gmax, dim, s["fnum"], O.cross_section_of(s["gas_diam"]), "n", w, gref)
    ppc = int(np.float32(s["density"]) * np.float32(sim.cell_volume) / np.float32(s["fnum"]))
    rng = np.random.default_rng(1)
    n = ppc * sim.cells
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 4), np.float32)
    # ppc particles uniform in every cell (GenerateUniformVelocitiesDevBlocks' fill)
    cell_idx = np.repeat(np.arange(sim.cells, dtype=np.int64), ppc)
    cx = cell_idx % dim[0]
    cy = (cell_idx // dim[0]) % dim[1]
    cz = cell_idx // (dim[0] * dim[1])
    cs = np.asarray(list(sim.cell), np.float64)
    pos[:, 0] = gmin[0] + (cx + rng.uniform(0, 1, n)) * cs[0]
    pos[:, 1] = gmin[1] + (cy + rng.uniform(0, 1, n)) * cs[1]
    pos[:, 2] = gmin[2] + (cz + rng.uniform(0, 1, n)) * cs[2]
    pos[:, 3] = 1.0
    del cell_idx, cx, cy, cz
    vstd = math.sqrt(KB * s["temp"] / s["gas_mass"])
    vel[:, :3] = rng.normal(0, vstd, (n, 3)) + np.asarray(s.get("stream_vel", (0, 0, 0)))
    geom = None
    m = wl["mesh"]
    if m is not None:
        if m["kind"] == "capsule":
            v, t = OM.capsule(m["nose_radius"], m["cone_deg"], m["length"], m["nose_center"],
                              m["ntarget"], m["seed"])
        else:
            v, t = OM.icosphere(m["level"], m["radius"], m["center"])
        bbox, gc, count, ids, flags = O.build_grid(v, t, m["grid"])
        nrm = np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
        nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
        geom = O.geom_from(bbox, gc, m["grid"], count, ids, flags, v, t, nrm)
    seeds = ((rng.integers(0, 2**32, (sim.cells, 4), dtype=np.uint64) % (2**32 - 129)) + 128).astype(np.uint32)
    mr = np.zeros((sim.cells, 2), np.float32)
    mr[:, 0] = O.max_rel_vel_of(s["gas_diam"], s["temp"])
    mr[:, 1] = rng.uniform(0, 1, sim.cells)
    st4 = np.zeros((sim.cells, 4), np.float32)
    dt = s["dt"]
    for _ in range(max(0, int(warmup))):
        pos, vel, _ = O.step(sim, geom, pos, vel, dt, float(ppc), mr, st4, seeds)
    steps, t_total = 0, 0.0
    while steps < 1 or (t_total < budget_s and steps < max_steps):
        t0 = time.perf_counter()
        pos, vel, _ = O.step(sim, geom, pos, vel, dt, float(ppc), mr, st4, seeds)
        t_total += time.perf_counter() - t0
        steps += 1
    desc = (f"oracle restatement of the reference step on the full workload grid ({dim[0]}x{dim[1]}x"
            f"{dim[2]} cells, {n} particles, {int(warmup)} untimed + {steps} timed steps, "
            f"{O.threads()} threads); closest reference physics: closed specular box for the "
            f"inflow/outflow faces, first-hit specular body for the diffuse nearest-hit wall, "
            f"HybridTaus for Philox")
    return n * steps / t_total, O.threads(), desc, n, steps, t_total


def legacy_cpu_sample(budget_s=5.0, particles_per_cell=90):
    """The reference's legacy 2-D CPU solver (src/dsmc_cpu.cpp: UpdateGridCPU,
    ComputeNanbuCPU, IntegrateCPU on its compile-time 30 x 18 grid), built
    unchanged from the reference's sources into oracle/_ref/dsmc_cpu_legacy,
    single thread, for about budget_s seconds.  It is not the 3-D step and
    its physics is not comparable; it is reported beside the port as the only
    CPU solver the reference ships.  None when the prebuilt driver is absent."""
    exe = os.path.join(ROOT, "oracle", "_ref", "dsmc_cpu_legacy")
    dat = os.path.join(ROOT, "oracle", "_ref", "MersenneTwister.dat")
    if not (os.path.isfile(exe) and os.path.isfile(dat)):
        return None
    r = subprocess.run([exe, dat, str(particles_per_cell), str(budget_s), "100000", "999"],
                       capture_output=True, text=True, timeout=budget_s + 120)
    if r.returncode != 0:
        return {"label": "reference dsmc_cpu (2-D legacy)", "unavailable": (r.stderr or r.stdout).strip()[-200:]}
    res = json.loads(r.stdout.strip().splitlines()[-1])
    return {"label": "reference dsmc_cpu (2-D legacy)", "value": res["value"],
            "unit": "particle-timesteps/s", "cores": 1,
            "sample": (f"{res['particles']} particles on the 30x18 2-D grid, {res['steps']} steps of "
                       f"UpdateGridCPU + ComputeNanbuCPU + IntegrateCPU, {res['seconds']:.1f} s")}


# ---------------------------------------------------------------- our arm ---

def reduce_over_ranks(elapsed, count, world, device):
    """Whole-job timing of independent replicas: the slowest rank's elapsed
    time and the units all ranks processed.  The only cross-rank traffic of
    the benchmark."""
    import torch
    t = torch.tensor([float(elapsed)], dtype=torch.float64, device=device)
    c = torch.tensor([float(count)], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(c, op=torch.distributed.ReduceOp.SUM)
    return float(t.item()), float(c.item())


def kernels_per_step(settings, variant, has_mesh):
    """Kernels one timestep launches: scan and scatter; the fused cell kernel,
    or the split variants' order, NTC, flight, mesh flights (with a body) and
    sampling (with sampling on: it returns at once on other steps); two per
    inflow face (plan, fill)."""
    n = 2
    if variant >= 4:
        n += 3 + (1 if has_mesh else 0) + (1 if settings.get("sample_every", 0) > 0 else 0)
    else:
        n += 1
    faces = settings.get("face_kind", {})
    return n + 2 * sum(1 for k in faces.values() if k == "inflow")


def algorithmic_bytes(kernel, n_particles, cells, rng_taus, sample_frac, split=True):
    """Bytes a kernel must move per launch (SoA FP32 state, 24 B/particle).

    scatter: key read 4 + orig written 4 (split variants; for the fused cell
    kernel it also moves the state: + 24 read + 24 written).  order: orig 4
    + state gathered 24 + sorted state written 24 per particle; per cell its
    start 4 and (sigma g)max/remainder read + written 16 (+ 32 of HybridTaus
    state in the reference RNG mode).  flight: state read 24 + written 24 +
    next-step key 4 per particle.  cell (fused): state + orig read 28, state +
    key written 28, the per-cell terms of order and 80 B of sampling sums on
    sampling steps."""
    per_cell = 4 + 16 + (32 if rng_taus else 0)
    if kernel == "scatter":
        return n_particles * (4 + 4 + (0 if split else 48))
    if kernel == "order":
        return n_particles * (4 + 24 + 24) + cells * per_cell
    if kernel == "flight":
        return n_particles * (24 + 24 + 4)
    if kernel == "cell":
        return n_particles * (24 + 4 + 24 + 4) + cells * (per_cell + sample_frac * 80)
    if kernel == "scan":
        return cells * 12
    return 0


def run_ours(args, rank, world):
    import torch
    import cudadsmc_b200 as cb
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    wl = WORKLOADS[args.workload]()
    sol = build_solver(wl, seed_offset=rank)
    sol.SetStream(torch.cuda.current_stream().cuda_stream)
    n0 = sol.InitSystemState()
    dt = wl["settings"]["dt"]
    # warm-up (also develops the flow a little), then the launch-shape
    # autotuner of the cell kernel on real steps of the run
    sol.RunSimulationStep(dt, args.warmup)
    if args.tune_steps > 0:
        variant, tune_ms = sol.Autotune(dt, steps=args.tune_steps)
    else:
        # a fixed launch shape (profiling runs)
        sol.SetKernelVariant(args.variant)
        variant, tune_ms = args.variant, None
    split = variant >= 4
    # per-kernel breakdown on a short window with events around every kernel
    # (an event pair costs the GPU a few microseconds, so the timed region
    # below keeps events around the dominant kernel only).  Both replay the
    # step's CUDA graph, the library's event-record nodes inside it.
    bsteps = max(1, min(50, args.steps))
    sol.Profile(True)
    sol.StepGraph(dt, bsteps)
    breakdown = sol.ProfileReadKernels()
    dom_slot = max((k for k in breakdown if k in ("scatter", "order", "flight")),
                   key=lambda k: breakdown[k][0])
    if not split:
        breakdown["cell"] = breakdown.pop("order")  # the fused cell kernel's slot
    # the timed region's graph (events around the dominant kernel only),
    # captured and run once before it
    sol.Profile(True)
    sol.ProfileOnly([dom_slot])
    sol.StepGraph(dt, 1)
    sol.ProfileReadKernels()
    sol.Sync()
    info0 = sol.Info()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    gpu_index = int(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0] or 0) if world == 1 else dev.index
    with ClockSampler(gpu_index) as clk:
        sol.Profile(True)
        sol.ProfileOnly([dom_slot])  # the same mask: the graph is not captured again
        ev0.record()
        sol.StepGraph(dt, args.steps)
        ev1.record()
        torch.cuda.synchronize()
        prof = sol.ProfileReadKernels()
    ms = ev0.elapsed_time(ev1)
    sol.Sync()
    info1 = sol.Info()
    pst = int(info1.particle_steps - info0.particle_steps)
    ms_max, total_ps = reduce_over_ranks(ms, pst, world, dev)
    value = total_ps / (ms_max * 1e-3)
    launches = args.steps * kernels_per_step(wl["settings"], variant, wl["mesh"] is not None)
    n_avg = pst / args.steps
    # dominant kernel and its roofline
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    dom = dom_slot if split or dom_slot != "order" else "cell"
    dom_ms = prof[dom_slot][0] / max(prof[dom_slot][1], 1)
    taus = wl["settings"].get("rng", "taus") == "taus"
    alg = algorithmic_bytes(dom, n_avg, sol.Info().cells, taus, 1.0 / 100, split)
    achieved = alg / (dom_ms * 1e-3) / 1e9
    traffic = None
    tr_path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(tr_path):
        try:
            tr = json.load(open(tr_path)).get(args.workload, {}).get(dom)
            if tr:
                traffic = tr["bytes_per_particle"] * n_avg
        except (OSError, ValueError, KeyError):
            traffic = None
    kernels = {k: {"ms_per_launch": (v[0] / v[1] if v[1] else None), "launches": v[1],
                   "share": v[0] / max(sum(x[0] for x in breakdown.values()), 1e-12)}
               for k, v in breakdown.items()}
    kernels["window"] = (f"{bsteps} graph-replayed steps before the timed region, CUDA events "
                         "around every kernel; the timed region times only the dominant kernel")
    # whole-step roofline at 128 B per particle-timestep (algorithmic)
    step_frac = value / max(world, 1) * 128 / (peak * 1e9)
    # end-to-end through the C ABI with host buffers
    e2e = run_e2e(args, wl, rank, world, dev, variant)
    out = {
        "metric": "particle-timesteps/s", "value": value, "unit": "particle-timesteps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded free-stream fill, generated mesh)",
        "config": {"workload": wl["name"], "description": wl["desc"], "particles_initial": n0,
                   "particles_avg_timed": n_avg, "cells": sol.Info().cells, "dt": dt,
                   "parallelism": f"replicas{world}" if world > 1 else "single-gpu",
                   "l2_policy": "working set (2 x 24 B x N state + 12 B x N keys) > 126 MB L2",
                   "rng": wl["settings"].get("rng"),
                   "cell_kernel_variant": {"chosen": variant, "autotune_ms_per_step": tune_ms}},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
                     "algorithmic_bytes_per_launch": alg, "ms_per_launch": dom_ms,
                     "step_frac_128B": step_frac},
        "kernels": kernels,
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "e2e": e2e,
    }
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        v, cores, desc, *_ = cpu_oracle_sample(wl, budget_s=args.cpu_budget)
        out["cpu_baseline"] = {"value": v, "unit": "particle-timesteps/s", "cores": cores, "kind": "port",
                               "sample": desc}
        legacy = legacy_cpu_sample()
        if legacy is not None:
            out["legacy_dsmc_cpu"] = legacy
    sol.close()
    return out


def run_batch(args, rank, world):
    """Aggregate particle-timesteps/s of the batched ensemble: one graph launch
    per timestep advances every member; also the same members stepped one
    after another (each with its own graph) for comparison."""
    import torch
    import cudadsmc_b200 as cb
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    wl = WORKLOADS[args.workload]()
    m = wl["mesh"]
    v, t = cb.mesh_icosphere(m["level"], m["radius"], m["center"])
    sols = []
    for mem in wl["members"]:
        st = dict(mem["settings"])
        st["seed"] += rank * 1000
        sol = cb.DSMCSolver().Init(cb.settings_t().set(**st))
        sol.SetModel(v, t, m["grid"])
        sol.InitSystemState()
        sols.append(sol)
    batch = cb.DSMCBatch(sols)
    stream = torch.cuda.Stream()  # a real stream: the batch's branches fork from it
    batch.SetStream(stream.cuda_stream)
    batch.Step(args.warmup + 2)
    batch.Sync()

    def particle_steps():
        return sum(s.Info().particle_steps for s in sols)

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0 = particle_steps()
    gpu_index = int(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0] or 0) if world == 1 else dev.index
    with ClockSampler(gpu_index) as clk:
        ev0.record(stream)
        batch.Step(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    batch.Sync()
    ms = ev0.elapsed_time(ev1)
    pst = particle_steps() - p0
    ms_max, total = reduce_over_ranks(ms, pst, world, dev)
    value = total / (ms_max * 1e-3)
    # the same members stepped one after another on one stream
    for s in sols:
        s.SetStream(stream.cuda_stream)
        s.StepGraph(s.settings.cfg.dt, 1)
    torch.cuda.synchronize()
    k2 = max(3, args.steps // 4)
    p1 = particle_steps()
    ev0.record(stream)
    for _ in range(k2):
        for s in sols:
            s.StepGraph(s.settings.cfg.dt, 1)
    ev1.record(stream)
    torch.cuda.synchronize()
    seq_ms = ev0.elapsed_time(ev1)
    seq_value = (particle_steps() - p1) / (seq_ms * 1e-3)
    n_now = [s.Info().num_particles for s in sols]
    out = {
        "metric": "particle-timesteps/s", "value": value, "unit": "particle-timesteps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded members, generated mesh)",
        "config": {"workload": wl["name"], "description": wl["desc"], "members": len(sols),
                   "particles_now_total": int(sum(n_now)), "particles_now_min": int(min(n_now)),
                   "particles_now_max": int(max(n_now)),
                   "batched_launches": "each stage once per step for all members (order kernel in "
                                       "the (128 particles, 4 warps) shape)",
                   "parallelism": f"replicas{world}" if world > 1 else "single-gpu",
                   "l2_policy": "working set of all members (several GB) > 126 MB L2"},
        "sequential": {"value": seq_value, "ms_per_step": seq_ms / k2,
                       "note": "same members, one graph launch per member per step, one stream"},
        # the batch launches each stage once for all members: scan, scatter,
        # order, inflow plan and fill, NTC, flight, mesh, sampling
        "gpu_launches": args.steps * 9,
        "clocks": clk.summary(),
    }
    batch.close()
    for s in sols:
        s.close()
    out["single_instance_same_size"] = single_same_size(args, int(sum(n_now)), len(sols), stream)
    sv = out["single_instance_same_size"]["value"]
    out["single_instance_same_size"]["batch_over_single"] = value / max(world, 1) / sv
    return out


def single_same_size(args, particles, members, stream):
    """One sphere flow as large as the whole ensemble (the members' cells
    together, 256 x 128 x 128 for 64 members of 64 x 32 x 32, and their
    particles together), stepped with the same kernels.  Not the same physics:
    its particles are spread evenly (7.5 per cell, where the members hold
    0.8-30) and one body covers a far smaller share of its cells than each
    member's does, so its kernels' work per particle is lower than the
    ensemble's."""
    import torch
    import cudadsmc_b200 as cb
    f = max(1, round(members ** (1.0 / 3.0)))
    dim = (64 * f, 32 * f, 32 * f)
    dom = (1.2, 0.6, 0.6)
    cells = dim[0] * dim[1] * dim[2]
    cell_v = (dom[0] / dim[0]) * (dom[1] / dim[1]) * (dom[2] / dim[2])
    T, m = 200.0, ARGON["gas_mass"]
    a = math.sqrt(5.0 / 3.0 * KB * T / m)
    cmp = math.sqrt(2 * KB * T / m)
    u, nd = 6.0 * a, 1e20
    st = dict(grid_min=(0, 0, 0), grid_max=dom, grid_dim=dim, density=nd,
              fnum=nd * cell_v / (particles / cells), temp=T, stream_vel=(u, 0.0, 0.0),
              dt=0.2 * min(dom[k] / dim[k] for k in range(3)) / (u + 3 * cmp), rng="philox",
              ntc_local=1, sample_every=100, init_kind="maxwell", wall_diffuse=1, wall_temp=400.0,
              capacity_factor=1.6, seed=77, geom_nearest=1,
              face_kind={"-x": "inflow", "+x": "outflow", "-y": "outflow", "+y": "outflow",
                         "-z": "outflow", "+z": "outflow"}, **ARGON)
    sol = cb.DSMCSolver().Init(cb.settings_t().set(**st))
    v, t = cb.mesh_icosphere(3, 0.1, (0.4, 0.3, 0.3))
    sol.SetModel(v, t, (8 * f, 8 * f, 8 * f))
    sol.SetStream(stream.cuda_stream)
    sol.InitSystemState()
    dt = st["dt"]
    sol.StepGraph(dt, max(3, args.warmup))
    sol.Sync()
    k = max(3, args.steps // 4)
    p0 = sol.Info().particle_steps
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    sol.StepGraph(dt, k)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    res = {"value": (sol.Info().particle_steps - p0) / (ms * 1e-3), "ms_per_step": ms / k,
           "particles": int(sol.Info().num_particles), "cells": cells, "grid": list(dim), "steps": k}
    sol.close()
    return res


def run_e2e(args, wl, rank, world, dev, variant):
    """The same metric through the C ABI with host buffers, driven as a host
    program would: per run the pinned initial state is uploaded (h2d); every
    step is one replay of the step's graph (dsmc_step_graph) followed by an
    asynchronous copy of that step's collision totals into pinned host memory
    (dsmc_totals_async), which the host reads while the next step runs (after
    enqueueing step i it waits for step i-4's copy, so that a pause of the
    host shorter than four steps leaves the GPU busy); the sampled fields are
    read back at the end (d2h).  Three such runs from the same initial state;
    the value is their median (a run on a shared machine now and then loses
    tens of milliseconds to a stall of the GPU outside this program), the
    runs are listed."""
    import torch
    sol = build_solver(wl, seed_offset=rank)
    sol.SetStream(torch.cuda.current_stream().cuda_stream)
    sol.SetKernelVariant(variant)
    sol.InitSystemState()
    state = sol.DownloadState()  # the initial state, as a host would provide it
    host = torch.from_numpy(state).pin_memory()
    lag, ring = 4, 8  # totals read 4 steps behind, from a ring of 8 pinned slots
    tot = torch.zeros((ring, 24), dtype=torch.uint8).pin_memory()
    fields_host = torch.zeros((sol.Info().cells, 5), dtype=torch.float64).pin_memory()
    ev = [torch.cuda.Event() for _ in range(ring)]
    dt = wl["settings"]["dt"]
    # runs of at least 1000 steps (as many as the device-timed region when
    # that is longer): a DSMC run uploads its state once and steps thousands
    # of times, so a short timed region would measure the upload instead
    k = max(3, max(args.steps, 1000) if args.e2e_steps is None else args.e2e_steps)
    # warm the path (captures the step graph, loads the field kernel on its
    # first use) and keep the GPU busy for about 40 ms right before the timed
    # runs, so that they start at full clocks
    sol.UploadState(host.numpy(), soa=True)
    sol.StepGraph(dt, 100)
    sol.Fields(out=fields_host.numpy())
    sol.TotalsAsync(tot[0].data_ptr())
    sol.StepGraph(dt, 100)
    sol.Sync()
    runs = []
    for _ in range(3):
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sol.UploadState(host.numpy(), soa=True)
        i0 = sol.Info().particle_steps
        totals = None
        for i in range(k):
            sol.StepGraph(dt, 1)
            sol.TotalsAsync(tot[i % ring].data_ptr())
            ev[i % ring].record()
            if i >= lag:
                ev[(i - lag) % ring].synchronize()
                totals = sol.TotalsFromBytes(tot[(i - lag) % ring].numpy())
        for j in range(max(0, k - lag), k):
            ev[j % ring].synchronize()
            totals = sol.TotalsFromBytes(tot[j % ring].numpy())
        fields = sol.Fields(out=fields_host.numpy())
        t1 = time.perf_counter()
        pst = sol.Info().particle_steps - i0
        assert totals[1] > 0 and totals[0] >= totals[1]
        el, total = reduce_over_ranks(t1 - t0, pst, world, dev)
        runs.append(total / el)
    sol.close()
    return {"value": statistics.median(runs), "unit": "particle-timesteps/s",
            "h2d_bytes_per_step": int(state.nbytes / k),
            "d2h_bytes_per_step": int(24 + fields.nbytes / k), "steps": k, "runs": runs,
            "note": f"median of 3 runs of {k} steps, each: upload of the initial pinned state + per "
                    "step one C-ABI dsmc_step_graph and an asynchronous totals read into pinned memory "
                    f"(read by the host {lag} steps later) + the sampled fields at the end"}


# ---------------------------------------------------------- reference arm ---

def run_reference(args):
    wl = WORKLOADS[args.workload]()
    if wl.get("members"):
        wl = dict(wl, settings=wl["members"][0]["settings"])
    budget = max(10.0, min(90.0, 4.0 * args.steps))
    from oracle import oracle as O
    O.set_threads(os.cpu_count() or 1)
    v, cores, desc, n, steps, tt = cpu_oracle_sample(wl, budget_s=budget, warmup=min(args.warmup, 2),
                                                     max_steps=args.steps)
    out = {"metric": "particle-timesteps/s", "value": v, "unit": "particle-timesteps/s", "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": tt / steps * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic", "impl": "reference",
           "config": {"workload": wl["name"], "description": wl["desc"]},
           "cpu_baseline": {"value": v, "unit": "particle-timesteps/s", "cores": cores, "kind": "port",
                            "sample": desc},
           "e2e": {"value": v, "unit": "particle-timesteps/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    legacy = legacy_cpu_sample()
    if legacy is not None:
        out["legacy_dsmc_cpu"] = legacy
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--e2e-steps", type=int, default=None,
                    help="steps of the end-to-end leg (default: --steps, at least 1000)")
    ap.add_argument("--tune-steps", type=int, default=10,
                    help="steps per launch shape of the autotuner (0: use --variant)")
    ap.add_argument("--variant", type=int, default=5,
                    help="cell-kernel launch shape when --tune-steps is 0")
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import torch
        import datetime
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    out = run_batch(args, rank, world) if args.workload == "batch64" else run_ours(args, rank, world)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
