"""Full runs on the GPU against the oracle: the sampled fields (particles per
step, ux, T per cell) of 8 GPU runs and 8 oracle runs agree within 3 sigma of
the sampling noise, under the acceptance rule of tests/fieldstats.py, which
the CPU tests check on the oracle itself (independent runs pass, planted
mistakes fail).  Fields are formed as the reference's
ProcessAndOutputStatistics forms them (kernels/dsmc_base.cu:104-163:
u = sum v / N, T = m (sum |v|^2 / N - |u|^2) / 3k) from the FP64 sums of
SampleCellStatisticsDev's loop (kernels/dsmc_kernel.cu:856-910).

Two modes, each on the same body (tests/sphereflow.py):
  - the reference's: HybridTaus per cell, hard spheres, the periodic-x
    boundary functor and the first-hit specular body, against the oracle's
    restatement of the reference step;
  - the extension mode the capsule workload runs: Philox streams, VHS
    omega = 0.81, inflow at x = 0 and outflow elsewhere, nearest wall
    crossings with a diffuse wall at 300 K, against oracle/fast_oracle.c.
Both sides start from independent draws of the same initial distribution."""
import numpy as np
import pytest

import fieldstats as F
import sphereflow as S
from cudadsmc_b200 import DSMCSolver, settings_t

pytestmark = pytest.mark.gpu

REPLICAS, SETTLE, STEPS, MIN_COUNT = 8, 100, 200, 50


def _gpu_run(seed):
    sim, geom, pos, vel, mr, seeds, ppc = S.initial_state(seed)
    s = settings_t().set(grid_min=S.GMIN, grid_max=S.GMAX, grid_dim=S.DIM, density=S.DENSITY,
                         fnum=S.fnum(), temp=S.TEMP, gas_mass=S.MASS, gas_diam=S.DIAM,
                         gas_tref=S.TREF, periodic="x", rng="taus", sample_every=1, geometry=1,
                         geom_nearest=0, wall_diffuse=0)
    sol = DSMCSolver().Init(s)
    assert sol.Info().part_per_cell == ppc
    verts, tris = S.icosphere(S.LEVEL, S.RADIUS, S.CENTER)
    nrm = np.cross(verts[tris[:, 1]] - verts[tris[:, 0]], verts[tris[:, 2]] - verts[tris[:, 0]])
    nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
    sol.SetModel(verts, tris, S.GEOM_DIM, nrm)
    sol.UploadState(pos, vel)
    sol.SetCellState(mr, seeds)
    sol.RunSimulationStep(S.DT, nsteps=SETTLE)
    sol.ResetSamples()
    sol.RunSimulationStep(S.DT, nsteps=STEPS)
    sums, _, nsamp = sol.SampleStatistics()
    assert nsamp == STEPS
    sol.close()
    return sums


def test_sampled_fields_agree_with_the_oracle_within_noise(cuda):
    gpu = np.stack([_gpu_run(1 + 10 * k) for k in range(REPLICAS)])
    ora = S.oracle_replicas(5001, REPLICAS, SETTLE, STEPS)
    r = F.compare(gpu, ora, STEPS, S.MASS, MIN_COUNT)
    print(f"GPU vs oracle (reference mode): {r['cells']} cells, beyond 3 sigma "
          f"{r['frac_beyond_3']:.4f}, mean z^2 per field {[round(v, 3) for v in r['mean_z2_per_field']]}")
    assert r["cells"] > 3000
    assert F.agree(r), r["mean_z2_per_field"]


def _gpu_run_fast(seed, run_seed):
    sim, st, mr = S.fast_initial_state(seed)
    s = S.fast_settings().set(seed=run_seed)
    sol = DSMCSolver().Init(s)
    verts, tris = S.fast_mesh()
    sol.SetModel(verts, tris, S.GEOM_DIM)
    sol.UploadState(st, soa=True)
    sol.SetCellState(mr)
    dt = s.cfg.dt
    sol.RunSimulationStep(dt, nsteps=SETTLE)
    sol.ResetSamples()
    sol.RunSimulationStep(dt, nsteps=STEPS)
    sums, _, nsamp = sol.SampleStatistics()
    assert nsamp == STEPS
    sol.close()
    return sums


def test_fast_mode_fields_agree_with_the_oracle_within_noise(cuda):
    gpu = np.stack([_gpu_run_fast(1 + 10 * k, 40 + k) for k in range(REPLICAS)])
    ora = S.oracle_replicas_fast(5001, REPLICAS, SETTLE, STEPS)
    r = F.compare(gpu, ora, STEPS, S.MASS, MIN_COUNT)
    print(f"GPU vs oracle (extension mode): {r['cells']} cells, beyond 3 sigma "
          f"{r['frac_beyond_3']:.4f}, mean z^2 per field {[round(v, 3) for v in r['mean_z2_per_field']]}")
    assert r["cells"] > 3000
    assert F.agree(r), r["mean_z2_per_field"]
