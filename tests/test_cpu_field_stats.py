"""The full-run field comparison (tests/fieldstats.py) on the oracle, on the
CPU: independent runs of the same flow agree within their sampling noise,
and the comparison rejects runs with a planted mistake - a 3 % hotter start,
or 1.5 times the NTC pairs.  The flow is tests/sphereflow.py: a stream past an
icosphere in a box periodic in x, with the reference's boundary functor and
first-hit specular body, 3,456 cells and about 55,000 particles."""
import pytest

import fieldstats as F
import sphereflow as S

REPLICAS, SETTLE, STEPS, MIN_COUNT = 8, 100, 200, 50


@pytest.fixture(scope="module")
def base():
    return S.oracle_replicas(1, REPLICAS, SETTLE, STEPS)


def _compare(base, **kw):
    other = S.oracle_replicas(1001, REPLICAS, SETTLE, STEPS, **kw)
    return F.compare(base, other, STEPS, S.MASS, MIN_COUNT)


def test_independent_runs_agree_within_noise(base):
    r = _compare(base)
    assert r["cells"] > 3000
    assert F.agree(r), r["mean_z2_per_field"]
    assert r["frac_beyond_3"] < 0.03


def test_planted_hotter_start_is_rejected(base):
    r = _compare(base, temp_scale=1.03)
    assert not F.agree(r)
    assert r["mean_z2_per_field"][2] > 2.0  # the temperature field carries it


def test_planted_collision_rate_is_rejected(base):
    r = _compare(base, pair_scale=1.5)
    assert not F.agree(r)
    assert min(r["mean_z2_per_field"]) > 1.6  # every field carries it


@pytest.fixture(scope="module")
def base_fast():
    return S.oracle_replicas_fast(1, REPLICAS, SETTLE, STEPS)


def test_fast_mode_independent_runs_agree_and_planted_wall_is_rejected(base_fast):
    """The extension-mode flow (inflow/outflow, VHS, diffuse 300 K sphere):
    independent oracle runs agree; a wall at 450 K and 1.5x the NTC pairs are
    rejected."""
    other = S.oracle_replicas_fast(1001, REPLICAS, SETTLE, STEPS)
    r = F.compare(base_fast, other, STEPS, S.MASS, MIN_COUNT)
    assert r["cells"] > 3000
    assert F.agree(r), r["mean_z2_per_field"]
    hot = S.oracle_replicas_fast(1001, REPLICAS, SETTLE, STEPS, wall_temp=450.0)
    r = F.compare(base_fast, hot, STEPS, S.MASS, MIN_COUNT)
    assert not F.agree(r), r["mean_z2_per_field"]
    pairs = S.oracle_replicas_fast(1001, REPLICAS, SETTLE, STEPS, pair_scale=1.5)
    r = F.compare(base_fast, pairs, STEPS, S.MASS, MIN_COUNT)
    assert not F.agree(r), r["mean_z2_per_field"]
