"""Host-side logic of the learned-proposal study and the benchmark, on CPU: the
annealing schedule (diffusion.rs:102-104 in f32), time to target, the JSON form of
unreached targets, and the study's configuration."""
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def test_annealing_schedule_matches_temperature(pkg, oracle):
    L = pkg.learned
    total = 600
    for start, n in ((0, 25), (275, 25), (575, 25)):
        got = L.annealing(n, total, start=start)
        exp = np.array([pkg.temperature(start + i, total) for i in range(n)], np.float32)
        assert got.dtype == np.float32 and np.array_equal(got, exp)
        ref = np.array([oracle.temperature(start + i, total) for i in range(n)], np.float32)
        assert np.allclose(got, ref, rtol=2e-7, atol=0)  # C powf vs numpy power: within an ulp
    t = L.annealing(total, total)
    assert t[0] == np.float32(3.0) and np.all(np.diff(t) < 0) and t[-1] > np.float32(0.02)


def test_time_to_target(pkg):
    L = pkg.learned
    plain = [[(10.0, -1.0, 0.0), (20.0, -5.0, 0.0)], [(10.0, -2.0, 0.0), (20.0, -3.0, 0.0)],
             [(10.0, -4.0, 0.0), (20.0, -4.0, 0.0)]]
    other = [[(5.0, -3.6, 0.0), (9.0, -6.0, 0.0)], [(5.0, 0.0, 0.0), (9.0, -1.0, 0.0)]]
    target, tp, to = L.time_to_target(plain, other, tol=0.5)
    assert target == -4.0  # median of the plain finals -5, -3, -4
    assert tp == [20.0, float("inf"), 10.0]
    assert to == [5.0, float("inf")]


def test_bench_strict_json_and_study_config():
    import bench
    assert bench._finite(float("inf")) is None and bench._finite(float("nan")) is None
    assert bench._finite(np.float64(2.5)) == 2.5
    json.dumps({"x": [bench._finite(v) for v in (1.0, float("inf"))]}, allow_nan=False)
    names = [m for m, _ in bench.LEARNED_METHODS]
    assert names[0] == "uniform" and len(set(names)) == len(names)
    assert bench.PHASE2_STEPS in bench.SCHEDULES  # the target is the uniform method's final champion there
    assert all(kw.get("t_prop_min") == bench.T_PROP_MIN for _, kw in bench.LEARNED_METHODS[1:])
    assert list(bench.SCHEDULES) == sorted(bench.SCHEDULES)
