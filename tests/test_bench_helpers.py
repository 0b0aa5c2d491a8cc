"""Host-side helpers of bench.py, on CPU: the stratified sample that the
reference arm times (its weights must add up to the batch, so that the
weighted per-scene times estimate the whole batch), the DRAM-traffic
estimate of the roofline, and the tet-balanced split of a batch across
ranks that the multi-GPU run uses."""
import importlib.util
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_stratified_sample_weights_cover_the_batch(bench):
    from avbd_b200.scenes import batched_cube_params
    ids, weights = bench.stratified_sample(1024, 0, 16)
    assert len(ids) == len(weights) == len(set(ids)) >= 8
    assert all(0 <= s < 1024 for s in ids)
    # every stratum's sampled scenes carry its whole population
    assert abs(sum(weights) - 1024) < 1e-9
    # every stratum (cells per side band x stiffness band) is represented
    strata = {(min(3, (batched_cube_params(0, s)[0] - 4) // 5), int(np.log10(batched_cube_params(0, s)[1]) >= 5.5))
              for s in ids}
    assert len(strata) == 8
    # deterministic
    assert bench.stratified_sample(1024, 0, 16) == (ids, weights)


def test_traffic_estimate_scales_the_measured_ratio(bench):
    import json
    with open(os.path.join(ROOT, "profiles", "solve_traffic.json")) as f:
        ratio = json.load(f)["batch1024_cubes"]["dram_over_algorithmic"]
    assert 1.0 <= ratio < 1.5
    assert bench.traffic_for("batch1024_cubes", 1e9) == pytest.approx(ratio * 1e9)
    assert bench.traffic_for("no_such_workload", 1e9) is None


def test_clock_record_from_sampler_rows(bench, tmp_path):
    """The clocks object of the JSON line from nvidia-smi's CSV rows: the
    median SM clock of the samples under load (above half the maximum), the
    maximum, and every throttle reason seen active."""
    class Done:
        def terminate(self):
            pass

        def wait(self, timeout=None):
            return 0

    rows = ["0, 345, 1965, 150.1, 0x0, Not Active, Not Active, Not Active, Not Active",
            "0, 1800, 1965, 990.5, 0x4, Not Active, Not Active, Not Active, Active",
            "0, 1830, 1965, 995.0, 0x4, Not Active, Not Active, Not Active, Active",
            "0, 1950, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active",
            "garbage line"]
    path = tmp_path / "clocks.csv"
    path.write_text("\n".join(rows) + "\n")
    c = bench.Clocks(0)
    c.proc, c.path = Done(), str(path)
    rec = c.stop()
    assert rec == {"sm_mhz": 1830.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 4}
    assert not path.exists()
    # no sampler (nvidia-smi missing): no record
    assert bench.Clocks(0).stop() is None


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun the reference arm's rank 0 alone times the CPU
    reference; the other ranks exit 0 without work or output."""
    import subprocess
    import sys
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


def test_batch_partition_is_balanced_by_tets():
    from avbd_b200 import dist
    from avbd_b200.scenes import batched_cube_params
    for world in (2, 4, 8):
        parts = dist.batch_partition(1024, 0, world)
        flat = sorted(s for p in parts for s in p)
        assert flat == list(range(1024))
        loads = [sum(6 * batched_cube_params(0, s)[0] ** 3 for s in p) for p in parts]
        # longest-processing-time first: within one largest scene of even
        assert max(loads) - min(loads) <= 6 * 24 ** 3
