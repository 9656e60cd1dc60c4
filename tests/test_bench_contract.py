"""bench.py's reference arm on CPU, as the round's driver launches it: one JSON line per run, with the keys the
driver reads (impl, metric, value, unit, e2e with no host copies, cpu_baseline with its cores and sample), for
each workload, on a bounded sample; ranks other than 0 exit 0 without work. And the product path without a GPU:
creating a world fails loudly, with no CPU fallback."""
import json
import os
import subprocess
import sys

import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def run_bench(*args, env=None):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, capture_output=True,
                         text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    return out.stdout.strip().splitlines()


@pytest.mark.parametrize("workload", ["large-mixed", "sphere-lattice", "batched-scenes", "sphere-pile"])
def test_reference_arm_prints_one_line_of_the_contract(workload):
    import bench
    lines = run_bench("--impl", "reference", "--steps", "2", "--warmup", "1", "--workload", workload)
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["warmup"] >= 1 and line["steps"] >= 1 and line["n_gpus"] == 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    base = line["cpu_baseline"]
    assert base["value"] == line["value"] and base["kind"] == "port" and base["cores"] >= 1 and base["sample"]
    assert line["config"]["workload"]


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="1")
    assert run_bench("--impl", "reference", "--steps", "2", "--warmup", "1", env=env) == []


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the behaviour with no GPU")
def test_a_world_without_a_gpu_fails_loudly():
    sys.path.insert(0, os.path.join(ROOT, "vexelray-sim-rigid_b200"))
    from vxr import boxes as B
    from vxr._lib import VxrError
    from vxr.box_simulation import BoxSimulation
    with pytest.raises((VxrError, RuntimeError, OSError)):
        BoxSimulation(8, 1, 1, False, B.grid(1.0, 1.0, 1.0, 0.1, 0.005))


class _Rep:
    def __init__(self, steps, touching=0, rounds=0, unplaced=0, unlisted=0):
        self.steps, self.touching, self.points, self.rounds = steps, touching, 2 * touching, rounds
        self.unplaced, self.unlisted, self.most_rounds = unplaced, unlisted, rounds
        self.unplaced_total, self.unlisted_total = unplaced * steps, unlisted * steps


class _World:
    """A world whose sync reports nothing when no step ran since the sync before, as vxr_box_sync does."""

    def __init__(self):
        self.pending = 0

    def step(self, k):
        self.pending += k

    def sync(self):
        k, self.pending = self.pending, 0
        return _Rep(k, 500, 7, 1, 2) if k else _Rep(0)


@pytest.mark.parametrize("steps", [20, 40, 25, 7])
def test_last_step_keeps_the_colouring_when_the_final_sync_has_nothing_new(steps):
    import bench
    w = _World()
    reports = bench.Reports()
    for k in range(steps):
        w.step(1)
        if k % 20 == 19:
            reports.add(w.sync())
    reports.finish(w, 20, steps)
    last = reports.last_step()
    assert last["touching"] > 0 and last["rounds"] > 0
    assert last["steps_reported"] == steps
    assert last["unplaced_total"] == steps and last["unlisted_total"] == 2 * steps


def test_clock_samples_give_the_median_the_peak_and_every_throttle_reason_seen():
    """The clock record a line carries, from nvidia-smi's CSV rows (index, clocks.sm, clocks.max.sm, power, active
    mask, then the hw_slowdown, hw_thermal_slowdown, sw_thermal_slowdown and sw_power_cap states): the median SM clock
    under load, the highest maximum, and every reason any sample saw active. Samples of two timed windows merge."""
    import bench
    row = lambda sm, hw="Not Active", sw_power="Not Active": ["0", str(sm), "1965", "900.0", "0x0", hw,  # noqa: E731
                                                              "Not Active", "Not Active", sw_power]
    a = bench.Clocks(0)
    a.samples = [row(1965), row(1950, sw_power="Active")]
    b = bench.Clocks(0)
    b.samples = [row(1965), row(1800, hw="Active"), row(1965)]
    a.samples += b.samples
    s = a.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 5
    assert s["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert bench.Clocks(0).summary()["reasons"] == ["unsampled"]
