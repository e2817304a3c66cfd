"""Host logic of bench.py (CPU): how a plan's units are cut into steps and
dealt to ranks, and the TEPS bookkeeping those steps feed."""
import numpy as np

import bench
from helpers import pkg

pkg()
from centrality_gpu_b200 import multigpu  # noqa: E402


class FakePlan:
    """unit_work of a plan whose units hold the given numbers of sources."""

    def __init__(self, per_unit):
        self.n_units = len(per_unit)
        self.c = np.concatenate([[0], np.cumsum(per_unit)])

    def unit_work(self, a, b):
        s = int(self.c[b] - self.c[a])
        return s, 10 * s, 3 * s


def test_step_ranges_are_minimal_and_cover_every_unit():
    rng = np.random.default_rng(7)
    for trial in range(20):
        per = rng.integers(1, 600, size=int(rng.integers(1, 300)))
        plan = FakePlan(per)
        target = int(rng.integers(1, 4000))
        ranges = bench.step_ranges(plan, target)
        assert ranges[0][0] == 0 and ranges[-1][1] == plan.n_units
        assert all(b0 == a1 for (_, a1), (b0, _) in zip(ranges, ranges[1:]))  # contiguous
        assert all(a < b for a, b in ranges)
        total = plan.unit_work(0, plan.n_units)[0]
        for k, (a, b) in enumerate(ranges[:-1]):
            # step k ends at the first unit boundary holding (k+1) * target sources
            assert plan.unit_work(0, b)[0] >= (k + 1) * target > plan.unit_work(0, b - 1)[0]
        assert plan.unit_work(0, ranges[-1][0])[0] < total or len(ranges) == 1


def test_shards_partition_the_steps():
    steps = [(i, i + 1) for i in range(11)]
    for world in (1, 2, 3, 4, 8):
        got = [multigpu.shard(steps, r, world) for r in range(world)]
        assert sorted(x for g in got for x in g) == steps
        assert max(map(len, got)) - min(map(len, got)) <= 1


def test_reference_arm_line(tmp_path):
    """bench.py --impl reference (the reference method's CPU path on the host
    cores) prints one JSON line with this engine's metric, unit and
    direction, its cpu_baseline and a zero-copy e2e; under torchrun every rank
    but 0 exits 0 without output."""
    import json
    import os
    import subprocess
    import sys

    from helpers import ROOT

    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", "small", "--steps", "2",
           "--warmup", "1", "--ref-step-s", "0.2"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC
    assert d["unit"] == "GTEPS" and d["higher_is_better"] is True and d["value"] > 0
    assert d["steps"] == 2 and d["warmup"] == 1 and d["config"]["workload"].startswith("small")
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["cores"] >= 1 and cb["kind"] == "port" and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=tmp_path,
                       env=dict(os.environ, RANK="1", WORLD_SIZE="2"))
    assert r.returncode == 0 and r.stdout.strip() == ""
