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
