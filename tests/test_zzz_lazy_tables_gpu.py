"""bc_opts.lazy_tables on the B200: a one-shot unit-range call that builds the
multi-source tables of its own passes only gives the same BC, bit for bit,
as one that builds every pass's tables (the CPU side checks the tables
themselves: tests/test_host_plumbing.py).

[multi]: every BCC in multi-source passes. [mixed]: a core threshold of 500
sends the five largest of the twelve BCCs to multi-source passes and the
seven others to the per-source schedule, so the ranges below cross from
passes into per-source items; per-source BC is deterministic (fixed-point
accumulation), so those units compare bit for bit too."""
import numpy as np
import pytest

from helpers import graphs, pkg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("route", ["multi", "mixed"])
def test_lazy_tables_give_the_same_bc(route):
    P = pkg()
    G = graphs()
    n, u, v = G.pack_graphs(G.gen_ba_batch(12, 40, 3000, seed=7))[:3]
    d = P.Decomposition(P.Graph.from_edges(n, u, v))
    opts = dict(mode=P.MODE_BATCHED, delta=P.DELTA_FP32C, batch_width=64, plain_core=-1 if route == "multi" else 500)
    full, lazy = P.Context(lazy_tables=False, **opts), P.Context(lazy_tables=True, **opts)
    plan = full.plan(d)
    units = plan.n_units
    arrs = d.arrays()
    owner = np.repeat(np.arange(arrs["n_bcc"]), np.diff(arrs["vtx_off"]))
    big = [b for b in range(arrs["n_bcc"]) if route == "multi" or arrs["n_plain"][b] >= 500]
    kinds = [bool(np.isin(owner[plan.unit_sources(k, k + 1)], big).all()) for k in range(units)]
    n_bat = kinds.index(False) if False in kinds else units  # the multi-source passes come first
    plan.close()
    assert n_bat > 0 and (route == "multi" or n_bat < units)
    ranges = [(0, 1), (3, 9), (units // 2, units // 2 + 5), (max(0, units - 4), units), (0, units)]
    if n_bat < units:
        ranges.append((max(0, n_bat - 3), n_bat + 3))  # across the last passes into the first per-source items
    for r0, r1 in ranges:
        a, _ = full.run_units(d, r0, r1)
        b, _ = lazy.run_units(d, r0, r1)
        assert np.array_equal(a, b), (r0, r1)
    full.close()
    lazy.close()
