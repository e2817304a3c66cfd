"""bc_opts.lazy_tables on the B200: a one-shot unit-range call that builds the
multi-source tables of its own passes only gives the same BC, bit for bit,
as one that builds every pass's tables (the CPU side checks the tables
themselves: tests/test_host_plumbing.py)."""
import numpy as np
import pytest

from helpers import graphs, pkg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("route", ["multi", "auto"])
def test_lazy_tables_give_the_same_bc(route):
    P = pkg()
    G = graphs()
    n, u, v = G.pack_graphs(G.gen_ba_batch(12, 40, 3000, seed=7))[:3]
    d = P.Decomposition(P.Graph.from_edges(n, u, v))
    opts = dict(mode=P.MODE_BATCHED, delta=P.DELTA_FP32C, batch_width=64, plain_core=-1 if route == "multi" else 0)
    full, lazy = P.Context(**opts), P.Context(lazy_tables=True, **opts)
    units = full.plan(d).n_units
    for r0, r1 in ((0, 1), (3, 9), (units // 2, units // 2 + 5), (max(0, units - 4), units), (0, units)):
        a, _ = full.run_units(d, r0, r1)
        b, _ = lazy.run_units(d, r0, r1)
        assert np.array_equal(a, b), (r0, r1)
    full.close()
    lazy.close()
