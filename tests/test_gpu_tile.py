"""The small-BCC schedule on the B200 (one CTA per range of sources of a BCC,
its CSR slice staged in shared memory by a bulk copy; a warp, a CTA or a
group of a CTA per source):
BC against the oracle in FP64 (1e-12) on its own and mixed with the other two
schedules in one plan, bit-identical reruns, and BCCs at the size limits of
the schedule (the smallest, 3 vertices; the largest that fits shared
memory)."""
import numpy as np
import pytest

from helpers import GOLDEN_CASES, graphs, load_case, oracle, pkg, rel_err

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32c": 1e-6}


def decomp(n, u, v):
    P = pkg()
    return P.Decomposition(P.Graph.from_edges(n, u, v))


def oracle_bc(n, u, v):
    O = oracle()
    row, col = O.csr(n, u, v)
    return O.brandes(n, row, col)


def ba(count=16, seed=11):
    G = graphs()
    n, u, v, _ = G.pack_graphs(G.gen_ba_batch(count, 40, 3000, seed=seed))
    return n, u, v


@pytest.mark.parametrize("name", ["ba16", "small2000"] + GOLDEN_CASES)
def test_tile_bc_matches_the_oracle(name):
    P = pkg()
    if name == "ba16":
        n, u, v = ba()
    elif name == "small2000":
        n, u, v = graphs().gen_small(2)
    else:
        n, u, v, _, _ = load_case(name)
    d = decomp(n, u, v)
    want = oracle_bc(n, u, v)
    for tmax in (0, 64):  # every BCC that fits, or only those of <= 64 vertices
        ctx = P.Context(mode=P.MODE_BATCHED, delta=P.DELTA_FP64, tile_max=tmax)
        got, st = ctx.run(d)
        ctx.close()
        assert rel_err(got, want) < TOL["fp64"], tmax
        assert st["sources"] == int(d.arrays()["n_packed"])


@pytest.mark.parametrize("delta", ["fp64", "fp32c"])
def test_three_schedules_in_one_plan(delta):
    """BA graphs with the multi-source threshold at 500 core vertices and the
    small-BCC limit at 600 vertices: the largest BCCs take multi-source
    passes, the middle ones per-source items, the smallest tile items."""
    P = pkg()
    n, u, v = ba(16, seed=12)
    d = decomp(n, u, v)
    arrs = d.arrays()
    nb = np.diff(arrs["vtx_off"])
    assert (nb <= 600).any() and (arrs["n_plain"] >= 500).any() and ((nb > 600) & (arrs["n_plain"] < 500)).any()
    ctx = P.Context(mode=P.MODE_BATCHED, delta=P.DELTA_FP64 if delta == "fp64" else P.DELTA_FP32C, plain_core=500,
                    tile_max=600)
    plan = ctx.plan(d)
    st = plan.run()
    got = plan.read()
    assert st["kernel_launches"] == 5  # multi-source, per-source + fold, tile (warp class) + fold
    assert rel_err(got, oracle_bc(n, u, v)) < TOL[delta]
    plan.close()
    ctx.close()


def test_tile_reruns_are_bit_identical():
    P = pkg()
    n, u, v = ba(24, seed=13)
    d = decomp(n, u, v)
    ctx = P.Context(mode=P.MODE_BATCHED, delta=P.DELTA_FP64)
    outs = []
    for _ in range(2):
        plan = ctx.plan(d)
        plan.run()
        outs.append(plan.read())
        plan.close()
    ctx.close()
    assert np.array_equal(outs[0], outs[1])


def test_grouped_ctas_match_the_oracle():
    """Six BA graphs of 2,500-6,000 vertices: their BCCs (3,800-8,300
    vertices with chains) fit a one-source CTA only once or twice per SM and
    take the 1024-thread CTAs of four and two source groups sharing the
    staged slice (classes 5 and 4) next to the one-source 1024-thread CTA;
    FP64 BC against the oracle, and a second run bit-identical."""
    P = pkg()
    G = graphs()
    n, u, v, _ = G.pack_graphs(G.gen_ba_batch(6, 2500, 6000, seed=21))
    d = decomp(n, u, v)
    ctx = P.Context(mode=P.MODE_BATCHED, delta=P.DELTA_FP64, tile_max=0)
    plan = ctx.plan(d)
    classes = [c for c, _ in plan.tile_launches()]
    assert 4 in classes and 5 in classes, classes
    plan.run()
    got = plan.read()
    plan.reset()
    plan.run()
    again = plan.read()
    plan.close()
    ctx.close()
    assert np.array_equal(got, again)
    assert rel_err(got, oracle_bc(n, u, v)) < TOL["fp64"]


def test_tile_unit_ranges_add_up():
    """Running the plan's units in several ranges gives the whole run's BC."""
    P = pkg()
    n, u, v = ba(16, seed=14)
    d = decomp(n, u, v)
    ctx = P.Context(mode=P.MODE_BATCHED, delta=P.DELTA_FP64)
    plan = ctx.plan(d)
    k = plan.n_units
    for r0, r1 in ((0, k // 3), (k // 3, 2 * k // 3), (2 * k // 3, k)):
        plan.run(r0, r1)
    got = plan.read()
    plan.close()
    ctx.close()
    assert rel_err(got, oracle_bc(n, u, v)) < TOL["fp64"]


def test_tile_limits():
    """A triangle (the smallest BCC) and one BCC near the shared-memory limit
    (a 2-out random core of 1,800 vertices with chains: 2,516 vertices and
    8,628 arcs, 211 KB of the 227 KB a CTA may have): both through the
    small-BCC schedule."""
    P = pkg()
    G = graphs()
    ctx = P.Context(mode=P.MODE_BATCHED, delta=P.DELTA_FP64)
    n, u, v = 3, np.array([0, 1, 0]), np.array([1, 2, 2])
    got, _ = ctx.run(decomp(n, u, v))
    ctx.close()
    assert rel_err(got, oracle_bc(n, u, v)) < TOL["fp64"]
    rng = np.random.default_rng(5)
    core = 1800
    u, v = G.simple_edges(core, np.repeat(np.arange(core), 2), rng.integers(0, core, 2 * core))
    n, u, v = G.subdivide(core, u, v, 0.1, 1, 3, rng)
    d = decomp(n, u, v)
    ctx = P.Context(mode=P.MODE_BATCHED, delta=P.DELTA_FP64)
    got, _ = ctx.run(d)
    ctx.close()
    assert rel_err(got, oracle_bc(n, u, v)) < TOL["fp64"]
