"""The per-source (PLAIN) schedule on the GPU: deterministic BC and path
counts beyond FP64's range.

* BC accumulates in fixed-point integer counters folded to FP64 in a fixed
  order, so rerunning a plan -- in BATCHED plans whose BCCs are routed to the
  per-source schedule, and in PLAIN plans -- gives bit-identical BC although
  the CTAs finish their sources in a different order each time.
* Path counts are stored per level relative to a power of two: forcing a
  rescale on almost every level (rescale_exp 4) leaves every exported level
  and path count, and the BC, bit-identical to the unforced run.
* A ring of 2,200 "diamonds" (4-cycles joined at their far corners) is one
  BCC whose path counts reach 2^1100, past FP64's largest finite value: with
  the default scaling the BC of sampled units matches a Brandes run with
  Python's unbounded integers for sigma; with scaling switched off the run
  fails with BCGPU_EOVERFLOW instead of returning wrong numbers.
"""
from collections import deque

import numpy as np
import pytest

from helpers import graphs, load_case, oracle, pkg, rel_err

pytestmark = pytest.mark.gpu


def decomp(n, u, v):
    P = pkg()
    return P.Decomposition(P.Graph.from_edges(n, u, v))


def ba_batch():
    G = graphs()
    n, u, v, _ = G.pack_graphs(G.gen_ba_batch(16, 40, 3000, seed=11))
    return n, u, v


def grid90():
    return graphs().gen_grid(90, leaves=800, seed=3)


@pytest.mark.parametrize("name,mode", [("ba", "batched"), ("grid", "batched"), ("ba", "plain"), ("grid", "plain")])
def test_bc_bit_identical_across_runs(name, mode):
    """Three runs of the same work (a fresh plan, a second fresh plan, the
    second plan reset and run again) give the same BC bit for bit; in the
    BATCHED plans every BCC of these graphs is routed per-source (cores under
    8192 vertices, or levels deeper than 96)."""
    P = pkg()
    n, u, v = ba_batch() if name == "ba" else grid90()
    d = decomp(n, u, v)
    ctx = P.Context(mode=P.MODE_BATCHED if mode == "batched" else P.MODE_PLAIN, delta=P.DELTA_FP64)
    outs = []
    for _ in range(2):
        plan = ctx.plan(d)
        plan.run()
        outs.append(plan.read())
    plan.reset()
    plan.run()
    outs.append(plan.read())
    plan.close()
    ctx.close()
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])
    O = oracle()
    row, col = O.csr(n, u, v)
    assert rel_err(outs[0], O.brandes(n, row, col)) < 1e-12


@pytest.mark.parametrize("name", ["small2000", "rand4", "grid40"])
def test_forced_rescaling_is_exact(name):
    """Rescaling by powers of two is exact: rows (levels and unscaled path
    counts, BFS and merged chain rows) and BC equal the unforced run's bit
    for bit, and the rows equal the oracle's."""
    P = pkg()
    if name == "grid40":
        n, u, v = graphs().gen_grid(40, leaves=200, seed=2)
    else:
        n, u, v, _, _ = load_case(name)
    d = decomp(n, u, v)
    arrs = d.arrays()
    O = oracle()
    res = {}
    for tag, rx in (("default", 0), ("forced", 4)):
        ctx = P.Context(mode=P.MODE_PLAIN, rescale_exp=rx)
        plan = ctx.plan(d)
        plan.run()
        rows = []
        for b in range(arrs["n_bcc"]):
            v0, v1 = int(arrs["vtx_off"][b]), int(arrs["vtx_off"][b + 1])
            npl = int(arrs["n_plain"][b])
            picks = sorted(set(range(0, npl, max(1, npl // 8))) | set(range(npl, v1 - v0, max(1, (v1 - v0 - npl) // 8 or 1))))
            for s in picks:
                rows.append((b, s) + plan.source_rows(v0 + s, v1 - v0))
        res[tag] = (plan.read(), rows)
        plan.close()
        ctx.close()
    assert np.array_equal(res["default"][0], res["forced"][0])
    for (b, s, d0, s0), (_, _, d1, s1) in zip(res["default"][1], res["forced"][1]):
        assert np.array_equal(d0, d1) and np.array_equal(s0, s1), (b, s)
        do, so = O.bcc_source_rows(arrs, b, s)
        assert np.array_equal(d1, do) and np.array_equal(s1, so), (b, s)


def diamond_ring(k):
    """k 4-cycles c_i - {a_i, b_i} - c_{i+1} closed into a ring (ids: c_i = 3i,
    a_i = 3i+1, b_i = 3i+2). One BCC; from c_0, c_j is reached by 2^j
    shortest paths while j < k/2."""
    u, v = [], []
    for i in range(k):
        c, a, b, c2 = 3 * i, 3 * i + 1, 3 * i + 2, 3 * ((i + 1) % k)
        u += [c, c, a, b]
        v += [a, b, c2, c2]
    return 3 * k, np.array(u, dtype=np.int64), np.array(v, dtype=np.int64)


def bigint_dependencies(n, u, v, sources):
    """Sum over the given sources of the Brandes dependency delta_s(v), with
    path counts as Python integers (no overflow) and each ratio
    sigma(v)/sigma(w) a correctly rounded float."""
    adj = [[] for _ in range(n)]
    for a, b in zip(u.tolist(), v.tolist()):
        adj[a].append(b)
        adj[b].append(a)
    out = np.zeros(n)
    for s in sources:
        dist = [-1] * n
        sigma = [0] * n
        dist[s], sigma[s] = 0, 1
        order, q = [], deque([s])
        while q:
            x = q.popleft()
            order.append(x)
            for y in adj[x]:
                if dist[y] < 0:
                    dist[y] = dist[x] + 1
                    q.append(y)
                if dist[y] == dist[x] + 1:
                    sigma[y] += sigma[x]
        delta = [0.0] * n
        for w in reversed(order):
            for x in adj[w]:
                if dist[x] == dist[w] - 1:
                    delta[x] += sigma[x] / sigma[w] * (1.0 + delta[w])
            if w != s:
                out[w] += delta[w]
    return out


@pytest.fixture(scope="module")
def ring():
    n, u, v = diamond_ring(2200)
    return n, u, v, decomp(n, u, v)


@pytest.mark.parametrize("mode", ["plain", "batched-routed", "batched-multi-fp64"])
def test_path_counts_beyond_fp64(ring, mode):
    P = pkg()
    n, u, v, d = ring
    arrs = d.arrays()
    assert int(arrs["n_bcc"]) == 1 and int(arrs["n_packed"]) == n
    opts = {"plain": dict(mode=P.MODE_PLAIN),
            "batched-routed": dict(mode=P.MODE_BATCHED),  # 2,200 core vertices: routed per-source
            "batched-multi-fp64": dict(mode=P.MODE_BATCHED, plain_core=-1, delta=P.DELTA_FP64, batch_width=64)}[mode]
    ctx = P.Context(**opts)
    plan = ctx.plan(d)
    units = [0, plan.n_units // 3, plan.n_units - 1]
    orig = np.asarray(arrs["orig"])
    for k in units:
        got, _ = ctx.run_units(d, k, k + 1)
        srcs = [int(orig[x]) for x in plan.unit_sources(k, k + 1)]
        want = bigint_dependencies(n, u, v, srcs)
        assert np.all(np.isfinite(got))
        assert rel_err(got, want) < 1e-12, (k, srcs[:4])
    plan.close()
    ctx.close()


def test_unscaled_path_counts_fail_loudly(ring):
    """With per-level scaling off (a threshold above FP64's exponent range)
    the path counts overflow: the run reports BCGPU_EOVERFLOW."""
    P = pkg()
    n, u, v, d = ring
    ctx = P.Context(mode=P.MODE_PLAIN, rescale_exp=2000)
    with pytest.raises(P.BcError) as e:
        ctx.run_units(d, 0, 1)
    assert e.value.code == P.EOVERFLOW
    ctx.close()
