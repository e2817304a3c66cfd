"""CUDA-graph mode (bc_opts.graph): each unit range's device work -- counter
resets and the persistent kernels, including the cooperative multi-source
kernel -- is recorded once by stream capture and replayed as one graph
launch. Recording runs nothing; replays give the oracle's BC within the
schedule's tolerance and accumulate like direct runs."""
import numpy as np
import pytest

from helpers import graphs, oracle, pkg, rel_err

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32c": 1e-6}


def decomp(n, u, v):
    P = pkg()
    return P.Decomposition(P.Graph.from_edges(n, u, v))


def oracle_bc(n, u, v):
    O = oracle()
    row, col = O.csr(n, u, v)
    return O.brandes(n, row, col)


def chunks(n_units, k):
    b = np.linspace(0, n_units, num=k + 1).round().astype(int)
    return [(int(x), int(y)) for x, y in zip(b[:-1], b[1:]) if y > x]


CASES = [
    # (mode, delta, plain_core): per-source items; every BCC in multi-source
    # passes (the cooperative kernel as a graph node); the default routing
    ("plain", "fp64", 0),
    ("batched", "fp64", -1),
    ("batched", "fp32c", -1),
    ("batched", "fp32c", 0),
]


@pytest.mark.parametrize("mode,delta,plain_core", CASES)
def test_graph_replay_matches_oracle_on_grid(mode, delta, plain_core):
    """Reduced road-like workload (40x40 grid, 10% of edges deleted, chains,
    300 leaves): record every chunk, check recording ran nothing, replay all
    chunks, compare with the oracle; replaying again doubles the sources'
    contributions."""
    P = pkg()
    n, u, v = graphs().gen_grid(40, leaves=300, seed=3)
    d = decomp(n, u, v)
    art = np.array(d.arrays()["art"], dtype=np.float64)
    want = oracle_bc(n, u, v)
    c = P.Context(mode=P.MODE_PLAIN if mode == "plain" else P.MODE_BATCHED,
                  delta=P.DELTA_FP64 if delta == "fp64" else P.DELTA_FP32C, plain_core=plain_core,
                  batch_width=128 if mode == "batched" else 0, graph=True)
    plan = c.plan(d)
    parts = chunks(plan.n_units, 3)
    for r0, r1 in parts:
        plan.record(r0, r1)
    assert np.array_equal(plan.read(), art)  # recording enqueued no device work
    launches = 0
    for r0, r1 in parts:
        st = plan.run(r0, r1, stats=True)
        launches += st["kernel_launches"]
    assert 1 <= launches <= 3 * len(parts)  # multi-source kernel, per-source kernel, fold
    got = plan.read()
    assert rel_err(got, want) < TOL[delta]
    for r0, r1 in parts:  # second replay of the same graphs
        plan.run(r0, r1, stats=False)
    again = plan.read()
    assert rel_err(again - art, 2.0 * (got - art)) < TOL[delta]
    plan.close()
    c.close()


def test_graph_and_direct_runs_agree_rmat():
    """Same plan options with and without graph mode on a reduced RMAT
    workload (one giant BCC plus small ones, routed to both schedules): the
    deterministic multi-source partials make the two results identical up to
    the order of the per-source FP64 atomics."""
    P = pkg()
    n, u, v = graphs().gen_rmat(11, 16, chain_frac=0.2, chain_hi=8, seed=2)
    d = decomp(n, u, v)
    out = []
    for graph in (False, True):
        c = P.Context(mode=P.MODE_BATCHED, delta=P.DELTA_FP64, batch_width=256, plain_core=300, graph=graph)
        got, st = c.run(d)
        assert st["sources"] == int(d.arrays()["n_packed"])
        out.append(got)
        c.close()
    assert rel_err(out[1], out[0]) < 1e-12
    assert rel_err(out[1], oracle_bc(n, u, v)) < 1e-12


def test_record_needs_graph_mode():
    P = pkg()
    n, u, v = graphs().gen_small(1)
    c = P.Context(mode=P.MODE_PLAIN)
    plan = c.plan(decomp(n, u, v))
    with pytest.raises(P.BcError):
        plan.record(0, plan.n_units)
    with pytest.raises(P.BcError):
        plan.run(0, plan.n_units + 1)
    plan.close()
    c.close()
