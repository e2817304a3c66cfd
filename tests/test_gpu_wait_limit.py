"""Bounded device-side waits on the B200. bc_wait_probe runs the library's
wait primitive (the one the multi-source kernel's grid barrier uses) on a
flag that nothing sets, with a limit of about a second: the wait runs out,
the call returns BCGPU_ETIMEOUT, and the same context then runs plans
correctly. A short bc_opts.wait_limit_ms does not trip the barrier waits of a
normal multi-source run. (The reference has no device-side waits; it exit()s
on any CUDA error, Codes/kernels.cuh:25-32.)"""
import pytest

from helpers import graphs, oracle, pkg, rel_err

pytestmark = pytest.mark.gpu


def small_graph():
    n, u, v = graphs().gen_small(3)
    O = oracle()
    row, col = O.csr(n, u, v)
    return n, u, v, O.brandes(n, row, col)


def test_wait_runs_out_and_the_context_survives():
    P = pkg()
    n, u, v, want = small_graph()
    d = P.Decomposition(P.Graph.from_edges(n, u, v))
    ctx = P.Context(mode=P.MODE_BATCHED, delta=P.DELTA_FP64, plain_core=-1, batch_width=64, wait_limit_ms=1000)
    rc, ms = ctx.wait_probe(1000)
    assert rc == P.ETIMEOUT
    assert 1000.0 <= ms < 10000.0
    got, _ = ctx.run(d)  # multi-source passes, grid barriers with the 1 s limit
    assert rel_err(got, want) < 1e-12
    rc, ms = ctx.wait_probe(200)  # and once more after a run
    assert rc == P.ETIMEOUT and 200.0 <= ms < 10000.0
    got, _ = ctx.run(d)
    assert rel_err(got, want) < 1e-12
    ctx.close()


def test_wait_probe_rejects_a_nonpositive_limit():
    P = pkg()
    ctx = P.Context(mode=P.MODE_PLAIN)
    rc, _ = ctx.wait_probe(0)
    assert rc == P.EINVAL
    ctx.close()
