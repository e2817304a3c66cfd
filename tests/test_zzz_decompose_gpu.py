"""bc_decompose_gpu on the B200: the decomposition as GPU steps (BCC split,
chains, packing) gives exactly bc_decompose's packed arrays (the same steps
run as host loops are checked on the CPU in test_host.py)."""
import numpy as np
import pytest

from helpers import GOLDEN, GOLDEN_CASES, graphs, load_case, pkg


def _same(g):
    P = pkg()
    a = P.Decomposition(g).arrays()
    b = P.Decomposition(g, gpu_device=0).arrays()
    return all(np.array_equal(a[k], b[k]) if hasattr(a[k], "shape") else a[k] == b[k] for k in a)


@pytest.mark.gpu
def test_gpu_decomposition_equals_host_on_fixtures():
    P = pkg()
    for name in GOLDEN_CASES:
        n, u, v, _, _ = load_case(name)
        assert _same(P.Graph.from_edges(n, u, v)), name


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["rmat16", "grid", "ba64"])
def test_gpu_decomposition_equals_host_at_scale(which):
    P = pkg()
    G = graphs()
    n, u, v = {
        "rmat16": lambda: G.gen_rmat(16, 16, 0.2, 1, 8, seed=2),
        "grid": lambda: G.gen_grid(seed=3),
        "ba64": lambda: G.pack_graphs(G.gen_ba_batch(64, seed=4))[:3],
    }[which]()
    assert _same(P.Graph.from_edges(n, u, v))
