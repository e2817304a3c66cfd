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


def _deep_cycle():
    """A 30000-vertex cycle with 12 chords and 200 pendant leaves (deep BFS levels)."""
    G = graphs()
    rng = np.random.default_rng(21)
    n = 30000
    u = np.concatenate([np.arange(n), rng.integers(0, n, 12)])
    v = np.concatenate([(np.arange(n) + 1) % n, rng.integers(0, n, 12)])
    uu, vv = G.simple_edges(n, u, v)
    return G.attach_leaves(n, uu, vv, 200, n, rng)


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["rmat16", "grid", "ba64", "deep"])
def test_gpu_decomposition_equals_host_at_scale(which):
    P = pkg()
    G = graphs()
    n, u, v = {
        "rmat16": lambda: G.gen_rmat(16, 16, 0.2, 1, 8, seed=2),
        "grid": lambda: G.gen_grid(seed=3),
        "ba64": lambda: G.pack_graphs(G.gen_ba_batch(64, seed=4))[:3],
        "deep": _deep_cycle,
    }[which]()
    assert _same(P.Graph.from_edges(n, u, v))


@pytest.mark.gpu
def test_betc_with_gpu_decomposition_matches_golden(tmp_path):
    import json
    import subprocess

    P = pkg()
    for name in ("sample4", "rand4", "small2000"):
        out = tmp_path / f"{name}.out"
        r = subprocess.run([str(P.BETC_PATH), str(GOLDEN / f"{name}.txt"), "--out", str(out), "--gpu-decomp"],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        vals = np.loadtxt(out, ndmin=2)
        bc = np.array(json.loads((GOLDEN / f"{name}.bc.json").read_text())["bc"])
        assert np.array_equal(vals[:, 0], np.arange(len(bc)))
        assert np.max(np.abs(vals[:, 1] - bc) / np.maximum(1.0, np.abs(bc))) < 1e-6
