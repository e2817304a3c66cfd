"""GPU parity: libbcgpu's CUDA path (through the C ABI) against the oracle
and the golden fixtures. Levels and path counts bit-exact; BC within 1e-12
relative (FP64 plain schedule)."""
import numpy as np
import pytest

from helpers import GOLDEN_CASES, graphs, load_case, oracle, pkg, rel_err

pytestmark = pytest.mark.gpu

TOL_PLAIN = 1e-12  # FP64 dependencies and BC accumulation


@pytest.fixture(scope="module")
def ctx():
    c = pkg().Context(mode=pkg().MODE_PLAIN)
    yield c
    c.close()


def decomp(n, u, v):
    P = pkg()
    return P.Decomposition(P.Graph.from_edges(n, u, v))


def oracle_bc(n, u, v):
    O = oracle()
    row, col = O.csr(n, u, v)
    return O.brandes(n, row, col)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_plain_bc_matches_golden(ctx, name):
    n, u, v, bc, _ = load_case(name)
    got, st = ctx.run(decomp(n, u, v))
    assert rel_err(got, bc) < TOL_PLAIN
    assert st["kernel_launches"] >= 1 or n < 3


@pytest.mark.parametrize("name", ["sample1", "sample3", "sample4", "parallel", "rand4", "small2000"])
def test_plain_rows_bit_exact(ctx, name):
    """Levels and path counts of every source (BFS rows, or merged rows for
    chain vertices) equal the oracle's, bit for bit."""
    n, u, v, _, _ = load_case(name)
    d = decomp(n, u, v)
    arrs = d.arrays()
    plan = ctx.plan(d)
    O = oracle()
    step = 7 if n > 500 else 1
    for b in range(arrs["n_bcc"]):
        v0, v1 = int(arrs["vtx_off"][b]), int(arrs["vtx_off"][b + 1])
        npl = int(arrs["n_plain"][b])
        picks = list(range(0, v1 - v0, step)) + list(range(npl, v1 - v0))  # every chain vertex
        for s in sorted(set(picks)):
            dg, sg = plan.source_rows(v0 + s, v1 - v0)
            do, so = O.bcc_source_rows(arrs, b, s)
            assert np.array_equal(dg, do), (b, s)
            assert np.array_equal(sg, so), (b, s)
    plan.close()


@pytest.mark.parametrize("seed", range(12))
def test_plain_random_graphs(ctx, seed):
    """Disconnected graphs, isolated vertices, cycles, chains, pendants."""
    G = graphs()
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(2, 300))
    m = int(rng.integers(0, 3 * n))
    u, v = G.simple_edges(n, rng.integers(0, n, m), rng.integers(0, n, m))
    if len(u):
        n, u, v = G.subdivide(n, u, v, 0.3, 1, 5, rng)
        n, u, v = G.attach_leaves(n, u, v, int(rng.integers(0, 20)), n, rng)
    got, _ = ctx.run(decomp(n, u, v))
    assert rel_err(got, oracle_bc(n, u, v)) < TOL_PLAIN


def test_plain_edge_cases(ctx):
    P = pkg()
    # empty graph, single vertex, single edge, path, triangle (cycle block), star
    cases = [(0, [], []), (1, [], []), (2, [0], [1]), (5, [0, 1, 2, 3], [1, 2, 3, 4]), (3, [0, 1, 0], [1, 2, 2]),
             (6, [0, 0, 0, 0, 0], [1, 2, 3, 4, 5])]
    for n, u, v in cases:
        u = np.array(u, dtype=np.int32)
        v = np.array(v, dtype=np.int32)
        got, st = ctx.run(decomp(n, u, v))
        assert rel_err(got, oracle_bc(n, u, v) if n else np.zeros(0)) < TOL_PLAIN
    # a long cycle: one BCC, every vertex free, deep levels
    n = 3001
    u = np.arange(n, dtype=np.int32)
    v = ((np.arange(n) + 1) % n).astype(np.int32)
    got, _ = ctx.run(decomp(n, *graphs().simple_edges(n, u, v)))
    assert rel_err(got, oracle_bc(n, *graphs().simple_edges(n, u, v))) < TOL_PLAIN


def test_small_config_2000(ctx):
    """The CPU-runnable configuration: 2,000-vertex core + pendants + chains."""
    n, u, v = graphs().gen_small(1)
    got, st = ctx.run(decomp(n, u, v))
    assert rel_err(got, oracle_bc(n, u, v)) < TOL_PLAIN
    assert st["sources"] == 1000 + 500  # every vertex of the one BCC (core + chains); pendants are bridges


@pytest.mark.parametrize("gen", ["rmat", "grid", "ba"])
def test_plain_reduced_configs(ctx, gen):
    """Reduced-size versions of the measured workloads, full BC vs the oracle."""
    G = graphs()
    if gen == "rmat":
        n, u, v = G.gen_rmat(11, 16, chain_frac=0.2, chain_hi=8, seed=2)
    elif gen == "grid":
        n, u, v = G.gen_grid(40, leaves=300, seed=3)
    else:
        n, u, v, _ = G.pack_graphs(G.gen_ba_batch(16, 50, 400, seed=4))
    got, _ = ctx.run(decomp(n, u, v))
    assert rel_err(got, oracle_bc(n, u, v)) < TOL_PLAIN


def test_unit_ranges_accumulate(ctx):
    """Running the work units in pieces adds up to the whole run."""
    n, u, v = graphs().gen_rmat(10, 8, chain_frac=0.2, seed=5)
    d = decomp(n, u, v)
    plan = ctx.plan(d)
    k = plan.n_units
    st1 = plan.run(0, k // 3)
    st2 = plan.run(k // 3, k)
    pieces = plan.read()
    assert st1["sources"] + st2["sources"] == plan.unit_work()[0]
    assert rel_err(pieces, oracle_bc(n, u, v)) < TOL_PLAIN
    plan.reset()
    plan.run(0, k)
    assert rel_err(plan.read(), pieces) < 1e-13
    plan.close()


def test_begin_gpu_mirrors(ctx):
    """The reference-shaped entry points on one BCC: free sources through
    bc_begin_free, endpoints + ears through bc_begin_active; together they give
    the BCC's within-block contributions."""
    P = pkg()
    O = oracle()
    n, u, v, _, ref = load_case("sample4")
    arrs = decomp(n, u, v).arrays()
    for b in range(arrs["n_bcc"]):
        v0, v1 = int(arrs["vtx_off"][b]), int(arrs["vtx_off"][b + 1])
        nb = v1 - v0
        R = (arrs["row"][v0:v1 + 1] - arrs["row"][v0]).astype(np.int32)
        Cc = arrs["col"][arrs["row"][v0]:arrs["row"][v1]]
        reach = arrs["reach"][v0:v1]
        npl = int(arrs["n_plain"][b])
        ears, ends = [], set()
        for c in range(int(arrs["chain_off"][b]), int(arrs["chain_off"][b + 1])):
            s, ln = int(arrs["chain_start"][c]), int(arrs["chain_len"][c])
            l, r = int(arrs["chain_l"][c]), int(arrs["chain_r"][c])
            ends |= {l, r}
            ears.append((l, r, [(i + 1, s + i, ln - i) for i in range(ln)]))
        free = [k for k in range(npl) if k not in ends]
        bc = np.zeros(nb, dtype=np.float32)
        t = P.begin_gpu_free(ctx, R, Cc, nb, len(Cc), free, reach, bc) if free else 0.0
        t = P.begin_gpu_active(ctx, R, Cc, nb, len(Cc), sorted(ends), ears, reach, bc, t) if ears else t
        want = O.bcc_sources(arrs, b, np.arange(nb, dtype=np.int32))
        assert rel_err(bc, want) < 1e-6  # the reference's float buffer
        assert t >= 0.0


def test_bad_input_is_rejected(ctx):
    P = pkg()
    with pytest.raises(P.BcError):
        P.begin_gpu_free(ctx, [0, 1, 2], [1, 0], 2, 2, [0], [0, 0], np.zeros(2, np.float32))  # BCC < 3 vertices
    with pytest.raises(P.BcError):
        P.begin_gpu_free(ctx, [0, 2, 4, 6], [1, 2, 0, 2, 0, 9], 3, 6, [0], [0, 0, 0], np.zeros(3, np.float32))


@pytest.mark.parametrize("mode", ["plain", "batched"])
def test_betc_cli_matches_golden(tmp_path, mode):
    """The drop-in command: same edge-list input, `v bc` per vertex out."""
    import json
    import subprocess

    from helpers import GOLDEN
    P = pkg()
    for name in ("sample4", "rand4", "small2000"):
        out = tmp_path / f"{name}.{mode}.out"
        r = subprocess.run([str(P.BETC_PATH), str(GOLDEN / f"{name}.txt"), "--out", str(out), "--mode", mode],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        assert "GPU total time is" in r.stderr
        vals = np.loadtxt(out, ndmin=2)
        bc = np.array(json.loads((GOLDEN / f"{name}.bc.json").read_text())["bc"])
        assert np.array_equal(vals[:, 0], np.arange(len(bc)))
        assert rel_err(vals[:, 1], bc) < (TOL_PLAIN if mode == "plain" else 1e-6)
