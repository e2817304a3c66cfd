"""GPU parity of the BATCHED schedule (bitmask multi-source BFS over the
chain-contracted graph) against the oracle: FP64 dependencies within 1e-12
relative, compensated FP32 dependencies within 1e-6 relative (the metric's
accuracy bar). "multi" forces every BCC into multi-source passes (the kernel
under test on small graphs); "auto" is the default routing, where small or
deep BCCs take the per-source schedule inside the same plan."""
import numpy as np
import pytest

from helpers import GOLDEN_CASES, graphs, load_case, oracle, pkg, rel_err

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32c": 1e-6}


def ctx_for(delta, width=0, rescale_exp=0, route="multi"):
    P = pkg()
    return P.Context(mode=P.MODE_BATCHED, delta=P.DELTA_FP64 if delta == "fp64" else P.DELTA_FP32C,
                     batch_width=width, rescale_exp=rescale_exp, plain_core=-1 if route == "multi" else 0)


@pytest.fixture(scope="module", params=["fp64-multi", "fp32c-multi", "fp32c-auto"])
def bctx(request):
    delta, route = request.param.split("-")
    c = ctx_for(delta, route=route)
    c.tol = TOL[delta]
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
def test_batched_bc_matches_golden(bctx, name):
    n, u, v, bc, _ = load_case(name)
    got, st = bctx.run(decomp(n, u, v))
    assert rel_err(got, bc) < bctx.tol


@pytest.mark.parametrize("seed", range(10))
def test_batched_random_graphs(bctx, seed):
    G = graphs()
    rng = np.random.default_rng(300 + seed)
    n = int(rng.integers(2, 400))
    m = int(rng.integers(0, 3 * n))
    u, v = G.simple_edges(n, rng.integers(0, n, m), rng.integers(0, n, m))
    if len(u):
        n, u, v = G.subdivide(n, u, v, 0.3, 1, 6, rng)
        n, u, v = G.attach_leaves(n, u, v, int(rng.integers(0, 30)), n, rng)
    got, _ = bctx.run(decomp(n, u, v))
    assert rel_err(got, oracle_bc(n, u, v)) < bctx.tol


@pytest.mark.parametrize("width", [32, 64, 96, 1024])
def test_batched_widths(width):
    """Several passes per BCC (width << sources): owners return as helper BFS
    slots, chains split across passes."""
    n, u, v = graphs().gen_small(2)
    for delta in ("fp64", "fp32c"):
        c = ctx_for(delta, width)
        got, st = c.run(decomp(n, u, v))
        assert st["batch_width"] == width
        assert rel_err(got, oracle_bc(n, u, v)) < TOL[delta]
        c.close()


@pytest.mark.parametrize("gen", ["rmat", "grid", "ba"])
def test_batched_reduced_configs(bctx, gen):
    G = graphs()
    if gen == "rmat":
        n, u, v = G.gen_rmat(11, 16, chain_frac=0.2, chain_hi=8, seed=2)
    elif gen == "grid":
        n, u, v = G.gen_grid(40, leaves=300, seed=3)
    else:
        n, u, v, _ = G.pack_graphs(G.gen_ba_batch(16, 50, 400, seed=4))
    got, _ = bctx.run(decomp(n, u, v))
    assert rel_err(got, oracle_bc(n, u, v)) < bctx.tol


def test_batched_deterministic():
    """Per-block FP64 partials in a fixed order: repeated runs agree bit for bit."""
    n, u, v = graphs().gen_rmat(10, 8, chain_frac=0.2, seed=6)
    d = decomp(n, u, v)
    for delta in ("fp64", "fp32c"):
        c = ctx_for(delta, 64)
        a, _ = c.run(d)
        b, _ = c.run(d)
        assert np.array_equal(a, b)
        c.close()


def test_sigma_rescaling_path():
    """Forcing a rescale above 2^12 (path counts here reach ~2^75) runs the
    per-level power-of-two scaling on every level; results are unchanged."""
    n, u, v = graphs().gen_grid(40, delete_frac=0.0, sub_p=0.0, leaves=0, seed=9)
    want = oracle_bc(n, u, v)
    for delta in ("fp64", "fp32c"):
        c = ctx_for(delta, 128, rescale_exp=12)
        got, _ = c.run(decomp(n, u, v))
        assert rel_err(got, want) < TOL[delta]
        c.close()


@pytest.mark.parametrize("rescale_exp", [0, 4])
def test_pass_rows_bit_exact(rescale_exp):
    """Levels and path counts of the multi-source passes -- every slot, every
    core vertex of its BCC, read back from the pass's workspace with the
    per-level power-of-two bases applied -- equal the oracle's per-source BFS
    rows bit for bit: core sources and chain sources (seeded at both chain
    ends), on the golden inputs, an RMAT graph with chains and a grid, with the
    default rescale limit and with a rescale on almost every level (2^4)."""
    P = pkg()
    O = oracle()
    G = graphs()
    cases = [load_case(name)[:3] for name in GOLDEN_CASES]
    cases += [G.gen_rmat(10, 8, 0.3, 1, 4, seed=9), G.gen_grid(24, seed=5)]
    c = ctx_for("fp64", 64, rescale_exp=rescale_exp)
    checked = 0
    for n, u, v in cases:
        d = decomp(n, u, v)
        arrs = d.arrays()
        vo = arrs["vtx_off"]
        plan = c.plan(d)
        for unit in range(plan.n_units):
            try:
                src, dd, ss = plan.pass_rows(unit)
            except P.BcError:  # the passes are the first units
                break
            packed = plan.unit_sources(unit, unit + 1)
            b = int(np.searchsorted(vo, packed[0], side="right") - 1)
            ncore = int(arrs["n_plain"][b])
            assert dd.shape == (len(src), ncore)
            assert np.array_equal(np.sort(src + vo[b]), np.sort(packed)), (b, unit)
            for i, s in enumerate(src):
                do, so = O.bcc_source_rows(arrs, b, int(s))
                assert np.array_equal(dd[i], do[:ncore]), (b, int(s))
                assert np.array_equal(ss[i], so[:ncore]), (b, int(s))
            checked += len(src)
        plan.close()
    c.close()
    assert checked > 1000


def test_fp32_range_is_reported():
    """Path counts beyond FP32's range (a 90x90 grid: ~2^174 corner to corner)
    make the compensated-FP32 mode fail loudly instead of returning wrong BC;
    the FP64 mode handles the same graph."""
    P = pkg()
    n, u, v = graphs().gen_grid(90, delete_frac=0.0, sub_p=0.0, leaves=0, seed=9)
    d = decomp(n, u, v)
    c = ctx_for("fp32c", 1024)
    with pytest.raises(P.BcError) as e:
        c.run(d)
    assert e.value.code == P.EOVERFLOW
    c.close()
    c = ctx_for("fp64", 1024)
    plan = c.plan(d)
    plan.run(0, 2)
    got = plan.read()
    ids = plan.unit_sources(0, 2)
    arrs = d.arrays()
    local = ids - int(arrs["vtx_off"][0])
    want = np.array(arrs["art"])
    np.add.at(want, arrs["orig"][arrs["vtx_off"][0]:arrs["vtx_off"][1]], oracle().bcc_sources(arrs, 0, local))
    assert rel_err(got, want) < 1e-12
    plan.close()
    c.close()


def test_sampled_units_match_oracle_rmat():
    """A larger RMAT (scale 14): a range of passes vs the oracle on exactly the
    sources those passes cover."""
    n, u, v = graphs().gen_rmat(14, 16, chain_frac=0.2, chain_hi=8, seed=2)
    d = decomp(n, u, v)
    arrs = d.arrays()
    for delta in ("fp64", "fp32c"):
        c = ctx_for(delta, 256)
        plan = c.plan(d)
        k = min(plan.n_units, 3)
        plan.run(0, k)
        got = plan.read()  # includes the articulation terms
        ids = plan.unit_sources(0, k)
        assert len(ids) > 256
        want = np.array(arrs["art"])
        b = 0
        local = ids - int(arrs["vtx_off"][b])
        np.add.at(want, arrs["orig"][arrs["vtx_off"][b]:arrs["vtx_off"][b + 1]], oracle().bcc_sources(arrs, b, local))
        assert rel_err(got, want) < TOL[delta]
        plan.close()
        c.close()


def test_batched_vs_plain_same_numbers():
    n, u, v = graphs().gen_rmat(11, 16, chain_frac=0.2, seed=8)
    d = decomp(n, u, v)
    P = pkg()
    p = P.Context(mode=P.MODE_PLAIN)
    a, sa = p.run(d)
    b_ctx = ctx_for("fp64")
    b, sb = b_ctx.run(d)
    assert sa["sources"] == sb["sources"] and sa["teps_edges"] == sb["teps_edges"]
    assert rel_err(b, a) < 1e-12
    p.close()
    b_ctx.close()


def test_routing_mixes_both_schedules():
    """Twelve BA graphs of mixed sizes: with the core threshold at 500, the
    five BCCs whose cores reach it take multi-source passes and the seven
    smaller ones per-source items, in one plan (three launches: the
    multi-source kernel, the per-source kernel and the fold of its counters;
    the small-BCC schedule is off here)."""
    G = graphs()
    n, u, v, _ = G.pack_graphs(G.gen_ba_batch(12, 40, 3000, seed=7))
    d = decomp(n, u, v)
    arrs = d.arrays()
    cores = [int(x) for x in arrs["n_plain"]]
    assert sum(c >= 500 for c in cores) == 5 and sum(c < 500 for c in cores) == 7
    P = pkg()
    for delta in ("fp64", "fp32c"):
        c = P.Context(mode=P.MODE_BATCHED, delta=P.DELTA_FP64 if delta == "fp64" else P.DELTA_FP32C, plain_core=500,
                      tile_max=-1)  # the small-BCC schedule off: test_gpu_tile.py mixes all three
        plan = c.plan(d)
        st = plan.run(0, plan.n_units)
        assert st["kernel_launches"] == 3
        assert st["sources"] == int(arrs["n_packed"])
        assert rel_err(plan.read(), oracle_bc(n, u, v)) < TOL[delta]
        plan.close()
        c.close()


def test_autotune_width():
    """The width autotuner times each candidate on this graph's passes and
    returns one of them; a plan at that width gives the oracle's BC."""
    n, u, v = graphs().gen_rmat(11, 16, chain_frac=0.2, chain_hi=8, seed=2)
    d = decomp(n, u, v)
    c = ctx_for("fp32c")
    w, per = c.autotune_width(d, passes=2)
    assert w in (128, 256, 512, 1024) and per[w] == max(per.values()) > 0
    c.close()
    c = ctx_for("fp32c", w)
    got, st = c.run(d)
    assert st["batch_width"] == w
    assert rel_err(got, oracle_bc(n, u, v)) < TOL["fp32c"]
    c.close()
