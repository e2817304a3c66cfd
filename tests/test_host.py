"""Host side of the product (C++ in libbcgpu.so): edge-list ingest and the
BCC / reach / chain decomposition, checked against the reference's own host
pipeline (golden dumps) and the brute-force oracle. CPU only."""
import subprocess

import numpy as np
import pytest

from helpers import GOLDEN, GOLDEN_CASES, graphs, has_gpu, load_case, oracle, pkg, product_bccs, rel_err
from test_oracle import _oracle_bccs, compare_to_reference


def decompose(n, u, v):
    P = pkg()
    return P.Decomposition(P.Graph.from_edges(n, u, v))


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_decomposition_matches_reference(name):
    n, u, v, _, ref = load_case(name)
    arrs = decompose(n, u, v).arrays()
    compare_to_reference(product_bccs(arrs), arrs["art"], ref, u, v)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_packed_bccs_give_golden_bc(name):
    """The product's packing, driven through the oracle's per-BCC kernel."""
    n, u, v, bc, _ = load_case(name)
    arrs = decompose(n, u, v).arrays()
    assert rel_err(oracle().method_bc_from_decomp(arrs), bc) < 1e-12


def random_graph(seed):
    """Disconnected graphs, isolated vertices, pendant cycles, loops and duplicates."""
    G = graphs()
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 70))
    m = int(rng.integers(0, 2 * n + 1))
    u = rng.integers(0, n, m)
    v = rng.integers(0, n, m)
    if seed % 3 == 0 and n > 3:  # a ring
        u = np.concatenate([u, np.arange(n)])
        v = np.concatenate([v, (np.arange(n) + 1) % n])
    uu, vv = G.simple_edges(n, u, v)
    if len(uu) and seed % 2:
        n, uu, vv = G.subdivide(n, uu, vv, 0.4, 1, 3, rng)
    # what the product is fed: the simple edges plus reversed duplicates and loops
    k = len(uu) // 3
    ru = np.concatenate([uu, vv[:k], np.arange(min(n, 3))])
    rv = np.concatenate([vv, uu[:k], np.arange(min(n, 3))])
    return n, ru, rv, uu, vv


@pytest.mark.parametrize("seed", range(40))
def test_decomposition_matches_oracle(seed):
    n, u_raw, v_raw, u, v = random_graph(seed)
    P = pkg()
    arrs = P.Decomposition(P.Graph.from_edges(n, u_raw, v_raw)).arrays()  # raw: loops + duplicates
    mine = {b["verts"]: b for b in product_bccs(arrs)}
    theirs, art = _oracle_bccs(n, u, v)
    assert set(mine) == {b["verts"] for b in theirs}
    for b in theirs:
        m = mine[b["verts"]]
        assert m["reach"] == b["reach"]
        assert m["chains"] == b["chains"]
        assert m["free"] == b["free"]
    assert np.array_equal(arrs["art"], art)
    row, col = oracle().csr(n, u, v)
    assert rel_err(oracle().method_bc_from_decomp(arrs), oracle().brandes(n, row, col)) < 1e-12


def test_packing_invariants():
    G = graphs()
    n, u, v = G.gen_rmat(10, 8, chain_frac=0.2, seed=11)
    arrs = decompose(n, u, v).arrays()
    vo, row, col = arrs["vtx_off"], arrs["row"], arrs["col"]
    sizes = np.diff(vo)
    assert np.all(sizes >= 3) and np.all(np.diff(sizes) <= 0)  # largest first
    for b in range(arrs["n_bcc"]):
        nb = sizes[b]
        seg = col[row[vo[b]]:row[vo[b + 1]]]
        assert seg.min() >= 0 and seg.max() < nb
        for k in range(vo[b], vo[b + 1]):
            adj = col[row[k]:row[k + 1]]
            assert np.all(np.diff(adj) > 0)  # sorted, no duplicates
        c0, c1 = arrs["chain_off"][b], arrs["chain_off"][b + 1]
        assert np.all(np.diff(arrs["chain_l"][c0:c1]) >= 0)  # grouped by owner
        covered = arrs["chain_len"][c0:c1].sum()
        assert covered == nb - arrs["n_plain"][b]
        for c in range(c0, c1):
            s, ln = arrs["chain_start"][c], arrs["chain_len"][c]
            for i in range(ln):  # every chain vertex has degree 2 and sits between its neighbours
                k = vo[b] + s + i
                assert row[k + 1] - row[k] == 2
                prev = arrs["chain_l"][c] if i == 0 else s + i - 1
                nxt = arrs["chain_r"][c] if i == ln - 1 else s + i + 1
                assert set(col[row[k]:row[k + 1]].tolist()) == {prev, nxt}


def test_graph_load_and_errors(tmp_path):
    P = pkg()
    g = P.Graph.load(GOLDEN / "sample1.txt")
    n, row, col = g.csr()
    assert n == 9 and row[-1] == 24
    dup = tmp_path / "dup.txt"
    dup.write_text("4 6\n0 1 1\n1 0 1\n1 1 1\n1 2 1\n2 3 1\n3 2 1\n")
    n, row, col = P.Graph.load(dup).csr()
    assert row.tolist() == [0, 1, 3, 5, 6]  # loop dropped, duplicates merged
    bad = tmp_path / "trunc.txt"
    bad.write_text("5 4\n0 1 1\n1 2 1\n")
    with pytest.raises(P.BcError) as e:
        P.Graph.load(bad)
    assert e.value.code == P.EIO and "truncated" in str(e.value)
    oob = tmp_path / "oob.txt"
    oob.write_text("3 1\n0 7 1\n")
    with pytest.raises(P.BcError) as e:
        P.Graph.load(oob)
    assert e.value.code == P.EIO
    with pytest.raises(P.BcError):
        P.Graph.load(tmp_path / "missing.txt")
    empty = tmp_path / "empty.txt"
    empty.write_text("0 0\n")
    d = P.Decomposition(P.Graph.load(empty))
    assert d.arrays()["n_bcc"] == 0


def test_generators_are_simple_and_seeded():
    G = graphs()
    for gen in (lambda: G.gen_small(1), lambda: G.gen_rmat(9, 8, seed=3), lambda: G.gen_grid(24, leaves=50),
                lambda: G.pack_graphs(G.gen_ba_batch(5, 50, 200))[:3]):
        n, u, v = gen()
        assert np.all(u < v) and len(np.unique(u.astype(np.int64) * n + v)) == len(u)
        n2, u2, v2 = gen()
        assert n == n2 and np.array_equal(u, u2) and np.array_equal(v, v2)
    n, u, v = G.gen_small(1)
    assert n == 2000
    deg = np.bincount(np.concatenate([u, v]), minlength=n)
    assert np.all(deg[1500:] == 2) and np.all(deg[1000:1500] >= 1)


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU failure path")
def test_betc_fails_loudly_without_gpu():
    P = pkg()
    r = subprocess.run([str(P.BETC_PATH), str(GOLDEN / "sample1.txt")], capture_output=True, text=True)
    assert r.returncode == 4 and "CUDA" in r.stderr
    r = subprocess.run([str(P.BETC_PATH), str(GOLDEN / "sample1.txt"), "--gpu-decomp"], capture_output=True, text=True)
    assert r.returncode == 4 and "CUDA" in r.stderr and not r.stdout
    with pytest.raises(P.BcError) as e:
        P.Context()
    assert e.value.code == P.ECUDA
    with pytest.raises(P.BcError) as e:
        P.Decomposition(P.Graph.load(GOLDEN / "sample1.txt"), gpu_device=0)
    assert e.value.code == P.ECUDA


_HASH_SCRIPT = """
import hashlib, sys
sys.path.insert(0, {tests!r})
from helpers import graphs, pkg
P = pkg()
n, u, v = graphs().gen_rmat(16, 16, 0.2, 1, 8, seed=2)
arrs = P.Decomposition(P.Graph.from_edges(n, u, v)).arrays()
h = hashlib.sha256()
for k in sorted(arrs):
    h.update(k.encode())
    h.update(arrs[k].tobytes() if hasattr(arrs[k], "tobytes") else str(arrs[k]).encode())
print(int(arrs["vtx_off"][1]), h.hexdigest())
"""


def test_decomposition_independent_of_thread_count():
    """The decomposition's parallel passes (the BCC split, whose BFS forest
    and union-finds depend on thread timing; arc-to-BCC assignment, packed
    writes; the RMAT-16 giant BCC takes the large-BCC path) give the same
    arrays with 1 and 4 host threads."""
    import os
    import sys
    from pathlib import Path

    script = _HASH_SCRIPT.format(tests=str(Path(__file__).resolve().parent))
    out = []
    for threads in ("1", "4"):
        env = dict(os.environ, OMP_NUM_THREADS=threads)
        r = subprocess.run([sys.executable, "-c", script], env=env, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        out.append(r.stdout.split())
    assert int(out[0][0]) >= 1 << 16  # the giant BCC is written with its vertices in parallel
    assert out[0] == out[1]


_LOAD_SCRIPT = """
import sys
sys.path.insert(0, {tests!r})
from helpers import pkg
P = pkg()
for path in sys.argv[1:]:
    try:
        n, row, col = P.Graph.load(path).csr()
        print("ok", n, row.tolist(), col.tolist())
    except P.BcError as e:
        print("err", e.code, str(e))
"""


def test_graph_load_token_rules_any_thread_count(tmp_path):
    """The parallel parser reads numbers exactly as a sequential scan would
    (whitespace of any kind between them, a leading minus sign, nothing
    after the m-th edge looked at) and reports the first bad edge, with 1,
    3 and 8 host threads (chunk cuts fall in different places)."""
    import os
    import sys
    from pathlib import Path

    cases = {
        "one_line": "4 3 0 1 1 1 2 1 2 3 1",
        "mixed_ws": "4 3\r\n0\t1 1\n\n1  2 1\r\n2 3 1",
        "glued": "4 2\n0 1 1 2-3 1\n",            # '2-3' reads as 2 then -3: out of range at edge 1
        "junk_after": "3 2\n0 1 1\n1 2 1\nthis is ignored",
        "bad_token": "5 3\n0 1 1\n1 x 1\n2 3 1\n",   # edge 1 is incomplete
        "oob_before_trunc": "5 3\n0 9 1\n1 2 1\n2 3",
        "lone_minus": "5 2\n0 1 - 2 3 1\n",   # no digit after the sign: edge 0 is incomplete
        "huge_m": "5 99999999999\n0 1 1\n",     # a header overstating m: truncated, nothing sized from it
    }
    paths = []
    for name, text in cases.items():
        f = tmp_path / f"{name}.txt"
        f.write_text(text)
        paths.append(str(f))
    script = _LOAD_SCRIPT.format(tests=str(Path(__file__).resolve().parent))
    runs = []
    for threads in ("1", "3", "8"):
        env = dict(os.environ, OMP_NUM_THREADS=threads)
        r = subprocess.run([sys.executable, "-c", script] + paths, env=env, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        runs.append(r.stdout.splitlines())
    assert runs[0] == runs[1] == runs[2]
    got = dict(zip(cases, runs[0]))
    path_graph = "ok 4 [0, 1, 3, 5, 6] [1, 0, 2, 1, 3, 2]"
    assert got["one_line"] == path_graph and got["mixed_ws"] == path_graph
    assert got["glued"].startswith("err 5") and "out of range at edge 1" in got["glued"]
    assert got["junk_after"] == "ok 3 [0, 1, 3, 4] [1, 0, 2, 1]"
    assert got["bad_token"].startswith("err 5") and "truncated edge list at edge 1 of 3" in got["bad_token"]
    assert "out of range at edge 0" in got["oob_before_trunc"]
    assert "truncated edge list at edge 0 of 2" in got["lone_minus"]  # the minus sign is edge 0's weight
    assert got["huge_m"].startswith("err 5") and "truncated edge list at edge 1 of 99999999999" in got["huge_m"]


def larger_random_graph(seed):
    """A few hundred vertices: a random core, parallel chains between some
    pairs of its vertices, every edge subdivided with probability 0.3 into
    chains of 1-6, pendant trees, and a second small component."""
    G = graphs()
    rng = np.random.default_rng(1000 + seed)
    n = int(rng.integers(80, 250))
    m = int(rng.integers(n, 3 * n))
    u = rng.integers(0, n, m)
    v = rng.integers(0, n, m)
    a, b = rng.integers(0, n, 2)
    u = np.concatenate([u, [a, a, a]])  # three parallel paths a-x-b after subdivision below
    v = np.concatenate([v, [b, b, b]])
    uu, vv = G.simple_edges(n, u, v)
    n, uu, vv = G.subdivide(n, uu, vv, 0.3, 1, 6, rng)
    for _ in range(3):  # parallel chains: new vertices x between a and b
        uu = np.concatenate([uu, [a, n]]).astype(np.int32)
        vv = np.concatenate([vv, [n, b]]).astype(np.int32)
        n += 1
    n, uu, vv = G.attach_leaves(n, uu, vv, int(rng.integers(5, 40)), n, rng)
    k = n  # a separate 5-cycle with a chord
    uu = np.concatenate([uu, [k, k + 1, k + 2, k + 3, k + 4, k]]).astype(np.int32)
    vv = np.concatenate([vv, [k + 1, k + 2, k + 3, k + 4, k, k + 2]]).astype(np.int32)
    n += 5
    return (n,) + G.simple_edges(n, uu, vv)


@pytest.mark.parametrize("seed", range(12))
def test_larger_decomposition_matches_oracle(seed):
    n, u, v = larger_random_graph(seed)
    P = pkg()
    arrs = P.Decomposition(P.Graph.from_edges(n, u, v)).arrays()
    mine = {b["verts"]: b for b in product_bccs(arrs)}
    theirs, art = _oracle_bccs(n, u, v)
    assert set(mine) == {b["verts"] for b in theirs}
    for b in theirs:
        m = mine[b["verts"]]
        assert m["reach"] == b["reach"] and m["chains"] == b["chains"] and m["free"] == b["free"]
    assert np.array_equal(arrs["art"], art)
    row, col = oracle().csr(n, u, v)
    assert rel_err(oracle().method_bc_from_decomp(arrs), oracle().brandes(n, row, col)) < 1e-12


def wide_level_graph(seed):
    """A component whose BFS forest has a level of more than 2048 vertices
    (vertex 0, the root, adjacent to 2600 others), so the BCC split takes its
    parallel BFS and sweep paths: random edges among the hub's neighbours,
    edges subdivided into chains, pendant trees, and a second, deep component
    (a long cycle with chords)."""
    G = graphs()
    rng = np.random.default_rng(2000 + seed)
    n = 3200
    u = np.concatenate([np.zeros(2600, np.int64), rng.integers(1, n, 1400)])
    v = np.concatenate([np.arange(1, 2601), rng.integers(1, n, 1400)])
    uu, vv = G.simple_edges(n, u, v)
    n, uu, vv = G.subdivide(n, uu, vv, 0.3, 1, 3, rng)
    n, uu, vv = G.attach_leaves(n, uu, vv, 300, n, rng)
    k = n  # a 600-cycle with 40 chords
    cu = np.concatenate([k + np.arange(600), k + rng.integers(0, 600, 40)])
    cv = np.concatenate([k + (np.arange(600) + 1) % 600, k + rng.integers(0, 600, 40)])
    return (n + 600,) + G.simple_edges(n + 600, np.concatenate([uu, cu]), np.concatenate([vv, cv]))


@pytest.mark.parametrize("seed", range(2))
def test_wide_level_decomposition_matches_oracle(seed):
    n, u, v = wide_level_graph(seed)
    P = pkg()
    arrs = P.Decomposition(P.Graph.from_edges(n, u, v)).arrays()
    mine = {b["verts"]: b for b in product_bccs(arrs)}
    theirs, art = _oracle_bccs(n, u, v)
    assert len(theirs) > 10 and set(mine) == {b["verts"] for b in theirs}
    for b in theirs:
        m = mine[b["verts"]]
        assert m["reach"] == b["reach"] and m["chains"] == b["chains"] and m["free"] == b["free"]
    assert np.array_equal(arrs["art"], art)
    row, col = oracle().csr(n, u, v)
    assert rel_err(oracle().method_bc_from_decomp(arrs), oracle().brandes(n, row, col)) < 1e-12


def test_binary_csr_round_trip(tmp_path):
    """A graph saved with bc_graph_save loads back (detected by its magic
    bytes, no text parsing) to the same CSR and the same decomposition."""
    P = pkg()
    G = graphs()
    n, u, v = G.gen_rmat(12, 8, chain_frac=0.2, seed=4)
    g = P.Graph.from_edges(n, u, v)
    path = tmp_path / "g.csr"
    g.save(path)
    h = P.Graph.load(path)
    n1, r1, c1 = g.csr()
    n2, r2, c2 = h.csr()
    assert n1 == n2 and np.array_equal(r1, r2) and np.array_equal(c1, c2)
    a = P.Decomposition(g).arrays()
    b = P.Decomposition(h).arrays()
    assert all(np.array_equal(a[k], b[k]) for k in a)
    empty = P.Graph.from_edges(3, np.zeros(0, np.int32), np.zeros(0, np.int32))
    empty.save(tmp_path / "e.csr")
    assert P.Graph.load(tmp_path / "e.csr").csr()[0] == 3


def test_binary_csr_is_checked(tmp_path):
    """A binary CSR that is not a simple undirected graph, or whose size does
    not match its header, is rejected with the reason."""
    import struct

    P = pkg()

    def write(n, row, col, pad=0, cut=0):
        data = b"BCGCSR1\0" + struct.pack("<iiq", n, pad, len(col)) + struct.pack(f"<{len(row)}q", *row) + \
            struct.pack(f"<{len(col)}i", *col)
        f = tmp_path / "g.csr"
        f.write_bytes(data[:len(data) - cut])
        return f

    def reason(*a, **k):
        with pytest.raises(P.BcError) as e:
            P.Graph.load(write(*a, **k))
        assert e.value.code == P.EIO
        return str(e.value)

    tri = (3, [0, 2, 4, 6], [1, 2, 0, 2, 0, 1])
    assert P.Graph.load(write(*tri)).csr()[0] == 3  # a triangle is fine
    assert "size" in reason(*tri, cut=4)
    assert "header" in reason(*tri, pad=1)
    assert "order" in reason(3, [0, 2, 1, 6], [1, 2, 0, 2, 0, 1])
    assert "not sorted" in reason(3, [0, 2, 4, 6], [2, 1, 0, 2, 0, 1])
    assert "not sorted" in reason(3, [0, 2, 4, 6], [1, 1, 0, 2, 0, 1])  # repeated neighbour
    assert "loop" in reason(2, [0, 1, 2], [0, 1])
    assert "out of range" in reason(2, [0, 1, 2], [1, 7])
    assert "reverse" in reason(3, [0, 1, 1, 1], [1])


def _same_arrays(a, b):
    return all(np.array_equal(a[k], b[k]) if hasattr(a[k], "shape") else a[k] == b[k] for k in a)


def _deep_cycle():
    """A 30000-vertex cycle with 12 chords and 200 pendant leaves: BFS levels
    in the tens of thousands."""
    G = graphs()
    rng = np.random.default_rng(21)
    n = 30000
    u = np.concatenate([np.arange(n), rng.integers(0, n, 12)])
    v = np.concatenate([(np.arange(n) + 1) % n, rng.integers(0, n, 12)])
    uu, vv = G.simple_edges(n, u, v)
    return G.attach_leaves(n, uu, vv, 200, n, rng)


@pytest.mark.parametrize("family", ["random", "larger", "wide", "rmat16", "grid", "deep"])
def test_gpu_decomposition_steps_on_host_equal_bc_decompose(family):
    """bc_decompose_gpu's data-parallel steps (union-find components, BFS
    forest, level sweeps, union-find over tree edges, member slots, the
    exact-order BFS of every BCC at once, chain numbering, packed CSR), run
    as host loops (device -1), give exactly bc_decompose's packed arrays."""
    P = pkg()
    G = graphs()
    cases = {
        "random": lambda: [random_graph(s)[:3] for s in range(0, 40, 3)],
        "larger": lambda: [larger_random_graph(s) for s in range(12)],
        "wide": lambda: [wide_level_graph(s) for s in range(2)],
        "rmat16": lambda: [G.gen_rmat(16, 16, 0.2, 1, 8, seed=2)],
        "grid": lambda: [G.gen_grid(seed=3)],
        "deep": lambda: [_deep_cycle()],
    }[family]()
    for n, u, v in cases:
        g = P.Graph.from_edges(n, u, v)
        assert _same_arrays(P.Decomposition(g).arrays(), P.Decomposition(g, gpu_device=-1).arrays())


@pytest.mark.parametrize("which", ["rmat16", "grid"])
def test_packed_plain_order_is_the_sequential_bfs(which):
    """The largest BCC's plain vertices are numbered in the order of a plain
    sequential queue BFS from its max-degree vertex (smallest vertex id among
    equals), neighbours visited in increasing vertex id -- recomputed here in
    Python, independently of the library's level-synchronous, top-down or
    bottom-up BFS (RMAT-16: 850k vertices, wide levels; the grid: deep)."""
    from collections import deque

    G = graphs()
    n, u, v = G.gen_rmat(16, 16, 0.2, 1, 8, seed=2) if which == "rmat16" else G.gen_grid(seed=3)
    a = decompose(n, u, v).arrays()
    v0, v1 = int(a["vtx_off"][0]), int(a["vtx_off"][1])
    nb = v1 - v0
    R = a["row"][v0:v1 + 1] - a["row"][v0]
    C = a["col"][a["row"][v0]:a["row"][v1]]
    o = a["orig"][v0:v1]
    deg = np.diff(R)
    rid = np.repeat(np.arange(nb), deg)
    Cs = C[np.lexsort((o[C], rid))]  # each row by increasing original id
    cands = np.flatnonzero(deg == deg.max())
    root = int(cands[np.argmin(o[cands])])
    seen = np.zeros(nb, bool)
    seen[root] = True
    q, order = deque([root]), []
    Rl, Cl = R.tolist(), Cs.tolist()
    while q:
        x = q.popleft()
        order.append(x)
        for y in Cl[Rl[x]:Rl[x + 1]]:
            if not seen[y]:
                seen[y] = True
                q.append(y)
    order = np.array(order)
    assert len(order) == nb and root == 0
    assert np.array_equal(order[deg[order] != 2], np.arange(int(a["n_plain"][0])))


def _cactus(count, rng):
    """count cycles of 3-30 vertices, most hung off a vertex of an earlier cycle."""
    us, vs, base = [], [], 0
    for c in range(count):
        k = int(rng.integers(3, 31))
        cyc = base + np.arange(k)
        us.append(cyc)
        vs.append(np.r_[cyc[1:], cyc[0]])
        if c and c % 7:
            us.append([int(rng.integers(0, base))])
            vs.append([base + int(rng.integers(0, k))])
        base += k
    return (base,) + graphs().simple_edges(base, np.concatenate(us), np.concatenate(vs))


@pytest.mark.parametrize("which", ["sparse", "ba", "cactus"])
def test_bccs_and_articulations_match_networkx(which):
    """BCC vertex sets (>= 3 vertices) and articulation points at sizes that
    take the split's parallel paths, against networkx's independent
    biconnected_components / articulation_points."""
    import networkx as nx

    G = graphs()
    rng = np.random.default_rng(11)
    if which == "sparse":  # random sparse core with chains and leaves: many bridges and cut vertices
        n = 60000
        u, v = G.simple_edges(n, rng.integers(0, n, int(1.3 * n)), rng.integers(0, n, int(1.3 * n)))
        n, u, v = G.subdivide(n, u, v, 0.2, 1, 4, rng)
        n, u, v = G.attach_leaves(n, u, v, 3000, n, rng)
    elif which == "ba":
        n, u, v = G.pack_graphs(G.gen_ba_batch(64, 50, 2000, seed=5))[:3]
    else:
        n, u, v = _cactus(3000, rng)
    a = decompose(n, u, v).arrays()
    g = nx.Graph()
    g.add_nodes_from(range(n))
    g.add_edges_from(zip(u.tolist(), v.tolist()))
    theirs = {frozenset(c) for c in nx.biconnected_components(g) if len(c) >= 3}
    vo, orig = a["vtx_off"], a["orig"]
    assert {frozenset(orig[vo[b]:vo[b + 1]].tolist()) for b in range(a["n_bcc"])} == theirs
    assert set(np.flatnonzero(a["art"] > 0).tolist()) == set(nx.articulation_points(g))


def test_reach_matches_components_of_g_minus_x():
    """Reach and articulation terms at scale, independently: for sampled
    members x of the largest BCC b of a sparse graph with chains and leaves,
    reach_b(x) = the number of vertices in the components of G - x next to x
    that hold no other vertex of b, and art(x) = S^2 - sum(part^2) over those
    components (S their total) -- scipy's connected components of G
    without x."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import connected_components

    G = graphs()
    rng = np.random.default_rng(12)
    n = 40000
    u, v = G.simple_edges(n, rng.integers(0, n, int(1.3 * n)), rng.integers(0, n, int(1.3 * n)))
    n, u, v = G.subdivide(n, u, v, 0.2, 1, 4, rng)
    n, u, v = G.attach_leaves(n, u, v, 3000, n, rng)
    a = decompose(n, u, v).arrays()
    v0, v1 = int(a["vtx_off"][0]), int(a["vtx_off"][1])
    members, reach = a["orig"][v0:v1], a["reach"][v0:v1]
    A = csr_matrix((np.ones(2 * len(u)), (np.r_[u, v], np.r_[v, u])), shape=(n, n))
    cut = np.flatnonzero(a["art"][members] > 0)
    picks = np.r_[rng.choice(cut, 24, replace=False), rng.choice(np.flatnonzero(a["art"][members] == 0), 6)]
    for k in picks:
        x = int(members[k])
        keep = np.ones(n, bool)
        keep[x] = False
        idx = np.flatnonzero(keep)
        _, lab = connected_components(A[idx][:, idx], directed=False)
        full = np.full(n, -1)
        full[idx] = lab
        sizes = np.bincount(lab)
        near = set(full[A.indices[A.indptr[x]:A.indptr[x + 1]]].tolist())
        in_b = set(full[members[members != x]].tolist())
        assert reach[k] == sum(int(sizes[c]) for c in near - in_b), x
        parts = [int(sizes[c]) for c in near]  # the component of x, less x, in pieces
        assert a["art"][x] == sum(parts) ** 2 - sum(p * p for p in parts), x
    assert np.all(reach[cut] > 0)
