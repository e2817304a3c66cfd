"""The oracle pinned before it is trusted: against networkx's independent
Brandes (BC values) and against the reference's own host pipeline run on the
same graphs (decomposition: BCCs, reach, articulation terms, chains, free
sets). CPU only."""
import numpy as np
import pytest

from helpers import GOLDEN_CASES, canonical_chains, graphs, load_case, oracle, pkg, rel_err


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_brandes_matches_networkx(name):
    O = oracle()
    n, u, v, bc, _ = load_case(name)
    row, col = O.csr(n, u, v)
    assert rel_err(O.brandes(n, row, col), bc) < 1e-12


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_method_matches_networkx(name):
    """The restated reference method (BCC split, reach weights, chain merge,
    articulation terms) gives exact BC."""
    n, u, v, bc, _ = load_case(name)
    assert rel_err(oracle().method_bc(n, u, v), bc) < 1e-12


def _oracle_bccs(n, u, v):
    """Brute-force decomposition in the reference dump's terms."""
    O = oracle()
    nb, eb, art = O.decompose(n, u, v)
    out = []
    for b in range(nb):
        sel = eb == b
        verts = set(u[sel].tolist()) | set(v[sel].tolist())
        if len(verts) <= 2:
            continue
        r = O.reach(n, u, v, eb, b)
        deg = {x: 0 for x in verts}
        adj = {x: [] for x in verts}
        for a, c in zip(u[sel].tolist(), v[sel].tolist()):
            deg[a] += 1
            deg[c] += 1
            adj[a].append(c)
            adj[c].append(a)
        cycle = all(d == 2 for d in deg.values())
        chains, seen = [], set()
        if not cycle:
            for x in sorted(verts):
                if deg[x] == 2:
                    continue
                for y in adj[x]:
                    if deg[y] != 2 or y in seen:
                        continue
                    path, prev, cur = [], x, y
                    while deg[cur] == 2:
                        seen.add(cur)
                        path.append(cur)
                        nxt = adj[cur][0] if adj[cur][1] == prev else adj[cur][1]
                        prev, cur = cur, nxt
                    chains.append((x, cur, [(i + 1, p, len(path) - i) for i, p in enumerate(path)]))
        ends = {c[0] for c in chains} | {c[1] for c in chains}
        out.append({"verts": frozenset(verts), "reach": {x: int(r[x]) for x in verts},
                    "free": set(verts) - seen - ends, "chains": canonical_chains(chains)})
    return out, art


def chain_members(chains):
    """{frozenset(endpoints): set(chain vertices)} (parallel chains merged, as the
    reference merges parallel ears, Codes/readeardata.cpp:50-100)."""
    out = {}
    for node, ends in chains.items():
        key = frozenset(e for e, _ in ends)
        out.setdefault(key, set()).add(node)
    return out


def chain_distances(u, v, chains):
    """Independent distances of each chain vertex to its two endpoints: BFS
    inside the subgraph induced by the vertex's chain plus one endpoint."""
    import networkx as nx
    g = nx.Graph()
    g.add_edges_from(zip(np.asarray(u).tolist(), np.asarray(v).tolist()))
    members = chain_members(chains)
    out = {}
    for ends, nodes in members.items():
        for e in ends:
            other = [x for x in ends if x != e]
            sub = g.subgraph(set(nodes) | {e})
            dist = nx.single_source_shortest_path_length(sub, e)
            for x in nodes:
                out.setdefault(x, set()).add((e, dist.get(x, -1)))
    return {x: frozenset(s) for x, s in out.items()}


def compare_to_reference(bccs, art, ref, u, v):
    """Exact match of BCC vertex sets, reach, free sets, chain membership and
    articulation terms. Chain distances are checked against an independent
    BFS; returns the chain vertices whose distances the REFERENCE gets wrong
    (its preSum, Codes/bcc_bfs.cpp:100-236, mis-orients or mis-measures some
    ears)."""
    by_verts = {b["verts"]: b for b in bccs}
    assert len(by_verts) == len(ref["bccs"])
    ref_defects = []
    for rb in ref["bccs"]:
        verts = frozenset(rb["reach"])
        assert verts in by_verts, f"reference BCC {sorted(verts)} missing"
        mine = by_verts[verts]
        assert mine["reach"] == rb["reach"]
        theirs = canonical_chains(rb["ears"])
        assert chain_members(mine["chains"]) == chain_members(theirs)
        truth = chain_distances(u, v, mine["chains"])
        assert mine["chains"] == truth
        ref_defects += sorted(x for x in theirs if theirs[x] != truth[x])
        assert mine["free"] == set(rb["free"])
    nz = {int(i): float(a) for i, a in enumerate(art) if a != 0}
    assert nz == ref["art"]
    return ref_defects


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_decomposition_matches_reference(name):
    n, u, v, _, ref = load_case(name)
    bccs, art = _oracle_bccs(n, u, v)
    defects = compare_to_reference(bccs, art, ref, u, v)
    if name.startswith("sample"):  # the reference's own inputs: its ears are right there
        assert defects == []


def test_rows_of_chain_vertex_equal_bfs():
    """Merged rows of a chain vertex equal a BFS from it (levels and counts)."""
    P = graphs()
    from helpers import pkg
    O = oracle()
    n, u, v = P.gen_small(3)
    d = pkg().Decomposition(pkg().Graph.from_edges(n, u, v))
    arrs = d.arrays()
    b = 0
    v0, v1 = int(arrs["vtx_off"][b]), int(arrs["vtx_off"][b + 1])
    row = arrs["row"][v0:v1 + 1] - arrs["row"][v0]
    col = arrs["col"][arrs["row"][v0]:arrs["row"][v1]]
    npl = int(arrs["n_plain"][b])
    for s in list(range(npl, v1 - v0))[:60] + [0, 1]:
        dm, sm = O.bcc_source_rows(arrs, b, s)
        db, sb = O.bfs_rows(v1 - v0, row, col, s)
        assert np.array_equal(dm, db)
        assert np.array_equal(sm, sb)


def test_linear_decomposition_equals_brute_force():
    """orc_decompose_linear (Hopcroft-Tarjan, DFS subtree sizes) gives
    orc_decompose's BCC ids and articulation terms, and orc_pack_bcc the
    reach of orc_reach, on random graphs with chains, leaves, isolated
    vertices and several components; BC through the linear packing equals
    Brandes."""
    G = graphs()
    O = oracle()
    rng = np.random.default_rng(7)
    for t in range(150):
        n = int(rng.integers(1, 70))
        m = int(rng.integers(0, 3 * n + 1))
        u, v = G.simple_edges(n, rng.integers(0, n, m), rng.integers(0, n, m))
        if len(u) and t % 2 == 0:
            n, u, v = G.subdivide(n, u, v, 0.3, 1, 4, rng)
            n, u, v = G.attach_leaves(n, u, v, int(rng.integers(0, 10)), n, rng)
        nb, eb, art = O.decompose(n, u, v)
        nl, el, artl = O.decompose_linear(n, u, v)
        assert nb == nl and np.array_equal(eb, el) and np.array_equal(art, artl), t
        bc = artl.copy()
        for b in range(nl):
            pk = O.pack_bcc(n, u, v, el, b)
            r = np.full(n, -1)
            r[pk["orig"]] = pk["reach"]
            assert np.array_equal(r, O.reach(n, u, v, eb, b)), (t, b)
            if pk["n_packed"] >= 3:
                np.add.at(bc, pk["orig"], O.bcc_sources(pk, 0, np.arange(pk["n_packed"], dtype=np.int32)))
        row, col = O.csr(n, u, v)
        want = O.brandes(n, row, col)
        assert np.max(np.abs(bc - want) / np.maximum(1.0, np.abs(want)), initial=0.0) < 1e-12, t


def test_linear_packing_of_the_largest_bcc_matches_the_product():
    """RMAT scale 14 with chains: the oracle's own packing of the largest BCC
    has the product's vertex set, core size, chain count and per-vertex
    reach."""
    G = graphs()
    O = oracle()
    P = pkg()
    n, u, v = G.gen_rmat(14, 16, 0.2, 1, 8, seed=3)
    nbcc, eb, _ = O.decompose_linear(n, u, v)
    pk = O.pack_bcc(n, u, v, eb, int(np.argmax(np.bincount(eb))))
    a = P.Decomposition(P.Graph.from_edges(n, u, v)).arrays()
    v1 = int(a["vtx_off"][1])
    assert int(pk["n_packed"]) == v1 and int(pk["n_plain"][0]) == int(a["n_plain"][0])
    assert len(pk["chain_len"]) == int(a["chain_off"][1])
    assert np.array_equal(np.sort(pk["orig"]), np.sort(a["orig"][:v1]))
    mine = dict(zip(a["orig"][:v1].tolist(), a["reach"][:v1].tolist()))
    assert all(mine[int(x)] == int(r) for x, r in zip(pk["orig"], pk["reach"]))
