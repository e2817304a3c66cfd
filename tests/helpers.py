"""Shared test helpers: load the package from its hyphenated directory, the
oracle, and the golden fixtures."""
from __future__ import annotations

import importlib.util
import json
import sys
from functools import lru_cache
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


@lru_cache(maxsize=1)
def pkg():
    name = "centrality_gpu_b200"
    if name in sys.modules:
        return sys.modules[name]
    d = ROOT / "centrality-gpu_b200"
    spec = importlib.util.spec_from_file_location(name, d / "__init__.py", submodule_search_locations=[str(d)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def graphs():
    pkg()
    from centrality_gpu_b200 import graphs as g
    return g


def oracle():
    from oracle import oracle as O
    return O


GOLDEN_CASES = sorted(p.name[:-len(".bc.json")] for p in GOLDEN.glob("*.bc.json"))


def load_case(name):
    """(n, u, v) simple edges, golden BC (networkx), parsed reference dump."""
    g = graphs()
    n, u, v = g.read_edge_list(GOLDEN / f"{name}.txt")
    u, v = g.simple_edges(n, u, v)
    bc = np.array(json.loads((GOLDEN / f"{name}.bc.json").read_text())["bc"])
    ref = oracle().parse_refdump(GOLDEN / f"{name}.ref.txt")
    return n, u, v, bc, ref


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.size == 0:
        return 0.0
    return float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b))))


def canonical_chains(chains):
    """node -> frozenset{(endpoint, distance)} from (l, r, [(ld, node, rd), ...])."""
    out = {}
    for l, r, trip in chains:
        for ld, node, rd in trip:
            out[node] = frozenset({(l, ld), (r, rd)})
    return out


def product_bccs(arrs):
    """Per packed BCC: vertex set, reach map, free set and canonical chains, in original ids."""
    res = []
    for b in range(arrs["n_bcc"]):
        v0, v1 = int(arrs["vtx_off"][b]), int(arrs["vtx_off"][b + 1])
        orig = arrs["orig"][v0:v1]
        reach = {int(orig[k]): int(arrs["reach"][v0 + k]) for k in range(v1 - v0)}
        chains = []
        ends = set()
        for c in range(int(arrs["chain_off"][b]), int(arrs["chain_off"][b + 1])):
            s, ln = int(arrs["chain_start"][c]), int(arrs["chain_len"][c])
            l, r = int(orig[arrs["chain_l"][c]]), int(orig[arrs["chain_r"][c]])
            ends |= {l, r}
            chains.append((l, r, [(i + 1, int(orig[s + i]), ln - i) for i in range(ln)]))
        npl = int(arrs["n_plain"][b])
        free = {int(orig[k]) for k in range(npl)} - ends
        res.append({"verts": frozenset(int(x) for x in orig), "reach": reach, "free": free,
                    "chains": canonical_chains(chains)})
    return res


def has_gpu():
    try:
        ctx = pkg().Context()
        ctx.close()
        return True
    except Exception:
        return False
