"""Regenerates the golden fixtures in this directory. Needs the reference
checkout (read-only) and oracle/_ref/refdump (make -C oracle/ref); run here,
never on the GPU box:

    python tests/golden/make_golden.py /path/to/reference

For every graph it writes
  <name>.txt      the input in the reference's edge-list format
  <name>.ref.txt  what the reference's own host pipeline hands to its GPU
                  entry points (BCCs, reach, free set, ears) and its
                  articulation terms -- produced by running the reference's
                  C++ host code (oracle/ref/Makefile)
  <name>.bc.json  exact BC (ordered pairs) from networkx's independent Brandes
                  (networkx.betweenness_centrality(normalized=False) x 2)
Graphs: the reference's four sample inputs (Codes/sample_input/test1-4.txt)
and seeded connected graphs with chains, pendants, parallel chains and cycle
blocks.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import networkx as nx
import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "centrality-gpu_b200"))
import graphs  # noqa: E402

REFDUMP = ROOT / "oracle" / "_ref" / "refdump"


def connected_graph(rng, n, extra, sub_frac, leaves, cycles):
    """Random spanning tree + extra edges, some edges subdivided, pendant
    leaves and pendant cycles (blocks that are a single cycle)."""
    parent = [int(rng.integers(0, i)) for i in range(1, n)]
    u = list(range(1, n))
    v = parent
    eu = np.array(u + list(rng.integers(0, n, extra)), dtype=np.int64)
    ev = np.array(v + list(rng.integers(0, n, extra)), dtype=np.int64)
    eu, ev = graphs.simple_edges(n, eu, ev)
    n, eu, ev = graphs.subdivide(n, eu, ev, sub_frac, 1, 4, rng)
    us, vs = [eu], [ev]
    for _ in range(cycles):  # a cycle of 3..6 new vertices hanging off one vertex
        a = int(rng.integers(0, n))
        k = int(rng.integers(2, 6))
        ring = [a] + list(range(n, n + k))
        n += k
        us.append(np.array(ring))
        vs.append(np.array(ring[1:] + ring[:1]))
    eu, ev = np.concatenate(us), np.concatenate(vs)
    eu, ev = graphs.simple_edges(n, eu, ev)
    return graphs.attach_leaves(n, eu, ev, leaves, n, rng)


def parallel_chains(rng):
    """Two hubs joined by several chains of equal and unequal length (the
    reference merges parallel ears, Codes/readeardata.cpp:50-100)."""
    edges = [(0, 1), (0, 2), (1, 2), (2, 3), (3, 0)]
    n = 4
    for length in (2, 2, 3, 1):
        path = [0] + list(range(n, n + length)) + [1]
        n += length
        edges += list(zip(path[:-1], path[1:]))
    e = np.array(edges)
    return (n,) + graphs.simple_edges(n, e[:, 0], e[:, 1])


def main(ref_root: str):
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle" / "ref"), f"REF={ref_root}/Codes"], check=True)
    cases = {}
    for t in range(1, 5):
        cases[f"sample{t}"] = graphs.read_edge_list(f"{ref_root}/Codes/sample_input/test{t}.txt")
    rng = np.random.default_rng(20261203)
    for k in range(6):
        cases[f"rand{k}"] = connected_graph(rng, int(rng.integers(8, 40)), int(rng.integers(2, 30)),
                                            0.3, int(rng.integers(0, 6)), int(rng.integers(0, 3)))
    cases["parallel"] = parallel_chains(rng)
    cases["small2000"] = graphs.gen_small(1)
    for name, (n, u, v) in cases.items():
        graphs.write_edge_list(HERE / f"{name}.txt", n, u, v)
        with tempfile.TemporaryDirectory() as tmp:  # the reference writes debug files to its CWD
            env = dict(os.environ, REFDUMP_OUT=str(HERE / f"{name}.ref.txt"))
            subprocess.run([str(REFDUMP), str(HERE / f"{name}.txt")], cwd=tmp, env=env, check=True,
                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        g = nx.Graph()
        g.add_nodes_from(range(n))
        g.add_edges_from(zip(np.asarray(u).tolist(), np.asarray(v).tolist()))
        bc = nx.betweenness_centrality(g, normalized=False)
        (HERE / f"{name}.bc.json").write_text(json.dumps({"n": int(n), "m": int(len(u)), "source": "networkx "
                                                          + nx.__version__, "bc": [2.0 * bc[i] for i in range(n)]}))
        print(name, n, len(u))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference checkout (the directory holding Codes/)>")
    main(sys.argv[1])
