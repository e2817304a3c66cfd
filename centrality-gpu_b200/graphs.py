"""Seeded synthetic graphs standing in for the workloads the engine is measured on,
plus the reference's edge-list file format.

Every generator returns ``(n, u, v)``: the vertex count and two int32 arrays
holding each undirected edge once, with no self loops and no duplicates
(the reference's BFS assumes a simple graph, Codes/kernels_free.cu:248).

Edge-list format (reference Codes/graph.cpp:38-59, Codes/ReadMe:6-13):
first line ``n m``, then ``m`` lines ``u v w`` with 0-based ids and w = 1.
"""
from __future__ import annotations

import numpy as np


def simple_edges(n: int, u, v):
    """Drop self loops and duplicate undirected edges; canonical u < v, sorted."""
    u = np.asarray(u, dtype=np.int64)
    v = np.asarray(v, dtype=np.int64)
    keep = u != v
    u, v = u[keep], v[keep]
    lo = np.minimum(u, v)
    hi = np.maximum(u, v)
    key = np.sort(lo * np.int64(n) + hi)
    if len(key):
        key = key[np.concatenate(([True], key[1:] != key[:-1]))]
    return (key // n).astype(np.int32), (key % n).astype(np.int32)


def subdivide(n: int, u, v, frac: float, lo: int, hi: int, rng, exact: bool = True):
    """Replace a random subset of edges by paths through new degree-2 vertices.

    ``exact``: subdivide exactly round(frac * m) edges; otherwise each edge
    independently with probability ``frac``. Chain lengths are uniform in
    [lo, hi] new vertices.
    """
    m = len(u)
    if exact:
        pick = np.zeros(m, dtype=bool)
        pick[rng.permutation(m)[: int(round(frac * m))]] = True
    else:
        pick = rng.random(m) < frac
    su, sv = u[pick].astype(np.int64), v[pick].astype(np.int64)
    k = rng.integers(lo, hi + 1, size=len(su))
    total = int(k.sum())
    # chain i owns new vertices first[i] .. first[i]+k[i]-1
    first = n + np.concatenate(([0], np.cumsum(k)[:-1])) if len(k) else np.zeros(0, np.int64)
    owner = np.repeat(np.arange(len(su)), k)
    new_ids = n + np.arange(total, dtype=np.int64)
    pos = new_ids - first[owner] if total else new_ids
    # edge into each new vertex from its predecessor on the chain
    prev = np.where(pos == 0, su[owner] if total else su, new_ids - 1)
    last = first + k - 1
    eu = np.concatenate([u[~pick].astype(np.int64), prev, last])
    ev = np.concatenate([v[~pick].astype(np.int64), new_ids, sv])
    n2 = n + total
    return (n2,) + simple_edges(n2, eu, ev)


def attach_leaves(n: int, u, v, count: int, targets: int, rng):
    """Attach ``count`` new pendant vertices to uniform random vertices in [0, targets)."""
    t = rng.integers(0, targets, size=count)
    new = n + np.arange(count, dtype=np.int64)
    n2 = n + count
    return (n2,) + simple_edges(n2, np.concatenate([u, t]), np.concatenate([v, new]))


def gen_small(seed: int = 1):
    """2,000 vertices: a 1,000-vertex core where each vertex links to 3 uniform
    others, 500 pendants on uniform core vertices, and 100 chains of 5
    degree-2 vertices each spliced between two distinct uniform core vertices."""
    rng = np.random.default_rng(seed)
    core = 1000
    a = np.repeat(np.arange(core), 3)
    b = rng.integers(0, core, size=3 * core)
    eu, ev = [a], [b]
    n = core
    pend = rng.integers(0, core, size=500)
    eu.append(pend)
    ev.append(n + np.arange(500))
    n += 500
    for _ in range(100):
        x = int(rng.integers(0, core))
        y = int(rng.integers(0, core - 1))
        y = y + 1 if y >= x else y
        path = [x] + list(range(n, n + 5)) + [y]
        eu.append(np.array(path[:-1]))
        ev.append(np.array(path[1:]))
        n += 5
    return (n,) + simple_edges(n, np.concatenate(eu), np.concatenate(ev))


def rmat_edges(scale: int, edge_factor: int, a: float, b: float, c: float, rng, chunk: int = 1 << 22):
    """R-MAT endpoints (before symmetrising): edge_factor * 2^scale pairs."""
    m = edge_factor << scale
    us, vs = [], []
    ab, abc = a + b, a + b + c
    for start in range(0, m, chunk):
        cnt = min(chunk, m - start)
        u = np.zeros(cnt, dtype=np.int64)
        v = np.zeros(cnt, dtype=np.int64)
        for bit in range(scale):
            r = rng.random(cnt, dtype=np.float32)
            ubit = r >= ab                       # quadrants c, d
            vbit = ((r >= a) & (r < ab)) | (r >= abc)  # quadrants b, d
            u |= ubit.astype(np.int64) << bit
            v |= vbit.astype(np.int64) << bit
        us.append(u)
        vs.append(v)
    return np.concatenate(us), np.concatenate(vs)


def gen_rmat(scale: int = 16, edge_factor: int = 16, chain_frac: float = 0.2, chain_lo: int = 1,
             chain_hi: int = 8, seed: int = 2, a: float = 0.57, b: float = 0.19, c: float = 0.19):
    """R-MAT(a,b,c,d=1-a-b-c), symmetrised, deduplicated, loops removed; then
    ``chain_frac`` of the remaining edges subdivided into chains of uniform
    length chain_lo..chain_hi."""
    rng = np.random.default_rng(seed)
    n = 1 << scale
    u, v = rmat_edges(scale, edge_factor, a, b, c, rng)
    u, v = simple_edges(n, u, v)
    return subdivide(n, u, v, chain_frac, chain_lo, chain_hi, rng)


def gen_grid(side: int = 512, delete_frac: float = 0.1, sub_p: float = 0.3, sub_lo: int = 1, sub_hi: int = 4,
             leaves: int = 15000, seed: int = 3):
    """side x side 4-neighbour grid, delete_frac of edges removed uniformly,
    each survivor subdivided with probability sub_p by sub_lo..sub_hi
    degree-2 vertices, then ``leaves`` pendants on uniform grid vertices."""
    rng = np.random.default_rng(seed)
    idx = np.arange(side * side, dtype=np.int64).reshape(side, side)
    hu, hv = idx[:, :-1].ravel(), idx[:, 1:].ravel()
    vu, vv = idx[:-1, :].ravel(), idx[1:, :].ravel()
    u = np.concatenate([hu, vu])
    v = np.concatenate([hv, vv])
    m = len(u)
    keep = np.ones(m, dtype=bool)
    keep[rng.permutation(m)[: int(round(delete_frac * m))]] = False
    n = side * side
    u, v = simple_edges(n, u[keep], v[keep])
    n, u, v = subdivide(n, u, v, sub_p, sub_lo, sub_hi, rng, exact=False)
    return attach_leaves(n, u, v, leaves, side * side, rng)


def gen_ba(n: int, m: int, rng):
    """Barabasi-Albert preferential attachment: start from a clique on m+1
    vertices; each new vertex links to m distinct earlier vertices chosen with
    probability proportional to degree."""
    eu = []
    ev = []
    rep = []  # every edge endpoint once: sampling from it is degree-proportional
    for i in range(m + 1):
        for j in range(i):
            eu.append(j)
            ev.append(i)
            rep += [i, j]
    rep = np.array(rep + [0] * (2 * m * max(n - m - 1, 0)), dtype=np.int64)
    fill = 2 * (m * (m + 1) // 2)
    draws = rng.integers(0, 1 << 62, size=(max(n - m - 1, 0), 4 * m))
    for t in range(m + 1, n):
        chosen = []
        row = draws[t - m - 1]
        k = 0
        while len(chosen) < m:
            if k < len(row):
                x = int(rep[row[k] % fill])
            else:
                x = int(rep[int(rng.integers(0, fill))])
            k += 1
            if x not in chosen:
                chosen.append(x)
        for x in chosen:
            eu.append(x)
            ev.append(t)
            rep[fill] = x
            rep[fill + 1] = t
            fill += 2
    return (n,) + simple_edges(n, np.array(eu), np.array(ev))


def gen_ba_batch(count: int = 4096, n_lo: int = 50, n_hi: int = 5000, m: int = 2, chain_frac: float = 0.1,
                 chain_lo: int = 1, chain_hi: int = 3, seed: int = 4):
    """``count`` independent graphs: BA(m) with n log-uniform in [n_lo, n_hi],
    chain_frac of each graph's edges subdivided into chains of chain_lo..chain_hi,
    then n/10 pendant leaves. Returns a list of (n, u, v)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), size=count)).astype(np.int64)
    out = []
    for n0 in sizes:
        n, u, v = gen_ba(int(n0), m, rng)
        n, u, v = subdivide(n, u, v, chain_frac, chain_lo, chain_hi, rng)
        n, u, v = attach_leaves(n, u, v, int(n0) // 10, int(n0), rng)
        out.append((n, u, v))
    return out


def pack_graphs(graphs):
    """Disjoint union of independent graphs (vertex ids offset per graph).
    Returns (n, u, v, vertex_offsets)."""
    offs = [0]
    us, vs = [], []
    for n, u, v in graphs:
        us.append(u.astype(np.int64) + offs[-1])
        vs.append(v.astype(np.int64) + offs[-1])
        offs.append(offs[-1] + n)
    return offs[-1], np.concatenate(us).astype(np.int32), np.concatenate(vs).astype(np.int32), np.array(offs)


def write_edge_list(path, n: int, u, v):
    """Writes the reference's input format (w = 1)."""
    with open(path, "w") as f:
        f.write(f"{n} {len(u)}\n")
        np.savetxt(f, np.stack([u, v, np.ones_like(u)], axis=1), fmt="%d")


def read_edge_list(path):
    """Reads the reference's input format; returns (n, u, v) as given (not deduplicated)."""
    with open(path) as f:
        head = f.readline().split()
        n, m = int(head[0]), int(head[1])
        data = np.loadtxt(f, dtype=np.int64, ndmin=2)
    data = data[:m]
    return n, data[:, 0].astype(np.int32), data[:, 1].astype(np.int32)
