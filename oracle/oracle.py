"""ORACLE — test infrastructure only. ctypes wrapper of oracle/_build/liboracle.so
(the C restatement in bc_oracle.c). Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg may use it, as the checker; the product library
never does.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SO = HERE / "_build" / "liboracle.so"
REFDUMP = HERE / "_ref" / "refdump"

_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)
_lib = None


def build():
    """Compiles liboracle.so (gcc + OpenMP)."""
    r = subprocess.run(["make", "-s", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return SO


def lib():
    global _lib
    if _lib is None:
        if not SO.exists():
            build()
        L = C.CDLL(str(SO))
        L.orc_brandes.argtypes = [C.c_int32, _i64p, _i32p, _i32p, C.c_int64, C.c_int, _f64p]
        L.orc_bfs_rows.argtypes = [C.c_int32, _i64p, _i32p, C.c_int32, _i32p, _f64p]
        L.orc_decompose.argtypes = [C.c_int32, C.c_int64, _i32p, _i32p, _i32p, _f64p]
        L.orc_decompose.restype = C.c_int32
        L.orc_reach.argtypes = [C.c_int32, C.c_int64, _i32p, _i32p, _i32p, C.c_int32, _i32p]
        L.orc_method_bc.argtypes = [C.c_int32, C.c_int64, _i32p, _i32p, C.c_int, _f64p]
        L.orc_method_bc.restype = C.c_int32
        L.orc_bcc_sources.argtypes = [C.c_int32, _i64p, _i32p, _i32p, C.c_int32, _i32p, _i32p, _i32p, _i32p, _i32p,
                                      C.c_int64, C.c_int, _f64p]
        L.orc_bcc_source_rows.argtypes = [C.c_int32, _i64p, _i32p, C.c_int32, _i32p, _i32p, _i32p, _i32p, C.c_int32,
                                          _i32p, _f64p]
        L.orc_decompose_linear.argtypes = [C.c_int32, C.c_int64, _i32p, _i32p, _i32p, _f64p]
        L.orc_decompose_linear.restype = C.c_int32
        L.orc_bcc_size.argtypes = [C.c_int64, _i32p, _i32p, _i32p, C.c_int32, C.c_int32, _i32p, _i64p]
        L.orc_pack_bcc.argtypes = [C.c_int32, C.c_int64, _i32p, _i32p, _i32p, C.c_int32, _i32p, _i64p, _i32p, _i32p,
                                   _i32p, _i32p, _i32p, _i32p]
        L.orc_pack_bcc.restype = C.c_int32
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def csr(n, u, v):
    """CSR (int64 rows, int32 sorted cols) of an undirected simple edge list."""
    u = np.asarray(u, dtype=np.int64)
    v = np.asarray(v, dtype=np.int64)
    src = np.concatenate([u, v])
    dst = np.concatenate([v, u])
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    row = np.zeros(n + 1, dtype=np.int64)
    np.add.at(row, src + 1, 1)
    return np.cumsum(row), dst.astype(np.int32)


def brandes(n, row, col, sources=None, nthreads=0):
    """Ground-truth BC (ordered pairs, FP64) from the listed sources (all if None)."""
    row = np.ascontiguousarray(row, dtype=np.int64)
    col = np.ascontiguousarray(col, dtype=np.int32)
    out = np.zeros(n, dtype=np.float64)
    if sources is None:
        lib().orc_brandes(n, _p(row, _i64p), _p(col, _i32p), None, 0, nthreads, _p(out, _f64p))
    else:
        s = np.ascontiguousarray(sources, dtype=np.int32)
        lib().orc_brandes(n, _p(row, _i64p), _p(col, _i32p), _p(s, _i32p), len(s), nthreads, _p(out, _f64p))
    return out


def bfs_rows(n, row, col, s):
    d = np.zeros(n, dtype=np.int32)
    sig = np.zeros(n, dtype=np.float64)
    lib().orc_bfs_rows(n, _p(np.ascontiguousarray(row, np.int64), _i64p), _p(np.ascontiguousarray(col, np.int32), _i32p),
                       int(s), _p(d, _i32p), _p(sig, _f64p))
    return d, sig


def decompose(n, u, v):
    """Brute-force BCC split: (n_bcc, edge_bcc, art_term)."""
    u = np.ascontiguousarray(u, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.int32)
    eb = np.zeros(len(u), dtype=np.int32)
    art = np.zeros(n, dtype=np.float64)
    nb = lib().orc_decompose(n, len(u), _p(u, _i32p), _p(v, _i32p), _p(eb, _i32p), _p(art, _f64p))
    return nb, eb, art


def decompose_linear(n, u, v):
    """Linear-time BCC split with decompose()'s outputs: (n_bcc, edge_bcc, art_term)."""
    u = np.ascontiguousarray(u, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.int32)
    eb = np.zeros(len(u), dtype=np.int32)
    art = np.zeros(n, dtype=np.float64)
    nb = lib().orc_decompose_linear(n, len(u), _p(u, _i32p), _p(v, _i32p), _p(eb, _i32p), _p(art, _f64p))
    return nb, eb, art


def pack_bcc(n, u, v, edge_bcc, b):
    """BCC b packed by the oracle alone, as a one-BCC arrays dict that
    bcc_sources(arrs, 0, ...) takes: orig (original ids), row, col, reach,
    n_plain and the chain table."""
    u = np.ascontiguousarray(u, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.int32)
    eb = np.ascontiguousarray(edge_bcc, dtype=np.int32)
    nb = C.c_int32()
    mb = C.c_int64()
    lib().orc_bcc_size(len(u), _p(u, _i32p), _p(v, _i32p), _p(eb, _i32p), n, int(b), C.byref(nb), C.byref(mb))
    k, m2 = nb.value, 2 * mb.value
    vert = np.zeros(max(k, 1), np.int32)
    row = np.zeros(k + 1, np.int64)
    col = np.zeros(max(m2, 1), np.int32)
    rch = np.zeros(max(k, 1), np.int32)
    ch = [np.zeros(max(k, 1), np.int32) for _ in range(4)]
    nch = lib().orc_pack_bcc(n, len(u), _p(u, _i32p), _p(v, _i32p), _p(eb, _i32p), int(b), _p(vert, _i32p),
                             _p(row, _i64p), _p(col, _i32p), _p(rch, _i32p), *[_p(c, _i32p) for c in ch])
    plain = k - int(ch[1][:nch].sum())
    return {"n_bcc": 1, "n_packed": k, "vtx_off": np.array([0, k], np.int64), "row": row, "col": col[:m2],
            "reach": rch[:k], "orig": vert[:k], "n_plain": np.array([plain], np.int32),
            "chain_off": np.array([0, nch], np.int64), "chain_start": ch[0][:nch], "chain_len": ch[1][:nch],
            "chain_l": ch[2][:nch], "chain_r": ch[3][:nch]}


def reach(n, u, v, edge_bcc, bcc):
    u = np.ascontiguousarray(u, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.int32)
    out = np.zeros(n, dtype=np.int32)
    lib().orc_reach(n, len(u), _p(u, _i32p), _p(v, _i32p), _p(np.ascontiguousarray(edge_bcc, np.int32), _i32p), bcc,
                    _p(out, _i32p))
    return out


def method_bc(n, u, v, nthreads=0):
    """BC by the restated reference method (BCC/reach/chain merge)."""
    u = np.ascontiguousarray(u, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.int32)
    out = np.zeros(n, dtype=np.float64)
    lib().orc_method_bc(n, len(u), _p(u, _i32p), _p(v, _i32p), nthreads, _p(out, _f64p))
    return out


def _bcc_arrays(arrs, b):
    """Local CSR + chains of packed BCC b from Decomposition.arrays()."""
    vo = arrs["vtx_off"]
    v0, v1 = int(vo[b]), int(vo[b + 1])
    row = arrs["row"][v0:v1 + 1] - arrs["row"][v0]
    col = arrs["col"][arrs["row"][v0]:arrs["row"][v1]]
    c0, c1 = int(arrs["chain_off"][b]), int(arrs["chain_off"][b + 1])
    ch = [np.ascontiguousarray(arrs[k][c0:c1], np.int32) for k in ("chain_start", "chain_len", "chain_l", "chain_r")]
    return v1 - v0, np.ascontiguousarray(row, np.int64), np.ascontiguousarray(col, np.int32), \
        np.ascontiguousarray(arrs["reach"][v0:v1], np.int32), ch


def bcc_sources(arrs, b, sources, nthreads=0):
    """Per-BCC kernel restatement on the packed format: local BC contributions."""
    nb, row, col, rch, ch = _bcc_arrays(arrs, b)
    src = np.ascontiguousarray(sources, dtype=np.int32)
    out = np.zeros(nb, dtype=np.float64)
    lib().orc_bcc_sources(nb, _p(row, _i64p), _p(col, _i32p), _p(rch, _i32p), len(ch[0]), *[_p(c, _i32p) for c in ch],
                          _p(src, _i32p), len(src), nthreads, _p(out, _f64p))
    return out


def bcc_source_rows(arrs, b, s):
    nb, row, col, _, ch = _bcc_arrays(arrs, b)
    d = np.zeros(nb, dtype=np.int32)
    sig = np.zeros(nb, dtype=np.float64)
    lib().orc_bcc_source_rows(nb, _p(row, _i64p), _p(col, _i32p), len(ch[0]), *[_p(c, _i32p) for c in ch], int(s),
                              _p(d, _i32p), _p(sig, _f64p))
    return d, sig


def method_bc_from_decomp(arrs, nthreads=0):
    """BC from a packed decomposition with the oracle's per-BCC kernel (tests the
    product's decomposition against the oracle's BC)."""
    out = np.array(arrs["art"], dtype=np.float64)
    for b in range(arrs["n_bcc"]):
        nb = int(arrs["vtx_off"][b + 1] - arrs["vtx_off"][b])
        loc = bcc_sources(arrs, b, np.arange(nb, dtype=np.int32), nthreads)
        np.add.at(out, arrs["orig"][arrs["vtx_off"][b]:arrs["vtx_off"][b + 1]], loc)
    return out


def parse_refdump(path):
    """Parses an oracle/_ref/refdump record file (see oracle/ref/refdump_stub.cpp)."""
    bccs = []
    art = {}
    counts = None
    cur = None
    for line in Path(path).read_text().splitlines():
        t = line.split()
        if not t:
            continue
        if t[0] == "BCC":
            cur = {"n": int(t[2]), "reach": {}, "free": [], "ears": []}
            bccs.append(cur)
        elif t[0] == "V":
            cur["reach"][int(t[1])] = int(t[2])
        elif t[0] == "FREE":
            cur["free"] = [int(x) for x in t[1:]]
        elif t[0] == "EAR":
            l, r, cnt = int(t[1]), int(t[2]), int(t[3])
            trip = [(int(t[4 + 3 * i]), int(t[5 + 3 * i]), int(t[6 + 3 * i])) for i in range(cnt)]
            cur["ears"].append((l, r, trip))
        elif t[0] == "ART":
            art[int(t[1])] = float(t[2])
        elif t[0] == "COUNTS":
            counts = (int(t[1]), int(t[2]))
    return {"bccs": bccs, "art": art, "counts": counts}
