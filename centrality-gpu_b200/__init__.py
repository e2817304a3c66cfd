"""Python host side of libbcgpu: exact betweenness centrality on one B200.

Thin ctypes layer over the C ABI in include/bcgpu.h and include/bchost.h; all
computation happens in libbcgpu.so (C++ host decomposition + sm_100a CUDA
kernels). There is no CPU fallback: if the library or a CUDA device is missing,
the calls raise.

Mirrors the reference's interfaces (Goutam363/centrality-GPU):
  * ``betc`` CLI                                -> lib/betc, ``betweenness``
  * Graph(char*) edge-list input                -> ``Graph.load``
  * begin_gpu free overload   (Codes/begin_gpupgm.cu:42-71)   -> ``begin_gpu_free``
  * begin_gpu active overload (Codes/begin_gpupgm.cu:73-89)   -> ``begin_gpu_active``
  * BiCC::to_eargraph loop    (Codes/to_eargraph_construct.cpp:54-200) -> ``Context.run``
"""
from __future__ import annotations

import atexit
import ctypes as C
import os
import weakref
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
# BCGPU_LIB_DIR selects another in-tree build (e.g. an instrumented variant from
# build.py --variant); the default is lib/.
_LIB_DIR = Path(os.environ["BCGPU_LIB_DIR"]) if os.environ.get("BCGPU_LIB_DIR") else _PKG / "lib"
LIB_PATH = _LIB_DIR / "libbcgpu.so"
BETC_PATH = _LIB_DIR / "betc"

OK, EINVAL, ECUDA, ENOMEM, ETIMEOUT, EIO, EOVERFLOW = range(7)
MODE_PLAIN, MODE_BATCHED = 0, 1
DELTA_FP64, DELTA_FP32C = 0, 1
_ERRNAMES = {1: "EINVAL", 2: "ECUDA", 3: "ENOMEM", 4: "ETIMEOUT", 5: "EIO", 6: "EOVERFLOW"}

_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)
_f32p = C.POINTER(C.c_float)


class BcOpts(C.Structure):
    _fields_ = [("device", C.c_int32), ("mode", C.c_int32), ("delta", C.c_int32), ("batch_width", C.c_int32),
                ("stream", C.c_void_p), ("workspace_limit", C.c_int64), ("rescale_exp", C.c_int32),
                ("plain_core", C.c_int32), ("graph", C.c_int32), ("plain_ctas_per_sm", C.c_int32),
                ("lazy_tables", C.c_int32), ("tile_max", C.c_int32), ("wait_limit_ms", C.c_int32)]


class BcBccs(C.Structure):
    _fields_ = [("n_bcc", C.c_int32), ("n_orig", C.c_int32), ("n_packed", C.c_int64), ("n_arcs", C.c_int64),
                ("n_chains", C.c_int64), ("vtx_off", _i64p), ("row", _i64p), ("col", _i32p), ("reach", _i32p),
                ("orig", _i32p), ("n_plain", _i32p), ("chain_off", _i64p), ("chain_start", _i32p),
                ("chain_len", _i32p), ("chain_l", _i32p), ("chain_r", _i32p), ("art", _f64p)]


class BcStats(C.Structure):
    _fields_ = [("sources", C.c_int64), ("bfs_sources", C.c_int64), ("aux_bfs", C.c_int64), ("teps_edges", C.c_int64),
                ("kernel_ms", C.c_double), ("total_ms", C.c_double), ("kernel_launches", C.c_int32),
                ("batch_width", C.c_int32), ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BcDecompInfo(C.Structure):
    _fields_ = [("n_components", C.c_int32), ("n_bcc_all", C.c_int32), ("n_bcc_packed", C.c_int32),
                ("n_articulation", C.c_int32), ("n_chain_vertices", C.c_int64), ("n_chains", C.c_int64),
                ("n_cycle_bccs", C.c_int64), ("host_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# Every symbol the C headers declare, with its ctypes signature.
_SIGS = {
    "bc_default_opts": (None, [C.POINTER(BcOpts)]),
    "bc_create": (C.c_int, [C.POINTER(BcOpts), C.POINTER(C.c_void_p)]),
    "bc_destroy": (None, [C.c_void_p]),
    "bc_last_error": (C.c_char_p, [C.c_void_p]),
    "bc_run_bccs": (C.c_int, [C.c_void_p, C.POINTER(BcBccs), _f64p, C.POINTER(BcStats)]),
    "bc_run_bccs_units": (C.c_int, [C.c_void_p, C.POINTER(BcBccs), C.c_int64, C.c_int64, C.c_int32, _f64p,
                                    C.POINTER(BcStats)]),
    "bc_begin_free": (C.c_int, [C.c_void_p, _i32p, _i32p, C.c_int32, C.c_int32, _i32p, C.c_int32, _i32p, _f32p,
                                _f64p]),
    "bc_begin_free_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                                        C.c_int32, C.c_void_p, C.c_void_p, _f64p]),
    "bc_begin_active": (C.c_int, [C.c_void_p, _i32p, _i32p, C.c_int32, C.c_int32, _i32p, C.c_int32, C.c_int32,
                                  _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _f32p, _f64p]),
    "bc_wait_probe": (C.c_int, [C.c_void_p, C.c_int32, _f64p]),
    "bc_plan_create": (C.c_int, [C.c_void_p, C.POINTER(BcBccs), C.POINTER(C.c_void_p)]),
    "bc_plan_destroy": (None, [C.c_void_p]),
    "bc_plan_num_units": (C.c_int64, [C.c_void_p]),
    "bc_plan_unit_work": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, _i64p, _i64p, _i64p]),
    "bc_plan_device_bytes": (C.c_int64, [C.c_void_p]),
    "bc_plan_tile_launches": (C.c_int, [C.c_void_p, _i32p, _i32p, C.c_int32]),
    "bc_plan_concurrency": (C.c_int, [C.c_void_p]),
    "bc_autotune_width": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "bc_plan_unit_sources": (C.c_int64, [C.c_void_p, C.c_int64, C.c_int64, _i64p, C.c_int64]),
    "bc_plan_reset": (C.c_int, [C.c_void_p]),
    "bc_plan_run": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.POINTER(BcStats)]),
    "bc_plan_record": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64]),
    "bc_plan_read": (C.c_int, [C.c_void_p, _f64p]),
    "bc_plan_source_rows": (C.c_int, [C.c_void_p, C.c_int64, _i32p, _f64p]),
    "bc_plan_pass_rows": (C.c_int, [C.c_void_p, C.c_int64, _i32p, _i32p, _i32p, _i32p, _f64p]),
    "bc_graph_load": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "bc_graph_from_edges": (C.c_int, [C.c_int32, C.c_int64, _i32p, _i32p, C.POINTER(C.c_void_p)]),
    "bc_graph_free": (None, [C.c_void_p]),
    "bc_graph_save": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_size_t]),
    "bc_graph_csr": (C.c_int, [C.c_void_p, _i32p, _i64p, C.POINTER(_i64p), C.POINTER(_i32p)]),
    "bc_decompose": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "bc_decompose_gpu": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "bc_decomp_free": (None, [C.c_void_p]),
    "bc_decomp_view": (C.POINTER(BcBccs), [C.c_void_p]),
    "bc_decomp_get_info": (None, [C.c_void_p, C.POINTER(BcDecompInfo)]),
}

_lib = None


def lib():
    """Loads libbcgpu.so (built in-tree by build.py). Raises if it is missing."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"libbcgpu.so not built ({LIB_PATH}); run centrality-gpu_b200/build.py")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class BcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


def _ptr(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Graph:
    """Simple undirected graph (loops dropped, duplicates merged) in CSR."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)

    @classmethod
    def load(cls, path):
        h = C.c_void_p()
        err = C.create_string_buffer(512)
        rc = lib().bc_graph_load(str(path).encode(), C.byref(h), err, 512)
        if rc:
            raise BcError(rc, err.value.decode())
        return cls(h.value)

    @classmethod
    def from_edges(cls, n, u, v):
        u, v = _i32(u), _i32(v)
        h = C.c_void_p()
        rc = lib().bc_graph_from_edges(int(n), len(u), _ptr(u, _i32p), _ptr(v, _i32p), C.byref(h))
        if rc:
            raise BcError(rc, "bc_graph_from_edges")
        return cls(h.value)

    def save(self, path):
        """Writes the CSR in the binary form Graph.load reads back (bc_graph_save)."""
        err = C.create_string_buffer(512)
        rc = lib().bc_graph_save(self._h, str(path).encode(), err, 512)
        if rc:
            raise BcError(rc, err.value.decode())

    def csr(self):
        n = C.c_int32()
        m = C.c_int64()
        row = _i64p()
        col = _i32p()
        lib().bc_graph_csr(self._h, C.byref(n), C.byref(m), C.byref(row), C.byref(col))
        r = np.ctypeslib.as_array(row, shape=(n.value + 1,)).copy()
        c = np.ctypeslib.as_array(col, shape=(max(m.value, 1),))[: m.value].copy() if m.value else np.zeros(0, np.int32)
        return n.value, r, c

    def close(self):
        if self._h:
            lib().bc_graph_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _arr(ptr, count, dtype):
    if count == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(count,)).copy()


class Decomposition:
    """BCC split + reach + articulation terms + degree-2 chains (bc_decompose).

    ``gpu_device``: run the decomposition on that GPU as data-parallel steps
    (bc_decompose_gpu; same result); -1 runs those GPU steps as host loops,
    a check of them without a GPU."""

    def __init__(self, graph: Graph, gpu_device: int | None = None):
        self._graph = graph
        h = C.c_void_p()
        if gpu_device is None:
            rc = lib().bc_decompose(graph._h, C.byref(h))
            if rc:
                raise BcError(rc, "bc_decompose")
        else:
            err = C.create_string_buffer(512)
            rc = lib().bc_decompose_gpu(graph._h, int(gpu_device), C.byref(h), err, 512)
            if rc:
                raise BcError(rc, "bc_decompose_gpu: " + err.value.decode(errors="replace"))
        self._h = h
        self.view = lib().bc_decomp_view(h)
        info = BcDecompInfo()
        lib().bc_decomp_get_info(h, C.byref(info))
        self.info = info.as_dict()

    def arrays(self):
        """Copies of the packed arrays as numpy (for tests and tools)."""
        V = self.view.contents
        nb, npk, na, nc = V.n_bcc, V.n_packed, V.n_arcs, V.n_chains
        return {
            "n_bcc": nb, "n_orig": V.n_orig, "n_packed": npk, "n_arcs": na, "n_chains": nc,
            "vtx_off": _arr(V.vtx_off, nb + 1, np.int64), "row": _arr(V.row, npk + 1, np.int64),
            "col": _arr(V.col, na, np.int32), "reach": _arr(V.reach, npk, np.int32),
            "orig": _arr(V.orig, npk, np.int32), "n_plain": _arr(V.n_plain, nb, np.int32),
            "chain_off": _arr(V.chain_off, nb + 1, np.int64), "chain_start": _arr(V.chain_start, nc, np.int32),
            "chain_len": _arr(V.chain_len, nc, np.int32), "chain_l": _arr(V.chain_l, nc, np.int32),
            "chain_r": _arr(V.chain_r, nc, np.int32), "art": _arr(V.art, V.n_orig, np.float64),
        }

    def close(self):
        if self._h:
            lib().bc_decomp_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """One CUDA device and stream (bc_create)."""

    _live = weakref.WeakSet()

    def __init__(self, mode=MODE_PLAIN, delta=DELTA_FP32C, batch_width=0, device=-1, stream=None,
                 workspace_limit=0, rescale_exp=0, plain_core=0, graph=False, plain_ctas_per_sm=0,
                 lazy_tables=True, tile_max=0, wait_limit_ms=0):
        o = BcOpts()
        lib().bc_default_opts(C.byref(o))
        o.mode, o.delta, o.batch_width, o.device = mode, delta, batch_width, device
        o.stream = stream
        o.workspace_limit = workspace_limit
        o.rescale_exp = rescale_exp
        o.plain_core = plain_core
        o.graph = 1 if graph else 0
        o.plain_ctas_per_sm = plain_ctas_per_sm
        o.lazy_tables = 1 if lazy_tables else 0
        o.wait_limit_ms = wait_limit_ms
        o.tile_max = tile_max
        h = C.c_void_p()
        rc = lib().bc_create(C.byref(o), C.byref(h))
        if rc:
            raise BcError(rc, lib().bc_last_error(None).decode())
        self._h = h
        self._plans = weakref.WeakSet()
        Context._live.add(self)

    def _check(self, rc):
        if rc:
            raise BcError(rc, lib().bc_last_error(self._h).decode())

    def run(self, decomp: Decomposition):
        """All sources of all BCCs, host buffers in and out. Returns (bc, stats)."""
        out = np.zeros(decomp.view.contents.n_orig, dtype=np.float64)
        st = BcStats()
        self._check(lib().bc_run_bccs(self._h, decomp.view, _ptr(out, _f64p), C.byref(st)))
        return out, st.as_dict()

    def run_units(self, decomp: Decomposition, begin, end, with_art=False, out=None):
        """Units [begin, end) only, host buffers in and out (uploads included)."""
        if out is None:
            out = np.zeros(decomp.view.contents.n_orig, dtype=np.float64)
        st = BcStats()
        self._check(lib().bc_run_bccs_units(self._h, decomp.view, int(begin), int(end), int(with_art),
                                            _ptr(out, _f64p), C.byref(st)))
        return out, st.as_dict()

    def plan(self, decomp: Decomposition):
        return Plan(self, decomp)

    def wait_probe(self, limit_ms: int):
        """bc_wait_probe: a device-side wait on a flag nothing sets, bounded by
        limit_ms. Returns (status code, device milliseconds the probe took)."""
        ms = C.c_double(0.0)
        rc = lib().bc_wait_probe(self._h, int(limit_ms), C.byref(ms))
        return rc, ms.value

    def autotune_width(self, decomp: Decomposition, passes: int = 4):
        """Times up to `passes` multi-source passes at widths 128/256/512/1024
        (bc_autotune_width); returns (best width or 0, {width: GTEPS})."""
        w = C.c_int32(0)
        g = (C.c_double * 4)()
        self._check(lib().bc_autotune_width(self._h, decomp.view, passes, C.byref(w), g))
        return w.value, {c: g[i] for i, c in enumerate((128, 256, 512, 1024))}

    def close(self):
        """Releases the context; its plans are released with it."""
        if self._h:
            for p in list(self._plans):
                p._h = C.c_void_p()  # freed by bc_destroy
            lib().bc_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@atexit.register
def _close_all():
    # before the CUDA runtime unloads: contexts (and with them their plans)
    for c in list(Context._live):
        try:
            c.close()
        except Exception:
            pass


class Plan:
    """Device-resident packed BCCs + BC accumulator (bc_plan_*)."""

    def __init__(self, ctx: Context, decomp: Decomposition):
        self.ctx = ctx
        self.decomp = decomp
        h = C.c_void_p()
        ctx._check(lib().bc_plan_create(ctx._h, decomp.view, C.byref(h)))
        self._h = h
        ctx._plans.add(self)
        self.n_units = lib().bc_plan_num_units(h)
        self.device_bytes = lib().bc_plan_device_bytes(h)
        self.concurrency = lib().bc_plan_concurrency(h)

    def unit_work(self, begin=0, end=None):
        """(sources, TEPS arcs, vertex visits) of units [begin, end)."""
        end = self.n_units if end is None else end
        s = C.c_int64()
        t = C.c_int64()
        w = C.c_int64()
        self.ctx._check(lib().bc_plan_unit_work(self._h, begin, end, C.byref(s), C.byref(t), C.byref(w)))
        return s.value, t.value, w.value

    def tile_launches(self):
        """[(class, grid)] of the small-BCC schedule's launches, in launch order
        (class: 0 warp per source; 1, 2, 3 one source per 256-, 512-, 1024-thread
        CTA; 4, 5 a 1024-thread CTA of two / four source groups)."""
        n = lib().bc_plan_tile_launches(self._h, None, None, 0)
        if n < 0:
            raise BcError(-n, "bc_plan_tile_launches")
        cls = np.zeros(max(n, 1), dtype=np.int32)
        grid = np.zeros(max(n, 1), dtype=np.int32)
        lib().bc_plan_tile_launches(self._h, _ptr(cls, _i32p), _ptr(grid, _i32p), n)
        return [(int(cls[i]), int(grid[i])) for i in range(n)]

    def unit_sources(self, begin=0, end=None):
        """Packed ids of the sources units [begin, end) accumulate."""
        end = self.n_units if end is None else end
        cnt = lib().bc_plan_unit_sources(self._h, begin, end, None, 0)
        if cnt < 0:
            raise BcError(-cnt, "bc_plan_unit_sources")
        out = np.zeros(max(cnt, 1), dtype=np.int64)
        lib().bc_plan_unit_sources(self._h, begin, end, _ptr(out, _i64p), cnt)
        return out[:cnt]

    def reset(self):
        self.ctx._check(lib().bc_plan_reset(self._h))

    def run(self, begin=0, end=None, stats=True):
        end = self.n_units if end is None else end
        st = BcStats() if stats else None
        self.ctx._check(lib().bc_plan_run(self._h, begin, end, C.byref(st) if stats else None))
        return st.as_dict() if stats else None

    def record(self, begin=0, end=None):
        """Graph mode: records units [begin, end) into a CUDA graph without running it."""
        end = self.n_units if end is None else end
        self.ctx._check(lib().bc_plan_record(self._h, begin, end))

    def read(self):
        out = np.zeros(self.decomp.view.contents.n_orig, dtype=np.float64)
        self.ctx._check(lib().bc_plan_read(self._h, _ptr(out, _f64p)))
        return out

    def source_rows(self, packed, nb):
        d = np.zeros(nb, dtype=np.int32)
        s = np.zeros(nb, dtype=np.float64)
        self.ctx._check(lib().bc_plan_source_rows(self._h, int(packed), _ptr(d, _i32p), _ptr(s, _f64p)))
        return d, s

    def pass_rows(self, unit):
        """Runs multi-source pass `unit` and returns (sources, d, sigma): the
        pass's sources (local ids in its BCC) and, per source (row) and core
        vertex (column), the level and the path count (level bases applied)."""
        ns, nc = C.c_int32(), C.c_int32()
        self.ctx._check(lib().bc_plan_pass_rows(self._h, int(unit), C.byref(ns), C.byref(nc), None, None, None))
        src = np.zeros(ns.value, dtype=np.int32)
        d = np.zeros((ns.value, nc.value), dtype=np.int32)
        s = np.zeros((ns.value, nc.value), dtype=np.float64)
        self.ctx._check(lib().bc_plan_pass_rows(self._h, int(unit), C.byref(ns), C.byref(nc), _ptr(src, _i32p),
                                                _ptr(d, _i32p), _ptr(s, _f64p)))
        return src, d, s

    def close(self):
        if self._h and self.ctx._h:
            lib().bc_plan_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def betweenness(n, u, v, mode=MODE_PLAIN, delta=DELTA_FP32C, batch_width=0, device=-1):
    """Exact BC (ordered pairs, FP64) of the graph given by edges (u, v)."""
    g = Graph.from_edges(n, u, v)
    d = Decomposition(g)
    ctx = Context(mode=mode, delta=delta, batch_width=batch_width, device=device)
    bc, st = ctx.run(d)
    ctx.close()
    return bc, st, d.info


def begin_gpu_free(ctx: Context, R, Cc, n, m, req_nodes, artnodes, bc, time_s=0.0):
    """Mirror of the reference's free-source begin_gpu: bc (float32, length n)
    is overwritten; returns the accumulated device seconds."""
    R, Cc, req, reach = _i32(R), _i32(Cc), _i32(req_nodes), _i32(artnodes)
    assert bc.dtype == np.float32 and bc.flags.c_contiguous
    t = C.c_double(time_s)
    ctx._check(lib().bc_begin_free(ctx._h, _ptr(R, _i32p), _ptr(Cc, _i32p), int(n), int(m), _ptr(req, _i32p), len(req),
                                   _ptr(reach, _i32p), _ptr(bc, _f32p), C.byref(t)))
    return t.value


def begin_gpu_free_noalloc(ctx: Context, R_dev, C_dev, n, m, req_dev, n_req, reach_dev, bc_dev, time_s=0.0):
    """bc_begin_free_noalloc: device pointers (ints) in and out, no allocation
    inside the call; bc_dev (FP64, n entries) is overwritten. Returns the
    accumulated device seconds."""
    t = C.c_double(time_s)
    ctx._check(lib().bc_begin_free_noalloc(ctx._h, C.c_void_p(R_dev), C.c_void_p(C_dev), int(n), int(m),
                                           C.c_void_p(req_dev), int(n_req), C.c_void_p(reach_dev),
                                           C.c_void_p(bc_dev), C.byref(t)))
    return t.value


def begin_gpu_active(ctx: Context, R, Cc, n, m, active, ears, artnodes, bc, time_s=0.0):
    """Mirror of the reference's active/chain begin_gpu. ``ears``: list of
    (lnode, rnode, [(ld, node, rd), ...]). bc (float32) is added to."""
    R, Cc, act, reach = _i32(R), _i32(Cc), _i32(active), _i32(artnodes)
    ln = _i32([e[0] for e in ears])
    rn = _i32([e[1] for e in ears])
    cnt = _i32([len(e[2]) for e in ears])
    off = _i32(np.concatenate(([0], np.cumsum(cnt)[:-1])) if len(ears) else [])
    flat = [x for e in ears for x in e[2]]
    ld = _i32([x[0] for x in flat])
    nodes = _i32([x[1] for x in flat])
    rd = _i32([x[2] for x in flat])
    assert bc.dtype == np.float32 and bc.flags.c_contiguous
    t = C.c_double(time_s)
    ctx._check(lib().bc_begin_active(ctx._h, _ptr(R, _i32p), _ptr(Cc, _i32p), int(n), int(m), _ptr(act, _i32p),
                                     len(act), len(ears), _ptr(ln, _i32p), _ptr(rn, _i32p), _ptr(cnt, _i32p),
                                     _ptr(off, _i32p), _ptr(nodes, _i32p), _ptr(ld, _i32p), _ptr(rd, _i32p),
                                     _ptr(reach, _i32p), _ptr(bc, _f32p), C.byref(t)))
    return t.value


def declared_symbols():
    """Names of every function declared in include/*.h."""
    return sorted(_SIGS)


# Phases of the multi-source kernel as numbered by its PHASE_MARK points.
PHASES = {0: "pass init", 1: "forward rows", 2: "forward heavy combine", 3: "forward level end",
          4: "chain inflow", 5: "backward heavy chunks", 6: "backward rows", 8: "chain vertices", 7: "fold into BC"}


def phase_times(reset=True):
    """Instrumented builds only (build.py --variant NAME -DBCGPU_PHASE_TIMERS,
    loaded with BCGPU_LIB_DIR): milliseconds CTA 0 spent in each phase of the
    multi-source kernel since the last reset, plus the forward and backward
    level counts; None with the default build."""
    L = lib()
    if not hasattr(L, "bc_debug_phase_times"):
        return None
    buf = (C.c_ulonglong * 32)()
    L.bc_debug_phase_times.restype = C.c_int
    if L.bc_debug_phase_times(buf, 1 if reset else 0) != 0:
        return None
    out = {name: buf[i] / 1e6 for i, name in PHASES.items()}
    out["forward levels"] = int(buf[16])
    out["backward levels"] = int(buf[17])
    return out
