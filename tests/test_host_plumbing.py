"""libbcgpu's host logic on the CPU: the library's own objects (built by
build.py) linked against a stand-in CUDA runtime (tests/stub_cudart/: device
memory is host memory, kernels are counted but do not run). This reaches
the code the rest of the CPU suite cannot -- plan construction, routing
between the two schedules, the pass and work-item scheduling, the unit
bookkeeping behind TEPS, CUDA-graph record/replay and the input checks of
every entry point. BC values are not checked here (no kernel runs): the GPU
tests pin them. Each check runs in a subprocess that loads the stub build
through BCGPU_LIB_DIR, so this process keeps the real library."""
import json
import os
import subprocess
import sys

import pytest

from helpers import ROOT

PKG = ROOT / "centrality-gpu_b200"
STUB = ROOT / "tests" / "stub_cudart"
BUILD = STUB / "_build"

PRELUDE = """
import json, sys
import ctypes as C
import numpy as np
sys.path.insert(0, {tests!r})
from helpers import GOLDEN_CASES, graphs, load_case, pkg
P = pkg()
L = P.lib()
L.stub_cudart_launches.restype = C.c_longlong
G = graphs()
out = {{}}

def decomp(n, u, v):
    return P.Decomposition(P.Graph.from_edges(n, u, v))

def raises(f):
    try:
        f()
    except P.BcError as e:
        return [int(e.code), str(e)]
    return None
"""


@pytest.fixture(scope="module")
def stub_dir():
    sys.path.insert(0, str(PKG))
    import build as pkg_build  # centrality-gpu_b200/build.py: its source list names the library's objects
    objs = [PKG / "_build" / (s + ".o") for s in pkg_build.CU_SOURCES + pkg_build.CXX_SOURCES]
    if not all(o.exists() for o in objs):
        pkg_build.build()
    BUILD.mkdir(exist_ok=True)
    # built under names of this process, then renamed into place: test
    # processes running side by side never load a half-written library
    tag = f".{os.getpid()}"
    stub_o = BUILD / f"stub_cudart{tag}.o"
    subprocess.run(["g++", "-O1", "-std=c++17", "-fPIC", "-I/usr/local/cuda/include", "-c",
                    str(STUB / "stub_cudart.cpp"), "-o", str(stub_o)], check=True)
    # -Bsymbolic: the library's calls bind to these stand-ins even when a real
    # CUDA runtime is already loaded in the process (torch brings one)
    lib_tmp = BUILD / f"libbcgpu.so{tag}"
    subprocess.run(["g++", "-shared", "-o", str(lib_tmp)] + [str(o) for o in objs] +
                   [str(stub_o), "-lgomp", "-Wl,--no-undefined", "-Wl,-Bsymbolic"], check=True)
    stub_o.unlink()
    os.replace(lib_tmp, BUILD / "libbcgpu.so")
    return BUILD


def run_stub(stub_dir, code):
    env = dict(os.environ, BCGPU_LIB_DIR=str(stub_dir))
    script = PRELUDE.format(tests=str(ROOT / "tests")) + code + "\nprint(json.dumps(out))\n"
    r = subprocess.run([sys.executable, "-c", script], env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_stub_library_is_loaded(stub_dir):
    res = run_stub(stub_dir, "out['lib'] = str(P.LIB_PATH)\nout['stub'] = hasattr(L, 'stub_cudart_launches')")
    assert res["lib"] == str(stub_dir / "libbcgpu.so") and res["stub"]


def test_every_source_is_scheduled_exactly_once(stub_dir):
    """In every schedule and batch width, the units of a plan hold every
    vertex of every BCC exactly once as a source, and the work they report
    (sources, TEPS arcs, vertex visits) adds up to the BCCs' own."""
    res = run_stub(stub_dir, """
graphs_ = [("small2000", G.gen_small(1)),
           ("rmat11", G.gen_rmat(11, 16, chain_frac=0.2, chain_hi=8, seed=2)),
           ("grid30", G.gen_grid(30, leaves=100, seed=3)),
           ("ba12", G.pack_graphs(G.gen_ba_batch(12, 40, 3000, seed=7))[:3])]
graphs_ += [(c, load_case(c)[:3]) for c in GOLDEN_CASES]
modes = [dict(mode=P.MODE_PLAIN), dict(mode=P.MODE_PLAIN, plain_ctas_per_sm=16), dict(mode=P.MODE_BATCHED),
         dict(mode=P.MODE_BATCHED, tile_max=-1), dict(mode=P.MODE_BATCHED, tile_max=300),
         dict(mode=P.MODE_BATCHED, plain_core=500, plain_ctas_per_sm=8),
         dict(mode=P.MODE_BATCHED, plain_core=-1, batch_width=32),
         dict(mode=P.MODE_BATCHED, plain_core=-1, batch_width=128),
         dict(mode=P.MODE_BATCHED, plain_core=-1, batch_width=1024)]
bad = []
for name, (n, u, v) in graphs_:
    d = decomp(n, u, v)
    a = d.arrays()
    nb = np.diff(a["vtx_off"])
    arcs = a["row"][a["vtx_off"][1:]] - a["row"][a["vtx_off"][:-1]]
    want = [int(a["n_packed"]), int((nb * arcs).sum()), int((nb * nb).sum())]
    for opts in modes:
        ctx = P.Context(**opts)
        plan = ctx.plan(d)
        ids = plan.unit_sources()
        if sorted(ids.tolist()) != list(range(int(a["n_packed"]))):
            bad.append([name, str(opts), "sources"])
        if list(plan.unit_work()) != want:
            bad.append([name, str(opts), "work", list(plan.unit_work()), want])
        for k in range(0, plan.n_units, max(1, plan.n_units // 7)):
            if len(plan.unit_sources(k, k + 1)) != plan.unit_work(k, k + 1)[0]:
                bad.append([name, str(opts), "unit", k])
        plan.close()
        ctx.close()
out["bad"] = bad
""")
    assert res["bad"] == []


def test_routing_between_the_schedules(stub_dir):
    """Twelve BA graphs with the core threshold at 500: the multi-source
    passes come first and hold exactly the sources of the five BCCs whose
    cores reach it; the per-source items hold the seven others; one run over
    all units launches each schedule once, plus the fold of the per-source
    schedule's fixed-point counters. A deep BCC is routed
    per-source by its depth alone (60x60 grid); forcing multi-source passes
    overrides it. (The small-BCC schedule is off here: tile_max -1.)"""
    res = run_stub(stub_dir, """
n, u, v = G.pack_graphs(G.gen_ba_batch(12, 40, 3000, seed=7))[:3]
d = decomp(n, u, v)
a = d.arrays()
big = [b for b in range(a["n_bcc"]) if a["n_plain"][b] >= 500]
owner = np.repeat(np.arange(a["n_bcc"]), np.diff(a["vtx_off"]))
ctx = P.Context(mode=P.MODE_BATCHED, plain_core=500, tile_max=-1)
plan = ctx.plan(d)
kinds = [bool(np.isin(owner[plan.unit_sources(k, k + 1)], big).all()) for k in range(plan.n_units)]
first_item = kinds.index(False)
out["big"] = len(big)
out["passes_first"] = all(kinds[:first_item]) and not any(kinds[first_item:])
out["pass_sources"] = int(plan.unit_work(0, first_item)[0])
out["big_vertices"] = int(sum(a["vtx_off"][b + 1] - a["vtx_off"][b] for b in big))
l0 = L.stub_cudart_launches()
st = plan.run()
out["launches"] = [st["kernel_launches"], L.stub_cudart_launches() - l0]
plan.close()
ctx.close()
g = decomp(*G.gen_grid(60, delete_frac=0.0, sub_p=0.0, leaves=0, seed=9))  # levels deeper than 96 from any vertex
ga = g.arrays()
units = {}
for name, opts in (("plain", dict(mode=P.MODE_PLAIN)), ("auto", dict(mode=P.MODE_BATCHED, plain_core=100, tile_max=-1)),
                   ("multi", dict(mode=P.MODE_BATCHED, plain_core=-1, batch_width=128))):
    c = P.Context(**opts)
    p = c.plan(g)
    units[name] = p.n_units
    p.close()
    c.close()
out["grid_core"] = int(ga["n_plain"][0])
out["grid_units"] = units
""")
    assert res["big"] == 5 and res["passes_first"]
    assert res["pass_sources"] == res["big_vertices"]
    assert res["launches"] == [3, 3]
    assert res["grid_core"] >= 100  # above the threshold given: only the depth routes it
    assert res["grid_units"]["auto"] == res["grid_units"]["plain"]
    assert res["grid_units"]["multi"] == -(-3600 // 128)


def test_small_bccs_take_the_tile_schedule(stub_dir):
    """BATCHED plan of twelve BA graphs (every core under the multi-source
    threshold): with tile_max 600 the BCCs of at most 600 vertices become
    small-BCC items of at most 128 sources each, listed after the per-source
    items of the larger BCCs; one run over all units launches the per-source
    kernel, the tile kernel and one counter fold after each; with tile_max -1
    every BCC stays per-source."""
    res = run_stub(stub_dir, """
n, u, v = G.pack_graphs(G.gen_ba_batch(12, 40, 3000, seed=7))[:3]
d = decomp(n, u, v)
a = d.arrays()
nb = np.diff(a["vtx_off"])
owner = np.repeat(np.arange(a["n_bcc"]), nb)
ctx = P.Context(mode=P.MODE_BATCHED, tile_max=600)
plan = ctx.plan(d)
sizes = [int(nb[owner[plan.unit_sources(k, k + 1)]].max()) for k in range(plan.n_units)]
counts = [int(plan.unit_work(k, k + 1)[0]) for k in range(plan.n_units)]
small = [s <= 600 for s in sizes]
first = small.index(True) if True in small else len(small)
out["order"] = all(not x for x in small[:first]) and all(small[first:])
out["small_units"] = len(small) - first
out["small_bccs"] = int((nb <= 600).sum())
out["max_small_unit"] = max(counts[first:]) if first < len(counts) else 0
l0 = L.stub_cudart_launches()
st = plan.run()
out["launches"] = [st["kernel_launches"], L.stub_cudart_launches() - l0]
plan.close()
ctx.close()
ctx = P.Context(mode=P.MODE_BATCHED, tile_max=-1)
plan = ctx.plan(d)
out["off_units"] = plan.n_units
out["off_launches"] = plan.run()["kernel_launches"]
plan.close()
ctx.close()
out["n_bcc"] = int(a["n_bcc"])
out["n_packed"] = int(a["n_packed"])
""")
    assert res["order"] and res["small_bccs"] > 0 and res["small_units"] >= res["small_bccs"]
    assert 0 < res["max_small_unit"] <= 128
    assert res["launches"] == [4, 4]  # per-source kernel + fold, tile kernel + fold
    assert res["off_launches"] == 2 and res["off_units"] < res["n_packed"]


def test_autotuner_measures_caches_and_rereads(stub_dir, tmp_path):
    """The shape autotuner (centrality-gpu_b200/autotune.py) on the stand-in
    runtime: it returns a batch width and a tile_max from the candidates,
    reports the size bands it sampled, writes its choice to the JSON cache
    under a key of the graph's shape and device, reads it back on a second
    call without measuring, and measures again for another graph. The
    sub-batches it times are exact: a subset of BCCs packed on its own holds
    their sources and work."""
    cache = tmp_path / "tune.json"
    res = run_stub(stub_dir, f"""
from centrality_gpu_b200 import autotune as A
n, u, v = G.pack_graphs(G.gen_ba_batch(24, 40, 3000, seed=7))[:3]
d = decomp(n, u, v)
a = d.arrays()
l0 = L.stub_cudart_launches()
r1 = A.tune(P, d, cache_path="{cache}", device_name="stub")
out["launches_first"] = L.stub_cudart_launches() - l0
l1 = L.stub_cudart_launches()
r2 = A.tune(P, d, cache_path="{cache}", device_name="stub")
out["launches_second"] = L.stub_cudart_launches() - l1
out["r1"] = r1
out["r2"] = r2
g = decomp(*G.gen_grid(30, leaves=100, seed=3))
out["r3_cached"] = A.tune(P, g, cache_path="{cache}", device_name="stub")["cached"]
out["keys"] = len(__import__("json").load(open("{cache}")))
pick = [1, 4, 9]
sub = A.PackedBccs(A.subset(a, pick))
ctx = P.Context(mode=P.MODE_BATCHED)
plan = ctx.plan(sub)
nb = np.diff(a["vtx_off"])[pick]
arcs = (a["row"][a["vtx_off"][1:]] - a["row"][a["vtx_off"][:-1]])[pick]
out["sub"] = [list(plan.unit_work()), [int(nb.sum()), int((nb * arcs).sum()), int((nb * nb).sum())]]
plan.close()
ctx.close()
""")
    r1, r2 = res["r1"], res["r2"]
    assert r1["batch_width"] in (0, 128, 256, 512, 1024) and not r1["cached"]
    assert r1["tile_max"] in [-1] + [b["hi"] for b in r1["bands"]] and len(r1["bands"]) >= 2
    assert all(b["sampled"] <= b["bccs"] for b in r1["bands"])
    assert res["launches_first"] > 0 and res["launches_second"] == 0
    assert r2["cached"] and r2["batch_width"] == r1["batch_width"] and r2["tile_max"] == r1["tile_max"]
    assert res["r3_cached"] is False and res["keys"] == 2
    assert res["sub"][0] == res["sub"][1]


def test_graph_mode_records_then_replays(stub_dir):
    """Recording enqueues nothing; each replay of a recorded range launches
    what the range holds; a range run without recording is recorded on its
    first run; without graph mode, recording is refused."""
    res = run_stub(stub_dir, """
n, u, v = G.pack_graphs(G.gen_ba_batch(12, 40, 3000, seed=7))[:3]  # both schedules at this threshold
d = decomp(n, u, v)
c = P.Context(mode=P.MODE_BATCHED, plain_core=500, graph=True, tile_max=-1)
plan = c.plan(d)
k = plan.n_units
l0 = L.stub_cudart_launches()
plan.record(0, k)
out["after_record"] = L.stub_cudart_launches() - l0
st1 = plan.run(0, k)
l1 = L.stub_cudart_launches()
st2 = plan.run(0, k)
out["replays"] = [st1["kernel_launches"], st2["kernel_launches"], L.stub_cudart_launches() - l1]
st3 = plan.run(1, k)  # not recorded before: recorded on this run
out["fresh"] = st3["kernel_launches"]
plan.close()
c.close()
c = P.Context(mode=P.MODE_PLAIN)
plan = c.plan(d)
out["refused"] = raises(lambda: plan.record(0, 1))
plan.close()
c.close()
""")
    assert res["after_record"] == 0
    assert res["replays"] == [3, 3, 3]
    assert res["fresh"] == 3
    assert res["refused"] is not None and res["refused"][0] == 1


def test_malformed_input_is_rejected(stub_dir):
    """Every structural check of the packed input, and of the begin_gpu
    mirrors, returns BCGPU_EINVAL (1) with its message; sizes beyond the
    no-allocation variant's fixed scratch return BCGPU_EOVERFLOW (6); a
    workspace limit below one BCC's rows returns BCGPU_ENOMEM (3)."""
    res = run_stub(stub_dir, """
n, u, v = G.gen_small(1)
d = decomp(n, u, v)
a = d.arrays()
ctx = P.Context(mode=P.MODE_PLAIN)

class Packed:  # a bc_bccs over numpy copies that a case may corrupt
    def __init__(self, **change):
        self.arr = {k: np.array(x, copy=True) for k, x in a.items() if isinstance(x, np.ndarray)}
        for k, x in change.items():
            self.arr[k] = x(self.arr[k])
        b = P.BcBccs()
        b.n_bcc, b.n_orig, b.n_packed, b.n_arcs, b.n_chains = a["n_bcc"], a["n_orig"], a["n_packed"], a["n_arcs"], a["n_chains"]
        for k, x in self.arr.items():
            ptype = dict(b._fields_)[k]
            setattr(b, k, x.ctypes.data_as(ptype))
        self.view = C.pointer(b)

def bump(i, val):
    def f(x):
        x[i] = val
        return x
    return f

cases = {
    "ok": Packed(),
    "col": Packed(col=bump(5, 10 ** 6)),
    "neg_col": Packed(col=bump(5, -1)),
    "reach": Packed(reach=bump(3, -2)),
    "orig": Packed(orig=bump(3, 10 ** 7)),
    "n_plain": Packed(n_plain=bump(0, 0)),
    "chain_len": Packed(chain_len=bump(0, 0)),
    "row": Packed(row=bump(5, 0)),
}
res = {}
for name, pk in cases.items():
    res[name] = raises(lambda: ctx.run(pk))
out["packed"] = res
R = [0, 2, 4, 6]
Cc = [1, 2, 0, 2, 0, 1]
out["free_ok"] = raises(lambda: P.begin_gpu_free(ctx, R, Cc, 3, 6, [0, 1, 2], [0, 0, 0], np.zeros(3, np.float32)))
out["free_small"] = raises(lambda: P.begin_gpu_free(ctx, [0, 1, 2], [1, 0], 2, 2, [0], [0, 0], np.zeros(2, np.float32)))
out["free_col"] = raises(lambda: P.begin_gpu_free(ctx, [0, 2, 4, 6], [1, 2, 0, 2, 0, 9], 3, 6, [0], [0, 0, 0], np.zeros(3, np.float32)))
out["free_src"] = raises(lambda: P.begin_gpu_free(ctx, R, Cc, 3, 6, [7], [0, 0, 0], np.zeros(3, np.float32)))
# a 4-cycle 0-1-2-3 seen as ears (0, 2) through 1 and 3
R4, C4 = [0, 2, 4, 6, 8], [1, 3, 0, 2, 1, 3, 0, 2]
good = [(0, 2, [(1, 1, 1)]), (0, 2, [(1, 3, 1)])]
out["active_ok"] = raises(lambda: P.begin_gpu_active(ctx, R4, C4, 4, 8, [0, 2], good, [0] * 4, np.zeros(4, np.float32)))
out["active_dist"] = raises(lambda: P.begin_gpu_active(ctx, R4, C4, 4, 8, [0, 2], [(0, 2, [(2, 1, 2)])], [0] * 4,
                                                      np.zeros(4, np.float32)))
out["active_end"] = raises(lambda: P.begin_gpu_active(ctx, R4, C4, 4, 8, [2], good, [0] * 4, np.zeros(4, np.float32)))
out["noalloc_big"] = raises(lambda: P.begin_gpu_free_noalloc(ctx, 16, 16, 20000, 4, 16, 1, 16, 16))
ctx.close()
small = P.Context(mode=P.MODE_PLAIN, workspace_limit=120 << 10)  # below two slots of rows
out["limit"] = raises(lambda: small.run(d))
small.close()
""")
    p = res["packed"]
    assert p["ok"] is None
    want = {"col": "column id outside its BCC", "neg_col": "negative column id", "reach": "orig/reach out of range",
            "orig": "orig/reach out of range", "n_plain": "n_plain out of range", "chain_len": "chain out of range",
            "row": "row offsets decrease"}
    for name, msg in want.items():
        assert p[name] is not None and p[name][0] == 1 and msg in p[name][1], (name, p[name])
    assert res["free_ok"] is None and res["active_ok"] is None
    for name in ("free_small", "free_col", "free_src", "active_dist", "active_end"):
        assert res[name] is not None and res[name][0] == 1, (name, res[name])
    assert res["noalloc_big"][0] == 6 and "16384" in res["noalloc_big"][1]
    assert res["limit"][0] == 3 and "exceeds the limit" in res["limit"][1]


def test_chain_shape_errors(stub_dir):
    """The multi-source builder's chain checks (run in parallel) report the
    error a pass in chain order meets first: equal ends, a vertex an earlier
    chain holds, a chain vertex whose neighbours are not its chain
    neighbours; with two faulty chains, the earlier one's error."""
    res = run_stub(stub_dir, """
n, u, v = G.gen_small(1)
d = decomp(n, u, v)
a = d.arrays()
ctx = P.Context(mode=P.MODE_BATCHED, plain_core=-1)
b = int(np.argmax(np.diff(a["chain_off"])))
c0 = int(a["chain_off"][b])
out["chains"] = int(a["chain_off"][b + 1]) - c0

def packed(**change):
    arr = {k: np.array(x, copy=True) for k, x in a.items() if isinstance(x, np.ndarray)}
    for k, f in change.items():
        f(arr[k])
    from centrality_gpu_b200 import autotune as A
    return A.PackedBccs(dict(a, **arr))

def put(i, val):
    def f(x):
        x[i] = val
    return f

def foreign(c):  # the first arc of chain c's first vertex leads to a core vertex off the chain
    e0 = int(a["row"][int(a["vtx_off"][b]) + int(a["chain_start"][c])])
    L, R = int(a["chain_l"][c]), int(a["chain_r"][c])
    w = next(x for x in range(int(a["n_plain"][b])) if x not in (L, R))
    return put(e0, w)

cases = {
    "ok": packed(),
    "same": packed(chain_r=put(c0 + 3, int(a["chain_l"][c0 + 3]))),
    "overlap": packed(chain_start=put(c0 + 6, int(a["chain_start"][c0 + 2]))),
    "neigh": packed(col=foreign(c0 + 3)),
    # chain 3 with foreign neighbours before chain 6 overlapping chain 2: chain 3's error
    "first": packed(col=foreign(c0 + 3), chain_start=put(c0 + 6, int(a["chain_start"][c0 + 2]))),
    # chain 2 with equal ends before chain 4 with foreign neighbours: chain 2's error
    "first2": packed(chain_r=put(c0 + 2, int(a["chain_l"][c0 + 2])), col=foreign(c0 + 4)),
}
out["res"] = {k: raises(lambda: ctx.run(pk)) for k, pk in cases.items()}
ctx.close()
""")
    r = res["res"]
    assert res["chains"] >= 10
    assert r["ok"] is None
    want = {"same": "two ends are the same vertex", "overlap": "chains overlap",
            "neigh": "neighbours are not its chain neighbours", "first": "neighbours are not its chain neighbours",
            "first2": "two ends are the same vertex"}
    for name, msg in want.items():
        assert r[name] is not None and r[name][0] == 1 and msg in r[name][1], (name, r[name])


def test_large_small_bccs_take_grouped_ctas(stub_dir):
    """BCCs whose one-source CTA fits only once or twice per SM go to a
    1024-thread CTA of two or four source groups sharing one staged slice
    (classes 4, 5) when the groups fit shared memory; every source is in
    exactly one item."""
    res = run_stub(stub_dir, """
n, u, v = G.pack_graphs(G.gen_ba_batch(12, 2500, 6000, seed=21))[:3]
d = decomp(n, u, v)
ctx = P.Context(mode=P.MODE_BATCHED, tile_max=0)
plan = ctx.plan(d)
out["launches"] = plan.tile_launches()
out["sources"] = int(plan.unit_work()[0])
out["n_packed"] = int(d.arrays()["n_packed"])
plan.close()
ctx.close()
""")
    classes = [c for c, _ in res["launches"]]
    assert 4 in classes and 5 in classes, res["launches"]
    assert res["sources"] == res["n_packed"]


def test_failed_plan_builds_release_everything(stub_dir):
    """A device allocation failing at any point of a plan build (PLAIN, and
    multi-source with per-source items) returns BCGPU_ENOMEM (3) and leaves
    no device allocation behind; the context stays usable."""
    res = run_stub(stub_dir, """
L.stub_cudart_live_allocs.restype = C.c_longlong
L.stub_cudart_fail_malloc_after.argtypes = [C.c_longlong]
n, u, v = G.pack_graphs(G.gen_ba_batch(12, 40, 3000, seed=7))[:3]
d = decomp(n, u, v)
seen = {}
leaks = []
for name, opts in (("plain", dict(mode=P.MODE_PLAIN)), ("mixed", dict(mode=P.MODE_BATCHED, plain_core=500))):
    ctx = P.Context(**opts)
    base = L.stub_cudart_live_allocs()
    codes = []
    for k in range(80):
        L.stub_cudart_fail_malloc_after(k)
        r = raises(lambda: ctx.run(d))
        codes.append(0 if r is None else r[0])
        if L.stub_cudart_live_allocs() != base:
            leaks.append([name, k, L.stub_cudart_live_allocs() - base])
        if r is None:
            break
    L.stub_cudart_fail_malloc_after(-1)
    ok = raises(lambda: ctx.run(d))
    seen[name] = [codes, ok]
    ctx.close()
out["seen"] = seen
out["leaks"] = leaks
""")
    assert res["leaks"] == []
    for name, (codes, ok) in res["seen"].items():
        assert codes[-1] == 0 and len(codes) > 10, name  # every allocation of the build was made to fail once
        assert set(codes[:-1]) == {3}, (name, codes)
        assert ok is None


def test_noalloc_entry_point_allocates_nothing(stub_dir):
    """bc_begin_free_noalloc makes no device allocation on any call, the
    first included (its scratch is the library's fixed __device__ array,
    found with cudaGetSymbolAddress), and rejects sizes beyond it."""
    res = run_stub(stub_dir, """
L.stub_cudart_mallocs.restype = C.c_longlong
n, u, v = G.gen_small(1)
a = decomp(n, u, v).arrays()
v0, v1 = int(a["vtx_off"][0]), int(a["vtx_off"][1])
R = (a["row"][v0:v1 + 1] - a["row"][v0]).astype(np.int32)
Cc = np.ascontiguousarray(a["col"][a["row"][v0]:a["row"][v1]], dtype=np.int32)
reach = np.ascontiguousarray(a["reach"][v0:v1], dtype=np.int32)
nb = v1 - v0
src = np.arange(nb, dtype=np.int32)
bc = np.zeros(nb, dtype=np.float64)
ctx = P.Context(mode=P.MODE_PLAIN)
m0 = L.stub_cudart_mallocs()
for _ in range(3):  # device memory is host memory here: host arrays stand in for the caller's buffers
    P.begin_gpu_free_noalloc(ctx, R.ctypes.data, Cc.ctypes.data, nb, len(Cc), src.ctypes.data, nb,
                             reach.ctypes.data, bc.ctypes.data)
out["mallocs"] = L.stub_cudart_mallocs() - m0
out["too_big"] = raises(lambda: P.begin_gpu_free_noalloc(ctx, R.ctypes.data, Cc.ctypes.data, 16385, len(Cc),
                                                         src.ctypes.data, 1, reach.ctypes.data, bc.ctypes.data))
ctx.close()
""")
    assert res["mallocs"] == 0
    assert res["too_big"][0] == 6


def test_integration_c_example_runs(stub_dir, tmp_path):
    """The whole-graph C example of INTEGRATION.md (Option 3) compiles as C
    against include/, links against the library and runs through every call
    it makes (here on the stand-in runtime)."""
    import re
    import shutil

    text = (ROOT / "INTEGRATION.md").read_text()
    body = re.search(r"## Option 3.*?```c\n(.*?)```", text, re.S).group(1)
    src = tmp_path / "example.c"
    src.write_text('#include <stdlib.h>\n#include <stdio.h>\n#include "bchost.h"\n'
                   "int main(void) {\n" + body +
                   '  if (!bc) return 1;\n  printf("%.6f\\n", bc[0]);\n  free(bc);\n  bc_destroy(c);\n'
                   "  bc_decomp_free(d);\n  bc_graph_free(g);\n  return 0;\n}\n")
    exe = tmp_path / "example"
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I" + str(ROOT / "include"), str(src), "-o", str(exe),
                    "-L" + str(stub_dir), "-lbcgpu", "-Wl,-rpath," + str(stub_dir)], check=True)
    shutil.copy(ROOT / "tests" / "golden" / "sample4.txt", tmp_path / "graph.txt")
    r = subprocess.run([str(exe)], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    float(r.stdout.strip())


def test_integration_python_example_runs(stub_dir, tmp_path):
    """The Python example of INTEGRATION.md runs as written from the
    repository root (here on the stand-in runtime)."""
    import re

    text = (ROOT / "INTEGRATION.md").read_text()
    body = re.search(r"## Python \(ctypes\) binding.*?```python\n(.*?)```", text, re.S).group(1)
    env = dict(os.environ, BCGPU_LIB_DIR=str(stub_dir))
    r = subprocess.run([sys.executable, "-c", body + "\nprint(len(bc), stats['sources'])\n"], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.split() == ["4", "4"]


def test_betc_cli_options_and_exit_codes(stub_dir, tmp_path):
    """The drop-in command's options, output format and exit codes, with the
    in-tree betc loading the stand-in library (its RUNPATH yields to
    LD_LIBRARY_PATH): `v bc` per vertex to --out, usage errors (1), unreadable
    input (2), a rejected option value (4), an unwritable output (6). The
    decomposition runs on the host (--host-decomp): the stand-in runtime runs
    no kernels, so the default GPU decomposition stops with its own error
    (exit 3) instead."""
    from helpers import GOLDEN

    betc = PKG / "lib" / "betc"
    env = dict(os.environ, LD_LIBRARY_PATH=str(stub_dir))

    def run(*args):
        return subprocess.run([str(betc)] + [str(a) for a in args], env=env, capture_output=True, text=True,
                              timeout=120, cwd=tmp_path)

    g = GOLDEN / "sample4.txt"
    n = int(g.read_text().split()[0])
    out = tmp_path / "bc.txt"
    for extra in ([], ["--mode", "plain"], ["--mode", "batched", "--delta", "fp64", "--batch", "64"],
                  ["--mode", "plain", "--plain-ctas", "16"]):
        r = run(g, "--out", out, "--host-decomp", *extra)
        assert r.returncode == 0, r.stderr
        assert "GPU total time is" in r.stderr
        rows = [ln.split() for ln in out.read_text().splitlines()]
        assert [int(a) for a, _ in rows] == list(range(n))
        [float(b) for _, b in rows]
    r = run(g, "--quiet", "--host-decomp")
    assert r.returncode == 0 and len(r.stdout.splitlines()) == n
    r = run(g, "--quiet")
    assert r.returncode == 3 and "GPU decomposition failed" in r.stderr
    assert run().returncode == 1
    assert run(g, "--mode", "bogus").returncode == 1
    assert run(g, "--delta").returncode == 1  # option without its value
    assert run("-h").returncode == 0
    r = run(tmp_path / "missing.txt")
    assert r.returncode == 2 and "cannot be opened" in r.stderr
    r = run(g, "--batch", "33")
    assert r.returncode == 4 and "multiple of 32" in r.stderr
    r = run(g, "--plain-ctas", "3")
    assert r.returncode == 4 and "plain_ctas_per_sm" in r.stderr
    r = run(g, "--out", tmp_path / "no" / "such" / "dir.txt", "--host-decomp")
    assert r.returncode == 6


def test_reported_copy_bytes_are_the_copies_made(stub_dir):
    """bc_run_bccs_units reports in bc_stats exactly the bytes it copied each
    way (counted by the stand-in runtime), in both schedules; the host->device
    bytes include the tables the library builds, beyond the packed input."""
    res = run_stub(stub_dir, """
L.stub_cudart_h2d.restype = C.c_longlong
L.stub_cudart_d2h.restype = C.c_longlong
n, u, v = G.pack_graphs(G.gen_ba_batch(12, 40, 3000, seed=7))[:3]
d = decomp(n, u, v)
a = d.arrays()
packed = sum(int(a[k].nbytes) for k in ("vtx_off", "row", "col", "reach", "chain_start", "chain_len", "chain_l",
                                        "chain_r"))
rows = []
for opts in (dict(mode=P.MODE_PLAIN), dict(mode=P.MODE_BATCHED, plain_core=500),
             dict(mode=P.MODE_BATCHED, plain_core=-1)):
    ctx = P.Context(**opts)
    h0, d0 = L.stub_cudart_h2d(), L.stub_cudart_d2h()
    _, st = ctx.run_units(d, 0, 3)
    rows.append([st["h2d_bytes"], L.stub_cudart_h2d() - h0, st["d2h_bytes"], L.stub_cudart_d2h() - d0])
    ctx.close()
out["rows"] = rows
out["packed"] = packed
out["n_packed"] = int(a["n_packed"])
""")
    for h2d, h2d_seen, d2h, d2h_seen in res["rows"]:
        assert h2d == h2d_seen and d2h == d2h_seen
        assert h2d >= res["packed"] and d2h >= 8 * res["n_packed"]
    assert res["rows"][2][0] > res["rows"][0][0]  # the multi-source schedule also uploads its contracted rows


def test_betc_reads_the_csr_it_saved(stub_dir, tmp_path):
    """betc --save-csr writes the loaded graph as a binary CSR; betc given
    that file prints what it printed for the edge list."""
    from helpers import GOLDEN

    betc = PKG / "lib" / "betc"
    env = dict(os.environ, LD_LIBRARY_PATH=str(stub_dir))
    csr = tmp_path / "g.csr"
    a = subprocess.run([str(betc), str(GOLDEN / "small2000.txt"), "--save-csr", str(csr), "--quiet", "--host-decomp"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert a.returncode == 0, a.stderr
    b = subprocess.run([str(betc), str(csr), "--quiet", "--host-decomp"], env=env, capture_output=True, text=True,
                       timeout=120)
    assert b.returncode == 0, b.stderr
    assert a.stdout == b.stdout and len(a.stdout.splitlines()) == 2000
    r = subprocess.run([str(betc), str(GOLDEN / "sample1.txt"), "--save-csr", str(tmp_path / "no" / "x.csr")], env=env,
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 6 and "cannot write" in r.stderr


def test_autotune_width_candidates(stub_dir):
    """bc_autotune_width builds a plan per candidate width, times passes from
    the middle of the source order, reports every candidate and returns one of
    them; a candidate whose workspace does not fit the limit scores 0 and is
    never chosen; a plan with no multi-source pass returns width 0."""
    res = run_stub(stub_dir, """
n, u, v = G.gen_rmat(12, 16, chain_frac=0.2, chain_hi=8, seed=2)
d = decomp(n, u, v)
c = P.Context(mode=P.MODE_BATCHED, plain_core=-1)
w, per = c.autotune_width(d, passes=2)
out["free"] = [w, per]
c.close()
c = P.Context(mode=P.MODE_BATCHED, plain_core=-1, workspace_limit=12 << 20)
w, per = c.autotune_width(d, passes=2)
out["tight"] = [w, per]
c.close()
c = P.Context(mode=P.MODE_BATCHED)  # default routing: every BCC of this graph runs per source
w, per = c.autotune_width(decomp(*G.gen_small(1)), passes=2)
out["none"] = w
c.close()
c = P.Context(mode=P.MODE_PLAIN)
out["plain"] = raises(lambda: c.autotune_width(d, passes=2))
c.close()
""")
    w, per = res["free"]
    assert w in (128, 256, 512, 1024) and sorted(per) == ["1024", "128", "256", "512"]
    assert per[str(w)] == max(per.values()) > 0
    w, per = res["tight"]
    assert per["1024"] == 0 and w in (128, 256, 512) and per[str(w)] > 0
    assert res["none"] == 0
    assert res["plain"] is not None and res["plain"][0] == 1


def test_source_rows_arguments(stub_dir):
    """Row export (for the parity tests) is for PLAIN plans and packed ids in
    range; anything else is BCGPU_EINVAL."""
    res = run_stub(stub_dir, """
n, u, v = G.gen_small(1)
d = decomp(n, u, v)
a = d.arrays()
nb = int(a["vtx_off"][1] - a["vtx_off"][0])
c = P.Context(mode=P.MODE_PLAIN)
plan = c.plan(d)
out["ok"] = raises(lambda: plan.source_rows(0, nb))
out["chain_vertex"] = raises(lambda: plan.source_rows(int(a["n_plain"][0]), nb))
out["range"] = raises(lambda: plan.source_rows(int(a["n_packed"]), nb))
plan.close()
c.close()
c = P.Context(mode=P.MODE_BATCHED, plain_core=-1)
plan = c.plan(d)
out["batched"] = raises(lambda: plan.source_rows(0, nb))
plan.close()
c.close()
""")
    assert res["ok"] is None and res["chain_vertex"] is None
    assert res["range"][0] == 1 and res["batched"][0] == 1 and "PLAIN" in res["batched"][1]


def test_pass_rows_arguments(stub_dir):
    """Multi-source row export (for the parity tests): the arrays have one row
    per slot of the pass and one column per core vertex of its BCC, the slots'
    sources are the pass's sources; a unit that is not a multi-source pass (a
    per-source unit, one beyond the plan, a PLAIN plan's) is BCGPU_EINVAL."""
    res = run_stub(stub_dir, """
n, u, v = G.gen_small(1)
d = decomp(n, u, v)
a = d.arrays()
c = P.Context(mode=P.MODE_BATCHED, plain_core=-1, batch_width=64)
plan = c.plan(d)
src, dd, ss = plan.pass_rows(0)
out["shape"] = [len(src), list(dd.shape), list(ss.shape), int(a["n_plain"][0])]
out["same_sources"] = sorted((src + int(a["vtx_off"][0])).tolist()) == sorted(plan.unit_sources(0, 1).tolist())
out["beyond"] = raises(lambda: plan.pass_rows(plan.n_units))
plan.close()
c.close()
c = P.Context(mode=P.MODE_PLAIN)
plan = c.plan(d)
out["plain"] = raises(lambda: plan.pass_rows(0))
plan.close()
c.close()
""")
    ns, dshape, sshape, ncore = res["shape"]
    assert ns == 64 and dshape == [64, ncore] and sshape == [64, ncore] and res["same_sources"]
    assert res["beyond"][0] == 1 and res["plain"][0] == 1 and "multi-source" in res["plain"][1]


@pytest.mark.parametrize("mode", ["batched", "plain"])
def test_bench_main_arm_line(stub_dir, tmp_path, mode):
    """bench.py's main arm runs end to end on the stand-in runtime (torch.cuda
    stood in by tests/stub_cudart/torch_cuda_stub.py) and prints one JSON line
    with every key of the contract; the numbers are meaningless here."""
    args = ["--workload", "small", "--steps", "3", "--warmup", "3", "--plain-waves", "1", "--e2e-steps", "1",
            "--mode", mode, "--host-decomp"]  # the stand-in runtime runs no decomposition kernels
    env = dict(os.environ, BCGPU_LIB_DIR=str(stub_dir))
    r = subprocess.run([sys.executable, str(STUB / "bench_on_stub.py")] + args, env=env, capture_output=True,
                       text=True, timeout=600, cwd=tmp_path)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    import bench
    assert d["metric"] == bench.METRIC and d["unit"] == "GTEPS" and d["higher_is_better"] is True
    for k in ("value", "n_gpus", "steps", "warmup", "ms_per_step", "scaling", "vs_baseline", "dtype", "data", "config",
              "roofline", "cpu_baseline", "e2e", "clocks", "gpu_launches", "plain", "accuracy"):
        assert k in d, k
    assert d["steps"] == 3 and d["warmup"] == 3 and d["n_gpus"] == 1 and d["gpu_launches"] >= 3
    assert d["config"]["workload"].startswith("small") and d["config"]["cuda_graph"] is True
    assert {"bound", "achieved", "peak", "unit", "frac", "traffic"} <= set(d["roofline"])
    assert {"value", "unit", "cores", "kind", "sample"} <= set(d["cpu_baseline"])
    e = d["e2e"]
    assert e["unit"] == "GTEPS" and e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] >= 8 * 1500
    assert d["config"]["host_decomposition_s"] >= 0 and d["config"]["generator_s"] >= 0
    assert d["config"]["mode"] == mode and (d["plain"] is None) == (mode == "plain")
    assert d["dtype"] == ("f64" if mode == "plain" else "f32c")


def test_bench_two_ranks_under_torchrun(stub_dir, tmp_path):
    """bench.py's multi-rank path (one process per GPU under torchrun) on two
    CPU ranks over gloo: every rank takes the same collective steps, rank 0
    alone prints the line, which reports 2 GPUs and the whole job's work."""
    import socket

    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        port = sock.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(STUB / "bench_on_stub.py"),
           "--gpus", "2", "--workload", "small", "--steps", "3", "--warmup", "3", "--e2e-steps", "1", "--host-decomp"]
    env = dict(os.environ, BCGPU_LIB_DIR=str(stub_dir), BCGPU_DIST_BACKEND="gloo", OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["scaling"] == "weak" and d["steps"] == 3
    assert d["cpu_baseline"] is None and d["plain"] is None  # single-GPU legs only
    assert d["e2e"]["h2d_bytes_per_step"] > 0
    assert "combined BC over 2 ranks" in r.stderr


@pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "refbetc").exists(), reason="reference sources absent")
def test_reference_betc_calls_are_accepted(stub_dir, tmp_path):
    """The reference's own betc rebuilt on the binding (oracle/_ref/refbetc),
    run on the library's host code (stand-in runtime: kernels do not run):
    on every golden fixture the library accepts every begin_gpu call the
    reference makes, and what is left in the result -- no kernel adds to it --
    is the articulation terms of the reference's reach computation."""
    from helpers import GOLDEN, GOLDEN_CASES, load_case
    from helpers import pkg as real_pkg

    env = dict(os.environ, LD_LIBRARY_PATH=str(stub_dir))
    for name in GOLDEN_CASES:
        n, u, v, _, _ = load_case(name)
        r = subprocess.run([str(ROOT / "oracle" / "_ref" / "refbetc"), str(GOLDEN / f"{name}.txt")], env=env,
                           cwd=tmp_path, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, (name, r.stderr[-2000:])
        rows = [ln.split() for ln in r.stdout.splitlines()][-n:]
        got = [float(b) for _, b in rows]
        art = real_pkg().Decomposition(real_pkg().Graph.from_edges(n, u, v)).arrays()["art"]
        assert [int(a) for a, _ in rows] == list(range(n))
        assert max(abs(g - a) / max(1.0, abs(a)) for g, a in zip(got, art)) < 1e-6, name


def test_gpu_decomposition_fails_cleanly_when_its_kernels_do_not_run(stub_dir):
    """bc_decompose_gpu on the stand-in runtime (kernels counted, not run):
    its consistency checks turn the missing results into an error status,
    and every device allocation of the failed call is released."""
    res = run_stub(stub_dir, """
L.stub_cudart_live_allocs.restype = C.c_longlong
before = L.stub_cudart_live_allocs()
n0 = L.stub_cudart_launches()
for name in ('sample4', 'small2000'):
    n, u, v, _, _ = load_case(name)
    g = P.Graph.from_edges(n, u, v)
    out[name] = raises(lambda: P.Decomposition(g, gpu_device=0))
out['live'] = L.stub_cudart_live_allocs() - before
out['launches'] = L.stub_cudart_launches() - n0
""")
    assert res["sample4"] and res["small2000"] and res["sample4"][0] == 1  # EINVAL
    assert res["live"] == 0 and res["launches"] > 0


def test_plain_ctas_per_sm_sets_the_sources_in_flight(stub_dir):
    """bc_opts.plain_ctas_per_sm: the per-source schedule runs that many CTAs
    per SM (the stand-in device has 148 SMs) while their rows fit, 0 means
    four; other values are rejected at bc_create."""
    res = run_stub(stub_dir, """
n, u, v = G.gen_small(1)
d = decomp(n, u, v)
for k in (0, 4, 8, 16):
    ctx = P.Context(mode=P.MODE_PLAIN, plain_ctas_per_sm=k)
    plan = ctx.plan(d)
    out[str(k)] = plan.concurrency
    plan.close()
    ctx.close()
out['bad'] = [raises(lambda: P.Context(mode=P.MODE_PLAIN, plain_ctas_per_sm=k)) for k in (-1, 2, 3, 32)]
""")
    assert [res[k] for k in ("0", "4", "8", "16")] == [148 * 4, 148 * 4, 148 * 8, 148 * 16]
    assert all(b and b[0] == 1 for b in res["bad"])


def test_lazy_tables_build_exactly_the_requested_passes(stub_dir, tmp_path):
    """bc_opts.lazy_tables restricts a plan's multi-source tables to a pass
    range (BatchedConfig::fill_begin/fill_end): every pass in the range runs
    from exactly the slots, seeds and arming list of the full build, and the
    unit accounting is unchanged (tests/stub_cudart/fill_range_check.cpp,
    linked against the stand-in runtime's library)."""
    exe = tmp_path / "fill_range_check"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", str(ROOT / "include"), "-I", str(PKG / "csrc"),
                    "-I/usr/local/cuda/include", str(STUB / "fill_range_check.cpp"), "-o", str(exe),
                    "-L", str(stub_dir), "-lbcgpu", "-Wl,-rpath," + str(stub_dir)], check=True)
    from helpers import graphs
    G = graphs()
    cases = {"rmat14": G.gen_rmat(14, 16, 0.2, 1, 8, seed=2), "grid30": G.gen_grid(30, leaves=100, seed=3),
             "ba12": G.pack_graphs(G.gen_ba_batch(12, 40, 3000, seed=7))[:3]}
    ranges = ["0", "1", "3", "7", "-2", "-1", "5", "5", "-3", "1000000000", "0", "1000000000"]
    for name, (n, u, v) in cases.items():
        path = tmp_path / f"{name}.txt"
        G.write_edge_list(path, n, u, v)
        for width in ("64", "128"):
            r = subprocess.run([str(exe), str(path), width] + ranges, capture_output=True, text=True, timeout=300)
            assert r.returncode == 0, r.stdout + r.stderr
            lines = [ln.split() for ln in r.stdout.splitlines() if ln.startswith("range")]
            assert len(lines) == len(ranges) // 2 and all(ln[3] == "ok" for ln in lines), (name, width, r.stdout)
            assert int(r.stdout.split()[1]) > 8  # several passes, so the ranges cut the order

