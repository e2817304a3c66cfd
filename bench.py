#!/usr/bin/env python
"""Benchmark: exact-BC TEPS on one B200 (or N, one process per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--mode batched|plain] [--workload rmat20|rmat16|grid|ba|small]

A step is one pass of the BC kernels over one batch of sources of the
workload graph (inputs resident in HBM). TEPS = sum over processed sources of
the arcs of the source's biconnected component / device time. Prints ONE
JSON line on rank 0.

--impl reference times the reference method's CPU restatement (the oracle's
per-BCC kernel, C + OpenMP, all host cores) on bounded source samples of the
same workload: the reference itself has no CPU BC path.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "centrality-gpu_b200"
PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
# the headline metric, reported by both arms (this engine, and the reference's CPU path)
METRIC = "exact-BC TEPS on 1 B200, batched vs plain, at FP64-oracle rel err \u22641e-6"


def load_graphs():
    """The seeded workload generators (numpy only; loads no native library)."""
    spec = importlib.util.spec_from_file_location("bench_graphs", PKG_DIR / "graphs.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_pkg():
    name = "centrality_gpu_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


WORKLOADS = {
    "rmat20": ("RMAT scale 20, edge factor 16 (a,b,c)=(0.57,0.19,0.19), symmetrised/deduplicated, "
               "10% of edges subdivided into chains of 1-4", lambda G: G.gen_rmat(20, 16, 0.1, 1, 4, seed=5)),
    "rmat16": ("RMAT scale 16, edge factor 16, 20% of edges subdivided into chains of 1-8",
               lambda G: G.gen_rmat(16, 16, 0.2, 1, 8, seed=2)),
    "grid": ("512x512 grid, 10% edges deleted, p=0.3 chains of 1-4, 15000 leaves", lambda G: G.gen_grid(seed=3)),
    "ba": ("4096 Barabasi-Albert m=2 graphs, n log-uniform 50..5000, 10% chains of 1-3, n/10 leaves, packed",
           lambda G: G.pack_graphs(G.gen_ba_batch(4096, seed=4))[:3]),
    "small": ("2000 vertices: 1000-vertex 3-out core, 500 pendants, 100 chains of 5", lambda G: G.gen_small(1)),
}


def clocks_start():
    f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    try:
        p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                             stdout=f, stderr=subprocess.DEVNULL)
    except OSError:
        p = None
    return p, f.name


def clocks_stop(handle, gpu_index):
    p, path = handle
    if p is None:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
    p.terminate()
    p.wait()
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in Path(path).read_text().splitlines():
        t = [x.strip() for x in line.split(",")]
        if len(t) < 9 or t[0] != str(gpu_index):
            continue
        try:
            sm.append(float(t[1]))
            mx.append(float(t[2]))
        except ValueError:
            continue
        for nme, val in zip(names, t[5:9]):
            if val.lower() == "active":
                reasons.add(nme)
    os.unlink(path)
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
            "samples": len(sm), "reasons": sorted(reasons)}


def peak_hbm():
    try:
        d = json.loads(PEAKS.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def step_ranges(plan, target_sources):
    """Contiguous unit ranges holding >= target_sources sources each."""
    n = plan.n_units
    total = plan.unit_work(0, n)[0]
    bounds = [0]
    k = 1
    while bounds[-1] < n:
        want = k * target_sources
        if want >= total:
            bounds.append(n)
            break
        lo, hi = bounds[-1] + 1, n
        while lo < hi:
            mid = (lo + hi) // 2
            if plan.unit_work(0, mid)[0] >= want:
                hi = mid
            else:
                lo = mid + 1
        bounds.append(lo)
        k += 1
    return list(zip(bounds[:-1], bounds[1:]))


def oracle_largest_bcc(n, u, v, edge=None):
    """A BCC as the oracle alone decomposes and packs it (linear-time BCC
    split, reach and chains in oracle/bc_oracle.c), with the oracle's
    articulation terms: the CPU legs compute with no part of the product.
    Which BCC: the one holding `edge` (a pair of original vertex ids, e.g. an
    edge of the GPU plan's largest BCC, so that both sides name the same
    one), else the one with the most edges."""
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O  # the checker: CPU legs only
    nbcc, eb, art = O.decompose_linear(n, u, v)
    if edge is None:
        big = int(np.argmax(np.bincount(eb, minlength=max(nbcc, 1))))
    else:
        a, b = edge
        hit = np.nonzero(((u == a) & (v == b)) | ((u == b) & (v == a)))[0]
        if len(hit) == 0:
            raise RuntimeError("the edge naming the BCC is not in the graph")
        big = int(eb[hit[0]])
    return O.pack_bcc(n, u, v, eb, big), art


def cpu_sample(arrs, budget_s, threads):
    """Times the oracle's per-BCC kernel (CPU restatement of the method) on an
    evenly spaced sample of the sources of the BCC in arrs (the oracle's own
    packing of the largest BCC), sized to ~budget_s."""
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O  # the checker: CPU-baseline leg only
    nb = int(arrs["vtx_off"][1] - arrs["vtx_off"][0])
    arcs = int(arrs["row"][arrs["vtx_off"][1]] - arrs["row"][arrs["vtx_off"][0]])
    probe = np.linspace(0, nb - 1, num=max(threads, 1), dtype=np.int64).astype(np.int32)
    t = time.perf_counter()
    O.bcc_sources(arrs, 0, probe, threads)
    dt = time.perf_counter() - t
    count = int(min(nb, max(len(probe), len(probe) * budget_s / max(dt, 1e-3))))
    sample = np.linspace(0, nb - 1, num=count, dtype=np.int64).astype(np.int32)
    t = time.perf_counter()
    O.bcc_sources(arrs, 0, sample, threads)
    dt = time.perf_counter() - t
    return {"sources": count, "arcs": arcs, "vertices": nb, "seconds": dt, "gteps": count * arcs / dt / 1e9}


def cpu_unit_check(plan, arrs, oarrs, oart, threads):
    """CPU-baseline and accuracy leg: times the oracle's per-BCC kernel (the
    method's CPU restatement) on exactly the sources of one GPU work unit of
    the largest BCC, on all host threads, on the oracle's own decomposition
    and packing of that BCC (oarrs, oart), and reports the max relative BC
    error of the unit's GPU result (plus the GPU's articulation terms) against
    the oracle's (plus the oracle's articulation terms)."""
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O  # the checker: CPU-baseline leg only
    v0, v1 = int(arrs["vtx_off"][0]), int(arrs["vtx_off"][1])
    # a unit of the largest BCC, the one nearest the middle of the unit list
    # (its units may sit anywhere: passes first, small-BCC items last)
    inside = [k for k in range(plan.n_units)
              if len(ids := plan.unit_sources(k, k + 1)) and ids.min() >= v0 and ids.max() < v1]
    if not inside:
        raise RuntimeError("no unit lies in the largest BCC")
    k0 = min(inside, key=lambda k: abs(k - plan.n_units // 2))
    ids = plan.unit_sources(k0, k0 + 1)
    plan.reset()
    plan.run(k0, k0 + 1, stats=False)
    got = plan.read()
    n = len(got)
    onb = int(oarrs["n_packed"])
    if onb != v1 - v0:
        raise RuntimeError(f"oracle's largest BCC has {onb} vertices, the product's {v1 - v0}")
    to_local = np.full(n, -1, dtype=np.int64)
    to_local[oarrs["orig"]] = np.arange(onb)
    local = to_local[arrs["orig"][ids]].astype(np.int32)  # the unit's sources in the oracle's packing
    if (local < 0).any():
        raise RuntimeError("a GPU source is not in the oracle's largest BCC")
    t = time.perf_counter()
    contrib = O.bcc_sources(oarrs, 0, local, threads)
    dt = time.perf_counter() - t
    want = np.array(oart, dtype=np.float64)
    np.add.at(want, oarrs["orig"], contrib)
    err = float(np.max(np.abs(got - want) / np.maximum(1.0, np.abs(want))))
    arcs = int(arrs["row"][v1] - arrs["row"][v0])
    return {"unit": k0, "sources": len(ids), "arcs": arcs, "vertices": v1 - v0, "seconds": dt,
            "gteps": len(ids) * arcs / dt / 1e9, "max_rel_err": err}


def batch_graph_check(P, plan, G, threads, count=16, graphs=4096):
    """Accuracy of a whole run of the batch of independent graphs: the GPU's BC
    of every vertex of a seeded sample of `count` graphs against the oracle's
    restatement of the method (its own decomposition) run on each graph alone."""
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O  # the checker
    batch = G.gen_ba_batch(graphs, seed=4)
    offs = np.concatenate(([0], np.cumsum([g[0] for g in batch])))
    plan.reset()
    plan.run(stats=False)
    got = plan.read()
    count = min(count, len(batch))
    pick = np.sort(np.random.default_rng(2024).choice(len(batch), size=count, replace=False))
    err, verts = 0.0, 0
    for i in pick:
        n, u, v = batch[i]
        want = O.method_bc(n, u, v, threads)
        mine = got[offs[i]:offs[i] + n]
        err = max(err, float(np.max(np.abs(mine - want) / np.maximum(1.0, np.abs(want)))))
        verts += n
    return {"max_rel_err": err, "vs": "FP64 CPU oracle (the method restated, its own decomposition), per graph",
            "graphs": int(count), "vertices": int(verts), "sample": f"seeded {count} of {len(batch)} graphs, every vertex",
            "bar": 1e-6}


def save_sample(P, d, arrs, plan, args, device, stream, width, tile_max):
    """Runs `args.sample_units` seeded random units of the plan's largest BCC
    (outside the timed region) in FP32C and in FP64, and saves their BC
    contributions (original ids, articulation terms excluded) with the original
    ids of their sources to args.save_bc."""
    v1 = int(arrs["vtx_off"][1])  # the largest BCC: the units whose sources all lie in it
    inside = [k for k in range(plan.n_units) if plan.unit_sources(k, k + 1).max(initial=-1) < v1]
    rng = np.random.default_rng(2025)
    units = np.sort(rng.choice(inside, size=min(args.sample_units, len(inside)), replace=False))
    srcs = np.concatenate([plan.unit_sources(int(k), int(k) + 1) for k in units])
    out = {"units": units, "sources_orig": arrs["orig"][srcs], "sources_packed": srcs,
           "workload": np.array(args.workload)}
    for name, dl in (("fp32c", P.DELTA_FP32C), ("fp64", P.DELTA_FP64)):
        c = P.Context(mode=P.MODE_BATCHED, delta=dl, batch_width=width, device=device, stream=stream.cuda_stream,
                      tile_max=tile_max, workspace_limit=int(args.workspace_gb * 2**30))
        pl = c.plan(d)
        for k in units:
            pl.run(int(k), int(k) + 1, stats=False)
        out["bc_" + name] = pl.read() - arrs["art"]
        pl.close()
        c.close()
    np.savez_compressed(args.save_bc, **out)


def traffic_per_source(mode, workload):
    """DRAM bytes per source of the dominant kernel from the committed ncu
    summary (profiles/<kernel>_<workload>.md, line 'traffic_bytes_per_source: X')."""
    import re
    name = ("batched_kernel" if mode == "batched" else "plain_kernel") + f"_{workload}.md"
    f = ROOT / "profiles" / name
    if not f.exists():
        return None, None
    m = re.search(r"traffic_bytes_per_source:\s*([0-9.eE+]+)", f.read_text())
    return (float(m.group(1)), f"profiles/{name}") if m else (None, None)


def plain_sample(P, d, device, stream, waves, batched_gteps, whole=False):
    """Times the plain FP64 schedule (one source per CTA) on `waves` full
    waves of its work items, taken from two places in the largest BCC's item
    list (or on all its items when `whole`), with CUDA events; returns its TEPS
    and the batched/plain ratio."""
    import torch
    pctx = P.Context(mode=P.MODE_PLAIN, device=device, stream=stream.cuda_stream)
    pplan = pctx.plan(d)
    slots = pplan.concurrency
    per = max(1, waves * slots // 2)
    n = pplan.n_units
    picks = [(max(0, int(f * n) - per // 2), max(0, int(f * n) - per // 2) + per) for f in (0.25, 0.75)]
    picks = [(a, min(n, b)) for a, b in picks]
    if whole:
        picks = [(0, n)]
    pplan.run(picks[0][0], min(picks[0][1], picks[0][0] + slots), stats=False)  # warm-up wave
    torch.cuda.synchronize()
    ms = teps = src = 0.0
    for a, b in picks:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pplan.run(a, b, stats=False)
        e1.record(stream)
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        w = pplan.unit_work(a, b)
        src += w[0]
        teps += w[1]
    pplan.close()
    pctx.close()
    g = teps / (ms * 1e-3) / 1e9
    return {"value": g, "unit": "GTEPS", "dtype": "f64", "items": sum(b - a for a, b in picks), "sources": int(src),
            "ms": ms, "resident_ctas": slots, "batched_over_plain": batched_gteps / g,
            "sample": "every plain work item (the whole workload)" if whole else
                      f"{waves} full waves of plain work items ({slots} resident CTAs) at 25% and 75% of the item list"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    G = load_graphs()  # the seeded generators only: nothing of libbcgpu is loaded on this arm
    desc, gen = WORKLOADS[args.workload]
    n, u, v = gen(G)
    arrs, _ = oracle_largest_bcc(n, u, v)
    threads = len(os.sched_getaffinity(0))
    for _ in range(args.warmup):
        cpu_sample(arrs, 0.5, threads)
    res = [cpu_sample(arrs, args.ref_step_s, threads) for _ in range(args.steps)]
    secs = sum(r["seconds"] for r in res)
    value = sum(r["sources"] * r["arcs"] for r in res) / secs / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value,
        "unit": "GTEPS", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": {"workload": f"{args.workload}: {desc}",
                   "sample": "evenly spaced sources of the largest BCC, decomposed and packed by the oracle"},
        "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": threads, "kind": "port",
                         "sample": f"{res[0]['sources']} sources/step of the largest BCC "
                                   f"({res[0]['vertices']} vertices, {res[0]['arcs']} arcs)"},
        "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1,
                    help="GPUs of the run: one process per GPU under torchrun, which sets the ranks (WORLD_SIZE)")
    ap.add_argument("--steps", type=int, default=5, help="timed steps (ranges of work units)")
    ap.add_argument("--warmup", type=int, default=3, help="untimed steps before them")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mode", choices=["batched", "plain"], default="batched")
    ap.add_argument("--delta", choices=["fp32c", "fp64"], default="fp32c")
    ap.add_argument("--batch", type=int, default=0, help="sources per multi-source pass (0 = autotune)")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="rmat20")
    ap.add_argument("--step-sources", type=int, default=0, help="sources per step (0 = by workload and mode)")
    ap.add_argument("--e2e-steps", type=int, default=5,
                    help="steps timed end to end through bc_run_bccs_units with host buffers (0 = skip)")
    ap.add_argument("--ref-step-s", type=float, default=8.0,
                    help="--impl reference: seconds of CPU work per step (its sources are sized to it)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-waves", type=int, default=6,
                    help="batched runs: also time the plain FP64 schedule on this many full waves of its work "
                         "items (one item per resident CTA), the denominator of batched vs plain (0 = skip)")
    ap.add_argument("--graph", type=int, choices=[0, 1], default=1,
                    help="1: every step is one launch of a CUDA graph of the step's device work, recorded "
                         "(stream capture, nothing runs) before the warm-up; 0: the work is enqueued directly")
    ap.add_argument("--phase-times", action="store_true",
                    help="print the multi-source kernel's per-phase times of the timed steps to stderr "
                         "(needs an instrumented build: build.py --variant phase -DBCGPU_PHASE_TIMERS, "
                         "BCGPU_LIB_DIR=centrality-gpu_b200/lib_phase)")
    ap.add_argument("--workspace-gb", type=float, default=0.0,
                    help="cap the device workspace (0 = library default); used to keep profiler captures small")
    ap.add_argument("--no-autotune", action="store_true",
                    help="take --batch / --tile-max as given (0 = the library's defaults) instead of measuring them")
    ap.add_argument("--tune-cache", default="",
                    help="JSON file the autotuner reads its choice from, or writes it to (keyed by graph shape and GPU)")
    ap.add_argument("--sample-units", type=int, default=0,
                    help="after the timed region: run this many seeded random units of the plan in the line's "
                         "delta mode and in FP64 and save their BC contributions to --save-bc (for "
                         "tests/sample_accuracy.py, which checks them against the oracle on the CPU)")
    ap.add_argument("--save-bc", default="", help="npz file for --sample-units")
    ap.add_argument("--ba-graphs", type=int, default=4096,
                    help="ba workload: graphs in the batch (fewer only for small profiler captures)")
    ap.add_argument("--tile-max", type=int, default=0,
                    help="small-BCC schedule: largest BCC it takes (bc_opts.tile_max; 0 = as large as shared "
                         "memory allows, -1 = off)")
    ap.add_argument("--plain-ctas", type=int, choices=[0, 4, 8, 16], default=0,
                    help="per-source schedule (and BCCs routed to it): CTAs per SM (bc_opts.plain_ctas_per_sm; "
                         "0 = the library's choice, four of 256 threads)")
    ap.add_argument("--full-tables", action="store_true",
                    help="e2e steps build the multi-source tables of every pass, not only of the passes "
                         "they run (bc_opts.lazy_tables = 0; lazy tables are the library's default)")
    ap.add_argument("--host-decomp", action="store_true",
                    help="decompose on the host cores (bc_decompose) only; by default the decomposition runs "
                         "on the GPU (bc_decompose_gpu, outside the timed region) and the host one is timed "
                         "beside it and checked to give the same arrays")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    # NCCL between the GPUs; BCGPU_DIST_BACKEND=gloo runs the ranks' reductions on
    # host tensors instead (the CPU tests of this multi-rank path use it)
    backend = os.environ.get("BCGPU_DIST_BACKEND", "nccl")
    rdev = "cuda" if backend == "nccl" else "cpu"
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))

    P = load_pkg()
    from centrality_gpu_b200 import graphs as G
    desc, gen = WORKLOADS[args.workload]
    if args.workload == "ba" and args.ba_graphs != 4096:
        desc = desc.replace("4096", str(args.ba_graphs))
        gen = lambda G: G.pack_graphs(G.gen_ba_batch(args.ba_graphs, seed=4))[:3]  # noqa: E731
    t0 = time.perf_counter()
    n, u, v = gen(G)
    gen_s = time.perf_counter() - t0  # the seeded workload generator (Python): not the product
    t0 = time.perf_counter()
    graph = P.Graph.from_edges(n, u, v)
    ingest_s = time.perf_counter() - t0  # the product's host side: CSR build
    t0 = time.perf_counter()
    dh = P.Decomposition(graph)
    host_s = time.perf_counter() - t0  # BCC/chain decomposition on the host cores
    arrs = dh.arrays()
    decomp = None
    if args.host_decomp:
        d = dh
    else:  # the decomposition the measured runs use: on this rank's GPU (first call in the process)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        d = P.Decomposition(graph, gpu_device=local)
        gpu_s = time.perf_counter() - t0
        ga = d.arrays()
        same = all(np.array_equal(arrs[k], ga[k]) if hasattr(arrs[k], "shape") else arrs[k] == ga[k] for k in arrs)
        if not same:
            raise SystemExit("bench: the GPU decomposition differs from the host decomposition")
        decomp = {"gpu_s": round(gpu_s, 3), "host_s": round(host_s, 3), "same_arrays": same}
        dh.close()
        del ga
    mode = P.MODE_BATCHED if args.mode == "batched" else P.MODE_PLAIN
    delta = P.DELTA_FP32C if args.delta == "fp32c" else P.DELTA_FP64
    # a dedicated stream: torch's legacy default stream has handle 0, which the
    # library reads as "use your own stream"
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    width, tile_max, tuned = args.batch, args.tile_max, None
    if mode == P.MODE_BATCHED and (args.batch == 0 or args.tile_max == 0) and not args.no_autotune:
        # the project autotuner, outside the timed region: pass width and the
        # small-BCC size limit, measured on this graph (or read from --tune-cache)
        if rank == 0:  # every rank must build the same plan: rank 0 tunes, the others take its shapes
            from centrality_gpu_b200 import autotune
            res = autotune.tune(P, d, dict(delta=delta, device=local, stream=stream.cuda_stream,
                                           workspace_limit=int(args.workspace_gb * 2**30)),
                                cache_path=args.tune_cache or None, device_name=torch.cuda.get_device_name(local))
            width = res["batch_width"] if args.batch == 0 else width
            tile_max = res["tile_max"] if args.tile_max == 0 else tile_max
            tuned = {"cached": res["cached"], "batch_width": res["batch_width"], "tile_max": res["tile_max"],
                     "width_gteps": {k: round(v, 2) for k, v in res["width_gteps"].items()},
                     "bands": [{"vertices": f"{b['lo']}-{b['hi']}", "bccs": b["bccs"], "sampled": b["sampled"],
                                "per_source_ms": round(b["per_source_ms"], 3), "tile_ms": round(b["tile_ms"], 3)}
                               for b in res["bands"]]}
        if dist:
            wt = torch.tensor([width, tile_max], dtype=torch.int64, device=rdev)
            dist.broadcast(wt, src=0)
            width, tile_max = int(wt[0].item()), int(wt[1].item())
    ctx = P.Context(mode=mode, delta=delta, batch_width=width, device=local, stream=stream.cuda_stream,
                    workspace_limit=int(args.workspace_gb * 2**30), graph=bool(args.graph),
                    plain_ctas_per_sm=args.plain_ctas, lazy_tables=not args.full_tables, tile_max=tile_max)
    plan = ctx.plan(d)
    # steps of this many sources, small enough that every rank gets at least one
    total_sources = plan.unit_work(0, plan.n_units)[0]
    # the batch of independent graphs runs whole, in one launch per schedule
    whole = args.workload == "ba"
    target = args.step_sources or (total_sources if whole else 8192 if mode == P.MODE_BATCHED else 512)
    target = max(1, min(target, total_sources // world))
    ranges = step_ranges(plan, target)
    if len(ranges) < world:  # the same on every rank (same plan): all stop here, before any collective
        print(f"bench: {len(ranges)} step(s) of work for {world} ranks: use a larger workload", file=sys.stderr)
        return 1
    from centrality_gpu_b200 import multigpu
    mine = multigpu.shard(ranges, rank, world)
    need = args.warmup + args.steps
    # steps evenly spaced over the whole source order (passes differ by region)
    pick = np.linspace(0, len(mine) - 1, num=need).round().astype(int) if len(mine) >= need else np.arange(need) % len(mine)
    sel = [mine[i] for i in pick]
    if args.graph:  # record each step's graph up front (capture only: no device work runs)
        for r0, r1 in dict.fromkeys(sel):
            plan.record(r0, r1)

    for r0, r1 in sel[:args.warmup]:
        plan.run(r0, r1, stats=False)
    torch.cuda.synchronize()
    st = plan.run(*sel[0], stats=True)  # launches per step
    launches_per_unit = st["kernel_launches"]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if args.phase_times:
        P.phase_times(reset=True)
    clk = clocks_start()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for i, (r0, r1) in enumerate(sel[args.warmup:]):
        evs[i][0].record(stream)
        plan.run(r0, r1, stats=False)
        evs[i][1].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = clocks_stop(clk, local)
    if args.phase_times:
        print(json.dumps({"phase_ms": P.phase_times(reset=True)}), file=sys.stderr, flush=True)
    elapsed = t_start.elapsed_time(t_end)
    per_step = [a.elapsed_time(b) for a, b in evs]
    work = np.array([plan.unit_work(r0, r1) for r0, r1 in sel[args.warmup:]], dtype=np.float64)
    sources, teps, visits = work.sum(axis=0)
    tot = torch.tensor([teps, sources, visits], dtype=torch.float64, device=rdev)
    mx = torch.tensor([elapsed], dtype=torch.float64, device=rdev)
    if dist:
        dist.all_reduce(tot)
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    teps_all, sources_all, visits_all = tot.tolist()
    elapsed_max = mx.item()
    value = teps_all / (elapsed_max * 1e-3) / 1e9

    # roofline: algorithmic bytes per source (16 B per arc + 48 B per vertex of its BCC)
    peak, peak_kind = peak_hbm()
    alg_bytes = 16.0 * teps + 48.0 * visits
    avg_launch_ms = float(np.mean(per_step))
    achieved = alg_bytes / args.steps / (avg_launch_ms * 1e-3) / 1e9
    tps, tsrc = traffic_per_source(args.mode, args.workload)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_kind,
                "traffic": tps * sources / args.steps if tps else None,
                "traffic_source": f"ncu dram__bytes_read.sum+dram__bytes_write.sum per source ({tsrc}) x sources "
                                  f"per launch" if tps else None,
                "alg_bytes_per_launch": alg_bytes / args.steps, "avg_launch_ms": avg_launch_ms}

    # end to end through the public API with host buffers (uploads + download inside)
    e2e = None
    if args.e2e_steps > 0:
        torch.cuda.synchronize()
        e_sel = sel[args.warmup:args.warmup + args.e2e_steps]
        out = np.zeros(n, dtype=np.float64)
        if dist:
            dist.barrier()  # ranks start together; the job's time is the slowest rank's
        te = time.perf_counter()
        copied = []
        for r0, r1 in e_sel:
            _, est = ctx.run_units(d, r0, r1, with_art=False, out=out)
            copied.append((est["h2d_bytes"], est["d2h_bytes"]))
        te = time.perf_counter() - te
        e_teps = float(sum(plan.unit_work(r0, r1)[1] for r0, r1 in e_sel))
        if dist:
            t_sum = torch.tensor([e_teps], dtype=torch.float64, device=rdev)
            t_max = torch.tensor([te], dtype=torch.float64, device=rdev)
            dist.all_reduce(t_sum)
            dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
            e_teps, te = t_sum.item(), t_max.item()
        # what the library reports it copied each step (the packed graph and the tables built from it in;
        # BC and status words out), on every rank
        h2d = int(np.mean([c[0] for c in copied]))
        d2h = int(np.mean([c[1] for c in copied]))
        e2e = {"value": e_teps / te / 1e9, "unit": "GTEPS", "h2d_bytes_per_step": h2d * world,
               "d2h_bytes_per_step": d2h * world, "steps": len(e_sel)}

    # combine the ranks' BC (one FP64 all-reduce, outside the timed region)
    if world > 1:
        from centrality_gpu_b200 import multigpu
        plan.reset()
        for r0, r1 in sel[args.warmup:]:
            plan.run(r0, r1, stats=False)
        total = multigpu.combine_bc(plan.read() - arrs["art"], arrs["art"], dist, device=rdev)
        if rank == 0:
            print(f"combined BC over {world} ranks: sum {float(total.sum()):.6e}", file=sys.stderr)

    if rank == 0 and world == 1 and args.sample_units > 0 and args.save_bc:
        save_sample(P, d, arrs, plan, args, local, stream, width, tile_max)

    plain = None
    if rank == 0 and world == 1 and mode == P.MODE_BATCHED and args.plain_waves > 0:
        plain = plain_sample(P, d, local, stream, args.plain_waves, value, whole=whole)

    cpu = None
    accuracy = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = len(os.sched_getaffinity(0))
        # the GPU plan's largest BCC, named for the oracle by its first arc's original end points
        e0 = int(arrs["row"][0])
        first_edge = (int(arrs["orig"][0]), int(arrs["orig"][arrs["col"][e0]]))
        oarrs, oart = oracle_largest_bcc(n, u, v, first_edge)
        s = cpu_unit_check(plan, arrs, oarrs, oart, threads)
        cpu = {"value": s["gteps"], "unit": "GTEPS", "cores": threads, "kind": "port",
               "sample": f"the {s['sources']} sources of GPU unit {s['unit']} (largest BCC: {s['vertices']} vertices, "
                         f"{s['arcs']} arcs), oracle per-BCC kernel, {s['seconds']:.1f} s"}
        accuracy = {"max_rel_err": s["max_rel_err"],
                    "vs": "FP64 CPU oracle on the same sources, on the oracle's own decomposition",
                    "sources": s["sources"], "bar": 1e-6}
        if whole:  # the batch of graphs: every vertex of sampled graphs, after one whole run
            unit_err = accuracy["max_rel_err"]
            accuracy = batch_graph_check(P, plan, G, threads, graphs=args.ba_graphs)
            accuracy["unit_check_max_rel_err"] = unit_err

    if rank == 0:
        info = d.info
        line = {
            "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if (mode == P.MODE_PLAIN or delta == P.DELTA_FP64) else "f32c",
            "data": "synthetic (seeded generator)",
            "config": {"workload": f"{args.workload}: {desc}", "mode": args.mode,
                       "delta": "fp64" if mode == P.MODE_PLAIN else args.delta, "vertices": int(n),
                       "edges": int(len(u)), "largest_bcc": int(arrs["vtx_off"][1]) if arrs["n_bcc"] else 0,
                       "chain_vertices": info["n_chain_vertices"], "sources_per_step": sources_all / args.steps / world,
                       "units_per_step": float(np.mean([r1 - r0 for r0, r1 in sel])),
                       "host_decomposition_s": round(host_s, 3), "ingest_s": round(ingest_s, 3), "generator_s": round(gen_s, 3), "l2": "inputs larger than L2 (CSR + per-CTA rows)",
                       "batch_width": st.get("batch_width"), "tile_max": tile_max, "autotune": tuned,
                       "cuda_graph": bool(args.graph), "decomposition": "host" if args.host_decomp else "gpu",
                       "gpu_decomposition": decomp,
                       "plain_ctas_per_sm": args.plain_ctas or None, "lazy_tables": not args.full_tables,

                       "parallelism": f"sources sharded over {world} GPU(s)"},
            "roofline": roofline, "cpu_baseline": cpu, "accuracy": accuracy, "e2e": e2e, "clocks": clocks,
            "plain": plain,
            "gpu_launches": int(launches_per_unit * args.steps),
        }
        print(json.dumps(line), flush=True)
    plan.close()
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
