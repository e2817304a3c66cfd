"""Schedule-shape autotuner for one graph on one device.

Two shapes are measured rather than guessed:

* the multi-source pass width (sources per pass: 128, 256, 512 or 1024),
  by bc_autotune_width on passes from the middle of the source order;
* which BCCs take the small-BCC schedule (bc_opts.tile_max). The BCCs that
  could take it are grouped in size bands; for each band a sample of its BCCs
  is packed into a plan of its own and timed on the small-BCC schedule and on
  the per-source schedule (the library's kernel times). tile_max is then the
  band bound whose choice -- every band up to it on the small-BCC schedule,
  the rest per source -- gives the least estimated time over the whole graph
  (each band's time scaled by its share of the graph's work).

The reference has no tuner: one source per launch, 1024 threads, one CTA per
SM (Codes/begin_gpupgm.cu:52-65).

The choice is cached in a JSON file keyed by the graph's shape (BCC count,
packed vertices, arcs and the histogram of BCC sizes) and the device's name,
so that a later run on the same graph and GPU reads it instead of measuring.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
from pathlib import Path

import numpy as np

# Size bands (vertices per BCC) of the small-BCC schedule's candidates; the
# largest bound is the schedule's own limit (16-bit neighbour ids).
BANDS = ((3, 640), (641, 1500), (1501, 2500), (2501, 3500), (3501, 65535))


class PackedBccs:
    """A bc_bccs view over numpy arrays (the layout of Decomposition.arrays()),
    usable wherever the library takes a decomposition (Context.run, plans)."""

    def __init__(self, arrs):
        from . import BcBccs, _f64p, _i32p, _i64p  # noqa: PLC0415 (package-internal types)

        self._keep = {k: np.ascontiguousarray(v) for k, v in arrs.items() if isinstance(v, np.ndarray)}
        self._arrs = dict(arrs)
        k = self._keep
        v = BcBccs()
        v.n_bcc, v.n_orig, v.n_packed = int(arrs["n_bcc"]), int(arrs["n_orig"]), int(arrs["n_packed"])
        v.n_arcs, v.n_chains = int(arrs["n_arcs"]), int(arrs["n_chains"])
        for name, t in (("vtx_off", _i64p), ("row", _i64p), ("col", _i32p), ("reach", _i32p), ("orig", _i32p),
                        ("n_plain", _i32p), ("chain_off", _i64p), ("chain_start", _i32p), ("chain_len", _i32p),
                        ("chain_l", _i32p), ("chain_r", _i32p), ("art", _f64p)):
            setattr(v, name, k[name].ctypes.data_as(t))
        self._struct = v
        self.view = C.pointer(v)

    def arrays(self):
        return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self._arrs.items()}


def subset(arrs, bccs):
    """The listed BCCs of a packed decomposition as one of their own (same
    original ids, no articulation terms)."""
    bccs = np.asarray(bccs, dtype=np.int64)
    vo, co = arrs["vtx_off"], arrs["chain_off"]
    vtx_off, row, chain_off = [0], [0], [0]
    cols, reach, orig, n_plain, cs, cl, cL, cR = [], [], [], [], [], [], [], []
    for b in bccs:
        v0, v1 = int(vo[b]), int(vo[b + 1])
        e0, e1 = int(arrs["row"][v0]), int(arrs["row"][v1])
        row.extend((arrs["row"][v0 + 1:v1 + 1] - e0 + row[-1]).tolist())
        cols.append(arrs["col"][e0:e1])
        reach.append(arrs["reach"][v0:v1])
        orig.append(arrs["orig"][v0:v1])
        n_plain.append(int(arrs["n_plain"][b]))
        c0, c1 = int(co[b]), int(co[b + 1])
        for dst, name in ((cs, "chain_start"), (cl, "chain_len"), (cL, "chain_l"), (cR, "chain_r")):
            dst.append(arrs[name][c0:c1])
        vtx_off.append(vtx_off[-1] + v1 - v0)
        chain_off.append(chain_off[-1] + c1 - c0)
    cat = lambda xs, t: np.concatenate(xs).astype(t) if xs else np.zeros(0, t)  # noqa: E731
    out = {"n_bcc": len(bccs), "n_orig": int(arrs["n_orig"]), "n_packed": vtx_off[-1], "n_arcs": row[-1],
           "n_chains": chain_off[-1], "vtx_off": np.array(vtx_off, np.int64), "row": np.array(row, np.int64),
           "col": cat(cols, np.int32), "reach": cat(reach, np.int32), "orig": cat(orig, np.int32),
           "n_plain": np.array(n_plain, np.int32), "chain_off": np.array(chain_off, np.int64),
           "chain_start": cat(cs, np.int32), "chain_len": cat(cl, np.int32), "chain_l": cat(cL, np.int32),
           "chain_r": cat(cR, np.int32), "art": np.zeros(int(arrs["n_orig"]), np.float64)}
    return out


def signature(arrs, device_name):
    """Cache key: the device and the graph's shape as the schedules see it."""
    sizes = np.diff(arrs["vtx_off"])
    hist = np.bincount(np.floor(np.log2(np.maximum(sizes, 1))).astype(np.int64), minlength=32)[:32]
    core = np.bincount(np.floor(np.log2(np.maximum(arrs["n_plain"], 1))).astype(np.int64), minlength=32)[:32]
    key = json.dumps([device_name, int(arrs["n_bcc"]), int(arrs["n_packed"]), int(arrs["n_arcs"]),
                      hist.tolist(), core.tolist()])
    return hashlib.sha1(key.encode()).hexdigest()


def _work(arrs, bccs):
    """TEPS work (sum over sources of their BCC's arcs) of the listed BCCs."""
    vo, row = arrs["vtx_off"], arrs["row"]
    nb = vo[bccs + 1] - vo[bccs]
    return float(np.sum(nb.astype(np.float64) * (row[vo[bccs + 1]] - row[vo[bccs]])))


def _timed(P, ctx_kwargs, sub, tile_max):
    """Kernel milliseconds of one whole run of `sub` (after one warm-up run)."""
    ctx = P.Context(tile_max=tile_max, **ctx_kwargs)
    try:
        plan = ctx.plan(sub)
        plan.run(stats=False)
        plan.reset()
        return plan.run(stats=True)["kernel_ms"]
    finally:
        ctx.close()


def tune(P, decomp, ctx_kwargs=None, cache_path=None, device_name=None, sample_bccs=48, passes=4):
    """Measures (or reads from the cache) the width and tile_max for
    `decomp` on the context options ctx_kwargs (mode BATCHED is implied).
    Returns {"batch_width", "tile_max", "cached", "width_gteps", "bands"}."""
    ctx_kwargs = dict(ctx_kwargs or {})
    ctx_kwargs["mode"] = P.MODE_BATCHED
    ctx_kwargs.pop("batch_width", None)
    ctx_kwargs.pop("tile_max", None)
    arrs = decomp.arrays()
    key = signature(arrs, device_name or "device")
    cache = {}
    if cache_path and os.path.exists(cache_path):
        try:
            cache = json.loads(Path(cache_path).read_text())
        except (OSError, ValueError):
            cache = {}
    if key in cache:
        return dict(cache[key], cached=True)

    ctx = P.Context(**ctx_kwargs)
    try:
        width, per = ctx.autotune_width(decomp, passes=passes)
    finally:
        ctx.close()
    kw = dict(ctx_kwargs, batch_width=width)

    sizes = np.diff(arrs["vtx_off"])
    bands = []
    for lo, hi in BANDS:
        members = np.nonzero((sizes >= lo) & (sizes <= hi))[0]
        if len(members) == 0:
            continue
        pick = members[np.linspace(0, len(members) - 1, num=min(sample_bccs, len(members))).round().astype(np.int64)]
        pick = np.unique(pick)
        sub = PackedBccs(subset(arrs, pick))
        t_src = _timed(P, kw, sub, -1)
        t_tile = _timed(P, kw, sub, hi)
        scale = _work(arrs, members) / max(_work(arrs, pick), 1.0)
        bands.append({"lo": lo, "hi": hi, "bccs": int(len(members)), "sampled": int(len(pick)),
                      "per_source_ms": t_src, "tile_ms": t_tile, "scale": scale})
    # the threshold with the least estimated time: bands up to it tiled, the rest per source
    best, best_t = -1, sum(b["per_source_ms"] * b["scale"] for b in bands)
    for b in bands:
        t = sum((c["tile_ms"] if c["hi"] <= b["hi"] else c["per_source_ms"]) * c["scale"] for c in bands)
        if t < best_t:
            best, best_t = b["hi"], t
    res = {"batch_width": int(width), "tile_max": int(best), "width_gteps": {str(k): v for k, v in per.items()},
           "bands": bands}
    if cache_path:
        cache[key] = res
        Path(cache_path).parent.mkdir(parents=True, exist_ok=True)
        Path(cache_path).write_text(json.dumps(cache, indent=1))
    return dict(res, cached=False)
