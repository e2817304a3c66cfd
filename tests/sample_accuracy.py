"""Accuracy of a sampled set of sources against the FP64 oracle, on the CPU.

    python bench.py --sample-units 86 --save-bc sample.npz      # on the GPU: ~1% of RMAT-20's sources
    python tests/sample_accuracy.py sample.npz [threads]       # here: the oracle on the same sources

bench.py saves the BC contributions of a seeded random set of the plan's
units (FP32C and FP64 runs) with the original ids of their sources; this
script rebuilds the same seeded workload, decomposes and packs it with the
oracle alone (oracle/bc_oracle.c), computes the same sources' contributions
with the oracle's per-BCC restatement of the method, and prints the maximum
relative error of both GPU runs (the sampled units all lie in the largest
BCC). Not a pytest test (the oracle on ~44k RMAT-20 sources is an hour
of CPU); tests/ is where the checker lives.
"""
import json
import sys
import time

import numpy as np

from helpers import graphs, oracle


WORKLOADS = {
    "rmat20": lambda G: G.gen_rmat(20, 16, 0.1, 1, 4, seed=5),
    "rmat16": lambda G: G.gen_rmat(16, 16, 0.2, 1, 8, seed=2),
    "grid": lambda G: G.gen_grid(seed=3),
}


def main(path, threads=0):
    z = np.load(path)
    name = str(z["workload"])
    G, O = graphs(), oracle()
    n, u, v = WORKLOADS[name](G)
    t0 = time.time()
    nbcc, eb, _ = O.decompose_linear(n, u, v)
    src = z["sources_orig"].astype(np.int64)
    want = np.zeros(n)
    # bench samples units of the plan's largest BCC only: the oracle packs that BCC
    sizes = np.bincount(eb, minlength=nbcc)
    big = int(np.argmax(sizes))
    pk = O.pack_bcc(n, u, v, eb, big)
    local = np.full(n, -1, np.int64)
    local[pk["orig"]] = np.arange(int(pk["n_packed"]))
    ls = local[src]
    if (ls < 0).any():
        raise SystemExit("a sampled source is outside the largest BCC: this checker handles the largest BCC only")
    t1 = time.time()
    np.add.at(want, pk["orig"], O.bcc_sources(pk, 0, ls.astype(np.int32), threads))
    t2 = time.time()
    res = {"workload": name, "units": int(len(z["units"])), "sources": int(len(src)),
           "vertices": int(n), "bcc_vertices": int(pk["n_packed"]),
           "sample_fraction_of_bcc_sources": float(len(src)) / float(pk["n_packed"]),
           "oracle_decompose_s": round(t1 - t0, 1), "oracle_sources_s": round(t2 - t1, 1)}
    for key in ("bc_fp32c", "bc_fp64"):
        got = z[key]
        err = np.abs(got - want) / np.maximum(1.0, np.abs(want))
        res[key + "_max_rel_err"] = float(err.max())
        res[key + "_median_rel_err"] = float(np.median(err[want != 0])) if (want != 0).any() else 0.0
    print(json.dumps(res))


if __name__ == "__main__":
    main(sys.argv[1], int(sys.argv[2]) if len(sys.argv) > 2 else 0)
