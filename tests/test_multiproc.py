"""Multi-rank path on CPU: 2 gloo ranks shard the sources, compute their
contributions, and one all-reduce combines them into the whole-graph BC.
The per-rank compute here is the oracle's per-BCC kernel (no GPU on CPU);
what is tested is the sharding and the combine the GPU runs use."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from helpers import graphs, oracle, pkg, rel_err


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from helpers import pkg as _pkg
        P = _pkg()
        from centrality_gpu_b200 import multigpu
        n, u, v = graphs().gen_small(4)
        arrs = P.Decomposition(P.Graph.from_edges(n, u, v)).arrays()
        O = oracle()
        # units = contiguous source blocks of every BCC, dealt round-robin
        units = []
        for b in range(arrs["n_bcc"]):
            nb = int(arrs["vtx_off"][b + 1] - arrs["vtx_off"][b])
            units += [(b, s, min(nb, s + 64)) for s in range(0, nb, 64)]
        local = np.zeros(n)
        for b, s0, s1 in multigpu.shard(units, rank, world):
            contrib = O.bcc_sources(arrs, b, np.arange(s0, s1, dtype=np.int32))
            np.add.at(local, arrs["orig"][arrs["vtx_off"][b]:arrs["vtx_off"][b + 1]], contrib)
        total = multigpu.combine_bc(local, arrs["art"], dist)
        if rank == 0:
            row, col = O.csr(n, u, v)
            q.put(rel_err(total, O.brandes(n, row, col)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_combine():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=5) < 1e-12


def test_shard_covers_every_unit_once():
    pkg()
    from centrality_gpu_b200 import multigpu
    items = list(range(37))
    for world in (1, 2, 3, 8):
        got = sorted(x for r in range(world) for x in multigpu.shard(items, r, world))
        assert got == items
    with pytest.raises(ValueError):
        multigpu.shard(items, 2, 2)
