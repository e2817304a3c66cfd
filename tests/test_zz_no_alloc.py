"""bc_begin_free_noalloc: the free-source BC call for callers that cannot
allocate device memory themselves (their device memory belongs to another
allocator). Called through the C ABI with device buffers the test owns, it
must give the same BC as the allocating bc_begin_free (whose output buffer is
the reference's float), on two calls in a row (the shared scratch keeps the
previous call's contents), match the FP64 oracle at the FP64 tolerance,
allocate nothing on a repeated call, and reject sizes beyond its fixed
scratch."""
import numpy as np
import pytest

from helpers import graphs, oracle, pkg, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-6  # bc_begin_free returns the reference's float buffer
TOL_FP64 = 1e-12  # the no-allocation call's own FP64 output against the oracle


def one_bcc(seed):
    P = pkg()
    n, u, v = graphs().gen_small(seed)
    arrs = P.Decomposition(P.Graph.from_edges(n, u, v)).arrays()
    v0, v1 = int(arrs["vtx_off"][0]), int(arrs["vtx_off"][1])
    R = (arrs["row"][v0:v1 + 1] - arrs["row"][v0]).astype(np.int32)
    Cc = np.ascontiguousarray(arrs["col"][arrs["row"][v0]:arrs["row"][v1]], dtype=np.int32)
    reach = np.ascontiguousarray(arrs["reach"][v0:v1], dtype=np.int32)
    return v1 - v0, R, Cc, reach, arrs


def test_noalloc_matches_begin_free_on_two_calls():
    import torch

    P = pkg()
    ctx = P.Context(mode=P.MODE_PLAIN)
    for seed in (1, 5):  # two different BCCs, one call after the other
        nb, R, Cc, reach, arrs = one_bcc(seed)
        src = np.arange(nb, dtype=np.int32)  # every vertex a BFS source
        want = np.zeros(nb, dtype=np.float32)
        P.begin_gpu_free(ctx, R, Cc, nb, len(Cc), src, reach, want)
        dev = [torch.from_numpy(x).cuda() for x in (R, Cc, src, reach)]
        out = torch.full((nb,), -1.0, dtype=torch.float64, device="cuda")  # stale values must not leak
        torch.cuda.synchronize()
        t = P.begin_gpu_free_noalloc(ctx, dev[0].data_ptr(), dev[1].data_ptr(), nb, len(Cc), dev[2].data_ptr(), nb,
                                     dev[3].data_ptr(), out.data_ptr())
        assert t > 0.0
        got = out.cpu().numpy()
        assert rel_err(got, want) < TOL
        assert rel_err(got, oracle().bcc_sources(arrs, 0, src)) < TOL_FP64
    # a repeated call allocates nothing
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    out.fill_(-1.0)
    torch.cuda.synchronize()
    P.begin_gpu_free_noalloc(ctx, dev[0].data_ptr(), dev[1].data_ptr(), nb, len(Cc), dev[2].data_ptr(), nb,
                             dev[3].data_ptr(), out.data_ptr())
    assert torch.cuda.mem_get_info()[0] == free0
    assert rel_err(out.cpu().numpy(), want) < TOL
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    P = pkg()
    ctx = P.Context(mode=P.MODE_PLAIN)
    buf = torch.zeros(8, dtype=torch.int32, device="cuda")
    out = torch.zeros(8, dtype=torch.float64, device="cuda")
    with pytest.raises(P.BcError) as e:
        P.begin_gpu_free_noalloc(ctx, buf.data_ptr(), buf.data_ptr(), 20000, 4, buf.data_ptr(), 1, buf.data_ptr(),
                                 out.data_ptr())
    assert e.value.code == P.EOVERFLOW and "16384" in str(e.value)
    ctx.close()
