"""The reference-side binding of INTEGRATION.md (CPU): the snippet there is
the file centrality-gpu_b200/reference_binding/begin_gpupgm_bcgpu.cpp, and
the reference's own host pipeline links against it and the in-tree
libbcgpu.so (oracle/_ref/refbetc, built from the reference's sources when
they are present). Running it needs a GPU; without one it must stop at its
first begin_gpu call with libbcgpu's error, not compute anything. On a GPU
(marked test) it prints what it prints with the oracle behind the binding."""
import os
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from helpers import GOLDEN, GOLDEN_CASES, ROOT, canonical_chains, has_gpu, load_case, oracle, product_bccs
from helpers import pkg as P

BINDING = ROOT / "centrality-gpu_b200" / "reference_binding" / "begin_gpupgm_bcgpu.cpp"
REFBETC = ROOT / "oracle" / "_ref" / "refbetc"


def test_integration_snippet_is_the_binding_file():
    text = (ROOT / "INTEGRATION.md").read_text()
    snippet = re.search(r"```cpp\n(.*?)```", text, re.S).group(1)
    assert snippet == BINDING.read_text()


@pytest.mark.skipif(not REFBETC.exists(), reason="reference sources absent: refbetc not built")
def test_reference_pipeline_links_the_binding(tmp_path):
    ldd = subprocess.run(["ldd", str(REFBETC)], capture_output=True, text=True).stdout
    resolved = [ln.split("=>")[1].split("(")[0].strip() for ln in ldd.splitlines() if "libbcgpu.so =>" in ln]
    assert resolved and Path(resolved[0]).resolve() == (ROOT / "centrality-gpu_b200" / "lib" / "libbcgpu.so").resolve()
    nm = subprocess.run(["nm", "-C", "--undefined-only", str(REFBETC)], capture_output=True, text=True).stdout
    assert "begin_gpu" not in nm  # both of the reference's entry points are defined by the binding
    assert "bc_begin_active" in nm and "bc_begin_free" in nm


@pytest.mark.skipif(not REFBETC.exists(), reason="reference sources absent: refbetc not built")
@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU failure path")
def test_reference_pipeline_fails_loudly_without_gpu(tmp_path):
    # the reference writes its debug files to the working directory
    r = subprocess.run([str(REFBETC), str(GOLDEN / "sample1.txt")], cwd=tmp_path, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode != 0
    assert "no CUDA device" in r.stderr
    assert not any(re.fullmatch(r"\d+ -?[0-9.]+", ln) for ln in r.stdout.splitlines())  # no BC printed


REFBINDCHECK = ROOT / "oracle" / "_ref" / "refbindcheck"


@pytest.mark.skipif(not REFBINDCHECK.exists(), reason="reference sources absent: refbindcheck not built")
@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_binding_hands_on_the_products_chains(tmp_path, name):
    """On each fixture, the chains the binding rebuilds from the reference's
    ear records (split where the reference merged parallel ears, distances
    from positions where its ld/rd are off) are exactly the chains of the
    product's own decomposition."""
    out = tmp_path / "chains.txt"
    env = dict(os.environ, BINDCHECK_OUT=str(out))
    r = subprocess.run([str(REFBINDCHECK), str(GOLDEN / f"{name}.txt")], cwd=tmp_path, env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    got = []
    for line in out.read_text().splitlines():
        t = [int(x) for x in line.split()[1:]]
        got.append((t[0], t[1], [tuple(t[2 + 3 * i:5 + 3 * i]) for i in range((len(t) - 2) // 3)]))
    n, u, v, _, _ = load_case(name)
    arrs = P().Decomposition(P().Graph.from_edges(n, u, v)).arrays()
    want = {}
    for b in product_bccs(arrs):
        want.update(b["chains"])
    assert canonical_chains(got) == want


REFBETC_CPU = ROOT / "oracle" / "_ref" / "refbetc_cpu"


def _bc_lines(stdout, n):
    """The per-vertex BC lines refbetc_main prints last (the reference prints progress before)."""
    rows = [ln.split() for ln in stdout.splitlines()][-n:]
    assert [int(r[0]) for r in rows] == list(range(n))
    return np.array([float(r[1]) for r in rows])


def reference_semantics_bc(n, u, v):
    """What the reference's betc computes when its two begin_gpu calls return
    exact contributions: per BCC of >= 3 vertices, the free call's buffer F
    is added to the result, and -- when the BCC has ears -- the active call,
    which starts from that same buffer, adds F + A again
    (Codes/to_eargraph_construct.cpp:117,163-180); A = the chain endpoints'
    and chain vertices' contributions. Plus the articulation terms. Built from
    the product's decomposition and the oracle's per-BCC Brandes."""
    arrs = P().Decomposition(P().Graph.from_edges(n, u, v)).arrays()
    O = oracle()
    out = np.array(arrs["art"], dtype=np.float64)
    for b in range(arrs["n_bcc"]):
        v0, v1 = int(arrs["vtx_off"][b]), int(arrs["vtx_off"][b + 1])
        c0, c1 = int(arrs["chain_off"][b]), int(arrs["chain_off"][b + 1])
        npl = int(arrs["n_plain"][b])
        ends = set(arrs["chain_l"][c0:c1].tolist()) | set(arrs["chain_r"][c0:c1].tolist())
        free = np.array([k for k in range(npl) if k not in ends], dtype=np.int32)
        act = np.array(sorted(ends) + list(range(npl, v1 - v0)), dtype=np.int32)
        F = O.bcc_sources(arrs, b, free) if len(free) else np.zeros(v1 - v0)
        A = O.bcc_sources(arrs, b, act) if len(act) else np.zeros(v1 - v0)
        part = F + ((F + A) if c1 > c0 else 0.0)
        np.add.at(out, arrs["orig"][v0:v1], part)
    return out


@pytest.mark.skipif(not REFBETC_CPU.exists(), reason="reference sources absent: refbetc_cpu not built")
@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_reference_betc_on_the_binding_gives_reference_semantics(tmp_path, name):
    """The reference's own betc rebuilt on the binding (library calls computed
    by the oracle on the CPU) prints the reference's semantics -- its free
    contributions counted twice in BCCs with ears -- and, where a BCC has no
    ears, the exact BC."""
    n, u, v, golden, _ = load_case(name)
    r = subprocess.run([str(REFBETC_CPU), str(GOLDEN / f"{name}.txt")], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    got = _bc_lines(r.stdout, n)
    want = reference_semantics_bc(n, u, v)
    assert np.max(np.abs(got - want) / np.maximum(1.0, np.abs(want))) < 1e-5  # the reference's float buffers
    if P().Decomposition(P().Graph.from_edges(n, u, v)).arrays()["n_chains"] == 0:
        assert np.max(np.abs(got - golden) / np.maximum(1.0, np.abs(golden))) < 1e-5


@pytest.mark.skipif(not REFBETC_CPU.exists(), reason="reference sources absent: refbetc_cpu not built")
def test_reference_betc_without_ears_gives_exact_bc(tmp_path):
    """A wheel (hub 0, rim 1..5: no degree-2 vertex, so no ears) with a
    pendant path 1-6-7: only free calls, so the reference's betc on the
    binding prints the exact BC (articulation terms through reach)."""
    edges = [(0, k) for k in range(1, 6)] + [(k, k % 5 + 1) for k in range(1, 6)] + [(1, 6), (6, 7)]
    f = tmp_path / "wheel.txt"
    f.write_text(f"8 {len(edges)}\n" + "".join(f"{a} {b} 1\n" for a, b in edges))
    r = subprocess.run([str(REFBETC_CPU), str(f)], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    got = _bc_lines(r.stdout, 8)
    O = oracle()
    u = np.array([a for a, _ in edges], dtype=np.int32)
    v = np.array([b for _, b in edges], dtype=np.int32)
    row, col = O.csr(8, u, v)
    want = O.brandes(8, row, col)
    assert want[1] > 0 and want[0] > 0
    assert np.max(np.abs(got - want) / np.maximum(1.0, np.abs(want))) < 1e-5


@pytest.mark.gpu
@pytest.mark.skipif(not REFBETC.exists(), reason="reference sources absent: refbetc not built")
@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_reference_betc_on_the_gpu_gives_reference_semantics(tmp_path, name):
    """The reference's own betc rebuilt on the binding, its begin_gpu calls
    now computed by libbcgpu on the GPU: the same output as with the oracle
    behind the binding (the reference's semantics; the exact BC where a BCC
    has no ears)."""
    n, u, v, golden, _ = load_case(name)
    r = subprocess.run([str(REFBETC), str(GOLDEN / f"{name}.txt")], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    got = _bc_lines(r.stdout, n)
    want = reference_semantics_bc(n, u, v)
    assert np.max(np.abs(got - want) / np.maximum(1.0, np.abs(want))) < 1e-5  # the reference's float buffers
    if P().Decomposition(P().Graph.from_edges(n, u, v)).arrays()["n_chains"] == 0:
        assert np.max(np.abs(got - golden) / np.maximum(1.0, np.abs(golden))) < 1e-5
