"""The reference-side binding of INTEGRATION.md (CPU): the snippet there is
the file centrality-gpu_b200/reference_binding/begin_gpupgm_bcgpu.cpp, and
the reference's own host pipeline links against it and the in-tree
libbcgpu.so (oracle/_ref/refbetc, built from the reference's sources when
they are present). Running it needs a GPU; without one it must stop at its
first begin_gpu call with libbcgpu's error, not compute anything."""
import os
import re
import subprocess
from pathlib import Path

import pytest

from helpers import GOLDEN, GOLDEN_CASES, ROOT, canonical_chains, has_gpu, load_case, product_bccs
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
