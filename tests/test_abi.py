"""The C-ABI library loads and exports every symbol include/*.h declares (no
compute calls: CPU only)."""
import re

from helpers import ROOT, pkg


def declared_in_headers():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(bc_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported():
    L = pkg().lib()
    names = declared_in_headers()
    assert len(names) >= 20
    for name in sorted(names):
        assert hasattr(L, name), name


def test_python_layer_binds_every_declared_symbol():
    assert declared_in_headers() == set(pkg().declared_symbols())


def test_library_is_the_in_tree_build():
    P = pkg()
    P.lib()
    maps = open("/proc/self/maps").read()
    assert str(P.LIB_PATH) in maps
