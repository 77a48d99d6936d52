"""CPU-side checks of the C ABI: the library loads and exports every declared symbol."""
import os
import re
import subprocess

from conftest import ROOT


def header_symbols():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", f)).read()
            names |= set(re.findall(r"^\s*(?:int|int32_t|int64_t|size_t|void|const char\s*\*)\s+(mw_\w+)\s*\(", txt,
                                    re.M))
    return names


def test_library_builds_and_exports_all_declared_symbols():
    from meeuuw_b200 import build as B
    lib = B.build()
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (mw_\w+)", out))
    declared = header_symbols()
    assert declared, "no declarations found"
    missing = declared - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"


def test_ctypes_prototypes_cover_header():
    import ctypes
    from meeuuw_b200 import _lib
    from meeuuw_b200 import build as B
    B.build()
    L = ctypes.CDLL(_lib.LIB_PATH)          # loading needs no GPU (static runtime, driver dlopened lazily)
    for name in header_symbols():
        assert hasattr(L, name)
    assert set(_lib.declared_symbols()) <= header_symbols()
    assert L.mw_bin_workspace_bytes(1000) > 0
