"""The C-ABI library loads and exports every symbol include/*.h declares (no GPU)."""
import ctypes
import os
import re

from seisfem_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"^\s*(?:[a-z_]+\s+\**)+\**(\w+)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if not n.startswith("SFG_")))


def test_library_exports_all_declared_symbols():
    L = ctypes.CDLL(api.LIBPATH)
    decl = declared_functions()
    assert "elastic_wave" in decl and "sfg_run" in decl and len(decl) >= 20
    for n in decl:
        assert hasattr(L, n), n
    assert sorted(api.EXPORTS) == decl


def test_status_strings_and_no_device_behaviour():
    L = api.lib()
    assert L.sfg_error_string(0) == b"ok"
    assert L.sfg_error_string(6) == b"energy bound exceeded"
    assert L.sfg_snapshot_rows(1000, 200) == 1 + 5
    assert L.sfg_snapshot_rows(1200, 200) == 7       # example 2 wavefield files hold 7 rows
    import torch
    if not torch.cuda.is_available():
        assert L.sfg_create(0) is None                # fails loudly, no fallback
