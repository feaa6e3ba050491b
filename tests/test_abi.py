"""The C-ABI library loads and exports every entry point the headers under
include/ declare (no compute: runs without a GPU)."""
import ctypes as C
import os
import re

from cupf_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header=None):
    inc = os.path.join(ROOT, "include")
    names = set()
    for h in sorted(os.listdir(inc)) if header is None else [header]:
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(inc, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(cupf_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol(built):
    lib = C.CDLL(abi.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layout_matches_ctypes_mirror(built):
    L = abi.lib()
    assert L.cupf_struct_size(0) == C.sizeof(abi.cupf_apt_params)
    assert L.cupf_struct_size(1) == C.sizeof(abi.cupf_apt_inputs)
    assert L.cupf_abi_version() == 1


def test_python_binding_covers_header():
    """Every declared entry point has argtypes in cupf_b200/abi.py (host-side
    helpers of include/cupf_host.h in cupf_b200/host_api.py)."""
    from cupf_b200 import host_api
    L = host_api._lib()
    for n in declared_functions():
        assert getattr(L, n).argtypes is not None or n in ("cupf_last_error", "cupf_abi_version"), n
