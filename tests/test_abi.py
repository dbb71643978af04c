"""The C-ABI library loads and exports every function include/*.h declares
(no compute calls: runs without a GPU)."""

import ctypes
import os
import re

from conftest import PKG, ROOT


def declared_functions():
    names = []
    inc = os.path.join(ROOT, "include")
    for fn in sorted(os.listdir(inc)):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(inc, fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b(?:int|double|float|void|long long|const char\s*\*)\s+(amr_\w+|helm_\w+)\s*\(", src):
            names.append(m.group(1))
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(os.path.join(PKG, "lib", "libamr_b200.so"))
    names = declared_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_host_only_context_rejects_device_calls():
    from conftest import load_amr
    amr = load_amr()
    a = amr.AMR(max_bricks=0)
    a.init()
    try:
        a.enforce_boundaries()
    except amr.AmrError as e:
        assert e.code == -8
    else:
        raise AssertionError("device call on a host-only context must fail")
