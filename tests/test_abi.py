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


def test_config_checks_reconstruction_and_ghost_width():
    """PPM reads cells f-3..f+2 of face f (reconstruct.cpp:22-58), so it needs
    bw >= 3; minmod needs bw >= 2; unknown reconstructions are rejected."""
    from conftest import load_amr
    amr = load_amr()
    for kw in (dict(reconstruction=1, bw=2), dict(reconstruction=2, bw=3), dict(bw=1), dict(bw=5)):
        try:
            amr.AMR(max_bricks=0, **kw)
        except amr.AmrError as e:
            assert e.code == -1, kw
        else:
            raise AssertionError("config accepted: %r" % kw)
    for kw in (dict(reconstruction=1, bw=3), dict(reconstruction=0, bw=3), dict(reconstruction=1, bw=4)):
        a = amr.AMR(max_bricks=0, **kw)
        assert a.gnx == 8 + 2 * kw["bw"]
        a.close()
