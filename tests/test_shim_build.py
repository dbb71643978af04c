"""The reference-side binding compiles against the reference and links.

3d-eulerian-amr_b200/shim/amr_b200_drivers.h is the code a maintainer adds
to the reference: GpuHydroDriver (EULER build) and GpuBinaryDriver (BINARY
build), subclasses of the reference's own drivers whose step calls the C
ABI.  Each is compiled here against the reference's headers with that
build's defs.h configuration (the scratch copies oracle/build_ref.py makes:
src_g05 with EULER selected, src_ztwd12 the unpatched BINARY build), linked
with the reference's own objects and libamr_b200.so, and the program is
started (it makes no driver, so it needs no GPU).  Compile and link only:
the drivers' device runs are what the GPU tests check through the same ABI.
"""

import os
import subprocess

import pytest

from conftest import PKG, REF_BIN, ROOT

LIB = os.path.join(PKG, "lib")

MAIN = {
    # EULER build: euler/initialize.cpp does not compile in the reference
    # (r_outer undefined, euler/initialize.cpp:26,34), so the program gives
    # the one symbol the driver's step_to_time refers to
    "g05": ("GridNode", "GpuHydroDriver",
            '#include "grid/grid_node.h"\n#include "euler/hydro_driver.h"\n',
            "void initialize(GridNode*) {}\n"),
    "ztwd12": ("Binary", "GpuBinaryDriver",
               '#include "binary/binary.h"\n#include "binary/binary_driver.h"\n', ""),
}


def program(variant):
    root_cls, drv, includes, extra = MAIN[variant]
    return ('#include "defs.h"\n' + includes + '#include "amr_b200_drivers.h"\n' + extra +
            "int main(int argc, char**) {\n"
            "    if (argc > 99) {\n"
            "        %s* r = new %s;\n"
            "        %s d(r);\n"
            "        d.step(d.max_dt());\n"
            "        d.sync_to_reference();\n"
            "    }\n"
            "    return 0;\n"
            "}\n") % (root_cls, root_cls, drv)


@pytest.mark.parametrize("variant", ["g05", "ztwd12"])
def test_binding_compiles_links_and_loads(variant, tmp_path, table_path):
    src = os.path.join(REF_BIN, "src_" + variant)
    objdir = os.path.join(src, "_obj")
    if not os.path.isdir(objdir):
        pytest.skip("reference scratch build %s not present (oracle/build_ref.py)" % src)
    assert os.path.exists(os.path.join(LIB, "libamr_b200.so")), "build the library first"
    main = tmp_path / "main.cpp"
    main.write_text(program(variant))
    flags = ["-std=c++17", "-O1", "-fopenmp", "-w", "-I", src, "-I", os.path.join(ROOT, "include"), "-I",
             os.path.join(PKG, "shim")]
    obj = str(tmp_path / "main.o")
    r = subprocess.run(["g++"] + flags + ["-c", str(main), "-o", obj], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    objs = sorted(os.path.join(objdir, f) for f in os.listdir(objdir) if f.endswith(".o") and f != "harness.o")
    exe = str(tmp_path / "binding")
    cuda_lib = "/usr/local/cuda/lib64"
    r = subprocess.run(["g++", "-fopenmp", "-o", exe, obj] + objs +
                       ["-L", LIB, "-lamr_b200", "-L", cuda_lib, "-lcudart",
                        "-Wl,-rpath," + LIB + ":" + cuda_lib], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    # the BINARY build reads ./helmholtz.table while it starts
    os.symlink(table_path, str(tmp_path / "helmholtz.table"))
    r = subprocess.run([exe], cwd=str(tmp_path), capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
