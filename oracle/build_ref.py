"""Build the reference code as a test oracle (oracle/_ref/).

Test infrastructure only.  The reference (STEllAR-GROUP/3d-eulerian-amr) is a
plain C++/OpenMP code with no build system beyond an Intel-compiler Makefile
that links Silo.  This recipe

  1. copies the read-only reference tree into a git-ignored scratch directory
     oracle/_ref/src_<variant>/ (the sources are never committed),
  2. applies the minimal scripted patches listed in PATCHES below,
  3. compiles the reference's own grid/, oct_node/, euler/, poisson/ sources
     together with the harness in oracle/harness/ using g++ -O3 -fopenmp
     -ffp-contract=off (no FMA contraction, like the reference's x86-64 build),
  4. writes the executables to oracle/_ref/<variant>_harness.

It also builds oracle/_ref/helm_harness from helmholtz/helmeos.cpp (which
compiles unpatched) for the Helmholtz EOS oracle.

Variants:
  g05  EULER physics, GRID_DIM 0.5, no Z_REFLECT  (unit cube [-0.5,0.5]^3)
  zr   EULER physics, GRID_DIM 1.0, Z_REFLECT     (the reference's stock
       euler/euler_defs.h domain: x,y in [-1,1], z in [0,2] mirrored at z=0)
  ppm  g05 with PPM reconstruction (euler_defs.h:24 switched on) and BW 3,
       the ghost width PPM needs (reconstruct.cpp:22-58 reads cells i-3..i+2
       of face i)
  ztwd12 BINARY physics with the ZTWD state exactly as binary/binary_defs.h
       sets it (PPM, BW 3, Z_REFLECT, GRID_DIM 1, 12^3 interior cells per
       brick); driven by oracle/harness/ztwd_harness.cpp, with the
       reference's own binary/initialize.cpp as the initial data
  ztwd the same with 8^3 interior cells per brick (GNX 8+2*BW), a second
       brick size the CUDA path also runs

Run:  python oracle/build_ref.py [--reference DIR]
The reference tree is DIR, else $AMR_REFERENCE, else a directory named
`reference` beside this repository's directory.  When it is absent (e.g. on
a GPU box) this is a no-op and the previously built binaries are used as
they are.
"""

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")

EULER_SOURCES = [
    "assert.cpp", "indexer_2d.cpp", "indexer_2d_by2.cpp", "reconstruct.cpp",
    "grid/grid.cpp", "grid/grid_node.cpp", "grid/grid_amr_bound.cpp",
    "grid/grid_phys_bound.cpp", "grid/grid_interface.cpp",
    "oct_node/child_index.cpp", "oct_node/oct_face.cpp", "oct_node/oct_node.cpp",
    "euler/state.cpp", "euler/hydro_driver.cpp",
    "poisson/poisson.cpp", "poisson/poisson_amr_bound.cpp",
    "poisson/poisson_phys_bound.cpp", "binary/lane_emden.cpp",
]

COMMON_SOURCES = [
    "assert.cpp", "indexer_2d.cpp", "indexer_2d_by2.cpp", "reconstruct.cpp",
    "grid/grid.cpp", "grid/grid_node.cpp", "grid/grid_amr_bound.cpp",
    "grid/grid_phys_bound.cpp", "grid/grid_interface.cpp",
    "oct_node/child_index.cpp", "oct_node/oct_face.cpp", "oct_node/oct_node.cpp",
    "poisson/poisson.cpp", "poisson/poisson_amr_bound.cpp",
    "poisson/poisson_phys_bound.cpp",
]
BINARY_SOURCES = COMMON_SOURCES + [
    "binary/binary.cpp", "binary/binary_driver.cpp", "binary/state_ztwd.cpp",
    "binary/state.cpp", "binary/lane_emden.cpp", "binary/initialize.cpp",
    "helmholtz/helmeos.cpp",
]

CXXFLAGS = ["-O3", "-fopenmp", "-ffp-contract=off", "-DNDEBUG", "-w"]


def _replace(path, old, new, count=1):
    with open(path) as f:
        s = f.read()
    if old not in s:
        raise RuntimeError("patch anchor not found in %s: %r" % (path, old))
    s = s.replace(old, new, count)
    with open(path, "w") as f:
        f.write(s)


def _patch(src, variant):
    # real.h:14,33-35 declares Real abs(Real), which clashes with libstdc++'s
    # abs(double) under g++ >= 6.
    _replace(os.path.join(src, "real.h"), "Real abs(Real);", "")
    _replace(os.path.join(src, "real.h"),
             "inline Real abs(Real a) {\n\treturn fabs(a);\n}", "")
    # Silo is not installed; only the output path uses it.
    shutil.copy(os.path.join(HERE, "stubs", "silo.h"), os.path.join(src, "silo.h"))
    if variant == "ztwd12":
        return
    if variant == "ztwd":
        # binary/binary_defs.h:31-35: 12^3 interior cells -> 8^3
        bdefs = os.path.join(src, "binary", "binary_defs.h")
        _replace(bdefs, "#define GNX \t\t\t\t(12+2*BW)", "#define GNX \t\t\t\t(8+2*BW)", count=2)
        return
    # defs.h:4 hard-codes the BINARY driver; select the Euler state.
    _replace(os.path.join(src, "defs.h"), "#define BINARY", "#define EULER")
    defs = os.path.join(src, "euler", "euler_defs.h")
    if variant in ("g05", "ppm"):
        _replace(defs, "#define GRID_DIM            (1.0)", "#define GRID_DIM            (0.5)")
        _replace(defs, "#define Z_REFLECT\n", "\n")
    if variant == "ppm":
        _replace(defs, "//#define PPM\n", "#define PPM\n")
        _replace(defs, "#define BW \t\t\t\t\t(2)", "#define BW \t\t\t\t\t(3)")
    # euler/initialize.cpp:26,34 does not compile (r_outer undefined); the
    # harness defines initialize(GridNode*) instead.
    with open(os.path.join(src, "euler", "initialize.cpp"), "w") as f:
        f.write("// replaced by oracle/harness/amr_harness.cpp\n")


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("command failed: %s" % " ".join(cmd))


def _stale(out, inputs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(p) > t for p in inputs)


def build_variant(reference, variant, jobs=8):
    src = os.path.join(REF_OUT, "src_" + variant)
    exe = os.path.join(REF_OUT, variant + "_harness")
    binary = variant in ("ztwd", "ztwd12")
    harness = os.path.join(HERE, "harness", "ztwd_harness.cpp" if binary else "amr_harness.cpp")
    sources = BINARY_SOURCES if binary else EULER_SOURCES
    inputs = [harness, os.path.abspath(__file__), os.path.join(HERE, "stubs", "silo.h"),
              os.path.join(HERE, "harness", "dump.h")]
    if not _stale(exe, inputs):
        return exe
    if os.path.exists(src):
        shutil.rmtree(src)
    shutil.copytree(reference, src, ignore=shutil.ignore_patterns(".git"))
    for root, dirs, files in os.walk(src):
        os.chmod(root, 0o755)
        for fn in files:
            os.chmod(os.path.join(root, fn), 0o644)
    _patch(src, variant)
    objdir = os.path.join(src, "_obj")
    os.makedirs(objdir, exist_ok=True)
    procs, objs = [], []
    for s in sources:
        o = os.path.join(objdir, s.replace("/", "_") + ".o")
        objs.append(o)
        procs.append(subprocess.Popen(["g++"] + CXXFLAGS + ["-I", src, "-c", os.path.join(src, s), "-o", o],
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
        if len(procs) >= jobs:
            p = procs.pop(0)
            out, err = p.communicate()
            if p.returncode:
                raise RuntimeError("compile failed:\n" + out + err)
    for p in procs:
        out, err = p.communicate()
        if p.returncode:
            raise RuntimeError("compile failed:\n" + out + err)
    ho = os.path.join(objdir, "harness.o")
    _run(["g++"] + CXXFLAGS + ["-I", src, "-I", os.path.join(HERE, "harness"), "-c", harness, "-o", ho])
    _run(["g++", "-fopenmp", "-o", exe] + objs + [ho])
    return exe


def build_helm(reference):
    exe = os.path.join(REF_OUT, "helm_harness")
    harness = os.path.join(HERE, "harness", "helm_harness.cpp")
    if not os.path.exists(harness):
        return None
    if not _stale(exe, [harness, os.path.abspath(__file__)]):
        return exe
    src = os.path.join(REF_OUT, "src_helm")
    if os.path.exists(src):
        shutil.rmtree(src)
    os.makedirs(src)
    for fn in ("helmeos.cpp", "helmholtz.h", "const.h"):
        shutil.copy(os.path.join(reference, "helmholtz", fn), os.path.join(src, fn))
    _run(["g++"] + CXXFLAGS + ["-I", src, "-o", exe, os.path.join(src, "helmeos.cpp"), harness])
    return exe


def default_reference():
    """$AMR_REFERENCE, else `reference` beside the repository's directory."""
    env = os.environ.get("AMR_REFERENCE")
    if env:
        return env
    return os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")


def build(reference=None, variants=("g05", "zr", "ppm", "ztwd", "ztwd12")):
    reference = reference or default_reference()
    if not os.path.isdir(reference):
        print("[oracle] reference tree not present; using prebuilt oracle/_ref binaries")
        return []
    os.makedirs(REF_OUT, exist_ok=True)
    built = [build_variant(reference, v) for v in variants]
    h = build_helm(reference)
    if h:
        built.append(h)
    return built


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None)
    a = ap.parse_args()
    for e in build(a.reference):
        print(e)
