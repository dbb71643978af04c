"""Build recipe for the CUDA library (sm_100a) and the ctypes wrapper.

    python 3d-eulerian-amr_b200/build.py

compiles csrc/*.cu and csrc/*.cpp with nvcc into
3d-eulerian-amr_b200/lib/libamr_b200.so (in-tree, so it travels with the
repository snapshot).  Two compilation rules matter for results:
  * --fmad=false on every FP64 kernel: the plain form must not contract
    a*b+c into FMA, so it rounds like the reference's x86-64 build;
  * the mixed-precision kernels (files named *_mixed.cu) allow FMA.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", INCLUDE]


def _sources():
    out = []
    for fn in sorted(os.listdir(CSRC)):
        if fn.endswith(".cu") or fn.endswith(".cpp"):
            out.append(os.path.join(CSRC, fn))
    return out


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def build(verbose=False, force=False):
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    lib = os.path.join(LIBDIR, "libamr_b200.so")
    hdr_time = max(os.path.getmtime(h) for h in _headers() + [os.path.abspath(__file__)])
    objs, procs = [], []
    for src in _sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) > max(os.path.getmtime(src), hdr_time)):
            continue
        flags = list(COMMON)
        if src.endswith(".cu"):
            flags += ARCH + ["-Xptxas", "-v"] if verbose else ARCH
            if not src.endswith("_mixed.cu"):
                flags += ["--fmad=false"]
        else:
            flags += ["-x", "cu"] + ARCH + ["--fmad=false"]
        cmd = [NVCC] + flags + ["-c", src, "-o", obj]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed = True
            sys.stderr.write("nvcc failed for %s:\n%s\n" % (src, out))
        elif verbose and out:
            sys.stderr.write(out)
    if failed:
        raise RuntimeError("CUDA build failed")
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(lib) or os.path.getmtime(lib) < newest:
        cmd = [NVCC, "-shared"] + ARCH + ["-o", lib] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
