"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference oracle harness (oracle/_ref/*_harness, built from the
reference sources by oracle/build_ref.py) on small cases and stores, per
case, the initial and final octree and the interior cells of every brick
(ghost slabs are recomputed from interiors), the per-step dt sequence and the
root flow-off accumulator.  Re-running this script must reproduce the
committed files bit for bit (tests/test_oracle_ref.py checks that).

    python tests/golden/make_golden.py [case ...]
"""

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from dumpio import read_dump  # noqa: E402

# name: (variant, mode, argv after mode)
CASES = {
    "hydro_blast_L2": ("g05", "hydro", ["blast", 2, 20, 1e-6]),
    "hydro_bump_L2": ("g05", "hydro", ["bump", 2, 5, 3.0]),
    "hydro_bump_L3": ("g05", "hydro", ["bump", 3, 4, 3.0]),
    "hydro_bump_zr_L3": ("zr", "hydro", ["bump", 3, 4, 3.0]),
    "hydro_ppm_bump_L2": ("ppm", "hydro", ["bump", 2, 5, 3.0]),
    "hydro_ppm_blast_L2": ("ppm", "hydro", ["blast", 2, 20, 1e-6]),
    "poisson_poly_L2": ("g05", "poisson", ["polytrope", 2, 4]),
    "poisson_poly_L3": ("g05", "poisson", ["polytrope", 3, 3]),
    "grav_poly_L2": ("g05", "grav", ["polytrope", 2, 3, 1e-6]),
    "grav_ppm_poly_L2": ("ppm", "grav", ["polytrope", 2, 3, 1e-6]),
    # ZTWD binary (BINARY build): maxlevel, steps
    "ztwd_L2": ("ztwd", "ztwd", [2, 3]),
    "ztwd_L3": ("ztwd", "ztwd", [3, 9]),
    # the same on the BINARY build's own 12^3-cell bricks
    "ztwd12_L2": ("ztwd12", "ztwd", [2, 3]),
    "ztwd12_L3": ("ztwd12", "ztwd", [3, 9]),
    # the configured sizes: the 4-level single star (9 coupled steps, regrids
    # at steps 0 and 8) and the 5-level binary on 12^3 bricks (10
    # BinaryDriver steps, regrids at steps 0 and 8)
    "grav_poly_L4": ("g05", "grav", ["polytrope", 4, 9, 1e-6]),
    "ztwd12_L5": ("ztwd12", "ztwd", [5, 10]),
}
# cases whose full state would make a large fixture keep only the tree and
# per-brick, per-field sums and absolute sums of the interior cells
SUMMARY_ONLY = {"hydro_bump_L3"}
# Poisson cases whose state is rebuilt by the test from the host initializer:
# sums of the state, every cell of the potential after each V-cycle
PHI_ONLY = {"poisson_poly_L3"}
# cases too large for every cell: the initial state as sums only (a test
# regenerates it with a zero-step run of the same harness and checks the
# sums), the final state as sums plus every cell of a fixed sample of bricks
# (evenly spaced in depth-first order) and the per-field maxima
SAMPLED = {"grav_poly_L4": 24, "ztwd12_L5": 24}


def sample_bricks(n, k):
    """Indices of k bricks evenly spaced over n (all of them when n <= k)."""
    return np.unique(np.linspace(0, n - 1, min(n, k)).round().astype(np.int64))


def interior(d, U):
    b = d.bw
    return U[:, :, b:-b, b:-b, b:-b].copy()


def pack(prefix, d, summary, sample=0, phi=False):
    U = interior(d, d.U)
    out = {
        prefix + "level": d.level, prefix + "loc": d.loc, prefix + "age": d.age,
        prefix + "child_mask": d.child_mask, prefix + "refine_mask": d.refine_mask,
        prefix + "FO": d.FO, prefix + "time": np.float64(d.time),
        prefix + "Usum": U.reshape(U.shape[0], U.shape[1], -1).sum(axis=2),
        prefix + "Uabs": np.abs(U).reshape(U.shape[0], U.shape[1], -1).sum(axis=2),
    }
    if not summary:
        out[prefix + "U"] = U
    if d.P is not None and (phi or not summary):
        out[prefix + "phi"] = d.P["phi"]
    if d.P is not None:
        out[prefix + "phisum"] = d.P["phi"][:, 1:-1, 1:-1, 1:-1].reshape(d.nnodes, -1).sum(axis=1)
    if sample:
        idx = sample_bricks(U.shape[0], sample)
        out[prefix + "sample"] = idx
        out[prefix + "sample_U"] = U[idx]
        out[prefix + "Umax"] = np.abs(U).max(axis=(0, 2, 3, 4))
        if d.P is not None:
            out[prefix + "sample_phi"] = d.P["phi"][idx]
            out[prefix + "phimax"] = np.float64(np.abs(d.P["phi"][:, 1:-1, 1:-1, 1:-1]).max())
    return out


def run_case(name, workdir, threads=1):
    variant, mode, args = CASES[name]
    exe = os.path.join(ROOT, "oracle", "_ref", variant + "_harness")
    out = os.path.join(workdir, name + ".bin")
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    if mode == "ztwd":
        # the BINARY build reads ./helmholtz.table at start-up (helmeos.cpp:73-130)
        sys.path.insert(0, os.path.join(ROOT, "3d-eulerian-amr_b200"))
        import helm_table
        helm_table.ensure_table(workdir)
    r = subprocess.run([exe, mode] + [str(a) for a in args] + [out], cwd=workdir, env=env,
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stdout + r.stderr)
    d0 = read_dump(out + ".init")
    summ = name in SUMMARY_ONLY or name in SAMPLED or name in PHI_ONLY
    res = {"variant": np.array(variant), "mode": np.array(mode), "args": np.array([str(a) for a in args]),
           "bw": np.int32(d0.bw), "nx": np.int32(d0.gnx - 2 * d0.bw)}
    res.update(pack("init_", d0, summ))
    if mode == "poisson":
        ncyc = int(args[2])
        for c in range(ncyc):
            dc = read_dump(out + ".%d" % c)
            res.update(pack("cycle%d_" % c, dc, summ, phi=name in PHI_ONLY))
            res["extra"] = dc.extra
    else:
        d1 = read_dump(out)
        res["extra"] = d1.extra
        res.update(pack("final_", d1, summ, SAMPLED.get(name, 0)))
    return res


def main(names):
    with tempfile.TemporaryDirectory() as td:
        for n in names:
            res = run_case(n, td)
            path = os.path.join(HERE, n + ".npz")
            np.savez_compressed(path, **res)
            print(n, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1:] or list(CASES))
