"""Shared helpers for the parity tests: golden cases and tolerances."""

import os

import numpy as np

from conftest import GOLDEN

# FP64 plain form vs the reference CPU path: relative error per field,
# measured as max|a-b| / max|b| over the compared cells.
FP64_FIELD_RTOL = 1.0e-12
# dt sequence (exact max/min reductions, identical arithmetic)
DT_RTOL = 1.0e-13

VARIANTS = {
    "g05": dict(grid_dim=0.5, z_reflect=0),
    "zr": dict(grid_dim=1.0, z_reflect=1),
    # PPM reconstruction (reconstruct.cpp:22-58) with BW 3, unit cube
    "ppm": dict(grid_dim=0.5, z_reflect=0, bw=3, reconstruction=1),
}


def oracle_recon(variant):
    """Reconstruction name of amr_oracle for a variant."""
    return "ppm" if VARIANTS[variant].get("reconstruction", 0) == 1 else "minmod"


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def golden_names(prefix):
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.startswith(prefix) and f.endswith(".npz"))


def field_rel_err(a, b):
    """Per-field relative error: max |a-b| / max |b| over all cells."""
    nf = a.shape[1]
    out = np.zeros(nf)
    for l in range(nf):
        den = np.abs(b[:, l]).max()
        out[l] = np.abs(a[:, l] - b[:, l]).max() / (den if den > 0 else 1.0)
    return out


def same_tree(t, g, prefix):
    return (np.array_equal(t["level"], g[prefix + "level"]) and np.array_equal(t["loc"], g[prefix + "loc"])
            and np.array_equal(t["child_mask"], g[prefix + "child_mask"]))


def live_initial_state(variant, args, workdir, table_path=None):
    """The initial tree and state of a golden case whose fixture keeps only
    their sums: a zero-step run of the same reference harness (oracle/_ref),
    read back from its dump.  Test infrastructure only."""
    import os
    import subprocess

    from conftest import ref_binary
    from dumpio import read_dump

    exe = ref_binary(variant)
    assert exe is not None, "oracle/_ref/%s_harness is needed for this case" % variant
    if table_path is not None:
        os.symlink(table_path, os.path.join(workdir, "helmholtz.table"))
    out = os.path.join(workdir, "init.bin")
    argv = [exe] + [str(a) for a in args] + [out]
    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
    r = subprocess.run(argv, cwd=workdir, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    return read_dump(out + ".init")


def check_initial_sums(d, g):
    """The live initial state is the one the golden run started from: same
    tree, per-brick sums and absolute sums equal bit for bit."""
    b = d.bw
    U = d.U[:, :, b:-b, b:-b, b:-b]
    assert np.array_equal(d.level, g["init_level"]) and np.array_equal(d.loc, g["init_loc"])
    assert np.array_equal(U.reshape(U.shape[0], U.shape[1], -1).sum(axis=2), g["init_Usum"])
    assert np.array_equal(np.abs(U).reshape(U.shape[0], U.shape[1], -1).sum(axis=2), g["init_Uabs"])


def check_final_sampled(U, phi, g, rtol=FP64_FIELD_RTOL):
    """A sampled golden's final state: every cell of the sampled bricks
    within rtol of the field's maximum over all bricks (max |a-b| / max |b|
    per field), and every brick's per-field sum within 1e-11 of its sum of
    absolute values.  U: interiors [n][nf][nx][nx][nx]; phi: [n][pnx]^3."""
    idx = g["final_sample"]
    den = np.where(g["final_Umax"] > 0, g["final_Umax"], 1.0)
    err = np.abs(U[idx] - g["final_sample_U"]).max(axis=(0, 2, 3, 4)) / den
    assert np.all(err <= rtol), err
    s = U.reshape(U.shape[0], U.shape[1], -1).sum(axis=2)
    rel = np.abs(s - g["final_Usum"]) / np.maximum(g["final_Uabs"], 1e-300)
    assert rel.max() <= 1e-11, rel.max()
    if phi is not None and "final_sample_phi" in g:
        ep = np.abs(phi[idx][:, 1:-1, 1:-1, 1:-1] - g["final_sample_phi"][:, 1:-1, 1:-1, 1:-1]).max()
        assert ep <= rtol * float(g["final_phimax"]), ep / float(g["final_phimax"])
    return err
