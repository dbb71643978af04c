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
