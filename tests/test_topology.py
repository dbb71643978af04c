"""Octree topology and refinement decisions vs the reference (host only).

The reference's tree after its initialize/check_for_refine rounds
(grid_node.cpp:620-1033) is stored in the golden fixtures; the library's host
octree must reproduce it bit for bit (levels, locations, child masks) from
the same initial data.  Host-only contexts: no GPU needed.
"""

import numpy as np
import pytest

from cases import VARIANTS, golden_names, load_golden, same_tree
from conftest import load_amr

import importlib.util
import os
from conftest import PKG

spec = importlib.util.spec_from_file_location("amr_initial", os.path.join(PKG, "initial.py"))
initial = importlib.util.module_from_spec(spec)
spec.loader.exec_module(initial)


@pytest.mark.parametrize("name", golden_names("hydro_"))
def test_tree_build_matches_reference(name):
    amr = load_amr()
    g = load_golden(name)
    variant = str(g["variant"])
    ic, maxlevel, _, thr = [x for x in g["args"]]
    maxlevel, thr = int(maxlevel), float(thr)
    v = VARIANTS[variant]
    a = amr.AMR(max_bricks=0, max_refine_level=maxlevel, **v)
    initial.build_tree(a, str(ic), thr, v["grid_dim"], v["z_reflect"], maxlevel, device=False)
    t = a.get_tree()
    assert same_tree(t, g, "init_"), "tree differs from the reference"
    assert np.array_equal(t["age"], g["init_age"])


@pytest.mark.parametrize("name", ["poisson_poly_L2", "poisson_poly_L3", "grav_poly_L2", "grav_ppm_poly_L2"])
def test_polytrope_tree_matches_reference(name):
    """The oracle harness builds gravity trees at min_refine_density 1e-6."""
    amr = load_amr()
    g = load_golden(name)
    maxlevel = int(g["args"][1])
    a = amr.AMR(max_bricks=0, max_refine_level=maxlevel, **VARIANTS[str(g["variant"])])
    initial.build_tree(a, "polytrope", 1.0e-6, 0.5, 0, maxlevel, device=False)
    assert same_tree(a.get_tree(), g, "init_")


def test_load_tree_roundtrip():
    amr = load_amr()
    g = load_golden("hydro_bump_L3")
    a = amr.AMR(max_bricks=0, max_refine_level=3, grid_dim=0.5, z_reflect=0)
    a.load_tree(g["final_level"], g["final_loc"], g["final_age"])
    t = a.get_tree()
    assert same_tree(t, g, "final_")
    assert np.array_equal(t["age"], g["final_age"])
    # Grid::offset = 2*parent offset + BW + c*(GNX-2BW) (grid_node.cpp:244)
    for i in range(len(t["level"])):
        L = t["level"][i]
        assert np.all(t["offset"][i] == t["loc"][i] * 8 + 2 * (2 ** L - 1))


def test_refine_from_flags_regrid_sequence():
    """Regrid from the final state of a reference run: flags computed on the
    reference's own pre-regrid interiors reproduce its next tree."""
    amr = load_amr()
    g = load_golden("hydro_bump_L2")
    a = amr.AMR(max_bricks=0, max_refine_level=2, grid_dim=0.5, z_reflect=0)
    a.load_tree(g["final_level"], g["final_loc"], g["final_age"])
    a.set_time(float(g["final_time"]))
    # the reference regrids every step; its final tree is a fixed point of the
    # regrid on the final state (no young bricks at level < max)
    fl = initial.octant_flags(g["final_U"], 3.0)
    a.refine_from_flags(fl, True)
    assert same_tree(a.get_tree(), g, "final_")


@pytest.mark.parametrize("name", ["ztwd_L2", "ztwd_L3"])
def test_binary_initial_data_match_reference(name):
    """initial.py's binary (binary/initialize.cpp + floor + synchronous
    rotation) gives the reference harness's tree and refinement threshold,
    and its leaf bricks' state to the last bits of pow/Lane-Emden."""
    amr = load_amr()
    g = load_golden(name)
    L = int(g["init_level"].max())
    a = amr.AMR(max_bricks=0, physics=2, nf=13, bw=3, nx=8, reconstruction=1, grid_dim=1.0, z_reflect=1,
                max_refine_level=L, rho_floor=1e-10)
    a.init()
    U = initial.evaluate("binary", a.get_tree(), 3, 8, 1.0, 1, L, ghosts=False)
    thr = U[:, 0].max() / 1e6
    assert thr == g["extra"][6]
    t, U = initial.build_tree(a, "binary", thr, 1.0, 1, L, device=False)
    assert same_tree(t, g, "init_")
    leaf = t["child_mask"] == 0
    Ui, G = U[leaf][:, :, 3:-3, 3:-3, 3:-3], g["init_U"][leaf]
    scale = np.abs(G).max(axis=(0, 2, 3, 4))
    err = np.abs(Ui - G).max(axis=(0, 2, 3, 4)) / np.maximum(scale, 1e-300)
    assert err.max() <= 1e-14, err
