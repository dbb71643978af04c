"""Hydro step parity: CUDA plain FP64 path vs the reference CPU path.

Each golden case holds the reference's initial tree/state and its state
after N HydroDriver::step calls (euler/hydro_driver.cpp:171-194) with dt from
GridNode::max_dt and the MAXDTINC clamp.  The library replays the same steps
through the C ABI; trees must match bit for bit, dt to 1e-13 and every field
to 1e-12 (max |a-b| / max |b| per field).
"""

import os
import tempfile

import numpy as np
import pytest

from cases import (DT_RTOL, FP64_FIELD_RTOL, VARIANTS, field_rel_err, golden_names, load_golden, same_tree)
from conftest import PKG, ref_binary, run_ref
import importlib.util

spec = importlib.util.spec_from_file_location("amr_initial", os.path.join(PKG, "initial.py"))
initial = importlib.util.module_from_spec(spec)
spec.loader.exec_module(initial)


def make(gpu, variant, maxlevel, **kw):
    v = VARIANTS[variant]
    return gpu.AMR(max_refine_level=maxlevel, max_bricks=2048, **v, **kw)


def load_state(a, level, loc, age, U_int):
    a.load_tree(level, loc, age)
    bw = a.bw
    U = np.zeros((a.nbricks, a.nf, a.gnx, a.gnx, a.gnx))
    U[:, :, bw:-bw, bw:-bw, bw:-bw] = U_int
    a.upload_state(U)
    a.enforce_boundaries()


def run_steps(a, nsteps, thr):
    dts = []
    last = 0.0
    for s in range(nsteps):
        dt = a.max_dt()
        if s > 0:
            dt = min(last * 1.25, dt)
        last = dt
        dts.append(dt)
        a.hydro_step(dt, thr)
    return np.array(dts)


def interior(a, U):
    b = a.bw
    return U[:, :, b:-b, b:-b, b:-b]


@pytest.mark.gpu
@pytest.mark.parametrize("name", golden_names("hydro_"))
def test_hydro_matches_reference(gpu, name):
    g = load_golden(name)
    variant = str(g["variant"])
    ic, maxlevel, nsteps, thr = [x for x in g["args"]]
    maxlevel, nsteps, thr = int(maxlevel), int(nsteps), float(thr)
    a = make(gpu, variant, maxlevel)
    v = VARIANTS[variant]
    if "init_U" in g:
        load_state(a, g["init_level"], g["init_loc"], g["init_age"], g["init_U"])
    else:
        initial.build_tree(a, str(ic), thr, v["grid_dim"], v["z_reflect"], maxlevel, device=True)
        assert same_tree(a.get_tree(), g, "init_")
    dts = run_steps(a, nsteps, thr)
    ref_dts = g["extra"][:nsteps]
    np.testing.assert_allclose(dts, ref_dts, rtol=DT_RTOL if "init_U" in g else 1e-11)
    t = a.get_tree()
    assert same_tree(t, g, "final_")
    assert np.array_equal(t["age"], g["final_age"])
    U = interior(a, a.download_state())
    if "final_U" in g:
        err = field_rel_err(U, g["final_U"])
        assert np.all(err <= FP64_FIELD_RTOL), err
    else:
        s = U.reshape(U.shape[0], U.shape[1], -1).sum(axis=2)
        sa = np.abs(U).reshape(U.shape[0], U.shape[1], -1).sum(axis=2)
        rel = np.abs(s - g["final_Usum"]) / np.maximum(g["final_Uabs"], 1e-300)
        assert rel.max() <= 1e-11, rel.max()
        np.testing.assert_allclose(sa, g["final_Uabs"], rtol=1e-11)
    fo = a.flow_off()
    np.testing.assert_allclose(fo, g["final_FO"], rtol=1e-11, atol=1e-14 * max(1.0, np.abs(g["final_FO"]).max()))
    a.close()


@pytest.mark.gpu
def test_hydro_matches_reference_live_bump_L3():
    """Full-state comparison against a live run of the reference binary
    (travels with the repository as oracle/_ref) when it is present."""
    if ref_binary("g05") is None:
        pytest.skip("oracle/_ref not built")
    import conftest
    gpu = conftest.load_amr()
    from dumpio import read_dump
    with tempfile.TemporaryDirectory() as td:
        run_ref(["hydro", "bump", 3, 6, 3.0, "o.bin"], td)
        d0 = read_dump(os.path.join(td, "o.bin.init"))
        d1 = read_dump(os.path.join(td, "o.bin"))
    a = make(gpu, "g05", 3)
    bw = d0.bw
    load_state(a, d0.level, d0.loc, d0.age, d0.U[:, :, bw:-bw, bw:-bw, bw:-bw])
    dts = run_steps(a, 6, 3.0)
    np.testing.assert_allclose(dts, d1.extra[:6], rtol=DT_RTOL)
    t = a.get_tree()
    assert np.array_equal(t["level"], d1.level) and np.array_equal(t["loc"], d1.loc)
    U = interior(a, a.download_state())
    err = field_rel_err(U, d1.U[:, :, bw:-bw, bw:-bw, bw:-bw])
    assert np.all(err <= FP64_FIELD_RTOL), err
    a.close()


@pytest.mark.gpu
def test_substep_operations_individually(gpu):
    """enforce_boundaries / compute_fluxes / add_difs / inject / store /
    restore through the ABI compose to one hydro_step."""
    g = load_golden("hydro_bump_L2")
    a = make(gpu, "g05", 2)
    load_state(a, g["init_level"], g["init_loc"], g["init_age"], g["init_U"])
    b = make(gpu, "g05", 2)
    load_state(b, g["init_level"], g["init_loc"], g["init_age"], g["init_U"])
    dt = a.max_dt()
    a.hydro_step(dt, 3.0)
    b.store()
    for beta in (1.0, 0.25, 2.0 / 3.0):
        b.enforce_boundaries()
        b.compute_fluxes()
        b.add_difs(dt, beta)
        b.inject_from_children()
    b.enforce_boundaries()
    b.check_for_refine(3.0)
    Ua, Ub = a.download_state(), b.download_state()
    assert np.array_equal(interior(a, Ua), interior(b, Ub))
    # store/restore round trip
    b.store()
    b.sub_step(dt, 1.0)
    b.restore()
    assert np.array_equal(b.download_state(), Ub)
