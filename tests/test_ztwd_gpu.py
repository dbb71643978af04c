"""ZTWD binary (BINARY build of the reference) through the C ABI.

ztwd_*: the reference's own two-polytrope initial data (binary/initialize.cpp)
for a q = 0.7 binary in the co-rotating frame, then BinaryDriver::step
(binary/binary_driver.cpp:346-459) with dt from GridNode::max_dt and the
MAXDTINC clamp, run by oracle/harness/ztwd_harness.cpp on the reference's
BINARY build (ZTWD state, PPM, BW 3; ztwd12_* on its own 12^3 bricks,
ztwd_* on 8^3 bricks) reading the synthetic Helmholtz table.  The library
replays the same steps (amr_ztwd_step); trees must match bit for bit, dt to
1e-12 and every cell of every field to 1e-12 (max |a-b| / max |b| per
field), across the regrids at steps 0 and 8.
"""

import os

import numpy as np
import pytest

from cases import FP64_FIELD_RTOL, field_rel_err, load_golden, same_tree
from conftest import _load_pkg_module

DT_RTOL = 1.0e-12
ELL_TOLER = 1.0e-7     # binary/binary_defs.h:64
DYNAMIC_RANGE = 1.0e6  # binary/binary_defs.h:14
MIXED_RTOL = 1.0e-6    # mixed + persistent form against FP64, density / energy rel L1 after the run
# the same forms' potential, relative L2 over the interior cells after the run:
# FP64 itself, solved to ELL_TOLER, moves by up to ~1e-9 in the potential when
# the density is perturbed by 1e-15 (the solve stops at a different iterate),
# so the bound is a small multiple of that, far below the 1e-6 solver error
MIXED_PHI_RTOL = 1.0e-8


def ztwd_config(maxlevel, nx=8, **kw):
    """The BINARY build's compile-time constants (binary/binary_defs.h) with
    nx^3 interior cells per brick (12 in the reference's build)."""
    cfg = dict(physics=2, nf=13, bw=3, nx=nx, reconstruction=1, grid_dim=1.0, z_reflect=1, mirror_refine_y=1,
               max_refine_level=maxlevel, rho_floor=1.0e-10, cfl=0.3, maxdtinc=1.25, max_bricks=1024)
    cfg.update(kw)
    return cfg


def make(gpu, g, table_path, **kw):
    helm = _load_pkg_module("helm_b200", "helm.py").Helm(table_path)
    K1, Ucm, Ug, Us, omega, omega0 = [float(x) for x in g["extra"][:6]]
    helm.set_cgs_units(Ucm, Ug, Us, 1.0)  # Binary::set_units (binary/binary.h:17-35)
    a = gpu.AMR(**ztwd_config(int(g["init_level"].max()), nx=int(g["nx"]), **kw))
    a.ztwd_set_eos(helm)
    a.ztwd_set_frame(omega, omega0, 0.0, 0.0)
    a.load_tree(g["init_level"], g["init_loc"], g["init_age"])
    bw = a.bw
    U = np.zeros((a.nbricks, a.nf, a.gnx, a.gnx, a.gnx))
    U[:, :, bw:-bw, bw:-bw, bw:-bw] = g["init_U"]
    a.upload_state(U)
    a.enforce_boundaries()
    return a


def run(a, nsteps):
    dts, last = [], 0.0
    for s in range(nsteps):
        dt = a.max_dt()
        if s > 0:
            dt = min(last * 1.25, dt)
        dt = a.ztwd_step(dt, ELL_TOLER, DYNAMIC_RANGE, s)
        last = dt
        dts.append(dt)
    return np.array(dts)


def interior(a):
    b = a.bw
    return a.download_state()[:, :, b:-b, b:-b, b:-b]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ztwd_L2", "ztwd_L3", "ztwd12_L2", "ztwd12_L3"])
def test_ztwd_steps_match_reference(gpu, table_path, name):
    g = load_golden(name)
    nsteps = int(g["args"][1])
    a = make(gpu, g, table_path)
    dts = run(a, nsteps)
    ex = g["extra"]
    np.testing.assert_allclose(dts, ex[8:8 + nsteps], rtol=DT_RTOL)
    t = a.get_tree()
    assert same_tree(t, g, "final_")
    assert np.array_equal(t["age"], g["final_age"])
    U = interior(a)
    if "final_U" in g:
        err = field_rel_err(U, g["final_U"])
        assert np.all(err <= FP64_FIELD_RTOL), err
    else:
        s = U.reshape(U.shape[0], U.shape[1], -1).sum(axis=2)
        rel = np.abs(s - g["final_Usum"]) / np.maximum(g["final_Uabs"], 1e-300)
        assert rel.max() <= 1e-11, rel.max()
    fo = a.flow_off()
    np.testing.assert_allclose(fo, g["final_FO"], rtol=1e-10, atol=1e-13 * max(1.0, np.abs(g["final_FO"]).max()))
    a.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ztwd_L2", "ztwd12_L2"])
@pytest.mark.parametrize("prec", ["PREC_MIXED", "PREC_MIXED_SOLVE"])
def test_ztwd_mixed_persistent_close_to_fp64(gpu, table_path, name, prec):
    """The mixed forms in the persistent solve -- FP32 multigrid correction,
    with (PREC_MIXED) or without (PREC_MIXED_SOLVE) the FP32 reconstruction
    and KT flux -- against the FP64 form after the same steps: same trees and
    steps, density and energy within MIXED_RTOL (relative L1), the potential
    within MIXED_PHI_RTOL (relative L2)."""
    g = load_golden(name)
    nsteps = int(g["args"][1])
    a = make(gpu, g, table_path)
    b = make(gpu, g, table_path, precision=getattr(gpu, prec), persistent_solve=2)
    run(a, nsteps)
    run(b, nsteps)
    assert same_tree(b.get_tree(), {"final_" + k: v for k, v in a.get_tree().items()}, "final_")
    ua, ub = interior(a), interior(b)
    for f in (0, 7):
        l1 = np.abs(ub[:, f] - ua[:, f]).sum() / np.abs(ua[:, f]).sum()
        assert l1 <= MIXED_RTOL, (f, l1)
    pa, pb = a.download_poisson()[0][:, 1:-1, 1:-1, 1:-1], b.download_poisson()[0][:, 1:-1, 1:-1, 1:-1]
    l2 = np.sqrt(((pb - pa) ** 2).sum() / (pa ** 2).sum())
    assert l2 <= MIXED_PHI_RTOL, l2
    a.close()
    b.close()


@pytest.mark.gpu
def test_ztwd_calls_need_the_eos(gpu):
    a = gpu.AMR(**ztwd_config(1))
    a.init()
    with pytest.raises(gpu.AmrError) as e:
        a.enforce_boundaries()
    assert e.value.code == -6  # AMR_ERR_STATE
    a.close()


@pytest.mark.gpu
def test_ztwd_diagnostics_match_reference(gpu, table_path):
    """Binary::mass_sum of both stars, Binary::sum_lz and GridNode::state_sum
    of the density, on the reference's own final state of ztwd_L2: equal to
    the reference's one-thread values bit for bit (same data, same order)."""
    g = load_golden("ztwd_L2")
    nsteps = int(g["args"][1])
    diag = g["extra"][8 + nsteps:]
    a = gpu.AMR(**ztwd_config(int(g["final_level"].max())))
    a.load_tree(g["final_level"], g["final_loc"], g["final_age"])
    bw = a.bw
    U = np.zeros((a.nbricks, a.nf, a.gnx, a.gnx, a.gnx))
    U[:, :, bw:-bw, bw:-bw, bw:-bw] = g["final_U"]
    a.upload_state(U)
    assert np.array_equal(a.mass_sum(0), diag[0:4])
    assert np.array_equal(a.mass_sum(1), diag[4:8])
    assert a.sum_lz() == diag[8]
    assert np.array_equal(a.state_sum(0), diag[9:13])
    a.close()


@pytest.mark.gpu
def test_ztwd_m1m2data_matches_reference(gpu, table_path):
    """Binary::M1M2data (the L1 point, the lobes, the per-star and total
    integrals) on the reference's own final state and potential of ztwd_L2,
    with the face forces formed from that potential: the reference's values
    bit for bit."""
    g = load_golden("ztwd_L2")
    nsteps = int(g["args"][1])
    ref = g["extra"][8 + nsteps + 13:]
    assert ref.size == 28
    a = gpu.AMR(**ztwd_config(int(g["final_level"].max())))
    a.ztwd_set_frame(float(g["extra"][4]), float(g["extra"][5]), 0.0, 0.0)
    a.load_tree(g["final_level"], g["final_loc"], g["final_age"])
    bw = a.bw
    U = np.zeros((a.nbricks, a.nf, a.gnx, a.gnx, a.gnx))
    U[:, :, bw:-bw, bw:-bw, bw:-bw] = g["final_U"]
    a.upload_state(U)
    P = np.zeros((8, a.nbricks, a.pnx, a.pnx, a.pnx))
    P[0] = g["final_phi"]
    a.upload_poisson(P)
    a.compute_forces()
    d, out = a.m1m2data()
    bad = [(i, out[i], ref[i]) for i in range(28) if out[i] != ref[i]]
    assert not bad, bad
    assert d["m1"] > 0 and d["m2"] > 0 and 0.0 < d["q"] < 2.0
    a.close()


@pytest.mark.gpu
def test_ztwd_configured_size_matches_reference(gpu, table_path, tmp_path):
    """The headline configuration: the 5-level binary on the BINARY build's
    12^3 bricks, 10 BinaryDriver steps (regrids at steps 0 and 8), plain
    FP64 form.  The reference's initial state comes from a zero-step run of
    its harness (checked against the golden's sums); trees bit for bit, dt
    to 1e-12, every cell of 24 sampled bricks to 1e-12 of the field maxima,
    every brick's sums to 1e-11, the potential of the sampled bricks to
    1e-12, the flow-off."""
    from cases import check_final_sampled, check_initial_sums, live_initial_state
    g = load_golden("ztwd12_L5")
    levels, nsteps = int(g["args"][0]), int(g["args"][1])
    d0 = live_initial_state("ztwd12", ["ztwd", levels, 0], str(tmp_path), table_path)
    check_initial_sums(d0, g)
    init = {"init_level": d0.level, "init_loc": d0.loc, "init_age": d0.age, "extra": g["extra"],
            "init_U": d0.U[:, :, 3:-3, 3:-3, 3:-3], "nx": g["nx"]}
    a = make(gpu, init, table_path, max_bricks=2048)
    dts = run(a, nsteps)
    np.testing.assert_allclose(dts, g["extra"][8:8 + nsteps], rtol=DT_RTOL)
    t = a.get_tree()
    assert same_tree(t, g, "final_")
    check_final_sampled(interior(a), a.download_poisson()[0], g)
    fo = a.flow_off()
    np.testing.assert_allclose(fo, g["final_FO"], rtol=1e-10, atol=1e-13 * max(1.0, np.abs(g["final_FO"]).max()))
    a.close()


@pytest.mark.gpu
def test_persistent_forms_bitwise_on_the_headline_tree(gpu, table_path, tmp_path):
    """The persistent solve on the headline tree (5 levels of 12^3 bricks,
    309 bricks, 148 on the finest level): two BinaryDriver steps in the FP64
    form give the plain form's state and potential bit for bit in every
    block layout and blocks-per-SM cap (one block per SM: the finest level
    has as many bricks as blocks and the last block holds one; two: the
    shared-memory loops leave blocks idle), and the mixed form gives the
    same bits in each of them.  Bricks of a level reach pass 1 at different
    times here, which the smaller trees of the other tests do not show."""
    from cases import live_initial_state
    g = load_golden("ztwd12_L5")
    levels = int(g["args"][0])
    d0 = live_initial_state("ztwd12", ["ztwd", levels, 0], str(tmp_path), table_path)
    init = {"init_level": d0.level, "init_loc": d0.loc, "init_age": d0.age, "extra": g["extra"],
            "init_U": d0.U[:, :, 3:-3, 3:-3, 3:-3], "nx": g["nx"]}

    def final(prec, pers, layout=None):
        a = make(gpu, init, table_path, max_bricks=2048, precision=prec, persistent_solve=pers)
        if layout is not None:
            a.set_solve_layout(*layout)
        run(a, 2)
        out = (interior(a), a.download_poisson()[0])
        a.close()
        return out

    U0, phi0 = final(gpu.PREC_FP64, 0)
    mixed = None
    for layout in ((0, 1), (0, 2), (1, 1), (2, 2)):
        U, phi = final(gpu.PREC_FP64, 2, layout)
        assert np.array_equal(U, U0) and np.array_equal(phi, phi0), layout
        m = final(gpu.PREC_MIXED, 2, layout)
        if mixed is None:
            mixed = m
        else:
            assert np.array_equal(m[0], mixed[0]) and np.array_equal(m[1], mixed[1]), layout
