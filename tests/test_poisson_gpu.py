"""Multigrid Poisson and self-gravitating step parity vs the reference.

poisson_poly_*: the reference's Poisson::vcycle (poisson/poisson.cpp:1069)
run on a polytrope after compute_source_sums / compute_physical_boundaries /
compute_forces; potential and L1 error after every V-cycle.
grav_poly_L2: RK3 steps of the binary/single driver sequence on the Euler
state with the restated gravity coupling (oracle/harness/amr_harness.cpp).
"""

import importlib.util
import os

import numpy as np
import pytest

from cases import FP64_FIELD_RTOL, DT_RTOL, VARIANTS, field_rel_err, load_golden, same_tree
from conftest import PKG

spec = importlib.util.spec_from_file_location("amr_initial", os.path.join(PKG, "initial.py"))
initial = importlib.util.module_from_spec(spec)
spec.loader.exec_module(initial)


def make(gpu, maxlevel, variant="g05"):
    return gpu.AMR(max_refine_level=maxlevel, max_bricks=2048, physics=gpu.PHYSICS_EULER_GRAVITY,
                   **VARIANTS[variant])


def load_state(a, g, prefix="init_"):
    a.load_tree(g[prefix + "level"], g[prefix + "loc"], g[prefix + "age"])
    bw = a.bw
    U = np.zeros((a.nbricks, a.nf, a.gnx, a.gnx, a.gnx))
    U[:, :, bw:-bw, bw:-bw, bw:-bw] = g[prefix + "U"]
    a.upload_state(U)
    a.enforce_boundaries()


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.gpu
def test_vcycles_match_reference(gpu):
    g = load_golden("poisson_poly_L2")
    a = make(gpu, 2)
    load_state(a, g)
    a.poisson_boundaries()
    a.compute_forces()
    errs = g["extra"]
    for c in range(len(errs)):
        e = a.vcycle()
        np.testing.assert_allclose(e, errs[c], rtol=1e-12)
        phi = a.download_poisson()[0]
        assert rel(phi, g["cycle%d_phi" % c]) <= FP64_FIELD_RTOL, c
    a.close()


@pytest.mark.gpu
def test_vcycles_match_reference_L3(gpu):
    """137 bricks, four levels of coarse-fine interfaces; initial data from
    the host initializer (the tree must still match bit for bit); the L1
    error and every cell of the potential after each V-cycle."""
    g = load_golden("poisson_poly_L3")
    a = make(gpu, 3)
    initial.build_tree(a, "polytrope", 1.0e-6, 0.5, 0, 3, device=True)
    assert same_tree(a.get_tree(), g, "init_")
    a.poisson_boundaries()
    a.compute_forces()
    errs = g["extra"]
    for c in range(len(errs)):
        e = a.vcycle()
        np.testing.assert_allclose(e, errs[c], rtol=1e-12)
        phi = a.download_poisson()[0]
        assert rel(phi[:, 1:-1, 1:-1, 1:-1], g["cycle%d_phi" % c][:, 1:-1, 1:-1, 1:-1]) <= FP64_FIELD_RTOL, c
    a.close()


@pytest.mark.gpu
def test_poisson_solve_converges_and_restricts(gpu):
    g = load_golden("poisson_poly_L2")
    a = make(gpu, 2)
    load_state(a, g)
    err, cycles = a.poisson_solve(1.0e-8)
    assert err <= 1.0e-8 and cycles > 4
    with pytest.raises(gpu.AmrError) as ei:
        a.poisson_solve(1.0e-30, max_cycles=2)
    assert ei.value.code == -4  # AMR_ERR_NOCONVERGE instead of the reference's abort()
    a.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["grav_poly_L2", "grav_ppm_poly_L2"])
def test_grav_steps_match_reference(gpu, name):
    """grav_ppm_poly_L2: the same run with PPM reconstruction and BW 3 (the
    Poisson frame then sits two cells inside the hydro brick)."""
    g = load_golden(name)
    ic, maxlevel, nsteps, tol = [x for x in g["args"]]
    maxlevel, nsteps, tol = int(maxlevel), int(nsteps), float(tol)
    a = make(gpu, maxlevel, str(g["variant"]))
    load_state(a, g)
    dts = []
    last = 0.0
    for s in range(nsteps):
        dt = a.max_dt()
        if s > 0:
            dt = min(1.25 * last, dt)
        last = dt
        dts.append(dt)
        a.grav_step(dt, tol, 1.0e6, s)
    ex = g["extra"]
    n = int(ex[0])
    np.testing.assert_allclose(dts, ex[1:1 + n], rtol=DT_RTOL)
    t = a.get_tree()
    assert same_tree(t, g, "final_")
    bw = a.bw
    U = a.download_state()[:, :, bw:-bw, bw:-bw, bw:-bw]
    err = field_rel_err(U, g["final_U"])
    assert np.all(err <= FP64_FIELD_RTOL), err
    phi = a.download_poisson()[0]
    assert rel(phi[:, 1:-1, 1:-1, 1:-1], g["final_phi"][:, 1:-1, 1:-1, 1:-1]) <= FP64_FIELD_RTOL
    np.testing.assert_allclose(a.flow_off(), g["final_FO"], rtol=1e-11,
                               atol=1e-14 * max(1.0, np.abs(g["final_FO"]).max()))
    a.close()


@pytest.mark.gpu
def test_grav_configured_size_matches_reference(gpu, tmp_path):
    """The single star at its configured size: the 4-level n=1.5 polytrope,
    9 coupled steps of the driver sequence (the first solve from phi = 0,
    regrids with their tol/10 solves at steps 0 and 8), plain FP64 form.  The
    reference's initial state comes from a zero-step run of its harness
    (checked against the golden's sums); trees bit for bit, dt to 1e-13,
    every cell of 24 sampled bricks to 1e-12 of the field maxima, every
    brick's sums to 1e-11, the sampled potential to 1e-12, the flow-off."""
    from cases import check_final_sampled, check_initial_sums, live_initial_state
    g = load_golden("grav_poly_L4")
    ic, maxlevel, nsteps, tol = [x for x in g["args"]]
    maxlevel, nsteps, tol = int(maxlevel), int(nsteps), float(tol)
    d0 = live_initial_state("g05", ["grav", ic, maxlevel, 0, tol], str(tmp_path))
    check_initial_sums(d0, g)
    a = make(gpu, maxlevel)
    b = d0.bw
    load_state(a, {"init_level": d0.level, "init_loc": d0.loc, "init_age": d0.age,
                   "init_U": d0.U[:, :, b:-b, b:-b, b:-b]})
    dts, last = [], 0.0
    for s in range(nsteps):
        dt = a.max_dt()
        if s > 0:
            dt = min(1.25 * last, dt)
        last = dt
        dts.append(dt)
        a.grav_step(dt, tol, 1.0e6, s)
    n = int(g["extra"][0])
    np.testing.assert_allclose(dts, g["extra"][1:1 + n], rtol=DT_RTOL)
    assert same_tree(a.get_tree(), g, "final_")
    U = a.download_state()[:, :, b:-b, b:-b, b:-b]
    check_final_sampled(U, a.download_poisson()[0], g)
    np.testing.assert_allclose(a.flow_off(), g["final_FO"], rtol=1e-11,
                               atol=1e-14 * max(1.0, np.abs(g["final_FO"]).max()))
    a.close()
