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

from cases import FP64_FIELD_RTOL, DT_RTOL, VARIANTS, load_golden, same_tree
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
    the host initializer (the tree must still match bit for bit)."""
    g = load_golden("poisson_poly_L3")
    a = make(gpu, 3)
    initial.build_tree(a, "polytrope", 1.0e-6, 0.5, 0, 3, device=True)
    assert same_tree(a.get_tree(), g, "init_")
    a.poisson_boundaries()
    a.compute_forces()
    errs = g["extra"]
    for c in range(len(errs)):
        e = a.vcycle()
        np.testing.assert_allclose(e, errs[c], rtol=1e-9)
        phi = a.download_poisson()[0]
        s = phi[:, 1:-1, 1:-1, 1:-1].reshape(phi.shape[0], -1).sum(axis=1)
        np.testing.assert_allclose(s, g["cycle%d_phisum" % c], rtol=1e-9)
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
    s = U.reshape(U.shape[0], U.shape[1], -1).sum(axis=2)
    relerr = np.abs(s - g["final_Usum"]) / np.maximum(g["final_Uabs"], 1e-300)
    assert relerr.max() <= 1e-11, relerr.max()
    phi = a.download_poisson()[0]
    assert rel(phi[:, 1:-1, 1:-1, 1:-1], g["final_phi"][:, 1:-1, 1:-1, 1:-1]) <= 1e-11
    a.close()
