"""The graph-captured forms reproduce the plain forms bit for bit.

amr_graph_solve / amr_graph_grav_step run the same kernels as
amr_poisson_solve / amr_grav_step, with the loop decisions (relaxation
ratios, the L1 error test, the CFL step) taken on the device from the same
nested sums; every array must come out identical.  With persistent_solve the
V-cycle loop of each solve is one cooperative kernel whose phases are
separated by grid barriers; it too must reproduce the plain form exactly.
"""

import numpy as np
import pytest

from cases import VARIANTS, load_golden, same_tree


def make(gpu, maxlevel, persistent=0, variant="g05"):
    return gpu.AMR(max_refine_level=maxlevel, max_bricks=2048, physics=gpu.PHYSICS_EULER_GRAVITY,
                   persistent_solve=persistent, **VARIANTS[variant])


def load_state(a, g):
    a.load_tree(g["init_level"], g["init_loc"], g["init_age"])
    U = np.zeros((a.nbricks, a.nf, a.gnx, a.gnx, a.gnx))
    b = a.bw
    U[:, :, b:-b, b:-b, b:-b] = g["init_U"]
    a.upload_state(U)
    a.enforce_boundaries()


@pytest.mark.gpu
@pytest.mark.parametrize("persistent", [0, 1])
def test_graph_solve_is_bitwise_plain(gpu, persistent):
    g = load_golden("poisson_poly_L2")
    a, b = make(gpu, 2), make(gpu, 2, persistent)
    load_state(a, g)
    load_state(b, g)
    ea, na = a.poisson_solve(1.0e-7)
    eb, nb = b.graph_solve(1.0e-7)
    assert na == nb and ea == eb
    assert np.array_equal(a.download_poisson(), b.download_poisson())
    assert np.array_equal(a.download_state(), b.download_state())
    # a second solve on the same graph (replay) from the converged state
    ea, na = a.poisson_solve(1.0e-9)
    eb, nb = b.graph_solve(1.0e-9)
    assert na == nb and ea == eb
    assert np.array_equal(a.download_poisson()[0], b.download_poisson()[0])


@pytest.mark.gpu
@pytest.mark.parametrize("persistent", [1, 2])
def test_persistent_solve_bitwise_plain_on_large_levels(gpu, persistent):
    """The 4-level single star has levels of 1, 8, 64, 160 and 408 bricks.
    With 148 or 296 cooperative blocks some levels have fewer bricks than
    blocks (the relaxation loop that forms each level sum in one block while
    the bricks compute the next pass) and some have more (two bricks per
    block, level sums in every block); the solve must reproduce the plain
    form bit for bit, pass for pass."""
    import importlib.util
    import os
    from conftest import PKG
    spec = importlib.util.spec_from_file_location("amr_initial", os.path.join(PKG, "initial.py"))
    initial = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(initial)
    a, b = make(gpu, 4), make(gpu, 4, persistent)
    for x in (a, b):
        initial.build_tree(x, "polytrope", 1.0e-6, 0.5, 0, 4, device=True)
    assert [int((a.get_tree()["level"] == l).sum()) for l in range(5)] == [1, 8, 64, 160, 408]
    ea, na = a.poisson_solve(1.0e-6)
    eb, nb = b.graph_solve(1.0e-6)
    assert na == nb and ea == eb
    assert np.array_equal(a.relax_passes(), b.relax_passes())
    assert np.array_equal(a.download_poisson(), b.download_poisson())
    a.close()
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("persistent", [0, 1])
def test_graph_grav_steps_are_bitwise_plain(gpu, persistent):
    g = load_golden("grav_poly_L2")
    a, b = make(gpu, 2), make(gpu, 2, persistent)
    load_state(a, g)
    load_state(b, g)
    last = 0.0
    for s in range(int(g["args"][2]) + 6):  # through a regrid at step 8
        dt = a.max_dt()
        if s > 0:
            dt = min(1.25 * last, dt)
        last = dt
        a.grav_step(dt, 1.0e-6, 1.0e6, s)
        dtb = b.graph_grav_step(1.0e-6, 1.0e6, s)
        assert dtb == dt, (s, dt, dtb)
        ta, tb = a.get_tree(), b.get_tree()
        assert np.array_equal(ta["loc"], tb["loc"]) and np.array_equal(ta["age"], tb["age"])
    assert np.array_equal(a.download_state(), b.download_state())
    assert np.array_equal(a.download_poisson()[0], b.download_poisson()[0])
    np.testing.assert_array_equal(a.flow_off(), b.flow_off())


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["grav_poly_L2", "grav_ppm_poly_L2"])
def test_graph_steps_match_reference(gpu, name):
    """The reference's 3-step coupled run, replayed through the graph form
    (minmod with BW 2, and PPM with BW 3)."""
    g = load_golden(name)
    a = make(gpu, 2, variant=str(g["variant"]))
    load_state(a, g)
    dts = [a.graph_grav_step(1.0e-6, 1.0e6, s) for s in range(3)]
    n = int(g["extra"][0])
    np.testing.assert_allclose(dts, g["extra"][1:1 + n], rtol=1e-13)
    assert same_tree(a.get_tree(), g, "final_")
    b = a.bw
    U = a.download_state()[:, :, b:-b, b:-b, b:-b]
    s = U.reshape(U.shape[0], U.shape[1], -1).sum(axis=2)
    rel = np.abs(s - g["final_Usum"]) / np.maximum(g["final_Uabs"], 1e-300)
    assert rel.max() <= 1e-11


@pytest.mark.gpu
def test_persistent_wait_limit_times_out_and_context_recovers(gpu):
    """A wait limit of one poll makes some grid barrier or level-sum wait of
    the persistent solve run out (no block is made to fault or hang): the
    solve returns AMR_ERR_TIMEOUT, and with the default limit back the same
    context solves again, bit for bit like the plain form."""
    g = load_golden("poisson_poly_L2")
    a, b = make(gpu, 2), make(gpu, 2, 2)
    load_state(a, g)
    load_state(b, g)
    b.set_wait_limit(1)
    with pytest.raises(gpu.AmrError) as e:
        b.graph_solve(1.0e-7)
    assert e.value.code == -5  # AMR_ERR_TIMEOUT
    b.set_wait_limit(0)
    load_state(b, g)
    b.upload_poisson(np.zeros_like(b.download_poisson()))
    ea, na = a.poisson_solve(1.0e-7)
    eb, nb = b.graph_solve(1.0e-7)
    assert na == nb and ea == eb
    assert np.array_equal(a.download_poisson()[0], b.download_poisson()[0])
    a.close()
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["poisson_poly_L2", "ztwd12_L2"])
def test_solve_layouts_bitwise_and_autotuner(gpu, table_path, case):
    """Every block layout of the persistent solve kernel (threads per block,
    cells per thread, blocks per SM) gives the same potential bit for bit;
    the autotuner times them all on the context's own solve, keeps one and
    leaves the state and the Poisson arrays unchanged (a ZTWD solve also
    writes the state's potential field and restricts the state).  The
    source S is the exception: every call of the graph API recomputes it
    from the density first, and so does the autotuner's last one."""
    if case.startswith("ztwd"):
        from test_ztwd_gpu import make as make_ztwd
        g = load_golden(case)
        a = make_ztwd(gpu, g, table_path, persistent_solve=2)
        a.ztwd_pot(1)  # pot_from_grid: phi from the state
        tol = 1.0e-7
    else:
        g = load_golden(case)
        a = make(gpu, 2, 2)
        load_state(a, g)
        tol = 1.0e-7
    P0 = a.download_poisson()
    _, _, _, _, count = a.solve_layout()
    assert count >= 2
    ref = None
    for layout in range(count):
        for per_sm in (1, 0):
            a.set_solve_layout(layout, per_sm)
            a.upload_poisson(P0)
            e, n = a.graph_solve(tol)
            phi = a.download_poisson()[0]
            if ref is None:
                ref = (e, n, phi)
            else:
                assert (e, n) == ref[:2], (layout, per_sm)
                assert np.array_equal(phi, ref[2]), (layout, per_sm)
    a.upload_poisson(P0)
    U0 = a.download_state()
    ms, best = a.autotune_solve(tol, reps=1)
    assert 0 <= best < len(ms) and ms[best] is not None and ms[best] > 0
    assert all(m is None or m >= ms[best] for m in ms)
    P1 = a.download_poisson()
    for q in (0, 1, 2, 3, 5, 6, 7):  # phi, phi0, dphi, dphi1, fx, fy, fz
        assert np.array_equal(P1[q], P0[q]), q
    assert np.array_equal(a.download_state(), U0)
    lay = a.solve_layout()
    assert lay[0] == best // 3
    a.close()
