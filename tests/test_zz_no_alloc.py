"""amr_poisson_boundaries_noalloc against amr_poisson_boundaries.

The no-allocation variant serves host codes that may not call cudaMalloc
once they are running (all free device memory handed to their own pool, or
a section where an allocation's implicit device synchronisation is not
allowed).  It must give the same domain-face potential as the ordinary entry
point.  Two contexts hold the same polytrope; one computes the boundary
potential the ordinary way, the other through the variant, and one V-cycle
then carries the boundary values into phi.  This is done twice in a row, the
second time on a changed density, so that a result left over in the shared
scratch from the first call would show.

The file name sorts last so that a run stopping at its first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest

from cases import FP64_FIELD_RTOL, VARIANTS, load_golden


def make(gpu):
    return gpu.AMR(max_refine_level=2, max_bricks=2048, physics=gpu.PHYSICS_EULER_GRAVITY, **VARIANTS["g05"])


def set_state(a, g, scale):
    bw = a.bw
    U = np.zeros((a.nbricks, a.nf, a.gnx, a.gnx, a.gnx))
    U[:, :, bw:-bw, bw:-bw, bw:-bw] = g["init_U"]
    U[:, 0] *= scale
    a.upload_state(U)
    a.enforce_boundaries()


@pytest.mark.gpu
def test_noalloc_boundaries_match_two_calls(gpu):
    g = load_golden("poisson_poly_L2")
    ref, var = make(gpu), make(gpu)
    fn = var.lib.amr_poisson_boundaries_noalloc
    fn.argtypes = [ctypes.c_void_p]
    fn.restype = ctypes.c_int
    for a in (ref, var):
        a.load_tree(g["init_level"], g["init_loc"], g["init_age"])
        set_state(a, g, 1.0)
    # one ordinary Poisson call sets up the context's own buffers
    assert var.lib.amr_poisson_set_source(var.ctx) == 0
    for call, scale in enumerate((1.0, 1.7)):
        if call:
            for a in (ref, var):
                set_state(a, g, scale)
        ref.poisson_boundaries()
        rc = fn(var.ctx)
        assert rc == 0, var.lib.amr_last_error(var.ctx)
        e_ref, e_var = ref.vcycle(), var.vcycle()
        p_ref, p_var = ref.download_poisson(), var.download_poisson()
        scale_ref = np.abs(p_ref[0]).max()
        assert scale_ref > 0
        assert np.abs(p_var[0] - p_ref[0]).max() <= FP64_FIELD_RTOL * scale_ref, call
        np.testing.assert_allclose(e_var, e_ref, rtol=1e-12)
    ref.close()
    var.close()


@pytest.mark.gpu
def test_noalloc_boundaries_bitwise_on_the_4_level_star(gpu, tmp_path):
    """The 4-level single star (the reference's configured size; its initial
    state from a zero-step run of the reference harness): the boundary
    points and subtree sums are many times those of the 2-level case, so the
    variant's static scratch is walked in batches of points.  The points are
    batched, not the sums of one point, so the domain-face potential -- and
    the V-cycle that carries it into phi -- must equal the ordinary entry
    point's bit for bit."""
    from cases import live_initial_state
    from test_poisson_gpu import load_state, make as make_grav
    g = load_golden("grav_poly_L4")
    ic, maxlevel, _, tol = [x for x in g["args"]]
    d0 = live_initial_state("g05", ["grav", ic, int(maxlevel), 0, float(tol)], str(tmp_path))
    b = d0.bw
    init = {"init_level": d0.level, "init_loc": d0.loc, "init_age": d0.age, "init_U": d0.U[:, :, b:-b, b:-b, b:-b]}
    ref, var = make_grav(gpu, int(maxlevel)), make_grav(gpu, int(maxlevel))
    for a in (ref, var):
        load_state(a, init)
    fn = var.lib.amr_poisson_boundaries_noalloc
    fn.argtypes = [ctypes.c_void_p]
    fn.restype = ctypes.c_int
    assert var.lib.amr_poisson_set_source(var.ctx) == 0
    ref.poisson_boundaries()
    rc = fn(var.ctx)
    assert rc == 0, var.lib.amr_last_error(var.ctx)
    e_ref, e_var = ref.vcycle(), var.vcycle()
    assert e_ref == e_var
    assert np.array_equal(ref.download_poisson()[0], var.download_poisson()[0])
    ref.close()
    var.close()
