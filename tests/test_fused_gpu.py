"""The fused persistent hydro substep against the one-launch-per-step substep.

amr_fused_sub_step computes ghost cells where they are needed, fluxes,
coarse-fine corrections and the RK combination brick by brick in one
persistent launch, finest level first; in the FP64 form every interior value
and the flow-off accumulator must equal those of amr_sub_step bit for bit.
Cases: the bump on three levels in the unit cube (outflow faces) and in the
z-mirrored domain (reflecting face), a full RK3 step with restriction
between substeps, and a block-count cap (work spread over fewer blocks).
The mixed form (FP32 fluxes) is held to single-precision agreement.
"""

import numpy as np
import pytest

from cases import VARIANTS, load_golden

FLUX_RTOL = 1e-5  # FP32 fluxes: per field, relative to the field's maximum


def make(gpu, variant, maxlevel, **kw):
    return gpu.AMR(max_refine_level=maxlevel, max_bricks=2048, **VARIANTS[variant], **kw)


def load_state(a, g):
    a.load_tree(g["init_level"], g["init_loc"], g["init_age"])
    bw = a.bw
    U = np.zeros((a.nbricks, a.nf, a.gnx, a.gnx, a.gnx))
    U[:, :, bw:-bw, bw:-bw, bw:-bw] = g["init_U"]
    a.upload_state(U)
    a.enforce_boundaries()


def rk3(a, dt, fused, blocks_per_sm=0):
    a.store()
    for beta in (1.0, 0.25, 2.0 / 3.0):
        if fused:
            a.fused_sub_step(dt, beta, blocks_per_sm)
        else:
            a.sub_step(dt, beta)
        a.inject_from_children()
    a.enforce_boundaries()


def interior(a):
    b = a.bw
    return a.download_state()[:, :, b:-b, b:-b, b:-b]


@pytest.mark.gpu
@pytest.mark.parametrize("case,variant", [("hydro_bump_L2", "g05"), ("hydro_bump_zr_L3", "zr")])
@pytest.mark.parametrize("blocks_per_sm", [0, 1])
def test_fused_rk3_step_is_bitwise_plain(gpu, case, variant, blocks_per_sm):
    g = load_golden(case)
    maxl = int(g["init_level"].max())
    a, b = make(gpu, variant, maxl), make(gpu, variant, maxl)
    load_state(a, g)
    load_state(b, g)
    for _ in range(2):
        dt = a.max_dt()
        assert b.max_dt() == dt
        rk3(a, dt, False)
        rk3(b, dt, True, blocks_per_sm)
        assert np.array_equal(interior(a), interior(b))
        assert np.array_equal(a.flow_off(), b.flow_off())
    a.close()
    b.close()


@pytest.mark.gpu
def test_fused_mixed_close_to_fp64(gpu):
    g = load_golden("hydro_bump_zr_L3")
    maxl = int(g["init_level"].max())
    a, b = make(gpu, "zr", maxl), make(gpu, "zr", maxl, precision=gpu.PREC_MIXED)
    load_state(a, g)
    load_state(b, g)
    dt = a.max_dt()
    rk3(a, dt, False)
    rk3(b, dt, True)
    u64, u32 = interior(a), interior(b)
    for f in range(u64.shape[1]):
        scale = np.abs(u64[:, f]).max()
        if scale > 0:
            assert np.abs(u32[:, f] - u64[:, f]).max() <= FLUX_RTOL * scale, f
    a.close()
    b.close()


@pytest.mark.gpu
def test_fused_rejects_ppm(gpu):
    """The fused substep is written for the minmod brick (bw 2); a PPM
    context gets AMR_ERR_ARG instead of a wrong answer."""
    g = load_golden("hydro_ppm_bump_L2")
    a = make(gpu, "ppm", int(g["init_level"].max()))
    load_state(a, g)
    a.store()
    with pytest.raises(gpu.AmrError) as e:
        a.fused_sub_step(a.max_dt(), 1.0, 0)
    assert e.value.code == -1
    a.close()


@pytest.mark.gpu
def test_fused_wait_limit_times_out_and_context_recovers(gpu):
    """A wait limit of one poll makes a coarse brick's wait for a finer
    neighbour's published faces run out (no block is made to fault or hang;
    the whole three-level tree is resident at once, so coarse bricks meet
    children still in flight): the substep returns AMR_ERR_TIMEOUT, and with
    the default limit back the same context steps bit for bit like the plain
    substep."""
    g = load_golden("hydro_bump_zr_L3")
    maxl = int(g["init_level"].max())
    a, b = make(gpu, "zr", maxl), make(gpu, "zr", maxl)
    load_state(a, g)
    dt = a.max_dt()
    b.set_wait_limit(1)
    timed_out = False
    for _ in range(5):
        load_state(b, g)
        b.store()
        try:
            b.fused_sub_step(dt, 1.0, 0)
        except gpu.AmrError as e:
            assert e.code == -5  # AMR_ERR_TIMEOUT
            timed_out = True
            break
    assert timed_out
    b.set_wait_limit(0)
    load_state(b, g)
    b.set_flow_off(np.zeros(b.nf))  # the failed substep's flow-off went in
    rk3(a, dt, False)
    rk3(b, dt, True)
    assert np.array_equal(interior(a), interior(b))
    assert np.array_equal(a.flow_off(), b.flow_off())
    a.close()
    b.close()
