"""Conservation over whole runs, through the C ABI.

The reference tracks the total of every conserved field as
GridNode::state_sum over the uncovered cells (grid/grid_node.cpp:1489-1527)
plus the root's flow-off accumulator FO, the flux that has left through the
domain boundary (grid/grid.cpp:346-404; written out each step by
BinaryDriver::state_sums_out, binary/binary_driver.cpp:248-294).  With the
coarse-fine flux correction (grid_node.cpp:1076-1274), the restriction of
covered cells (grid_node.cpp:1035-1074) and the regrid's prolongation
(grid_node.cpp:193-233) all conservative, state_sum + FO stays constant to
round-off for every field without a source:

* the Euler blast (no gravity): mass, the three momenta and the energy;
* the self-gravitating star: the mass (the momenta and energy have the
  gravity sources).

The ZTWD binary is not conservative in the reference itself: State::floor
(binary/state_ztwd.cpp:482-554) raises the density of evacuated cells to
rho_floor, which adds mass (3.2e-9 of the total over the 9 steps of ztwd_L3,
1.4e-9 for ztwd12_L3, computed from the reference's own initial and final
states in the goldens).  There the test holds the library's drift of the
total density and of the two stars' densities to the reference's drift.

The bound is round-off: 1e-13 of the field's total absolute content
(sum |u| dV) per step.
"""

import numpy as np
import pytest

from cases import load_golden
from test_ztwd_gpu import ELL_TOLER, DYNAMIC_RANGE, make as make_ztwd

ROUNDOFF_PER_STEP = 1.0e-13


def totals(a, fields):
    """state_sum + FO of each field, and sum |u| dV as its scale."""
    fo = a.flow_off()
    out, scale = [], []
    bw = a.bw
    U = a.download_state()[:, :, bw:-bw, bw:-bw, bw:-bw]
    t = a.get_tree()
    nx = a.nx
    half = nx // 2
    idx = np.arange(nx) // half
    oc = idx[None, None, :] | (idx[None, :, None] << 1) | (idx[:, None, None] << 2)
    leaf = ((t["child_mask"][:, None, None, None] >> oc[None]) & 1) == 0
    vol = (t["h"] ** 3)[:, None, None, None] * leaf
    for f in fields:
        out.append(a.state_sum(f)[0] + fo[f])
        scale.append(float((np.abs(U[:, f]) * vol).sum()))
    return np.array(out), np.array(scale)


def check_run(a, step, nsteps, fields):
    m0, s0 = totals(a, fields)
    worst = np.zeros(len(fields))
    for s in range(nsteps):
        step(s)
        m, sc = totals(a, fields)
        worst = np.maximum(worst, np.abs(m - m0) / np.maximum(np.maximum(sc, s0), 1e-300))
    return worst


def hydro_steps(a, thr):
    state = {"last": 0.0}

    def step(s):
        dt = a.max_dt()
        if s > 0:
            dt = min(1.25 * state["last"], dt)
        state["last"] = dt
        a.hydro_step(dt, thr)
    return step


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["hydro_blast_L2", "hydro_ppm_blast_L2"])
def test_euler_blast_conserves_mass_momentum_energy(gpu, name):
    from test_hydro_gpu import load_state, make
    g = load_golden(name)
    variant = str(g["variant"])
    _, maxlevel, nsteps, thr = [x for x in g["args"]]
    a = make(gpu, variant, int(maxlevel))
    load_state(a, g["init_level"], g["init_loc"], g["init_age"], g["init_U"])
    n = int(nsteps)
    worst = check_run(a, hydro_steps(a, float(thr)), n, [0, 1, 2, 3, 4])
    assert np.all(worst <= ROUNDOFF_PER_STEP * n), worst
    a.close()


@pytest.mark.gpu
def test_self_gravitating_star_conserves_mass(gpu):
    from test_poisson_gpu import load_state, make
    g = load_golden("grav_poly_L2")
    _, maxlevel, nsteps, tol = [x for x in g["args"]]
    a = make(gpu, int(maxlevel))
    load_state(a, g)
    state = {"last": 0.0}

    def step(s):
        dt = a.max_dt()
        if s > 0:
            dt = min(1.25 * state["last"], dt)
        state["last"] = dt
        a.grav_step(dt, float(tol), 1.0e6, s)

    n = int(nsteps)
    worst = check_run(a, step, n, [0])
    assert worst[0] <= ROUNDOFF_PER_STEP * n, worst
    a.close()


def reference_drift(g, fields):
    """state_sum + FO of the reference's final state minus its initial one,
    from a golden holding both states per cell, over sum |u| dV."""
    nx = int(g["nx"])
    half = nx // 2
    idx = np.arange(nx) // half
    oc = idx[None, None, :] | (idx[None, :, None] << 1) | (idx[:, None, None] << 2)

    def tot(prefix):
        h = 2.0 * 1.0 / nx / 2.0 ** g[prefix + "level"]
        leaf = ((g[prefix + "child_mask"][:, None, None, None] >> oc[None]) & 1) == 0
        vol = (h ** 3)[:, None, None, None] * leaf
        U = g[prefix + "U"]
        return (np.array([(U[:, f] * vol).sum() for f in fields]) + g[prefix + "FO"][fields],
                np.array([(np.abs(U[:, f]) * vol).sum() for f in fields]))

    m0, s0 = tot("init_")
    m1, _ = tot("final_")
    return (m1 - m0) / s0


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ztwd_L3", "ztwd12_L3"])
def test_ztwd_binary_mass_drift_is_the_references(gpu, table_path, name):
    """Total density and the two stars' densities over the binary's steps
    (regrids at steps 0 and 8): the change of state_sum + FO equals the
    reference's own (its density floor adds mass) to round-off in the plain
    FP64 form, and to 1e-3 of it in the mixed form (FP32 fluxes stay
    conservative; only the floored cells differ)."""
    g = load_golden(name)
    n = int(g["args"][1])
    fields = [0, 1, 2]
    ref = reference_drift(g, fields)
    for kw in ({}, {"precision": gpu.PREC_MIXED, "persistent_solve": 2}):
        a = make_ztwd(gpu, g, table_path, **kw)
        m0, s0 = totals(a, fields)
        last = 0.0
        for s in range(n):
            dt = a.max_dt()
            if s > 0:
                dt = min(1.25 * last, dt)
            last = a.ztwd_step(dt, ELL_TOLER, DYNAMIC_RANGE, s)
        m1, _ = totals(a, fields)
        drift = (m1 - m0) / s0
        tol = ROUNDOFF_PER_STEP * n + (1e-3 * np.abs(ref) if kw else 0.0)
        assert np.all(np.abs(drift - ref) <= tol), (kw, drift, ref)
        a.close()
