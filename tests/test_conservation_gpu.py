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
* the self-gravitating star and the ZTWD binary: the mass (the momenta and
  energies have the gravity sources; the binary's angular momentum and
  radial momentum the rotating frame's).

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


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ztwd_L3", "ztwd12_L3"])
def test_ztwd_binary_conserves_mass(gpu, table_path, name):
    """Total density and the two stars' tracer densities over the binary's
    steps, across its step-8 regrid, plain FP64 and mixed persistent."""
    g = load_golden(name)
    n = int(g["args"][1])
    for kw in ({}, {"precision": gpu.PREC_MIXED, "persistent_solve": 2}):
        a = make_ztwd(gpu, g, table_path, **kw)
        state = {"last": 0.0}

        def step(s):
            dt = a.max_dt()
            if s > 0:
                dt = min(1.25 * state["last"], dt)
            state["last"] = a.ztwd_step(dt, ELL_TOLER, DYNAMIC_RANGE, s)

        worst = check_run(a, step, n, [0, 1, 2])
        assert np.all(worst <= ROUNDOFF_PER_STEP * n), (kw, worst)
        a.close()
