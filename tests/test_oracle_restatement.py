"""The numpy restatement (oracle/amr_oracle.py) reproduces the reference.

Golden runs whose tree does not change over the run are replayed step by
step with the restatement from the reference's own initial state; dt and
every field must agree to 1e-12 (the restatement keeps the reference's
operation order, so in practice to the last bit or one ulp).
"""

import numpy as np
import pytest

import amr_oracle as O
from cases import FP64_FIELD_RTOL, VARIANTS, field_rel_err, load_golden, oracle_recon


@pytest.mark.parametrize("name", ["hydro_bump_L2", "hydro_bump_zr_L3", "hydro_ppm_bump_L2"])
def test_restatement_matches_reference(name):
    g = load_golden(name)
    assert np.array_equal(g["init_level"], g["final_level"]) and np.array_equal(g["init_loc"], g["final_loc"])
    v = VARIANTS[str(g["variant"])]
    recon = oracle_recon(str(g["variant"]))
    T = O.Tree(g["init_level"], g["init_loc"], bw=int(g["bw"]), grid_dim=v["grid_dim"],
               z_reflect=bool(v["z_reflect"]))
    bw, gnx = T.bw, T.gnx
    U = np.zeros((T.n, 6, gnx, gnx, gnx))
    U[:, :, bw:-bw, bw:-bw, bw:-bw] = g["init_U"]
    U = O.enforce_boundaries(T, U)
    nsteps = int(g["args"][2])
    last = 0.0
    dts = []
    for s in range(nsteps):
        dt = O.max_dt(T, U, 1.3, 5.0 / 3.0, 0.4, recon)
        if s > 0:
            dt = min(last * 1.25, dt)
        last = dt
        dts.append(dt)
        U = O.step(T, U, dt, recon=recon)
    np.testing.assert_allclose(dts, g["extra"][:nsteps], rtol=1e-14)
    err = field_rel_err(U[:, :, bw:-bw, bw:-bw, bw:-bw], g["final_U"])
    assert np.all(err <= FP64_FIELD_RTOL), err
