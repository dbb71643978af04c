"""Generate tests/golden/helm_eos.npz from the reference Helmholtz EOS.

Writes the synthetic table (3d-eulerian-amr_b200/helm_table.py) into a
temporary directory, runs the reference (oracle/_ref/helm_harness, compiled
from the unpatched helmholtz/helmeos.cpp) there on seeded points, and stores
inputs and outputs.  Re-running reproduces the file bit for bit.

Cases
  fwd     helmholtz_eos on 2048 points of the throughput workload's
          distribution (log-uniform rho in [1e-2, 1e9] g/cm^3 and T in
          [1e4, 1e9] K, abar in [12, 16], zbar = abar/2) plus 64 points at
          the edges: T at and below the 1e3 K floor, ye*rho near both ends.
  units   helmholtz_eos on 256 points in code units (solar radius, solar
          mass, hour, kelvin) after helmholtz_set_cgs_units.
  inv     helmholtz_compute_T from e on 256 points (guess within a factor
          10^0.5 of the true T) plus 16 points whose e lies below e(1e3 K).
  invs    helmholtz_compute_T from s on 64 points of positive entropy.

    python tests/golden/make_helm_golden.py
"""

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "3d-eulerian-amr_b200"))
import helm_table  # noqa: E402

EXE = os.path.join(ROOT, "oracle", "_ref", "helm_harness")
UNITS = (1.0 / 6.96e10, 1.0 / 1.989e33, 1.0 / 3600.0, 1.0)
SEED = 20261203


def run(mode, records, workdir, units=None):
    n = records.shape[0]
    fin, fout = os.path.join(workdir, "in.bin"), os.path.join(workdir, "out.bin")
    with open(fin, "wb") as f:
        np.array([n], np.int64).tofile(f)
        np.ascontiguousarray(records, np.float64).tofile(f)
    argv = [EXE, mode, fin, fout] + ([repr(u) for u in units] if units else [])
    subprocess.run(argv, cwd=workdir, check=True)
    return np.fromfile(fout).reshape(n, 6)


def points(rng, n):
    rho = 10.0 ** rng.uniform(-2.0, 9.0, n)
    T = 10.0 ** rng.uniform(4.0, 9.0, n)
    abar = rng.uniform(12.0, 16.0, n)
    return rho, T, abar, abar / 2.0


def make(workdir):
    helm_table.ensure_table(workdir)
    rng = np.random.default_rng(SEED)
    out = {}
    # forward
    rho, T, abar, zbar = points(rng, 2048)
    e_rho = np.concatenate([10.0 ** rng.uniform(-2, 9, 16), np.full(16, 2.1e-12), np.full(16, 0.9e15),
                            10.0 ** rng.uniform(-2, 9, 16)])
    e_T = np.concatenate([np.full(16, 1.0e3), np.full(16, 5.0e2), 10.0 ** rng.uniform(4, 9, 16),
                          10.0 ** rng.uniform(3, 13, 16)])
    e_abar = rng.uniform(12.0, 16.0, 64)
    e_zbar = e_abar / 2.0
    e_rho[32:48] = 0.9e15 / (e_zbar[32:48] / e_abar[32:48])  # ye*rho just below the table's 1e15
    e_rho[16:32] = 2.1e-12 / (e_zbar[16:32] / e_abar[16:32])  # ye*rho just above 1e-12
    rho, T = np.concatenate([rho, e_rho]), np.concatenate([T, e_T])
    abar, zbar = np.concatenate([abar, e_abar]), np.concatenate([zbar, e_zbar])
    fin = np.stack([rho, T, abar, zbar], 1)
    out["fwd_in"] = fin
    out["fwd_out"] = run("fwd", fin, workdir)
    # units
    cm, g, s, K = UNITS
    f_rho = g / cm ** 3
    urho, uT, uabar, uzbar = points(rng, 256)
    uin = np.stack([urho * f_rho, uT * K, uabar, uzbar], 1)
    out["units"] = np.array(UNITS)
    out["units_in"] = uin
    out["units_out"] = run("fwd", uin, workdir, UNITS)
    # inverse from e
    irho, iT, iabar, izbar = points(rng, 256)
    e_true = run("fwd", np.stack([irho, iT, iabar, izbar], 1), workdir)[:, 1]
    guess = iT * 10.0 ** rng.uniform(-0.5, 0.5, 256)
    lrho, _, labar, lzbar = points(rng, 16)
    e_floor = run("fwd", np.stack([lrho, np.full(16, 1.0e3), labar, lzbar], 1), workdir)[:, 1]
    iin = np.concatenate([np.stack([irho, e_true, iabar, izbar, guess], 1),
                          np.stack([lrho, 0.5 * e_floor, labar, lzbar, np.full(16, 1.0e5)], 1)])
    out["inv_in"] = iin
    out["inv_true_T"] = np.concatenate([iT, np.full(16, 1.0e3)])
    out["inv_out"] = run("inv", iin, workdir)
    # inverse from s, at points of positive entropy (at negative entropy the
    # relative stopping test of helmeos.cpp:476 fails and the reference aborts)
    srho, sT, sabar, szbar = points(rng, 96)
    s_true = run("fwd", np.stack([srho, sT, sabar, szbar], 1), workdir)[:, 4]
    sguess = sT * 10.0 ** rng.uniform(-0.3, 0.3, 96)
    keep = np.nonzero(s_true > 0.0)[0][:64]
    srho, sT, sabar, szbar, s_true, sguess = (a[keep] for a in (srho, sT, sabar, szbar, s_true, sguess))
    sin = np.stack([srho, s_true, sabar, szbar, sguess], 1)
    out["invs_in"] = sin
    out["invs_true_T"] = sT
    out["invs_out"] = run("invs", sin, workdir)
    return out


def main():
    with tempfile.TemporaryDirectory() as td:
        out = make(td)
    np.savez_compressed(os.path.join(HERE, "helm_eos.npz"), **out)


if __name__ == "__main__":
    main()
