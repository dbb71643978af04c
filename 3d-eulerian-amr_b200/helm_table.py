"""Synthetic Helmholtz free-energy table in the reference's text format.

The reference EOS (helmholtz/helmeos.cpp:73-130) reads `helmholtz.table`:
JMAX=401 temperatures (log10 T from 3 to 13) outer, IMAX=1081 densities
(log10 of ye*rho from -12 to 15) inner, one line per node holding

    f  f_d  f_t  f_dd  f_tt  f_dt  f_ddt  f_dtt  f_ddtt

(the electron-positron free energy and its derivatives in density d and
temperature T).  The real table is a third-party data file that is not
shipped with the reference, so this module writes a stand-in with the same
layout from a closed-form free energy

    F(d, T) = A d^(2/3) - B T^2 d^(-2/3),

whose derivatives are exact.  It gives positive pressure, positive specific
heat and positive sound speed everywhere (the reference aborts otherwise,
helmeos.cpp:405-415): p_e = d^2 F_d = (2/3)(A d^(5/3) + B T^2 d^(1/3)),
c_v,e = -ye T F_tt = 2 ye B T d^(-2/3).  A = 1.5 x 1.0036e13 makes the cold
part the non-relativistic degenerate electron gas.

    python helm_table.py OUT_PATH
"""

import os
import sys

import numpy as np

IMAX, JMAX = 1081, 401
TLO, THI = 3.0, 13.0
DLO, DHI = -12.0, 15.0
A_COLD = 1.5 * 1.0036e13
B_THERM = 1.0e4


def grid():
    """Node densities d[i] and temperatures t[j] (helmeos.cpp:90-97)."""
    tstp = (THI - TLO) / float(JMAX - 1)
    dstp = (DHI - DLO) / float(IMAX - 1)
    t = np.power(10.0, TLO + np.arange(JMAX) * tstp)
    d = np.power(10.0, DLO + np.arange(IMAX) * dstp)
    return d, t


def free_energy(d, T, a=A_COLD, b=B_THERM):
    """F and its eight tabulated derivatives at (d, T), broadcasting."""
    d = np.asarray(d, np.float64)
    T = np.asarray(T, np.float64)
    d23 = np.cbrt(d) ** 2
    dm23 = 1.0 / d23
    dm13 = 1.0 / np.cbrt(d)
    dm43 = dm13 ** 4
    dm53 = dm23 / d
    dm83 = dm53 / d
    f = a * d23 - b * T * T * dm23
    fd = (2.0 / 3.0) * a * dm13 + (2.0 / 3.0) * b * T * T * dm53
    ft = -2.0 * b * T * dm23
    fdd = -(2.0 / 9.0) * a * dm43 - (10.0 / 9.0) * b * T * T * dm83
    ftt = -2.0 * b * dm23 + 0.0 * T
    fdt = (4.0 / 3.0) * b * T * dm53
    fddt = -(20.0 / 9.0) * b * T * dm83
    fdtt = (4.0 / 3.0) * b * dm53 + 0.0 * T
    fddtt = -(20.0 / 9.0) * b * dm83 + 0.0 * T
    return np.stack(np.broadcast_arrays(f, fd, ft, fdd, ftt, fdt, fddt, fdtt, fddtt), axis=-1)


def write_table(path):
    d, t = grid()
    vals = free_energy(d[None, :], t[:, None])  # [JMAX][IMAX][9], j outer
    rows = vals.reshape(-1, 9)
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        np.savetxt(fh, rows, fmt="%.17e")
    os.replace(tmp, path)
    return path


def ensure_table(directory):
    """Write helmholtz.table into `directory` unless it is already there."""
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, "helmholtz.table")
    if not os.path.exists(path):
        write_table(path)
    return path


if __name__ == "__main__":
    write_table(sys.argv[1] if len(sys.argv) > 1 else "helmholtz.table")
