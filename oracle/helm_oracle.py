"""CPU restatement of the reference Helmholtz EOS (numpy, vectorised).

Test infrastructure only: the checker for the CUDA EOS kernels, never part
of the product path.  Each function follows helmholtz/helmeos.cpp of the
reference (line numbers cited below) operation by operation; it is pinned
against the reference itself (oracle/_ref/helm_harness, built from the
unpatched helmeos.cpp) on the synthetic table that
3d-eulerian-amr_b200/helm_table.py writes (the reference's real
helmholtz.table is not shipped with it).
"""

import ctypes
import ctypes.util

import numpy as np

IMAX, JMAX = 1081, 401
TMIN, TMAX = 1.0e3, 1.0e13

# physical constants of helmholtz/const.h
PI = 3.1415926535897932384e0
H_PLANCK = 6.6260689633e-27
AVO = 6.0221417930e23
KERG = 1.380650424e-16
AMU = 1.66053878283e-24


def _libm_pow(x, y):
    return _LIBM.pow(x, y)


_LIBM = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_LIBM.pow.restype = ctypes.c_double
_LIBM.pow.argtypes = [ctypes.c_double, ctypes.c_double]


class Table:
    """helmeos.cpp:73-130: node values and the per-interval deltas."""

    def __init__(self, path):
        raw = np.fromfile(path, sep=" ")
        assert raw.size == IMAX * JMAX * 9, raw.size
        v = raw.reshape(JMAX, IMAX, 9)  # j outer, i inner
        self.f = np.ascontiguousarray(v.transpose(2, 1, 0))  # [9][IMAX][JMAX]
        self.tlo, thi = 3.0, 13.0
        self.tstp = (thi - self.tlo) / float(JMAX - 1)
        self.tstpi = 1.0 / self.tstp
        self.dlo, dhi = -12.0, 15.0
        self.dstp = (dhi - self.dlo) / float(IMAX - 1)
        self.dstpi = 1.0 / self.dstp
        # node positions through the C library's pow, as the reference computes
        # them (numpy's vectorised pow can differ in the last bit, and the
        # interpolated derivatives are sensitive to that)
        self.t = np.array([_libm_pow(10.0, self.tlo + j * self.tstp) for j in range(JMAX)])
        self.d = np.array([_libm_pow(10.0, self.dlo + i * self.dstp) for i in range(IMAX)])
        dth = self.t[1:] - self.t[:-1]
        self.dt_sav, self.dt2_sav = dth, dth * dth
        self.dti_sav = 1.0 / dth
        self.dt2i_sav = 1.0 / (dth * dth)
        dd = self.d[1:] - self.d[:-1]
        self.dd_sav, self.dd2_sav = dd, dd * dd
        self.ddi_sav = 1.0 / dd
        self.dd2i_sav = 1.0 / (dd * dd)


def _psi(z):
    psi0 = z * z * z * (z * (-6.0 * z + 15.0) - 10.0) + 1.0
    dpsi0 = z * z * (z * (-30.0 * z + 60.0) - 30.0)
    ddpsi0 = z * (z * (-120.0 * z + 180.0) - 60.0)
    psi1 = z * (z * z * (z * (-3.0 * z + 8.0) - 6.0) + 1.0)
    dpsi1 = z * z * (z * (-15.0 * z + 32.0) - 18.0) + 1.0
    ddpsi1 = z * (z * (-60.0 * z + 96.0) - 36.0)
    psi2 = 0.5 * z * z * (z * (z * (-z + 3.0) - 3.0) + 1.0)
    dpsi2 = 0.5 * z * (z * (z * (-5.0 * z + 12.0) - 9.0) + 2.0)
    ddpsi2 = 0.5 * (z * (z * (-20.0 * z + 36.0) - 18.0) + 2.0)
    return psi0, dpsi0, ddpsi0, psi1, dpsi1, ddpsi1, psi2, dpsi2, ddpsi2


def _h5(fi, w0t, w1t, w2t, w0mt, w1mt, w2mt, w0d, w1d, w2d, w0md, w1md, w2md):
    # the 36-term biquintic sum of helmeos.cpp:20-37, left to right
    terms = [
        (0, w0d, w0t), (1, w0md, w0t), (2, w0d, w0mt), (3, w0md, w0mt),
        (4, w0d, w1t), (5, w0md, w1t), (6, w0d, w1mt), (7, w0md, w1mt),
        (8, w0d, w2t), (9, w0md, w2t), (10, w0d, w2mt), (11, w0md, w2mt),
        (12, w1d, w0t), (13, w1md, w0t), (14, w1d, w0mt), (15, w1md, w0mt),
        (16, w2d, w0t), (17, w2md, w0t), (18, w2d, w0mt), (19, w2md, w0mt),
        (20, w1d, w1t), (21, w1md, w1t), (22, w1d, w1mt), (23, w1md, w1mt),
        (24, w2d, w1t), (25, w2md, w1t), (26, w2d, w1mt), (27, w2md, w1mt),
        (28, w1d, w2t), (29, w1md, w2t), (30, w1d, w2mt), (31, w1md, w2mt),
        (32, w2d, w2t), (33, w2md, w2t), (34, w2d, w2mt), (35, w2md, w2mt),
    ]
    acc = None
    for k, a, b in terms:
        v = fi[k] * a * b
        acc = v if acc is None else acc + v
    return acc


class Units:
    """helmholtz_set_cgs_units (helmeos.cpp:142-151): factors code <- cgs."""

    def __init__(self, cm=1.0, g=1.0, s=1.0, K=1.0):
        self.cm, self.g, self.s, self.K = cm, g, s, K
        self.erg = g * cm * cm / s / s
        self.dyne = g * cm / s / s
        self.f_p = self.dyne / cm ** 2
        self.f_e = self.erg / g
        self.f_T = K
        self.f_cs = cm / s
        self.f_cv = self.erg / g / K
        self.f_rho = g / cm ** 3
        self.f_s = self.erg / K / g
        self.f_dsdt = self.erg / K / K / g


def eos(tab, rho, T, abar, zbar, units=None):
    """helmholtz_eos (helmeos.cpp:164-421) on arrays (code units in and out).

    Returns dict p, e, cs, cv, s, dsdt, rho, T (rho, T after the code->cgs->code
    round trip the reference applies to them) and status (0 ok, 1 out of the
    table, 2 cv < 0, 3 cs^2 < 0: the reference aborts on 1-3).
    """
    u = units or Units()
    rho = np.asarray(rho, np.float64) * u.f_rho
    Tin = np.asarray(T, np.float64) * u.f_T
    abar = np.asarray(abar, np.float64)
    zbar = np.asarray(zbar, np.float64)
    den = rho
    temp = np.maximum(Tin, TMIN)
    ytot1 = 1.0 / abar
    ye = np.maximum(1.0 - 16, ytot1 * zbar)  # the reference writes 1.0d - 16
    deni = 1.0 / den
    kt = KERG * temp
    xni = AVO * ytot1 * den
    dxnidd = AVO * ytot1
    pion = xni * kt
    dpiondd = dxnidd * kt
    dpiondt = xni * KERG
    eion = 1.5 * pion * deni
    deiondt = 1.5 * dpiondt * deni
    x = abar * abar * np.sqrt(abar) * deni / AVO
    s = ((2.0 * PI * AMU * KERG) / (H_PLANCK * H_PLANCK)) * temp
    z = x * s * np.sqrt(s)
    y = np.log(z)
    tempi = 1.0 / temp
    sion = (pion * deni + eion) * tempi + KERG * AVO * ytot1 * y
    dsiondt = (dpiondt * deni + deiondt) * tempi - (pion * deni + eion) * tempi * tempi \
        + 1.5 * KERG * AVO * tempi * ytot1
    din = ye * den
    status = np.zeros(np.shape(den), np.int32)
    bad = (temp > tab.t[JMAX - 1]) | (temp < tab.t[0]) | (din > tab.d[IMAX - 1]) | (din < tab.d[0])
    status[bad] = 1
    with np.errstate(all="ignore"):
        jat = ((np.log10(temp) - tab.tlo) * tab.tstpi).astype(np.int64) + 1
        jat = np.maximum(1, np.minimum(jat, JMAX - 1)) - 1
        iat = ((np.log10(np.where(bad, 1.0, din)) - tab.dlo) * tab.dstpi).astype(np.int64) + 1
        iat = np.maximum(1, np.minimum(iat, IMAX - 1)) - 1
    F = tab.f  # [9][IMAX][JMAX]: f fd ft fdd ftt fdt fddt fdtt fddtt
    order = [0, 2, 4, 1, 3, 5, 6, 7, 8]  # fi blocks: f ft ftt fd fdd fdt fddt fdtt fddtt
    fi = []
    for q in order:
        fi += [F[q][iat, jat], F[q][iat + 1, jat], F[q][iat, jat + 1], F[q][iat + 1, jat + 1]]
    xt = np.maximum((temp - tab.t[jat]) * tab.dti_sav[jat], 0.0)
    xd = np.maximum((din - tab.d[iat]) * tab.ddi_sav[iat], 0.0)
    mxt = 1.0 - xt
    mxd = 1.0 - xd
    dt, dt2, dti, dt2i = tab.dt_sav[jat], tab.dt2_sav[jat], tab.dti_sav[jat], tab.dt2i_sav[jat]
    dd, dd2, ddi, dd2i = tab.dd_sav[iat], tab.dd2_sav[iat], tab.ddi_sav[iat], tab.dd2i_sav[iat]
    p0t, dp0t, ddp0t, p1t, dp1t, ddp1t, p2t, dp2t, ddp2t = _psi(xt)
    p0mt, dp0mt, ddp0mt, p1mt, dp1mt, ddp1mt, p2mt, dp2mt, ddp2mt = _psi(mxt)
    p0d, dp0d, ddp0d, p1d, dp1d, ddp1d, p2d, dp2d, ddp2d = _psi(xd)
    p0md, dp0md, ddp0md, p1md, dp1md, ddp1md, p2md, dp2md, ddp2md = _psi(mxd)
    si0t, si1t, si2t = p0t, p1t * dt, p2t * dt2
    si0mt, si1mt, si2mt = p0mt, -p1mt * dt, p2mt * dt2
    si0d, si1d, si2d = p0d, p1d * dd, p2d * dd2
    si0md, si1md, si2md = p0md, -p1md * dd, p2md * dd2
    dsi0t, dsi1t, dsi2t = dp0t * dti, dp1t, dp2t * dt
    dsi0mt, dsi1mt, dsi2mt = -dp0mt * dti, dp1mt, -dp2mt * dt
    dsi0d, dsi1d, dsi2d = dp0d * ddi, dp1d, dp2d * dd
    dsi0md, dsi1md, dsi2md = -dp0md * ddi, dp1md, -dp2md * dd
    ddsi0t, ddsi1t, ddsi2t = ddp0t * dt2i, ddp1t * dti, ddp2t
    ddsi0mt, ddsi1mt, ddsi2mt = ddp0mt * dt2i, -ddp1mt * dti, ddp2mt
    ddsi0d, ddsi1d, ddsi2d = ddp0d * dd2i, ddp1d * ddi, ddp2d
    ddsi0md, ddsi1md, ddsi2md = ddp0md * dd2i, -ddp1md * ddi, ddp2md
    T_ = (si0t, si1t, si2t, si0mt, si1mt, si2mt)
    dT_ = (dsi0t, dsi1t, dsi2t, dsi0mt, dsi1mt, dsi2mt)
    ddT_ = (ddsi0t, ddsi1t, ddsi2t, ddsi0mt, ddsi1mt, ddsi2mt)
    D_ = (si0d, si1d, si2d, si0md, si1md, si2md)
    dD_ = (dsi0d, dsi1d, dsi2d, dsi0md, dsi1md, dsi2md)
    ddD_ = (ddsi0d, ddsi1d, ddsi2d, ddsi0md, ddsi1md, ddsi2md)
    free = _h5(fi, *T_, *D_)
    df_d = _h5(fi, *T_, *dD_)
    df_t = _h5(fi, *dT_, *D_)
    df_dd = _h5(fi, *T_, *ddD_)
    df_tt = _h5(fi, *ddT_, *D_)
    df_dt = _h5(fi, *dT_, *dD_)
    x = din * din
    pele = x * df_d
    dpepdd = ye * (x * df_dd + 2.0 * din * df_d)
    dpepdt = x * df_dt
    sele = -df_t * ye
    dsepdt = -df_tt * ye
    eele = ye * free + temp * sele
    deepdt = temp * dsepdt
    p = pele + pion
    e = eele + eion
    s_out = sele + sion
    dsdt = dsiondt + dsepdt
    cv = deiondt + deepdt
    dpgasdd = dpiondd + dpepdd
    dpgasdt = dpiondt + dpepdt
    with np.errstate(all="ignore"):
        x = (p * deni * deni) * (dpgasdt / cv) + dpgasdd
        status[(status == 0) & (cv < 0.0)] = 2
        status[(status == 0) & (x < 0.0)] = 3
        cs = np.sqrt(np.maximum(x, 0.0))
    return {
        "p": p / u.f_p, "e": e / u.f_e, "cs": cs / u.f_cs, "cv": cv / u.f_cv, "s": s_out / u.f_s,
        "dsdt": dsdt / u.f_dsdt, "rho": rho / u.f_rho, "T": Tin / u.f_T, "status": status,
    }


def invert_T(tab, rho, e0, abar, zbar, T_guess, units=None, from_entropy=False):
    """helmholtz_compute_T (helmeos.cpp:436-486), point by point.

    Returns dict T, p, e, cs, cv, s, iters, status (4: no convergence in 100
    iterations, 5: T fell below TMIN; the reference aborts on both).
    """
    rho = np.atleast_1d(np.asarray(rho, np.float64))
    n = rho.size
    e0 = np.broadcast_to(np.asarray(e0, np.float64), (n,))
    abar = np.broadcast_to(np.asarray(abar, np.float64), (n,))
    zbar = np.broadcast_to(np.asarray(zbar, np.float64), (n,))
    Tg = np.broadcast_to(np.asarray(T_guess, np.float64), (n,))
    out = {k: np.zeros(n) for k in ("T", "p", "e", "cs", "cv", "s")}
    out["iters"] = np.zeros(n, np.int32)
    out["status"] = np.zeros(n, np.int32)
    key = "s" if from_entropy else "e"
    dkey = "dsdt" if from_entropy else "cv"

    def call(r, T, q):
        res = eos(tab, np.array([r]), np.array([T]), abar[q:q + 1], zbar[q:q + 1], units)
        return {k: v[0] for k, v in res.items()}

    for q in range(n):
        r = rho[q]
        T0 = Tg[q]
        res = call(r, TMIN, q)
        r = res["rho"]
        st = int(res["status"])
        T = T0
        iters = 0
        if res[key] >= e0[q]:
            T = TMIN
        else:
            a = 1.0
            while True:
                T0 = max(T, TMIN)
                res = call(r, T, q)
                r, T = res["rho"], res["T"]
                st = st or int(res["status"])
                f = res[key] - e0[q]
                dT = -f / res[dkey]
                T = T + a * dT
                T = max(T, (T0 + TMIN) / 2.0)
                iters += 1
                if iters % 10 == 0:
                    a *= 0.9
                if T < TMIN:
                    st = st or 5
                    break
                if not (abs(f / e0[q]) >= 1.0e-9 and iters < 100):
                    break
            res = call(r, T, q)
            r, T = res["rho"], res["T"]
            st = st or int(res["status"])
            if iters >= 100:
                st = st or 4
        if T < TMIN:
            st = st or 5
        out["T"][q] = T
        for k in ("p", "e", "cs", "cv", "s"):
            out[k][q] = res[k]
        out["iters"][q] = iters
        out["status"][q] = st
    return out
