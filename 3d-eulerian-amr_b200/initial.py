"""Initial data and tree construction on the host (setup, not the hot path).

The reference builds its octree by alternating initialize() and
check_for_refine() (euler/hydro_driver.cpp:84-107); build_tree() does the
same through the library: the initial data are evaluated on the host for the
current bricks, uploaded, and the device computes the refinement flags.

Initial conditions (cell centres, FP64, Euler state d sx sy sz et tau):
  blast      rho=1, v=0, p=1e-5; total energy 1.0 spread uniformly over the
             finest-level cells with centre radius < 0.05 (unit cube)
  bump       rho = 1 + 9 exp(-|x-c|^2/0.15^2), c=(0.08,-0.05,0.06), uniform
             p=0.6, v=(0.4, 0.25, -0.15+0.1 sin 2 pi x)
  polytrope  n=1.5 Lane-Emden star, central density 1, radius 0.25, at the
             origin, 2^3 sub-samples per cell, ambient floor 1e-10
  random     seeded log-normal field: Gaussian random field with P(k)~k^-3,
             sigma 1, on a periodic 256^3 grid, trilinearly sampled;
             v ~ N(0, 0.1), p = rho^(5/3)
  binary     (ZTWD state, 13 fields) the reference's two-polytrope binary of
             binary/initialize.cpp:12-92 with q = 0.7, separation 0.5, donor
             radius 0.17 (its Roche lobe radius at this q is 0.174),
             M1 = 2.4e-3, n = 1.5, followed by State::floor (T at the table
             floor, et = 0: a zero-temperature binary) and synchronous
             rotation in the co-rotating frame (lz = rho Omega R^2)
"""

import numpy as np

GAMMA = 5.0 / 3.0
POLY_R = 0.25


def cell_centres(tree, bw, nx, grid_dim, z_reflect, ghosts=False):
    """Centres of every brick's cells, Grid::xc/yc/zc (grid/grid.cpp:500-526)."""
    gnx = nx + 2 * bw
    h0 = 2.0 * grid_dim / nx
    idx = np.arange(gnx) if ghosts else np.arange(bw, gnx - bw)
    off = tree["offset"].astype(np.float64)
    h = tree["h"][:, None]
    xs = []
    for d in range(3):
        f = (off[:, d:d + 1] + idx[None, :]) * h - grid_dim - bw * h0
        if d == 2 and z_reflect:
            f = (off[:, d:d + 1] + idx[None, :]) * h - bw * h0
        xs.append(f + 0.5 * h)
    return xs  # each (n, len(idx))


# ZTWD binary parameters (Binary statics of binary/binary.cpp:8-26, set for
# this configuration)
BINARY = dict(q=0.7, a=0.5, R2=0.17, M1=2.4e-3, n=1.5, rho_floor=1.0e-10, T_floor=1.0e3)


def binary_params():
    """Derived constants of binary/initialize.cpp:13-19 and the code units of
    Binary::set_units (binary/binary.h:17-35): K1, (cm, g, s) and Omega."""
    q, a, R2, M1, n = (BINARY[k] for k in ("q", "a", "R2", "M1", "n"))
    rho_c2 = q * M1 * (pow(3.65375 / R2, 3.0) / (2.71406 * 4.0 * np.pi))
    rho_c1 = rho_c2 / pow(q, 2.0 * n / (3.0 - n))
    K = pow(R2 / 3.65375, 2) * 4.0 * np.pi / (2.5) * pow(rho_c2, 1.0 / 3.0)
    A, B, G = 6.0023e+22, 2.0 * 9.7393e+5, 6.6745e-8
    g = pow(K, -1.5) * (pow(A / G, 1.5) / B / B)
    cm = pow(K, -0.5) * (1.0 / B * np.sqrt(A / G))
    s = 1.0 * (1.0 / np.sqrt(B * G))
    omega = np.sqrt(M1 * (q + 1.0) / (a * a * a))
    return dict(K1=K, rho_c1=rho_c1, rho_c2=rho_c2, cm=cm, g=g, s=s, omega=omega,
                R1=R2 * pow(q, 1.0 / 3.0))


def _minmod(a, b):  # real.h:63-65
    sg = np.sign(a) + np.sign(b)
    return 0.5 * sg * np.minimum(np.abs(a), np.abs(b))


def _binary_state(tree, bw, nx, grid_dim, z_reflect, ghosts):
    """binary/initialize.cpp:12-92 + State::floor + synchronous rotation."""
    P = binary_params()
    q, a, n, floor = BINARY["q"], BINARY["a"], BINARY["n"], BINARY["rho_floor"]
    gnx = nx + 2 * bw
    h0 = 2.0 * grid_dim / nx
    idx = np.arange(gnx) if ghosts else np.arange(bw, gnx - bw)
    off = tree["offset"].astype(np.float64)
    h = tree["h"][:, None]
    faces = []
    for d in range(3):  # Grid::xf/yf/zf of cells idx and idx + 1
        lo = (off[:, d:d + 1] + idx[None, :]) * h - bw * h0
        hi = (off[:, d:d + 1] + idx[None, :] + 1) * h - bw * h0
        if not (d == 2 and z_reflect):
            lo, hi = lo - grid_dim, hi - grid_dim
        faces.append((lo, hi))
    nb, m = off.shape[0], len(idx)
    rho_c1, rho_c2, K = P["rho_c1"], P["rho_c2"], P["K1"]
    E1 = np.sqrt((4.0 * np.pi * pow(rho_c1, 1.0 - 1.0 / n)) / ((n + 1.0) * K))
    E2 = np.sqrt((4.0 * np.pi * pow(rho_c2, 1.0 - 1.0 / n)) / ((n + 1.0) * K))
    x1, x2 = a * q / (q + 1.0), -a / (q + 1.0)
    (xl, xh), (yl, yh), (zl, zh) = faces
    XL = np.broadcast_to(xl[:, None, None, :], (nb, m, m, m))
    XH = np.broadcast_to(xh[:, None, None, :], (nb, m, m, m))
    YL = np.broadcast_to(yl[:, None, :, None], (nb, m, m, m))
    YH = np.broadcast_to(yh[:, None, :, None], (nb, m, m, m))
    ZL = np.broadcast_to(zl[:, :, None, None], (nb, m, m, m))
    ZH = np.broadcast_to(zh[:, :, None, None], (nb, m, m, m))
    y = _minmod(YL, YH)
    z = _minmod(ZL, ZH)
    xa = _minmod(XL - x1, XH - x1)
    xb = _minmod(XL - x2, XH - x2)
    near = (np.sqrt(xa * xa + y * y + z * z) * E1 < 3.7) | (np.sqrt(xb * xb + y * y + z * z) * E2 < 3.7)
    finest = tree["child_mask"] == 0
    M0 = np.where(finest, (tree["h"] / P["R1"] + 2.0).astype(np.int64), 2)
    rho1 = np.zeros((nb, m, m, m))
    rho2 = np.zeros((nb, m, m, m))
    hb = tree["h"][:, None, None, None]
    for M in np.unique(M0):
        sel = (M0 == M)[:, None, None, None] & near
        for k0 in range(M):
            zz = ZL + (k0 + 0.5) * hb / M
            for j0 in range(M):
                yy = YL + (j0 + 0.5) * hb / M
                for i0 in range(M):
                    xx = XL + (i0 + 0.5) * hb / M
                    r1 = np.sqrt((xx - x1) * (xx - x1) + yy * yy + zz * zz) * E1
                    r2 = np.sqrt((xx - x2) * (xx - x2) + yy * yy + zz * zz) * E2
                    t1 = np.where(sel & (r1 < 3.7), lane_emden(np.where(r1 < 3.7, r1, 0.0)) ** n / M ** 3 * rho_c1, 0.0)
                    t2 = np.where(sel & (r2 < 3.7), lane_emden(np.where(r2 < 3.7, r2, 0.0)) ** n / M ** 3 * rho_c2, 0.0)
                    rho1 = rho1 + t1
                    rho2 = rho2 + t2
    rho1 = np.maximum(rho1, floor / 2.0)
    rho2 = np.maximum(rho2, floor / 2.0)
    rho = rho1 + rho2
    U = np.zeros((nb, 13, m, m, m))
    U[:, 0], U[:, 1], U[:, 2] = rho, rho1, rho2
    U[:, 9] = BINARY["T_floor"]  # Newton from e = 0 stops at the table floor
    U[:, 10] = rho               # all species zero -> species 0 (state_ztwd.cpp:520-526)
    XC = XL + 0.5 * hb
    YC = YL + 0.5 * hb
    U[:, 4] = rho * P["omega"] * (XC * XC + YC * YC)
    return U


def _lane_emden_table(dr=0.05, rmax=3.7):
    """Full RK4 steps of binary/lane_emden.cpp:17-77 from the centre."""
    ys, zs, rs = [1.0], [0.0], [0.0]
    y, z, r = 1.0, 0.0, 0.0
    while r + dr <= rmax + dr:
        y0, z0 = y, z
        f = lambda yy, zz, rr: -((max(yy, 0.0)) ** 1.5 + 2.0 * zz / rr) if rr != 0.0 else -3.0
        dy1, dz1 = z * dr, f(y, z, r) * dr
        y, zz = y0 + 0.5 * dy1, z0 + 0.5 * dz1
        dy2, dz2 = zz * dr, f(y, zz, r + 0.5 * dr) * dr
        y, zz = y0 + 0.5 * dy2, z0 + 0.5 * dz2
        dy3, dz3 = zz * dr, f(y, zz, r + 0.5 * dr) * dr
        y, zz = y0 + dy3, z0 + dz3
        dy4, dz4 = zz * dr, f(y, zz, r + dr) * dr
        y = y0 + (dy1 + dy4 + 2.0 * (dy3 + dy2)) / 6.0
        z = z0 + (dz1 + dz4 + 2.0 * (dz3 + dz2)) / 6.0
        r += dr
        ys.append(y)
        zs.append(z)
        rs.append(r)
        if y <= 0.0:
            break
    return np.array(ys), np.array(zs), np.array(rs)


_LE = None


def lane_emden(r0):
    """theta(xi) of the n=1.5 Lane-Emden equation, vectorised: full 0.05
    steps from a table, then one partial RK4 step to r0 (lane_emden.cpp)."""
    global _LE
    if _LE is None:
        _LE = _lane_emden_table()
    Y, Z, R = _LE
    r0 = np.asarray(r0, np.float64)
    m = np.searchsorted(R + 0.05, r0, side="right")  # first m with R[m]+dr > r0
    m = np.clip(m, 0, len(R) - 1)
    y, z, r = Y[m], Z[m], R[m]
    dr = r0 - r

    def fz(yy, zz, rr):
        with np.errstate(divide="ignore", invalid="ignore"):
            out = -(np.maximum(yy, 0.0) ** 1.5 + 2.0 * zz / rr)
        return np.where(rr != 0.0, out, -3.0)

    dy1, dz1 = z * dr, fz(y, z, r) * dr
    y1, z1 = y + 0.5 * dy1, z + 0.5 * dz1
    dy2, dz2 = z1 * dr, fz(y1, z1, r + 0.5 * dr) * dr
    y2, z2 = y + 0.5 * dy2, z + 0.5 * dz2
    dy3, dz3 = z2 * dr, fz(y2, z2, r + 0.5 * dr) * dr
    y3, z3 = y + dy3, z + dz3
    dy4 = z3 * dr
    yf = y + (dy1 + dy4 + 2.0 * (dy3 + dy2)) / 6.0
    return np.maximum(yf, 0.0)


def poly_K():
    return (POLY_R / 3.65375) ** 2 * 4.0 * np.pi / 2.5


def _state(rho, vx, vy, vz, ei):
    return np.stack([rho, rho * vx, rho * vy, rho * vz, ei + 0.5 * rho * (vx * vx + vy * vy + vz * vz),
                     ei ** (1.0 / GAMMA)], axis=1)


_GRF = {}


def random_field(seed=20261203, n=256, slope=-3.0, sigma=1.0):
    key = (seed, n, slope, sigma)
    if key not in _GRF:
        rng = np.random.default_rng(seed)
        k = np.fft.fftfreq(n) * n
        kx, ky, kz = np.meshgrid(k, k, np.fft.rfftfreq(n) * n, indexing="ij")
        kk = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
        amp = np.zeros_like(kk)
        amp[kk > 0] = kk[kk > 0] ** (slope / 2.0)
        noise = rng.standard_normal((n, n, n // 2 + 1)) + 1j * rng.standard_normal((n, n, n // 2 + 1))
        f = np.fft.irfftn(noise * amp, s=(n, n, n))
        f = (f - f.mean()) / f.std() * sigma
        _GRF[key] = np.exp(f)
    return _GRF[key]


def evaluate(ic, tree, bw, nx, grid_dim, z_reflect, max_level, ghosts=True, seed=20261203):
    """Conserved state [n, 6, g, g, g] of every brick (g = gnx with ghosts)."""
    xs = cell_centres(tree, bw, nx, grid_dim, z_reflect, ghosts=ghosts)
    n, m = xs[0].shape
    X = np.broadcast_to(xs[0][:, None, None, :], (n, m, m, m))
    Y = np.broadcast_to(xs[1][:, None, :, None], (n, m, m, m))
    Z = np.broadcast_to(xs[2][:, :, None, None], (n, m, m, m))
    if ic == "blast":
        h = 2.0 * grid_dim / nx / 2 ** max_level
        q = int(0.05 / h) + 2
        g = (np.arange(-q, q) + 0.5) * h
        gx, gy, gz = np.meshgrid(g, g, g, indexing="ij")
        cnt = int((np.sqrt(gx * gx + gy * gy + gz * gz) < 0.05).sum())
        eblast = 1.0 / (cnt * h ** 3) if cnt else 0.0
        rho = np.ones_like(X)
        ei = np.full_like(X, 1.0e-5 / (GAMMA - 1.0))
        ei = np.where(np.sqrt(X * X + Y * Y + Z * Z) < 0.05, ei + eblast, ei)
        zero = np.zeros_like(X)
        return _state(rho, zero, zero, zero, ei)
    if ic == "bump":
        r2 = (X - 0.08) ** 2 + (Y + 0.05) ** 2 + (Z - 0.06) ** 2
        rho = 1.0 + 9.0 * np.exp(-r2 / (0.15 * 0.15))
        vz = -0.15 + 0.1 * np.sin(2.0 * np.pi * X)
        ei = np.full_like(X, 0.6 / (GAMMA - 1.0))
        return _state(rho, np.full_like(X, 0.4), np.full_like(X, 0.25), vz, ei)
    if ic == "polytrope":
        K = poly_K()
        E1 = np.sqrt((4.0 * np.pi) / ((1.5 + 1.0) * K))
        h = tree["h"][:, None, None, None]
        acc = np.zeros_like(X)
        for k0 in range(2):
            for j0 in range(2):
                for i0 in range(2):
                    xs_ = X - 0.5 * h + (i0 + 0.5) * h / 2
                    ys_ = Y - 0.5 * h + (j0 + 0.5) * h / 2
                    zs_ = Z - 0.5 * h + (k0 + 0.5) * h / 2
                    r = np.sqrt(xs_ * xs_ + ys_ * ys_ + zs_ * zs_) * E1
                    inside = r < 3.65375
                    val = np.where(inside, lane_emden(np.where(inside, r, 0.0)) ** 1.5, 0.0)
                    acc += val / 8.0
        rho = np.maximum(acc, 1.0e-10)
        ei = K * rho ** (1.0 + 1.0 / 1.5) / (GAMMA - 1.0)
        zero = np.zeros_like(X)
        return _state(rho, zero, zero, zero, ei)
    if ic == "binary":
        return _binary_state(tree, bw, nx, grid_dim, z_reflect, ghosts)
    if ic == "random":
        F = random_field(seed)
        nn = F.shape[0]
        L = 2.0 * grid_dim
        zlo = 0.0 if z_reflect else -grid_dim
        u = [(X + grid_dim) / L * nn - 0.5, (Y + grid_dim) / L * nn - 0.5, (Z - zlo) / L * nn - 0.5]
        i0 = [np.floor(c).astype(np.int64) for c in u]
        fr = [c - f for c, f in zip(u, i0)]
        rho = np.zeros_like(X)
        for dz in (0, 1):
            for dy in (0, 1):
                for dx in (0, 1):
                    w = ((fr[0] if dx else 1 - fr[0]) * (fr[1] if dy else 1 - fr[1]) * (fr[2] if dz else 1 - fr[2]))
                    rho += w * F[(i0[0] + dx) % nn, (i0[1] + dy) % nn, (i0[2] + dz) % nn]
        rng = np.random.default_rng(seed + 1)
        v = rng.normal(0.0, 0.1, size=(3,) + X.shape)
        p = rho ** GAMMA
        return _state(rho, v[0], v[1], v[2], p / (GAMMA - 1.0))
    raise ValueError(ic)


def octant_flags(U_interior, thr):
    """set_refine_flags' density test on host data: [n, 8] bools."""
    rho = U_interior[:, 0]
    n, m = rho.shape[0], rho.shape[1]
    h = m // 2
    out = np.zeros((n, 8), np.uint8)
    for c in range(8):
        sx, sy, sz = c & 1, (c >> 1) & 1, (c >> 2) & 1
        blk = rho[:, sz * h:(sz + 1) * h, sy * h:(sy + 1) * h, sx * h:(sx + 1) * h]
        out[:, c] = (blk.reshape(n, -1) > thr).any(axis=1)
    return out


def _evaluate_padded(ic, t, bw, nx, grid_dim, z_reflect, max_level, ghosts):
    if ghosts:
        return evaluate(ic, t, bw, nx, grid_dim, z_reflect, max_level, ghosts=True)
    Ui = evaluate(ic, t, bw, nx, grid_dim, z_reflect, max_level, ghosts=False)
    g = nx + 2 * bw
    U = np.zeros((Ui.shape[0], Ui.shape[1], g, g, g))
    U[:, :, bw:-bw, bw:-bw, bw:-bw] = Ui
    return U


def build_tree(amr, ic, min_refine_density, grid_dim, z_reflect, max_level, device=True, ghosts=None):
    """Tree construction of the reference drivers (hydro_driver.cpp:84-107
    condensed): max_level rounds of initialize + check_for_refine, a final
    initialize, then restriction and ghost zones.  With device=False the
    density test runs on the host (host-only contexts).  ghosts=False
    evaluates interiors only (the ghost fill sets the face ghosts; edge and
    corner ghosts are never read); the default is False for the random
    field (large trees) and True otherwise."""
    if ghosts is None:
        ghosts = ic != "random"
    amr.init()
    amr.set_time(0.0)
    bw, nx = amr.bw, amr.nx
    for _ in range(max_level):
        t = amr.get_tree()
        U = _evaluate_padded(ic, t, bw, nx, grid_dim, z_reflect, max_level, ghosts)
        if device:
            amr.upload_state(U)
            amr.check_for_refine(min_refine_density, True)
        else:
            fl = octant_flags(U[:, :, bw:-bw, bw:-bw, bw:-bw], min_refine_density)
            amr.refine_from_flags(fl, True)
    t = amr.get_tree()
    U = _evaluate_padded(ic, t, bw, nx, grid_dim, z_reflect, max_level, ghosts)
    if device:
        amr.upload_state(U)
        amr.inject_from_children()
        amr.enforce_boundaries()
    return t, U
