"""CPU restatement (numpy) of the reference's hydro step on an octree.

Test infrastructure only: the oracle the CUDA path is checked against, itself
pinned to the reference (tests/test_oracle_restatement.py replays golden runs
of the reference built in oracle/_ref).  Nothing in the product imports it.

Data: a tree given as depth-first pre-order lists (level, location) and the
conserved state U[n, 6, gnx, gnx, gnx] (fields d sx sy sz et tau, index
[f][k][j][i]).  Topology (neighbours, parents, offsets) is derived here from
the locations alone.  Every arithmetic expression keeps the reference's
operation order; numpy elementwise operations round like the reference's
scalar FP64 code (no FMA contraction), and np.power calls the C library pow.
"""

import numpy as np

XL, XU, YL, YU, ZL, ZU = range(6)


class Tree:
    """Octree topology from a DFS pre-order node list (oct_node/oct_node.cpp)."""

    def __init__(self, level, loc, bw=2, nx=8, grid_dim=0.5, z_reflect=False):
        self.level = np.asarray(level, np.int64)
        self.loc = np.asarray(loc, np.int64).reshape(-1, 3)
        self.n = len(self.level)
        self.bw, self.nx, self.gnx = bw, nx, nx + 2 * bw
        self.grid_dim, self.z_reflect = grid_dim, z_reflect
        self.h0 = 2.0 * grid_dim / nx  # Grid::h0, grid/grid.cpp:70
        self.index = {(int(self.level[i]),) + tuple(int(x) for x in self.loc[i]): i for i in range(self.n)}
        self.parent = np.full(self.n, -1, np.int64)
        self.cidx = np.zeros(self.n, np.int64)
        self.child = np.full((self.n, 8), -1, np.int64)
        for i in range(1, self.n):
            L = int(self.level[i])
            pl = tuple(int(x) // 2 for x in self.loc[i])
            p = self.index[(L - 1,) + pl]
            c = int(self.loc[i][0] % 2) | (int(self.loc[i][1] % 2) << 1) | (int(self.loc[i][2] % 2) << 2)
            self.parent[i], self.cidx[i] = p, c
            self.child[p, c] = i
        # Grid::offset (grid_node.cpp:244): 2*parent offset + BW + c*(GNX-2BW)
        self.offset = np.zeros((self.n, 3), np.int64)
        for i in range(1, self.n):
            p, c = self.parent[i], self.cidx[i]
            for d in range(3):
                self.offset[i, d] = 2 * self.offset[p, d] + bw + ((c >> d) & 1) * nx
        self.h = np.array([self.h0 * 0.5 ** int(L) for L in self.level])

    def is_phys(self, i, face):
        hi = (1 << int(self.level[i])) - 1
        ax = face >> 1
        return self.loc[i][ax] == (hi if face & 1 else 0)

    def neighbor(self, i, face):
        if self.is_phys(i, face):
            return None
        l = [int(x) for x in self.loc[i]]
        l[face >> 1] += 1 if face & 1 else -1
        return self.index.get((int(self.level[i]),) + tuple(l))

    def levels(self):
        return range(int(self.level.max()) + 1)


# ---------------------------------------------------------------------------
# real.h / vector.h / euler/state.cpp
# ---------------------------------------------------------------------------
def sgn(a):
    return np.where(a > 0.0, 1.0, np.where(a < 0.0, -1.0, 0.0))


def rmin(a, b):  # real.h:41-43: a > b ? b : a
    return np.where(a > b, b, a)


def rmax(a, b):  # real.h:21-23
    return np.where(a > b, a, b)


def minmod2(a, b):  # real.h:63-65
    return 0.5 * (sgn(a) + sgn(b)) * rmin(np.abs(a), np.abs(b))


def minmod_theta(up, um, th):  # vector.h:195-202
    return minmod2(th * up, minmod2(th * um, 0.5 * (up + um)))


def ek(u):  # euler/state.cpp:181-183
    return 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0]


def pg(u, gamma):  # euler/state.cpp:189-196
    ei0 = u[4] - ek(u)
    return np.where(ei0 < 0.001 * u[4], (gamma - 1.0) * np.power(u[5], gamma), (gamma - 1.0) * ei0)


def to_prim(u):  # euler/state.cpp:246-251
    u = u.copy()
    u[4] = u[4] - ek(u)
    u[1] = u[1] / u[0]
    u[2] = u[2] / u[0]
    u[3] = u[3] / u[0]
    return u


def to_con(u):  # euler/state.cpp:253-258
    u = u.copy()
    u[1] = u[1] * u[0]
    u[2] = u[2] * u[0]
    u[3] = u[3] * u[0]
    u[4] = u[4] + ek(u)
    return u


def floor(u, gamma, rho_floor=1.0e-20, ei_floor=1.0e-20):  # euler/state.cpp:86-92
    u = u.copy()
    u[0] = rmax(u[0], rho_floor)
    ei0 = u[4] - ek(u)
    with np.errstate(invalid="ignore"):
        tau = np.power(rmax(ei0, ei_floor), 1.0 / gamma)
    u[5] = np.where(ei0 > 0.1 * u[4], tau, u[5])
    return u


def flux_eigen(u, d, gamma):  # euler/state.cpp:198-244
    v = u[1 + d] / u[0]
    p = pg(u, gamma)
    f = u * v
    f[1 + d] = f[1 + d] + p
    f[4] = f[4] + v * p
    cs = np.sqrt(gamma * p / u[0])
    return f, np.abs(v) + cs


def enforce_outflow(u, bface):  # euler/state.cpp:45-84 (bface: the proxy's face)
    u = u.copy()
    m = 1 + (bface >> 1)
    if bface in (ZU, ZL):
        zero = u[3] > 0.0 if bface == ZU else u[3] < 0.0
    else:
        v = u[m] / u[0]
        zero = v > 0.0 if bface & 1 else v < 0.0
    u[4] = np.where(zero, u[4] - 0.5 * u[m] * u[m] / u[0], u[4])
    u[m] = np.where(zero, 0.0, u[m])
    return u


# ---------------------------------------------------------------------------
# ghost zones (grid_node.cpp:59-112, grid_amr_bound.cpp, grid_phys_bound.cpp)
# ---------------------------------------------------------------------------
def _sl(ax, lo, hi, bw, gnx):
    """index tuple (f, k, j, i) for cells lo..hi-1 along axis ax (0=x..2=z)
    and the transverse interior."""
    s = [slice(None), slice(bw, gnx - bw), slice(bw, gnx - bw), slice(bw, gnx - bw)]
    s[3 - ax] = slice(lo, hi)
    return tuple(s)


def enforce_boundaries(T, U):
    bw, gnx = T.bw, T.gnx
    order = np.argsort(T.level, kind="stable")
    for i in order:  # parents before children
        for face in range(6):
            ax, up = face >> 1, face & 1
            g0, g1 = (gnx - bw, gnx) if up else (0, bw)
            dst = _sl(ax, g0, g1, bw, gnx)
            if T.is_phys(i, face):
                if T.z_reflect and face == ZL:
                    src = U[i][_sl(ax, bw, 2 * bw, bw, gnx)]
                    v = np.flip(src, axis=3 - ax).copy()
                    v[3] = -v[3]
                    U[i][dst] = v
                else:
                    c = gnx - bw - 1 if up else bw
                    src = U[i][_sl(ax, c, c + 1, bw, gnx)]
                    v = np.repeat(src, bw, axis=3 - ax)
                    U[i][dst] = enforce_outflow(v, face ^ 1)
                continue
            j = T.neighbor(i, face)
            if j is not None:
                s0 = g0 - (gnx - 2 * bw) if up else g0 + (gnx - 2 * bw)
                U[i][dst] = U[j][_sl(ax, s0, s0 + bw, bw, gnx)]
                continue
            # coarse-fine: parent cell -/+ a quarter of the face-normal minmod slope
            p = T.parent[i]
            rel = T.offset[i] - 2 * T.offset[p]
            idx = [np.arange(bw, gnx - bw)] * 3
            idx = list(idx)
            idx[ax] = np.arange(g0, g1)
            fine = [rel[d] + idx[d] for d in range(3)]
            pi = [f // 2 for f in fine]
            par = fine[ax] % 2
            K, J, I = np.meshgrid(pi[2], pi[1], pi[0], indexing="ij")
            P = U[p]
            u = P[:, K, J, I]
            e = [0, 0, 0]
            e[ax] = 1
            up_ = P[:, K + e[2], J + e[1], I + e[0]]
            um_ = P[:, K - e[2], J - e[1], I - e[0]]
            m = minmod2(up_ - u, u - um_)
            parity = [None, None, None]
            shape = [1, 1, 1]
            shape[2 - ax] = -1
            parg = par.reshape(shape)
            m = np.where(parg == 1, -m, m)
            U[i][dst] = u - m * 0.25
    return U


# ---------------------------------------------------------------------------
# fluxes (grid.cpp:215-302, reconstruct.cpp:60-71) and corrections
# ---------------------------------------------------------------------------
def ppm_faces(q, bw):
    """Left and right states of faces bw..gnx-bw of pencils q[..., gnx]
    (primitives along the last axis): Reconstruct::ppm
    (reconstruct.cpp:22-58) as Reconstruct::operator() calls it,
    ppm(q0, qr, ql) (reconstruct.cpp:94).  Inside ppm the array named qr
    holds the interface to the right of cell i, ql the one to its left; after
    the monotonisation the right edges are shifted up one cell (:55-57), so
    the caller's ql[f] is the right edge of cell f-1 and its qr[f] the left
    edge of cell f.  The Euler state has no low-order or smooth field
    (euler/state.h:37-42), so every field is treated alike."""
    n = q.shape[-1]
    six = 1.0 / 6.0
    s = np.zeros_like(q)
    s[..., 1:-1] = minmod_theta(q[..., 2:] - q[..., 1:-1], q[..., 1:-1] - q[..., :-2], 2.0)
    # interface to the right of cell i, i = 1..n-3
    I = np.zeros_like(q)
    I[..., 1:n - 2] = (q[..., 1:n - 2] + q[..., 2:n - 1]) * 0.5
    I[..., 1:n - 2] = I[..., 1:n - 2] + (s[..., 1:n - 2] - s[..., 2:n - 1]) * six
    # Colella-Woodward monotonisation of cells 2..n-3 (edges L = I[i-1], R = I[i])
    c = q[..., 2:n - 2]
    L = I[..., 1:n - 3]
    R = I[..., 2:n - 2]
    tmp1 = R - L
    tmp2 = R + L
    flat = (R - c) * (c - L) <= 0.0
    steep_l = tmp1 * (c - 0.5 * tmp2) > six * tmp1 * tmp1
    steep_r = -six * tmp1 * tmp1 > tmp1 * (c - 0.5 * tmp2)
    Lm = np.where(flat, c, np.where(steep_l, 3.0 * c - 2.0 * R, L))
    Rm = np.where(flat, c, np.where(~steep_l & steep_r, 3.0 * c - 2.0 * L, R))
    # Lm/Rm index m holds cell m + 2; face f: left = Rm[f-1], right = Lm[f]
    f = np.arange(bw, n - bw + 1)
    return Rm[..., f - 3], Lm[..., f - 2]


def brick_fluxes(Ub, bw, theta, gamma, recon="minmod"):
    """Face fluxes of one brick: F[d] of shape (nf, nx+1, nx, nx) indexed
    (field, face along d, lower transverse, higher transverse), and the max
    face eigenvalue (Grid::max_dt's inner max).  recon: "minmod"
    (reconstruct.cpp:60-71) or "ppm" (reconstruct.cpp:22-58, needs bw >= 3)."""
    gnx = Ub.shape[-1]
    nx = gnx - 2 * bw
    out, lam = [], 0.0
    for d in range(3):
        # move axis d to last, transverse interior: V[f, t2, t1, n]
        if d == 0:
            V = Ub[:, bw:-bw, bw:-bw, :]
        elif d == 1:
            V = np.transpose(Ub[:, bw:-bw, :, bw:-bw], (0, 1, 3, 2))
        else:
            V = np.transpose(Ub[:, :, bw:-bw, bw:-bw], (0, 2, 3, 1))
        q = to_prim(V)
        if recon == "ppm":
            ql, qr = ppm_faces(q, bw)
        else:
            s = np.zeros_like(q)
            s[..., 1:-1] = minmod_theta(q[..., 2:] - q[..., 1:-1], q[..., 1:-1] - q[..., :-2], theta)
            f = np.arange(bw, gnx - bw + 1)
            ql = q[..., f - 1] + s[..., f - 1] / 2.0
            qr = q[..., f] - s[..., f] / 2.0
        ql, qr = to_con(ql), to_con(qr)
        fl, al = flux_eigen(ql, d, gamma)
        fr, ar = flux_eigen(qr, d, gamma)
        a = rmax(al, ar)
        F = ((fl + fr) - (qr - ql) * a) * 0.5  # (f, t2, t1, face)
        lam = max(lam, float(np.max(rmax(al, ar))))
        out.append(np.transpose(F, (0, 3, 2, 1)))  # (f, face, t1, t2)
    return out, lam


def reflux(T, F):
    """GridNode::adjust_{x,y,z}_flux (grid_node.cpp:1076-1274), finest
    coarse level first."""
    bw, gnx, nx = T.bw, T.gnx, T.nx
    half = nx // 2
    for L in sorted(T.levels(), reverse=True):
        for P in [i for i in range(T.n) if T.level[i] == L]:
            for d in range(3):
                nlo, nhi = T.neighbor(P, 2 * d), T.neighbor(P, 2 * d + 1)
                ta, tb = (1, 2) if d == 0 else ((0, 2) if d == 1 else (0, 1))
                for l in range(3):
                    for ck in range(2):
                        for cj in range(2):
                            base = (cj << ta) | (ck << tb)
                            c0, c1 = base, base | (1 << d)
                            if l == 0:
                                cr = T.child[P, c0]
                                cl = T.child[nlo, c1] if nlo is not None else -1
                                i0 = 0
                            elif l == 1:
                                cl, cr, i0 = T.child[P, c0], T.child[P, c1], half
                            else:
                                cr = T.child[nhi, c0] if nhi is not None else -1
                                cl, i0 = T.child[P, c1], nx
                            if cr < 0 and cl >= 0:
                                ch, ic = cl, nx
                            elif cl < 0 and cr >= 0:
                                ch, ic = cr, 0
                            else:
                                continue
                            C = F[ch][d][:, ic]
                            v = +C[:, 0::2, 0::2]
                            v = v + C[:, 1::2, 0::2]
                            v = v + C[:, 0::2, 1::2]
                            v = v + C[:, 1::2, 1::2]
                            v = v * 0.25
                            F[P][d][:, i0, cj * half:(cj + 1) * half, ck * half:(ck + 1) * half] = v
    return F


def add_difs(T, U, U0, F, dt, beta, gamma):
    """clear_difs + sum_{x,y,z}_difs + Grid::add_difs (grid.cpp:201-420)."""
    bw, gnx = T.bw, T.gnx
    for i in range(T.n):
        hinv = 1.0 / T.h[i]
        Fx, Fy, Fz = F[i]
        D = np.zeros((6, T.nx, T.nx, T.nx))
        # x: Fx (f, face_i, j, k) -> D (f, k, j, i)
        gx = np.transpose(Fx, (0, 3, 2, 1))
        D = D - (gx[..., 1:] - gx[..., :-1]) * hinv
        gy = np.transpose(Fy, (0, 3, 1, 2))  # (f, k, face_j, i)
        D = D - (gy[:, :, 1:, :] - gy[:, :, :-1, :]) * hinv
        gz = np.transpose(Fz, (0, 1, 3, 2))  # (f, face_k, j, i)
        D = D - (gz[:, 1:] - gz[:, :-1]) * hinv
        D = D + 0.0
        u = U[i][:, bw:-bw, bw:-bw, bw:-bw]
        u0 = U0[i][:, bw:-bw, bw:-bw, bw:-bw]
        u = (u + D * dt) * beta + u0 * (1.0 - beta)
        U[i][:, bw:-bw, bw:-bw, bw:-bw] = floor(u, gamma)
    return U


def inject_from_children(T, U, gamma):
    """GridNode::inject_from_children (grid_node.cpp:1035-1074)."""
    bw, gnx, nx = T.bw, T.gnx, T.nx
    half = nx // 2
    for L in sorted(T.levels(), reverse=True):
        for P in [i for i in range(T.n) if T.level[i] == L]:
            for c in range(8):
                ch = T.child[P, c]
                if ch < 0:
                    continue
                C = U[ch][:, bw:-bw, bw:-bw, bw:-bw]
                s = 0.0 + C[:, 0::2, 0::2, 0::2]
                s = s + C[:, 0::2, 0::2, 1::2]
                s = s + C[:, 0::2, 1::2, 0::2]
                s = s + C[:, 0::2, 1::2, 1::2]
                s = s + C[:, 1::2, 0::2, 0::2]
                s = s + C[:, 1::2, 0::2, 1::2]
                s = s + C[:, 1::2, 1::2, 0::2]
                s = s + C[:, 1::2, 1::2, 1::2]
                s = s * 0.125
                ox, oy, oz = (c & 1) * half, ((c >> 1) & 1) * half, ((c >> 2) & 1) * half
                U[P][:, bw + oz:bw + oz + half, bw + oy:bw + oy + half, bw + ox:bw + ox + half] = floor(s, gamma)
    return U


def max_dt(T, U, theta, gamma, cfl, recon="minmod"):
    """Grid::max_dt per brick and GridNode::max_dt's recursion."""
    own = np.zeros(T.n)
    for i in range(T.n):
        _, lam = brick_fluxes(U[i], T.bw, theta, gamma, recon)
        dtinv = lam / T.h[i]
        if dtinv == 0.0:
            dtinv = 1.0e-10
        own[i] = (1.0 / dtinv) * cfl

    def rec(i):
        dtinv = 0.0
        for c in range(8):
            ch = T.child[i, c]
            if ch >= 0:
                cdt = 1.0 / rec(ch)
                dtinv = cdt if cdt > dtinv else dtinv
        o = 1.0 / own[i]
        dtinv = o if o > dtinv else dtinv
        return 1.0 / dtinv

    return rec(0)


def sub_step(T, U, U0, dt, beta, theta=1.3, gamma=5.0 / 3.0, recon="minmod"):
    """HydroDriver::sub_step (euler/hydro_driver.cpp:200-214) without
    regrid; returns the updated U."""
    U = enforce_boundaries(T, U)
    F = [brick_fluxes(U[i], T.bw, theta, gamma, recon)[0] for i in range(T.n)]
    F = reflux(T, F)
    return add_difs(T, U, U0, F, dt, beta, gamma)


def step(T, U, dt, theta=1.3, gamma=5.0 / 3.0, recon="minmod"):
    """HydroDriver::step (euler/hydro_driver.cpp:171-194) on a fixed tree."""
    U0 = U.copy()
    for beta in (1.0, 0.25, 2.0 / 3.0):
        U = sub_step(T, U, U0, dt, beta, theta, gamma, recon)
        U = inject_from_children(T, U, gamma)
    return enforce_boundaries(T, U)
