"""Reader for the raw dumps written by oracle/harness/amr_harness.cpp.

Test infrastructure.  A dump is a depth-first (pre-order, children 0..7) list
of octree nodes, each with its level, location, offset, age, child and
refinement masks, cell width and the full conserved state including ghost
cells, optionally followed by the Poisson arrays of that node.
"""

import numpy as np

POISSON_ARRAYS = ("phi", "phi0", "dphi", "dphi1", "S", "fx", "fy", "fz")


class Dump:
    pass


def read_dump(path):
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != b"AMRDUMP1":
        raise ValueError("not an AMR dump: %s" % path)
    off = 8
    bw, gnx, nf, pnx, has_p, nnodes, nextra, _ = np.frombuffer(data, np.int32, 8, off)
    off += 32
    time = float(np.frombuffer(data, np.float64, 1, off)[0])
    off += 8
    d = Dump()
    d.bw, d.gnx, d.nf, d.pnx = int(bw), int(gnx), int(nf), int(pnx)
    d.time = time
    n = int(nnodes)
    d.level = np.zeros(n, np.int32)
    d.loc = np.zeros((n, 3), np.int32)
    d.offset = np.zeros((n, 3), np.int32)
    d.age = np.zeros(n, np.int32)
    d.child_mask = np.zeros(n, np.int32)
    d.refine_mask = np.zeros(n, np.int32)
    d.h = np.zeros(n, np.float64)
    d.U = np.zeros((n, d.nf, d.gnx, d.gnx, d.gnx), np.float64)
    if has_p:
        d.P = {k: np.zeros((n, d.pnx, d.pnx, d.pnx), np.float64) for k in POISSON_ARRAYS}
    else:
        d.P = None
    ucount = d.nf * d.gnx ** 3
    pcount = d.pnx ** 3
    for b in range(n):
        hdr = np.frombuffer(data, np.int32, 10, off)
        off += 40
        d.level[b] = hdr[0]
        d.loc[b] = hdr[1:4]
        d.offset[b] = hdr[4:7]
        d.age[b] = hdr[7]
        d.child_mask[b] = hdr[8]
        d.refine_mask[b] = hdr[9]
        d.h[b] = np.frombuffer(data, np.float64, 1, off)[0]
        off += 8
        d.U[b] = np.frombuffer(data, np.float64, ucount, off).reshape(d.nf, d.gnx, d.gnx, d.gnx)
        off += 8 * ucount
        if has_p:
            for k in POISSON_ARRAYS:
                d.P[k][b] = np.frombuffer(data, np.float64, pcount, off).reshape(d.pnx, d.pnx, d.pnx)
                off += 8 * pcount
    d.FO = np.frombuffer(data, np.float64, d.nf, off).copy()
    off += 8 * d.nf
    d.extra = np.frombuffer(data, np.float64, int(nextra), off).copy()
    d.nnodes = n
    return d


def leaf_mask(d):
    """Boolean (n, nx, nx, nx) mask of interior cells not covered by a child
    (GridNode::zone_is_refined, grid_node.cpp:1401-1408)."""
    bw, gnx = d.bw, d.gnx
    nx = gnx - 2 * bw
    idx = np.arange(bw, gnx - bw)
    oct_ = (2 * idx) // gnx
    m = np.ones((d.nnodes, nx, nx, nx), bool)
    for b in range(d.nnodes):
        cm = int(d.child_mask[b])
        if cm == 0:
            continue
        c = oct_[None, None, :] + 2 * oct_[None, :, None] + 4 * oct_[:, None, None]
        covered = ((cm >> c) & 1).astype(bool)
        m[b] = ~covered
    return m
