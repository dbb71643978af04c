// Internal declarations shared by the host octree code and the CUDA kernels.
#pragma once

#include <cstddef>
#include <cstdint>

#include "amr_b200.h"

namespace amr {

enum Face { XL = 0, XU = 1, YL = 2, YU = 3, ZL = 4, ZU = 5 };
// Ghost-zone source of one brick face (grid_node.cpp:59-112 sibling kinds).
enum FaceKind : int {
    FACE_SIB = 0,      // same-level neighbour brick: copy its interior
    FACE_AMR = 1,      // coarse-fine: GridAMRBound, interpolate from the parent
    FACE_OUTFLOW = 2,  // GridPhysBound, copy + State::enforce_outflow
    FACE_REFLECT = 3,  // GridPhysBound with Z_REFLECT: mirror, negate sz
};

// Geometry and physics constants passed by value to every kernel.
struct Geom {
    int bw, nx, gnx, nf, pnx;
    int gnx3, pnx3, ucount;  // gnx^3, pnx^3, nf*gnx^3
    int z_reflect;
    int precision;  // correction type of the multigrid solve: AMR_PREC_FP64 / AMR_PREC_MIXED (FP32)
    int flux32;     // the KT reconstruction and flux in FP32 (AMR_PREC_MIXED)
    int recon;      // AMR_RECON_MINMOD / AMR_RECON_PPM (same values as RECON_* in recon.cuh)
    double grid_dim, h0;
    double origin[3];
    double theta, cfl, gamma, rho_floor, ei_floor, grav_g;
};

// Device brick table (struct of arrays, indexed by brick slot).
struct BrickTable {
    int* level;    // [cap]
    int* off;      // [3*cap] Grid::offset
    double* h;     // [cap]
    int* ftype;    // [6*cap] FaceKind
    int* fnbr;     // [6*cap] neighbour slot (SIB) or parent slot (AMR), -1 otherwise
    int* parent;   // [cap]
    int* cidx;     // [cap] child index within the parent
    int* child;    // [8*cap] child slots or -1
};

// Device state arrays (all FP64, indexed [slot][...]).
struct DevState {
    double* U;    // [cap][nf][gnx^3]
    double* U0;   // [cap][nf][gnx^3]
    double* Fx;   // [cap][nf][nx][nx][nx+1]   x faces i=bw..gnx-bw
    double* Fy;   // [cap][nf][nx][nx+1][nx]
    double* Fz;   // [cap][nf][nx+1][nx][nx]
    double* phi;  // [cap][pnx^3] ... Poisson arrays
    double* phi0;
    double* dphi;
    double* dphi1;
    double* S;
    double* fx;
    double* fy;
    double* fz;
    // mixed-precision form: the V-cycle correction (dphi, dphi1) in FP32;
    // null in the FP64 form
    float* fdphi;
    float* fdphi1;
    // ZTWD state only (null otherwise): primitives [cap][nf][gnx^3] and the
    // face-averaged normal velocities [cap][nx][nx][nx+1] per direction
    double* W;
    double* Vx;
    double* Vy;
    double* Vz;
};

// One coarse-fine flux (or force) correction task: coarse brick's face
// quadrant (dir, i0, cj, ck) := mean of the child's four faces at index ic
// (GridNode::adjust_x_flux, grid_node.cpp:1076-1140).
struct RefluxItem {
    int coarse, child, dir, i0, ic, cj, ck, pad;
};

// Kernels launched (or recorded into a graph) by the calling host thread.
extern thread_local long long g_launch_tally;

}  // namespace amr
