// Diagnostics as device reductions: GridNode::state_sum
// (grid/grid_node.cpp:1489-1527), Binary::mass_sum (binary/binary.cpp:28-68)
// and Binary::sum_lz (binary.cpp:363-388).  Each brick's sums over its
// uncovered interior cells are formed by one thread in the reference's loop
// order (one-thread OpenMP order), the bricks in parallel; the host adds
// them over the tree as the reference's recursion does (own sums first, then
// each child's subtree in child order).
#include <cuda_runtime.h>

#include <cmath>
#include <functional>
#include <vector>

#include "context.h"
#include "launch.cuh"

using namespace amr;

namespace {

__device__ __forceinline__ double centre(const Geom& g, int axis, int off, double h, int gi) {
    double f;
    if (axis < 2)
        f = double(off + gi) * h - g.grid_dim - double(g.bw) * g.h0 - g.origin[axis];
    else if (g.z_reflect)
        f = double(off + gi) * h - double(g.bw) * g.h0 - g.origin[2];
    else
        f = double(off + gi) * h - g.grid_dim - double(g.bw) * g.h0;
    return f + 0.5 * h;
}

// mode 0: (sum u h3, sum u h3 x, sum u h3 y, sum u h3 z) of field `field`,
// cells in (k, j, i) order, h3 = pow(h, 3) from the host;
// mode 1: sum lz dx*dx*dx, cells in (i, j, k) order, each (i, j) pencil
// summed separately (Binary::sum_lz)
__global__ void k_leaf_moments(Geom g, BrickTable bt, DevState st, const int* __restrict__ slots, int n,
                               const double* __restrict__ h3s, int field, int mode, double* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int b = slots[e];
    const int nx = g.nx, gnx = g.gnx, bw = g.bw;
    const double* u = st.U + (size_t)b * g.ucount + (size_t)field * g.gnx3;
    const double h = bt.h[b];
    const int* off = bt.off + 3 * b;
    const int* child = bt.child + 8 * b;
    auto covered = [&](int i, int j, int k) {
        return child[(2 * i / gnx) | ((2 * j / gnx) << 1) | ((2 * k / gnx) << 2)] >= 0;
    };
    if (mode == 0) {
        const double h3 = h3s[e];
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        for (int k = bw; k < bw + nx; k++)
            for (int j = bw; j < bw + nx; j++)
                for (int i = bw; i < bw + nx; i++) {
                    if (covered(i, j, k)) continue;
                    const double ds = u[(k * gnx + j) * gnx + i] * h3;
                    a0 += ds;
                    a1 += ds * centre(g, 0, off[0], h, i);
                    a2 += ds * centre(g, 1, off[1], h, j);
                    a3 += ds * centre(g, 2, off[2], h, k);
                }
        out[4 * e + 0] = a0;
        out[4 * e + 1] = a1;
        out[4 * e + 2] = a2;
        out[4 * e + 3] = a3;
    } else {
        // the k loop is an OpenMP reduction of its own (binary.cpp:372-378):
        // each (i, j) pencil is summed from 0 and then added to s
        const double dx3 = h * h * h;
        double s = 0.0;
        for (int i = bw; i < bw + nx; i++)
            for (int j = bw; j < bw + nx; j++) {
                double p = 0.0;
                for (int k = bw; k < bw + nx; k++)
                    if (!covered(i, j, k)) p += u[(k * gnx + j) * gnx + i] * dx3;
                s += p;
            }
        out[4 * e] = s;
    }
}

#define TRY(x)                        \
    do {                              \
        int rc_ = (x);                \
        if (rc_ != AMR_OK) return rc_; \
    } while (0)
#define CUDA_TRY(x)                                   \
    do {                                              \
        cudaError_t e_ = (x);                         \
        if (e_ != cudaSuccess) {                      \
            c->err = cudaGetErrorString(e_);          \
            return AMR_ERR_CUDA;                      \
        }                                             \
    } while (0)

// per-brick moments of one field, in DFS order
int moments(amr_ctx* c, int field, int mode, std::vector<double>& per) {
    if (!c) return AMR_ERR_ARG;
    if (!c->has_device) {
        c->err = "context has no device pool";
        return AMR_ERR_NODEVICE;
    }
    if (field < 0 || field >= c->geom.nf) return AMR_ERR_ARG;
    const int n = (int)c->order.size();
    std::vector<double> h3(n);
    for (int e = 0; e < n; e++) h3[e] = std::pow(c->order[e]->h, 3);  // pow(get_dx(), 3)
    double* d = nullptr;
    CUDA_TRY(cudaMalloc(&d, sizeof(double) * 5 * (size_t)n));
    int rc = AMR_OK;
    do {
        if (cudaMemcpyAsync(d, h3.data(), sizeof(double) * n, cudaMemcpyHostToDevice, c->stream) != cudaSuccess) {
            rc = AMR_ERR_CUDA;
            break;
        }
        launch_k(k_leaf_moments, (n + 63) / 64, 64, 0, c->stream, c->geom, c->bt, c->st, c->d_slots + c->off_all[0], n,
                 (const double*)d, field, mode, d + n);
        per.assign(4 * (size_t)n, 0.0);
        if (cudaMemcpyAsync(per.data(), d + n, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, c->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(c->stream) != cudaSuccess)
            rc = AMR_ERR_CUDA;
    } while (0);
    cudaFree(d);
    if (rc != AMR_OK) c->err = "diagnostic reduction failed";
    return rc;
}

// the reference's recursion: own values, then each child's subtree in order
void tree_sum(const Node* nd, const std::vector<double>& per, int ncomp, const std::function<void(double*)>& own_fix,
              double* out) {
    for (int q = 0; q < ncomp; q++) out[q] = per[4 * (size_t)nd->dfs + q];
    own_fix(out);
    for (int ch = 0; ch < 8; ch++)
        if (nd->child[ch]) {
            double s[4];
            tree_sum(nd->child[ch], per, ncomp, own_fix, s);
            for (int q = 0; q < ncomp; q++) out[q] += s[q];
        }
}

}  // namespace

extern "C" {

int amr_state_sum(amr_ctx* c, int field, double* out) {
    if (!out) return AMR_ERR_ARG;
    std::vector<double> per;
    TRY(moments(c, field, 0, per));
    tree_sum(c->tree.root(), per, 4, [](double*) {}, out);
    return AMR_OK;
}

int amr_mass_sum(amr_ctx* c, int frac, double* out) {
    if (!out || (frac != 0 && frac != 1)) return AMR_ERR_ARG;
    if (c && !is_ztwd(c)) {
        c->err = "mass_sum needs the ZTWD state (accretor / donor densities)";
        return AMR_ERR_ARG;
    }
    std::vector<double> per;
    TRY(moments(c, frac == 0 ? 1 : 2, 0, per));  // rho_accretor / rho_donor
    const bool zr = c->geom.z_reflect != 0;
    tree_sum(c->tree.root(), per, 4, [zr](double* a) {
        if (zr) a[3] = 0.0;  // Z_REFLECT: the z moment is zero by symmetry (binary.cpp:51-55)
    }, out);
    out[1] /= out[0];
    out[2] /= out[0];
    out[3] /= out[0];
    return AMR_OK;
}

int amr_sum_lz(amr_ctx* c, double* out) {
    if (!out) return AMR_ERR_ARG;
    if (c && !is_ztwd(c)) {
        c->err = "sum_lz needs the ZTWD state";
        return AMR_ERR_ARG;
    }
    std::vector<double> per;
    TRY(moments(c, 4, 1, per));
    tree_sum(c->tree.root(), per, 1, [](double*) {}, out);
    return AMR_OK;
}

}  // extern "C"
