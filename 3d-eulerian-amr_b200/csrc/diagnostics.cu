// Diagnostics as device reductions: GridNode::state_sum
// (grid/grid_node.cpp:1489-1527), Binary::mass_sum (binary/binary.cpp:28-68),
// Binary::sum_lz (binary.cpp:363-388) and Binary::M1M2data
// (binary.cpp:718-823 with find_l1 :390-447, mark_lobes :449-492,
// find_phimin :642-690).  Each brick's sums (or searches) over its cells are
// formed by one thread in the reference's loop order (one-thread OpenMP
// order), the bricks in parallel; the host combines them over the tree in
// the order of the reference's recursion.
#include <cuda_runtime.h>

#include <cmath>
#include <functional>
#include <vector>

#include "context.h"
#include "launch.cuh"
#include "poisson.h"

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

// ---- Binary::M1M2data -------------------------------------------------

// cell centre of Poisson-frame index p (Poisson::pxc = Grid::xc(p + BW - 1))
__device__ __forceinline__ double pcentre(const Geom& g, int axis, int off, double h, int p) {
    return centre(g, axis, off, h, p + g.bw - 1);
}

// Binary::find_phimin over one brick (lobe ln: x > 0 or x < 0), cells in
// (i, j, k) order, from phi_min = 1e99: the first strict minimum of the
// effective potential among uncovered local minima -> out[3 e ..] = (min,
// x, y).  The reference's pow(c, 2) is formed as c * c.
__global__ void k_phimin(Geom g, BrickTable bt, DevState st, const int* __restrict__ slots, int n, double O2, int ln,
                         double* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int b = slots[e];
    const int P = g.pnx;
    const double* phi = st.phi + (size_t)b * g.pnx3;
    const double h = bt.h[b];
    const int* off = bt.off + 3 * b;
    const int* child = bt.child + 8 * b;
    auto xc = [&](int i) { return pcentre(g, 0, off[0], h, i); };
    auto yc = [&](int j) { return pcentre(g, 1, off[1], h, j); };
    auto ph = [&](int i, int j, int k) { return phi[(k * P + j) * P + i]; };
    auto eff = [&](double v, double a, double c) { return v - 0.5 * (a * a + c * c) * O2; };
    double pmin = 1.0e99, x0 = 0.0, y0 = 0.0;
    for (int i = 1; i < P - 1; i++)
        for (int j = 1; j < P - 1; j++)
            for (int k = 1; k < P - 1; k++) {
                const double x = xc(i), y = yc(j);
                const bool covered = child[((2 * i) / P) | (((2 * j) / P) << 1) | (((2 * k) / P) << 2)] >= 0;
                if (!(((ln == 1 && x > 0.0) || (ln == 2 && x < 0.0)) && !covered)) continue;
                const double phi1 = ph(i, j, k) - 0.5 * (x * x + y * y) * O2;
                const double phi_px = eff(ph(i + 1, j, k), xc(i + 1), yc(j));
                const double phi_mx = eff(ph(i - 1, j, k), xc(i - 1), yc(j));
                const double phi_py = eff(ph(i, j + 1, k), xc(i), yc(j + 1));
                const double phi_my = eff(ph(i, j - 1, k), xc(i), yc(j - 1));
                const double phi_pz = eff(ph(i, j, k + 1), xc(i), yc(j));
                const double phi_mz = eff(ph(i, j, k - 1), xc(i), yc(j));
                if (pmin > phi1 && phi1 <= phi_px && phi1 <= phi_py && phi1 <= phi_pz && phi1 <= phi_mx &&
                    phi1 <= phi_my && phi1 <= phi_mz) {
                    pmin = phi1;
                    x0 = x;
                    y0 = y;
                }
            }
    out[3 * e + 0] = pmin;
    out[3 * e + 1] = x0;
    out[3 * e + 2] = y0;
}

// Binary::find_l1 over one brick, cells in (i, j, k) order, from -1e99: the
// first strict maximum of the effective potential among uncovered cells in
// the band |z| <= h near the segment between the two centres of mass
// (m1x, m1y), (m2x, m2y) -> out[4 e ..] = (phi0, x, y, z).
__global__ void k_find_l1(Geom g, BrickTable bt, DevState st, const int* __restrict__ slots, int n, double O2,
                          double m1x, double m1y, double m2x, double m2y, double* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int b = slots[e];
    const int P = g.pnx;
    const double* phi = st.phi + (size_t)b * g.pnx3;
    const double h = bt.h[b];
    const int* off = bt.off + 3 * b;
    const int* child = bt.child + 8 * b;
    double v0 = -1.0e99, v1 = 0.0, v2 = 0.0, v3 = 0.0;
    for (int i = 1; i < P - 1; i++)
        for (int j = 1; j < P - 1; j++)
            for (int k = 1; k < P - 1; k++) {
                const double x = pcentre(g, 0, off[0], h, i), y = pcentre(g, 1, off[1], h, j);
                const double z = pcentre(g, 2, off[2], h, k);
                if (fabs(z) > h) continue;
                const double dx0 = m2x - m1x, dx1 = x - m1x, dx2 = x - m2x;
                const double dy0 = m2y - m1y, dy1 = y - m1y, dy2 = y - m2y;
                const double a2 = dx0 * dx0 + dy0 * dy0;
                const double b2 = dx1 * dx1 + dy1 * dy1;
                const double c2 = dx2 * dx2 + dy2 * dy2;
                const double bc = b2 - c2;
                const double z2 = 0.5 * ((b2 + c2) - (0.5 / a2) * (bc * bc) - 0.5 * a2);
                if (z2 > (3.0 * h * h / 4.0) || z2 < 0.0) continue;
                if (dx1 * dx2 + dy1 * dy2 > 0.0) continue;
                const double phi0 = phi[(k * P + j) * P + i] - 0.5 * (x * x + y * y) * O2;
                const bool covered = child[((2 * i) / P) | (((2 * j) / P) << 1) | (((2 * k) / P) << 2)] >= 0;
                if (!covered && phi0 > v0) {
                    v0 = phi0;
                    v1 = x;
                    v2 = y;
                    v3 = z;
                }
            }
    out[4 * e + 0] = v0;
    out[4 * e + 1] = v1;
    out[4 * e + 2] = v2;
    out[4 * e + 3] = v3;
}

struct LobeFrame {
    double l1, l1x, l1y, c1x, c2x, c1y, c2y;
};

constexpr int M1M2_N = 28;  // m1 m2 mc js1 js2 jorb jc a q E K I1 I2 Ic V1 V2, x1 xdot1 x2 xdot2

// Binary::mark_lobes (the lobe of each cell from the effective potential,
// the face forces and the L1 frame) fused with one brick's share of
// Binary::M1M2data: uncovered interior cells in (k, j, i) order (Indexer2d
// over (j, k), j fastest), sums in the reference's expression order.
// h3s[e] = pow(h, 3) from the host.
__global__ void k_m1m2(Geom g, BrickTable bt, DevState st, const int* __restrict__ slots, int n,
                       const double* __restrict__ h3s, double omega, double omega0, LobeFrame L,
                       double* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int b = slots[e];
    const int nx = g.nx, gnx = g.gnx, bw = g.bw, P = g.pnx;
    const double* U = st.U + (size_t)b * g.ucount;
    const size_t pb = (size_t)b * g.pnx3;
    const double* phi = st.phi + pb;
    const double *fx = st.fx + pb, *fy = st.fy + pb, *fz = st.fz + pb;
    const double h = bt.h[b];
    const double h3 = h3s[e];
    const int* off = bt.off + 3 * b;
    const int* child = bt.child + 8 * b;
    const double O2 = omega * omega;
    double m1 = 0, m2 = 0, mc = 0, js1 = 0, js2 = 0, jc = 0, E = 0, K = 0, I1 = 0, I2 = 0, Ic = 0, V1 = 0, V2 = 0;
    double x1[3] = {0, 0, 0}, xd1[3] = {0, 0, 0}, x2[3] = {0, 0, 0}, xd2[3] = {0, 0, 0};
    for (int k = bw; k < bw + nx; k++)
        for (int j = bw; j < bw + nx; j++)
            for (int i = bw; i < bw + nx; i++) {
                if (child[(2 * i / gnx) | ((2 * j / gnx) << 1) | ((2 * k / gnx) << 2)] >= 0) continue;
                const double X[3] = {centre(g, 0, off[0], h, i), centre(g, 1, off[1], h, j),
                                     centre(g, 2, off[2], h, k)};
                // mark_lobes at Poisson cell (i, j, k) - (BW - 1)
                const int c = ((k - bw + 1) * P + (j - bw + 1)) * P + (i - bw + 1);
                const double x = X[0], y = X[1], z = X[2];
                const double phi0 = phi[c] - 0.5 * (x * x + y * y) * O2;
                int lobe = 0;
                if (phi0 < L.l1) {
                    const double nxx = 0.5 * (fx[c] + fx[c + 1]) + x * O2;
                    const double nyy = 0.5 * (fy[c] + fy[c + P]) + y * O2;
                    const double nzz = 0.5 * (fz[c] + fz[c + P * P]);
                    if ((x - L.l1x) * (L.c1x - L.c2x) + (y - L.l1y) * (L.c1y - L.c2y) > 0.0) {
                        if (nxx * (x - L.c1x) + nyy * (y - L.c1y) + nzz * z < 0.0) lobe = 1;
                    } else {
                        if (nxx * (x - L.c2x) + nyy * (y - L.c2y) + nzz * z < 0.0) lobe = 2;
                    }
                }
                const size_t cell = (size_t)(k * gnx + j) * gnx + i;
                auto u = [&](int f) { return U[(size_t)f * g.gnx3 + cell]; };
                const double rho = u(0), sr = u(3), lz = u(4), sz = u(5), pot = u(6), et = u(7);
                const double R2 = X[0] * X[0] + X[1] * X[1];
                const double R = sqrt(X[0] * X[0] + X[1] * X[1]);
                const double st_ = lz / R - rho * R * omega;  // State::st
                const double V[3] = {(X[0] * sr - X[1] * st_) / R / rho, (X[1] * sr + X[0] * st_) / R / rho, sz / rho};
                if (lobe != 0) {
                    double* xs = lobe == 1 ? x1 : x2;
                    double* xd = lobe == 1 ? xd1 : xd2;
                    (lobe == 1 ? V1 : V2) += h3;
                    (lobe == 1 ? m1 : m2) += rho * h3;
                    for (int q = 0; q < 3; q++) xs[q] += X[q] * rho * h3;
                    for (int q = 0; q < 3; q++) xd[q] += V[q] * rho * h3;
                    xd[0] -= omega * X[1] * rho * h3;
                    xd[1] += omega * X[0] * rho * h3;
                    (lobe == 1 ? js1 : js2) += lz * h3;
                    (lobe == 1 ? I1 : I2) += (X[0] * X[0] + X[1] * X[1]) * rho * h3;
                }
                // State::et_inertial, State::pot_inertial (Omega0)
                const double eti = et + omega0 * (lz - 0.5 * rho * omega0 * R2);
                const double poti = pot + 0.5 * rho * omega0 * omega0 * R2;
                mc += rho * h3;
                jc += lz * h3;
                E += eti * h3 + poti * h3 * 0.5;
                K += eti * h3;
                Ic += (X[0] * X[0] + X[1] * X[1]) * rho * h3;
            }
    double* o = out + (size_t)M1M2_N * e;
    const double sc[16] = {m1, m2, mc, js1, js2, 0.0, jc, 0.0, 0.0, E, K, I1, I2, Ic, V1, V2};
    for (int q = 0; q < 16; q++) o[q] = sc[q];
    for (int q = 0; q < 3; q++) {
        o[16 + q] = x1[q];
        o[19 + q] = xd1[q];
        o[22 + q] = x2[q];
        o[25 + q] = xd2[q];
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

// Binary::M1M2data at the root (binary.cpp:718-823): the centres of mass
// of both stars (mass_sum), the L1 point (find_l1, pre-order, first strict
// maximum), the lobe centres (find_phimin in mark_lobes, pre-order, first
// strict minimum), then the lobe-marked integrals summed in the
// recursion's post order (children first, then the node's own) and the
// root's closing arithmetic.
int m1m2data(amr_ctx* c, double* out, double* l1out) {
    double mf1[4], mf2[4];
    TRY(amr_mass_sum(c, 0, mf1));
    TRY(amr_mass_sum(c, 1, mf2));
    TRY(poisson_need(c));
    const int n = (int)c->order.size();
    const int* slots = c->d_slots + c->off_all[0];
    const double O = c->zpar.omega, O2 = O * O;
    std::vector<double> h3(n);
    for (int e = 0; e < n; e++) h3[e] = std::pow(c->order[e]->h, 3);  // pow(get_dx(), 3)
    double* d = nullptr;
    const size_t per_n = (size_t)M1M2_N * n;
    CUDA_TRY(cudaMalloc(&d, sizeof(double) * (n + per_n)));
    double* dout = d + n;
    std::vector<double> per(per_n);
    auto run = [&](auto launch, int ncomp) -> int {
        launch();
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(per.data(), dout, sizeof(double) * ncomp * n, cudaMemcpyDeviceToHost, c->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(c->stream) != cudaSuccess)
            return AMR_ERR_CUDA;
        return AMR_OK;
    };
    const int nb = (n + 63) / 64;
    int rc = AMR_OK;
    double L1[4] = {-1.0e99, 0.0, 0.0, 0.0};
    LobeFrame F{};
    do {
        if (cudaMemcpyAsync(d, h3.data(), sizeof(double) * n, cudaMemcpyHostToDevice, c->stream) != cudaSuccess) {
            rc = AMR_ERR_CUDA;
            break;
        }
        // find_l1: own cells, then each child's subtree
        rc = run([&] { launch_k(k_find_l1, nb, 64, 0, c->stream, c->geom, c->bt, c->st, slots, n, O2, mf1[1], mf1[2],
                                mf2[1], mf2[2], dout); }, 4);
        if (rc) break;
        std::function<void(const Node*)> l1rec = [&](const Node* nd) {
            const double* v = &per[4 * (size_t)nd->dfs];
            if (v[0] > L1[0]) std::copy(v, v + 4, L1);
            for (int ch = 0; ch < 8; ch++)
                if (nd->child[ch]) l1rec(nd->child[ch]);
        };
        l1rec(c->tree.root());
        F = LobeFrame{L1[0], L1[1], L1[2], mf1[1], mf2[1], mf1[2], mf2[2]};
        // find_phimin(&c1x, &c1y, 1) and (&c2x, &c2y, 2)
        for (int ln = 1; ln <= 2 && rc == AMR_OK; ln++) {
            rc = run([&] { launch_k(k_phimin, nb, 64, 0, c->stream, c->geom, c->bt, c->st, slots, n, O2, ln, dout); },
                     3);
            if (rc) break;
            double pmin = 1.0e99;
            double& cx = ln == 1 ? F.c1x : F.c2x;
            double& cy = ln == 1 ? F.c1y : F.c2y;
            std::function<void(const Node*)> mrec = [&](const Node* nd) {
                const double* v = &per[3 * (size_t)nd->dfs];
                if (v[0] < pmin) {
                    pmin = v[0];
                    cx = v[1];
                    cy = v[2];
                }
                for (int ch = 0; ch < 8; ch++)
                    if (nd->child[ch]) mrec(nd->child[ch]);
            };
            mrec(c->tree.root());
        }
        if (rc) break;
        rc = run([&] { launch_k(k_m1m2, nb, 64, 0, c->stream, c->geom, c->bt, c->st, slots, n, (const double*)d, O,
                                c->zpar.omega0, F, dout); }, M1M2_N);
    } while (0);
    cudaFree(d);
    if (rc != AMR_OK) {
        c->err = "M1M2data reduction failed";
        return rc;
    }
    // post order: the children's subtrees, then the node's own sums
    double b[M1M2_N] = {};
    std::function<void(const Node*)> prec = [&](const Node* nd) {
        for (int ch = 0; ch < 8; ch++)
            if (nd->child[ch]) prec(nd->child[ch]);
        const double* v = &per[(size_t)M1M2_N * nd->dfs];
        for (int q = 0; q < M1M2_N; q++)
            if (q != 5 && q != 7 && q != 8) b[q] += v[q];  // jorb, a, q are formed at the root
    };
    prec(c->tree.root());
    double &m1 = b[0], &m2 = b[1], &js1 = b[3], &js2 = b[4], &jorb = b[5], &a = b[7], &q = b[8], &I1 = b[11],
           &I2 = b[12];
    double *x1 = b + 16, *xd1 = b + 19, *x2 = b + 22, *xd2 = b + 25;
    if (c->geom.z_reflect) x1[2] = xd1[2] = x2[2] = xd2[2] = 0.0;
    q = m2 / m1;
    for (int k = 0; k < 3; k++) {
        x1[k] /= m1;
        x2[k] /= m2;
        xd1[k] /= m1;
        xd2[k] /= m2;
    }
    auto dot = [](const double* u, const double* v) {  // Vector::dot
        double s = 0;
        for (int k = 0; k < 3; k++) s += u[k] * v[k];
        return s;
    };
    const double dx[3] = {x1[0] - x2[0], x1[1] - x2[1], x1[2] - x2[2]};
    a = std::sqrt(dot(dx, dx));
    const double j1 = m1 * (x1[0] * xd1[1] - x1[1] * xd1[0]);
    const double j2 = m2 * (x2[0] * xd2[1] - x2[1] * xd2[0]);
    jorb = j1 + j2;
    js1 -= j1;
    js2 -= j2;
    I1 -= m1 * dot(x1, x1);
    I2 -= m2 * dot(x2, x2);
    std::copy(b, b + M1M2_N, out);
    if (l1out) std::copy(L1, L1 + 4, l1out);
    return AMR_OK;
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

int amr_m1m2data(amr_ctx* c, double* out, double* l1) {
    if (!c || !out) return AMR_ERR_ARG;
    if (!is_ztwd(c)) {
        c->err = "M1M2data needs the ZTWD state";
        return AMR_ERR_ARG;
    }
    if (!c->has_device) {
        c->err = "context has no device pool";
        return AMR_ERR_NODEVICE;
    }
    return m1m2data(c, out, l1);
}

}  // extern "C"
