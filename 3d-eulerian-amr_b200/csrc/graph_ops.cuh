// Device pieces shared by the graph-captured relaxation loop
// (graph_kernels.cu) and the persistent solve (persistent.cu): the
// reference's nested residual sums, the dphi ghost of a brick face taken from
// the previous pass's snapshot, and one relaxation pass of a brick.
#pragma once

#include "corr.cuh"
#include "graph.h"
#include "relax_brick.cuh"

namespace amr {

// Bottom-up nested sums over levels [0, top).  Values of level `top` are in
// `leaf` (per slot); S(node at m < top) = ((0 + S(c0)) + S(c1)) + ... in
// child order (withown = false), or ((own + S(c0)) + ...) (withown = true:
// own values in `leaf` for every level, `nest` preset to own at level top).  Result for the root is returned to
// thread 0.  Called by one whole block.
__device__ inline double nested_sum_block(const LevelLists& L, const int* __restrict__ child, const double* leaf,
                                   double* nest, int top, bool withown) {
    for (int m = top - 1; m >= 0; m--) {
        const int* sl = L.slots + L.off[m];
        for (int q = threadIdx.x; q < L.cnt[m]; q += blockDim.x) {
            const int p = sl[q];
            double s = withown ? __ldcg(leaf + p) : 0.0;
            for (int c = 0; c < 8; c++) {
                const int ch = child[8 * p + c];
                if (ch < 0) continue;
                s += (m + 1 == top && !withown) ? __ldcg(leaf + ch) : __ldcg(nest + ch);
            }
            nest[p] = s;
        }
        __threadfence_block();
        __syncthreads();
    }
    return __ldcg(nest + L.slots[L.off[0]]);
}

// Ghost zones of a relaxation pass (Poisson::vcycle_relax,
// poisson.cpp:88-130): in mode 0 they come from the brick's own dphi array (filled
// just before by the face ghost kernel).  In mode 1 the block fills them
// itself -- what Poisson::enforce_dphi_boundaries (poisson.cpp:890-929) would
// copy: a same-level neighbour's first interior layer from the snapshot the
// previous pass published, the parent's value across a coarse-fine face
// (PoissonAMRBound::get_dphi), 0 on a domain face, the mirror on z = 0 -- and
// also stores them into its global ghost cells, so the arrays end the loop
// exactly as the reference leaves them.  Every pass publishes its new first
// interior layers for the next pass.
// The same nested sum staged level by level in shared memory (buf:
// 2 * NEST_SMEM doubles) through the child-position table: leaves are the
// bricks of level `top` with values leaf[slot]; S(p) = ((own + S(c0)) +
// S(c1)) + ... in child order, own = leaf[p] when withown, else 0.  Same
// additions in the same order as nested_sum_block; the result is returned
// to every thread.  Needs L.max_cnt <= NEST_SMEM.
__device__ inline double nested_sum_smem_in(const LevelLists& L, const double* leaf, int top, bool withown,
                                            double* buf);
__device__ inline double nested_sum_smem(const LevelLists& L, const double* leaf, int top, bool withown,
                                         double* buf) {
    for (int q = threadIdx.x; q < L.cnt[top]; q += blockDim.x) buf[q] = __ldcg(leaf + L.slots[L.off[top] + q]);
    __syncthreads();
    return nested_sum_smem_in(L, leaf, top, withown, buf);
}

// nested_sum_smem with level `top`'s values already in buf[0 .. cnt[top])
// (level list order, made visible to the block); leaf is read only for the
// own values of the levels above (withown).
__device__ inline double nested_sum_smem_in(const LevelLists& L, const double* leaf, int top, bool withown,
                                            double* buf) {
    double* vb = buf;
    double* ub = buf + NEST_SMEM;
    const int e0 = L.off[0];
    for (int m = top - 1; m >= 0; m--) {
        for (int q = threadIdx.x; q < L.cnt[m]; q += blockDim.x) {
            const int* cp = L.cpos + 8 * (L.off[m] - e0 + q);
            double s = withown ? __ldcg(leaf + L.slots[L.off[m] + q]) : 0.0;
#pragma unroll
            for (int c = 0; c < 8; c++) {
                const int pos = cp[c];
                if (pos >= 0) s += vb[pos];
            }
            ub[q] = s;
        }
        __syncthreads();
        double* t = vb;
        vb = ub;
        ub = t;
    }
    const double r = vb[0];
    __syncthreads();
    return r;
}

// Entry of a snapshot layer: face f's first-interior layer, at face
// coordinates t1 (along the lower of the two other axes) and t2 (the
// higher), 1..NX.  t1 runs fastest, so the cells a warp relaxes (x fastest)
// write neighbouring entries of every face, and the ghost faces a warp
// fetches (relax_ghost_cell, t1 fastest) read neighbouring entries.
template <int NX>
__device__ __forceinline__ int layer_entry(int f, int t1, int t2) {
    return (f * NX + (t2 - 1)) * NX + (t1 - 1);
}

// `self`, when given, holds the brick's own values before this pass (a
// brick kept in shared memory); else they are read from dphi.
template <int NX, typename CT>
__device__ __forceinline__ CT ghost_dphi(const Geom& g, const BrickTable& bt, const DevState& st, const CT* snap_rd,
                                         size_t stride, int b, int face, int t1, int t2,
                                         const CT* self = nullptr) {
    constexpr int P = NX + 2;
    const int kind = bt.ftype[6 * b + face];
    const int nbr = bt.fnbr[6 * b + face];
    const CT* D = Corr<CT>::dphi(st);
    if (kind == FACE_SIB) return __ldcg(snap_rd + (size_t)nbr * stride + layer_entry<NX>(face ^ 1, t1, t2));
    if (kind == FACE_OUTFLOW) return CT(0);
    const int ax = face >> 1;
    const int qa = (face & 1) ? 1 : P - 2;  // the source layer along the face normal
    const int q0 = ax == 0 ? qa : t1;
    const int q1 = ax == 1 ? qa : (ax == 0 ? t1 : t2);
    const int q2 = ax == 2 ? qa : t2;
    if (kind == FACE_REFLECT) {  // own value mirrored through z = 0, before this pass
        const int kk = q2 == 1 ? P - 2 : 1;
        return self ? self[(kk * P + q1) * P + q0] : D[(size_t)b * P * P * P + (kk * P + q1) * P + q0];
    }
    const int v = (face & 1) ? 1 : -1;
    const int r0 = (bt.off[3 * b + 0] + (ax == 0 ? v * (P - 2) : 0) - 2 * bt.off[3 * nbr + 0] - (g.bw - 1) + q0) / 2;
    const int r1 = (bt.off[3 * b + 1] + (ax == 1 ? v * (P - 2) : 0) - 2 * bt.off[3 * nbr + 1] - (g.bw - 1) + q1) / 2;
    const int r2 = (bt.off[3 * b + 2] + (ax == 2 ? v * (P - 2) : 0) - 2 * bt.off[3 * nbr + 2] - (g.bw - 1) + q2) / 2;
    return D[(size_t)nbr * P * P * P + (r2 * P + r1) * P + r0];
}

// Ghost face cell q (< 6 NX^2) of the (NX+2)^3 brick, and its face
// coordinates.
template <int NX>
__device__ __forceinline__ int relax_ghost_cell(int q, int& face, int& t1, int& t2) {
    constexpr int P = NX + 2, F = NX * NX;
    face = q / F;
    const int qq = q % F;
    t1 = qq % NX + 1;
    t2 = qq / NX + 1;
    const int ax = face >> 1;
    int d[3];
    d[ax] = (face & 1) ? P - 1 : 0;
    d[ax == 0 ? 1 : 0] = t1;
    d[ax == 2 ? 1 : 2] = t2;
    return (d[2] * P + d[1]) * P + d[0];
}

// Where interior cell t (interior index) lies on a face, writes its value to
// that face's first-interior layer of the snapshot (layer of face f holds
// the cells adjacent to it).
template <int NX, typename CT>
__device__ __forceinline__ void relax_layer_put(CT* sw, int t, CT v) {
    const int ci = t % NX + 1, cj = (t / NX) % NX + 1, ck = t / (NX * NX) + 1;
    if (ci == 1) sw[layer_entry<NX>(0, cj, ck)] = v;
    if (ci == NX) sw[layer_entry<NX>(1, cj, ck)] = v;
    if (cj == 1) sw[layer_entry<NX>(2, ci, ck)] = v;
    if (cj == NX) sw[layer_entry<NX>(3, ci, ck)] = v;
    if (ck == 1) sw[layer_entry<NX>(4, ci, cj)] = v;
    if (ck == NX) sw[layer_entry<NX>(5, ci, cj)] = v;
}

// relax_layer_put for a snapshot of tagged entries (64 bits: the FP32 value
// in the low half, the pass word `tag` in the high half), each written with
// one relaxed 64-bit store: a reader that sees the tag it waits for sees
// that pass's value, with no fence and no flag between them.
__device__ __forceinline__ void tagged_put(unsigned long long* p, float v, unsigned tag) {
    const unsigned long long w = ((unsigned long long)tag << 32) | __float_as_uint(v);
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(w) : "memory");
}
// Only the faces in `faces` (bit f for face f) are written: a layer is read
// only by the same-level neighbour across that face.
template <int NX>
__device__ __forceinline__ void relax_layer_put_tagged(unsigned long long* sw, int t, float v, unsigned tag,
                                                       unsigned faces) {
    const int ci = t % NX + 1, cj = (t / NX) % NX + 1, ck = t / (NX * NX) + 1;
    if ((faces & 1u) && ci == 1) tagged_put(sw + layer_entry<NX>(0, cj, ck), v, tag);
    if ((faces & 2u) && ci == NX) tagged_put(sw + layer_entry<NX>(1, cj, ck), v, tag);
    if ((faces & 4u) && cj == 1) tagged_put(sw + layer_entry<NX>(2, ci, ck), v, tag);
    if ((faces & 8u) && cj == NX) tagged_put(sw + layer_entry<NX>(3, ci, ck), v, tag);
    if ((faces & 16u) && ck == 1) tagged_put(sw + layer_entry<NX>(4, ci, cj), v, tag);
    if ((faces & 32u) && ck == NX) tagged_put(sw + layer_entry<NX>(5, ci, cj), v, tag);
}

// Writes a relaxed interior value of cell t to dphi and to the snapshot.
template <int NX, typename CT>
__device__ __forceinline__ void relax_put(CT* D, CT* sw, int t, CT v) {
    constexpr int P = NX + 2;
    D[((t / (NX * NX) + 1) * P + (t / NX) % NX + 1) * P + t % NX + 1] = v;
    relax_layer_put<NX, CT>(sw, t, v);
}

// One relaxation pass of brick b by TH threads (local index lt, barrier
// `sync`): mode 1 fills the ghost faces from the snapshot snap_rd first; the
// relaxed interior goes to dphi, its first interior layers to snap_wr, the
// last sweep's sum to pres[b].  Called by every one of the TH threads.
template <int NX, int TH, typename CT, typename Sync>
__device__ __forceinline__ void op_relax_pass(const Geom& g, const BrickTable& bt, const DevState& st, int b,
                                              int mode, const CT* snap_rd, CT* snap_wr, size_t stride,
                                              double* pres, RelaxSmem<NX, CT>& sm, int lt, Sync sync) {
    constexpr int P = NX + 2, P3 = P * P * P, F = NX * NX, K = NX * NX * NX / TH;
    CT* D = Corr<CT>::dphi(st) + (size_t)b * P3;
    if (mode == 1) {
        for (int q = lt; q < 6 * F; q += TH) {
            int face, t1, t2;
            const int gi = relax_ghost_cell<NX>(q, face, t1, t2);
            D[gi] = ghost_dphi<NX, CT>(g, bt, st, snap_rd, stride, b, face, t1, t2);
        }
        sync();
    }
    int c[K];
    CT v[K];
    const double resid = relax_brick<NX, TH, CT>(sm, D, Corr<CT>::dphi1(st) + (size_t)b * P3, lt, c, v, sync);
    CT* sw = snap_wr + (size_t)b * stride;
#pragma unroll
    for (int r = 0; r < K; r++) relax_put<NX, CT>(D, sw, lt + r * TH, v[r]);
    if (lt == 0) pres[b] = resid;
}

// op_relax_pass in mode 1 split in two, so that a pass can be computed
// before the loop has decided whether it runs.  op_relax_spec computes it
// from the current dphi and the snapshot snap_rd with nothing written to
// global memory (the ghost faces go to the staged brick only, where the
// sweeps leave them); op_relax_commit then writes what op_relax_pass
// writes: the ghost faces and the relaxed interior to dphi, the first
// interior layers to snap_wr, the sum to pres[b].  Same values as
// op_relax_pass; called by every thread of a block of TH threads, with the
// brick's shared memory untouched in between.
template <typename CT, int K>
struct RelaxSpec {
    CT v[K];       // this thread's relaxed interior cells
    double resid;  // the brick's last sweep sum
};

template <int NX, int TH, typename CT>
__device__ __forceinline__ RelaxSpec<CT, NX * NX * NX / TH> op_relax_spec(const Geom& g, const BrickTable& bt,
                                                                        const DevState& st, int b, const CT* snap_rd,
                                                                        size_t stride, RelaxSmem<NX, CT>& sm) {
    constexpr int P = NX + 2, P3 = P * P * P, F = NX * NX, K = NX * NX * NX / TH, G = (6 * F + TH - 1) / TH;
    const CT* D = Corr<CT>::dphi(st) + (size_t)b * P3;
    const int lt = threadIdx.x;
    CT gv[G];
    int gi[G];
#pragma unroll
    for (int r = 0; r < G; r++) {
        const int q = lt + r * TH;
        gi[r] = -1;
        if (q < 6 * F) {
            int face, t1, t2;
            gi[r] = relax_ghost_cell<NX>(q, face, t1, t2);
            gv[r] = ghost_dphi<NX, CT>(g, bt, st, snap_rd, stride, b, face, t1, t2);
        }
    }
    relax_stage<NX, TH, CT>(sm, D, lt);
    int c[K];
    CT d1[K];
    relax_cells<NX, TH, CT>(lt, Corr<CT>::dphi1(st) + (size_t)b * P3, c, d1);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < G; r++)
        if (gi[r] >= 0) {
            sm.buf[0][gi[r]] = gv[r];
            sm.buf[1][gi[r]] = gv[r];
        }
    __syncthreads();
    RelaxSpec<CT, K> out;
    out.resid = relax_sweeps<NX, TH, CT>(sm, lt, c, d1, out.v, BlockSync{});
    return out;
}

template <int NX, int TH, typename CT>
__device__ __forceinline__ void op_relax_commit(const DevState& st, int b, const RelaxSpec<CT, NX * NX * NX / TH>& r,
                                                const RelaxSmem<NX, CT>& sm, CT* snap_wr, size_t stride,
                                                double* pres) {
    constexpr int P = NX + 2, P3 = P * P * P, F = NX * NX, K = NX * NX * NX / TH;
    CT* D = Corr<CT>::dphi(st) + (size_t)b * P3;
    const int lt = threadIdx.x;
    for (int q = lt; q < 6 * F; q += TH) {
        int face, t1, t2;
        const int gi = relax_ghost_cell<NX>(q, face, t1, t2);
        D[gi] = sm.buf[0][gi];
    }
    CT* sw = snap_wr + (size_t)b * stride;
#pragma unroll
    for (int q = 0; q < K; q++) relax_put<NX, CT>(D, sw, lt + q * TH, r.v[q]);
    if (lt == 0) pres[b] = r.resid;
}

}  // namespace amr
