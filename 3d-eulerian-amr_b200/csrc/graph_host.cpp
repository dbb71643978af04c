// Graph-captured self-gravitating step.
//
// The whole RK3 step -- CFL step, store, three substeps of hydro + gravity
// sources, each followed by a multigrid solve whose V-cycle loop and
// relaxation loops are CUDA-graph WHILE nodes decided on the device -- is
// captured once per topology and replayed every step; the graph is
// re-instantiated only after a regrid changes the tree.  The kernels and the
// order of every floating-point operation are those of the plain path, so
// the graph form reproduces it bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <functional>
#include <string>
#include <vector>

#include "context.h"
#include "graph.h"
#include "kernels.h"
#include "persistent.h"
#include "poisson.h"

using namespace amr;

#define CUDA_TRY(call)                                                                        \
    do {                                                                                      \
        cudaError_t e__ = (call);                                                             \
        if (e__ != cudaSuccess) {                                                             \
            c->err = std::string("CUDA error: ") + cudaGetErrorString(e__) + " at " + #call; \
            return AMR_ERR_CUDA;                                                              \
        }                                                                                     \
    } while (0)

#define TRY(x)                 \
    do {                       \
        int rc__ = (x);        \
        if (rc__) return rc__; \
    } while (0)

// entries per brick in one face-snapshot buffer: 6 faces of nx*nx
inline size_t snap_stride(const amr_ctx* c) { return 6 * (size_t)c->geom.nx * c->geom.nx; }

struct GraphState {
    Control* d_ctl = nullptr;
    Control* h_ctl = nullptr;  // pinned mirror
    double* d_nest = nullptr;
    double* d_snap = nullptr;  // [2][cap][6][nx][nx] first-interior dphi layers
    unsigned int* d_counter = nullptr;
    int* h_steps = nullptr;     // pinned scalar staging
    cudaGraphExec_t step_exec = nullptr;
    long long step_version = -1;
    double step_tol = -1.0;
    cudaGraphExec_t solve_exec = nullptr;
    long long solve_version = -1;
    double solve_tol = -1.0;
    int solve_max = -1;
    std::vector<cudaStream_t> streams;  // capture streams of nested bodies
    LevelLists L{};
    // kernels recorded into the captured graphs (counted by the launch
    // tally while recording): top level of the step / solve graph, one
    // V-cycle body outside its relaxation loops, one relaxation loop body
    long long k_step = 0, k_solve = 0, k_vbody = 0, k_rbody = 0;
    // persistent solve: cooperative blocks, [3][cap] per-brick sums,
    // [blocks][cap] nested-sum scratch, barrier word
    int pblocks = 0;
    int layout = 0;        // block layout of the solve kernel (solve_layout_threads)
    int per_sm = 0;        // blocks per SM cap of the launch (0: as many as fit)
    int pnest_blocks = 0;  // blocks d_pnest has room for (the most of any layout)
    double* d_pres3 = nullptr;
    double* d_pnest = nullptr;
    GridBarrier* d_bar = nullptr;
    unsigned* d_rpub = nullptr;  // [cap] relaxation pass words of the persistent solve
    unsigned long long* d_tsnap = nullptr;  // [2][cap][6][nx][nx] tagged face snapshots (FP32 correction)
    unsigned long long* d_tpres = nullptr;  // [2][cap][2] tagged per-brick relaxation sums (FP32 correction)
    cudaEvent_t ev_ps[2] = {nullptr, nullptr};  // around the last persistent launch
    double ps_ms_total = 0.0;                   // persistent launches of amr_graph_solve: device time, count
    long long ps_count = 0;
    long long rec_in_bodies = 0;  // kernels recorded inside outermost WHILE bodies
    long long rec_nested = 0;     // kernels recorded inside the bodies of the body being recorded
    int while_depth = 0;
    int nlevels_captured = 0;
    long long last_cycles = 0, last_relax = 0;  // device counters at the last read
    long long last_relax_level[MAX_LEVELS] = {};
};

namespace {

int ensure_state(amr_ctx* c) {
    if (c->gs) return AMR_OK;
    GraphState* g = new GraphState;
    c->gs = g;
    CUDA_TRY(cudaMalloc(&g->d_ctl, sizeof(Control)));
    CUDA_TRY(cudaMemsetAsync(g->d_ctl, 0, sizeof(Control), c->stream));
    CUDA_TRY(cudaMallocHost(&g->h_ctl, sizeof(Control)));
    CUDA_TRY(cudaMallocHost(&g->h_steps, sizeof(int) * 5));
    CUDA_TRY(cudaMalloc(&g->d_nest, sizeof(double) * c->cap));
    CUDA_TRY(cudaMalloc(&g->d_snap, sizeof(double) * 2 * snap_stride(c) * (size_t)c->cap));
    if (relax_dev_attributes() != 0 || solve_persistent_attributes() != 0) {
        c->err = "shared-memory attributes of the relaxation kernels";
        return AMR_ERR_CUDA;
    }
    CUDA_TRY(cudaMalloc(&g->d_counter, sizeof(unsigned int) * 4));
    CUDA_TRY(cudaMemsetAsync(g->d_counter, 0, sizeof(unsigned int) * 4, c->stream));
    if (c->cfg.persistent_solve) {
        g->layout = 0;
        g->per_sm = c->cfg.persistent_solve;
        g->pblocks = solve_persistent_blocks(c->geom.nx, c->geom.precision, g->per_sm, g->layout);
        if (g->pblocks <= 0) {
            c->err = "no cooperative launch configuration for the persistent solve";
            return AMR_ERR_CUDA;
        }
        g->pnest_blocks = g->pblocks;
        for (int l = 0; l < solve_layouts(c->geom.nx); l++)
            g->pnest_blocks = std::max(g->pnest_blocks, solve_persistent_blocks(c->geom.nx, c->geom.precision, 0, l));
        CUDA_TRY(cudaMalloc(&g->d_pres3, sizeof(double) * 3 * (size_t)c->cap));
        CUDA_TRY(cudaMalloc(&g->d_pnest, sizeof(double) * (size_t)g->pnest_blocks * c->cap));
        CUDA_TRY(cudaMalloc(&g->d_bar, sizeof(GridBarrier)));
        CUDA_TRY(cudaMalloc(&g->d_rpub, sizeof(unsigned) * (size_t)c->cap));
        if (c->geom.precision == AMR_PREC_MIXED) {
            CUDA_TRY(cudaMalloc(&g->d_tsnap, sizeof(unsigned long long) * 2 * snap_stride(c) * (size_t)c->cap));
            CUDA_TRY(cudaMalloc(&g->d_tpres, sizeof(unsigned long long) * 4 * (size_t)c->cap));
        }
        CUDA_TRY(cudaEventCreate(&g->ev_ps[0]));
        CUDA_TRY(cudaEventCreate(&g->ev_ps[1]));
    }
    // side streams for capturing nested loop bodies, created outside any capture
    for (int d = 0; d < 4; d++) {
        cudaStream_t s;
        CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        g->streams.push_back(s);
    }
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return AMR_OK;
}

int max_level_present(amr_ctx* c) {
    int m = 0;
    for (Node* n : c->order) m = std::max(m, n->level);
    return m;
}

void fill_lists(amr_ctx* c) {
    LevelLists& L = c->gs->L;
    L.slots = c->d_slots;
    L.all = c->d_slots + c->off_all[0];
    L.nall = (int)c->all_slots.size();
    L.cap = c->cap;
    for (int m = 0; m < MAX_LEVELS; m++) {
        const bool ok = m < (int)c->level_slots.size();
        L.off[m] = ok ? c->off_level[m] : 0;
        L.cnt[m] = ok ? (int)c->level_slots[m].size() : 0;
    }
    L.cpos = c->d_cpos;
    L.max_cnt = c->max_level_cnt;
}

cudaStream_t body_stream(amr_ctx* c, int depth) {
    GraphState* g = c->gs;
    while ((int)g->streams.size() <= depth) {
        cudaStream_t s;
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        g->streams.push_back(s);
    }
    return g->streams[depth];
}

// At the current capture point of s: run pre(s, h), then add a WHILE node on
// handle h whose body is captured from body(s2, h) on a side stream.
int add_while(amr_ctx* c, cudaStream_t s, int depth, const std::function<int(cudaStream_t, cudaGraphConditionalHandle)>& pre,
              const std::function<int(cudaStream_t, cudaGraphConditionalHandle)>& body) {
    cudaStreamCaptureStatus status;
    cudaGraph_t graph;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    CUDA_TRY(cudaStreamGetCaptureInfo(s, &status, nullptr, &graph, &deps, &ndeps));
    if (status != cudaStreamCaptureStatusActive) {
        c->err = "add_while outside an active capture";
        return AMR_ERR_STATE;
    }
    cudaGraphConditionalHandle h;
    CUDA_TRY(cudaGraphConditionalHandleCreate(&h, graph, 0, 0));
    TRY(pre(s, h));
    CUDA_TRY(cudaStreamGetCaptureInfo(s, &status, nullptr, &graph, &deps, &ndeps));
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    CUDA_TRY(cudaGraphAddNode(&node, graph, deps, ndeps, &p));
    cudaGraph_t bodyg = p.conditional.phGraph_out[0];
    CUDA_TRY(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    cudaStream_t s2 = body_stream(c, depth);
    CUDA_TRY(cudaStreamBeginCaptureToGraph(s2, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    GraphState* gs = c->gs;
    const long long t0 = g_launch_tally, n0 = gs->rec_nested;
    gs->rec_nested = 0;
    gs->while_depth++;
    const int rc = body(s2, h);
    gs->while_depth--;
    const long long all_k = g_launch_tally - t0, own = all_k - gs->rec_nested;
    gs->rec_nested = n0 + all_k;
    if (gs->while_depth == 0) gs->rec_in_bodies += all_k;
    (depth == 0 ? gs->k_vbody : gs->k_rbody) = own;
    cudaGraph_t out;
    const cudaError_t e = cudaStreamEndCapture(s2, &out);
    if (rc) return rc;
    if (e != cudaSuccess) {
        c->err = std::string("body capture failed: ") + cudaGetErrorString(e);
        return AMR_ERR_CUDA;
    }
    return AMR_OK;
}

int launched(amr_ctx* c, int line) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        c->err = std::string("CUDA launch error at graph_host.cpp:") + std::to_string(line) + ": " + cudaGetErrorString(e);
        return AMR_ERR_CUDA;
    }
    return AMR_OK;
}

const int* lvl(amr_ctx* c, int l) { return c->d_slots + c->off_level[l]; }
int nlvl(amr_ctx* c, int l) { return (int)c->level_slots[l].size(); }
const int* all(amr_ctx* c) { return c->d_slots + c->off_all[0]; }
int nall(amr_ctx* c) { return (int)c->all_slots.size(); }

int rec_relax_until(amr_ctx* c, cudaStream_t s, int l, double ratio, int depth) {
    GraphState* g = c->gs;
    launch_dphi_boundaries(c->geom, c->bt, c->st, c->d_bphi, c->d_perr, lvl(c, l), nlvl(c, l), s);
    return add_while(
        c, s, depth,
        [&](cudaStream_t q, cudaGraphConditionalHandle h) {
            launch_relax_dev(c->geom, c->bt, c->st, g->L, l, 0, ratio, h, g->d_ctl, c->d_pres, g->d_nest,
                             g->d_counter, g->d_snap, snap_stride(c), q);
            return launched(c, __LINE__);
        },
        [&](cudaStream_t q, cudaGraphConditionalHandle h) {
            // ghost fill folded into the pass (face snapshot of the previous pass)
            launch_relax_dev(c->geom, c->bt, c->st, g->L, l, 1, ratio, h, g->d_ctl, c->d_pres, g->d_nest,
                             g->d_counter, g->d_snap, snap_stride(c), q);
            return launched(c, __LINE__);
        });
}

int rec_forces(amr_ctx* c, cudaStream_t s) {
    launch_forces(c->geom, c->bt, c->st, all(c), nall(c), s);
    for (int l = c->tree.prm.max_level; l >= 0; l--) {
        const int n = c->off_reflux[l + 1] - c->off_reflux[l];
        launch_adjust_force(c->geom, c->st, c->d_reflux + c->off_reflux[l], n, s);
    }
    return launched(c, __LINE__);
}

// Poisson::vcycle (poisson.cpp:1069-1074) ending in the loop decision.
int rec_vcycle(amr_ctx* c, cudaStream_t s, int depth, cudaGraphConditionalHandle hsolve, double tol) {
    GraphState* g = c->gs;
    const int maxlevel = max_level_present(c);
    launch_set_source(c->geom, c->st, all(c), nall(c), s);
    for (int l = maxlevel - 1; l >= 0; l--)
        launch_phi_from_children(c->geom, c->bt, c->st, c->d_slots + c->off_parent[l], (int)c->parent_slots[l].size(),
                                 s);
    for (int l = 0; l <= maxlevel; l++)
        launch_phi_boundaries(c->geom, c->bt, c->st, c->d_bphi, c->d_perr, lvl(c, l), nlvl(c, l), s);
    launch_init_vcycle(c->geom, c->st, all(c), nall(c), s);
    TRY(launched(c, __LINE__));
    for (int l = maxlevel; l >= 0; l--) {
        launch_vdown(c->geom, c->bt, c->st, lvl(c, l), nlvl(c, l), c->d_vitems, c->d_vranges + 4 * c->off_vrange[l],
                     s);
        TRY(launched(c, __LINE__));
        TRY(rec_relax_until(c, s, l, 1.0, depth));
    }
    for (int l = 0; l <= maxlevel; l++) {
        if (l > 0) launch_coarse_correction(c->geom, c->bt, c->st, lvl(c, l), nlvl(c, l), s);
        TRY(launched(c, __LINE__));
        TRY(rec_relax_until(c, s, l, 0.05, depth));
        launch_retire(c->geom, c->st, lvl(c, l), nlvl(c, l), s);
        launch_phi_boundaries(c->geom, c->bt, c->st, c->d_bphi, c->d_perr, lvl(c, l), nlvl(c, l), s);
    }
    TRY(rec_forces(c, s));
    launch_error_dev(c->geom, c->bt, c->st, g->L, maxlevel + 1, tol, hsolve, g->d_ctl, c->d_pres, g->d_nest,
                     g->d_counter, s);
    return launched(c, __LINE__);
}

// The V-cycle loop as one persistent cooperative kernel (persistent.cu).
int rec_persistent(amr_ctx* c, cudaStream_t s, double tol) {
    GraphState* g = c->gs;
    SolveArgs a{};
    a.g = c->geom;
    a.bt = c->bt;
    a.st = c->st;
    a.L = g->L;
    a.aux = PoissonAux{c->d_bphi, c->d_perr};
    a.parents = c->d_slots;
    const int nlev = (int)c->level_slots.size();
    if (nlev > MAX_LEVELS || c->tree.prm.max_level + 1 > MAX_LEVELS) {
        c->err = "too many levels for the persistent solve";
        return AMR_ERR_ARG;
    }
    for (int l = 0; l < nlev; l++) {
        a.poff[l] = c->off_parent[l];
        a.pcnt[l] = (int)c->parent_slots[l].size();
        a.voff[l] = c->off_vrange[l];
    }
    a.fitems = c->d_reflux;
    a.force_levels = c->tree.prm.max_level + 1;
    for (int l = 0; l <= a.force_levels; l++) a.foff[l] = c->off_reflux[l];
    a.vitems = c->d_vitems;
    a.vranges = c->d_vranges;
    a.nlevels = max_level_present(c) + 1;
    a.tol = tol;
    a.ctl = g->d_ctl;
    a.pres = g->d_pres3;
    a.nest = g->d_pnest;
    a.snap = g->d_snap;
    a.stride = snap_stride(c);
    a.snap_half = snap_stride(c) * (size_t)c->cap;
    a.bar = g->d_bar;
    CUDA_TRY(cudaMemsetAsync(g->d_bar, 0, sizeof(GridBarrier), s));
    a.rpub = g->d_rpub;
    CUDA_TRY(cudaMemsetAsync(g->d_rpub, 0, sizeof(unsigned) * (size_t)c->cap, s));
    a.tsnap = g->d_tsnap;
    a.tpres = g->d_tpres;
    if (g->d_tsnap) {
        CUDA_TRY(cudaMemsetAsync(g->d_tsnap, 0, sizeof(unsigned long long) * 2 * snap_stride(c) * (size_t)c->cap, s));
        CUDA_TRY(cudaMemsetAsync(g->d_tpres, 0, sizeof(unsigned long long) * 4 * (size_t)c->cap, s));
    }
    // event nodes bracketing the launch: the elapsed time of the latest
    // replay is the kernel's duration on this stream
    CUDA_TRY(cudaEventRecordWithFlags(g->ev_ps[0], s, cudaEventRecordExternal));
    CUDA_TRY(launch_solve_persistent(a, g->pblocks, g->layout, s));
    CUDA_TRY(cudaEventRecordWithFlags(g->ev_ps[1], s, cudaEventRecordExternal));
    g->k_vbody = 0;
    g->k_rbody = 0;
    return launched(c, __LINE__);
}

// solve(): boundaries, forces, V-cycles while the L1 error > tol, restriction.
int rec_solve(amr_ctx* c, cudaStream_t s, double tol, int depth) {
    GraphState* g = c->gs;
    launch_set_source(c->geom, c->st, all(c), nall(c), s);
    launch_source_sums(c->geom, c->bt, c->st, all(c), nall(c), c->d_msrc, c->d_allref, s);
    if (launch_phys_bound(c->geom, c->bt, c->d_bfaces, c->n_bfaces, all(c), phys_walk(c), c->d_msrc, c->d_allref,
                          c->d_bphi, c->d_own, c->own_cap, s)) {
        c->err = "domain-face potential scratch too small";
        return AMR_ERR_STATE;
    }
    TRY(rec_forces(c, s));
    if (c->cfg.persistent_solve) {
        TRY(rec_persistent(c, s, tol));
    } else {
        TRY(add_while(
            c, s, depth,
            [&](cudaStream_t q, cudaGraphConditionalHandle h) {
                launch_open_loop(h, g->d_ctl, 1, q);
                return launched(c, __LINE__);
            },
            [&](cudaStream_t q, cudaGraphConditionalHandle h) { return rec_vcycle(c, q, depth + 1, h, tol); }));
    }
    if (is_ztwd(c)) {  // Binary's solve: pot_to_grid, then the ZTWD restriction
        launch_zt_pot(c->geom, c->bt, c->st, c->zpar, all(c), nall(c), 0, s);
        for (int l = c->tree.prm.max_level; l >= 0; l--)
            launch_zt_inject(c->geom, c->bt, c->st, c->zpar, c->d_slots + c->off_parent[l],
                             (int)c->parent_slots[l].size(), c->d_zerr, s);
    } else {
        for (int l = c->tree.prm.max_level; l >= 0; l--)
            launch_inject(c->geom, c->bt, c->st, c->d_slots + c->off_parent[l], (int)c->parent_slots[l].size(),
                          s);
    }
    return launched(c, __LINE__);
}

int rec_enforce_boundaries(amr_ctx* c, cudaStream_t s) {
    for (int l = 0; l <= c->tree.prm.max_level; l++)
        launch_ghost_fill(c->geom, c->bt, c->st, lvl(c, l), nlvl(c, l), s);
    return launched(c, __LINE__);
}

int maxslot(amr_ctx* c) {
    int m = 0;
    for (int sl : c->all_slots) m = std::max(m, sl + 1);
    return m;
}

// One RK3 step of the self-gravitating driver (binary_driver.cpp:346-459 on
// the Euler state) with the CFL step reduced on the device.
int rec_step(amr_ctx* c, cudaStream_t s, double tol) {
    GraphState* g = c->gs;
    double* dtp = &g->d_ctl->dt;
    launch_max_dt(c->geom, c->st, all(c), nall(c), c->bt.h, c->d_dt, s);
    launch_dt_reduce(c->bt, g->L, max_level_present(c) + 1, c->d_dt, g->d_nest, g->d_ctl, c->cfg.maxdtinc, s);
    CUDA_TRY(cudaMemcpyAsync(c->st.U0, c->st.U, sizeof(double) * (size_t)maxslot(c) * c->geom.ucount,
                             cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(c->d_fo + c->geom.nf, c->d_fo, sizeof(double) * c->geom.nf, cudaMemcpyDeviceToDevice, s));
    const double betas[3] = {1.0, 0.25, 2.0 / 3.0};
    for (int rk = 0; rk < 3; rk++) {
        TRY(rec_enforce_boundaries(c, s));
        launch_flux(c->geom, c->st, all(c), nall(c), s);
        for (int l = c->tree.prm.max_level; l >= 0; l--) {
            const int n = c->off_reflux[l + 1] - c->off_reflux[l];
            launch_reflux(c->geom, c->st, c->d_reflux + c->off_reflux[l], n, s);
        }
        launch_flow_off(c->geom, c->st, c->tree.root()->slot, c->tree.root()->h, 0.0, betas[rk], c->d_fo, s, dtp);
        launch_add_difs(c->geom, c->st, all(c), nall(c), c->bt.h, 0.0, betas[rk], 1, s, dtp);
        launch_phi_time(c->geom, c->st, all(c), nall(c), rk == 0 ? 0 : (rk == 1 ? 2 : 1), s);
        TRY(launched(c, __LINE__));
        TRY(rec_solve(c, s, tol, 0));
    }
    return rec_enforce_boundaries(c, s);
}

int capture(amr_ctx* c, const std::function<int(cudaStream_t)>& rec, cudaGraphExec_t* exec, long long* kernels) {
    if (*exec) {
        cudaGraphExecDestroy(*exec);
        *exec = nullptr;
    }
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    {
        const cudaError_t pre = cudaGetLastError();
        if (pre != cudaSuccess) {
            c->err = std::string("error pending before capture: ") + cudaGetErrorString(pre);
            return AMR_ERR_CUDA;
        }
    }
    CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
    GraphState* gs = c->gs;
    gs->rec_in_bodies = 0;
    gs->rec_nested = 0;
    gs->while_depth = 0;
    const long long t0 = g_launch_tally;
    const int rc = rec(c->stream);
    *kernels = g_launch_tally - t0 - gs->rec_in_bodies;
    cudaGraph_t graph;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (rc) {
        if (e == cudaSuccess) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) {
        c->err = std::string("capture failed: ") + cudaGetErrorString(e);
        return AMR_ERR_CUDA;
    }
    const cudaError_t ei = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
        c->err = std::string("graph instantiation failed: ") + cudaGetErrorString(ei);
        *exec = nullptr;
        return AMR_ERR_CUDA;
    }
    return AMR_OK;
}

int set_limits(amr_ctx* c, int max_cycles, int steps) {
    GraphState* g = c->gs;
    int* hs = g->h_steps;
    hs[0] = max_cycles;
    hs[1] = c->vcycle_max_outer;
    hs[2] = 0;
    hs[3] = steps;
    CUDA_TRY(cudaMemcpyAsync(&g->d_ctl->max_cycles, &hs[0], sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(&g->d_ctl->max_outer, &hs[1], sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(&g->d_ctl->status, &hs[2], sizeof(int), cudaMemcpyHostToDevice, c->stream));
    hs[4] = c->wait_limit;
    CUDA_TRY(cudaMemcpyAsync(&g->d_ctl->wait_limit, &hs[4], sizeof(int), cudaMemcpyHostToDevice, c->stream));
    if (steps >= 0)
        CUDA_TRY(cudaMemcpyAsync(&g->d_ctl->steps, &hs[3], sizeof(int), cudaMemcpyHostToDevice, c->stream));
    return AMR_OK;
}

int read_ctl(amr_ctx* c) {
    GraphState* g = c->gs;
    CUDA_TRY(cudaMemcpyAsync(g->h_ctl, g->d_ctl, sizeof(Control), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return AMR_OK;
}

// Kernels executed by the replay just read back: the graph's top-level
// kernels, one V-cycle body per V-cycle, one relaxation loop body per pass
// beyond the first of each loop (the first is part of the V-cycle body).
void count_replay(amr_ctx* c, long long top_kernels) {
    GraphState* g = c->gs;
    const long long dc = g->h_ctl->cycles_total - g->last_cycles;
    const long long dr = g->h_ctl->relax_calls - g->last_relax;
    const long long loops = dr - dc * 2LL * g->nlevels_captured;
    c->prof.kernels += top_kernels + dc * g->k_vbody + loops * g->k_rbody;
    c->relax_calls += dr;
    for (int l = 0; l < MAX_LEVELS; l++) {
        c->relax_level[l] += g->h_ctl->relax_level[l] - g->last_relax_level[l];
        g->last_relax_level[l] = g->h_ctl->relax_level[l];
    }
    g->last_cycles = g->h_ctl->cycles_total;
    g->last_relax = g->h_ctl->relax_calls;
}

int need(amr_ctx* c) {
    if (!c) return AMR_ERR_ARG;
    if (!c->has_device) return AMR_ERR_NODEVICE;
    if (!has_gravity(c)) {
        c->err = "graph solve needs a self-gravitating context";
        return AMR_ERR_ARG;
    }
    if (c->geom.nx != 8 && c->geom.nx != 12) {
        c->err = "graph step built for nx == 8 or 12";
        return AMR_ERR_ARG;
    }
    TRY(amr_poisson_set_source(c));  // allocates the Poisson scratch on first use
    TRY(ensure_state(c));
    return AMR_OK;
}

}  // namespace

namespace amr {
void graph_release(amr_ctx* c) {
    GraphState* g = c->gs;
    if (!g) return;
    if (g->step_exec) cudaGraphExecDestroy(g->step_exec);
    if (g->solve_exec) cudaGraphExecDestroy(g->solve_exec);
    for (cudaStream_t s : g->streams) cudaStreamDestroy(s);
    if (g->d_ctl) cudaFree(g->d_ctl);
    if (g->h_ctl) cudaFreeHost(g->h_ctl);
    if (g->h_steps) cudaFreeHost(g->h_steps);
    if (g->d_nest) cudaFree(g->d_nest);
    if (g->d_snap) cudaFree(g->d_snap);
    if (g->d_counter) cudaFree(g->d_counter);
    if (g->d_pres3) cudaFree(g->d_pres3);
    if (g->d_pnest) cudaFree(g->d_pnest);
    if (g->d_bar) cudaFree(g->d_bar);
    if (g->d_rpub) cudaFree(g->d_rpub);
    if (g->d_tsnap) cudaFree(g->d_tsnap);
    if (g->d_tpres) cudaFree(g->d_tpres);
    for (cudaEvent_t e : g->ev_ps)
        if (e) cudaEventDestroy(e);
    delete g;
    c->gs = nullptr;
}
}  // namespace amr

extern "C" {

// Device time per phase class of the persistent solve, accumulated over all
// persistent solves of the context (ms[PH_COUNT], counts[PH_COUNT]).
int amr_solve_phases(amr_ctx* c, double* ms, long long* counts, double* bytes, int n) {
    if (!c || !ms || !counts || !bytes || n < PH_COUNT) return AMR_ERR_ARG;
    if (!c->gs) {
        for (int p = 0; p < PH_COUNT; p++) ms[p] = 0.0, counts[p] = 0, bytes[p] = 0.0;
        return AMR_OK;
    }
    TRY(read_ctl(c));
    for (int p = 0; p < PH_COUNT; p++) {
        ms[p] = c->gs->h_ctl->phase_ns[p] * 1e-6;
        counts[p] = (long long)c->gs->h_ctl->phase_n[p];
        bytes[p] = c->gs->h_ctl->phase_bytes[p];
    }
    return AMR_OK;
}

// The barrier share of each phase class (wait_ms[PH_COUNT]) and the time of
// the relaxation level sums formed after a barrier (*level_sum_ms, over
// *level_sums of them), as block 0 of the persistent solve sees them.
int amr_solve_phase_waits(amr_ctx* c, double* wait_ms, int n, double* level_sum_ms, long long* level_sums) {
    if (!c || !wait_ms || !level_sum_ms || !level_sums || n < PH_COUNT) return AMR_ERR_ARG;
    if (!c->gs) {
        for (int p = 0; p < PH_COUNT; p++) wait_ms[p] = 0.0;
        *level_sum_ms = 0.0;
        *level_sums = 0;
        return AMR_OK;
    }
    TRY(read_ctl(c));
    for (int p = 0; p < PH_COUNT; p++) wait_ms[p] = c->gs->h_ctl->phase_wait_ns[p] * 1e-6;
    *level_sum_ms = c->gs->h_ctl->level_sum_ns * 1e-6;
    *level_sums = (long long)c->gs->h_ctl->level_sum_n;
    return AMR_OK;
}

// The shared-memory relaxation loops of the persistent solve as block 0
// sees them (its brick is in every level): ms[0..3] = waiting for the
// neighbours' passes, computing passes, waiting for the loop decision,
// publishing; the passes and the Jacobi sweeps block 0 computed.
int amr_solve_relax_split(amr_ctx* c, double* ms, long long* passes, long long* sweeps) {
    if (!c || !ms || !passes || !sweeps) return AMR_ERR_ARG;
    if (!c->gs) {
        for (int q = 0; q < 4; q++) ms[q] = 0.0;
        *passes = *sweeps = 0;
        return AMR_OK;
    }
    TRY(read_ctl(c));
    for (int q = 0; q < 4; q++) ms[q] = c->gs->h_ctl->relax_split_ns[q] * 1e-6;
    *passes = (long long)c->gs->h_ctl->relax_split_passes;
    *sweeps = (long long)c->gs->h_ctl->relax_split_sweeps;
    return AMR_OK;
}

// Block 0's time (ms) in the persistent solve's relaxation loops of each
// level since the context started; levels past n are not written.
int amr_solve_relax_level_ms(amr_ctx* c, double* ms, int n) {
    if (!c || !ms || n < 0) return AMR_ERR_ARG;
    if (c->gs) TRY(read_ctl(c));
    for (int l = 0; l < n; l++) ms[l] = c->gs && l < MAX_LEVELS ? c->gs->h_ctl->relax_level_ns[l] * 1e-6 : 0.0;
    return AMR_OK;
}

// Device time and number of the persistent solve launches made by
// amr_graph_solve (CUDA events around each launch on its stream).
int amr_solve_totals(amr_ctx* c, double* ms, long long* count) {
    if (!c || !ms || !count) return AMR_ERR_ARG;
    *ms = c->gs ? c->gs->ps_ms_total : 0.0;
    *count = c->gs ? c->gs->ps_count : 0;
    return AMR_OK;
}

// Polls per bounded wait of the persistent solve and of the fused substep
// before they give up with AMR_ERR_TIMEOUT; 0 restores the defaults (2^22
// and 2^24).
int amr_set_wait_limit(amr_ctx* c, int polls) {
    if (!c || polls < 0) return AMR_ERR_ARG;
    c->wait_limit = polls > 0 ? polls : (1 << 22);
    c->fused_wait_limit = polls > 0 ? polls : (1 << 24);
    return AMR_OK;
}

// Relaxation passes per level since the context started (every form:
// host-driven, captured graph, persistent solve).
static_assert(MAX_LEVELS == 16, "amr_ctx::relax_level holds 16 levels");
int amr_relax_passes(amr_ctx* c, long long* per_level, int n) {
    if (!c || !per_level || n < 0) return AMR_ERR_ARG;
    for (int l = 0; l < n; l++) per_level[l] = l < MAX_LEVELS ? c->relax_level[l] : 0;
    return AMR_OK;
}

// Duration of the most recent persistent solve launch (CUDA events recorded
// around it on the launching stream).
int amr_solve_last_ms(amr_ctx* c, float* ms) {
    if (!c || !ms) return AMR_ERR_ARG;
    if (!c->gs || !c->gs->ev_ps[0]) {
        c->err = "no persistent solve has run";
        return AMR_ERR_STATE;
    }
    CUDA_TRY(cudaEventSynchronize(c->gs->ev_ps[1]));
    CUDA_TRY(cudaEventElapsedTime(ms, c->gs->ev_ps[0], c->gs->ev_ps[1]));
    return AMR_OK;
}

// Block layout of the persistent solve kernel: layout (0 .. count-1 of the
// brick size's layouts) and blocks per SM (0: as many as fit).  Every layout
// gives the same results bit for bit; the captured graphs are re-captured
// with the new launch at their next call.
int amr_set_solve_layout(amr_ctx* c, int layout, int blocks_per_sm) {
    TRY(need(c));
    GraphState* g = c->gs;
    if (!c->cfg.persistent_solve) {
        c->err = "solve layouts belong to the persistent solve (amr_config.persistent_solve > 0)";
        return AMR_ERR_STATE;
    }
    if (layout < 0 || layout >= solve_layouts(c->geom.nx) || blocks_per_sm < 0) return AMR_ERR_ARG;
    const int nb = solve_persistent_blocks(c->geom.nx, c->geom.precision, blocks_per_sm, layout);
    if (nb <= 0 || nb > g->pnest_blocks) {
        c->err = "no cooperative launch configuration for this layout";
        return AMR_ERR_ARG;
    }
    g->layout = layout;
    g->per_sm = blocks_per_sm;
    g->pblocks = nb;
    g->solve_version = -1;
    g->step_version = -1;
    return AMR_OK;
}

int amr_get_solve_layout(amr_ctx* c, int* layout, int* blocks_per_sm, int* threads, int* blocks, int* count) {
    TRY(need(c));
    GraphState* g = c->gs;
    if (layout) *layout = g->layout;
    if (blocks_per_sm) *blocks_per_sm = g->per_sm;
    if (threads) *threads = solve_layout_threads(c->geom.nx, g->layout);
    if (blocks) *blocks = g->pblocks;
    if (count) *count = solve_layouts(c->geom.nx);
    return AMR_OK;
}

// Times one persistent solve (to L1 tolerance tol) from the context's
// current potential in every layout and blocks-per-SM cap (1, 2, as many as
// fit) of its brick size -- reps timed solves each after an untimed one,
// the potential restored before every solve -- keeps the fastest and leaves
// the potential as it was.  ms[t] receives the mean time of trial t
// (layout = t / 3, cap = 1, 2, 0 for t % 3; a negative value where the
// trial gives the same launch as an earlier one or has none); *ntrials the
// trials (3 per layout), *best the fastest.
int amr_autotune_solve(amr_ctx* c, double tol, int max_cycles, int reps, double* ms, int ms_cap, int* ntrials,
                       int* best) {
    TRY(need(c));
    GraphState* g = c->gs;
    if (!c->cfg.persistent_solve) {
        c->err = "the autotuner times the persistent solve (amr_config.persistent_solve > 0)";
        return AMR_ERR_STATE;
    }
    if (reps < 1 || max_cycles < 1) return AMR_ERR_ARG;
    const int nl = solve_layouts(c->geom.nx);
    const int caps[3] = {1, 2, 0};
    const int nt = 3 * nl;
    if (ntrials) *ntrials = nt;
    // the trials run whole solves, which write the Poisson arrays and, for
    // the ZTWD state, the potential field and the parents' covered cells of
    // the state: all of them are saved here and put back after every trial
    // and at the end, so tuning leaves the run's trajectory unchanged
    const size_t pbytes = sizeof(double) * (size_t)c->cap * c->geom.pnx3;
    const size_t ubytes = sizeof(double) * (size_t)c->cap * c->geom.ucount;
    double* arr[9] = {c->st.phi, c->st.phi0, c->st.dphi, c->st.dphi1, c->st.S, c->st.fx, c->st.fy, c->st.fz, c->st.U};
    double* saved = nullptr;
    CUDA_TRY(cudaMalloc(&saved, 8 * pbytes + ubytes));
    auto copy_all = [&](bool save) {
        for (int q = 0; q < 9; q++) {
            double* keep = saved + (size_t)q * (pbytes / sizeof(double));
            const size_t nb = q < 8 ? pbytes : ubytes;
            if (cudaMemcpyAsync(save ? keep : arr[q], save ? arr[q] : keep, nb, cudaMemcpyDeviceToDevice,
                                c->stream) != cudaSuccess)
                return false;
        }
        return true;
    };
    if (!copy_all(true)) {
        cudaFree(saved);
        c->err = "autotuner: saving the state failed";
        return AMR_ERR_CUDA;
    }
    const int l0 = g->layout, p0 = g->per_sm;
    double best_ms = 1e300;
    int best_t = -1;
    int rc = AMR_OK;
    std::vector<std::pair<int, int>> seen;  // (layout, blocks)
    for (int t = 0; t < nt && rc == AMR_OK; t++) {
        const int l = t / 3, cap = caps[t % 3];
        const int nb = solve_persistent_blocks(c->geom.nx, c->geom.precision, cap, l);
        double mean = -1.0;
        bool dup = nb <= 0 || nb > g->pnest_blocks;
        for (auto& q : seen) dup = dup || (q.first == l && q.second == nb);
        if (!dup) {
            seen.push_back({l, nb});
            rc = amr_set_solve_layout(c, l, cap);
            double sum = 0.0;
            for (int r = 0; r <= reps && rc == AMR_OK; r++) {
                if (!copy_all(false)) {
                    rc = AMR_ERR_CUDA;
                    break;
                }
                rc = amr_graph_solve(c, tol, max_cycles, nullptr, nullptr);
                float one = 0.0f;
                if (rc == AMR_OK) rc = amr_solve_last_ms(c, &one);
                if (r > 0) sum += one;
            }
            mean = sum / reps;
            if (rc == AMR_OK && mean < best_ms) {
                best_ms = mean;
                best_t = t;
            }
        }
        if (ms && t < ms_cap) ms[t] = mean;
    }
    if (!copy_all(false) && rc == AMR_OK) rc = AMR_ERR_CUDA;
    cudaStreamSynchronize(c->stream);
    cudaFree(saved);
    if (rc != AMR_OK) {
        amr_set_solve_layout(c, l0, p0);
        return rc;
    }
    if (best) *best = best_t;
    return amr_set_solve_layout(c, best_t / 3, caps[best_t % 3]);
}

// The Poisson solve as one graph launch (see amr_poisson_solve).
int amr_graph_solve(amr_ctx* c, double tol, int max_cycles, double* l1_error, int* cycles) {
    TRY(need(c));
    GraphState* g = c->gs;
    if (!g->solve_exec || g->solve_version != c->topo_version || g->solve_tol != tol) {
        fill_lists(c);
        TRY(capture(c, [&](cudaStream_t s) { return rec_solve(c, s, tol, 0); }, &g->solve_exec, &g->k_solve));
        g->solve_version = c->topo_version;
        g->solve_tol = tol;
        g->nlevels_captured = max_level_present(c) + 1;
    }
    TRY(set_limits(c, max_cycles, -1));
    CUDA_TRY(cudaGraphLaunch(g->solve_exec, c->stream));
    TRY(read_ctl(c));
    count_replay(c, g->k_solve);
    if (c->cfg.persistent_solve > 0) {
        float ms = 0.0f;
        CUDA_TRY(cudaEventElapsedTime(&ms, g->ev_ps[0], g->ev_ps[1]));
        g->ps_ms_total += ms;
        g->ps_count++;
    }
    if (l1_error) *l1_error = g->h_ctl->err;
    if (cycles) *cycles = g->h_ctl->cycles;
    if (g->h_ctl->status == 3) {
        c->err = "persistent solve: a grid barrier timed out";
        return AMR_ERR_TIMEOUT;
    }
    if (g->h_ctl->status) {
        c->err = g->h_ctl->status == 2 ? "Poisson solve exceeded max_cycles" : "relaxation loop exceeded its cap";
        return AMR_ERR_NOCONVERGE;
    }
    return AMR_OK;
}

// amr_grav_step with the whole RK3 step replayed from a captured graph and
// the CFL step (GridNode::max_dt + MAXDTINC clamp against the previous
// graph step) formed on the device.  step_index 0 starts the clamp afresh.
int amr_graph_grav_step(amr_ctx* c, double tol, double dynamic_range, int step_index, double* dt_out) {
    TRY(need(c));
    if (c->cfg.physics != AMR_PHYSICS_EULER_GRAVITY) {
        c->err = "graph step needs AMR_PHYSICS_EULER_GRAVITY";
        return AMR_ERR_ARG;
    }
    GraphState* g = c->gs;
    const int max_cycles = 10000;
    if (step_index <= 0) {
        TRY(amr_graph_solve(c, tol, max_cycles, nullptr, nullptr));
        TRY(amr_store_phi(c));
    }
    if (!g->step_exec || g->step_version != c->topo_version || g->step_tol != tol) {
        fill_lists(c);
        TRY(capture(c, [&](cudaStream_t s) { return rec_step(c, s, tol); }, &g->step_exec, &g->k_step));
        g->step_version = c->topo_version;
        g->step_tol = tol;
        g->nlevels_captured = max_level_present(c) + 1;
    }
    TRY(set_limits(c, max_cycles, step_index <= 0 ? 0 : -1));
    CUDA_TRY(cudaGraphLaunch(g->step_exec, c->stream));
    TRY(read_ctl(c));
    count_replay(c, g->k_step);
    if (g->h_ctl->status == 3) {
        c->err = "persistent solve: a grid barrier timed out";
        return AMR_ERR_TIMEOUT;
    }
    if (g->h_ctl->status) {
        c->err = "solve inside the captured step did not converge";
        return AMR_ERR_NOCONVERGE;
    }
    const double dt = g->h_ctl->dt;
    for (Node* n : c->order) n->age += 3;  // three add_difs calls
    if (step_index % 8 == 0) {
        double smax;
        TRY(amr_state_max(c, 0, &smax));
        int changed = 0;
        TRY(amr_check_for_refine(c, smax / dynamic_range, 1, &changed));
        if (changed) {
            TRY(amr_graph_solve(c, tol / 10.0, max_cycles, nullptr, nullptr));
            TRY(amr_store_phi(c));
        }
    }
    TRY(amr_set_time(c, c->time + dt));
    if (dt_out) *dt_out = dt;
    return AMR_OK;
}

}  // extern "C"
