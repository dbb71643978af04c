// Per-tree context: host octree, device brick pool and brick table.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "amr_internal.h"
#include "octree.h"
#include "profiler.h"
#include "ztwd.h"

struct amr_ctx {
    amr_config cfg{};
    amr::Geom geom{};
    amr::Octree tree;
    std::string err;
    double time = 0.0;
    bool has_device = false;
    cudaStream_t stream = nullptr;

    // device pool
    int cap = 0;
    amr::DevState st{};
    amr::BrickTable bt{};
    double* d_fo = nullptr;      // FO[nf], FO0[nf] of the root
    double* d_dt = nullptr;      // per-slot dt / scratch [cap]
    double* d_red = nullptr;     // per-entry reduction scratch [cap]
    unsigned char* d_flags = nullptr;  // [8*cap]
    double* d_stage = nullptr;   // host<->device staging [stage_cap]
    size_t stage_cap = 0;

    // host mirror of the brick table
    std::vector<int> h_level, h_off, h_ftype, h_fnbr, h_parent, h_cidx, h_child;
    std::vector<double> h_h;
    std::vector<int> free_slots;

    // derived topology (rebuilt after every tree change)
    std::vector<amr::Node*> order;              // DFS pre-order
    std::vector<int> all_slots;                 // slots in DFS order
    std::vector<std::vector<int>> level_slots;  // per level, DFS order
    std::vector<std::vector<int>> parent_slots; // per level: bricks with >=1 child
    std::vector<std::vector<amr::RefluxItem>> reflux;  // per coarse level
    int* d_slots = nullptr;                     // all_slots | level lists | parent lists
    std::vector<int> off_all, off_level, off_parent;
    amr::RefluxItem* d_reflux = nullptr;
    std::vector<int> off_reflux;
    int d_slots_cap = 0, d_reflux_cap = 0;
    std::vector<amr::Node*> pending_new;
    int reflux_hazards = 0;

    // Poisson
    double* d_bphi = nullptr;   // [cap][6][pnx][pnx] domain-face potential tables
    double* d_msrc = nullptr;   // [n][8][4] octant monopoles per DFS entry
    int* d_allref = nullptr;    // [n] node fully covered by children
    double* d_pres = nullptr;   // [cap] per-brick relax residual / L1 error
    int* d_bfaces = nullptr;    // [nbf][2] (slot, face) of physical (non-mirror) faces
    int* d_perr = nullptr;      // device error word (bad mirror index)
    int n_bfaces = 0, msrc_cap = 0, bfaces_cap = 0;
    double* d_own = nullptr;    // (point, subtree) partial sums of the domain-face potential
    size_t own_cap = 0;
    int* d_pwalk = nullptr;     // subtree ranges [nseg][2] | top-level walk [ntop]
    int pwalk_cap = 0, n_pseg = 0, n_ptop = 0;
    std::vector<int> off_reflux_dir;  // [(maxl+1)*3+1] items sorted by (level, dir)
    // the same items grouped by coarse brick for the fused V-cycle down
    // sweep: d_vitems in level-list order, x then y then z per brick;
    // d_vranges[4 (off_vrange[l] + q) + 0..3] = first x, y, z item, end
    amr::RefluxItem* d_vitems = nullptr;
    int* d_vranges = nullptr;
    // [8 e + c]: list position of child c of level-list entry e (-1: none)
    int* d_cpos = nullptr;
    int cpos_cap = 0, max_level_cnt = 0;
    // fused hydro substep: second state array, work list finest level first,
    // publish masks and buffer, done stamps, counters
    double* d_U1 = nullptr;
    int2* d_fwork = nullptr;
    unsigned char* d_pubmask = nullptr;
    double* d_pub = nullptr;
    int* d_fdone = nullptr;
    unsigned int* d_fctl = nullptr;  // [0] work counter, [1] error word
    int fwork_cap = 0, nfwork = 0, fused_epoch = 0, fused_blocks = 0;
    long long fused_version = -1;  // topology the work list was built for
    int vitems_cap = 0, vranges_cap = 0;
    std::vector<int> off_vrange;
    int vcycle_max_outer = 1000;
    long long relax_calls = 0, relax_sweeps_total = 0;
    long long relax_level[16] = {};  // relaxation passes per level
    int wait_limit = 1 << 22;        // polls per bounded wait of the persistent solve
    int fused_wait_limit = 1 << 24;  // polls per wait of the fused substep for a child's faces
    double chk_refine_alpha = 1.0;   // GridNode::refine_alpha of the last checkpoint read
    bool topo_dirty = true;
    long long topo_version = 0;  // bumped by every rebuild_topology
    // ZTWD state: frame + EOS passed to its kernels, EOS-failure word
    amr::ZtwdPar zpar{};
    bool zt_eos = false;
    int* d_zerr = nullptr;
    int zt_first_solve = 1;  // BinaryDriver::solve's first_call (binary_driver.cpp:297-301)
    amr::Profiler prof;
    struct GraphState* gs = nullptr;  // captured step/solve graphs (graph_host.cpp)

    amr_ctx(const amr::TreeParams& p) : tree(p) {}
};

namespace amr {
inline bool is_ztwd(const amr_ctx* c) { return c->cfg.physics == AMR_PHYSICS_ZTWD; }
inline bool has_gravity(const amr_ctx* c) {
    return c->cfg.physics == AMR_PHYSICS_EULER_GRAVITY || c->cfg.physics == AMR_PHYSICS_ZTWD;
}
int zt_ready(amr_ctx* c);  // ZTWD context has its EOS (ztwd_host.cpp)
int zt_check(amr_ctx* c);  // reads and clears the EOS-failure word
int rebuild_topology(amr_ctx* c);
int alloc_slot(amr_ctx* c);
void graph_release(amr_ctx* c);
// the staging buffer of the host copies holds at least `count` doubles
int stage_reserve(amr_ctx* c, size_t count);
}  // namespace amr
