// Host side of the C ABI: context, brick pool, topology tables and the
// reference's driver sequences.  Every numerical operation is a CUDA kernel
// (kernels.h); the host only orchestrates and keeps the octree.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>

#include "context.h"
#include "profiler.h"
#include "kernels.h"
#include "poisson.h"
#include "hydro_fused.h"

using namespace amr;

thread_local long long amr::g_launch_tally = 0;

#define CUDA_TRY(call)                                                                                  \
    do {                                                                                                \
        cudaError_t e__ = (call);                                                                       \
        if (e__ != cudaSuccess) {                                                                       \
            c->err = std::string("CUDA error: ") + cudaGetErrorString(e__) + " at " + #call;           \
            return AMR_ERR_CUDA;                                                                        \
        }                                                                                               \
    } while (0)

#define NEED_DEVICE(c)                                                                   \
    do {                                                                                 \
        if (!(c)) return AMR_ERR_ARG;                                                    \
        if (!(c)->has_device) {                                                          \
            (c)->err = "context has no device pool (created with max_bricks == 0)";      \
            return AMR_ERR_NODEVICE;                                                     \
        }                                                                                \
    } while (0)

#define TRY(x)               \
    do {                     \
        int rc__ = (x);      \
        if (rc__) return rc__; \
    } while (0)

namespace {

int check_launch(amr_ctx* c) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        c->err = std::string("CUDA launch error: ") + cudaGetErrorString(e);
        return AMR_ERR_CUDA;
    }
    return AMR_OK;
}

const int* dslots_all(amr_ctx* c) { return c->d_slots + c->off_all[0]; }
const int* dslots_level(amr_ctx* c, int l) { return c->d_slots + c->off_level[l]; }
const int* dslots_parent(amr_ctx* c, int l) { return c->d_slots + c->off_parent[l]; }

}  // namespace

namespace amr {

int alloc_slot(amr_ctx* c) {
    if (!c->has_device) return (int)c->tree.count();  // host-only: slots are bookkeeping only
    if (c->free_slots.empty()) return -1;
    const int s = c->free_slots.back();
    c->free_slots.pop_back();
    return s;
}

// Rebuild the derived topology after a tree change: DFS order, per-slot
// brick table, per-level lists, coarse-fine correction items; upload.
int rebuild_topology(amr_ctx* c) {
    Octree& T = c->tree;
    c->order = T.dfs_order();
    const int n = (int)c->order.size();
    for (int i = 0; i < n; i++) c->order[i]->dfs = i;
    const int maxl = T.prm.max_level;
    c->all_slots.resize(n);
    c->level_slots.assign(maxl + 1, {});
    c->parent_slots.assign(maxl + 1, {});
    c->reflux.assign(maxl + 1, {});
    const int bw = c->geom.bw, gnx = c->geom.gnx;
    for (int i = 0; i < n; i++) {
        Node* nd = c->order[i];
        const int s = nd->slot;
        c->all_slots[i] = s;
        if (nd->level <= maxl) c->level_slots[nd->level].push_back(s);
        if (nd->nchildren() > 0 && nd->level <= maxl) c->parent_slots[nd->level].push_back(s);
        if (!c->has_device) continue;
        c->h_level[s] = nd->level;
        for (int d = 0; d < 3; d++) c->h_off[3 * s + d] = nd->off[d];
        c->h_h[s] = nd->h;
        c->h_parent[s] = nd->parent ? nd->parent->slot : -1;
        c->h_cidx[s] = nd->cidx;
        for (int ch = 0; ch < 8; ch++) c->h_child[8 * s + ch] = nd->child[ch] ? nd->child[ch]->slot : -1;
        for (int f = 0; f < 6; f++) {
            int kind, nbr = -1;
            if (T.is_phys_bound(nd, f)) {
                kind = (c->cfg.z_reflect && f == ZL) ? FACE_REFLECT : FACE_OUTFLOW;
            } else if (Node* sn = T.same_level_neighbor(nd, f)) {
                kind = FACE_SIB;
                nbr = sn->slot;
            } else {
                kind = FACE_AMR;
                nbr = nd->parent ? nd->parent->slot : -1;
            }
            c->h_ftype[6 * s + f] = kind;
            c->h_fnbr[6 * s + f] = nbr;
        }
    }
    // Coarse-fine correction items, GridNode::adjust_{x,y,z}_flux
    // (grid_node.cpp:1076-1274): for each brick P, direction, the three
    // face planes l = 0 (P's lower face), 1 (P's middle), 2 (P's upper face)
    // and the four transverse quadrants; correct when exactly one side has a
    // child brick touching the face.
    c->reflux_hazards = 0;
    for (int i = 0; i < n; i++) {
        Node* P = c->order[i];
        if (P->level > maxl) continue;
        for (int dir = 0; dir < 3; dir++) {
            const int lo_face = 2 * dir, hi_face = 2 * dir + 1;
            Node* nlo = T.same_level_neighbor(P, lo_face);
            Node* nhi = T.same_level_neighbor(P, hi_face);
            for (int l = 0; l < 3; l++)
                for (int ck = 0; ck < 2; ck++)
                    for (int cj = 0; cj < 2; cj++) {
                        // transverse bits: lower transverse axis <- cj, higher <- ck
                        const int ta = dir == 0 ? 1 : 0, tb = dir == 2 ? 1 : 2;
                        const int base = (cj << ta) | (ck << tb);
                        const int c0 = base, c1 = base | (1 << dir);
                        Node *cl = nullptr, *cr = nullptr;
                        int i0;
                        if (l == 0) {
                            cr = P->child[c0];
                            cl = nlo ? nlo->child[c1] : nullptr;
                            i0 = bw;
                        } else if (l == 1) {
                            cl = P->child[c0];
                            cr = P->child[c1];
                            i0 = gnx / 2;
                        } else {
                            cr = nhi ? nhi->child[c0] : nullptr;
                            cl = P->child[c1];
                            i0 = gnx - bw;
                        }
                        Node* ch = nullptr;
                        int ic = 0;
                        if (!cr && cl) {
                            ch = cl;
                            ic = gnx - bw;
                        } else if (!cl && cr) {
                            ch = cr;
                            ic = bw;
                        }
                        if (!ch) continue;
                        RefluxItem it{P->slot, ch->slot, dir, i0, ic, cj, ck, 0};
                        c->reflux[P->level].push_back(it);
                        // The reference corrects in depth-first order; a child
                        // owned by a later-visited neighbour whose own face is
                        // still to be corrected would be read uncorrected there.
                        // Under proper nesting that face never has children.
                        if (ch->parent != P && ch->dfs > P->dfs) {
                            const int f = (ic == bw) ? lo_face : hi_face;
                            for (int q = 0; q < 8; q++)
                                if (ch->child[q] && (((q >> dir) & 1) == (f & 1))) c->reflux_hazards++;
                        }
                    }
        }
    }
    if (!c->has_device) {
        c->topo_dirty = false;
        return AMR_OK;
    }
    // pack slot lists: all | level 0..maxl | parents 0..maxl
    std::vector<int> packed;
    c->off_all.assign(1, 0);
    packed.insert(packed.end(), c->all_slots.begin(), c->all_slots.end());
    c->off_level.assign(maxl + 1, 0);
    for (int l = 0; l <= maxl; l++) {
        c->off_level[l] = (int)packed.size();
        packed.insert(packed.end(), c->level_slots[l].begin(), c->level_slots[l].end());
    }
    c->off_parent.assign(maxl + 1, 0);
    for (int l = 0; l <= maxl; l++) {
        c->off_parent[l] = (int)packed.size();
        packed.insert(packed.end(), c->parent_slots[l].begin(), c->parent_slots[l].end());
    }
    if ((int)packed.size() > c->d_slots_cap) {
        if (c->d_slots) cudaFree(c->d_slots);
        c->d_slots_cap = (int)packed.size() * 2 + 64;
        CUDA_TRY(cudaMalloc(&c->d_slots, sizeof(int) * c->d_slots_cap));
    }
    CUDA_TRY(cudaMemcpyAsync(c->d_slots, packed.data(), sizeof(int) * packed.size(), cudaMemcpyHostToDevice,
                             c->stream));
    // items grouped by (coarse level, direction): the hydro reflux runs a
    // whole level at once; the Poisson dphi corrections must apply x, y, z
    // in turn (adjust_x_dphi .. adjust_z_dphi, poisson.cpp:989-1046)
    std::vector<RefluxItem> items;
    c->off_reflux.assign(maxl + 2, 0);
    c->off_reflux_dir.assign(3 * (maxl + 1) + 1, 0);
    for (int l = 0; l <= maxl; l++) {
        c->off_reflux[l] = (int)items.size();
        for (int dir = 0; dir < 3; dir++) {
            c->off_reflux_dir[3 * l + dir] = (int)items.size();
            for (const RefluxItem& it : c->reflux[l])
                if (it.dir == dir) items.push_back(it);
        }
    }
    c->off_reflux[maxl + 1] = (int)items.size();
    c->off_reflux_dir[3 * (maxl + 1)] = (int)items.size();
    // physical (non-mirror) domain faces for the multipole boundary tables
    {
        std::vector<int> bf;
        for (int i = 0; i < n; i++) {
            Node* nd = c->order[i];
            for (int f = 0; f < 6; f++)
                if (c->h_ftype[6 * nd->slot + f] == FACE_OUTFLOW) {
                    bf.push_back(nd->slot);
                    bf.push_back(f);
                }
        }
        c->n_bfaces = (int)bf.size() / 2;
        if (has_gravity(c)) {
            if ((int)bf.size() > c->bfaces_cap) {
                if (c->d_bfaces) cudaFree(c->d_bfaces);
                c->bfaces_cap = (int)bf.size() * 2 + 64;
                CUDA_TRY(cudaMalloc(&c->d_bfaces, sizeof(int) * c->bfaces_cap));
            }
            if (!bf.empty())
                CUDA_TRY(cudaMemcpyAsync(c->d_bfaces, bf.data(), sizeof(int) * bf.size(), cudaMemcpyHostToDevice,
                                         c->stream));
            if (n > c->msrc_cap) {
                if (c->d_msrc) cudaFree(c->d_msrc);
                if (c->d_allref) cudaFree(c->d_allref);
                c->msrc_cap = n * 2 + 64;
                CUDA_TRY(cudaMalloc(&c->d_msrc, sizeof(double) * 32 * c->msrc_cap));
                CUDA_TRY(cudaMalloc(&c->d_allref, sizeof(int) * c->msrc_cap));
            }
            // walk program of the domain-face potential: subtrees of at most
            // ~sqrt(n) bricks summed in parallel, then the walk above them
            std::vector<int> lv(n), segs, top;
            for (int i = 0; i < n; i++) lv[i] = c->order[i]->level;
            const int limit = std::max(4, (int)std::ceil(std::sqrt((double)n)));
            build_phys_walk(lv.data(), n, limit, segs, top);
            c->n_pseg = (int)segs.size() / 2;
            c->n_ptop = (int)top.size();
            std::vector<int> walk(segs);
            walk.insert(walk.end(), top.begin(), top.end());
            if ((int)walk.size() > c->pwalk_cap) {
                if (c->d_pwalk) cudaFree(c->d_pwalk);
                c->pwalk_cap = (int)walk.size() * 2 + 64;
                CUDA_TRY(cudaMalloc(&c->d_pwalk, sizeof(int) * c->pwalk_cap));
            }
            if (!walk.empty())
                CUDA_TRY(cudaMemcpyAsync(c->d_pwalk, walk.data(), sizeof(int) * walk.size(), cudaMemcpyHostToDevice,
                                         c->stream));
            // (subtree, point) scratch: all points at once up to 32 Mi
            // doubles, batched beyond
            const size_t per = (size_t)std::max(c->n_pseg, 1);
            const size_t need = (size_t)c->n_bfaces * c->geom.pnx * c->geom.pnx * per;
            const size_t want = std::min<size_t>(std::max<size_t>(need, per), (size_t)32 << 20);
            if (want > c->own_cap) {
                if (c->d_own) cudaFree(c->d_own);
                c->own_cap = want;
                CUDA_TRY(cudaMalloc(&c->d_own, sizeof(double) * c->own_cap));
            }
        }
    }
    // child positions within the next level's list, for the level sums
    {
        std::vector<int> pos(c->cap > 0 ? c->cap : 1, -1), cp;
        c->max_level_cnt = 0;
        for (int l = 0; l <= maxl; l++) {
            const std::vector<int>& ls = c->level_slots[l];
            c->max_level_cnt = std::max(c->max_level_cnt, (int)ls.size());
            for (int q = 0; q < (int)ls.size(); q++) pos[ls[q]] = q;
        }
        for (int l = 0; l <= maxl; l++)
            for (int s : c->level_slots[l])
                for (int q = 0; q < 8; q++) {
                    const int ch = c->h_child[8 * s + q];
                    cp.push_back(ch >= 0 ? pos[ch] : -1);
                }
        if ((int)cp.size() > c->cpos_cap) {
            if (c->d_cpos) cudaFree(c->d_cpos);
            c->cpos_cap = (int)cp.size() * 2 + 64;
            CUDA_TRY(cudaMalloc(&c->d_cpos, sizeof(int) * c->cpos_cap));
        }
        if (!cp.empty())
            CUDA_TRY(cudaMemcpyAsync(c->d_cpos, cp.data(), sizeof(int) * cp.size(), cudaMemcpyHostToDevice,
                                     c->stream));
    }
    // per coarse brick, in level-list order: its x, then y, then z items
    {
        std::vector<RefluxItem> vitems;
        std::vector<int> vr;
        c->off_vrange.assign(maxl + 1, 0);
        std::vector<int> pos(c->cap > 0 ? c->cap : 1, -1);
        for (int l = 0; l <= maxl; l++) {
            c->off_vrange[l] = (int)vr.size() / 4;
            const std::vector<int>& ls = c->level_slots[l];
            for (int q = 0; q < (int)ls.size(); q++) pos[ls[q]] = q;
            std::vector<std::vector<RefluxItem>> by(ls.size() * 3);
            for (const RefluxItem& it : c->reflux[l]) by[3 * pos[it.coarse] + it.dir].push_back(it);
            for (int q = 0; q < (int)ls.size(); q++) {
                for (int d = 0; d < 3; d++) {
                    vr.push_back((int)vitems.size());
                    vitems.insert(vitems.end(), by[3 * q + d].begin(), by[3 * q + d].end());
                }
                vr.push_back((int)vitems.size());
            }
        }
        if ((int)vitems.size() > c->vitems_cap) {
            if (c->d_vitems) cudaFree(c->d_vitems);
            c->vitems_cap = (int)vitems.size() * 2 + 64;
            CUDA_TRY(cudaMalloc(&c->d_vitems, sizeof(RefluxItem) * c->vitems_cap));
        }
        if ((int)vr.size() > c->vranges_cap) {
            if (c->d_vranges) cudaFree(c->d_vranges);
            c->vranges_cap = (int)vr.size() * 2 + 64;
            CUDA_TRY(cudaMalloc(&c->d_vranges, sizeof(int) * c->vranges_cap));
        }
        if (!vitems.empty())
            CUDA_TRY(cudaMemcpyAsync(c->d_vitems, vitems.data(), sizeof(RefluxItem) * vitems.size(),
                                     cudaMemcpyHostToDevice, c->stream));
        if (!vr.empty())
            CUDA_TRY(cudaMemcpyAsync(c->d_vranges, vr.data(), sizeof(int) * vr.size(), cudaMemcpyHostToDevice,
                                     c->stream));
    }
    if ((int)items.size() > c->d_reflux_cap) {
        if (c->d_reflux) cudaFree(c->d_reflux);
        c->d_reflux_cap = (int)items.size() * 2 + 64;
        CUDA_TRY(cudaMalloc(&c->d_reflux, sizeof(RefluxItem) * c->d_reflux_cap));
    }
    if (!items.empty())
        CUDA_TRY(cudaMemcpyAsync(c->d_reflux, items.data(), sizeof(RefluxItem) * items.size(),
                                 cudaMemcpyHostToDevice, c->stream));
    // brick table: upload the used slot range
    int maxslot = 0;
    for (int s : c->all_slots) maxslot = std::max(maxslot, s + 1);
    const int m = maxslot;
    CUDA_TRY(cudaMemcpyAsync(c->bt.level, c->h_level.data(), sizeof(int) * m, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->bt.off, c->h_off.data(), sizeof(int) * 3 * m, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->bt.h, c->h_h.data(), sizeof(double) * m, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->bt.ftype, c->h_ftype.data(), sizeof(int) * 6 * m, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->bt.fnbr, c->h_fnbr.data(), sizeof(int) * 6 * m, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->bt.parent, c->h_parent.data(), sizeof(int) * m, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->bt.cidx, c->h_cidx.data(), sizeof(int) * m, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->bt.child, c->h_child.data(), sizeof(int) * 8 * m, cudaMemcpyHostToDevice, c->stream));
    // host vectors may be rewritten before the async copies finish
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->topo_dirty = false;
    c->topo_version++;  // captured graphs embed the slot lists: rebuild them
    return AMR_OK;
}

}  // namespace amr

namespace {

// Prolongation of the bricks created by the last refinement pass.
int finish_refine(amr_ctx* c) {
    TRY(rebuild_topology(c));
    if (!c->has_device || c->pending_new.empty()) {
        c->pending_new.clear();
        return AMR_OK;
    }
    std::vector<int> slots;
    for (Node* nd : c->pending_new)
        if (nd->parent) slots.push_back(nd->slot);
    c->pending_new.clear();
    if (slots.empty()) return AMR_OK;
    int* d;
    CUDA_TRY(cudaMalloc(&d, sizeof(int) * slots.size()));
    CUDA_TRY(cudaMemcpyAsync(d, slots.data(), sizeof(int) * slots.size(), cudaMemcpyHostToDevice, c->stream));
    {
        ProfScope ps_(c->prof, KC_PROLONG, c->stream);
        if (is_ztwd(c))
            launch_zt_prolong(c->geom, c->bt, c->st, c->zpar, d, (int)slots.size(), c->d_zerr, c->stream);
        else
            launch_prolong(c->geom, c->bt, c->st, d, (int)slots.size(), c->stream);
    }
    if (has_gravity(c))
        launch_poisson_new_bricks(c->geom, c->bt, c->st, d, (int)slots.size(), c->stream);
    if (is_ztwd(c))  // Binary::inject_from_parent: then pot_from_grid (binary.cpp:852-855)
        launch_zt_pot(c->geom, c->bt, c->st, c->zpar, d, (int)slots.size(), 1, c->stream);
    TRY(check_launch(c));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    cudaFree(d);
    return AMR_OK;
}

void install_callbacks(amr_ctx* c) {
    c->tree.on_create = [c](Node* n) {
        n->slot = alloc_slot(c);
        c->pending_new.push_back(n);
    };
    c->tree.on_destroy = [c](Node* n) {
        if (c->has_device && n->slot >= 0) c->free_slots.push_back(n->slot);
        auto it = std::find(c->pending_new.begin(), c->pending_new.end(), n);
        if (it != c->pending_new.end()) c->pending_new.erase(it);
    };
}

template <class T>
int dev_alloc(amr_ctx* c, T** p, size_t count) {
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(count, 1));
    if (e != cudaSuccess) {
        c->err = std::string("cudaMalloc failed: ") + cudaGetErrorString(e);
        return AMR_ERR_CUDA;
    }
    e = cudaMemsetAsync(*p, 0, sizeof(T) * std::max<size_t>(count, 1), c->stream);
    if (e != cudaSuccess) {
        c->err = std::string("cudaMemset failed: ") + cudaGetErrorString(e);
        return AMR_ERR_CUDA;
    }
    return AMR_OK;
}

// The staging buffer of the host copies (gather / scatter of the bricks'
// arrays), sized on first use for the whole brick pool (its largest user,
// the state of every slot): a tree that grows later never makes a copy
// reallocate it, which cost from 5 ms to half a second per call (the free
// and allocation of a few hundred MB) on the copy after a regrid.
int ensure_stage(amr_ctx* c, size_t count) {
    if (count <= c->stage_cap) return AMR_OK;
    if (c->d_stage) cudaFree(c->d_stage);
    c->d_stage = nullptr;
    c->stage_cap = std::max(count, (size_t)c->cap * (size_t)std::max(c->geom.ucount, c->geom.pnx3));
    return dev_alloc(c, &c->d_stage, c->stage_cap);
}

int check_slots(amr_ctx* c) {
    for (Node* nd : c->order)
        if (nd->slot < 0) {
            c->err = "brick pool exhausted: raise amr_config.max_bricks";
            return AMR_ERR_CAPACITY;
        }
    return AMR_OK;
}

}  // namespace

namespace amr {
int stage_reserve(amr_ctx* c, size_t count) { return ensure_stage(c, count); }
}  // namespace amr

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int amr_default_config(amr_config* cfg) {
    if (!cfg) return AMR_ERR_ARG;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->bw = 2;
    cfg->nx = 8;
    cfg->nf = 6;
    cfg->physics = AMR_PHYSICS_EULER;
    cfg->precision = AMR_PREC_FP64;
    cfg->z_reflect = 1;
    cfg->mirror_refine_y = 1;
    cfg->max_refine_level = 4;
    cfg->min_level = 1;
    cfg->min_grid_life = 3 * 8;
    cfg->max_bricks = 4096;
    cfg->grid_dim = 1.0;
    cfg->minmod_theta = 1.3;
    cfg->cfl = 0.4;
    cfg->gamma = 5.0 / 3.0;
    cfg->rho_floor = 1.0e-20;
    cfg->ei_floor = 1.0e-20;
    cfg->maxdtinc = 1.25;
    cfg->grav_g = 1.0;
    return AMR_OK;
}

int amr_create(const amr_config* cfg, amr_ctx** out) {
    if (!cfg || !out) return AMR_ERR_ARG;
    *out = nullptr;
    // minmod reads cells f-2..f+1 of face f (bw >= 2), PPM cells f-3..f+2 (bw >= 3)
    const int min_bw = cfg->reconstruction == AMR_RECON_PPM ? 3 : 2;
    const bool ztwd = cfg->physics == AMR_PHYSICS_ZTWD;
    if (cfg->physics < AMR_PHYSICS_EULER || cfg->physics > AMR_PHYSICS_ZTWD ||
        (ztwd && (cfg->reconstruction != AMR_RECON_PPM || (cfg->nx != 8 && cfg->nx != 12))))
        return AMR_ERR_ARG;
    if (cfg->precision < AMR_PREC_FP64 || cfg->precision > AMR_PREC_MIXED_SOLVE) return AMR_ERR_ARG;
    if (cfg->nf != (ztwd ? (int)ZTWD_NF : 6) || cfg->bw < min_bw || cfg->bw > 4 || cfg->nx < 4 || (cfg->nx % 4) != 0 ||
        cfg->max_refine_level < 0 || cfg->max_refine_level > 12 || cfg->max_bricks < 0 ||
        (cfg->reconstruction != AMR_RECON_MINMOD && cfg->reconstruction != AMR_RECON_PPM))
        return AMR_ERR_ARG;
    TreeParams tp;
    tp.bw = cfg->bw;
    tp.nx = cfg->nx;
    tp.max_level = cfg->max_refine_level;
    tp.min_level = cfg->min_level;
    tp.min_grid_life = cfg->min_grid_life;
    tp.mirror_y = cfg->mirror_refine_y;
    tp.h0 = 2.0 * cfg->grid_dim / double(cfg->nx);
    amr_ctx* c = new amr_ctx(tp);
    c->cfg = *cfg;
    Geom& g = c->geom;
    g.bw = cfg->bw;
    g.nx = cfg->nx;
    g.gnx = cfg->nx + 2 * cfg->bw;
    g.nf = cfg->nf;
    g.pnx = cfg->nx + 2;
    g.gnx3 = g.gnx * g.gnx * g.gnx;
    g.pnx3 = g.pnx * g.pnx * g.pnx;
    g.ucount = g.nf * g.gnx3;
    g.z_reflect = cfg->z_reflect;
    // AMR_PREC_MIXED_SOLVE: the mixed multigrid correction, fluxes in FP64
    g.precision = cfg->precision == AMR_PREC_FP64 ? AMR_PREC_FP64 : AMR_PREC_MIXED;
    g.flux32 = cfg->precision == AMR_PREC_MIXED;
    g.recon = cfg->reconstruction;
    g.grid_dim = cfg->grid_dim;
    g.h0 = tp.h0;
    for (int d = 0; d < 3; d++) g.origin[d] = cfg->origin[d];
    g.theta = cfg->minmod_theta;
    g.cfl = cfg->cfl;
    g.gamma = cfg->gamma;
    g.rho_floor = cfg->rho_floor;
    g.ei_floor = cfg->ei_floor;
    g.grav_g = cfg->grav_g;
    install_callbacks(c);
    if (cfg->max_bricks > 0) {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            delete c;
            return AMR_ERR_NODEVICE;
        }
        c->has_device = true;
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            return AMR_ERR_CUDA;
        }
        const int cap = cfg->max_bricks;
        c->cap = cap;
        const size_t fcount = (size_t)g.nf * g.nx * g.nx * (g.nx + 1);
        int rc = 0;
        rc |= dev_alloc(c, &c->st.U, (size_t)cap * g.ucount);
        rc |= dev_alloc(c, &c->st.U0, (size_t)cap * g.ucount);
        rc |= dev_alloc(c, &c->st.Fx, (size_t)cap * fcount);
        rc |= dev_alloc(c, &c->st.Fy, (size_t)cap * fcount);
        rc |= dev_alloc(c, &c->st.Fz, (size_t)cap * fcount);
        if (cfg->physics != AMR_PHYSICS_EULER) {
            double** parr[8] = {&c->st.phi, &c->st.phi0, &c->st.dphi, &c->st.dphi1,
                                &c->st.S,   &c->st.fx,   &c->st.fy,   &c->st.fz};
            for (auto p : parr) rc |= dev_alloc(c, p, (size_t)cap * g.pnx3);
            if (g.precision == AMR_PREC_MIXED) {
                rc |= dev_alloc(c, &c->st.fdphi, (size_t)cap * g.pnx3);
                rc |= dev_alloc(c, &c->st.fdphi1, (size_t)cap * g.pnx3);
            }
        }
        rc |= dev_alloc(c, &c->bt.level, cap);
        rc |= dev_alloc(c, &c->bt.off, 3 * (size_t)cap);
        rc |= dev_alloc(c, &c->bt.h, cap);
        rc |= dev_alloc(c, &c->bt.ftype, 6 * (size_t)cap);
        rc |= dev_alloc(c, &c->bt.fnbr, 6 * (size_t)cap);
        rc |= dev_alloc(c, &c->bt.parent, cap);
        rc |= dev_alloc(c, &c->bt.cidx, cap);
        rc |= dev_alloc(c, &c->bt.child, 8 * (size_t)cap);
        rc |= dev_alloc(c, &c->d_fo, 2 * (size_t)g.nf);
        rc |= dev_alloc(c, &c->d_dt, cap);
        rc |= dev_alloc(c, &c->d_red, cap);
        rc |= dev_alloc(c, &c->d_flags, 8 * (size_t)cap);
        if (ztwd) {
            rc |= dev_alloc(c, &c->st.W, (size_t)cap * g.ucount);
            const size_t fc = (size_t)g.nx * g.nx * (g.nx + 1);
            rc |= dev_alloc(c, &c->st.Vx, (size_t)cap * fc);
            rc |= dev_alloc(c, &c->st.Vy, (size_t)cap * fc);
            rc |= dev_alloc(c, &c->st.Vz, (size_t)cap * fc);
            rc |= dev_alloc(c, &c->d_zerr, 1);
            if (!rc && cudaMemsetAsync(c->d_zerr, 0, sizeof(int), c->stream) != cudaSuccess) rc = 1;
            // State::abar (state_ztwd.cpp:27), State::rho_floor from the config
            c->zpar.abar[0] = 4.0;
            c->zpar.abar[1] = 14.12;
            c->zpar.abar[2] = 17.52;
            c->zpar.rho_floor = cfg->rho_floor;
        }
        if (rc) {
            std::string e = c->err;
            amr_destroy(c);
            fprintf(stderr, "amr_create: %s\n", e.c_str());
            return AMR_ERR_CUDA;
        }
        c->h_level.assign(cap, 0);
        c->h_off.assign(3 * cap, 0);
        c->h_h.assign(cap, 0.0);
        c->h_ftype.assign(6 * cap, 0);
        c->h_fnbr.assign(6 * cap, -1);
        c->h_parent.assign(cap, -1);
        c->h_cidx.assign(cap, 0);
        c->h_child.assign(8 * cap, -1);
        c->free_slots.reserve(cap);
        for (int s = cap - 1; s >= 0; s--) c->free_slots.push_back(s);
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
            amr_destroy(c);
            return AMR_ERR_CUDA;
        }
    }
    *out = c;
    return AMR_OK;
}

int amr_destroy(amr_ctx* c) {
    if (!c) return AMR_ERR_ARG;
    c->tree.on_create = nullptr;
    c->tree.on_destroy = nullptr;
    c->tree.clear();
    if (c->has_device) {
        cudaStreamSynchronize(c->stream);
        void* ptrs[] = {c->st.U,    c->st.U0,   c->st.Fx,     c->st.Fy,     c->st.Fz,      c->st.phi,
                        c->st.phi0, c->st.dphi, c->st.dphi1,  c->st.S,      c->st.fx,      c->st.fy,
                        c->st.fz,   c->bt.level, c->bt.off,   c->bt.h,      c->bt.ftype,   c->bt.fnbr,
                        c->bt.parent, c->bt.cidx, c->bt.child, c->d_fo,     c->d_dt,       c->d_red,
                        c->d_flags, c->d_stage, c->d_slots,  c->d_reflux, c->d_vitems, c->d_vranges, c->d_cpos,
                        c->d_U1, c->d_fwork, c->d_pubmask, c->d_pub, c->d_fdone, c->d_fctl,
                        c->st.fdphi, c->st.fdphi1, c->st.W, c->st.Vx, c->st.Vy, c->st.Vz, c->d_zerr};
        for (void* p : ptrs)
            if (p) cudaFree(p);
        amr_poisson_release(c);
        amr::graph_release(c);
        cudaStreamDestroy(c->stream);
    }
    delete c;
    return AMR_OK;
}

const char* amr_last_error(const amr_ctx* c) { return c ? c->err.c_str() : "null context"; }

int amr_init_root(amr_ctx* c) {
    if (!c) return AMR_ERR_ARG;
    c->pending_new.clear();
    c->tree.init_root();
    c->pending_new.clear();
    c->time = 0.0;
    TRY(rebuild_topology(c));
    return check_slots(c);
}

int amr_load_tree(amr_ctx* c, int n, const int* level, const int* loc, const int* age) {
    if (!c || n <= 0 || !level || !loc) return AMR_ERR_ARG;
    c->tree.init_root();
    if (level[0] != 0) return AMR_ERR_ARG;
    std::vector<Node*> stack{c->tree.root()};
    if (age) c->tree.root()->age = age[0];
    for (int i = 1; i < n; i++) {
        while (!stack.empty() && stack.back()->level >= level[i]) stack.pop_back();
        if (stack.empty() || stack.back()->level != level[i] - 1) {
            c->err = "amr_load_tree: list is not a depth-first pre-order";
            return AMR_ERR_ARG;
        }
        Node* p = stack.back();
        int cidx = 0;
        for (int d = 0; d < 3; d++) {
            const int bit = loc[3 * i + d] - 2 * p->loc[d];
            if (bit != 0 && bit != 1) {
                c->err = "amr_load_tree: location is not a child of the preceding node";
                return AMR_ERR_ARG;
            }
            cidx |= bit << d;
        }
        if (p->child[cidx]) return AMR_ERR_ARG;
        Node* ch = c->tree.create_child(p, cidx);
        if (age) ch->age = age[i];
        stack.push_back(ch);
    }
    c->pending_new.clear();
    TRY(rebuild_topology(c));
    return check_slots(c);
}

int amr_num_bricks(const amr_ctx* c) { return c ? (int)c->order.size() : 0; }

int amr_get_tree(const amr_ctx* c, int* level, int* loc, int* offset, int* age, int* child_mask, int* refine_mask,
                 double* h) {
    if (!c) return AMR_ERR_ARG;
    for (size_t i = 0; i < c->order.size(); i++) {
        const Node* n = c->order[i];
        if (level) level[i] = n->level;
        for (int d = 0; d < 3; d++) {
            if (loc) loc[3 * i + d] = n->loc[d];
            if (offset) offset[3 * i + d] = n->off[d];
        }
        if (age) age[i] = n->age;
        int cm = 0, rm = 0;
        for (int q = 0; q < 8; q++) {
            if (n->child[q]) cm |= 1 << q;
            if (n->refine[q]) rm |= 1 << q;
        }
        if (child_mask) child_mask[i] = cm;
        if (refine_mask) refine_mask[i] = rm;
        if (h) h[i] = n->h;
    }
    return AMR_OK;
}

int amr_refine_from_flags(amr_ctx* c, const unsigned char* flags, int clear, int* changed) {
    if (!c || !flags) return AMR_ERR_ARG;
    std::vector<Node*> snapshot = c->order;  // flags are indexed by the current DFS order
    auto fl = [&](const Node* n, int q) -> bool {
        if (n->dfs < 0 || n->dfs >= (int)snapshot.size() || snapshot[n->dfs] != n) return false;
        return flags[8 * n->dfs + q] != 0;
    };
    c->pending_new.clear();
    const bool rc = c->tree.check_for_refine(fl, clear != 0, c->time);
    if (changed) *changed = rc ? 1 : 0;
    TRY(finish_refine(c));
    return check_slots(c);
}

int amr_set_time(amr_ctx* c, double t) {
    if (!c) return AMR_ERR_ARG;
    if (t == 0.0)
        for (Node* n : c->order) n->age = -1;
    c->time = t;
    return AMR_OK;
}

double amr_get_time(const amr_ctx* c) { return c ? c->time : 0.0; }

long long amr_zone_count(const amr_ctx* c) { return c ? c->tree.zone_count() : 0; }

int amr_upload_state(amr_ctx* c, const double* U) {
    NEED_DEVICE(c);
    if (!U) return AMR_ERR_ARG;
    const int n = (int)c->order.size();
    const size_t cnt = (size_t)n * c->geom.ucount;
    TRY(ensure_stage(c, cnt));
    CUDA_TRY(cudaMemcpyAsync(c->d_stage, U, sizeof(double) * cnt, cudaMemcpyHostToDevice, c->stream));
    launch_scatter(c->d_stage, dslots_all(c), n, c->geom.ucount, c->st.U, c->stream);
    TRY(check_launch(c));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return AMR_OK;
}

int amr_download_state(amr_ctx* c, double* U) {
    NEED_DEVICE(c);
    if (!U) return AMR_ERR_ARG;
    const int n = (int)c->order.size();
    const size_t cnt = (size_t)n * c->geom.ucount;
    TRY(ensure_stage(c, cnt));
    launch_gather(c->st.U, dslots_all(c), n, c->geom.ucount, c->d_stage, c->stream);
    TRY(check_launch(c));
    CUDA_TRY(cudaMemcpyAsync(U, c->d_stage, sizeof(double) * cnt, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return AMR_OK;
}

int amr_get_flow_off(amr_ctx* c, double* fo) {
    NEED_DEVICE(c);
    CUDA_TRY(cudaMemcpyAsync(fo, c->d_fo, sizeof(double) * c->geom.nf, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return AMR_OK;
}

int amr_set_flow_off(amr_ctx* c, const double* fo) {
    NEED_DEVICE(c);
    CUDA_TRY(cudaMemcpyAsync(c->d_fo, fo, sizeof(double) * c->geom.nf, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return AMR_OK;
}

int amr_synchronize(amr_ctx* c) {
    NEED_DEVICE(c);
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return AMR_OK;
}

// GridNode::enforce_boundaries: levels in ascending order so every
// coarse-fine ghost reads a parent whose own ghosts are already filled.
int amr_enforce_boundaries(amr_ctx* c) {
    NEED_DEVICE(c);
    if (is_ztwd(c)) TRY(zt_ready(c));
    for (int l = 0; l <= c->tree.prm.max_level; l++)
        {
            ProfScope ps_(c->prof, KC_GHOST, c->stream, (long long)c->level_slots[l].size());
            if (is_ztwd(c))
                launch_zt_ghost_fill(c->geom, c->bt, c->st, c->zpar, dslots_level(c, l),
                                     (int)c->level_slots[l].size(), c->stream);
            else
                launch_ghost_fill(c->geom, c->bt, c->st, dslots_level(c, l), (int)c->level_slots[l].size(),
                                  c->stream);
        }
    return check_launch(c);
}

// Grid::store for every brick (U0 <- U incl. ghosts) and FO0 <- FO.
int amr_store(amr_ctx* c) {
    NEED_DEVICE(c);
    int maxslot = 0;
    for (int s : c->all_slots) maxslot = std::max(maxslot, s + 1);
    CUDA_TRY(cudaMemcpyAsync(c->st.U0, c->st.U, sizeof(double) * (size_t)maxslot * c->geom.ucount,
                             cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->d_fo + c->geom.nf, c->d_fo, sizeof(double) * c->geom.nf, cudaMemcpyDeviceToDevice,
                             c->stream));
    return AMR_OK;
}

int amr_restore(amr_ctx* c) {
    NEED_DEVICE(c);
    int maxslot = 0;
    for (int s : c->all_slots) maxslot = std::max(maxslot, s + 1);
    CUDA_TRY(cudaMemcpyAsync(c->st.U, c->st.U0, sizeof(double) * (size_t)maxslot * c->geom.ucount,
                             cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->d_fo, c->d_fo + c->geom.nf, sizeof(double) * c->geom.nf, cudaMemcpyDeviceToDevice,
                             c->stream));
    return AMR_OK;
}

// Fluxes of every brick, then coarse-fine corrections from the finest coarse
// level upward so a corrected child face is final before its parent uses it.
int amr_compute_fluxes(amr_ctx* c) {
    NEED_DEVICE(c);
    if (is_ztwd(c)) TRY(zt_ready(c));
    {
        ProfScope ps_(c->prof, KC_FLUX, c->stream, (long long)c->all_slots.size());
        if (is_ztwd(c))
            launch_zt_flux(c->geom, c->bt, c->st, c->zpar, dslots_all(c), (int)c->all_slots.size(), c->d_zerr,
                           c->stream);
        else
            launch_flux(c->geom, c->st, dslots_all(c), (int)c->all_slots.size(), c->stream);
    }
    for (int l = c->tree.prm.max_level; l >= 0; l--) {
        const int n = c->off_reflux[l + 1] - c->off_reflux[l];
        {
            ProfScope ps_(c->prof, KC_REFLUX, c->stream);
            launch_reflux(c->geom, c->st, c->d_reflux + c->off_reflux[l], n, c->stream);
        }
    }
    return check_launch(c);
}

int amr_add_difs(amr_ctx* c, double dt, double beta) {
    NEED_DEVICE(c);
    if (is_ztwd(c)) TRY(zt_ready(c));
    const int grav = c->cfg.physics == AMR_PHYSICS_EULER_GRAVITY;
    {
        ProfScope ps_(c->prof, KC_ADD_DIFS, c->stream);
        launch_flow_off(c->geom, c->st, c->tree.root()->slot, c->tree.root()->h, dt, beta, c->d_fo, c->stream);
    }
    {
        ProfScope ps_(c->prof, KC_ADD_DIFS, c->stream, (long long)c->all_slots.size());
        if (is_ztwd(c))
            launch_zt_add_difs(c->geom, c->bt, c->st, c->zpar, dslots_all(c), (int)c->all_slots.size(), dt, beta,
                               c->d_zerr, c->stream);
        else
            launch_add_difs(c->geom, c->st, dslots_all(c), (int)c->all_slots.size(), c->bt.h, dt, beta, grav,
                            c->stream);
    }
    for (Node* n : c->order) n->age++;  // GridNode::add_difs, grid_node.cpp:338
    return check_launch(c);
}

// Restriction from the finest parents to the root (children first).
int amr_inject_from_children(amr_ctx* c) {
    NEED_DEVICE(c);
    if (is_ztwd(c)) TRY(zt_ready(c));
    for (int l = c->tree.prm.max_level; l >= 0; l--)
        {
            ProfScope ps_(c->prof, KC_INJECT, c->stream);
            if (is_ztwd(c))
                launch_zt_inject(c->geom, c->bt, c->st, c->zpar, dslots_parent(c, l), (int)c->parent_slots[l].size(),
                                 c->d_zerr, c->stream);
            else
                launch_inject(c->geom, c->bt, c->st, dslots_parent(c, l), (int)c->parent_slots[l].size(),
                              c->stream);
        }
    return check_launch(c);
}

// Grid::max_dt per brick on the device, then GridNode::max_dt's recursion
// (1/max of inverse child steps) on the host in the reference's order.
int amr_max_dt(amr_ctx* c, double* dt) {
    NEED_DEVICE(c);
    if (!dt) return AMR_ERR_ARG;
    if (is_ztwd(c)) TRY(zt_ready(c));
    const int n = (int)c->all_slots.size();
    {
        ProfScope ps_(c->prof, KC_MAX_DT, c->stream, (long long)n);
        if (is_ztwd(c))
            launch_zt_max_dt(c->geom, c->bt, c->st, c->zpar, dslots_all(c), n, c->d_dt, c->d_zerr, c->stream);
        else
            launch_max_dt(c->geom, c->st, dslots_all(c), n, c->bt.h, c->d_dt, c->stream);
    }
    TRY(check_launch(c));
    if (is_ztwd(c)) TRY(zt_check(c));
    std::vector<double> per(c->cap);
    int maxslot = 0;
    for (int s : c->all_slots) maxslot = std::max(maxslot, s + 1);
    CUDA_TRY(cudaMemcpyAsync(per.data(), c->d_dt, sizeof(double) * maxslot, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    std::function<double(const Node*)> rec = [&](const Node* nd) -> double {
        double dtinv = 0.0;
        for (int q = 0; q < 8; q++)
            if (nd->child[q]) {
                const double cdtinv = 1.0 / rec(nd->child[q]);
                dtinv = cdtinv > dtinv ? cdtinv : dtinv;
            }
        const double own = 1.0 / per[nd->slot];
        dtinv = own > dtinv ? own : dtinv;
        return 1.0 / dtinv;
    };
    *dt = rec(c->tree.root());
    return AMR_OK;
}

int amr_check_for_refine(amr_ctx* c, double min_refine_density, int clear, int* changed) {
    NEED_DEVICE(c);
    const int n = (int)c->all_slots.size();
    {
        ProfScope ps_(c->prof, KC_REFINE, c->stream);
        launch_refine_flags(c->geom, c->st, dslots_all(c), n, min_refine_density, c->d_flags, c->stream);
    }
    TRY(check_launch(c));
    std::vector<unsigned char> fl(8 * (size_t)n);
    CUDA_TRY(cudaMemcpyAsync(fl.data(), c->d_flags, fl.size(), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    int ch = 0;
    TRY(amr_refine_from_flags(c, fl.data(), clear, &ch));
    if (changed) *changed = ch;
    if (ch) TRY(amr_enforce_boundaries(c));  // grid_node.cpp:1028-1030
    return AMR_OK;
}

int amr_state_max(amr_ctx* c, int field, double* vmax) {
    NEED_DEVICE(c);
    if (field < 0 || field >= c->geom.nf || !vmax) return AMR_ERR_ARG;
    const int n = (int)c->all_slots.size();
    {
        ProfScope ps_(c->prof, KC_OTHER, c->stream);
        launch_state_max(c->geom, c->bt, c->st, dslots_all(c), n, field, c->d_red, c->stream);
    }
    TRY(check_launch(c));
    std::vector<double> v(n);
    CUDA_TRY(cudaMemcpyAsync(v.data(), c->d_red, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    double m = -1.0E+99;
    for (double x : v) m = x > m ? x : m;
    *vmax = m;
    return AMR_OK;
}

// HydroDriver::sub_step (euler/hydro_driver.cpp:200-214).
int amr_sub_step(amr_ctx* c, double dt, double beta) {
    NEED_DEVICE(c);
    TRY(amr_enforce_boundaries(c));
    TRY(amr_compute_fluxes(c));
    TRY(amr_add_difs(c, dt, beta));
    return AMR_OK;
}

namespace {

// Work list (finest level first, depth-first within a level) and publish
// masks of the fused substep, rebuilt when the topology changes.
int fused_setup(amr_ctx* c) {
    const int cap = c->cap;
    if (!c->d_U1) {
        CUDA_TRY(cudaMalloc(&c->d_U1, sizeof(double) * (size_t)cap * c->geom.ucount));
        CUDA_TRY(cudaMemcpyAsync(c->d_U1, c->st.U, sizeof(double) * (size_t)cap * c->geom.ucount,
                                 cudaMemcpyDeviceToDevice, c->stream));
        CUDA_TRY(cudaMalloc(&c->d_pubmask, (size_t)cap));
        CUDA_TRY(cudaMalloc(&c->d_pub, sizeof(double) * (size_t)cap * 6 * c->geom.nf * c->geom.nx * c->geom.nx));
        CUDA_TRY(cudaMalloc(&c->d_fdone, sizeof(int) * (size_t)cap));
        CUDA_TRY(cudaMemsetAsync(c->d_fdone, 0, sizeof(int) * (size_t)cap, c->stream));
        CUDA_TRY(cudaMalloc(&c->d_fctl, sizeof(unsigned int) * 2));
    }
    if (c->fused_version == c->topo_version) return AMR_OK;
    std::vector<int2> work;
    const int maxl = (int)c->level_slots.size() - 1;
    for (int l = maxl; l >= 0; l--)
        for (int q = 0; q < (int)c->level_slots[l].size(); q++) {
            const int s = c->level_slots[l][q];
            const int vr = c->off_vrange[l] + q;
            work.push_back(make_int2(s, vr));
        }
    std::vector<unsigned char> mask((size_t)cap, 0);
    for (int l = 0; l <= maxl; l++)
        for (const RefluxItem& it : c->reflux[l])
            mask[it.child] |= (unsigned char)(1u << (2 * it.dir + (it.ic == c->geom.bw ? 0 : 1)));
    if ((int)work.size() > c->fwork_cap) {
        if (c->d_fwork) cudaFree(c->d_fwork);
        c->fwork_cap = (int)work.size() * 2 + 64;
        CUDA_TRY(cudaMalloc(&c->d_fwork, sizeof(int2) * c->fwork_cap));
    }
    CUDA_TRY(cudaMemcpyAsync(c->d_fwork, work.data(), sizeof(int2) * work.size(), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->d_pubmask, mask.data(), mask.size(), cudaMemcpyHostToDevice, c->stream));
    c->nfwork = (int)work.size();
    c->fused_version = c->topo_version;
    return AMR_OK;
}

}  // namespace

// amr_sub_step of the Euler driver as one persistent launch (plus the root's
// flow-off): ghost zones, fluxes, coarse-fine corrections and the RK
// combination per brick, the result written to the second state array which
// then becomes the state.  Interiors are bitwise those of amr_sub_step (FP64
// form); the ghost zones of the new state are not filled.
int amr_fused_sub_step(amr_ctx* c, double dt, double beta, int blocks_per_sm) {
    NEED_DEVICE(c);
    if (c->cfg.physics != AMR_PHYSICS_EULER || c->geom.nf != 6) {
        c->err = "fused substep: Euler physics without gravity only";
        return AMR_ERR_ARG;
    }
    if (c->geom.bw != 2 || c->geom.recon != AMR_RECON_MINMOD) {
        c->err = "fused substep: minmod reconstruction with bw 2 only";
        return AMR_ERR_ARG;
    }
    TRY(fused_setup(c));
    CUDA_TRY(cudaMemsetAsync(c->d_fctl, 0, sizeof(unsigned int) * 2, c->stream));
    FusedArgs a{};
    a.g = c->geom;
    a.bt = c->bt;
    a.Uin = c->st.U;
    a.U0 = c->st.U0;
    a.Uout = c->d_U1;
    a.work = c->d_fwork;
    a.nwork = c->nfwork;
    a.next = c->d_fctl;
    a.done = c->d_fdone;
    a.epoch = ++c->fused_epoch;
    a.pubmask = c->d_pubmask;
    a.pub = c->d_pub;
    a.vitems = c->d_vitems;
    a.vranges = c->d_vranges;
    a.dt = dt;
    a.beta = beta;
    a.root = c->tree.root()->slot;
    a.Fx = c->st.Fx;
    a.Fy = c->st.Fy;
    a.Fz = c->st.Fz;
    a.err = reinterpret_cast<int*>(c->d_fctl + 1);
    a.wait_limit = (unsigned long long)c->fused_wait_limit;
    cudaError_t e;
    {
        ProfScope ps_(c->prof, KC_FUSED, c->stream, (long long)c->nfwork);
        e = c->geom.flux32 ? launch_substep_fused_f32(a, blocks_per_sm, c->stream, &c->fused_blocks)
                                                : launch_substep_fused_f64(a, blocks_per_sm, c->stream, &c->fused_blocks);
    }
    if (e != cudaSuccess) {
        c->err = std::string("fused substep launch: ") + cudaGetErrorString(e);
        return AMR_ERR_CUDA;
    }
    {
        ProfScope ps_(c->prof, KC_ADD_DIFS, c->stream);
        launch_flow_off(c->geom, c->st, c->tree.root()->slot, c->tree.root()->h, dt, beta, c->d_fo, c->stream);
    }
    std::swap(c->st.U, c->d_U1);
    for (Node* n : c->order) n->age++;  // GridNode::add_difs, grid_node.cpp:338
    unsigned int err = 0;
    CUDA_TRY(cudaMemcpyAsync(&err, c->d_fctl + 1, sizeof(unsigned int), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (err & 1u) {
        c->err = "fused substep: a wait for a child's face fluxes timed out";
        return AMR_ERR_TIMEOUT;
    }
    if (err & 2u) {
        c->err = "fused substep: coarse-fine ghost of a coarse-fine ghost (tree not properly nested)";
        return AMR_ERR_STATE;
    }
    return check_launch(c);
}

// HydroDriver::step (euler/hydro_driver.cpp:171-194), RK_ORDER 3.
int amr_hydro_step(amr_ctx* c, double dt, double min_refine_density) {
    NEED_DEVICE(c);
    if (!(dt > 0.0)) return AMR_ERR_ARG;
    TRY(amr_store(c));
    TRY(amr_sub_step(c, dt, 1.0));
    TRY(amr_inject_from_children(c));
    TRY(amr_sub_step(c, dt, 0.25));
    TRY(amr_inject_from_children(c));
    TRY(amr_sub_step(c, dt, 2.0 / 3.0));
    TRY(amr_inject_from_children(c));
    TRY(amr_enforce_boundaries(c));
    TRY(amr_check_for_refine(c, min_refine_density, 1, nullptr));
    TRY(amr_set_time(c, c->time + dt));
    return AMR_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// instrumentation
// ---------------------------------------------------------------------------
extern "C" {

static const char* kClassNames[amr::KC_COUNT] = {
    "ghost_fill", "flux", "reflux", "add_difs", "inject", "max_dt", "refine_flags", "prolong",
    "relax", "vcycle_down", "phi_boundaries", "dphi_boundaries", "forces", "solution_error",
    "source", "phys_boundary", "coarse_correction", "phi_time", "other", "fused_substep"};

int amr_get_stream(amr_ctx* c, void** stream) {
    NEED_DEVICE(c);
    if (!stream) return AMR_ERR_ARG;
    *stream = (void*)c->stream;
    return AMR_OK;
}

int amr_profile_enable(amr_ctx* c, int on) {
    NEED_DEVICE(c);
    c->prof.collect();
    c->prof.on = on != 0;
    return AMR_OK;
}

int amr_profile_reset(amr_ctx* c) {
    NEED_DEVICE(c);
    c->prof.reset();
    return AMR_OK;
}

int amr_profile_get(amr_ctx* c, int cls, double* ms, long long* launches, const char** name) {
    NEED_DEVICE(c);
    if (cls < 0 || cls >= amr::KC_COUNT) return AMR_ERR_ARG;
    c->prof.collect();
    if (ms) *ms = c->prof.ms[cls];
    if (launches) *launches = c->prof.launches[cls];
    if (name) *name = kClassNames[cls];
    return AMR_OK;
}

int amr_launch_count(amr_ctx* c, long long* kernels) {
    if (!c || !kernels) return AMR_ERR_ARG;
    *kernels = c->prof.kernels;
    return AMR_OK;
}

int amr_profile_units(amr_ctx* c, int cls, long long* units) {
    NEED_DEVICE(c);
    if (cls < 0 || cls >= amr::KC_COUNT || !units) return AMR_ERR_ARG;
    c->prof.collect();
    *units = c->prof.units[cls];
    return AMR_OK;
}

int amr_stats(amr_ctx* c, long long* relax_calls, int* reflux_hazards, int* nbricks, int* max_level) {
    if (!c) return AMR_ERR_ARG;
    if (relax_calls) *relax_calls = c->relax_calls;
    if (reflux_hazards) *reflux_hazards = c->reflux_hazards;
    if (nbricks) *nbricks = (int)c->order.size();
    if (max_level) *max_level = c->tree.max_level_present();
    return AMR_OK;
}

}  // extern "C"
