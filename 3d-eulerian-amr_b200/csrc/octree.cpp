// Host octree: topology and refinement decisions (bit-exact with the
// reference's GridNode/OctNode logic, cited per function).
#include "octree.h"

#include <algorithm>

namespace amr {

Octree::Octree(const TreeParams& p) : prm(p) {}

Octree::~Octree() { clear(); }

uint64_t Octree::key(int level, int x, int y, int z) {
    return (uint64_t(level) << 60) | (uint64_t(uint32_t(x) & 0xFFFFF) << 40) | (uint64_t(uint32_t(y) & 0xFFFFF) << 20) |
           uint64_t(uint32_t(z) & 0xFFFFF);
}

void Octree::clear() {
    if (root_) destroy_subtree(root_);
    root_ = nullptr;
    index_.clear();
}

void Octree::destroy_subtree(Node* n) {
    for (int c = 0; c < 8; c++)
        if (n->child[c]) {
            destroy_subtree(n->child[c]);
            n->child[c] = nullptr;
        }
    if (on_destroy) on_destroy(n);
    index_.erase(key(n->level, n->loc[0], n->loc[1], n->loc[2]));
    delete n;
}

void Octree::link(Node* n) { index_[key(n->level, n->loc[0], n->loc[1], n->loc[2])] = n; }

// GridNode::init (grid_node.cpp:1410-1418): one root brick, offset 0,
// h = h0 (Grid::h0 = 2*GRID_DIM/(GNX-2*BW), grid.cpp:70), age -1.
void Octree::init_root() {
    clear();
    root_ = new Node;
    root_->h = prm.h0;
    root_->age = -1;
    link(root_);
    if (on_create) on_create(root_);
}

Node* Octree::find(int level, int x, int y, int z) const {
    const int n = 1 << level;
    if (x < 0 || y < 0 || z < 0 || x >= n || y >= n || z >= n) return nullptr;
    auto it = index_.find(key(level, x, y, z));
    return it == index_.end() ? nullptr : it->second;
}

// OctNode::is_phys_bound (oct_node.cpp:86-109).
bool Octree::is_phys_bound(const Node* n, int face) const {
    const int hi = (1 << n->level) - 1;
    const int ax = face >> 1;
    return (face & 1) ? n->loc[ax] == hi : n->loc[ax] == 0;
}

Node* Octree::same_level_neighbor(const Node* n, int face) const {
    if (is_phys_bound(n, face)) return nullptr;
    int l[3] = {n->loc[0], n->loc[1], n->loc[2]};
    l[face >> 1] += (face & 1) ? 1 : -1;
    return find(n->level, l[0], l[1], l[2]);
}

// OctNode::create_child (oct_node.cpp:172-240) + GridNode::create_child
// (grid_node.cpp:235-270): location 2*loc + c, offset 2*offset + BW +
// c*(GNX-2*BW), h/2, refine flags cleared, age -1 (the GridNode constructor;
// set_time keeps it).  Prolongation (inject_from_parent) is the on_create
// callback's job.
Node* Octree::create_child(Node* p, int c) {
    Node* n = new Node;
    n->level = p->level + 1;
    n->parent = p;
    n->cidx = c;
    const int cv[3] = {c & 1, (c >> 1) & 1, (c >> 2) & 1};
    for (int d = 0; d < 3; d++) {
        n->loc[d] = 2 * p->loc[d] + cv[d];
        n->off[d] = 2 * p->off[d] + prm.bw + cv[d] * prm.nx;
    }
    n->h = p->h * 0.5;
    n->age = -1;
    p->child[c] = n;
    link(n);
    if (on_create) on_create(n);
    return n;
}

// OctNode::destroy_child (oct_node.cpp:242-303): the whole subtree goes.
void Octree::destroy_child(Node* p, int c) {
    Node* n = p->child[c];
    if (!n) return;
    p->child[c] = nullptr;
    destroy_subtree(n);
}

std::vector<Node*> Octree::dfs_order() const {
    std::vector<Node*> out;
    if (!root_) return out;
    std::vector<Node*> stack{root_};
    while (!stack.empty()) {
        Node* n = stack.back();
        stack.pop_back();
        out.push_back(n);
        for (int c = 7; c >= 0; c--)
            if (n->child[c]) stack.push_back(n->child[c]);
    }
    return out;
}

int Octree::max_level_present() const {
    int m = 0;
    for (auto& kv : index_) m = std::max(m, kv.second->level);
    return m;
}

// GridNode::get_zone_cnt (grid_node.cpp:1276-1288): every octant without a
// child contributes nx^3/8 cells.
long long Octree::zone_count() const {
    const long long per = (long long)prm.nx * prm.nx * prm.nx / 8;
    long long cnt = 0;
    for (auto& kv : index_)
        for (int c = 0; c < 8; c++)
            if (!kv.second->child[c]) cnt += per;
    return cnt;
}

// ---------------------------------------------------------------------------
// refinement (grid_node.cpp:620-1033)
// ---------------------------------------------------------------------------
void Octree::clear_refine_flags(Node* n) {
    for (int c = 0; c < 8; c++) n->refine[c] = false;
    for (int c = 0; c < 8; c++)
        if (n->child[c]) clear_refine_flags(n->child[c]);
}

// GridNode::set_refine_flags (grid_node.cpp:631-685).
void Octree::set_refine_flags(Node* n, const std::function<bool(const Node*, int)>& flags, double time) {
    if (n->level < prm.min_level) {
        for (int c = 0; c < 8; c++) n->refine[c] = true;
    } else if (n->level < prm.max_level) {
        for (int c = 0; c < 8; c++) {
            const Node* ch = n->child[c];
            if (!ch) continue;
            for (int j = 0; j < 8; j++)
                if (ch->refine[j] || ch->child[j]) n->refine[c] = true;
        }
        for (int c = 0; c < 8; c++)
            if (flags(n, c)) n->refine[c] = true;
    }
    for (int c = 0; c < 8; c++) {
        Node* ch = n->child[c];
        if (!ch) continue;
        if (ch->nchildren() > 0) n->refine[c] = true;
        set_refine_flags(ch, flags, time);
        if (ch->age < prm.min_grid_life && time != 0.0 && n->level < prm.max_level) n->refine[c] = true;
    }
}

// GridNode::propagate_refine_flags_up (grid_node.cpp:902-914).
void Octree::propagate_refine_flags_up(Node* n) {
    for (int c = 0; c < 8; c++) {
        Node* ch = n->child[c];
        if (!ch) continue;
        propagate_refine_flags_up(ch);
        for (int j = 0; j < 8; j++)
            if (ch->refine[j]) {
                n->refine[c] = true;
                break;
            }
    }
}

// GridNode::enforce_proper_nesting (grid_node.cpp:687-900).  For every
// octant ci flagged for refinement, the level-(L) bricks that touch it across
// faces, edges and corners get their own refine flag set on the parent level.
// The seven neighbour directions are the non-empty subsets of {x,y,z}; along a
// flipped axis the neighbour lies in the parent's sibling when the octant sits
// on the same side as this node within its parent and that side is not a
// domain face, otherwise inside the parent.  Siblings are visited in x, y, z
// order exactly as the reference chains get_sibling().
void Octree::enforce_proper_nesting(Node* n) {
    for (int c = 0; c < 8; c++)
        if (n->child[c] && n->refine[c]) enforce_proper_nesting(n->child[c]);
    if (n->level == 0) return;
    const int mi = n->cidx;
    Node* parent = n->parent;
    for (int ci = 0; ci < 8; ci++) {
        if (!n->refine[ci]) continue;
        // subsets in the reference's order: x, y, z, xy, xz, yz, xyz
        static const int subsets[7] = {1, 2, 4, 3, 5, 6, 7};
        for (int s = 0; s < 7; s++) {
            const int mask = subsets[s];
            const int target = mi ^ mask;
            Node* g = parent;
            bool hopped_proxy = false;
            for (int ax = 0; ax < 3; ax++) {
                if (!(mask & (1 << ax))) continue;
                const int mbit = (mi >> ax) & 1, cbit = (ci >> ax) & 1;
                const int face = 2 * ax + cbit;  // ChildIndex::x_face/y_face/z_face
                if (mbit == cbit && !is_phys_bound(n, face)) {
                    if (!g) {
                        hopped_proxy = true;
                        break;
                    }
                    g = same_level_neighbor(g, face);
                }
            }
            if (hopped_proxy || !g) {
                anomalies++;
                continue;
            }
            g->refine[target] = true;
        }
    }
}

// GridNode::mirror_refine (grid_node.cpp:936-955).
void Octree::mirror_refine(Node* n, const Node* mirror, int dir) {
    if (n->level >= prm.max_level) return;
    const int mask = 1 << dir;
    for (int c = 0; c < 8; c++)
        if (mirror->refine[c ^ mask]) n->refine[c] = true;
    for (int c = 0; c < 8; c++) {
        const Node* cm = mirror->child[c ^ mask];
        if (n->child[c] && cm) mirror_refine(n->child[c], cm, dir);
    }
}

// GridNode::use_refine_flags (grid_node.cpp:916-934).
bool Octree::use_refine_flags(Node* n) {
    bool rc = false;
    for (int c = 0; c < 8; c++) {
        if (n->refine[c] && !n->child[c] && n->level + 1 <= prm.max_level) {
            Node* ch = create_child(n, c);
            for (int j = 0; j < 8; j++) ch->refine[j] = false;
            rc = true;
        } else if (!n->refine[c] && n->child[c]) {
            destroy_child(n, c);
            rc = true;
        }
    }
    for (int c = 0; c < 8; c++)
        if (n->child[c]) rc = use_refine_flags(n->child[c]) || rc;
    return rc;
}

// GridNode::check_for_refine (grid_node.cpp:957-1033), MIRROR_REFINE_Y only.
bool Octree::check_for_refine(const std::function<bool(const Node*, int)>& flags, bool clear, double time) {
    if (prm.max_level == 0 || !root_) return false;
    if (clear) clear_refine_flags(root_);
    set_refine_flags(root_, flags, time);
    propagate_refine_flags_up(root_);
    enforce_proper_nesting(root_);
    if (prm.mirror_y) mirror_refine(root_, root_, 1);
    propagate_refine_flags_up(root_);
    return use_refine_flags(root_);
}

}  // namespace amr
