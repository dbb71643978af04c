// Host octree with the reference's refinement semantics.
//
// The reference keeps explicit sibling pointers to real nodes or to proxy
// objects (GridAMRBound for a coarse-fine face, GridPhysBound for a domain
// face; grid/grid_node.cpp:256-290, oct_node/oct_node.cpp:172-303).  Here a
// node's face neighbour is derived from its (level, location): a physical face
// when the location touches the domain edge (OctNode::is_phys_bound,
// oct_node.cpp:86-109), otherwise the same-level node at location +- 1 if it
// exists, otherwise a coarse-fine face served by the parent.  This gives the
// same adjacency the reference's pointer bookkeeping maintains.
#pragma once

#include <cstdint>
#include <functional>
#include <unordered_map>
#include <vector>

namespace amr {

struct Node {
    int level = 0;
    int loc[3] = {0, 0, 0};
    int off[3] = {0, 0, 0};  // Grid::offset, grid_node.cpp:244-247
    double h = 0.0;
    Node* parent = nullptr;
    int cidx = 0;  // ChildIndex within the parent (x | y<<1 | z<<2)
    Node* child[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    int age = -1;  // GridNode::age
    bool refine[8] = {false, false, false, false, false, false, false, false};
    int slot = -1;  // device brick slot
    int dfs = -1;   // position in depth-first pre-order
    int nchildren() const {
        int n = 0;
        for (int c = 0; c < 8; c++) n += child[c] != nullptr;
        return n;
    }
};

struct TreeParams {
    int bw = 2, nx = 8;
    int max_level = 2, min_level = 1, min_grid_life = 24;
    int mirror_y = 1;
    double h0 = 0.25;
};

class Octree {
public:
    explicit Octree(const TreeParams& p);
    ~Octree();
    void clear();
    void init_root();
    Node* root() const { return root_; }

    // Tree queries.
    Node* find(int level, int x, int y, int z) const;
    bool is_phys_bound(const Node* n, int face) const;
    Node* same_level_neighbor(const Node* n, int face) const;  // nullptr for phys/coarse-fine
    std::vector<Node*> dfs_order() const;
    int max_level_present() const;
    long long zone_count() const;
    int count() const { return (int)index_.size(); }

    // Structural edits (GridNode::create_child / destroy_child).
    Node* create_child(Node* p, int c);
    void destroy_child(Node* p, int c);

    // GridNode::check_for_refine decision.  flags(n, c) returns the density
    // test for octant c of node n (set_refine_flags' cell loop).  Returns
    // use_refine_flags()'s result; created/destroyed nodes are reported
    // through the callbacks.
    bool check_for_refine(const std::function<bool(const Node*, int)>& flags, bool clear, double time);

    std::function<void(Node*)> on_create;   // after a node is linked
    std::function<void(Node*)> on_destroy;  // before a node is unlinked
    int anomalies = 0;  // nesting lookups that hit a missing node

    TreeParams prm;

private:
    Node* root_ = nullptr;
    std::unordered_map<uint64_t, Node*> index_;
    static uint64_t key(int level, int x, int y, int z);
    void link(Node* n);
    void destroy_subtree(Node* n);

    void clear_refine_flags(Node* n);
    void set_refine_flags(Node* n, const std::function<bool(const Node*, int)>& flags, double time);
    void propagate_refine_flags_up(Node* n);
    void enforce_proper_nesting(Node* n);
    void mirror_refine(Node* n, const Node* mirror, int dir);
    bool use_refine_flags(Node* n);
};

}  // namespace amr
