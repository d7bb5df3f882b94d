// Host-side order bookkeeping of a world step: the structures of
// ReactPhysics3D v0.10.2 whose history decides in which order pairs,
// contacts and bodies are processed.  The floating-point work of a step runs
// on the GPU (world.cu); these structures only decide order, and they do it
// exactly as the reference does, so that the GPU replays the reference's
// sequence of operations:
//
//   Tree   the broad-phase dynamic AABB tree (src/collision/broadphase/
//          DynamicAABBTree.cpp): node allocation from a free list (:93-143),
//          volume-cost insertion (:219-345), leaf removal (:348-412), AVL-style
//          rotations (:420-586) and the stack query whose visiting order is
//          the order of the reported pairs (:589-638).
//   IdSet  the moved-collider set BroadPhaseSystem::mMovedShapes, a
//          Set<int32> (include/reactphysics3d/containers/Set.h): power-of-two
//          buckets, identity hash, new entries at the head of their bucket
//          chain, rehash on growth, iteration bucket by bucket (:119-170,
//          :263-341, :380-420, :475-484, :571-600).
//   PairMap  the id-to-index maps of OverlappingPairs (a flat hash table;
//          lookups only, so its own order never shows).
//   Comps  component order of Components (src/components/Components.cpp:
//          67-193): enabled components first, additions and enable/disable
//          by moving or swapping with the first disabled / last enabled one.
//
// Fat AABBs enter the tree as computed on the GPU (bit-identical to the
// reference's); the tree only merges them (min/max) and compares volumes,
// with the reference's float expressions.
//
// The tree's insertion, removal and rotations are written once (TreeT) for
// two node stores: a growing host vector (Tree, the host replica) and a
// fixed device span (DevTree, one world's tree in a world group's device
// pool, updated by one GPU thread per world).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#if defined(__CUDACC__)
#define ORDER_HD __host__ __device__
#define ORDER_NO_EXEC_CHECK _Pragma("nv_exec_check_disable")
#else
#define ORDER_HD
#define ORDER_NO_EXEC_CHECK
#endif

namespace rp3dg {
namespace order {

struct Box {
    float mn[3], mx[3];
};

// std::min / std::max as the reference's AABB code uses them (signed zeros)
ORDER_HD inline float rmin(float a, float b) { return (b < a) ? b : a; }
ORDER_HD inline float rmax(float a, float b) { return (a < b) ? b : a; }

// AABB::mergeTwoAABBs (AABB.h:235-243)
ORDER_HD inline Box merge(const Box& a, const Box& b) {
    Box r;
    for (int k = 0; k < 3; k++) {
        r.mn[k] = rmin(a.mn[k], b.mn[k]);
        r.mx[k] = rmax(a.mx[k], b.mx[k]);
    }
    return r;
}
// AABB::getVolume (AABB.h:190-193)
ORDER_HD inline float volume(const Box& a) {
    const float dx = a.mx[0] - a.mn[0], dy = a.mx[1] - a.mn[1], dz = a.mx[2] - a.mn[2];
    return dx * dy * dz;
}
// AABB::testCollision, inclusive (AABB.h:179-187)
ORDER_HD inline bool overlap(const Box& a, const Box& b) {
    for (int k = 0; k < 3; k++)
        if (a.mx[k] < b.mn[k] || b.mx[k] < a.mn[k]) return false;
    return true;
}

// One node of DynamicAABBTree (TreeNode, 48 bytes so that a device thread
// reads it as three 16-byte words).
struct alignas(16) TreeNode {
    int parent = -1;    // parentID, or nextNodeID while the node is free
    int child[2] = {-1, -1};
    int height = -1;    // 0 = leaf, -1 = free
    Box box{};
    int data = -1;      // collider id of a leaf
    int unused = 0;
};
static_assert(sizeof(TreeNode) == 48, "tree node layout");

// DynamicAABBTree::allocateNode's growth (double the array, chain the new
// nodes into the free list): the host vector grows; a device span cannot.
inline bool grow_nodes(std::vector<TreeNode>& nodes, int nb_nodes, int& free_id) {
    const int old = int(nodes.size());
    nodes.resize(size_t(old) * 2);
    for (int i = nb_nodes; i < int(nodes.size()) - 1; i++) {
        nodes[size_t(i)].parent = i + 1;
        nodes[size_t(i)].height = -1;
    }
    nodes.back().parent = -1;
    nodes.back().height = -1;
    free_id = nb_nodes;
    return true;
}

// One world's nodes in device memory: n nodes, no growth.
struct NodeSpan {
    TreeNode* p = nullptr;
    int n = 0;
    ORDER_HD TreeNode& operator[](int i) const { return p[i]; }
    ORDER_HD int size() const { return n; }
};
ORDER_HD inline bool grow_nodes(NodeSpan&, int, int&) { return false; }

template <class Nodes>
struct TreeT {
    static constexpr int NIL = -1;
    using Node = TreeNode;
    Nodes nodes;
    int root = NIL;
    int free_id = 0;
    int nb_nodes = 0;
    bool failed = false;   // a device tree that would have had to grow

    ORDER_NO_EXEC_CHECK
    ORDER_HD bool leaf(int id) const { return nodes[id].height == 0; }

    ORDER_NO_EXEC_CHECK
    ORDER_HD int alloc() {
        if (free_id == NIL && !grow_nodes(nodes, nb_nodes, free_id)) {
            failed = true;
            return NIL;
        }
        const int id = free_id;
        free_id = nodes[id].parent;
        nodes[id].parent = NIL;
        nodes[id].height = 0;
        nb_nodes++;
        return id;
    }
    ORDER_NO_EXEC_CHECK
    ORDER_HD void release(int id) {
        nodes[id].parent = free_id;
        nodes[id].height = -1;
        free_id = id;
        nb_nodes--;
    }

    ORDER_NO_EXEC_CHECK
    ORDER_HD int balance(int a_id) {
        Node* A = &nodes[a_id];
        if (A->height == 0 || A->height < 2) return a_id;
        const int b_id = A->child[0], c_id = A->child[1];
        Node* B = &nodes[b_id];
        Node* C = &nodes[c_id];
        const int bf = C->height - B->height;
        if (bf > 1) {
            const int f_id = C->child[0], g_id = C->child[1];
            Node* F = &nodes[f_id];
            Node* G = &nodes[g_id];
            C->child[0] = a_id;
            C->parent = A->parent;
            A->parent = c_id;
            if (C->parent != NIL) {
                if (nodes[C->parent].child[0] == a_id) nodes[C->parent].child[0] = c_id;
                else nodes[C->parent].child[1] = c_id;
            } else {
                root = c_id;
            }
            if (F->height > G->height) {
                C->child[1] = f_id;
                A->child[1] = g_id;
                G->parent = a_id;
                A->box = merge(B->box, G->box);
                C->box = merge(A->box, F->box);
                A->height = (B->height < G->height ? G->height : B->height) + 1;
                C->height = (A->height < F->height ? F->height : A->height) + 1;
            } else {
                C->child[1] = g_id;
                A->child[1] = f_id;
                F->parent = a_id;
                A->box = merge(B->box, F->box);
                C->box = merge(A->box, G->box);
                A->height = (B->height < F->height ? F->height : B->height) + 1;
                C->height = (A->height < G->height ? G->height : A->height) + 1;
            }
            return c_id;
        }
        if (bf < -1) {
            const int f_id = B->child[0], g_id = B->child[1];
            Node* F = &nodes[f_id];
            Node* G = &nodes[g_id];
            B->child[0] = a_id;
            B->parent = A->parent;
            A->parent = b_id;
            if (B->parent != NIL) {
                if (nodes[B->parent].child[0] == a_id) nodes[B->parent].child[0] = b_id;
                else nodes[B->parent].child[1] = b_id;
            } else {
                root = b_id;
            }
            if (F->height > G->height) {
                B->child[1] = f_id;
                A->child[0] = g_id;
                G->parent = a_id;
                A->box = merge(C->box, G->box);
                B->box = merge(A->box, F->box);
                A->height = (C->height < G->height ? G->height : C->height) + 1;
                B->height = (A->height < F->height ? F->height : A->height) + 1;
            } else {
                B->child[1] = g_id;
                A->child[0] = f_id;
                F->parent = a_id;
                A->box = merge(C->box, F->box);
                B->box = merge(A->box, G->box);
                A->height = (C->height < F->height ? F->height : C->height) + 1;
                B->height = (A->height < G->height ? G->height : A->height) + 1;
            }
            return b_id;
        }
        return a_id;
    }

    ORDER_NO_EXEC_CHECK
    ORDER_HD void refit_up(int cur) {
        while (cur != NIL) {
            cur = balance(cur);
            const int l = nodes[cur].child[0], r = nodes[cur].child[1];
            nodes[cur].height = (nodes[l].height < nodes[r].height ? nodes[r].height : nodes[l].height) + 1;
            nodes[cur].box = merge(nodes[l].box, nodes[r].box);
            cur = nodes[cur].parent;
        }
    }

    ORDER_NO_EXEC_CHECK
    ORDER_HD void insert_leaf(int id) {
        if (root == NIL) {
            root = id;
            nodes[id].parent = NIL;
            return;
        }
        const Box nb = nodes[id].box;
        int cur = root;
        while (!leaf(cur)) {
            const int l = nodes[cur].child[0], r = nodes[cur].child[1];
            const float vol = volume(nodes[cur].box);
            const float merged = volume(merge(nodes[cur].box, nb));
            const float costS = 2.0f * merged;
            const float costI = 2.0f * (merged - vol);
            float costL, costR;
            const float vl = volume(merge(nb, nodes[l].box));
            if (leaf(l)) costL = vl + costI;
            else costL = costI + vl - volume(nodes[l].box);
            const float vr = volume(merge(nb, nodes[r].box));
            if (leaf(r)) costR = vr + costI;
            else costR = costI + vr - volume(nodes[r].box);
            if (costS < costL && costS < costR) break;
            cur = costL < costR ? l : r;
        }
        const int sib = cur;
        const int old_parent = nodes[sib].parent;
        const int np = alloc();
        if (np == NIL) return;
        nodes[np].parent = old_parent;
        nodes[np].box = merge(nodes[sib].box, nb);
        nodes[np].height = nodes[sib].height + 1;
        if (old_parent != NIL) {
            if (nodes[old_parent].child[0] == sib) nodes[old_parent].child[0] = np;
            else nodes[old_parent].child[1] = np;
        } else {
            root = np;
        }
        nodes[np].child[0] = sib;
        nodes[np].child[1] = id;
        nodes[sib].parent = np;
        nodes[id].parent = np;
        refit_up(nodes[id].parent);
    }

    ORDER_NO_EXEC_CHECK
    ORDER_HD void remove_leaf(int id) {
        if (root == id) {
            root = NIL;
            return;
        }
        const int parent = nodes[id].parent;
        const int grand = nodes[parent].parent;
        const int sib = nodes[parent].child[0] == id ? nodes[parent].child[1] : nodes[parent].child[0];
        if (grand != NIL) {
            if (nodes[grand].child[0] == parent) nodes[grand].child[0] = sib;
            else nodes[grand].child[1] = sib;
            nodes[sib].parent = grand;
            release(parent);
            refit_up(grand);
        } else {
            root = sib;
            nodes[sib].parent = NIL;
            release(parent);
        }
    }

    // updateObject after the fat-AABB test failed (the new fat AABB given)
    ORDER_NO_EXEC_CHECK
    ORDER_HD void reinsert(int id, const Box& fat) {
        remove_leaf(id);
        nodes[id].box = fat;
        insert_leaf(id);
    }
};

// The host replica: nodes in a vector that grows as the reference's array.
struct Tree : TreeT<std::vector<TreeNode>> {
    Tree() { init(); }

    // DynamicAABBTree::init (GLOBAL_ALIGNMENT = 16 nodes to start with)
    void init() {
        nodes.assign(16, Node());
        for (int i = 0; i < 15; i++) nodes[size_t(i)].parent = i + 1;
        nodes[15].parent = NIL;
        root = NIL;
        free_id = 0;
        nb_nodes = 0;
    }

    // addObject with the fat AABB already inflated (addObjectInternal)
    int add_object(const Box& fat, int data) {
        const int id = alloc();
        nodes[size_t(id)].box = fat;
        nodes[size_t(id)].height = 0;
        nodes[size_t(id)].data = data;
        insert_leaf(id);
        return id;
    }

    // reportAllShapesOverlappingWithShapes for one shape: leaves in the
    // stack order (children[1] popped before children[0])
    void query(const Box& box, std::vector<int>& out, std::vector<int>& stack) const {
        stack.clear();
        stack.push_back(root);
        while (!stack.empty()) {
            const int id = stack.back();
            stack.pop_back();
            if (id == NIL) continue;
            const Node& n = nodes[size_t(id)];
            if (overlap(box, n.box)) {
                if (n.height == 0) {
                    out.push_back(id);
                } else {
                    stack.push_back(n.child[0]);
                    stack.push_back(n.child[1]);
                }
            }
        }
    }
};

// One world's tree in a world group's device pool.
using DevTree = TreeT<NodeSpan>;

// Set<int32> with std::hash<int32> (identity).
struct IdSet {
    static constexpr uint64_t INVALID = ~uint64_t(0);
    uint64_t hash_size = 0, nb_alloc = 0, nb = 0, free_idx = INVALID;
    std::vector<uint64_t> buckets, next;
    std::vector<int32_t> entries;

    static uint64_t next_pow2(uint64_t x) {
        uint64_t p = 1;
        while (p < x) p <<= 1;
        return p;
    }
    void reserve(uint64_t cap) {
        if (cap <= hash_size) return;
        if (cap < 16) cap = 16;
        cap = next_pow2(cap);
        std::vector<uint64_t> nbk(cap, INVALID);
        uint64_t na = uint64_t(double(cap) * 0.75);
        na = uint64_t(float(std::ceil(float(na) / float(16))) * 16.0f);
        std::vector<uint64_t> nnext(na, INVALID);
        std::vector<int32_t> nent(na, 0);
        for (uint64_t i = 0; i < nb_alloc; i++) nnext[i] = next[i];
        for (uint64_t i = 0; i < hash_size; i++) {
            uint64_t e = buckets[i];
            while (e != INVALID) {
                const uint64_t b = uint64_t(uint64_t(int64_t(entries[e])) & (cap - 1));
                nnext[e] = nbk[b];
                nbk[b] = e;
                nent[e] = entries[e];
                e = next[e];
            }
        }
        for (uint64_t i = nb_alloc; i + 1 < na; i++) nnext[i] = i + 1;
        nnext[na - 1] = free_idx;
        free_idx = nb_alloc;
        hash_size = cap;
        nb_alloc = na;
        buckets.swap(nbk);
        next.swap(nnext);
        entries.swap(nent);
    }
    bool add(int32_t v) {
        const uint64_t h = uint64_t(int64_t(v));
        uint64_t b = INVALID;
        if (hash_size > 0) {
            b = h & (hash_size - 1);
            for (uint64_t i = buckets[b]; i != INVALID; i = next[i])
                if (entries[i] == v) return false;
        }
        if (free_idx == INVALID) {
            reserve(hash_size == 0 ? 16 : hash_size * 2);
            b = h & (hash_size - 1);
        }
        const uint64_t e = free_idx;
        free_idx = next[e];
        nb++;
        next[e] = buckets[b];
        entries[e] = v;
        buckets[b] = e;
        return true;
    }
    void clear() {
        for (uint64_t i = 0; i < hash_size; i++) {
            uint64_t e = buckets[i];
            while (e != INVALID) {
                const uint64_t n = next[e];
                next[e] = free_idx;
                free_idx = e;
                e = n;
            }
            buckets[i] = INVALID;
        }
        nb = 0;
    }
    void to_array(std::vector<int32_t>& out) const {
        out.clear();
        for (uint64_t i = 0; i < hash_size; i++)
            for (uint64_t e = buckets[i]; e != INVALID; e = next[e]) out.push_back(entries[e]);
    }
};

// Pair id -> index in its pair array (OverlappingPairs' mMapConvexPairIdToPairIndex
// and the three other maps; only looked up, never iterated, so its order is
// free): open addressing with linear probing, deletion by backward shift,
// at most half full.  find / end / operator[] / erase as std::unordered_map.
struct PairMap {
    static constexpr uint64_t EMPTY = ~uint64_t(0);
    struct Entry {
        uint64_t first = EMPTY;
        uint32_t second = 0;
    };
    std::vector<Entry> slots;
    uint32_t mask = 0;
    size_t n = 0;

    static uint32_t hash(uint64_t k) {
        k ^= k >> 33;
        k *= 0xff51afd7ed558ccdull;
        k ^= k >> 33;
        return uint32_t(k);
    }
    Entry* end() const { return nullptr; }
    bool empty() const { return n == 0; }
    Entry* find(uint64_t k) {
        if (!n) return nullptr;
        for (uint32_t h = hash(k) & mask;; h = (h + 1) & mask) {
            if (slots[h].first == k) return &slots[h];
            if (slots[h].first == EMPTY) return nullptr;
        }
    }
    void rehash(size_t cap) {
        std::vector<Entry> old;
        old.swap(slots);
        slots.assign(cap, Entry());
        mask = uint32_t(cap - 1);
        for (const Entry& e : old)
            if (e.first != EMPTY) {
                uint32_t h = hash(e.first) & mask;
                while (slots[h].first != EMPTY) h = (h + 1) & mask;
                slots[h] = e;
            }
    }
    uint32_t& operator[](uint64_t k) {
        if (2 * (n + 1) > slots.size()) rehash(std::max<size_t>(16, 2 * slots.size()));
        uint32_t h = hash(k) & mask;
        while (slots[h].first != EMPTY && slots[h].first != k) h = (h + 1) & mask;
        if (slots[h].first == EMPTY) {
            slots[h].first = k;
            slots[h].second = 0;
            n++;
        }
        return slots[h].second;
    }
    void erase(uint64_t k) {
        Entry* e = find(k);
        if (!e) return;
        uint32_t i = uint32_t(e - slots.data()), j = i;
        for (;;) {
            j = (j + 1) & mask;
            if (slots[j].first == EMPTY) break;
            const uint32_t home = hash(slots[j].first) & mask;
            // the entry at j stays where it is if its home lies cyclically in (i, j]
            const bool stays = i <= j ? (i < home && home <= j) : (i < home || home <= j);
            if (stays) continue;
            slots[i] = slots[j];
            i = j;
        }
        slots[i] = Entry();
        n--;
    }
};

// Component order: ids at slots, enabled ones first.
struct Comps {
    std::vector<int> at;    // slot -> id
    std::vector<int> slot;  // id -> slot
    uint32_t n_enabled = 0;

    void reserve_ids(size_t n) { slot.resize(n, -1); }
    void place(int id, uint32_t s) {
        if (s >= at.size()) at.resize(size_t(s) + 1, -1);
        at[s] = id;
        slot[size_t(id)] = int(s);
    }
    // prepareAddComponent + addComponent
    void add(int id, bool disabled) {
        const uint32_t n = uint32_t(at.size());
        if (disabled) {
            place(id, n);
            return;
        }
        if (n_enabled != n) place(at[n_enabled], n);  // moveComponentToIndex(first disabled, end)
        place(id, n_enabled);
        n_enabled++;
    }
    void swap_slots(uint32_t a, uint32_t b) {
        const int ia = at[a], ib = at[b];
        place(ia, b);
        place(ib, a);
    }
    // Components::setIsEntityDisabled
    void set_disabled(int id, bool dis) {
        const uint32_t s = uint32_t(slot[size_t(id)]);
        if (!dis && s >= n_enabled) {
            if (n_enabled != s) swap_slots(s, n_enabled);
            n_enabled++;
        } else if (dis && s < n_enabled) {
            if (s != n_enabled - 1) swap_slots(s, n_enabled - 1);
            n_enabled--;
        }
    }
    bool enabled(int id) const { return uint32_t(slot[size_t(id)]) < n_enabled; }
};

}  // namespace order
}  // namespace rp3dg
