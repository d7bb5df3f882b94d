// Randomised checks of the world step's host structures (test program, built
// and run by tests/test_host_structures.py):
//   1. PairMap against std::unordered_map under random inserts, updates,
//      erases and lookups;
//   2. the tree code on a device-style node span holding only the nodes in
//      use plus the free list's head (what a world group's device pool
//      holds), against the host tree, under random reinsertions: every
//      access must stay inside the span and both trees must end identical.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <unordered_map>
#include <vector>

#include "../../reactphysics3d_b200/csrc/world_order.h"

using namespace rp3dg::order;

struct CheckedSpan {
    TreeNode* p = nullptr;
    int n = 0;
    TreeNode& operator[](int i) const {
        if (i < 0 || i >= n) {
            std::printf("node %d outside the span of %d\n", i, n);
            std::exit(1);
        }
        return p[i];
    }
    int size() const { return n; }
};
inline bool grow_nodes(CheckedSpan&, int, int&) { return false; }

static int pair_map_fuzz() {
    std::mt19937_64 rng(7);
    for (int trial = 0; trial < 200; trial++) {
        PairMap m;
        std::unordered_map<uint64_t, uint32_t> ref;
        const uint64_t range = 1 + rng() % 4000;
        for (int op = 0; op < 20000; op++) {
            const uint64_t k = ((rng() % range) * 0x9E3779B97F4A7C15ull) >> (rng() % 3);
            const int r = int(rng() % 10);
            if (r < 5) {
                const uint32_t v = uint32_t(rng());
                m[k] = v;
                ref[k] = v;
            } else if (r < 8) {
                m.erase(k);
                ref.erase(k);
            } else {
                const PairMap::Entry* e = m.find(k);
                const auto it = ref.find(k);
                if ((e == nullptr) != (it == ref.end()) || (e && e->second != it->second)) return 1;
            }
            if (m.n != ref.size()) return 2;
        }
        for (const auto& kv : ref) {
            const PairMap::Entry* e = m.find(kv.first);
            if (!e || e->second != kv.second) return 3;
        }
    }
    return 0;
}

static int tree_span_fuzz() {
    std::mt19937 rng(3);
    std::uniform_real_distribution<float> U(-50.f, 50.f), S(0.1f, 3.f);
    auto box = [&]() {
        Box b;
        for (int k = 0; k < 3; k++) {
            const float c = U(rng), h = S(rng);
            b.mn[k] = c - h;
            b.mx[k] = c + h;
        }
        return b;
    };
    for (int trial = 0; trial < 300; trial++) {
        Tree host;
        const int nleaves = 1 + int(rng() % 400);
        std::vector<int> leaves;
        for (int i = 0; i < nleaves; i++) leaves.push_back(host.add_object(box(), i));
        const int n = std::min<int>(int(host.nodes.size()), host.nb_nodes + 1);
        std::vector<TreeNode> span(host.nodes.begin(), host.nodes.begin() + n);
        TreeT<CheckedSpan> dev;
        dev.nodes.p = span.data();
        dev.nodes.n = n;
        dev.root = host.root;
        dev.free_id = host.free_id;
        dev.nb_nodes = host.nb_nodes;
        for (int op = 0; op < 2000; op++) {
            const int leaf = leaves[rng() % leaves.size()];
            const Box b = box();
            host.reinsert(leaf, b);
            dev.reinsert(leaf, b);
            if (dev.failed) return 4;
        }
        if (host.root != dev.root || host.free_id != dev.free_id || host.nb_nodes != dev.nb_nodes) return 5;
        for (int i = 0; i < n; i++) {
            const TreeNode &a = host.nodes[size_t(i)], &c = span[size_t(i)];
            if (a.parent != c.parent || a.child[0] != c.child[0] || a.child[1] != c.child[1] || a.height != c.height)
                return 6;
            for (int k = 0; k < 3; k++)
                if (a.box.mn[k] != c.box.mn[k] || a.box.mx[k] != c.box.mx[k]) return 7;
        }
    }
    return 0;
}

int main() {
    const int a = pair_map_fuzz();
    const int b = tree_span_fuzz();
    std::printf("pair map %d tree span %d\n", a, b);
    return a || b;
}
