// The world broadphase's dynamic tree, restated only as far as the order in
// which a query reports static proxies.
//
// b3DynamicTree (src/bounce/collision/trees/dynamic_tree.cpp:107-117,
// 144-260) inserts a proxy as a new leaf next to the sibling of least
// surface-area cost, with a new parent holding (sibling, leaf) as (child1,
// child2), and refits the ancestors.  Its QueryAABB
// (include/bounce/collision/trees/dynamic_tree.h:152-183) walks the tree with
// a stack, pushing child1 then child2, so child2's subtree is reported first.
// Leaves whose subtree misses the query AABB are skipped, which never
// changes the relative order of two reported leaves: the report order is the
// child2-first depth-first order of the leaves.  The cost arithmetic follows
// the reference's float expressions, so ties and near-ties fall the same
// way.
#include "broadphase_order.h"

#include <vector>

namespace b3g {

namespace {

struct Node {
    float lo[3], hi[3];
    int parent = -1, child1 = -1, child2 = -1;
    int height = 0;
    int shape = -1;  // leaves: the shape they stand for
    bool leaf() const { return child1 < 0; }
};

// b3AABB3::SurfaceArea (include/bounce/collision/shapes/aabb3.h:130-133)
float area(const float lo[3], const float hi[3])
{
    const float w = hi[0] - lo[0], h = hi[1] - lo[1], d = hi[2] - lo[2];
    return 2.0f * (w * d + w * h + d * h);
}

// b3Combine (aabb3.h:238-244)
void combine(const float alo[3], const float ahi[3], const float blo[3], const float bhi[3], float lo[3],
             float hi[3])
{
    for (int q = 0; q < 3; ++q) {
        lo[q] = alo[q] < blo[q] ? alo[q] : blo[q];
        hi[q] = ahi[q] > bhi[q] ? ahi[q] : bhi[q];
    }
}

struct Tree {
    std::vector<Node> nodes;
    int root = -1;

    // FindBest: descend while a child is cheaper than a new parent here
    int find_best(const float lo[3], const float hi[3]) const
    {
        int index = root;
        while (!nodes[index].leaf()) {
            const Node& nd = nodes[index];
            const float branch_area = area(nd.lo, nd.hi);
            float clo[3], chi[3];
            combine(lo, hi, nd.lo, nd.hi, clo, chi);
            const float combined_area = area(clo, chi);
            const float branch_cost = 2.0f * combined_area;
            const float inheritance_cost = 2.0f * (combined_area - branch_area);
            float cost[2];
            const int kids[2] = {nd.child1, nd.child2};
            for (int k = 0; k < 2; ++k) {
                const Node& ch = nodes[kids[k]];
                float xlo[3], xhi[3];
                combine(lo, hi, ch.lo, ch.hi, xlo, xhi);
                cost[k] = ch.leaf() ? area(xlo, xhi) : (area(xlo, xhi) - area(ch.lo, ch.hi)) + inheritance_cost;
            }
            if (branch_cost < cost[0] && branch_cost < cost[1]) break;
            index = cost[0] < cost[1] ? kids[0] : kids[1];
        }
        return index;
    }

    void insert(int leaf)
    {
        if (root < 0) {
            root = leaf;
            nodes[leaf].parent = -1;
            return;
        }
        const int sibling = find_best(nodes[leaf].lo, nodes[leaf].hi);
        const int old_parent = nodes[sibling].parent;
        nodes.push_back(Node());
        const int np = (int)nodes.size() - 1;
        nodes[np].parent = old_parent;
        nodes[np].child1 = sibling;
        nodes[np].child2 = leaf;
        nodes[sibling].parent = np;
        nodes[leaf].parent = np;
        if (old_parent >= 0) {
            if (nodes[old_parent].child1 == sibling) nodes[old_parent].child1 = np;
            else nodes[old_parent].child2 = np;
        } else {
            root = np;
        }
        // refit the ancestors (WalkBackNodeAndCombineVolumes)
        for (int a = np; a >= 0; a = nodes[a].parent) {
            const Node &c1 = nodes[nodes[a].child1], &c2 = nodes[nodes[a].child2];
            nodes[a].height = 1 + (c1.height > c2.height ? c1.height : c2.height);
            combine(c1.lo, c1.hi, c2.lo, c2.hi, nodes[a].lo, nodes[a].hi);
        }
    }
};

}  // namespace

void query_report_ranks(const float (*lo)[3], const float (*hi)[3], uint32_t count, uint32_t* rank)
{
    if (count == 0) return;
    Tree t;
    t.nodes.reserve(2 * (size_t)count);
    for (uint32_t s = 0; s < count; ++s) {
        Node leaf;
        for (int q = 0; q < 3; ++q) {
            leaf.lo[q] = lo[s][q];
            leaf.hi[q] = hi[s][q];
        }
        leaf.shape = (int)s;
        t.nodes.push_back(leaf);
        t.insert((int)t.nodes.size() - 1);
    }
    // report order: a stack with child1 pushed before child2
    std::vector<int> stack{t.root};
    uint32_t next = 0;
    while (!stack.empty()) {
        const int nd = stack.back();
        stack.pop_back();
        if (t.nodes[nd].leaf()) {
            rank[t.nodes[nd].shape] = next++;
        } else {
            stack.push_back(t.nodes[nd].child1);
            stack.push_back(t.nodes[nd].child2);
        }
    }
}

}  // namespace b3g
