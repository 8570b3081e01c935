/* Test infrastructure (the oracle): the order in which a world AABB query
 * reports static shape proxies, restated from b3DynamicTree
 * (src/bounce/collision/trees/dynamic_tree.cpp:144-260, InsertLeaf with
 * FindBest and the ancestor refit; include/bounce/collision/trees/
 * dynamic_tree.h:152-183, QueryAABB).  Proxies are inserted in shape order;
 * a query pops child2 before child1, so among the shapes it reports, order
 * is the child2-first depth-first order of the leaves.  Bounce pushes each
 * new contact to its list's front as the shape is reported. */
#ifndef ORACLE_WORLD_ORDER_H
#define ORACLE_WORLD_ORDER_H

#include <stdint.h>

#define WO_MAX 8 /* shapes; nodes are 2 * WO_MAX - 1 */

typedef struct {
    float lo[3], hi[3];
    int parent, c1, c2;
    int shape; /* leaves: the shape; -1 for inner nodes */
} wo_node;

static float wo_area(const float* lo, const float* hi) /* b3AABB3::SurfaceArea */
{
    float w = hi[0] - lo[0], h = hi[1] - lo[1], d = hi[2] - lo[2];
    return 2.0f * (w * d + w * h + d * h);
}

static void wo_union(const float* alo, const float* ahi, const float* blo, const float* bhi, float* lo, float* hi)
{
    for (int q = 0; q < 3; ++q) {
        lo[q] = alo[q] < blo[q] ? alo[q] : blo[q];
        hi[q] = ahi[q] > bhi[q] ? ahi[q] : bhi[q];
    }
}

/* order[k]: the shape reported k-th */
static void world_report_order(const float (*lo)[3], const float (*hi)[3], uint32_t count, uint32_t* order)
{
    wo_node nd[2 * WO_MAX];
    int nnodes = 0, root = -1;
    for (uint32_t s = 0; s < count && s < WO_MAX; ++s) {
        int leaf = nnodes++;
        for (int q = 0; q < 3; ++q) {
            nd[leaf].lo[q] = lo[s][q];
            nd[leaf].hi[q] = hi[s][q];
        }
        nd[leaf].c1 = nd[leaf].c2 = -1;
        nd[leaf].parent = -1;
        nd[leaf].shape = (int)s;
        if (root < 0) {
            root = leaf;
            continue;
        }
        int at = root;
        while (nd[at].c1 >= 0) {
            float ulo[3], uhi[3];
            wo_union(nd[leaf].lo, nd[leaf].hi, nd[at].lo, nd[at].hi, ulo, uhi);
            float here = wo_area(nd[at].lo, nd[at].hi), joint = wo_area(ulo, uhi);
            float new_parent = 2.0f * joint, inherit = 2.0f * (joint - here);
            float c[2];
            for (int k = 0; k < 2; ++k) {
                const wo_node* ch = nd + (k == 0 ? nd[at].c1 : nd[at].c2);
                float xlo[3], xhi[3];
                wo_union(nd[leaf].lo, nd[leaf].hi, ch->lo, ch->hi, xlo, xhi);
                c[k] = ch->c1 < 0 ? wo_area(xlo, xhi) : (wo_area(xlo, xhi) - wo_area(ch->lo, ch->hi)) + inherit;
            }
            if (new_parent < c[0] && new_parent < c[1]) break;
            at = c[0] < c[1] ? nd[at].c1 : nd[at].c2;
        }
        int p = nnodes++, gp = nd[at].parent;
        nd[p].shape = -1;
        nd[p].parent = gp;
        nd[p].c1 = at;
        nd[p].c2 = leaf;
        nd[at].parent = p;
        nd[leaf].parent = p;
        if (gp < 0) root = p;
        else if (nd[gp].c1 == at) nd[gp].c1 = p;
        else nd[gp].c2 = p;
        for (int a = p; a >= 0; a = nd[a].parent)
            wo_union(nd[nd[a].c1].lo, nd[nd[a].c1].hi, nd[nd[a].c2].lo, nd[nd[a].c2].hi, nd[a].lo, nd[a].hi);
    }
    int stack[2 * WO_MAX], top = 0;
    uint32_t k = 0;
    if (root >= 0) stack[top++] = root;
    while (top > 0) {
        int a = stack[--top];
        if (nd[a].c1 < 0) {
            order[k++] = (uint32_t)nd[a].shape;
        } else {
            stack[top++] = nd[a].c1;
            stack[top++] = nd[a].c2;
        }
    }
}

#endif
