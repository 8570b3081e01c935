// Host check of the slot-major assembly's term lists (topology.cpp,
// build_slot_terms), built by tests/test_slot_terms.py with g++.
//
// For grid cloths with bending springs, sewing springs, created particles and
// mouse forces it checks, from the meaning of a term rather than from how the
// lists are built:
//   * every term of block (row r, slot k) names an element that holds r at
//     the term's row corner and the block's column at its column corner;
//   * the terms of a block follow the row's force-list (incidence) order;
//   * every element appears in exactly (vertices)^2 block lists: 9 for a
//     triangle, 4 for a spring, 16 for a mouse force;
//   * the codes sit where the kernel reads them (term j of the block at SELL
//     position slice_off[q] + 32 k + lane at term_qk[slice_off[q] / 32 + k]
//     + 32 j + lane), inside the array.
// Prints one line per case and exits non-zero on the first failure.
#include <cstdio>
#include <map>
#include <vector>

#include "../bounce_b200/csrc/topology.h"

using namespace b3g;

static int fail(const char* what, int side, uint32_t r, uint32_t k)
{
    std::printf("FAIL side %d row %u slot %u: %s\n", side, r, k, what);
    return 1;
}

int main()
{
    const int sides[] = {2, 5, 20, 37};
    for (int side : sides) {
        std::vector<float> X;
        std::vector<uint32_t> T;
        for (int i = 0; i < side; ++i)
            for (int j = 0; j < side; ++j) {
                X.push_back((float)j);
                X.push_back(0.0f);
                X.push_back((float)i);
            }
        for (int i = 0; i + 1 < side; ++i)
            for (int j = 0; j + 1 < side; ++j) {
                const uint32_t v1 = i * side + j, v2 = v1 + 1, v3 = v1 + side + 1, v4 = v1 + side;
                T.insert(T.end(), {v3, v2, v1, v1, v4, v3});
            }
        const uint32_t n0 = (uint32_t)(side * side), t = (uint32_t)(T.size() / 3);
        // a sewing line between the first and last vertex of the first row
        const uint32_t sew[4] = {0, 0, 0, (uint32_t)(side - 1)};
        const float def[8] = {1.0f, 1e4f, 1e3f, 1e2f, 1e3f, 0.05f, 0.0f, 0.0f};
        // two created particles, each tied to a triangle by a mouse force
        const MouseForceDesc mice[2] = {{n0, 0, 0.2f, 0.3f, 0.5f, 800.0f, 4.0f},
                                        {n0 + 1, t - 1, 0.1f, 0.6f, 0.3f, 500.0f, 0.0f}};
        ClothTopology c;
        const int rc = build_topology(n0, X.data(), t, T.data(), 1, sew, def, &c, 2, mice, 2);
        if (rc != 0) {
            std::printf("FAIL side %d: build_topology %d\n", side, rc);
            return 1;
        }
        if (!c.slot_terms) return fail("no term lists", side, 0, 0);
        if (c.term_qk.size() != c.E / 32 || c.term_slot.size() != c.E) return fail("array sizes", side, 0, 0);
        // element vertices: triangles, springs, mouse forces
        auto verts = [&](uint32_t code, uint32_t out[4]) -> uint32_t {
            const uint32_t id = code & ((1u << kTermIdBits) - 1u), kind = code >> 30;
            if (kind == 0) {
                for (int q = 0; q < 3; ++q) out[q] = T[3 * id + q];
                return 3;
            }
            if (kind == 2) {
                out[0] = c.spring_pairs[2 * id];
                out[1] = c.spring_pairs[2 * id + 1];
                return 2;
            }
            out[0] = mice[id].particle;
            for (int q = 0; q < 3; ++q) out[q + 1] = T[3 * mice[id].triangle + q];
            return 4;
        };
        std::map<uint32_t, uint32_t> seen;  // code without corners -> count
        size_t used = 0;
        for (uint32_t r = 0; r < c.n; ++r) {
            const uint32_t q = r / 32, lane = r % 32, base = c.slice_off[q] + lane;
            // the row's elements in force-list order, as kind|id keys
            std::vector<uint32_t> order;
            for (uint32_t e = c.inc_ptr[r]; e < c.inc_ptr[r + 1]; ++e) {
                const uint32_t el = c.inc_elem[e];
                if ((el & 0xc0000000u) == 0xc0000000u) order.push_back(kTermKindMouse | (el & 0x3fffffffu));
                else if (el & 0x80000000u) order.push_back(kTermKindSpring | (el & 0x7fffffffu));
                else order.push_back(el);
            }
            for (uint32_t k = 0; k < c.row_deg[r]; ++k) {
                const uint32_t col = c.sell_cols[base + 32 * k], cnt = c.term_slot[base + 32 * k];
                const size_t first = (size_t)c.term_qk[(base >> 5) + k] + lane;
                size_t pos_in_order = 0;
                for (uint32_t j = 0; j < cnt; ++j) {
                    const size_t at = first + 32 * (size_t)j;
                    if (at >= c.terms.size()) return fail("term outside the array", side, r, k);
                    const uint32_t code = c.terms[at];
                    uint32_t v[4];
                    const uint32_t nv = verts(code, v);
                    const uint32_t cr = (code >> 28) & 3u, cj = (code >> 26) & 3u;
                    if (cr >= nv || cj >= nv || v[cr] != r || v[cj] != col)
                        return fail("term does not couple the row and the column", side, r, k);
                    const uint32_t key = code & ~(15u << 26);
                    // non-decreasing position in the row's force list
                    size_t p = pos_in_order;
                    while (p < order.size() && order[p] != key) ++p;
                    if (p == order.size()) return fail("term out of force-list order", side, r, k);
                    pos_in_order = p;
                    seen[key] += 1;
                    ++used;
                }
            }
        }
        for (const auto& kv : seen) {
            const uint32_t kind = kv.first >> 30;
            const uint32_t want = kind == 0 ? 9u : kind == 2 ? 4u : 16u;
            if (kv.second != want) return fail("element in the wrong number of blocks", side, kv.first, kv.second);
        }
        if (seen.size() != (size_t)t + c.ns + 2) return fail("an element has no terms", side, 0, 0);
        std::printf("side %d: %u rows, %u blocks, %zu terms in %zu slots, max degree %u\n", side, c.n,
                    (unsigned)c.row_cols.size(), used, c.terms.size(), c.max_deg);
    }
    std::printf("ok\n");
    return 0;
}
