#include "topology.h"

#include <algorithm>
#include <cmath>
#include <tuple>

namespace b3g {

namespace {

struct V3 {
    float x, y, z;
};
inline V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float len(V3 v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
inline V3 divs(V3 v, float s) { return V3{v.x / s, v.y / s, v.z / s}; }
inline V3 at(const float* p, uint32_t i) { return V3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }

struct DEdge {
    uint32_t a, b, tri, slot;
    bool operator<(const DEdge& o) const { return std::tie(a, b, tri, slot) < std::tie(o.a, o.b, o.tri, o.slot); }
};

constexpr int kOk = 0, kDegenerate = 2, kUnsupported = 9;
constexpr uint32_t kMaxDegree = 64;

}  // namespace

void bending_pairs(uint32_t t, const uint32_t* tris, std::vector<uint32_t>* pairs)
{
    std::vector<DEdge> edges(3 * (size_t)t);
    for (uint32_t k = 0; k < t; ++k)
        for (uint32_t e = 0; e < 3; ++e) edges[3 * k + e] = DEdge{tris[3 * k + e], tris[3 * k + (e + 1) % 3], k, e};
    std::sort(edges.begin(), edges.end());
    pairs->clear();
    for (uint32_t i = 0; i < t; ++i) {
        const uint32_t* t1 = tris + 3 * i;
        for (uint32_t j1 = 0; j1 < 3; ++j1) {
            uint32_t k1 = j1 + 1 < 3 ? j1 + 1 : 0;
            uint32_t a = t1[j1], b = t1[k1];
            auto it = std::lower_bound(edges.begin(), edges.end(), DEdge{b, a, i + 1, 0});
            uint32_t last = UINT32_MAX;
            for (; it != edges.end() && it->a == b && it->b == a; ++it) {
                if (it->tri == last) continue;
                last = it->tri;
                const uint32_t* t2 = tris + 3 * it->tri;
                uint32_t k2 = it->slot + 1 < 3 ? it->slot + 1 : 0;
                uint32_t k3 = k1 + 1 < 3 ? k1 + 1 : 0;
                uint32_t k4 = k2 + 1 < 3 ? k2 + 1 : 0;
                pairs->push_back(t1[k3]);
                pairs->push_back(t2[k4]);
            }
        }
    }
}

int build_topology(uint32_t n, const float* X, uint32_t t, const uint32_t* tris, uint32_t nsew,
                   const uint32_t* sewing, const float* def, ClothTopology* out, uint32_t n_extra,
                   const MouseForceDesc* mice, uint32_t nmice, bool slot_terms)
{
    ClothTopology& c = *out;
    c.n_mesh = n;
    c.t = t;
    for (uint64_t k = 0; k < 3ull * t; ++k)
        if (tris[k] >= n) return kDegenerate;
    for (uint32_t s = 0; s < nsew; ++s)
        if (sewing[4 * s + 2] >= n || sewing[4 * s + 3] >= n) return kDegenerate;

    // lumped masses (cloth.cpp:388-427)
    c.mass.assign(n, 0.0f);
    const float inv3 = 1.0f / 3.0f, rho = def[0];
    for (uint32_t k = 0; k < t; ++k) {
        V3 a = at(X, tris[3 * k]), b = at(X, tris[3 * k + 1]), cc = at(X, tris[3 * k + 2]);
        float area = 0.5f * len(cross(sub(b, a), sub(cc, a)));
        if (!(area > 0.0f)) return kDegenerate;
        float m = rho * area;
        for (int q = 0; q < 3; ++q) c.mass[tris[3 * k + q]] += inv3 * m;
    }
    for (uint32_t i = 0; i < n; ++i)
        if (!(c.mass[i] > 0.0f)) return kDegenerate;  // a vertex outside every triangle
    const uint32_t n_mesh = n;
    n += n_extra;
    c.n = n;
    c.mass.resize(n, 1.0f);
    for (uint32_t m = 0; m < nmice; ++m) {
        const MouseForceDesc& f = mice[m];
        if (f.particle >= n || f.triangle >= t) return kDegenerate;
    }

    // rest-state frames (cloth.cpp:152-191)
    c.rest.resize(6 * (size_t)t);
    for (uint32_t k = 0; k < t; ++k) {
        V3 A = at(X, tris[3 * k]), B = at(X, tris[3 * k + 1]), C = at(X, tris[3 * k + 2]);
        V3 AB = sub(B, A), AC = sub(C, A);
        float u1 = 0.0f, v1 = 0.0f, u2 = len(AB), v2 = 0.0f;
        if (!(u2 > 0.0f)) return kDegenerate;
        V3 n_AB = divs(AB, u2);
        float A2 = len(cross(AB, AC));
        float u3 = dot(AC, n_AB), v3 = A2 / u2;
        float du1 = u2 - u1, dv1 = v2 - v1, du2 = u3 - u1, dv2 = v3 - v1;
        float det = du1 * dv2 - du2 * dv1;
        if (det == 0.0f) return kDegenerate;
        float* r = &c.rest[6 * (size_t)k];
        r[0] = du1; r[1] = dv1; r[2] = du2; r[3] = dv2; r[4] = 1.0f / det; r[5] = 0.5f * A2;
    }

    // springs in creation order: bending (cloth.cpp:227-243), sewing (:248-262)
    c.spring_pairs.clear();
    c.spring_par.clear();
    if (def[3] > 0.0f) {
        std::vector<uint32_t> bp;
        bending_pairs(t, tris, &bp);
        for (size_t q = 0; q < bp.size(); q += 2) {
            c.spring_pairs.push_back(bp[q]);
            c.spring_pairs.push_back(bp[q + 1]);
            c.spring_par.push_back(len(sub(at(X, bp[q]), at(X, bp[q + 1]))));
            c.spring_par.push_back(def[3]);
            c.spring_par.push_back(def[5]);
        }
    }
    if (def[4] > 0.0f) {
        for (uint32_t s = 0; s < nsew; ++s) {
            uint32_t p1 = sewing[4 * s + 2], p2 = sewing[4 * s + 3];
            c.spring_pairs.push_back(p1);
            c.spring_pairs.push_back(p2);
            c.spring_par.push_back(len(sub(at(X, p1), at(X, p2))));
            c.spring_par.push_back(def[4]);
            c.spring_par.push_back(def[5]);
        }
    }
    c.ns = (uint32_t)(c.spring_pairs.size() / 2);

    (void)n_mesh;
    // row pattern
    std::vector<std::vector<uint32_t>> nb(n);
    for (uint32_t i = 0; i < n; ++i) nb[i].push_back(i);
    for (uint32_t k = 0; k < t; ++k)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                if (a != b) nb[tris[3 * k + a]].push_back(tris[3 * k + b]);
    for (uint32_t s = 0; s < c.ns; ++s) {
        uint32_t p = c.spring_pairs[2 * s], q = c.spring_pairs[2 * s + 1];
        if (p != q) {
            nb[p].push_back(q);
            nb[q].push_back(p);
        }
    }
    auto mouse_vertices = [&](uint32_t m, uint32_t (&ids)[4]) {
        ids[0] = mice[m].particle;
        for (int q = 0; q < 3; ++q) ids[q + 1] = tris[3 * (size_t)mice[m].triangle + q];
    };
    for (uint32_t m = 0; m < nmice; ++m) {
        uint32_t ids[4];
        mouse_vertices(m, ids);
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b)
                if (ids[a] != ids[b]) nb[ids[a]].push_back(ids[b]);
    }
    c.row_ptr.assign(n + 1, 0);
    c.row_cols.clear();
    c.max_deg = 0;
    for (uint32_t i = 0; i < n; ++i) {
        auto& v = nb[i];
        std::sort(v.begin() + 1, v.end());
        v.erase(std::unique(v.begin() + 1, v.end()), v.end());
        // drop a repeated diagonal
        v.erase(std::remove(v.begin() + 1, v.end(), i), v.end());
        if (v.size() > kMaxDegree) return kUnsupported;
        c.max_deg = std::max<uint32_t>(c.max_deg, (uint32_t)v.size());
        c.row_cols.insert(c.row_cols.end(), v.begin(), v.end());
        c.row_ptr[i + 1] = (uint32_t)c.row_cols.size();
    }
    auto slot_of = [&](uint32_t i, uint32_t j) -> uint32_t {
        if (i == j) return 0;
        auto b = c.row_cols.begin() + c.row_ptr[i] + 1, e = c.row_cols.begin() + c.row_ptr[i + 1];
        return (uint32_t)(std::lower_bound(b, e, j) - (c.row_cols.begin() + c.row_ptr[i]));
    };

    // SELL-32
    c.nslices = (n + 31) / 32;
    c.slice_off.assign(c.nslices + 1, 0);
    c.row_deg.assign(n, 0);
    for (uint32_t q = 0; q < c.nslices; ++q) {
        uint32_t w = 0;
        for (uint32_t r = q * 32; r < std::min(n, q * 32 + 32); ++r) {
            uint32_t d = c.row_ptr[r + 1] - c.row_ptr[r];
            c.row_deg[r] = (uint8_t)d;
            w = std::max(w, d);
        }
        c.slice_off[q + 1] = c.slice_off[q] + 32 * w;
    }
    c.E = c.slice_off[c.nslices];
    c.sell_cols.assign(c.E, 0);
    for (uint32_t r = 0; r < n; ++r) {
        uint32_t q = r / 32, lane = r % 32;
        uint32_t w = (c.slice_off[q + 1] - c.slice_off[q]) / 32;
        for (uint32_t k = 0; k < w; ++k) {
            uint32_t d = c.row_deg[r];
            c.sell_cols[c.slice_off[q] + 32 * k + lane] = k < d ? c.row_cols[c.row_ptr[r] + k] : r;
        }
    }

    // incidence in force-list order: mouse forces newest first (created after
    // the constructor's forces, cloth.cpp:353-358), springs newest first, then
    // triangles newest first (each triangle's shear element precedes its
    // stretch element)
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> inc(n);
    for (uint32_t m = nmice; m-- > 0;) {
        uint32_t ids[4];
        mouse_vertices(m, ids);
        for (uint32_t role = 0; role < 4; ++role) {
            const uint32_t i = ids[role];
            uint32_t meta = role;
            for (int q = 0; q < 4; ++q) meta |= slot_of(i, ids[q]) << (4 + 7 * q);
            inc[i].push_back({kIncSpring | kIncMouse | m, meta});
        }
    }
    for (uint32_t s = c.ns; s-- > 0;) {
        uint32_t p = c.spring_pairs[2 * s], q = c.spring_pairs[2 * s + 1];
        for (uint32_t end = 0; end < 2; ++end) {
            uint32_t i = end == 0 ? p : q;
            uint32_t meta = end | (slot_of(i, p) << 8) | (slot_of(i, q) << 16);
            inc[i].push_back({kIncSpring | s, meta});
        }
    }
    const bool tri_forces = def[1] > 0.0f || def[2] > 0.0f;
    if (tri_forces) {
        for (uint32_t k = t; k-- > 0;) {
            const uint32_t* tv = tris + 3 * k;
            for (uint32_t cn = 0; cn < 3; ++cn) {
                uint32_t i = tv[cn];
                uint32_t meta = cn | (slot_of(i, tv[0]) << 8) | (slot_of(i, tv[1]) << 16) | (slot_of(i, tv[2]) << 24);
                inc[i].push_back({k, meta});
            }
        }
    }
    c.inc_ptr.assign(n + 1, 0);
    c.inc_elem.clear();
    c.inc_meta.clear();
    for (uint32_t i = 0; i < n; ++i) {
        for (auto& pr : inc[i]) {
            c.inc_elem.push_back(pr.first);
            c.inc_meta.push_back(pr.second);
        }
        c.inc_ptr[i + 1] = (uint32_t)c.inc_elem.size();
    }
    if (slot_terms) build_slot_terms(&c);
    else c.slot_terms = false;
    return kOk;
}

void build_slot_terms(ClothTopology* out)
{
    ClothTopology& c = *out;
    c.slot_terms = false;
    c.term_qk.clear();
    c.term_slot.clear();
    c.terms.clear();
    const uint64_t id_limit = 1ull << kTermIdBits;
    if (c.max_deg > kSlotMajorMaxDeg || c.t >= id_limit || c.ns >= id_limit) return;
    c.term_qk.assign(c.E / 32, 0);
    c.term_slot.assign(c.E, 0);
    // per lane of the slice, per slot: the block's terms in the order the
    // row's dfdx accumulation adds them: per element (force-list order) its
    // vertices in element order
    std::vector<std::vector<uint32_t>> per(32 * kSlotMajorMaxDeg);
    for (uint32_t q = 0; q < c.nslices; ++q) {
        for (auto& v : per) v.clear();
        const uint32_t r0 = 32 * q, r1 = std::min(c.n, r0 + 32);
        for (uint32_t i = r0; i < r1; ++i) {
            auto slot_list = [&](uint32_t k) -> std::vector<uint32_t>& { return per[(i - r0) * kSlotMajorMaxDeg + k]; };
            for (uint32_t e = c.inc_ptr[i]; e < c.inc_ptr[i + 1]; ++e) {
                const uint32_t el = c.inc_elem[e], meta = c.inc_meta[e], cn = meta & 3u;
                if ((el & (kIncSpring | kIncMouse)) == (kIncSpring | kIncMouse)) {
                    const uint32_t id = el & ~(kIncSpring | kIncMouse);
                    if (id >= id_limit) return;
                    for (uint32_t v = 0; v < 4; ++v)
                        slot_list((meta >> (4 + 7 * v)) & 0x7fu).push_back(kTermKindMouse | cn << 28 | v << 26 | id);
                } else if (el & kIncSpring) {
                    const uint32_t id = el & ~kIncSpring;
                    for (uint32_t v = 0; v < 2; ++v)
                        slot_list((meta >> (8 + 8 * v)) & 0xffu).push_back(kTermKindSpring | cn << 28 | v << 26 | id);
                } else {
                    for (uint32_t v = 0; v < 3; ++v) slot_list((meta >> (8 + 8 * v)) & 0xffu).push_back(cn << 28 | v << 26 | el);
                }
            }
        }
        // slot k of the slice: term j of lane l at term_qk[.] + 32 j + l
        const uint32_t width = (c.slice_off[q + 1] - c.slice_off[q]) / 32;
        for (uint32_t k = 0; k < width; ++k) {
            size_t w = 0;
            for (uint32_t l = 0; l < r1 - r0; ++l) w = std::max(w, per[l * kSlotMajorMaxDeg + k].size());
            if (w > 255 || c.terms.size() + 32 * w >= (1ull << 32)) return;
            const size_t base = c.terms.size();
            c.term_qk[c.slice_off[q] / 32 + k] = (uint32_t)base;
            c.terms.resize(base + 32 * w, 0u);
            for (uint32_t l = 0; l < r1 - r0; ++l) {
                const auto& v = per[l * kSlotMajorMaxDeg + k];
                for (size_t j = 0; j < v.size(); ++j) c.terms[base + 32 * j + l] = v[j];
                c.term_slot[c.slice_off[q] + 32 * k + l] = (uint32_t)v.size();
            }
        }
    }
    c.slot_terms = true;
}

}  // namespace b3g
