// Soft body preparation on the host.  The element matrices follow the
// reference constructor's float arithmetic step for step (compiled without
// FMA contraction), so the device step starts from bit-identical data:
//   lumped mass rho V / 4 per vertex in element order   softbody.cpp:640-680
//   invE = (e1 e2 e3)^-1 by the adjugate                softbody.cpp:511-520, common/math/math.cpp:111-133
//   D (isotropic elasticity), B (strain-displacement)   softbody.cpp:43-155
//   Ke = V B^T D B as 16 blocks, lower = upper^T        softbody.cpp:522-545, :157-435
//   P = V B^T D                                         softbody.cpp:547-553
#include "softbody_prep.h"

#include <cmath>
#include <cstring>

#include "../../include/b3g.h"

namespace b3g {

namespace {

struct V3 {
    float x, y, z;
};
inline V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

// b3Volume with b3Sign (include/bounce/common/math/vec3.h:226-233, math.h:80-83)
float tet_volume(V3 a, V3 b, V3 c, V3 d)
{
    const float v = dot(sub(b, a), cross(sub(c, a), sub(d, a)));
    const float sign = (float)(0.0f < v) - (float)(v < 0.0f);
    const float inv6 = 1.0f / 6.0f;
    return sign * inv6 * v;
}

// C = A B, column-major, each entry summed from 0 in k order (softbody.cpp:26-42)
void matmul(float* C, const float* A, uint32_t am, uint32_t an, const float* B, uint32_t bm, uint32_t bn)
{
    for (uint32_t i = 0; i < am; ++i)
        for (uint32_t j = 0; j < bn; ++j) {
            float acc = 0.0f;
            for (uint32_t k = 0; k < an; ++k) acc += A[i + am * k] * B[k + bm * j];
            C[i + am * j] = acc;
        }
}

// the element matrices of one tetrahedron (columns e1, e2, e3 of E)
void element_matrices(V3 p1, V3 p2, V3 p3, V3 p4, float E, float nu, float* Ke, float* invE, float* Bo, float* Po)
{
    const float vol = tet_volume(p1, p2, p3, p4);
    const V3 e1 = sub(p2, p1), e2 = sub(p3, p1), e3 = sub(p4, p1);
    // inverse by the adjugate: rows of adj are the cross products
    float det = dot(e1, cross(e2, e3));
    if (det != 0.0f) det = 1.0f / det;
    const V3 c1 = cross(e2, e3), c2 = cross(e3, e1), c3 = cross(e1, e2);
    // column-major 3x3: inv[r + 3 c]; adjugate column c holds (c1[c], c2[c], c3[c])
    const float adj[9] = {c1.x, c2.x, c3.x, c1.y, c2.y, c3.y, c1.z, c2.z, c3.z};
    for (int k = 0; k < 9; ++k) invE[k] = det * adj[k];
    // elasticity matrix (symmetric 6 x 6)
    const float lambda = (nu * E) / ((1 + nu) * (1 - 2 * nu));
    const float mu = E / (2 * (1 + nu));
    const float l2m = lambda + 2 * mu;
    float D[36];
    std::memset(D, 0, sizeof(D));
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) D[i + 6 * j] = i == j ? l2m : lambda;
    D[3 + 6 * 3] = mu;
    D[4 + 6 * 4] = mu;
    D[5 + 6 * 5] = mu;
    // strain-displacement matrix (b3ComputeB, softbody.cpp:76-155): its
    // coefficients are the entries of invE with the signs the reference's
    // cofactor expression gives, vertices 2..4 the negated rows of invE and
    // vertex 1 the sum of the rows, summed in the reference's order
    const float* m = invE;  // m[r + 3 c]
    const float g1[3] = {(m[0] + m[1]) + m[2], (m[3] + m[4]) + m[5], (m[6] + m[7]) + m[8]};
    const float g2[3] = {-m[0], -m[3], -m[6]}, g3[3] = {-m[1], -m[4], -m[7]}, g4[3] = {-m[2], -m[5], -m[8]};
    const float* g[4] = {g1, g2, g3, g4};
    std::memset(Bo, 0, 72 * sizeof(float));
    for (int v = 0; v < 4; ++v) {
        const float b = g[v][0], c = g[v][1], d = g[v][2];
        float* colx = Bo + 6 * (3 * v);      // strain rows: xx yy zz xy xz yz
        float* coly = Bo + 6 * (3 * v + 1);
        float* colz = Bo + 6 * (3 * v + 2);
        colx[0] = b, colx[3] = c, colx[4] = d;
        coly[1] = c, coly[3] = b, coly[5] = d;
        colz[2] = d, colz[4] = b, colz[5] = c;
    }
    float BT[72], BTD[72], BTDB[144];
    for (uint32_t i = 0; i < 6; ++i)
        for (uint32_t j = 0; j < 12; ++j) BT[j + 12 * i] = Bo[i + 6 * j];
    matmul(BTD, BT, 12, 6, D, 6, 6);
    matmul(BTDB, BTD, 12, 6, Bo, 6, 12);
    for (int k = 0; k < 144; ++k) BTDB[k] *= vol;
    // 16 blocks: upper and diagonal from the matrix, lower = upper^T
    for (uint32_t bi = 0; bi < 4; ++bi)
        for (uint32_t bj = bi; bj < 4; ++bj) {
            float* blk = Ke + 9 * (bi + 4 * bj);
            for (uint32_t c = 0; c < 3; ++c)
                for (uint32_t r = 0; r < 3; ++r) blk[r + 3 * c] = BTDB[3 * bi + r + 12 * (3 * bj + c)];
        }
    for (uint32_t bi = 1; bi < 4; ++bi)
        for (uint32_t bj = 0; bj < bi; ++bj) {
            const float* up = Ke + 9 * (bj + 4 * bi);
            float* lo = Ke + 9 * (bi + 4 * bj);
            for (uint32_t c = 0; c < 3; ++c)
                for (uint32_t r = 0; r < 3; ++r) lo[r + 3 * c] = up[c + 3 * r];
        }
    matmul(Po, BT, 12, 6, D, 6, 6);
    for (int k = 0; k < 72; ++k) Po[k] *= vol;
}

}  // namespace

int prepare_softbody(uint32_t n, const float* vertices, uint32_t t, const uint32_t* tets, float density, float E,
                     float nu, SoftBodyPrep* out)
{
    SoftBodyPrep& S = *out;
    S = SoftBodyPrep();
    S.n = n;
    S.t = t;
    auto vert = [&](uint32_t i) { return V3{vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]}; };
    for (uint64_t k = 0; k < 4ull * t; ++k)
        if (tets[k] >= n) return B3G_ERR_DEGENERATE_MESH;
    S.mass.assign(n, 0.0f);
    S.Ke.resize(144 * (size_t)t);
    S.invE.resize(9 * (size_t)t);
    S.B.resize(72 * (size_t)t);
    S.P.resize(72 * (size_t)t);
    const float inv4 = 1.0f / 4.0f;
    for (uint32_t e = 0; e < t; ++e) {
        const uint32_t* tv = tets + 4 * (size_t)e;
        if (tv[0] == tv[1] || tv[0] == tv[2] || tv[0] == tv[3] || tv[1] == tv[2] || tv[1] == tv[3] || tv[2] == tv[3])
            return B3G_ERR_DEGENERATE_MESH;
        const float vol = tet_volume(vert(tv[0]), vert(tv[1]), vert(tv[2]), vert(tv[3]));
        if (!(vol > 0.0f) || !std::isfinite(vol)) return B3G_ERR_DEGENERATE_MESH;
        const float mass = density * vol;
        for (int k = 0; k < 4; ++k) S.mass[tv[k]] += inv4 * mass;
        element_matrices(vert(tv[0]), vert(tv[1]), vert(tv[2]), vert(tv[3]), E, nu, &S.Ke[144 * (size_t)e],
                         &S.invE[9 * (size_t)e], &S.B[72 * (size_t)e], &S.P[72 * (size_t)e]);
    }
    for (uint32_t i = 0; i < n; ++i)
        if (!(S.mass[i] > 0.0f)) return B3G_ERR_DEGENERATE_MESH;  // a vertex no element uses
    // incidence in element order
    std::vector<uint32_t> cnt(n + 1, 0);
    for (uint64_t k = 0; k < 4ull * t; ++k) ++cnt[tets[k] + 1];
    S.inc_ptr.assign(n + 1, 0);
    for (uint32_t i = 0; i < n; ++i) S.inc_ptr[i + 1] = S.inc_ptr[i] + cnt[i + 1];
    S.inc_elem.resize(4 * (size_t)t);
    S.inc_meta.resize(4 * (size_t)t);
    std::vector<uint32_t> fill(S.inc_ptr.begin(), S.inc_ptr.end() - 1);
    for (uint32_t e = 0; e < t; ++e)
        for (uint32_t k = 0; k < 4; ++k) {
            const uint32_t i = tets[4 * (size_t)e + k];
            S.inc_elem[fill[i]] = e;
            S.inc_meta[fill[i]] = k;
            ++fill[i];
        }
    // block rows in first-touch order, and each incidence's slots
    S.rowptr.assign(n + 1, 0);
    S.diag.assign(n, 0);
    std::vector<uint32_t> row;
    for (uint32_t i = 0; i < n; ++i) {
        row.clear();
        for (uint32_t q = S.inc_ptr[i]; q < S.inc_ptr[i + 1]; ++q) {
            const uint32_t* tv = tets + 4 * (size_t)S.inc_elem[q];
            uint32_t meta = S.inc_meta[q];
            for (uint32_t j = 0; j < 4; ++j) {
                uint32_t slot = 0;
                while (slot < row.size() && row[slot] != tv[j]) ++slot;
                if (slot == row.size()) row.push_back(tv[j]);
                if (slot > 127) return B3G_ERR_UNSUPPORTED;
                meta |= slot << (4 + 7 * j);
            }
            S.inc_meta[q] = meta;
        }
        S.rowptr[i + 1] = S.rowptr[i] + (uint32_t)row.size();
        for (uint32_t k = 0; k < row.size(); ++k) {
            if (row[k] == i) S.diag[i] = S.rowptr[i] + k;
            S.cols.push_back(row[k]);
        }
        if (row.size() > S.max_deg) S.max_deg = (uint32_t)row.size();
    }
    return 0;
}

}  // namespace b3g
