// Static hull colliders: b3HullShape::TestSphere
// (src/bounce/dynamics/shapes/hull_shape.cpp:187-254) for one particle,
// with b3GJK (src/bounce/collision/gjk/gjk.cpp:579-740, no cache, no radius)
// between the hull (body at the origin, identity rotation) and the
// particle's point.  The simplex solvers follow gjk.cpp:32-577 operation for
// operation (-fmad=false), so the contact's normal and point are the
// reference's.
#pragma once

#include <cfloat>
#include <cstdint>

#include "vec.cuh"

namespace b3g {
namespace hull {
namespace {  // internal linkage: every file that includes this gets its own copy

struct Vtx {
    f3 p1, p2, p;
    float w;
    uint32_t i1;
};

// b3Mul / b3MulT with the static body's transform (identity rotation, origin)
__device__ __forceinline__ f3 xf_mul(f3 v)
{
    const f3 r = (v.x * mk(1.0f, 0.0f, 0.0f) + v.y * mk(0.0f, 1.0f, 0.0f)) + v.z * mk(0.0f, 0.0f, 1.0f);
    return r + zero3();
}
__device__ __forceinline__ f3 xf_mult(f3 v)
{
    const f3 d = v - zero3();
    return mk(dot(mk(1.0f, 0.0f, 0.0f), d), dot(mk(0.0f, 1.0f, 0.0f), d), dot(mk(0.0f, 0.0f, 1.0f), d));
}
__device__ __forceinline__ f3 neg(f3 v) { return mk(-v.x, -v.y, -v.z); }

__device__ __forceinline__ void bary2(float o[3], f3 A, f3 B, f3 Q)
{
    const f3 AB = B - A, QA = A - Q, QB = B - Q;
    o[0] = dot(QB, AB);
    o[1] = -dot(QA, AB);
    o[2] = o[0] + o[1];
}

__device__ __forceinline__ void bary3(float o[4], f3 A, f3 B, f3 C, f3 Q)
{
    const f3 AB = B - A, AC = C - A, QA = A - Q, QB = B - Q, QC = C - Q;
    const f3 a = cross(QB, QC), b = cross(QC, QA), c = cross(QA, QB), n = cross(AB, AC);
    o[0] = dot(a, n);
    o[1] = dot(b, n);
    o[2] = dot(c, n);
    o[3] = o[0] + o[1] + o[2];
}

__device__ __forceinline__ float det3(f3 a, f3 b, f3 c) { return dot(a, cross(b, c)); }
__device__ __forceinline__ float sgn(float x) { return (float)(0.0f < x) - (float)(x < 0.0f); }

__device__ __forceinline__ void bary4(float o[5], f3 A, f3 B, f3 C, f3 D, f3 Q)
{
    const f3 AB = B - A, AC = C - A, AD = D - A, QA = A - Q, QB = B - Q, QC = C - Q, QD = D - Q;
    const float divisor = det3(AB, AC, AD);
    const float s = sgn(divisor);
    o[0] = s * det3(QB, QC, QD);
    o[1] = s * det3(QA, QD, QC);
    o[2] = s * det3(QA, QB, QD);
    o[3] = s * det3(QA, QC, QB);
    o[4] = s * divisor;
}

struct Simplex {
    Vtx v[4];
    uint32_t n;
    __device__ void set1(const Vtx& a)
    {
        n = 1;
        v[0] = a;
        v[0].w = 1.0f;
    }
    __device__ void set2(const Vtx& a, float wa, const Vtx& b, float wb)
    {
        n = 2;
        v[0] = a;
        v[0].w = wa;
        v[1] = b;
        v[1].w = wb;
    }
    __device__ void set3(const Vtx& a, float wa, const Vtx& b, float wb, const Vtx& c, float wc)
    {
        n = 3;
        v[0] = a;
        v[0].w = wa;
        v[1] = b;
        v[1].w = wb;
        v[2] = c;
        v[2].w = wc;
    }
};

// b3Simplex::Solve2 / Solve3 / Solve4 with Q the origin
__device__ void solve2(Simplex& s, f3 Q)
{
    const Vtx A = s.v[0], B = s.v[1];
    float wAB[3];
    bary2(wAB, A.p, B.p, Q);
    if (wAB[1] <= 0.0f) { s.set1(A); return; }
    if (wAB[0] <= 0.0f) { s.set1(B); return; }
    const float sc = 1.0f / wAB[2];
    s.set2(A, sc * wAB[0], B, sc * wAB[1]);
}

__device__ void solve3(Simplex& s, f3 Q)
{
    const Vtx A = s.v[0], B = s.v[1], C = s.v[2];
    float wAB[3], wBC[3], wCA[3];
    bary2(wAB, A.p, B.p, Q);
    bary2(wBC, B.p, C.p, Q);
    bary2(wCA, C.p, A.p, Q);
    if (wAB[1] <= 0.0f && wCA[0] <= 0.0f) { s.set1(A); return; }
    if (wAB[0] <= 0.0f && wBC[1] <= 0.0f) { s.set1(B); return; }
    if (wBC[0] <= 0.0f && wCA[1] <= 0.0f) { s.set1(C); return; }
    float wABC[4];
    bary3(wABC, A.p, B.p, C.p, Q);
    const float area = wABC[3];
    if (wAB[0] > 0.0f && wAB[1] > 0.0f && area * wABC[2] <= 0.0f) {
        const float sc = 1.0f / wAB[2];
        s.set2(A, sc * wAB[0], B, sc * wAB[1]);
        return;
    }
    if (wBC[0] > 0.0f && wBC[1] > 0.0f && area * wABC[0] <= 0.0f) {
        const float sc = 1.0f / wBC[2];
        s.set2(B, sc * wBC[0], C, sc * wBC[1]);
        return;
    }
    if (wCA[0] > 0.0f && wCA[1] > 0.0f && area * wABC[1] <= 0.0f) {
        const float sc = 1.0f / wCA[2];
        s.set2(C, sc * wCA[0], A, sc * wCA[1]);
        return;
    }
    const float divisor = wABC[3];
    if (divisor <= 0.0f) return;  // give up: the simplex and its weights stay
    const float sc = 1.0f / divisor;
    s.set3(A, sc * wABC[0], B, sc * wABC[1], C, sc * wABC[2]);
}

__device__ void solve4(Simplex& s, f3 Q)
{
    const Vtx A = s.v[0], B = s.v[1], C = s.v[2], D = s.v[3];
    float wAB[3], wAC[3], wAD[3], wBC[3], wCD[3], wDB[3];
    bary2(wAB, A.p, B.p, Q);
    bary2(wBC, B.p, C.p, Q);
    bary2(wAC, A.p, C.p, Q);
    bary2(wAD, A.p, D.p, Q);
    bary2(wCD, C.p, D.p, Q);
    bary2(wDB, D.p, B.p, Q);
    if (wAB[1] <= 0.0f && wAC[1] <= 0.0f && wAD[1] <= 0.0f) { s.set1(A); return; }
    if (wAB[0] <= 0.0f && wDB[0] <= 0.0f && wBC[1] <= 0.0f) { s.set1(B); return; }
    if (wAC[0] <= 0.0f && wBC[0] <= 0.0f && wCD[1] <= 0.0f) { s.set1(C); return; }
    if (wAD[0] <= 0.0f && wCD[0] <= 0.0f && wDB[1] <= 0.0f) { s.set1(D); return; }
    float wACB[4], wABD[4], wADC[4], wBCD[4];
    bary3(wACB, A.p, C.p, B.p, Q);
    bary3(wABD, A.p, B.p, D.p, Q);
    bary3(wADC, A.p, D.p, C.p, Q);
    bary3(wBCD, B.p, C.p, D.p, Q);
    if (wABD[2] <= 0.0f && wACB[1] <= 0.0f && wAB[0] > 0.0f && wAB[1] > 0.0f) {
        const float sc = 1.0f / wAB[2];
        s.set2(A, sc * wAB[0], B, sc * wAB[1]);
        return;
    }
    if (wACB[2] <= 0.0f && wADC[1] <= 0.0f && wAC[0] > 0.0f && wAC[1] > 0.0f) {
        const float sc = 1.0f / wAC[2];
        s.set2(A, sc * wAC[0], C, sc * wAC[1]);
        return;
    }
    if (wADC[2] <= 0.0f && wABD[1] <= 0.0f && wAD[0] > 0.0f && wAD[1] > 0.0f) {
        const float sc = 1.0f / wAD[2];
        s.set2(A, sc * wAD[0], D, sc * wAD[1]);
        return;
    }
    if (wACB[0] <= 0.0f && wBCD[2] <= 0.0f && wBC[0] > 0.0f && wBC[1] > 0.0f) {
        const float sc = 1.0f / wBC[2];
        s.set2(B, sc * wBC[0], C, sc * wBC[1]);
        return;
    }
    if (wADC[0] <= 0.0f && wBCD[0] <= 0.0f && wCD[0] > 0.0f && wCD[1] > 0.0f) {
        const float sc = 1.0f / wCD[2];
        s.set2(C, sc * wCD[0], D, sc * wCD[1]);
        return;
    }
    if (wABD[0] <= 0.0f && wBCD[1] <= 0.0f && wDB[0] > 0.0f && wDB[1] > 0.0f) {
        const float sc = 1.0f / wDB[2];
        s.set2(D, sc * wDB[0], B, sc * wDB[1]);
        return;
    }
    float wABCD[5];
    bary4(wABCD, A.p, B.p, C.p, D.p, Q);
    if (wABCD[3] <= 0.0f && wACB[0] > 0.0f && wACB[1] > 0.0f && wACB[2] > 0.0f) {
        const float sc = 1.0f / (wACB[0] + wACB[1] + wACB[2]);
        s.set3(A, sc * wACB[0], C, sc * wACB[1], B, sc * wACB[2]);
        return;
    }
    if (wABCD[2] <= 0.0f && wABD[0] > 0.0f && wABD[1] > 0.0f && wABD[2] > 0.0f) {
        const float sc = 1.0f / (wABD[0] + wABD[1] + wABD[2]);
        s.set3(A, sc * wABD[0], B, sc * wABD[1], D, sc * wABD[2]);
        return;
    }
    if (wABCD[1] <= 0.0f && wADC[0] > 0.0f && wADC[1] > 0.0f && wADC[2] > 0.0f) {
        const float sc = 1.0f / (wADC[0] + wADC[1] + wADC[2]);
        s.set3(A, sc * wADC[0], D, sc * wADC[1], C, sc * wADC[2]);
        return;
    }
    if (wABCD[0] <= 0.0f && wBCD[0] > 0.0f && wBCD[1] > 0.0f && wBCD[2] > 0.0f) {
        const float sc = 1.0f / (wBCD[0] + wBCD[1] + wBCD[2]);
        s.set3(B, sc * wBCD[0], C, sc * wBCD[1], D, sc * wBCD[2]);
        return;
    }
    const float divisor = wABCD[0] + wABCD[1] + wABCD[2] + wABCD[3];
    if (divisor <= 0.0f) return;
    const float sc = 1.0f / divisor;
    s.n = 4;
    s.v[0].w = sc * wABCD[0];
    s.v[1].w = sc * wABCD[1];
    s.v[2].w = sc * wABCD[2];
    s.v[3].w = sc * wABCD[3];
}

// b3Simplex::GetSearchDirection toward the origin
__device__ __forceinline__ f3 search(const Simplex& s)
{
    const f3 Q = zero3();
    if (s.n == 1) return Q - s.v[0].p;
    if (s.n == 2) {
        const f3 AB = s.v[1].p - s.v[0].p, AQ = Q - s.v[0].p;
        return cross(cross(AB, AQ), AB);
    }
    const f3 AB = s.v[1].p - s.v[0].p, AC = s.v[2].p - s.v[0].p, AQ = Q - s.v[0].p;
    const f3 n = cross(AB, AC);
    return dot(n, AQ) > 0.0f ? n : neg(n);
}

// b3Simplex::GetClosestPoints
__device__ __forceinline__ void witness(const Simplex& s, f3& p1, f3& p2)
{
    const Vtx* v = s.v;
    if (s.n == 1) {
        p1 = v[0].p1;
        p2 = v[0].p2;
    } else if (s.n == 2) {
        p1 = v[0].w * v[0].p1 + v[1].w * v[1].p1;
        p2 = v[0].w * v[0].p2 + v[1].w * v[1].p2;
    } else if (s.n == 3) {
        p1 = (v[0].w * v[0].p1 + v[1].w * v[1].p1) + v[2].w * v[2].p1;
        p2 = (v[0].w * v[0].p2 + v[1].w * v[1].p2) + v[2].w * v[2].p2;
    } else {
        p1 = ((v[0].w * v[0].p1 + v[1].w * v[1].p1) + v[2].w * v[2].p1) + v[3].w * v[3].p1;
        p2 = p1;
    }
}

// b3Mul(xf, v) and b3MulT(xf.rotation, v) for the hull's body transform
// (rotation R, column-major, position p); with the identity and the origin
// they are the static forms above, bit for bit.
__device__ __forceinline__ f3 xr_mul(const m3& R, f3 p, f3 v) { return ((v.x * R.x + v.y * R.y) + v.z * R.z) + p; }
__device__ __forceinline__ f3 r_mult(const m3& R, f3 v) { return mk(dot(R.x, v), dot(R.y, v), dot(R.z, v)); }

// b3GJK between the hull (vertices hv[0, nv), in its body's frame R, p) and
// the point Q; returns the distance and the witness points (p1 on the hull).
__device__ __noinline__ float gjk(const float* hv, uint32_t nv, const m3 R, const f3 P, f3 Q, f3& p1, f3& p2)
{
    Simplex s;
    s.v[0].p1 = xr_mul(R, P, mk(hv[0], hv[1], hv[2]));
    s.v[0].p2 = xf_mul(Q);
    s.v[0].p = s.v[0].p2 - s.v[0].p1;
    s.v[0].w = 1.0f;
    s.v[0].i1 = 0;
    for (int k = 1; k < 4; ++k) {
        s.v[k].p1 = s.v[k].p2 = s.v[k].p = zero3();
        s.v[k].w = 0.0f;
        s.v[k].i1 = 0;
    }
    s.n = 1;
    const f3 O = zero3();
    uint32_t save[4];
    for (uint32_t iter = 0; iter < 20;) {
        const uint32_t saved = s.n;
        for (uint32_t i = 0; i < saved; ++i) save[i] = s.v[i].i1;
        if (s.n == 2) solve2(s, O);
        else if (s.n == 3) solve3(s, O);
        else if (s.n == 4) solve4(s, O);
        if (s.n == 4) break;
        const f3 d = search(s);
        if (dot(d, d) < FLT_EPSILON * FLT_EPSILON) break;
        // the hull's support vertex in -d (b3GJKProxy::GetSupportIndex)
        const f3 dl = r_mult(R, neg(d));
        uint32_t best = 0;
        float bestp = dot(dl, mk(hv[0], hv[1], hv[2]));
        for (uint32_t i = 1; i < nv; ++i) {
            const float pr = dot(dl, mk(hv[3 * i], hv[3 * i + 1], hv[3 * i + 2]));
            if (pr > bestp) {
                best = i;
                bestp = pr;
            }
        }
        Vtx& x = s.v[s.n];
        x.i1 = best;
        x.p1 = xr_mul(R, P, mk(hv[3 * best], hv[3 * best + 1], hv[3 * best + 2]));
        x.p2 = xf_mul(Q);
        x.p = x.p2 - x.p1;
        ++iter;
        bool duplicate = false;  // the point proxy's index is always 0
        for (uint32_t i = 0; i < saved; ++i)
            if (best == save[i]) {
                duplicate = true;
                break;
            }
        if (duplicate) break;
        ++s.n;
    }
    witness(s, p1, p2);
    const f3 d = p1 - p2;
    return sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
}

// b3HullShape::TestSphere for a particle at Q of radius r against the hull
// (vertices, then planes as normal xyz + offset, in its body's frame R, P).
// false: no contact.
__device__ __forceinline__ bool test_sphere(const float* hv, uint32_t nv, const float* hp, uint32_t nf, float radius,
                                            const m3& R, f3 P, f3 Q, f3& normal, f3& point)
{
    f3 c1, c2;
    const float distance = gjk(hv, nv, R, P, Q, c1, c2);
    if (distance > radius) return false;
    if (distance > 0.0f) {
        normal = (c2 - c1) / distance;
        point = c1;
        return true;
    }
    const f3 support = r_mult(R, Q - P);
    uint32_t best = 0;
    float best_sep = -FLT_MAX;
    for (uint32_t f = 0; f < nf; ++f) {
        const float sep = dot(mk(hp[4 * f], hp[4 * f + 1], hp[4 * f + 2]), support) - hp[4 * f + 3];
        if (sep > radius) return false;
        if (sep > best_sep) {
            best = f;
            best_sep = sep;
        }
    }
    // b3Mul(xf, plane) and b3ClosestPointOnPlane (geometry.h:77-100)
    const f3 n0 = mk(hp[4 * best], hp[4 * best + 1], hp[4 * best + 2]);
    const f3 n = (n0.x * R.x + n0.y * R.y) + n0.z * R.z;
    const float off = hp[4 * best + 3] + dot(n, P);
    const float fraction = dot(n, Q) - off;
    point = Q - fraction * n;
    normal = n;
    return true;
}

}  // namespace
}  // namespace hull
}  // namespace b3g
