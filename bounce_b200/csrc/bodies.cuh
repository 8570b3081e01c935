// Colliders on rigid bodies: the body's transform, quaternion arithmetic and
// the shape tests with a body transform, on the device.
//
// Every expression follows the reference's float order (b3Mul / b3MulT,
// include/bounce/common/math/transform.h:74-110, mat33.h:129-160; b3Quat,
// quat.h:88-100, 172-180, 225-232, 306-318; b3Derivative,
// include/bounce/dynamics/time_step.h:105-109), so that with -fmad=false the
// results are the reference's bit for bit.
#pragma once

#include <cfloat>
#include <cstdint>

#include "../../include/b3g.h"
#include "cloth_dev.cuh"
#include "hull_gjk.cuh"
#include "vec.cuh"

namespace b3g {
namespace body {

struct Q4 {
    float x, y, z, w;
};

__device__ __forceinline__ f3 ld3a(const float* a) { return f3{a[0], a[1], a[2]}; }
__device__ __forceinline__ void st3a(float* a, f3 v) { a[0] = v.x, a[1] = v.y, a[2] = v.z; }
__device__ __forceinline__ m3 ld9(const float* a) { return m3{ld3a(a), ld3a(a + 3), ld3a(a + 6)}; }
__device__ __forceinline__ void st9(float* a, const m3& m) { st3a(a, m.x), st3a(a + 3, m.y), st3a(a + 6, m.z); }
__device__ __forceinline__ Q4 ldq(const float* a) { return Q4{a[0], a[1], a[2], a[3]}; }
__device__ __forceinline__ void stq(float* a, Q4 q) { a[0] = q.x, a[1] = q.y, a[2] = q.z, a[3] = q.w; }

// b3Mul(xf, v), b3MulT(xf, v), b3MulT(A, v)
__device__ __forceinline__ f3 xmul(const m3& R, f3 p, f3 v) { return R * v + p; }
__device__ __forceinline__ f3 mult(const m3& R, f3 v) { return mk(dot(R.x, v), dot(R.y, v), dot(R.z, v)); }
__device__ __forceinline__ f3 xmult(const m3& R, f3 p, f3 v) { return mult(R, v - p); }
// b3Mat33 * b3Mat33 (columns A * B.x ...) and b3Transpose
__device__ __forceinline__ m3 mmul(const m3& A, const m3& B) { return m3{A * B.x, A * B.y, A * B.z}; }
__device__ __forceinline__ m3 transpose(const m3& A)
{
    return m3{mk(A.x.x, A.y.x, A.z.x), mk(A.x.y, A.y.y, A.z.y), mk(A.x.z, A.y.z, A.z.z)};
}

__device__ __forceinline__ Q4 qmul(Q4 a, Q4 b)
{
    return Q4{a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z,
              a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
__device__ __forceinline__ void qnormalize(Q4& q)
{
    const float length = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    if (length > FLT_EPSILON) {
        const float s = 1.0f / length;
        q.x *= s, q.y *= s, q.z *= s, q.w *= s;
    }
}
__device__ __forceinline__ m3 qmat(Q4 q)
{
    const float x = q.x, y = q.y, z = q.z, w = q.w;
    const float x2 = x + x, y2 = y + y, z2 = z + z;
    const float xx = x * x2, xy = x * y2, xz = x * z2;
    const float yy = y * y2, yz = y * z2, zz = z * z2;
    const float wx = w * x2, wy = w * y2, wz = w * z2;
    return m3{mk(1.0f - (yy + zz), xy + wz, xz - wy), mk(xy - wz, 1.0f - (xx + zz), yz + wx),
              mk(xz + wy, yz - wx, 1.0f - (xx + yy))};
}
__device__ __forceinline__ f3 qrot(Q4 q, f3 v)
{
    const f3 qv = mk(q.x, q.y, q.z);
    const f3 t = 2.0f * cross(qv, v);
    return (v + q.w * t) + cross(qv, t);
}
__device__ __forceinline__ Q4 qderiv(Q4 q, f3 w) { return qmul(Q4{0.5f * w.x, 0.5f * w.y, 0.5f * w.z, 0.0f}, q); }

// b3Sweep::GetTransform (transform.h:224-234)
__device__ __forceinline__ void sweep_xf(const b3g_body_state& b, float t, m3& R, f3& p)
{
    const f3 cc = (1.0f - t) * ld3a(b.world_center0) + t * ld3a(b.world_center);
    const Q4 q0 = ldq(b.orientation0), q1 = ldq(b.orientation);
    Q4 q{(1.0f - t) * q0.x + t * q1.x, (1.0f - t) * q0.y + t * q1.y, (1.0f - t) * q0.z + t * q1.z,
         (1.0f - t) * q0.w + t * q1.w};
    qnormalize(q);
    R = qmat(q);
    p = cc - qrot(q, ld3a(b.local_center));
}

// b3Shape::ComputeAABB with a transform (sphere_shape.cpp:53-59,
// capsule_shape.cpp:130-137, hull_shape.cpp:162-166)
__device__ __forceinline__ void shape_aabb(const SphereDev& sp, const m3& R, f3 p, f3& lo, f3& hi)
{
    const f3 r = mk(sp.radius, sp.radius, sp.radius);
    if (sp.kind == 0) {
        const f3 ctr = xmul(R, p, mk(sp.cx, sp.cy, sp.cz));
        lo = ctr - r;
        hi = ctr + r;
    } else if (sp.kind == 1) {
        const f3 c1 = xmul(R, p, mk(sp.ax, sp.ay, sp.az)), c2 = xmul(R, p, mk(sp.bx, sp.by, sp.bz));
        lo = mk(c1.x < c2.x ? c1.x : c2.x, c1.y < c2.y ? c1.y : c2.y, c1.z < c2.z ? c1.z : c2.z) - r;
        hi = mk(c1.x > c2.x ? c1.x : c2.x, c1.y > c2.y ? c1.y : c2.y, c1.z > c2.z ? c1.z : c2.z) + r;
    } else {
        f3 l = xmul(R, p, mk(sp.hull[0], sp.hull[1], sp.hull[2])), h = l;
        for (uint32_t i = 1; i < sp.nhv; ++i) {
            const f3 w = xmul(R, p, mk(sp.hull[3 * i], sp.hull[3 * i + 1], sp.hull[3 * i + 2]));
            l = mk(l.x < w.x ? l.x : w.x, l.y < w.y ? l.y : w.y, l.z < w.z ? l.z : w.z);
            h = mk(h.x > w.x ? h.x : w.x, h.y > w.y ? h.y : w.y, h.z > w.z ? h.z : w.z);
        }
        lo = l - r;
        hi = h + r;
    }
}

// TestSphere of a shape on a body (transform R, p) against the particle at
// Q with the summed radius: the normal (shape to particle) and the world
// point on the shape (sphere_shape.cpp:71-95, capsule_shape.cpp:186-284,
// hull_shape.cpp:187-254).
__device__ __forceinline__ bool test_sphere(const SphereDev& sp, const m3& R, f3 p, f3 Q, float radius, f3& normal,
                                            f3& point)
{
    if (sp.kind == 2)
        return hull::test_sphere(sp.hull, sp.nhv, sp.hull + 3 * sp.nhv, sp.nhf, radius, R, p, Q, normal, point);
    if (sp.kind == 0) {
        const f3 center = xmul(R, p, mk(sp.cx, sp.cy, sp.cz));
        const float rr = radius * radius;
        const f3 d = Q - center;
        const float dd = dot(d, d);
        if (!(dd <= rr)) return false;
        const float d_len = sqrtf(dd);
        normal = mk(0.0f, 1.0f, 0.0f);
        if (d_len > FLT_EPSILON) normal = d / d_len;
        point = center;
        return true;
    }
    const f3 A = xmul(R, p, mk(sp.ax, sp.ay, sp.az)), B = xmul(R, p, mk(sp.bx, sp.by, sp.bz));
    const f3 AB = B - A;
    const float u = dot(B - Q, AB);
    const float v = dot(Q - A, AB);
    if (v <= 0.0f || u <= 0.0f) {
        const f3 P = v <= 0.0f ? A : B;
        const f3 d = Q - P;
        const float dd = dot(d, d);
        if (dd > radius * radius) return false;
        normal = mk(0.0f, 1.0f, 0.0f);
        const float len = sqrtf(dd);
        if (len > FLT_EPSILON) normal = d / len;
        point = P;
        return true;
    }
    const float ss = dot(AB, AB);
    const f3 P = ss < 0.005f * 0.005f ? A : (u * A + v * B) / ss;
    const f3 d = Q - P;
    const float dd = dot(d, d);
    if (dd > radius * radius) return false;
    const f3 QA = A - Q;
    const f3 e = cross(AB, QA);
    f3 nn3 = cross(AB, e);
    if (dot(nn3, QA) < 0.0f) nn3 = mk(-nn3.x, -nn3.y, -nn3.z);
    const float len = sqrtf(nn3.x * nn3.x + nn3.y * nn3.y + nn3.z * nn3.z);
    if (len > FLT_EPSILON) {
        const float s1 = 1.0f / len;
        nn3 = mk(nn3.x * s1, nn3.y * s1, nn3.z * s1);
    }
    normal = mk(-nn3.x, -nn3.y, -nn3.z);
    point = P;
    return true;
}

// The transform m_xf of a body state
__device__ __forceinline__ void body_xf(const b3g_body_state& b, m3& R, f3& p)
{
    R = ld9(b.rotation);
    p = ld3a(b.position);
}

}  // namespace body
}  // namespace b3g
