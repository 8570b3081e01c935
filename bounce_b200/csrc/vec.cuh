// Small 3-vector / 3x3-matrix helpers for the cloth kernels.
//
// They evaluate in the same order as Bounce's inline operators
// (include/bounce/common/math/vec3.h, mat33.h): with -fmad=false (set for
// every kernel of this library) the element force and Jacobian arithmetic is
// the reference's, operation for operation, so the assembled system matches
// the CPU reference bit for bit.
#pragma once

#include <cuda_runtime.h>

namespace b3g {

struct f3 {
    float x, y, z;
};

struct m3 {  // column-major, like b3Mat33
    f3 x, y, z;
};

__host__ __device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__host__ __device__ __forceinline__ f3 zero3() { return f3{0.0f, 0.0f, 0.0f}; }
__host__ __device__ __forceinline__ f3 operator+(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ f3 operator-(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ f3 operator*(float s, f3 v) { return f3{s * v.x, s * v.y, s * v.z}; }
__host__ __device__ __forceinline__ f3 operator/(f3 v, float s) { return f3{v.x / s, v.y / s, v.z / s}; }
__host__ __device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ f3 cross(f3 a, f3 b)
{
    return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float length(f3 v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }

__host__ __device__ __forceinline__ m3 mzero() { return m3{zero3(), zero3(), zero3()}; }
__host__ __device__ __forceinline__ m3 mident()
{
    return m3{f3{1.0f, 0.0f, 0.0f}, f3{0.0f, 1.0f, 0.0f}, f3{0.0f, 0.0f, 1.0f}};
}
__host__ __device__ __forceinline__ m3 operator+(const m3& a, const m3& b) { return m3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ m3 operator-(const m3& a, const m3& b) { return m3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ m3 operator*(float s, const m3& a) { return m3{s * a.x, s * a.y, s * a.z}; }
// b3Outer(a, b) = a b^T, columns b.x a, b.y a, b.z a (mat33.h:229-232)
__host__ __device__ __forceinline__ m3 outer(f3 a, f3 b) { return m3{b.x * a, b.y * a, b.z * a}; }
// A v = v.x A.x + v.y A.y + v.z A.z (mat33.h:129-132)
__host__ __device__ __forceinline__ f3 operator*(const m3& a, f3 v) { return (v.x * a.x + v.y * a.y) + v.z * a.z; }

// b3Perp (vec3.h:255-266): an unnormalised perpendicular.
__device__ __forceinline__ f3 perp(f3 v)
{
    if (fabsf(v.x) >= 0.57735027f) return f3{v.y, -v.x, 0.0f};
    return f3{0.0f, v.z, -v.y};
}

__device__ __forceinline__ f3 ld3(const float* p, uint32_t n, uint32_t i)
{
    return f3{p[i], p[n + i], p[2 * n + i]};
}
__device__ __forceinline__ void st3(float* p, uint32_t n, uint32_t i, f3 v)
{
    p[i] = v.x;
    p[n + i] = v.y;
    p[2 * n + i] = v.z;
}

}  // namespace b3g
