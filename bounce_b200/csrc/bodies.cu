// Colliders on rigid bodies of any type: the body-contact solve of a cloth
// in a world whose bodies move, and the C ABI that exchanges the bodies'
// state with the caller's world.
//
// With a dynamic body every contact on it reads and writes the body's
// velocity (and, in the position solve, its sweep), so the contacts form one
// chain in the contact list's order.  The reference solves that list one
// contact after another (cloth_contact_solver.cpp:54-177, 264-307, 388-472,
// 598-718, in b3ClothSolver::Solve, cloth_solver.cpp:103-182); here one
// thread does the same, in the same order, after a radix sort has put the
// active contacts into list order: newest first (the creation step), then by
// particle (a step's new contacts are pushed particle by particle in the
// particle list's order, cloth_contact_manager.cpp:64-123), then by the
// world query's report order, last reported first.  The particle
// integration between the velocity and the position solve runs on the
// whole block.
#include <cub/device/device_radix_sort.cuh>

#include <cstring>
#include <vector>

#include "../../include/b3g.h"
#include "bodies.cuh"
#include "cloth_dev.cuh"
#include "cloth_internal.h"
#include "vec.cuh"

namespace b3g {

namespace {

constexpr int kSolveThreads = 256;
constexpr float kSlop = 0.005f;       // B3_LINEAR_SLOP (include/bounce/common/settings.h:63)
constexpr float kMaxCorr = 0.2f;      // B3_MAX_LINEAR_CORRECTION (:95)
constexpr float kBaum = 0.1f;         // B3_BAUMGARTE (:101)
constexpr float kAabbExt = 0.2f;      // B3_AABB_EXTENSION (:54)
constexpr float kAabbMul = 2.0f;      // B3_AABB_MULTIPLIER (:59)

// One active body contact's constraint (the velocity and the position
// constraint of cloth_contact_solver.h in one record).
struct BodyCon {
    uint32_t slot, body1;
    float mA, mB, friction, normal_mass;
    float tm_xx, tm_xy, tm_yx, tm_yy;
    f3 normal, t1, t2, point, rA, rB;
    float ni, tix, tiy;
    m3 iB;
    float radius_a, radius_b;
    f3 lcB, lpB;
};

// The sort key of a contact slot: list order ascending, inactive slots last.
__global__ void k_body_keys(const __grid_constant__ ClothDev c, unsigned long long* keys, uint32_t* idx)
{
    const uint32_t m = c.nsph * c.n;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        idx[q] = q;
        if (!c.c_exists[q] || !c.c_active[q]) {
            keys[q] = ~0ull;
            continue;
        }
        const uint32_t i = q % c.n;
        const uint32_t step = c.c_key[q] / (uint32_t)kMaxSpheres, rank = c.c_key[q] % (uint32_t)kMaxSpheres;
        keys[q] = ((unsigned long long)(0xffffffffu - step) << 32) | ((unsigned long long)i << 2) |
                  (unsigned long long)(3u - rank);
    }
}

// The force solver's state update before the contact solve
// (cloth_force_solver.cpp:211-222): v += dv, x += y, m_x = dv.
__global__ void k_body_prepare(const __grid_constant__ ClothDev c)
{
    const uint32_t n = c.n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const f3 dv = ld3(c.dv, n, i);
        st3(c.v, n, i, ld3(c.v, n, i) + dv);
        st3(c.x, n, i, ld3(c.x, n, i) + ld3(c.y, n, i));
        st3(c.mx, n, i, dv);
    }
}

// b3BroadPhase::MoveProxy (broad_phase.cpp:99-149) of a shape's proxy.
__device__ void move_shape_proxy(float* fat, f3 lo, f3 hi, f3 disp)
{
    const bool contains = fat[0] <= lo.x && lo.x <= fat[3] && fat[1] <= lo.y && lo.y <= fat[4] && fat[2] <= lo.z &&
                          lo.z <= fat[5] && fat[0] <= hi.x && hi.x <= fat[3] && fat[1] <= hi.y && hi.y <= fat[4] &&
                          fat[2] <= hi.z && hi.z <= fat[5];
    if (contains) return;
    float l[3] = {lo.x - kAabbExt, lo.y - kAabbExt, lo.z - kAabbExt};
    float h[3] = {hi.x + kAabbExt, hi.y + kAabbExt, hi.z + kAabbExt};
    const float d[3] = {kAabbMul * disp.x, kAabbMul * disp.y, kAabbMul * disp.z};
    for (int k = 0; k < 3; ++k) {
        if (d[k] < 0.0f) l[k] += d[k];
        else h[k] += d[k];
        fat[k] = l[k];
        fat[3 + k] = h[k];
    }
}

// After the position solve: SynchronizeTransform, the world inverse inertia
// and SynchronizeShapes of a non-static body (body.cpp:176-202,
// time_step.h:86-89).
__device__ void sync_body(const ClothDev& c, b3g_body_state& b, uint32_t body)
{
    if (b.type == 0) return;
    m3 R;
    f3 p;
    body::sweep_xf(b, 1.0f, R, p);
    body::st9(b.rotation, R);
    body::st3a(b.position, p);
    body::st9(b.world_inv_inertia, body::mmul(body::mmul(R, body::ld9(b.inv_inertia)), body::transpose(R)));
    m3 R1;
    f3 p1;
    body::sweep_xf(b, 0.0f, R1, p1);
    const f3 disp = p - p1;
    for (uint32_t s = 0; s < c.nsph; ++s) {
        const SphereDev& sp = c.sph[s];
        if (sp.body1 != body + 1) continue;
        f3 lo1, hi1, lo2, hi2;
        body::shape_aabb(sp, R1, p1, lo1, hi1);
        body::shape_aabb(sp, R, p, lo2, hi2);
        const f3 lo = mk(lo1.x < lo2.x ? lo1.x : lo2.x, lo1.y < lo2.y ? lo1.y : lo2.y, lo1.z < lo2.z ? lo1.z : lo2.z);
        const f3 hi = mk(hi1.x > hi2.x ? hi1.x : hi2.x, hi1.y > hi2.y ? hi1.y : hi2.y, hi1.z > hi2.z ? hi1.z : hi2.z);
        move_shape_proxy(c.shape_fat + 6 * s, lo, hi, disp);
    }
}

// The body of collider s; a static world-frame collider's implicit body (at
// the sphere's centre, or the origin, identity orientation, at rest).
__device__ b3g_body_state implicit_body(const SphereDev& sp)
{
    b3g_body_state b;
    memset(&b, 0, sizeof(b));
    b.rotation[0] = b.rotation[4] = b.rotation[8] = 1.0f;
    const f3 p = sp.kind == 0 ? mk(sp.cx, sp.cy, sp.cz) : zero3();
    body::st3a(b.position, p);
    body::st3a(b.world_center0, p);
    body::st3a(b.world_center, p);
    b.orientation0[3] = b.orientation[3] = 1.0f;
    return b;
}

__device__ __forceinline__ void set_velocity(b3g_body_state* b, f3 v, f3 w)
{
    if (b->type == 0) return;  // b3Body::SetLinearVelocity / SetAngularVelocity skip static bodies
    body::st3a(b->linear_velocity, v);
    body::st3a(b->angular_velocity, w);
}

// The body contact solve of one cloth, in list order, on one block.  Thread 0
// walks the list; the bodies live in shared memory meanwhile (the cloth's
// bodies at [0, nbody), the implicit static body of each world-frame
// collider at kMaxSpheres + s), so that the chain of dependent body updates
// waits on shared memory rather than on L2.
__global__ void __launch_bounds__(kSolveThreads) k_body_solve(const __grid_constant__ ClothDev c,
                                                              const unsigned long long* keys, const uint32_t* idx,
                                                              BodyCon* con)
{
    __shared__ uint32_t s_na;
    __shared__ b3g_body_state sb[2 * kMaxSpheres];
    StepScalars* sc = c.sc;
    const uint32_t n = c.n, nn = c.nsph * n;
    const float h = sc->dt;
    auto body_of = [&](uint32_t body1, uint32_t s) -> b3g_body_state* {
        return body1 ? sb + (body1 - 1) : sb + kMaxSpheres + s;
    };
    if (threadIdx.x == 0) {
        // the active contacts are the sorted keys' prefix below ~0
        uint32_t lo = 0, hi = nn;
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2;
            if (keys[mid] == ~0ull) hi = mid;
            else lo = mid + 1;
        }
        const uint32_t na = lo;
        s_na = na;
        sc->active_contacts = na;
        for (uint32_t b = 0; b < c.nbody; ++b) sb[b] = c.bodies[b];
        for (uint32_t s = 0; s < c.nsph; ++s) sb[kMaxSpheres + s] = implicit_body(c.sph[s]);
        // InitializeBodyContactConstraints (cloth_contact_solver.cpp:54-177)
        for (uint32_t k = 0; k < na; ++k) {
            BodyCon& x = con[k];
            const uint32_t q = idx[k], s = q / n, i = q % n;
            const SphereDev& sp = c.sph[s];
            const b3g_body_state& b = *body_of(sp.body1, s);
            x.slot = q;
            x.body1 = sp.body1;
            x.mA = c.type[i] == 0 ? 0.0f : 1.0f / c.mass[i];
            x.mB = b.inv_mass;
            x.iB = body::ld9(b.world_inv_inertia);
            x.friction = sqrtf(c.p_friction[i] * sp.friction);
            x.radius_a = c.p_radius[i];
            x.radius_b = sp.radius;
            x.lcB = body::ld3a(b.local_center);
            // the contact's point in the body's frame: body shapes, capsules
            // and hulls keep it in c_point; a world sphere's body sits at its centre
            x.lpB = sp.body1 || sp.kind != 0 ? ld3(c.c_point, nn, q) : zero3();
            const f3 xA = ld3(c.x, n, i), xB = body::ld3a(b.world_center);
            const m3 RA = body::qmat(body::Q4{0.0f, 0.0f, 0.0f, 1.0f});
            const f3 pA = xA - RA * zero3();
            const m3 RB = body::qmat(body::ldq(b.orientation));
            const f3 pB = xB - RB * x.lcB;
            // b3ParticleBodyContactWorldPoint::Initialize (cloth_particle_body_contact.cpp:49-62)
            const f3 nA = ld3(c.c_normal, nn, q);
            const f3 cA = body::xmul(RA, pA, zero3());
            const f3 cB = body::xmul(RB, pB, x.lpB);
            const f3 wA = cA + x.radius_a * nA, wB = cB - x.radius_b * nA;
            x.point = 0.5f * (wA + wB);
            x.normal = nA;
            x.t1 = ld3(c.c_t1, nn, q);
            x.t2 = ld3(c.c_t2, nn, q);
            x.rA = x.point - xA;
            x.rB = x.point - xB;
            x.ni = c.c_imp[q];
            x.tix = c.c_imp[nn + q];
            x.tiy = c.c_imp[2 * nn + q];
            const float mA = x.mA, mB = x.mB;
            const m3 iA = mzero(), iB = x.iB;
            {
                const f3 rnA = cross(x.rA, x.normal), rnB = cross(x.rB, x.normal);
                const float K = mA + mB + dot(iA * rnA, rnA) + dot(iB * rnB, rnB);
                x.normal_mass = K > 0.0f ? 1.0f / K : 0.0f;
            }
            {
                // b3Inverse of the 2x2 tangent mass (math.cpp:77-93)
                const f3 rn1A = cross(x.rA, x.t1), rn1B = cross(x.rB, x.t1);
                const f3 rn2A = cross(x.rA, x.t2), rn2B = cross(x.rB, x.t2);
                const float k11 = mA + mB + dot(iA * rn1A, rn1A) + dot(iB * rn1B, rn1B);
                const float k12 = dot(iA * rn1A, rn2A) + dot(iB * rn1B, rn2B);
                const float k22 = mA + mB + dot(iA * rn2A, rn2A) + dot(iB * rn2B, rn2B);
                float det = k11 * k22 - k12 * k12;
                if (det != 0.0f) det = 1.0f / det;
                x.tm_xx = det * k22;
                x.tm_yx = -det * k12;
                x.tm_xy = -det * k12;
                x.tm_yy = det * k11;
            }
        }
        // WarmStartBodyContactConstraints (:264-307)
        for (uint32_t k = 0; k < na; ++k) {
            const BodyCon& x = con[k];
            const uint32_t i = x.slot % n;
            b3g_body_state* b = body_of(x.body1, x.slot / n);
            f3 vA = ld3(c.v, n, i), vB = body::ld3a(b->linear_velocity), wB = body::ld3a(b->angular_velocity);
            const f3 P = x.ni * x.normal;
            vA = vA - x.mA * P;
            vB = vB + x.mB * P;
            wB = wB + x.iB * cross(x.rB, P);
            const f3 P1 = x.tix * x.t1, P2 = x.tiy * x.t2;
            vA = vA - x.mA * (P1 + P2);
            vB = vB + x.mB * (P1 + P2);
            wB = wB + x.iB * cross(x.rB, P1 + P2);
            st3(c.v, n, i, vA);
            set_velocity(b, vB, wB);
        }
        // SolveBodyContactVelocityConstraints (:388-472)
        for (uint32_t it = 0; it < sc->vel_iters; ++it) {
            for (uint32_t k = 0; k < na; ++k) {
                BodyCon& x = con[k];
                const uint32_t i = x.slot % n;
                b3g_body_state* b = body_of(x.body1, x.slot / n);
                f3 vA = ld3(c.v, n, i), vB = body::ld3a(b->linear_velocity), wB = body::ld3a(b->angular_velocity);
                const f3 wA = zero3();
                {
                    const f3 dv = ((vB + cross(wB, x.rB)) - vA) - cross(wA, x.rA);
                    const float Cdot = dot(x.normal, dv);
                    float impulse = x.normal_mass * (-Cdot + 0.0f);
                    const float old = x.ni;
                    const float sum = old + impulse;
                    x.ni = sum > 0.0f ? sum : 0.0f;
                    impulse = x.ni - old;
                    const f3 P = impulse * x.normal;
                    vA = vA - x.mA * P;
                    vB = vB + x.mB * P;
                    wB = wB + x.iB * cross(x.rB, P);
                }
                {
                    const f3 dv = ((vB + cross(wB, x.rB)) - vA) - cross(wA, x.rA);
                    const float cx = dot(dv, x.t1), cy = dot(dv, x.t2);
                    const float ncx = -cx, ncy = -cy;
                    // Mat22 * Vec2 (mat22.h:56-59)
                    const float ix = ncx * x.tm_xx + ncy * x.tm_yx;
                    const float iy = ncx * x.tm_xy + ncy * x.tm_yy;
                    const float ox = x.tix, oy = x.tiy;
                    x.tix += ix;
                    x.tiy += iy;
                    const float maxImpulse = x.friction * x.ni;
                    if (x.tix * x.tix + x.tiy * x.tiy > maxImpulse * maxImpulse) {
                        float tx = x.tix, ty = x.tiy;
                        const float sl = sqrtf(tx * tx + ty * ty);
                        if (sl > FLT_EPSILON) {
                            tx /= sl;
                            ty /= sl;
                        }
                        x.tix = tx * maxImpulse;
                        x.tiy = ty * maxImpulse;
                    }
                    const f3 P = (x.tix - ox) * x.t1 + (x.tiy - oy) * x.t2;
                    vA = vA - x.mA * P;
                    vB = vB + x.mB * P;
                    wB = wB + x.iB * cross(x.rB, P);
                }
                st3(c.v, n, i, vA);
                set_velocity(b, vB, wB);
            }
        }
        // StoreImpulses (:598-616)
        for (uint32_t k = 0; k < na; ++k) {
            const BodyCon& x = con[k];
            c.c_imp[x.slot] = x.ni;
            c.c_imp[nn + x.slot] = x.tix;
            c.c_imp[2 * nn + x.slot] = x.tiy;
        }
    }
    __syncthreads();
    // integrate positions (cloth_solver.cpp:143-147)
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) st3(c.x, n, i, ld3(c.x, n, i) + h * ld3(c.v, n, i));
    __syncthreads();
    if (threadIdx.x != 0) return;
    const uint32_t na = s_na;
    // SolveBodyContactPositionConstraints (:620-718), early out (cloth_solver.cpp:151-164)
    for (uint32_t it = 0; it < sc->pos_iters; ++it) {
        float min_sep = 0.0f;
        for (uint32_t k = 0; k < na; ++k) {
            const BodyCon& x = con[k];
            const uint32_t i = x.slot % n;
            b3g_body_state* b = body_of(x.body1, x.slot / n);
            f3 cA = ld3(c.x, n, i);
            f3 cB = body::ld3a(b->world_center);
            body::Q4 qB = body::ldq(b->orientation);
            const m3 RA = body::qmat(body::Q4{0.0f, 0.0f, 0.0f, 1.0f}), RB = body::qmat(qB);
            const f3 pA = cA - RA * zero3(), pB = cB - RB * x.lcB;
            const f3 nA = ld3(c.c_normal, nn, x.slot);
            const f3 wcA = body::xmul(RA, pA, zero3()), wcB = body::xmul(RB, pB, x.lpB);
            const f3 point = wcB;
            const float separation = dot(wcB - wcA, nA) - x.radius_a - x.radius_b;
            min_sep = min_sep < separation ? min_sep : separation;
            const float Cv = kBaum * (separation + kSlop);
            float C = Cv < 0.0f ? Cv : 0.0f;
            C = -kMaxCorr > C ? -kMaxCorr : C;
            const f3 rA = point - cA, rB = point - cB;
            const f3 rnA = cross(rA, nA), rnB = cross(rB, nA);
            const m3 iA = mzero();
            const float K = x.mA + x.mB + dot(rnA, iA * rnA) + dot(rnB, x.iB * rnB);
            const float impulse = K > 0.0f ? -C / K : 0.0f;
            const f3 P = impulse * nA;
            cA = cA - x.mA * P;
            cB = cB + x.mB * P;
            const body::Q4 dB = body::qderiv(qB, x.iB * cross(rB, P));
            qB = body::Q4{qB.x + dB.x, qB.y + dB.y, qB.z + dB.z, qB.w + dB.w};
            body::qnormalize(qB);
            st3(c.x, n, i, cA);
            body::st3a(b->world_center, cB);
            body::stq(b->orientation, qB);
        }
        if (min_sep >= -3.0f * kSlop) break;
    }
    // synchronize the bodies of the active contacts (cloth_solver.cpp:167-181);
    // a body's synchronisation is idempotent, so once per touched body
    bool touched[kMaxSpheres] = {};
    for (uint32_t k = 0; k < na; ++k)
        if (con[k].body1) touched[con[k].body1 - 1] = true;
    for (uint32_t b = 0; b < c.nbody; ++b) {
        if (touched[b]) sync_body(c, sb[b], b);
        c.bodies[b] = sb[b];
    }
}
}  // namespace

// Scratch of the body solve, sized for every contact slot of the cloth.
struct BodyScratch {
    size_t slots = 0, temp_bytes = 0;
    unsigned long long *keys = nullptr, *keys_sorted = nullptr;
    uint32_t *idx = nullptr, *idx_sorted = nullptr;
    BodyCon* con = nullptr;
    void* temp = nullptr;
};

void body_scratch_free(BodyScratch* s)
{
    if (!s) return;
    cudaFree(s->keys);
    cudaFree(s->keys_sorted);
    cudaFree(s->idx);
    cudaFree(s->idx_sorted);
    cudaFree(s->con);
    cudaFree(s->temp);
    delete s;
}

// The contact solve of a cloth with body colliders, after its CG: the force
// solver's state update, the list order, then the ordered solve.
cudaError_t launch_body_solve(const ClothDev& c, BodyScratch*& s, cudaStream_t st)
{
    const size_t m = (size_t)c.nsph * c.n;
    if (m == 0) {
        k_body_prepare<<<(c.n + 255) / 256, 256, 0, st>>>(c);
        count_launches(1);
        return cudaGetLastError();
    }
    if (!s || s->slots < m) {
        body_scratch_free(s);
        s = new BodyScratch();
        s->slots = m;
        cudaError_t e = cudaMalloc(&s->keys, m * 8);
        if (e == cudaSuccess) e = cudaMalloc(&s->keys_sorted, m * 8);
        if (e == cudaSuccess) e = cudaMalloc(&s->idx, m * 4);
        if (e == cudaSuccess) e = cudaMalloc(&s->idx_sorted, m * 4);
        if (e == cudaSuccess) e = cudaMalloc(&s->con, m * sizeof(BodyCon));
        if (e == cudaSuccess)
            e = cub::DeviceRadixSort::SortPairs(nullptr, s->temp_bytes, s->keys, s->keys_sorted, s->idx,
                                                s->idx_sorted, (int)m);
        if (e == cudaSuccess) e = cudaMalloc(&s->temp, s->temp_bytes);
        if (e != cudaSuccess) {
            body_scratch_free(s);
            s = nullptr;
            return e;
        }
    }
    k_body_prepare<<<(c.n + 255) / 256, 256, 0, st>>>(c);
    const uint32_t grid = (uint32_t)std::min<size_t>((m + 255) / 256, 148 * 8);
    k_body_keys<<<grid, 256, 0, st>>>(c, s->keys, s->idx);
    size_t tb = s->temp_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(s->temp, tb, s->keys, s->keys_sorted, s->idx, s->idx_sorted,
                                                    (int)m, 0, 64, st);
    if (e != cudaSuccess) return e;
    k_body_solve<<<1, kSolveThreads, 0, st>>>(c, s->keys_sorted, s->idx_sorted, s->con);
    count_launches(3);
    return cudaGetLastError();
}

}  // namespace b3g
