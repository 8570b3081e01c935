// Test-only harness around the reference library (Bounce), compiled from the
// reference's unmodified sources by oracle/Makefile into oracle/_ref/.
//
// This file is test infrastructure.  It is linked only into the checker
// library oracle/_ref/libbounce_ref.so, which the parity tests, the golden
// fixture generator and the reference arm of bench.py load through ctypes.
// Nothing in the product (bounce_b200/, include/) links or calls it.
//
// What it adds around the reference, without editing any reference file:
//  * the two profile hooks the library leaves to its user
//    (include/bounce/common/settings.h:146-152), implemented as wall-clock
//    accumulators per scope name ("Cloth Step", "Cloth Solve",
//    "Cloth Solve MPCG", "Cloth Update Body Contacts", ...);
//  * harness_step(): b3Cloth::Step (src/bounce/cloth/cloth.cpp:551-601) with
//    the cloth self-collision pass left out (UpdateClothContacts,
//    triangle AABB sync, FindNewClothContacts).  At thickness 0 a
//    particle-triangle contact can only become active when the particle lies
//    exactly on a non-adjacent triangle
//    (src/bounce/cloth/contacts/cloth_particle_triangle_contact.cpp:144-170),
//    so leaving the pass out does not change the solve; the real Step is
//    also exported (ref_cloth_step with full=1) to show that on small cloths;
//  * restated_cloth(): the constructor (cloth.cpp:96-266) with its O(T^2)
//    shared-edge search (cloth.cpp:40-94) replaced by a directed-edge hash
//    that yields the same pairs in the same order.  Particles are still
//    created by the reference constructor, masses by b3Cloth::ComputeMass,
//    forces by b3Cloth::CreateForce / b3SpringForceDef::Initialize.  The
//    tests check it field by field against the real constructor;
//  * export of the assembled system A, b of one force solve
//    (cloth_force_solver.cpp:142-204), in the reference's own row order,
//    so the oracle's MPCG can be checked on identical inputs.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

// Reach members of b3Cloth / b3Particle / the contact manager without
// touching the reference headers.
#define private public
#define protected public
#include <bounce/bounce.h>
#include <bounce/cloth/cloth.h>
#include <bounce/cloth/cloth_mesh.h>
#include <bounce/cloth/particle.h>
#include <bounce/cloth/cloth_triangle.h>
#include <bounce/cloth/cloth_solver.h>
#include <bounce/cloth/cloth_force_solver.h>
#include <bounce/cloth/forces/force.h>
#include <bounce/cloth/forces/strech_force.h>
#include <bounce/cloth/forces/shear_force.h>
#include <bounce/cloth/forces/spring_force.h>
#include <bounce/cloth/forces/mouse_force.h>
#include <bounce/cloth/contacts/cloth_particle_body_contact.h>
#include <bounce/cloth/contacts/cloth_particle_triangle_contact.h>
#include <bounce/sparse/dense_vec3.h>
#include <bounce/sparse/diag_mat33.h>
#include <bounce/sparse/sparse_mat33.h>
#include <bounce/sparse/sparse_mat33_view.h>
#include <bounce/dynamics/world.h>
#include <bounce/dynamics/body.h>
#include <bounce/dynamics/shapes/sphere_shape.h>
#include <bounce/dynamics/shapes/hull_shape.h>
#include <bounce/collision/shapes/qhull.h>
#undef private
#undef protected

extern u32 b3_clothSolverIterations;

// ---------------------------------------------------------------------------
// Profile hooks
// ---------------------------------------------------------------------------

namespace {

typedef std::chrono::steady_clock clk;

struct ScopeAcc {
    double seconds = 0.0;
    uint64_t calls = 0;
};

std::vector<std::pair<std::string, clk::time_point>> g_scope_stack;
std::map<std::string, ScopeAcc> g_scopes;

}  // namespace

void b3BeginProfileScope(const char* name)
{
    g_scope_stack.emplace_back(std::string(name), clk::now());
}

void b3EndProfileScope()
{
    if (g_scope_stack.empty()) return;
    auto top = g_scope_stack.back();
    g_scope_stack.pop_back();
    ScopeAcc& a = g_scopes[top.first];
    a.seconds += std::chrono::duration<double>(clk::now() - top.second).count();
    a.calls += 1;
}

// ---------------------------------------------------------------------------
// Handle
// ---------------------------------------------------------------------------

namespace {

struct RefCloth {
    // The mesh must outlive the cloth (cloth.cpp:102 keeps the pointer).
    std::vector<b3Vec3> vertices;
    std::vector<b3ClothMeshTriangle> triangles;
    std::vector<b3ClothMeshSewingLine> sewing;
    b3ClothMeshMesh sub;
    b3ClothMesh mesh;
    b3Cloth* cloth = nullptr;
    b3World* world = nullptr;
    std::vector<b3SphereShape*> sphere_protos;
    std::vector<b3CapsuleShape*> capsule_protos;
    std::vector<b3HullShape*> hull_protos;
    std::vector<b3QHull*> hulls;  // the hulls the shapes point to
    std::vector<const b3Shape*> shapes;  // the world's shapes, in creation order
    std::vector<b3Body*> bodies;         // bodies made by ref_cloth_add_body
    // Particles made with b3Cloth::CreateParticle, addressed after the mesh
    // vertices (index vertexCount + k), and mouse forces by id - 1 (null once
    // destroyed).
    std::vector<b3Particle*> extra;
    std::vector<b3MouseForce*> mice;

    // Last exported system (solver-row order).
    std::vector<uint32_t> sys_rowptr, sys_cols, sys_vertex_of_row;
    std::vector<float> sys_vals, sys_b, sys_S, sys_x0;
};

b3Particle* particle_at(RefCloth* h, uint32_t i)
{
    u32 n = h->mesh.vertexCount;
    return i < n ? h->cloth->m_particles[i] : h->extra[i - n];
}

// Same pairs, same order as b3FindSharedEdges (cloth.cpp:40-94): for each
// triangle i, each of its edges (a -> b) in vertex order, every later
// triangle j > i that holds the reversed directed edge (b -> a), ascending j,
// taking the first matching edge slot of j.
struct SharedEdge {
    u32 v1, v2, nsv1, nsv2;
};

std::vector<SharedEdge> shared_edges_hashed(const b3ClothMesh* m)
{
    std::unordered_map<uint64_t, std::vector<std::pair<u32, u32>>> by_edge;
    by_edge.reserve(size_t(m->triangleCount) * 3);
    for (u32 t = 0; t < m->triangleCount; ++t) {
        const b3ClothMeshTriangle* tr = m->triangles + t;
        u32 vs[3] = {tr->v1, tr->v2, tr->v3};
        for (u32 e = 0; e < 3; ++e) {
            u32 a = vs[e], b = vs[e + 1 < 3 ? e + 1 : 0];
            by_edge[(uint64_t(a) << 32) | b].push_back(std::make_pair(t, e));
        }
    }
    std::vector<SharedEdge> out;
    for (u32 i = 0; i < m->triangleCount; ++i) {
        const b3ClothMeshTriangle* t1 = m->triangles + i;
        u32 i1s[3] = {t1->v1, t1->v2, t1->v3};
        for (u32 j1 = 0; j1 < 3; ++j1) {
            u32 k1 = j1 + 1 < 3 ? j1 + 1 : 0;
            u32 a = i1s[j1], b = i1s[k1];
            auto it = by_edge.find((uint64_t(b) << 32) | a);
            if (it == by_edge.end()) continue;
            u32 last_tri = ~0u;
            for (const auto& te : it->second) {
                u32 j = te.first;
                if (j <= i || j == last_tri) continue;
                last_tri = j;
                const b3ClothMeshTriangle* t2 = m->triangles + j;
                u32 i2s[3] = {t2->v1, t2->v2, t2->v3};
                u32 k2 = te.second + 1 < 3 ? te.second + 1 : 0;
                u32 k3 = k1 + 1 < 3 ? k1 + 1 : 0;
                u32 k4 = k2 + 1 < 3 ? k2 + 1 : 0;
                SharedEdge se;
                se.v1 = a;
                se.v2 = b;
                se.nsv1 = i1s[k3];
                se.nsv2 = i2s[k4];
                out.push_back(se);
            }
        }
    }
    return out;
}

// Constructor restated around an O(T) shared-edge search; follows
// cloth.cpp:96-266 step by step (see the file comment).
b3Cloth* restated_cloth(const b3ClothDef& def)
{
    const b3ClothMesh* m = def.mesh;

    // Particles: the reference constructor on a triangle-free copy of the
    // mesh creates them in the same order with the same defs (cloth.cpp:109-123).
    b3ClothMesh m0 = *m;
    m0.triangleCount = 0;
    m0.sewingLineCount = 0;
    b3ClothDef d0 = def;
    d0.mesh = &m0;
    b3Cloth* c = new b3Cloth(d0);
    c->m_mesh = m;

    // Lumped masses from the full mesh (cloth.cpp:126, :388-427).
    c->ComputeMass();

    // Triangles: rest-state frame, proxies and forces (cloth.cpp:129-215).
    b3Free(c->m_triangles);
    c->m_triangles = (b3ClothTriangle*)b3Alloc(m->triangleCount * sizeof(b3ClothTriangle));
    for (u32 i = 0; i < m->triangleCount; ++i) {
        b3ClothMeshTriangle* mt = m->triangles + i;
        b3ClothTriangle* tri = c->m_triangles + i;
        tri->m_cloth = c;
        tri->m_radius = def.thickness;
        tri->m_friction = def.friction;
        tri->m_triangle = i;

        b3Vec3 A = m->vertices[mt->v1];
        b3Vec3 B = m->vertices[mt->v2];
        b3Vec3 C = m->vertices[mt->v3];

        b3AABB3 aabb;
        aabb.Set(A, B, C);
        aabb.Extend(tri->m_radius);
        tri->m_aabbProxy.type = e_triangleProxy;
        tri->m_aabbProxy.owner = tri;
        tri->m_broadPhaseId = c->m_contactManager.m_broadPhase.CreateProxy(aabb, &tri->m_aabbProxy);

        b3Vec3 AB = B - A;
        b3Vec3 AC = C - A;
        float32 u1 = 0.0f, v1 = 0.0f;
        float32 u2 = b3Length(AB), v2 = 0.0f;
        b3Vec3 n_AB = AB / u2;
        float32 A2 = b3Length(b3Cross(AB, AC));
        float32 u3 = b3Dot(AC, n_AB);
        float32 v3 = A2 / u2;

        float32 du1 = u2 - u1, dv1 = v2 - v1;
        float32 du2 = u3 - u1, dv2 = v3 - v1;
        tri->m_du1 = du1;
        tri->m_dv1 = dv1;
        tri->m_du2 = du2;
        tri->m_dv2 = dv2;
        float32 det = du1 * dv2 - du2 * dv1;
        tri->m_inv_det = 1.0f / det;
        tri->m_alpha = 0.5f * A2;

        b3StrechForceDef sfdef;
        sfdef.triangle = tri;
        sfdef.streching = def.streching;
        sfdef.damping = def.damping;
        sfdef.bu = 1.0f;
        sfdef.bv = 1.0f;
        if (def.streching > 0.0f) c->CreateForce(sfdef);

        b3ShearForceDef shdef;
        shdef.triangle = tri;
        shdef.shearing = def.shearing;
        shdef.damping = def.damping;
        if (def.shearing > 0.0f) c->CreateForce(shdef);
    }

    // Bending springs between the non-shared vertices (cloth.cpp:227-243).
    std::vector<SharedEdge> shared = shared_edges_hashed(m);
    for (const SharedEdge& e : shared) {
        b3Particle* p3 = c->m_particles[e.nsv1];
        b3Particle* p4 = c->m_particles[e.nsv2];
        b3SpringForceDef fd;
        fd.Initialize(p3, p4, def.bending, def.damping);
        if (def.bending > 0.0f) c->CreateForce(fd);
    }

    // Sewing springs (cloth.cpp:248-262).
    for (u32 i = 0; i < m->sewingLineCount; ++i) {
        b3ClothMeshSewingLine* line = m->sewingLines + i;
        b3SpringForceDef fd;
        fd.Initialize(c->m_particles[line->v1], c->m_particles[line->v2], def.sewing, def.damping);
        if (def.sewing > 0.0f) c->CreateForce(fd);
    }
    return c;
}

// b3Cloth::Step without the self-collision pass (see the file comment).
void harness_step(b3Cloth* c, float32 dt, u32 vel_iters, u32 pos_iters)
{
    b3ProfileScope scope("Cloth Step");
    c->m_contactManager.UpdateBodyContacts();
    if (dt > 0.0f) c->Solve(dt, c->m_gravity, vel_iters, pos_iters);
    for (b3Particle* p = c->m_particleList.m_head; p; p = p->m_next) {
        p->m_force.SetZero();
        p->m_translation.SetZero();
    }
    for (b3Particle* p = c->m_particleList.m_head; p; p = p->m_next) {
        b3Vec3 displacement = dt * p->m_velocity;
        p->Synchronize(displacement);
    }
    c->m_contactManager.FindNewBodyContacts();
    // FindPairs would empty the move buffer (broad_phase.h:182); nothing reads it here.
    c->m_contactManager.m_broadPhase.m_moveBufferCount = 0;
}

inline void put3(float* dst, const b3Vec3& v)
{
    dst[0] = v.x;
    dst[1] = v.y;
    dst[2] = v.z;
}

}  // namespace

// ---------------------------------------------------------------------------
// C API (ctypes)
// ---------------------------------------------------------------------------

extern "C" {

// def: density, streching, shearing, bending, sewing, damping, thickness, friction
void* ref_cloth_create(const float* vertices, uint32_t vertex_count, const uint32_t* triangles,
                       uint32_t triangle_count, const uint32_t* sewing_lines, uint32_t sewing_count,
                       const float* def, int restated)
{
    RefCloth* h = new RefCloth();
    h->vertices.resize(vertex_count);
    for (uint32_t i = 0; i < vertex_count; ++i)
        h->vertices[i].Set(vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]);
    h->triangles.resize(triangle_count);
    for (uint32_t i = 0; i < triangle_count; ++i) {
        h->triangles[i].v1 = triangles[3 * i];
        h->triangles[i].v2 = triangles[3 * i + 1];
        h->triangles[i].v3 = triangles[3 * i + 2];
    }
    h->sewing.resize(sewing_count);
    for (uint32_t i = 0; i < sewing_count; ++i) {
        h->sewing[i].s1 = sewing_lines[4 * i];
        h->sewing[i].s2 = sewing_lines[4 * i + 1];
        h->sewing[i].v1 = sewing_lines[4 * i + 2];
        h->sewing[i].v2 = sewing_lines[4 * i + 3];
    }
    h->sub.vertexCount = vertex_count;
    h->sub.startVertex = 0;
    h->sub.triangleCount = triangle_count;
    h->sub.startTriangle = 0;
    h->mesh.vertexCount = vertex_count;
    h->mesh.vertices = h->vertices.data();
    h->mesh.triangleCount = triangle_count;
    h->mesh.triangles = h->triangles.data();
    h->mesh.meshCount = 1;
    h->mesh.meshes = &h->sub;
    h->mesh.sewingLineCount = sewing_count;
    h->mesh.sewingLines = sewing_count ? h->sewing.data() : nullptr;

    b3ClothDef d;
    d.mesh = &h->mesh;
    d.density = def[0];
    d.streching = def[1];
    d.shearing = def[2];
    d.bending = def[3];
    d.sewing = def[4];
    d.damping = def[5];
    d.thickness = def[6];
    d.friction = def[7];
    h->cloth = restated ? restated_cloth(d) : new b3Cloth(d);
    return h;
}

void ref_cloth_destroy(void* hp)
{
    RefCloth* h = (RefCloth*)hp;
    if (!h) return;
    if (h->cloth) {
        h->cloth->SetWorld(nullptr);
        delete h->cloth;
    }
    delete h->world;
    for (b3SphereShape* s : h->sphere_protos) delete s;
    for (b3CapsuleShape* s : h->capsule_protos) delete s;
    for (b3HullShape* s : h->hull_protos) delete s;
    for (b3QHull* q : h->hulls) delete q;
    delete h;
}

void ref_cloth_set_gravity(void* hp, const float* g)
{
    ((RefCloth*)hp)->cloth->SetGravity(b3Vec3(g[0], g[1], g[2]));
}

void ref_cloth_set_type(void* hp, uint32_t vertex, int type)
{
    particle_at((RefCloth*)hp, vertex)->SetType((b3ParticleType)type);
}

void ref_cloth_set_radius(void* hp, uint32_t vertex, float radius)
{
    particle_at((RefCloth*)hp, vertex)->SetRadius(radius);
}

void ref_cloth_set_friction(void* hp, uint32_t vertex, float friction)
{
    particle_at((RefCloth*)hp, vertex)->SetFriction(friction);
}

void ref_cloth_apply_force(void* hp, uint32_t vertex, const float* f)
{
    particle_at((RefCloth*)hp, vertex)->ApplyForce(b3Vec3(f[0], f[1], f[2]));
}

void ref_cloth_apply_translation(void* hp, uint32_t vertex, const float* t)
{
    particle_at((RefCloth*)hp, vertex)->ApplyTranslation(b3Vec3(t[0], t[1], t[2]));
}

void ref_cloth_set_position(void* hp, uint32_t vertex, const float* x)
{
    particle_at((RefCloth*)hp, vertex)->SetPosition(b3Vec3(x[0], x[1], x[2]));
}

void ref_cloth_set_velocity(void* hp, uint32_t vertex, const float* v)
{
    particle_at((RefCloth*)hp, vertex)->SetVelocity(b3Vec3(v[0], v[1], v[2]));
}

// A static body at `center` carrying one sphere shape of `radius`, in a world
// attached to the cloth as its collider provider (cloth.cpp:290).
void ref_cloth_add_sphere(void* hp, const float* center, float radius, float friction)
{
    RefCloth* h = (RefCloth*)hp;
    if (!h->world) {
        h->world = new b3World();
        h->cloth->SetWorld(h->world);
    }
    b3BodyDef bd;
    bd.type = e_staticBody;
    bd.position.Set(center[0], center[1], center[2]);
    b3Body* body = h->world->CreateBody(bd);
    b3SphereShape* sphere = new b3SphereShape();
    sphere->m_center.SetZero();
    sphere->m_radius = radius;
    h->sphere_protos.push_back(sphere);
    b3ShapeDef sd;
    sd.shape = sphere;
    sd.friction = friction;
    h->shapes.push_back(body->CreateShape(sd));
}

// A body of any type (b3BodyDef: type 0 static, 1 kinematic, 2 dynamic,
// position, orientation x y z w, linear and angular velocity) in the cloth's
// world; shapes are added to it with the calls below.  Returns its index.
uint32_t ref_cloth_add_body(void* hp, int type, const float* position, const float* orientation,
                            const float* velocity, const float* angular_velocity)
{
    RefCloth* h = (RefCloth*)hp;
    if (!h->world) {
        h->world = new b3World();
        h->cloth->SetWorld(h->world);
    }
    b3BodyDef bd;
    bd.type = (b3BodyType)type;
    bd.position.Set(position[0], position[1], position[2]);
    bd.orientation.Set(orientation[0], orientation[1], orientation[2], orientation[3]);
    bd.linearVelocity.Set(velocity[0], velocity[1], velocity[2]);
    bd.angularVelocity.Set(angular_velocity[0], angular_velocity[1], angular_velocity[2]);
    h->bodies.push_back(h->world->CreateBody(bd));
    return (uint32_t)h->bodies.size() - 1;
}

// A shape on one of those bodies, its geometry in the body's frame, with
// density (the body's mass follows, b3Body::ResetMass) and friction.
// kind 0 sphere (centre, radius), 1 capsule (a, b, radius); returns the
// shape's index among the world's shapes.
uint32_t ref_cloth_add_body_shape(void* hp, uint32_t body, int kind, const float* geom, float radius, float density,
                                  float friction)
{
    RefCloth* h = (RefCloth*)hp;
    b3ShapeDef sd;
    sd.density = density;
    sd.friction = friction;
    if (kind == 0) {
        b3SphereShape* sphere = new b3SphereShape();
        sphere->m_center.Set(geom[0], geom[1], geom[2]);
        sphere->m_radius = radius;
        h->sphere_protos.push_back(sphere);
        sd.shape = sphere;
    } else {
        b3CapsuleShape* cap = new b3CapsuleShape();
        cap->m_centers[0].Set(geom[0], geom[1], geom[2]);
        cap->m_centers[1].Set(geom[3], geom[4], geom[5]);
        cap->m_radius = radius;
        h->capsule_protos.push_back(cap);
        sd.shape = cap;
    }
    h->shapes.push_back(h->bodies[body]->CreateShape(sd));
    return (uint32_t)h->shapes.size() - 1;
}

// A hull (the reference's quickhull of `points`) on one of those bodies;
// writes its vertices and planes like ref_cloth_add_hull.
uint32_t ref_cloth_add_body_hull(void* hp, uint32_t body, const float* points, uint32_t count, float density,
                                 float friction, float* vertices, float* planes, uint32_t* face_count)
{
    RefCloth* h = (RefCloth*)hp;
    std::vector<b3Vec3> pts(count);
    for (uint32_t i = 0; i < count; ++i) pts[i].Set(points[3 * i], points[3 * i + 1], points[3 * i + 2]);
    b3QHull* hull = new b3QHull();
    hull->Set(sizeof(b3Vec3), pts.data(), count);
    h->hulls.push_back(hull);
    b3HullShape* shape = new b3HullShape();
    shape->m_hull = hull;
    h->hull_protos.push_back(shape);
    b3ShapeDef sd;
    sd.shape = shape;
    sd.density = density;
    sd.friction = friction;
    h->shapes.push_back(h->bodies[body]->CreateShape(sd));
    for (uint32_t i = 0; i < hull->vertexCount; ++i) put3(vertices + 3 * i, hull->vertices[i]);
    for (uint32_t i = 0; i < hull->faceCount; ++i) {
        put3(planes + 4 * i, hull->planes[i].normal);
        planes[4 * i + 3] = hull->planes[i].offset;
    }
    *face_count = hull->faceCount;
    return hull->vertexCount;
}

// A body's state as 55 floats: type, m_xf (rotation column-major, position),
// m_sweep (local center, world center 0, world center, orientation 0,
// orientation), velocities, inverse mass, local and world inverse inertia.
void ref_cloth_get_body(void* hp, uint32_t body, float* d)
{
    const b3Body* b = ((RefCloth*)hp)->bodies[body];
    d[0] = (float)b->m_type;
    put3(d + 1, b->m_xf.rotation.x); put3(d + 4, b->m_xf.rotation.y); put3(d + 7, b->m_xf.rotation.z);
    put3(d + 10, b->m_xf.position);
    put3(d + 13, b->m_sweep.localCenter); put3(d + 16, b->m_sweep.worldCenter0); put3(d + 19, b->m_sweep.worldCenter);
    const b3Quat& q0 = b->m_sweep.orientation0;
    const b3Quat& q = b->m_sweep.orientation;
    d[22] = q0.x; d[23] = q0.y; d[24] = q0.z; d[25] = q0.w;
    d[26] = q.x; d[27] = q.y; d[28] = q.z; d[29] = q.w;
    put3(d + 30, b->m_linearVelocity); put3(d + 33, b->m_angularVelocity);
    d[36] = b->m_invMass;
    put3(d + 37, b->m_invI.x); put3(d + 40, b->m_invI.y); put3(d + 43, b->m_invI.z);
    put3(d + 46, b->m_worldInvI.x); put3(d + 49, b->m_worldInvI.y); put3(d + 52, b->m_worldInvI.z);
}

// A shape's proxy in the world broadphase (b3Shape::GetAABB).
void ref_cloth_get_shape_proxy(void* hp, uint32_t shape, float* lo, float* hi)
{
    const b3AABB3& a = ((RefCloth*)hp)->shapes[shape]->GetAABB();
    put3(lo, a.m_lower);
    put3(hi, a.m_upper);
}

// The world's shapes in the order a query over everything reports them (its
// dynamic tree's order, b3World::QueryAABB, world.cpp:464-470); returns the
// count written.
struct ReportAll : public b3QueryListener {
    RefCloth* h;
    std::vector<uint32_t> out;
    bool ReportShape(b3Shape* s) override
    {
        uint32_t k = 0;
        while (k < h->shapes.size() && h->shapes[k] != s) ++k;
        out.push_back(k);
        return true;
    }
};

uint32_t ref_world_report_order(void* hp, uint32_t* order)
{
    RefCloth* h = (RefCloth*)hp;
    if (!h->world) return 0;
    ReportAll all;
    all.h = h;
    b3AABB3 box;
    box.m_lower.Set(-1e30f, -1e30f, -1e30f);
    box.m_upper.Set(1e30f, 1e30f, 1e30f);
    h->world->QueryAABB(&all, box);
    for (size_t k = 0; k < all.out.size(); ++k) order[k] = all.out[k];
    return (uint32_t)all.out.size();
}

// b3World::Step of the cloth's world (rigid bodies only).
void ref_world_step(void* hp, float dt, uint32_t velocity_iterations, uint32_t position_iterations)
{
    RefCloth* h = (RefCloth*)hp;
    if (h->world) h->world->Step(dt, velocity_iterations, position_iterations);
}

void ref_world_set_gravity(void* hp, const float* g)
{
    RefCloth* h = (RefCloth*)hp;
    if (h->world) h->world->SetGravity(b3Vec3(g[0], g[1], g[2]));
}

// A static body at the origin carrying one capsule shape, segment a-b.
void ref_cloth_add_capsule(void* hp, const float* a, const float* b, float radius, float friction)
{
    RefCloth* h = (RefCloth*)hp;
    if (!h->world) {
        h->world = new b3World();
        h->cloth->SetWorld(h->world);
    }
    b3BodyDef bd;
    bd.type = e_staticBody;
    b3Body* body = h->world->CreateBody(bd);
    b3CapsuleShape* cap = new b3CapsuleShape();
    cap->m_centers[0].Set(a[0], a[1], a[2]);
    cap->m_centers[1].Set(b[0], b[1], b[2]);
    cap->m_radius = radius;
    h->capsule_protos.push_back(cap);
    b3ShapeDef sd;
    sd.shape = cap;
    sd.friction = friction;
    h->shapes.push_back(body->CreateShape(sd));
}

// A static body at the origin with a b3HullShape: the hull b3QHull::Set
// builds from `points` (quickhull), friction as given.  Its vertices (3 floats
// each, at most 256) and face planes (normal and offset, 4 floats each, at most
// 256) are written out; returns the vertex count, *face_count the face count.
uint32_t ref_cloth_add_hull(void* hp, const float* points, uint32_t count, float friction, float* vertices,
                            float* planes, uint32_t* face_count)
{
    RefCloth* h = (RefCloth*)hp;
    if (!h->world) {
        h->world = new b3World();
        h->cloth->SetWorld(h->world);
    }
    std::vector<b3Vec3> pts(count);
    for (uint32_t i = 0; i < count; ++i) pts[i].Set(points[3 * i], points[3 * i + 1], points[3 * i + 2]);
    b3QHull* hull = new b3QHull();
    hull->Set(sizeof(b3Vec3), pts.data(), count);
    h->hulls.push_back(hull);
    b3BodyDef bd;
    bd.type = e_staticBody;
    b3Body* body = h->world->CreateBody(bd);
    b3HullShape* shape = new b3HullShape();
    shape->m_hull = hull;
    h->hull_protos.push_back(shape);
    b3ShapeDef sd;
    sd.shape = shape;
    sd.friction = friction;
    h->shapes.push_back(body->CreateShape(sd));
    for (uint32_t i = 0; i < hull->vertexCount; ++i) put3(vertices + 3 * i, hull->vertices[i]);
    for (uint32_t i = 0; i < hull->faceCount; ++i) {
        put3(planes + 4 * i, hull->planes[i].normal);
        planes[4 * i + 3] = hull->planes[i].offset;
    }
    *face_count = hull->faceCount;
    return hull->vertexCount;
}

// full = 1: the reference's own b3Cloth::Step; full = 0: harness_step.
void ref_cloth_step(void* hp, float dt, uint32_t vel_iters, uint32_t pos_iters, int full)
{
    RefCloth* h = (RefCloth*)hp;
    if (full)
        h->cloth->Step(dt, vel_iters, pos_iters);
    else
        harness_step(h->cloth, dt, vel_iters, pos_iters);
}

uint32_t ref_last_iterations() { return b3_clothSolverIterations; }

// Per vertex index: position, velocity, last CG solution m_x (3 floats each),
// mass and type.
void ref_cloth_get_state(void* hp, float* x, float* v, float* dv, float* mass, uint8_t* type)
{
    RefCloth* h = (RefCloth*)hp;
    u32 n = h->mesh.vertexCount + (u32)h->extra.size();
    for (u32 i = 0; i < n; ++i) {
        b3Particle* p = particle_at(h, i);
        if (x) put3(x + 3 * i, p->m_position);
        if (v) put3(v + 3 * i, p->m_velocity);
        if (dv) put3(dv + 3 * i, p->m_x);
        if (mass) mass[i] = p->m_mass;
        if (type) type[i] = (uint8_t)p->m_type;
    }
}

float ref_cloth_energy(void* hp) { return ((RefCloth*)hp)->cloth->GetEnergy(); }

// b3Cloth::CreateParticle (cloth.cpp:307-322); returns the particle's index.
uint32_t ref_cloth_create_particle(void* hp, const float* position, const float* velocity, float mass, float radius,
                                   float friction)
{
    RefCloth* h = (RefCloth*)hp;
    b3ParticleDef pd;
    pd.mass = mass;
    pd.position.Set(position[0], position[1], position[2]);
    if (velocity) pd.velocity.Set(velocity[0], velocity[1], velocity[2]);
    pd.radius = radius;
    pd.friction = friction;
    h->extra.push_back(h->cloth->CreateParticle(pd));
    return h->mesh.vertexCount + (uint32_t)h->extra.size() - 1;
}

// b3Cloth::DestroyParticle (cloth.cpp:324-351) of a created particle; the
// mouse forces it takes with it are forgotten here too.
int ref_cloth_destroy_particle(void* hp, uint32_t i)
{
    RefCloth* h = (RefCloth*)hp;
    u32 n = h->mesh.vertexCount;
    if (i < n || i >= n + h->extra.size()) return -1;
    b3Particle* p = h->extra[i - n];
    for (b3MouseForce*& m : h->mice)
        if (m && m->HasParticle(p)) m = nullptr;
    h->cloth->DestroyParticle(p);
    h->extra.erase(h->extra.begin() + (i - n));
    return 0;
}

// b3Cloth::CreateForce (cloth.cpp:353-358) of a b3MouseForceDef; returns its id.
uint32_t ref_cloth_create_mouse_force(void* hp, uint32_t particle, uint32_t triangle, float w2, float w3, float w4,
                                      float mouse, float damping)
{
    RefCloth* h = (RefCloth*)hp;
    b3MouseForceDef def;
    def.particle = particle_at(h, particle);
    def.triangle = h->cloth->GetTriangle(triangle);
    def.w2 = w2;
    def.w3 = w3;
    def.w4 = w4;
    def.mouse = mouse;
    def.damping = damping;
    h->mice.push_back((b3MouseForce*)h->cloth->CreateForce(def));
    return (uint32_t)h->mice.size();
}

// b3Cloth::DestroyForce (cloth.cpp:360-364)
int ref_cloth_destroy_force(void* hp, uint32_t id)
{
    RefCloth* h = (RefCloth*)hp;
    if (id == 0 || id > h->mice.size() || !h->mice[id - 1]) return -1;
    h->cloth->DestroyForce(h->mice[id - 1]);
    h->mice[id - 1] = nullptr;
    return 0;
}

uint32_t ref_cloth_particle_count(void* hp)
{
    RefCloth* h = (RefCloth*)hp;
    return h->mesh.vertexCount + (uint32_t)h->extra.size();
}

// Rest state per triangle (du1, dv1, du2, dv2, inv_det, alpha), particle fat
// AABBs (lower xyz, upper xyz) and the force list in application order.
// force_desc: 8 floats per force: type, a, b, c (vertex ids), p0, p1, p2, p3
//   stretch: ks, kd, bu, bv   shear: ks, kd, 0, 0   spring: ks, kd, L0, 0
uint32_t ref_cloth_describe(void* hp, float* tri_rest, float* fat_aabb, float* force_desc)
{
    RefCloth* h = (RefCloth*)hp;
    b3Cloth* c = h->cloth;
    if (tri_rest) {
        for (u32 i = 0; i < h->mesh.triangleCount; ++i) {
            b3ClothTriangle* t = c->m_triangles + i;
            float* o = tri_rest + 6 * i;
            o[0] = t->m_du1;
            o[1] = t->m_dv1;
            o[2] = t->m_du2;
            o[3] = t->m_dv2;
            o[4] = t->m_inv_det;
            o[5] = t->m_alpha;
        }
    }
    if (fat_aabb) {
        for (u32 i = 0; i < h->mesh.vertexCount; ++i) {
            b3Particle* p = c->m_particles[i];
            b3AABB3 a = c->m_contactManager.m_broadPhase.GetAABB(p->m_broadPhaseId);
            put3(fat_aabb + 6 * i, a.m_lower);
            put3(fat_aabb + 6 * i + 3, a.m_upper);
        }
    }
    uint32_t k = 0;
    for (b3Force* f = c->m_forceList.m_head; f; f = f->m_next, ++k) {
        if (!force_desc) continue;
        float* o = force_desc + 8 * k;
        std::memset(o, 0, 8 * sizeof(float));
        o[0] = (float)f->m_type;
        if (f->m_type == e_strechForce || f->m_type == e_shearForce) {
            b3ClothTriangle* t = f->m_type == e_strechForce ? ((b3StrechForce*)f)->m_triangle
                                                            : ((b3ShearForce*)f)->m_triangle;
            b3ClothMeshTriangle* mt = h->mesh.triangles + t->m_triangle;
            o[1] = (float)mt->v1;
            o[2] = (float)mt->v2;
            o[3] = (float)mt->v3;
            if (f->m_type == e_strechForce) {
                b3StrechForce* s = (b3StrechForce*)f;
                o[4] = s->m_ks;
                o[5] = s->m_kd;
                o[6] = s->m_bu;
                o[7] = s->m_bv;
            } else {
                b3ShearForce* s = (b3ShearForce*)f;
                o[4] = s->m_ks;
                o[5] = s->m_kd;
            }
        } else if (f->m_type == e_springForce) {
            b3SpringForce* s = (b3SpringForce*)f;
            o[1] = (float)s->m_p1->m_vertex;
            o[2] = (float)s->m_p2->m_vertex;
            o[3] = -1.0f;
            o[4] = s->m_ks;
            o[5] = s->m_kd;
            o[6] = s->m_L0;
        }
    }
    return k;
}

// Body contacts per vertex: exists, active, normal impulse, tangent impulse (2).
uint32_t ref_cloth_get_contacts(void* hp, uint8_t* exists, uint8_t* active, float* impulses)
{
    RefCloth* h = (RefCloth*)hp;
    u32 n = h->mesh.vertexCount;
    if (exists) std::memset(exists, 0, n);
    if (active) std::memset(active, 0, n);
    if (impulses) std::memset(impulses, 0, 3 * n * sizeof(float));
    uint32_t count = 0;
    for (b3ParticleBodyContact* c = h->cloth->m_contactManager.m_particleBodyContactList.m_head; c;
         c = c->m_next, ++count) {
        u32 vtx = c->m_p1->m_vertex;
        if (exists) exists[vtx] = 1;
        if (active) active[vtx] = c->m_active ? 1 : 0;
        if (impulses) {
            impulses[3 * vtx] = c->m_normalImpulse;
            impulses[3 * vtx + 1] = c->m_tangentImpulse.x;
            impulses[3 * vtx + 2] = c->m_tangentImpulse.y;
        }
    }
    return count;
}

// The particle-body contact list from its head: particle, shape (creation
// index), active flag, impulses; at most `cap` written, the count returned.
uint32_t ref_cloth_get_contact_list(void* hp, uint32_t cap, uint32_t* particle, uint32_t* shape, uint8_t* active,
                                    float* impulses)
{
    RefCloth* h = (RefCloth*)hp;
    uint32_t count = 0;
    for (b3ParticleBodyContact* c = h->cloth->m_contactManager.m_particleBodyContactList.m_head; c;
         c = c->m_next, ++count) {
        if (count >= cap) continue;
        particle[count] = c->m_p1->m_vertex;
        uint32_t s = 0;
        while (s < h->shapes.size() && h->shapes[s] != c->m_s2) ++s;
        shape[count] = s;
        active[count] = c->m_active ? 1 : 0;
        impulses[3 * count] = c->m_normalImpulse;
        impulses[3 * count + 1] = c->m_tangentImpulse.x;
        impulses[3 * count + 2] = c->m_tangentImpulse.y;
    }
    return count;
}

// b3Cloth::RayCastSingle: 1 on a hit, with the triangle, fraction and normal.
int ref_cloth_ray_cast_single(void* hp, const float* p1, const float* p2, uint32_t* triangle, float* fraction,
                              float* normal)
{
    RefCloth* h = (RefCloth*)hp;
    b3ClothRayCastSingleOutput out;
    if (!h->cloth->RayCastSingle(&out, b3Vec3(p1[0], p1[1], p1[2]), b3Vec3(p2[0], p2[1], p2[2]))) return 0;
    *triangle = out.triangle;
    *fraction = out.fraction;
    put3(normal, out.normal);
    return 1;
}

// Particle-triangle contacts in list order (head first): particle vertex and
// triangle index (2 per contact), active flag, barycentric weights
// m_w2, m_w3, m_w4 and the normal and two tangent impulses.  Any pointer may
// be null.  Returns the number of contacts.
uint32_t ref_cloth_get_tri_contacts(void* hp, uint32_t* pt, uint8_t* active, float* w, float* impulses)
{
    RefCloth* h = (RefCloth*)hp;
    uint32_t k = 0;
    for (b3ParticleTriangleContact* c = h->cloth->m_contactManager.m_particleTriangleContactList.m_head; c;
         c = c->m_next, ++k) {
        if (pt) {
            pt[2 * k] = c->m_p1->m_vertex;
            pt[2 * k + 1] = c->m_t2->m_triangle;
        }
        if (active) active[k] = c->m_active ? 1 : 0;
        if (w) {
            w[3 * k] = c->m_w2;
            w[3 * k + 1] = c->m_w3;
            w[3 * k + 2] = c->m_w4;
        }
        if (impulses) {
            impulses[3 * k] = c->m_normalImpulse;
            impulses[3 * k + 1] = c->m_tangentImpulse1;
            impulses[3 * k + 2] = c->m_tangentImpulse2;
        }
    }
    return k;
}

// Assemble A and b exactly as one force solve would (the gather of
// cloth_force_solver.cpp:164-188 restated, then the reference's own
// ApplyForces and sparse operators, :191-204) and keep them in the handle.
// Rows are in solver order (particle-list order, b3ClothSolver::Add); each
// row's blocks are in the order of the reference's b3SparseMat33View.
// Returns the number of blocks.
uint32_t ref_cloth_build_system(void* hp, float dt)
{
    RefCloth* h = (RefCloth*)hp;
    b3Cloth* c = h->cloth;
    u32 n = c->m_particleList.m_count;
    std::vector<b3Particle*> particles;
    std::vector<b3Force*> forces;
    for (b3Particle* p = c->m_particleList.m_head; p; p = p->m_next) {
        p->m_solverId = (u32)particles.size();
        particles.push_back(p);
    }
    for (b3Force* f = c->m_forceList.m_head; f; f = f->m_next) forces.push_back(f);

    b3ClothForceSolverDef fdef;
    fdef.stack = &c->m_stackAllocator;
    fdef.particleCount = n;
    fdef.particles = particles.data();
    fdef.forceCount = (u32)forces.size();
    fdef.forces = forces.data();
    b3ClothForceSolver fs(fdef);

    float32 hstep = dt;
    b3Vec3 gravity = c->m_gravity;
    b3DenseVec3 sx(n), sv(n), sf(n), sy(n), sz(n), sx0(n);
    b3SparseMat33 M(n), dfdx(n), dfdv(n);
    b3DiagMat33 S(n);
    fs.m_solverData.x = &sx;
    fs.m_solverData.v = &sv;
    fs.m_solverData.f = &sf;
    fs.m_solverData.y = &sy;
    fs.m_solverData.z = &sz;
    fs.m_solverData.dfdx = &dfdx;
    fs.m_solverData.dfdv = &dfdv;
    fs.m_solverData.S = &S;
    for (u32 i = 0; i < n; ++i) {
        b3Particle* p = particles[i];
        M(i, i) = b3Diagonal(p->m_mass);
        sx[i] = p->m_position;
        sv[i] = p->m_velocity;
        sf[i] = p->m_force;
        sz[i].SetZero();
        if (p->m_type == e_dynamicParticle) {
            sf[i] += p->m_mass * gravity;
            S[i].SetIdentity();
        } else {
            S[i].SetZero();
        }
        sy[i] = p->m_translation;
        sx0[i] = p->m_x;
    }
    fs.ApplyForces();
    b3SparseMat33 A = M - hstep * dfdv - (hstep * hstep) * dfdx;
    b3SparseMat33View viewA(A);
    b3DenseVec3 b = hstep * (sf + hstep * (dfdx * sv) + dfdx * sy);

    h->sys_rowptr.assign(n + 1, 0);
    h->sys_cols.clear();
    h->sys_vals.clear();
    h->sys_b.assign(3 * n, 0.0f);
    h->sys_S.assign(n, 0.0f);
    h->sys_x0.assign(3 * n, 0.0f);
    h->sys_vertex_of_row.assign(n, 0);
    for (u32 i = 0; i < n; ++i) {
        b3RowValueArray* row = viewA.rows + i;
        for (u32 k = 0; k < row->count; ++k) {
            h->sys_cols.push_back(row->values[k].column);
            const b3Mat33& m = row->values[k].value;
            const float vals[9] = {m.x.x, m.x.y, m.x.z, m.y.x, m.y.y, m.y.z, m.z.x, m.z.y, m.z.z};
            h->sys_vals.insert(h->sys_vals.end(), vals, vals + 9);
        }
        h->sys_rowptr[i + 1] = (uint32_t)h->sys_cols.size();
        put3(&h->sys_b[3 * i], b[i]);
        put3(&h->sys_x0[3 * i], sx0[i]);
        h->sys_S[i] = S[i].x.x;
    {
        // created particles have no mesh vertex: report their index
        uint32_t v = particles[i]->m_vertex;
        if (v == ~0u)
            for (size_t k = 0; k < h->extra.size(); ++k)
                if (h->extra[k] == particles[i]) v = h->mesh.vertexCount + (uint32_t)k;
        h->sys_vertex_of_row[i] = v;
    }
    }
    return (uint32_t)h->sys_cols.size();
}

void ref_cloth_get_system(void* hp, uint32_t* rowptr, uint32_t* cols, float* vals, float* b,
                          float* S, float* x0, uint32_t* vertex_of_row)
{
    RefCloth* h = (RefCloth*)hp;
    std::copy(h->sys_rowptr.begin(), h->sys_rowptr.end(), rowptr);
    std::copy(h->sys_cols.begin(), h->sys_cols.end(), cols);
    std::copy(h->sys_vals.begin(), h->sys_vals.end(), vals);
    std::copy(h->sys_b.begin(), h->sys_b.end(), b);
    std::copy(h->sys_S.begin(), h->sys_S.end(), S);
    std::copy(h->sys_x0.begin(), h->sys_x0.end(), x0);
    std::copy(h->sys_vertex_of_row.begin(), h->sys_vertex_of_row.end(), vertex_of_row);
}

// Profile scopes: names joined by '\n' into `names` (capacity bytes), seconds
// and call counts in the same order.  Returns the number of scopes.
uint32_t ref_profile_read(char* names, uint32_t capacity, double* seconds, uint64_t* calls)
{
    std::string joined;
    uint32_t k = 0;
    for (const auto& kv : g_scopes) {
        joined += kv.first;
        joined += '\n';
        if (seconds) seconds[k] = kv.second.seconds;
        if (calls) calls[k] = kv.second.calls;
        ++k;
    }
    if (names && capacity) {
        size_t m = std::min<size_t>(capacity - 1, joined.size());
        std::memcpy(names, joined.data(), m);
        names[m] = 0;
    }
    return k;
}

void ref_profile_reset() { g_scopes.clear(); }

}  // extern "C"
