// Test-only harness around the reference's soft body (b3SoftBody), compiled
// with the reference's unmodified sources into oracle/_ref/libbounce_ref.so
// (see ref_harness.cpp for the profile hooks the library needs).
//
// One adjustment, without editing any reference file: the constructor
// (src/bounce/softbody/softbody.cpp:484-553) never sets b3SoftBodyElement::q,
// the rotation b3ExtractRotation (softbody_force_solver.cpp:53-91) starts
// from, so the reference reads whatever its allocator left there (with
// zero-filled memory q = 0, which the extraction can never leave, and the
// stiffness warping is silently off).  The harness sets every q to the
// identity, the rotation of the rest state, right after construction.

#include <cstdint>
#include <cstring>
#include <vector>

#define private public
#define protected public
#include <bounce/bounce.h>
#include <bounce/softbody/softbody.h>
#include <bounce/softbody/softbody_mesh.h>
#include <bounce/softbody/softbody_node.h>
#include <bounce/softbody/contacts/softbody_node_body_contact.h>
#include <bounce/dynamics/world.h>
#include <bounce/dynamics/body.h>
#include <bounce/dynamics/shapes/hull_shape.h>
#include <bounce/collision/shapes/qhull.h>
#undef private
#undef protected

extern u32 b3_softBodySolverIterations;

namespace {

struct RefSoftBody {
    std::vector<b3Vec3> vertices;
    std::vector<b3SoftBodyMeshTetrahedron> tets;
    b3SoftBodyMesh mesh;
    b3SoftBody* body = nullptr;
    b3World* world = nullptr;
    std::vector<b3QHull*> hulls;
    std::vector<b3HullShape*> protos;
    std::vector<const b3Shape*> shapes;  // the world's shapes, in creation order
};

}  // namespace

extern "C" {

// def: density, E, nu, c_yield, c_creep, c_max
void* ref_softbody_create(const float* vertices, uint32_t vertex_count, const uint32_t* tets, uint32_t tet_count,
                          const float* def)
{
    RefSoftBody* h = new RefSoftBody();
    h->vertices.resize(vertex_count);
    for (uint32_t i = 0; i < vertex_count; ++i)
        h->vertices[i].Set(vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]);
    h->tets.resize(tet_count);
    for (uint32_t i = 0; i < tet_count; ++i) {
        h->tets[i].v1 = tets[4 * i];
        h->tets[i].v2 = tets[4 * i + 1];
        h->tets[i].v3 = tets[4 * i + 2];
        h->tets[i].v4 = tets[4 * i + 3];
    }
    h->mesh.vertexCount = vertex_count;
    h->mesh.vertices = h->vertices.data();
    h->mesh.tetrahedronCount = tet_count;
    h->mesh.tetrahedrons = h->tets.data();
    b3SoftBodyDef d;
    d.mesh = &h->mesh;
    d.density = def[0];
    d.E = def[1];
    d.nu = def[2];
    d.c_yield = def[3];
    d.c_creep = def[4];
    d.c_max = def[5];
    h->body = new b3SoftBody(d);
    for (uint32_t e = 0; e < tet_count; ++e) h->body->m_elements[e].q.SetIdentity();
    return h;
}

void ref_softbody_destroy(void* p)
{
    RefSoftBody* h = static_cast<RefSoftBody*>(p);
    delete h->body;
    delete h->world;
    for (b3HullShape* s : h->protos) delete s;
    for (b3QHull* q : h->hulls) delete q;
    delete h;
}

// A world with a static body at the origin carrying a b3HullShape built by
// the reference's quickhull from `points` (b3SoftBody::SetWorld); writes the
// hull's vertices and planes (at most 256 each), returns the vertex count.
uint32_t ref_softbody_add_hull(void* p, const float* points, uint32_t count, float friction, float* vertices,
                               float* planes, uint32_t* face_count)
{
    RefSoftBody* h = static_cast<RefSoftBody*>(p);
    if (!h->world) {
        h->world = new b3World();
        h->body->SetWorld(h->world);
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
    h->protos.push_back(shape);
    b3ShapeDef sd;
    sd.shape = shape;
    sd.friction = friction;
    h->shapes.push_back(body->CreateShape(sd));
    for (uint32_t i = 0; i < hull->vertexCount; ++i) {
        vertices[3 * i] = hull->vertices[i].x;
        vertices[3 * i + 1] = hull->vertices[i].y;
        vertices[3 * i + 2] = hull->vertices[i].z;
    }
    for (uint32_t i = 0; i < hull->faceCount; ++i) {
        planes[4 * i] = hull->planes[i].normal.x;
        planes[4 * i + 1] = hull->planes[i].normal.y;
        planes[4 * i + 2] = hull->planes[i].normal.z;
        planes[4 * i + 3] = hull->planes[i].offset;
    }
    *face_count = hull->faceCount;
    return hull->vertexCount;
}

// b3SoftBodyNode::SetRadius / SetFriction
void ref_softbody_set_node_radius(void* p, uint32_t i, float r)
{
    static_cast<RefSoftBody*>(p)->body->m_nodes[i].SetRadius(r);
}
void ref_softbody_set_node_friction(void* p, uint32_t i, float f)
{
    static_cast<RefSoftBody*>(p)->body->m_nodes[i].SetFriction(f);
}

// Node-body contacts (one shape): per node exists, active, normal and
// tangent impulses; returns the contact count.
uint32_t ref_softbody_get_contacts(void* p, uint8_t* exists, uint8_t* active, float* impulses)
{
    RefSoftBody* h = static_cast<RefSoftBody*>(p);
    const uint32_t n = h->mesh.vertexCount;
    std::memset(exists, 0, n);
    std::memset(active, 0, n);
    std::memset(impulses, 0, 3 * (size_t)n * sizeof(float));
    uint32_t count = 0;
    for (b3NodeBodyContact* c = h->body->m_contactManager.m_nodeBodyContactList.m_head; c; c = c->m_next, ++count) {
        const uint32_t v = c->m_n1->m_vertex;
        exists[v] = 1;
        active[v] = c->m_active ? 1 : 0;
        impulses[3 * v] = c->m_normalImpulse;
        impulses[3 * v + 1] = c->m_tangentImpulse.x;
        impulses[3 * v + 2] = c->m_tangentImpulse.y;
    }
    return count;
}

// The node-body contact list from its head: node, hull (creation index),
// active flag, impulses; at most `cap` written, the count returned.
uint32_t ref_softbody_get_contact_list(void* p, uint32_t cap, uint32_t* node, uint32_t* shape, uint8_t* active,
                                       float* impulses)
{
    RefSoftBody* h = static_cast<RefSoftBody*>(p);
    uint32_t count = 0;
    for (b3NodeBodyContact* c = h->body->m_contactManager.m_nodeBodyContactList.m_head; c; c = c->m_next, ++count) {
        if (count >= cap) continue;
        node[count] = c->m_n1->m_vertex;
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

void ref_softbody_set_type(void* p, uint32_t i, int type)
{
    static_cast<RefSoftBody*>(p)->body->GetVertexNode(i)->SetType((b3SoftBodyNodeType)type);
}

void ref_softbody_set_mass_damping(void* p, uint32_t i, float d)
{
    static_cast<RefSoftBody*>(p)->body->GetVertexNode(i)->SetMassDamping(d);
}

void ref_softbody_set_gravity(void* p, const float* g)
{
    static_cast<RefSoftBody*>(p)->body->SetGravity(b3Vec3(g[0], g[1], g[2]));
}

void ref_softbody_apply_force(void* p, uint32_t i, const float* f)
{
    static_cast<RefSoftBody*>(p)->body->GetVertexNode(i)->ApplyForce(b3Vec3(f[0], f[1], f[2]));
}

void ref_softbody_set_velocity(void* p, uint32_t i, const float* v)
{
    static_cast<RefSoftBody*>(p)->body->GetVertexNode(i)->SetVelocity(b3Vec3(v[0], v[1], v[2]));
}

void ref_softbody_step(void* p, float dt, uint32_t vel_iters, uint32_t pos_iters)
{
    static_cast<RefSoftBody*>(p)->body->Step(dt, vel_iters, pos_iters);
}

uint32_t ref_softbody_last_iterations() { return b3_softBodySolverIterations; }

void ref_softbody_get_state(void* p, float* x, float* v)
{
    RefSoftBody* h = static_cast<RefSoftBody*>(p);
    for (uint32_t i = 0; i < h->mesh.vertexCount; ++i) {
        const b3SoftBodyNode* n = h->body->GetVertexNode(i);
        if (x) {
            x[3 * i] = n->m_position.x;
            x[3 * i + 1] = n->m_position.y;
            x[3 * i + 2] = n->m_position.z;
        }
        if (v) {
            v[3 * i] = n->m_velocity.x;
            v[3 * i + 1] = n->m_velocity.y;
            v[3 * i + 2] = n->m_velocity.z;
        }
    }
}

void ref_softbody_get_masses(void* p, float* m)
{
    RefSoftBody* h = static_cast<RefSoftBody*>(p);
    for (uint32_t i = 0; i < h->mesh.vertexCount; ++i) m[i] = h->body->GetVertexNode(i)->m_mass;
}

// per element: q (4), plastic strain (6)
void ref_softbody_get_elements(void* p, float* q, float* eps)
{
    RefSoftBody* h = static_cast<RefSoftBody*>(p);
    for (uint32_t e = 0; e < h->mesh.tetrahedronCount; ++e) {
        const b3SoftBodyElement& el = h->body->m_elements[e];
        if (q) {
            q[4 * e] = el.q.x;
            q[4 * e + 1] = el.q.y;
            q[4 * e + 2] = el.q.z;
            q[4 * e + 3] = el.q.w;
        }
        if (eps) std::memcpy(eps + 6 * (size_t)e, el.epsilon_plastic, 6 * sizeof(float));
    }
}

// one element's K blocks (16 x 9, column-major b3Mat33), invE (9), B (72), P (72)
void ref_softbody_get_element_data(void* p, uint32_t e, float* K, float* invE, float* B, float* P)
{
    const b3SoftBodyElement& el = static_cast<RefSoftBody*>(p)->body->m_elements[e];
    if (K) std::memcpy(K, el.K, sizeof(el.K));
    if (invE) std::memcpy(invE, &el.invE, sizeof(b3Mat33));
    if (B) std::memcpy(B, el.B, sizeof(el.B));
    if (P) std::memcpy(P, el.P, sizeof(el.P));
}

float ref_softbody_energy(void* p) { return static_cast<RefSoftBody*>(p)->body->GetEnergy(); }

}  // extern "C"
