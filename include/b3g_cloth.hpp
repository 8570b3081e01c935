// C++ shim with the shape of Bounce's b3Cloth / b3Particle
// (include/bounce/cloth/cloth.h:99-158, include/bounce/cloth/particle.h:63-111)
// over the C ABI of libb3g.so.  Header-only; link with -lb3g.  Every method
// forwards to the GPU; errors surface as b3gError exceptions.
#ifndef B3G_CLOTH_HPP
#define B3G_CLOTH_HPP

#include <stdexcept>
#include <string>
#include <vector>

#include "b3g.h"

class b3gError : public std::runtime_error {
public:
    b3gError(b3g_status s, const char* what)
        : std::runtime_error(std::string(what) + ": " + b3g_status_string(s)), status(s) {}
    b3g_status status;
};

inline void b3gCheck(b3g_status s, const char* what)
{
    if (s != B3G_OK) throw b3gError(s, what);
}

class b3gCloth;

class b3gParticle {
public:
    b3gParticle(b3g_cloth* c, uint32_t v) : m_cloth(c), m_vertex(v) {}
    void SetType(b3g_particle_type t) { b3gCheck(b3g_particle_set_type(m_cloth, m_vertex, t), "SetType"); }
    b3g_particle_type GetType() const
    {
        b3g_particle_type t;
        b3gCheck(b3g_particle_get_type(m_cloth, m_vertex, &t), "GetType");
        return t;
    }
    uint32_t GetVertex() const { return m_vertex; }
    void SetPosition(const float p[3]) { b3gCheck(b3g_particle_set_position(m_cloth, m_vertex, p), "SetPosition"); }
    void GetPosition(float p[3]) const { b3gCheck(b3g_particle_get_position(m_cloth, m_vertex, p), "GetPosition"); }
    void SetVelocity(const float v[3]) { b3gCheck(b3g_particle_set_velocity(m_cloth, m_vertex, v), "SetVelocity"); }
    void GetVelocity(float v[3]) const { b3gCheck(b3g_particle_get_velocity(m_cloth, m_vertex, v), "GetVelocity"); }
    float GetMass() const
    {
        float m;
        b3gCheck(b3g_particle_get_mass(m_cloth, m_vertex, &m), "GetMass");
        return m;
    }
    void ApplyForce(const float f[3]) { b3gCheck(b3g_particle_apply_force(m_cloth, m_vertex, f), "ApplyForce"); }
    void ApplyTranslation(const float t[3])
    {
        b3gCheck(b3g_particle_apply_translation(m_cloth, m_vertex, t), "ApplyTranslation");
    }
    void SetRadius(float r) { b3gCheck(b3g_particle_set_radius(m_cloth, m_vertex, r), "SetRadius"); }
    float GetRadius() const
    {
        float r;
        b3gCheck(b3g_particle_get_radius(m_cloth, m_vertex, &r), "GetRadius");
        return r;
    }
    void SetFriction(float f) { b3gCheck(b3g_particle_set_friction(m_cloth, m_vertex, f), "SetFriction"); }
    float GetFriction() const
    {
        float f;
        b3gCheck(b3g_particle_get_friction(m_cloth, m_vertex, &f), "GetFriction");
        return f;
    }

private:
    b3g_cloth* m_cloth;
    uint32_t m_vertex;
};

class b3gCloth {
public:
    // b3Cloth(const b3ClothDef&): the mesh is copied to the device.
    b3gCloth(const b3g_mesh_desc& mesh, const b3g_cloth_def& def, int device = 0)
    {
        b3gCheck(b3g_cloth_create(&mesh, &def, device, &m_cloth), "b3gCloth");
    }
    ~b3gCloth() { b3g_cloth_destroy(m_cloth); }
    b3gCloth(const b3gCloth&) = delete;
    b3gCloth& operator=(const b3gCloth&) = delete;

    void SetGravity(const float g[3]) { b3gCheck(b3g_cloth_set_gravity(m_cloth, g), "SetGravity"); }
    void GetGravity(float g[3]) const { b3gCheck(b3g_cloth_get_gravity(m_cloth, g), "GetGravity"); }
    // SetWorld(world) with one static sphere body, as a collider list
    uint32_t AddStaticSphere(const float c[3], float radius, float friction)
    {
        uint32_t id;
        b3gCheck(b3g_cloth_add_static_sphere(m_cloth, c, radius, friction, &id), "AddStaticSphere");
        return id;
    }
    // a static capsule body: segment a-b (world frame), radius
    uint32_t AddStaticCapsule(const float a[3], const float b[3], float radius, float friction)
    {
        uint32_t id;
        b3gCheck(b3g_cloth_add_static_capsule(m_cloth, a, b, radius, friction, &id), "AddStaticCapsule");
        return id;
    }
    void ClearColliders() { b3gCheck(b3g_cloth_clear_colliders(m_cloth), "ClearColliders"); }
    // SetWorld(world) with moving bodies: the cloth's copy of a b3Body, the
    // shapes on it (body frame), and the state exchange around each Step
    uint32_t AddBody(const b3g_body_state& b)
    {
        uint32_t id;
        b3gCheck(b3g_cloth_add_body(m_cloth, &b, &id), "AddBody");
        return id;
    }
    void SetBody(uint32_t id, const b3g_body_state& b) { b3gCheck(b3g_cloth_set_body(m_cloth, id, &b), "SetBody"); }
    b3g_body_state GetBody(uint32_t id) const
    {
        b3g_body_state b;
        b3gCheck(b3g_cloth_get_body(m_cloth, id, &b), "GetBody");
        return b;
    }
    uint32_t AddBodySphere(uint32_t body, const float c[3], float radius, float friction)
    {
        uint32_t id;
        b3gCheck(b3g_cloth_add_body_sphere(m_cloth, body, c, radius, friction, &id), "AddBodySphere");
        return id;
    }
    uint32_t AddBodyCapsule(uint32_t body, const float a[3], const float b[3], float radius, float friction)
    {
        uint32_t id;
        b3gCheck(b3g_cloth_add_body_capsule(m_cloth, body, a, b, radius, friction, &id), "AddBodyCapsule");
        return id;
    }
    uint32_t AddBodyHull(uint32_t body, const float* vertices, uint32_t vertexCount, const float* planes,
                         uint32_t faceCount, float friction)
    {
        uint32_t id;
        b3gCheck(b3g_cloth_add_body_hull(m_cloth, body, vertices, vertexCount, planes, faceCount, friction, &id),
                 "AddBodyHull");
        return id;
    }
    void SetShapeProxy(uint32_t shape, const float lo[3], const float hi[3])
    {
        b3gCheck(b3g_cloth_set_shape_proxy(m_cloth, shape, lo, hi), "SetShapeProxy");
    }
    void GetShapeProxy(uint32_t shape, float lo[3], float hi[3]) const
    {
        b3gCheck(b3g_cloth_get_shape_proxy(m_cloth, shape, lo, hi), "GetShapeProxy");
    }
    void SetReportOrder(const uint32_t* order, uint32_t count)
    {
        b3gCheck(b3g_cloth_set_report_order(m_cloth, order, count), "SetReportOrder");
    }
    void SetSolver(const b3g_solver_opts& o) { b3gCheck(b3g_cloth_set_solver(m_cloth, &o), "SetSolver"); }
    b3gParticle GetParticle(uint32_t i) { return b3gParticle(m_cloth, i); }
    // b3Cloth::CreateParticle / DestroyParticle (cloth.cpp:307-351): a particle
    // outside the mesh, addressed after the mesh vertices.
    b3gParticle CreateParticle(const b3g_particle_def& def)
    {
        uint32_t i;
        b3gCheck(b3g_cloth_create_particle(m_cloth, &def, &i), "CreateParticle");
        return b3gParticle(m_cloth, i);
    }
    void DestroyParticle(const b3gParticle& p)
    {
        b3gCheck(b3g_cloth_destroy_particle(m_cloth, p.GetVertex()), "DestroyParticle");
    }
    // b3Cloth::CreateForce of a b3MouseForceDef, and DestroyForce (cloth.cpp:353-364)
    uint32_t CreateMouseForce(const b3g_mouse_force_def& def)
    {
        uint32_t id;
        b3gCheck(b3g_cloth_create_mouse_force(m_cloth, &def, &id), "CreateForce");
        return id;
    }
    void DestroyForce(uint32_t id) { b3gCheck(b3g_cloth_destroy_force(m_cloth, id), "DestroyForce"); }
    float GetEnergy() const
    {
        float e;
        b3gCheck(b3g_cloth_get_energy(m_cloth, &e), "GetEnergy");
        return e;
    }
    b3g_step_stats Step(float dt, uint32_t velocityIterations, uint32_t positionIterations)
    {
        b3g_step_stats s;
        b3gCheck(b3g_cloth_step(m_cloth, dt, velocityIterations, positionIterations, &s), "Step");
        return s;
    }
    uint32_t GetVertexCount() const { return b3g_cloth_vertex_count(m_cloth); }
    void ReadPositions(float* xyz) const { b3gCheck(b3g_cloth_read_state(m_cloth, xyz, nullptr, nullptr), "ReadPositions"); }
    void ReadVelocities(float* xyz) const
    {
        b3gCheck(b3g_cloth_read_state(m_cloth, nullptr, xyz, nullptr), "ReadVelocities");
    }
    b3g_cloth* Handle() { return m_cloth; }

private:
    b3g_cloth* m_cloth = nullptr;
};

#endif
