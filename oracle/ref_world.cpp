// Test infrastructure, not product code: reference worlds (ReactPhysics3D
// v0.10.2, built from its own sources by oracle/Makefile) stepped by the
// reference itself, with the dynamics stage of one step captured.
//
// ref_world_create builds a seeded scene (a jittered grid of boxes, spheres
// and capsules with random sizes, orientations, materials, dampings, lock
// factors, external forces and a few kinematic / gravity-free bodies above a
// static ground box).  ref_world_step runs PhysicsWorld::update.
// ref_world_capture runs one step by calling the phases of
// PhysicsWorld::update (src/engine/PhysicsWorld.cpp:239-307) in the same order
// and records, between createContacts/reportContacts and the end of
// updateBodiesState, every input and output of the dynamics stage: the
// enabled rigid-body and collider components, the contact manifolds and
// points in the contact solver's order (islands in order, each island's
// manifold range in order), the islands as manifold ranges, and the world
// settings.  Private members are reached because this translation unit is
// compiled with -fno-access-control (oracle/Makefile), which lifts access
// checks without changing any class layout; the reference objects are
// compiled unchanged.
#include <algorithm>
#include <array>
#include <atomic>
#include <cassert>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>
#include <reactphysics3d/reactphysics3d.h>

#include "../include/rp3dg.h"

using namespace reactphysics3d;

namespace {

struct Capture {
    std::map<std::string, std::vector<uint8_t>> f;
    template <class T>
    void put(const std::string& name, const std::vector<T>& v) {
        std::vector<uint8_t> b(v.size() * sizeof(T));
        if (!v.empty()) std::memcpy(b.data(), v.data(), b.size());
        f[name] = std::move(b);
    }
};

// The contact events of the last update (EventListener::onContact), in the
// rp3dg_contact_event layout: body and collider creation indices, event type,
// first point and point count, and the points (normal + depth, local points).
struct EventRecorder : public EventListener {
    const std::vector<RigidBody*>* bodies = nullptr;
    const std::vector<Collider*>* colliders = nullptr;
    std::vector<rp3dg_contact_event> events;
    std::vector<rp3dg_contact_event> triggers;   // EventListener::onTrigger, no points
    std::vector<float> nd, l1, l2;
    void clear() { events.clear(); triggers.clear(); nd.clear(); l1.clear(); l2.clear(); }
    void onTrigger(const OverlapCallback::CallbackData& data) override {
        std::unordered_map<const void*, int32_t> bi, ci;
        for (size_t i = 0; i < bodies->size(); i++) bi[static_cast<const void*>(static_cast<Body*>((*bodies)[i]))] = int32_t(i);
        for (size_t i = 0; i < colliders->size(); i++) ci[static_cast<const void*>((*colliders)[i])] = int32_t(i);
        for (uint32 k = 0; k < data.getNbOverlappingPairs(); k++) {
            const OverlapCallback::OverlapPair pair = data.getOverlappingPair(k);
            rp3dg_contact_event ev{};
            ev.body1 = bi.at(static_cast<const void*>(pair.getBody1()));
            ev.body2 = bi.at(static_cast<const void*>(pair.getBody2()));
            ev.collider1 = ci.at(static_cast<const void*>(pair.getCollider1()));
            ev.collider2 = ci.at(static_cast<const void*>(pair.getCollider2()));
            const auto t = pair.getEventType();
            ev.type = t == OverlapCallback::OverlapPair::EventType::OverlapStart ? 0
                    : (t == OverlapCallback::OverlapPair::EventType::OverlapStay ? 1 : 2);
            triggers.push_back(ev);
        }
    }
    void onContact(const CollisionCallback::CallbackData& data) override {
        std::unordered_map<const void*, int32_t> bi, ci;
        for (size_t i = 0; i < bodies->size(); i++) bi[static_cast<const void*>(static_cast<Body*>((*bodies)[i]))] = int32_t(i);
        for (size_t i = 0; i < colliders->size(); i++) ci[static_cast<const void*>((*colliders)[i])] = int32_t(i);
        for (uint32 k = 0; k < data.getNbContactPairs(); k++) {
            const CollisionCallback::ContactPair pair = data.getContactPair(k);
            rp3dg_contact_event ev{};
            ev.body1 = bi.at(static_cast<const void*>(pair.getBody1()));
            ev.body2 = bi.at(static_cast<const void*>(pair.getBody2()));
            ev.collider1 = ci.at(static_cast<const void*>(pair.getCollider1()));
            ev.collider2 = ci.at(static_cast<const void*>(pair.getCollider2()));
            const auto t = pair.getEventType();
            ev.type = t == CollisionCallback::ContactPair::EventType::ContactStart ? 0
                    : (t == CollisionCallback::ContactPair::EventType::ContactStay ? 1 : 2);
            ev.first_point = uint32_t(nd.size() / 4);
            ev.nb_points = pair.getNbContactPoints();
            for (uint32 c = 0; c < pair.getNbContactPoints(); c++) {
                const CollisionCallback::ContactPoint cp = pair.getContactPoint(c);
                const Vector3 n = cp.getWorldNormal(), a = cp.getLocalPointOnCollider1(), b = cp.getLocalPointOnCollider2();
                const float v[12] = {float(n.x), float(n.y), float(n.z), float(cp.getPenetrationDepth()),
                                     float(a.x), float(a.y), float(a.z), 0.0f, float(b.x), float(b.y), float(b.z), 0.0f};
                nd.insert(nd.end(), v, v + 4);
                l1.insert(l1.end(), v + 4, v + 8);
                l2.insert(l2.end(), v + 8, v + 12);
            }
            events.push_back(ev);
        }
    }
};

struct World {
    PhysicsCommon common;
    PhysicsWorld* world = nullptr;
    std::vector<RigidBody*> bodies;
    std::vector<Joint*> joints;  // in creation order
    std::vector<Collider*> colliders;  // in creation order
    EventRecorder recorder;
    Capture cap;
};

std::vector<std::unique_ptr<World>>& worlds() {
    static std::vector<std::unique_ptr<World>> w;
    return w;
}

void f4(std::vector<float>& out, const Vector3& v, float w = 0.0f) {
    out.push_back(float(v.x)); out.push_back(float(v.y)); out.push_back(float(v.z)); out.push_back(w);
}
void q4(std::vector<float>& out, const Quaternion& q) {
    out.push_back(float(q.x)); out.push_back(float(q.y)); out.push_back(float(q.z)); out.push_back(float(q.w));
}

// Uniform unit quaternion (Shoemake).
Quaternion random_rotation(std::mt19937_64& rng) {
    std::uniform_real_distribution<double> u(0.0, 1.0);
    const double u1 = u(rng), u2 = u(rng), u3 = u(rng);
    const double a = std::sqrt(1.0 - u1), b = std::sqrt(u1);
    const double t1 = 2.0 * 3.14159265358979323846 * u2, t2 = 2.0 * 3.14159265358979323846 * u3;
    Quaternion q(decimal(a * std::sin(t1)), decimal(a * std::cos(t1)), decimal(b * std::sin(t2)), decimal(b * std::cos(t2)));
    q.normalize();
    return q;
}

// Bodies and colliders of the enabled component ranges, as the dynamics
// stage sees them.
void capture_state(World& W, const std::string& pre, bool inputs) {
    PhysicsWorld& w = *W.world;
    RigidBodyComponents& rb = w.mRigidBodyComponents;
    ColliderComponents& cc = w.mCollidersComponents;
    TransformComponents& tc = w.mTransformComponents;
    // every component: the solver also reads bodies outside the enabled range
    // (static bodies are never enabled), through their constrained
    // velocities and world inverse inertia
    const uint32 nb = rb.getNbComponents();
    std::vector<float> pos, ori, comw, coml, lv, av, force, torque, iil, mass, llock, alock, iiw, clv, cav, sv;
    std::vector<uint8_t> grav;
    for (uint32 i = 0; i < nb; i++) {
        const Transform& t = tc.getTransform(rb.mBodiesEntities[i]);
        f4(pos, t.getPosition());
        q4(ori, t.getOrientation());
        f4(comw, rb.mCentersOfMassWorld[i]);
        f4(lv, rb.mLinearVelocities[i]);
        f4(av, rb.mAngularVelocities[i]);
        if (inputs) {
            f4(coml, rb.mCentersOfMassLocal[i]);
            f4(force, rb.mExternalForces[i]);
            f4(torque, rb.mExternalTorques[i]);
            f4(iil, rb.mInverseInertiaTensorsLocal[i]);
            mass.push_back(float(rb.mMasses[i])); mass.push_back(float(rb.mInverseMasses[i]));
            mass.push_back(float(rb.mLinearDampings[i])); mass.push_back(float(rb.mAngularDampings[i]));
            f4(llock, rb.mLinearLockAxisFactors[i]);
            f4(alock, rb.mAngularLockAxisFactors[i]);
            grav.push_back(rb.mIsGravityEnabled[i] ? 1 : 0);
            f4(clv, rb.mConstrainedLinearVelocities[i]);
            f4(cav, rb.mConstrainedAngularVelocities[i]);
            f4(sv, rb.mSplitLinearVelocities[i]);
            f4(sv, rb.mSplitAngularVelocities[i]);
            const Matrix3x3& m = rb.mInverseInertiaTensorsWorld[i];
            for (int r = 0; r < 3; r++) f4(iiw, m[r]);
        } else {
            const Matrix3x3& m = rb.mInverseInertiaTensorsWorld[i];
            for (int r = 0; r < 3; r++) f4(iiw, m[r]);
        }
    }
    W.cap.put(pre + "body_position", pos);
    W.cap.put(pre + "body_orientation", ori);
    W.cap.put(pre + "body_com_world", comw);
    W.cap.put(pre + "body_linear_velocity", lv);
    W.cap.put(pre + "body_angular_velocity", av);
    if (inputs) {
        W.cap.put(pre + "body_com_local", coml);
        W.cap.put(pre + "body_force", force);
        W.cap.put(pre + "body_torque", torque);
        W.cap.put(pre + "body_inv_inertia_local", iil);
        W.cap.put(pre + "body_mass", mass);
        W.cap.put(pre + "body_linear_lock", llock);
        W.cap.put(pre + "body_angular_lock", alock);
        W.cap.put(pre + "body_gravity", grav);
        W.cap.put(pre + "body_constrained_linear_velocity", clv);
        W.cap.put(pre + "body_constrained_angular_velocity", cav);
        W.cap.put(pre + "body_split_velocity", sv);
        W.cap.put(pre + "body_inv_inertia_world", iiw);
        std::vector<uint32_t> ne = {rb.getNbEnabledComponents()};
        W.cap.put(pre + "body_nb_enabled", ne);
    } else {
        W.cap.put(pre + "body_inv_inertia_world", iiw);
    }
    const uint32 nc = cc.getNbComponents();
    std::vector<int32_t> cbody;
    std::vector<float> clp, clo, cwp, cwo, cmat;
    for (uint32 i = 0; i < nc; i++) {
        const Transform& lw = cc.mLocalToWorldTransforms[i];
        f4(cwp, lw.getPosition());
        q4(cwo, lw.getOrientation());
        if (inputs) {
            cbody.push_back(int32_t(rb.getEntityIndex(cc.mBodiesEntities[i])));
            const Transform& lb = cc.mLocalToBodyTransforms[i];
            f4(clp, lb.getPosition());
            q4(clo, lb.getOrientation());
            const Material& m = cc.mMaterials[i];
            cmat.push_back(float(m.getFrictionCoefficientSqrt()));
            cmat.push_back(float(m.getBounciness()));
            cmat.push_back(0.0f); cmat.push_back(0.0f);
        }
    }
    W.cap.put(pre + "collider_world_position", cwp);
    W.cap.put(pre + "collider_world_orientation", cwo);
    if (inputs) {
        W.cap.put(pre + "collider_body", cbody);
        W.cap.put(pre + "collider_local_position", clp);
        W.cap.put(pre + "collider_local_orientation", clo);
        W.cap.put(pre + "collider_material", cmat);
        std::vector<uint32_t> ne = {cc.getNbEnabledComponents()};
        W.cap.put(pre + "collider_nb_enabled", ne);
    }
}

// Manifolds in the solver's order: islands in order, each island's range.
std::vector<uint32_t> solver_order(World& W) {
    Islands& isl = W.world->mIslands;
    std::vector<uint32_t> order;
    for (uint32 i = 0; i < isl.getNbIslands(); i++)
        for (uint32 m = isl.contactManifoldsIndices[i]; m < isl.contactManifoldsIndices[i] + isl.nbContactManifolds[i]; m++)
            order.push_back(m);
    return order;
}

void capture_contacts(World& W, const std::string& pre, const std::vector<uint32_t>& order, bool inputs) {
    PhysicsWorld& w = *W.world;
    Array<ContactManifold>& mans = *w.mCollisionDetection.mCurrentContactManifolds;
    Array<ContactPoint>& pts = *w.mCollisionDetection.mCurrentContactPoints;
    RigidBodyComponents& rb = w.mRigidBodyComponents;
    ColliderComponents& cc = w.mCollidersComponents;
    std::vector<int32_t> ids;
    std::vector<uint32_t> pstart, src;
    std::vector<uint8_t> npts, resting;
    std::vector<float> fv1, fv2, fimp, nd, l1, l2, pimp;
    for (uint32_t k = 0; k < order.size(); k++) {
        const ContactManifold& m = mans[order[k]];
        src.push_back(order[k]);
        ids.push_back(int32_t(rb.getEntityIndex(m.bodyEntity1)));
        ids.push_back(int32_t(rb.getEntityIndex(m.bodyEntity2)));
        ids.push_back(int32_t(cc.getEntityIndex(m.colliderEntity1)));
        ids.push_back(int32_t(cc.getEntityIndex(m.colliderEntity2)));
        pstart.push_back(uint32_t(pimp.size()));
        npts.push_back(m.nbContactPoints);
        f4(fv1, m.frictionVector1);
        f4(fv2, m.frictionVector2);
        fimp.push_back(float(m.frictionImpulse1)); fimp.push_back(float(m.frictionImpulse2));
        fimp.push_back(float(m.frictionTwistImpulse)); fimp.push_back(0.0f);
        for (uint32 c = m.contactPointsIndex; c < m.contactPointsIndex + m.nbContactPoints; c++) {
            const ContactPoint& p = pts[c];
            f4(nd, p.getNormal(), float(p.getPenetrationDepth()));
            f4(l1, p.getLocalPointOnShape1());
            f4(l2, p.getLocalPointOnShape2());
            pimp.push_back(float(p.getPenetrationImpulse()));
            resting.push_back(p.getIsRestingContact() ? 1 : 0);
        }
    }
    W.cap.put(pre + "manifold_friction_vector1", fv1);
    W.cap.put(pre + "manifold_friction_vector2", fv2);
    W.cap.put(pre + "manifold_friction_impulse", fimp);
    W.cap.put(pre + "point_penetration_impulse", pimp);
    W.cap.put(pre + "point_is_resting", resting);
    if (inputs) {
        W.cap.put(pre + "manifold_ids", ids);
        W.cap.put(pre + "manifold_point_start", pstart);
        W.cap.put(pre + "manifold_nb_points", npts);
        W.cap.put(pre + "manifold_source", src);
        W.cap.put(pre + "point_normal_depth", nd);
        W.cap.put(pre + "point_local1", l1);
        W.cap.put(pre + "point_local2", l2);
        Islands& isl = w.mIslands;
        std::vector<uint32_t> is, in;
        uint32_t at = 0;
        for (uint32 i = 0; i < isl.getNbIslands(); i++) {
            is.push_back(at);
            in.push_back(isl.nbContactManifolds[i]);
            at += isl.nbContactManifolds[i];
        }
        W.cap.put(pre + "island_manifold_start", is);
        W.cap.put(pre + "island_manifold_count", in);
    }
}

// Fat AABB of every collider component (zeros for colliders outside the
// broad phase), by collider index.
void capture_fat(World& W, const std::string& pre) {
    PhysicsWorld& w = *W.world;
    ColliderComponents& cc = w.mCollidersComponents;
    const DynamicAABBTree& tree = w.mCollisionDetection.mBroadPhaseSystem.mDynamicAABBTree;
    std::vector<float> mn, mx;
    for (uint32 i = 0; i < cc.getNbComponents(); i++) {
        const int32 id = cc.mBroadPhaseIds[i];
        if (id >= 0) {
            const AABB& a = tree.getFatAABB(id);
            f4(mn, a.getMin()); f4(mx, a.getMax());
        } else {
            f4(mn, Vector3(0, 0, 0)); f4(mx, Vector3(0, 0, 0));
        }
    }
    W.cap.put(pre + "fat_min", mn);
    W.cap.put(pre + "fat_max", mx);
}

// Static broad-phase data of the colliders: shape (kind as in rp3dg.h: 0
// sphere, 1 capsule, 2 box; params), local bounds, filter bits, broad-phase id.
void capture_bp_static(World& W) {
    PhysicsWorld& w = *W.world;
    ColliderComponents& cc = w.mCollidersComponents;
    std::vector<float> shape, lmin, lmax;
    std::vector<int32_t> bits, bpid;
    for (uint32 i = 0; i < cc.getNbComponents(); i++) {
        const CollisionShape* cs = cc.mCollisionShapes[i];
        float kind = -1, p0 = 0, p1 = 0, p2 = 0;
        switch (cs->getName()) {
            case CollisionShapeName::SPHERE: kind = 0; p0 = float(static_cast<const SphereShape*>(cs)->getRadius()); break;
            case CollisionShapeName::CAPSULE:
                kind = 1; p0 = float(static_cast<const CapsuleShape*>(cs)->getRadius());
                p1 = float(static_cast<const CapsuleShape*>(cs)->mHalfHeight); break;
            case CollisionShapeName::BOX: {
                kind = 2; const Vector3 h = static_cast<const BoxShape*>(cs)->getHalfExtents();
                p0 = float(h.x); p1 = float(h.y); p2 = float(h.z); break;
            }
            default: break;
        }
        shape.push_back(p0); shape.push_back(p1); shape.push_back(p2); shape.push_back(kind);
        const AABB lb = cs->getLocalBounds();
        f4(lmin, lb.getMin()); f4(lmax, lb.getMax());
        bits.push_back(int32_t(cc.mCollisionCategoryBits[i]));
        bits.push_back(int32_t(cc.mCollideWithMaskBits[i]));
        bpid.push_back(cc.mBroadPhaseIds[i]);
    }
    W.cap.put("bp_shape", shape);
    W.cap.put("bp_local_min", lmin);
    W.cap.put("bp_local_max", lmax);
    W.cap.put("bp_bits", bits);
    W.cap.put("bp_id", bpid);
}

// Every overlapping pair (enabled and disabled arrays) as (lower, higher)
// collider index.
void capture_pairs(World& W, const std::string& name) {
    PhysicsWorld& w = *W.world;
    ColliderComponents& cc = w.mCollidersComponents;
    OverlappingPairs& op = w.mCollisionDetection.mOverlappingPairs;
    std::vector<int32_t> out;
    auto add = [&](const OverlappingPairs::OverlappingPair& p) {
        const int32_t a = int32_t(cc.getEntityIndex(p.collider1)), b = int32_t(cc.getEntityIndex(p.collider2));
        out.push_back(a < b ? a : b);
        out.push_back(a < b ? b : a);
    };
    for (uint32 i = 0; i < op.mConvexPairs.size(); i++) add(op.mConvexPairs[i]);
    for (uint32 i = 0; i < op.mDisabledConvexPairs.size(); i++) add(op.mDisabledConvexPairs[i]);
    W.cap.put(name, out);
}

}  // namespace

extern "C" {

// kind 0: boxes only; 1: boxes, spheres and capsules.  variety bit 0: random
// materials, dampings, locks, kinematic bodies...; bit 1: collision filters.
// Returns a world id.
int ref_world_create(int kind, uint64_t seed, int nx, int ny, int nz, float spacing, int variety) {
    auto W = std::make_unique<World>();
    PhysicsWorld::WorldSettings s;
    W->world = W->common.createPhysicsWorld(s);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    auto U = [&](double a, double b) { return decimal(a + (b - a) * u(rng)); };
    // static ground box 50 x 0.5 x 50 (half-extents 25, 0.25, 25) with its top at y = 0
    RigidBody* ground = W->world->createRigidBody(Transform(Vector3(0, decimal(-0.25), 0), Quaternion::identity()));
    ground->setType(BodyType::STATIC);
    Collider* gc = ground->addCollider(W->common.createBoxShape(Vector3(25, decimal(0.25), 25)), Transform::identity());
    if (variety & 1) gc->getMaterial().setFrictionCoefficient(decimal(0.6));
    W->bodies.push_back(ground);
    int count = 0;
    for (int iy = 0; iy < ny; iy++)
        for (int ix = 0; ix < nx; ix++)
            for (int iz = 0; iz < nz; iz++) {
                const Vector3 p(decimal((ix - 0.5 * (nx - 1)) * spacing) + U(-0.1, 0.1),
                                decimal(1.0 + iy * spacing) + U(-0.1, 0.1),
                                decimal((iz - 0.5 * (nz - 1)) * spacing) + U(-0.1, 0.1));
                RigidBody* b = W->world->createRigidBody(Transform(p, random_rotation(rng)));
                const int shape = kind == 0 ? 0 : int(u(rng) * 3.0);
                CollisionShape* cs;
                if (shape == 0) cs = W->common.createBoxShape(Vector3(U(0.25, 0.75), U(0.25, 0.75), U(0.25, 0.75)));
                else if (shape == 1) cs = W->common.createSphereShape(U(0.2, 0.5));
                else cs = W->common.createCapsuleShape(decimal(0.2), decimal(0.6));
                Collider* c = b->addCollider(cs, Transform::identity());
                if (variety & 1) {
                    c->getMaterial().setFrictionCoefficient(U(0.1, 1.0));
                    c->getMaterial().setBounciness(U(0.0, 0.6));
                }
                b->updateMassPropertiesFromColliders();
                if (variety & 1) {
                    const int k = count % 23;
                    if (k == 3) b->setLinearDamping(U(0.0, 0.5));
                    if (k == 4) b->setAngularDamping(U(0.0, 0.5));
                    if (k == 5) b->setLinearLockAxisFactor(Vector3(1, 0, 1));
                    if (k == 6) b->setAngularLockAxisFactor(Vector3(0, 1, 0));
                    if (k == 7) b->enableGravity(false);
                    if (k == 8) b->setLinearVelocity(Vector3(U(-2, 2), U(-2, 0), U(-2, 2)));
                    if (k == 9) b->setAngularVelocity(Vector3(U(-3, 3), U(-3, 3), U(-3, 3)));
                    if (k == 10) {
                        b->setType(BodyType::KINEMATIC);
                        b->setLinearVelocity(Vector3(U(-0.5, 0.5), 0, U(-0.5, 0.5)));
                    }
                }
                if (variety & 2) {
                    // collision filtering: categories 1, 2, 4; every 3rd collider ignores category 2
                    c->setCollisionCategoryBits((unsigned short)(1u << (count % 3)));
                    if (count % 3 == 0) c->setCollideWithMaskBits((unsigned short)(0xffffu & ~2u));
                }
                W->bodies.push_back(b);
                count++;
            }
    worlds().push_back(std::move(W));
    return int(worlds().size()) - 1;
}

// External forces/torques on every 5th dynamic body (they are reset by each
// update, so they are applied right before a step).
int ref_world_apply_forces(int id, uint64_t seed) {
    World& W = *worlds().at(size_t(id));
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    for (size_t i = 1; i < W.bodies.size(); i += 5) {
        RigidBody* b = W.bodies[i];
        if (b->getType() != BodyType::DYNAMIC) continue;
        b->applyWorldForceAtCenterOfMass(Vector3(decimal(20 * u(rng)), decimal(20 * u(rng)), decimal(20 * u(rng))));
        b->applyLocalTorque(Vector3(decimal(5 * u(rng)), decimal(5 * u(rng)), decimal(5 * u(rng))));
    }
    return 0;
}

int ref_world_step(int id, float dt, int nsteps) {
    World& W = *worlds().at(size_t(id));
    for (int i = 0; i < nsteps; i++) {
        W.recorder.clear();
        W.world->update(decimal(dt));
    }
    return 0;
}

// The trigger events of the last update (EventListener::onTrigger).
int ref_scene_trigger_events(int id, rp3dg_contact_event* events, uint32_t cap, uint32_t* nb_events) {
    World& W = *worlds().at(size_t(id));
    const EventRecorder& R = W.recorder;
    *nb_events = uint32_t(R.triggers.size());
    for (size_t k = 0; k < R.triggers.size() && k < cap; k++) events[k] = R.triggers[k];
    return 0;
}

// The contact events of the last update (counts always written).
int ref_scene_events(int id, rp3dg_contact_event* events, uint32_t cap, float* nd, float* l1, float* l2,
                     uint32_t cap_points, uint32_t* nb_events, uint32_t* nb_points) {
    World& W = *worlds().at(size_t(id));
    const EventRecorder& R = W.recorder;
    *nb_events = uint32_t(R.events.size());
    *nb_points = uint32_t(R.nd.size() / 4);
    for (size_t k = 0; k < R.events.size() && k < cap; k++) events[k] = R.events[k];
    const size_t np = std::min<size_t>(R.nd.size() / 4, cap_points);
    if (nd) std::memcpy(nd, R.nd.data(), np * 16);
    if (l1) std::memcpy(l1, R.l1.data(), np * 16);
    if (l2) std::memcpy(l2, R.l2.data(), np * 16);
    return 0;
}

// One step, phase by phase in the order of PhysicsWorld::update, recording
// the dynamics stage's inputs ("in_") and outputs ("out_").
int ref_world_capture(int id, float dt) {
    World& W = *worlds().at(size_t(id));
    PhysicsWorld& w = *W.world;
    W.cap.f.clear();
    const decimal timeStep = decimal(dt);
    capture_bp_static(W);
    capture_fat(W, "bp_start_");
    w.mCollisionDetection.computeCollisionDetection();
    capture_pairs(W, "bp_pairs");
    w.createIslands();
    w.mCollisionDetection.createContacts();
    w.mCollisionDetection.reportContactsAndTriggers();

    const std::vector<uint32_t> order = solver_order(W);
    capture_state(W, "in_", true);
    capture_contacts(W, "in_", order, true);
    std::vector<float> params = {float(timeStep), float(w.mConfig.gravity.x), float(w.mConfig.gravity.y),
                                 float(w.mConfig.gravity.z), w.mIsGravityEnabled ? 1.0f : 0.0f,
                                 float(w.mNbVelocitySolverIterations), w.mContactSolverSystem.isSplitImpulseActive() ? 1.0f : 0.0f,
                                 float(w.mContactSolverSystem.mRestitutionVelocityThreshold)};
    W.cap.put("params", params);

    // the dynamics stage, timed (the CPU figure of the same stage on the GPU)
    const auto t_dyn = std::chrono::steady_clock::now();
    w.updateBodiesInverseWorldInertiaTensors();
    w.enableDisableJoints();
    w.mDynamicsSystem.integrateRigidBodiesVelocities(timeStep);
    w.solveContactsAndConstraints(timeStep);
    w.mDynamicsSystem.integrateRigidBodiesPositions(timeStep, w.mContactSolverSystem.isSplitImpulseActive());
    w.solvePositionCorrection();
    w.mDynamicsSystem.updateBodiesState();
    W.cap.put("dyn_seconds",
              std::vector<double>{std::chrono::duration<double>(std::chrono::steady_clock::now() - t_dyn).count()});

    capture_state(W, "out_", false);
    capture_contacts(W, "out_", order, false);

    capture_fat(W, "bp_in_");
    w.mCollisionDetection.updateColliders();
    capture_fat(W, "bp_out_");
    {
        // colliders reinserted by this update (BroadPhaseSystem::mMovedShapes)
        ColliderComponents& cc = w.mCollidersComponents;
        std::vector<uint8_t> moved(cc.getNbComponents(), 0);
        const Set<int>& ms = w.mCollisionDetection.mBroadPhaseSystem.mMovedShapes;
        for (uint32 i = 0; i < cc.getNbComponents(); i++)
            if (cc.mBroadPhaseIds[i] >= 0 && ms.contains(cc.mBroadPhaseIds[i])) moved[i] = 1;
        W.cap.put("bp_moved", moved);
    }
    if (w.mIsSleepingEnabled) w.updateSleepingBodies(timeStep);
    w.mDynamicsSystem.resetBodiesForceAndTorque();
    w.mIslands.clear();
    w.mProcessContactPairsOrderIslands.clear(true);
    w.mMemoryManager.resetFrameAllocator();
    return 0;
}

// Size in bytes of a captured field (-1 if absent) and a copy of it.
long ref_world_field_size(int id, const char* name) {
    World& W = *worlds().at(size_t(id));
    auto it = W.cap.f.find(name);
    return it == W.cap.f.end() ? -1 : long(it->second.size());
}

int ref_world_field(int id, const char* name, void* dst) {
    World& W = *worlds().at(size_t(id));
    auto it = W.cap.f.find(name);
    if (it == W.cap.f.end()) return -1;
    if (!it->second.empty()) std::memcpy(dst, it->second.data(), it->second.size());
    return 0;
}

// Names of the captured fields, separated by spaces.
int ref_world_field_names(int id, char* dst, int cap) {
    World& W = *worlds().at(size_t(id));
    std::string s;
    for (auto& kv : W.cap.f) { s += kv.first; s += ' '; }
    if (int(s.size()) + 1 > cap) return -1;
    std::memcpy(dst, s.c_str(), s.size() + 1);
    return 0;
}

// ---- scenes described with the library's own world description -----------
// Height fields named by rp3dg_shape.mesh (kind RP3DG_SHAPE_HEIGHTFIELD):
// registered here with the arguments of rp3dg_create_heightfield, then built
// by ref_scene_create with PhysicsCommon::createHeightField (float heights)
// and createHeightFieldShape(scale).
struct HeightFieldSpec {
    int ncol, nrow;
    std::vector<float> heights;
    float scale[3];
};
static std::vector<HeightFieldSpec>& heightfields() {
    static std::vector<HeightFieldSpec> h;
    return h;
}
// Convex meshes for world scenes (shape kind RP3DG_SHAPE_CONVEX_MESH, the
// shape's mesh field naming the id returned here): ref_scene_create builds
// each with PhysicsCommon::createConvexMesh(PolygonVertexArray) and
// createConvexMeshShape(mesh, scale) in the world's PhysicsCommon.
struct ConvexSpec {
    std::vector<float> vertices;
    std::vector<uint32_t> indices;
    std::vector<PolygonVertexArray::PolygonFace> faces;
    float scale[3];
};
static std::vector<ConvexSpec>& convex_specs() {
    static std::vector<ConvexSpec> c;
    return c;
}
// A triangle mesh and its concave-mesh-shape scale, registered for
// ref_scene_create (rp3dg_shape.mesh names this id for RP3DG_SHAPE_CONCAVE_MESH).
struct ConcaveSpec {
    std::vector<float> vertices, normals;   // normals empty: computed by TriangleMesh::init
    std::vector<uint32_t> indices;
    float scale[3];
};
static std::vector<ConcaveSpec>& concave_specs() {
    static std::vector<ConcaveSpec> c;
    return c;
}
int ref_concave_register(const float* vertices, uint32_t nv, const uint32_t* indices, uint32_t nt,
                         const float* normals, float sx, float sy, float sz) {
    ConcaveSpec c;
    c.vertices.assign(vertices, vertices + 3 * size_t(nv));
    if (normals) c.normals.assign(normals, normals + 3 * size_t(nv));
    c.indices.assign(indices, indices + 3 * size_t(nt));
    c.scale[0] = sx; c.scale[1] = sy; c.scale[2] = sz;
    concave_specs().push_back(std::move(c));
    return int(concave_specs().size()) - 1;
}

// The TriangleMesh of a registered spec as the reference builds it: vertices,
// vertex normals, triangles (counts always written; -1 when it is invalid).
int ref_concave_mesh_data(int id, float* vertices, float* normals, uint32_t* triangles, uint32_t cap_v, uint32_t cap_t,
                          uint32_t* nv, uint32_t* nt) {
    ConcaveSpec& c = concave_specs().at(size_t(id));
    PhysicsCommon common;
    const uint32 n = uint32(c.vertices.size() / 3), m = uint32(c.indices.size() / 3);
    std::unique_ptr<TriangleVertexArray> tva;
    if (c.normals.empty())
        tva.reset(new TriangleVertexArray(n, c.vertices.data(), 3 * sizeof(float), m, c.indices.data(),
                                          3 * sizeof(uint32_t), TriangleVertexArray::VertexDataType::VERTEX_FLOAT_TYPE,
                                          TriangleVertexArray::IndexDataType::INDEX_INTEGER_TYPE));
    else
        tva.reset(new TriangleVertexArray(n, c.vertices.data(), 3 * sizeof(float), c.normals.data(), 3 * sizeof(float),
                                          m, c.indices.data(), 3 * sizeof(uint32_t),
                                          TriangleVertexArray::VertexDataType::VERTEX_FLOAT_TYPE,
                                          TriangleVertexArray::NormalDataType::NORMAL_FLOAT_TYPE,
                                          TriangleVertexArray::IndexDataType::INDEX_INTEGER_TYPE));
    std::vector<Message> messages;
    TriangleMesh* mesh = common.createTriangleMesh(*tva, messages);
    if (!mesh) return -1;
    *nv = mesh->getNbVertices();
    *nt = mesh->getNbTriangles();
    for (uint32_t v = 0; v < *nv && v < cap_v; v++) {
        const Vector3& p = mesh->getVertex(v);
        const Vector3& q = mesh->getVertexNormal(v);
        vertices[3 * v] = float(p.x); vertices[3 * v + 1] = float(p.y); vertices[3 * v + 2] = float(p.z);
        normals[3 * v] = float(q.x); normals[3 * v + 1] = float(q.y); normals[3 * v + 2] = float(q.z);
    }
    for (uint32_t t = 0; t < *nt && t < cap_t; t++) {
        uint32 a, b, d;
        mesh->getTriangleVerticesIndices(t, a, b, d);
        triangles[3 * t] = a; triangles[3 * t + 1] = b; triangles[3 * t + 2] = d;
    }
    return 0;
}

int ref_convex_register(const float* vertices, uint32_t nv, const uint32_t* face_indices, const uint32_t* face_sizes,
                        uint32_t nf, float sx, float sy, float sz) {
    ConvexSpec c;
    c.vertices.assign(vertices, vertices + 3 * size_t(nv));
    uint32_t total = 0;
    for (uint32_t f = 0; f < nf; f++) {
        PolygonVertexArray::PolygonFace pf;
        pf.nbVertices = face_sizes[f];
        pf.indexBase = total;
        c.faces.push_back(pf);
        total += face_sizes[f];
    }
    c.indices.assign(face_indices, face_indices + total);
    c.scale[0] = sx; c.scale[1] = sy; c.scale[2] = sz;
    convex_specs().push_back(std::move(c));
    return int(convex_specs().size()) - 1;
}

// ref_scene_create builds a reference world from the rp3dg_world_settings /
// rp3dg_body_desc / rp3dg_collider_desc arrays that rp3dg_world_create takes,
// with the call sequence documented there (include/rp3dg.h), so that both
// engines start from identical worlds.
int ref_heightfield_register(uint32_t ncol, uint32_t nrow, const float* heights, float sx, float sy, float sz) {
    HeightFieldSpec h;
    h.ncol = int(ncol);
    h.nrow = int(nrow);
    h.heights.assign(heights, heights + size_t(ncol) * nrow);
    h.scale[0] = sx; h.scale[1] = sy; h.scale[2] = sz;
    heightfields().push_back(h);
    return int(heightfields().size()) - 1;
}

// PhysicsWorld::setIsDebugRenderingEnabled(items != 0) and
// DebugRenderer::setIsDebugItemDisplayed for the six DebugItem bits.
int ref_scene_set_debug(int id, uint32_t items) {
    World& W = *worlds().at(size_t(id));
    W.world->setIsDebugRenderingEnabled(items != 0);
    DebugRenderer& r = W.world->getDebugRenderer();
    for (uint32_t bit = 1; bit <= 32; bit <<= 1)
        r.setIsDebugItemDisplayed(static_cast<DebugRenderer::DebugItem>(bit), (items & bit) != 0);
    return 0;
}

// Body::setIsDebugEnabled for one body (body >= 0) or all of them.
int ref_scene_set_body_debug(int id, int body, int enabled) {
    World& W = *worlds().at(size_t(id));
    for (size_t b = 0; b < W.bodies.size(); b++)
        if (body < 0 || size_t(body) == b) W.bodies[b]->setIsDebugEnabled(enabled != 0);
    return 0;
}

// DebugRenderer::getLinesArray / getTrianglesArray of the last update
// (counts always written), converted field by field to the C-ABI structs.
int ref_scene_debug_primitives(int id, rp3dg_debug_line* lines, uint32_t cap_lines, rp3dg_debug_triangle* tris,
                               uint32_t cap_tris, uint32_t* nb_lines, uint32_t* nb_tris) {
    World& W = *worlds().at(size_t(id));
    DebugRenderer& r = W.world->getDebugRenderer();
    *nb_lines = r.getNbLines();
    *nb_tris = r.getNbTriangles();
    auto put = [](float* o, const Vector3& v) { o[0] = float(v.x); o[1] = float(v.y); o[2] = float(v.z); };
    const DebugRenderer::DebugLine* L = r.getLinesArray();
    for (uint32_t k = 0; k < r.getNbLines() && k < cap_lines; k++) {
        put(lines[k].p1, L[k].point1); lines[k].color1 = L[k].color1;
        put(lines[k].p2, L[k].point2); lines[k].color2 = L[k].color2;
    }
    const DebugRenderer::DebugTriangle* T = r.getTrianglesArray();
    for (uint32_t k = 0; k < r.getNbTriangles() && k < cap_tris; k++) {
        put(tris[k].p1, T[k].point1); tris[k].color1 = T[k].color1;
        put(tris[k].p2, T[k].point2); tris[k].color2 = T[k].color2;
        put(tris[k].p3, T[k].point3); tris[k].color3 = T[k].color3;
    }
    return 0;
}

int ref_scene_create(const rp3dg_world_settings* s, const rp3dg_shape* shapes, uint32_t nshapes,
                     const rp3dg_body_desc* bd, uint32_t nb, const rp3dg_collider_desc* cd, uint32_t nc) {
    auto W = std::make_unique<World>();
    PhysicsWorld::WorldSettings ws;
    ws.gravity = Vector3(s->gravity[0], s->gravity[1], s->gravity[2]);
    ws.defaultVelocitySolverNbIterations = uint16(s->velocity_iterations);
    ws.isSleepingEnabled = s->sleeping_enabled != 0;
    ws.defaultSleepLinearVelocity = s->sleep_linear_velocity;
    ws.defaultSleepAngularVelocity = s->sleep_angular_velocity;
    ws.defaultTimeBeforeSleep = s->time_before_sleep;
    ws.restitutionVelocityThreshold = s->restitution_velocity_threshold;
    ws.persistentContactDistanceThreshold = s->persistent_contact_distance_threshold;
    ws.cosAngleSimilarContactManifold = s->cos_angle_similar_contact_manifold;
    ws.defaultPositionSolverNbIterations = uint16(s->position_iterations);
    W->world = W->common.createPhysicsWorld(ws);
    W->recorder.bodies = &W->bodies;
    W->recorder.colliders = &W->colliders;
    W->world->setEventListener(&W->recorder);
    std::vector<CollisionShape*> cs(nshapes, nullptr);
    for (uint32_t i = 0; i < nshapes; i++) {
        const rp3dg_shape& sh = shapes[i];
        if (sh.kind == RP3DG_SHAPE_SPHERE) cs[i] = W->common.createSphereShape(sh.params[0]);
        else if (sh.kind == RP3DG_SHAPE_CAPSULE) cs[i] = W->common.createCapsuleShape(sh.params[0], sh.params[1] * 2.0f);
        else if (sh.kind == RP3DG_SHAPE_BOX) cs[i] = W->common.createBoxShape(Vector3(sh.params[0], sh.params[1], sh.params[2]));
        else if (sh.kind == RP3DG_SHAPE_HEIGHTFIELD) {
            if (sh.mesh < 0 || size_t(sh.mesh) >= heightfields().size()) return -1;
            const HeightFieldSpec& h = heightfields()[size_t(sh.mesh)];
            std::vector<Message> messages;
            HeightField* hf = W->common.createHeightField(h.ncol, h.nrow, h.heights.data(),
                                                          HeightField::HeightDataType::HEIGHT_FLOAT_TYPE, messages);
            if (!hf) return -1;
            cs[i] = W->common.createHeightFieldShape(hf, Vector3(h.scale[0], h.scale[1], h.scale[2]));
        }
        else if (sh.kind == RP3DG_SHAPE_CONCAVE_MESH) {
            if (sh.mesh < 0 || size_t(sh.mesh) >= concave_specs().size()) return -1;
            ConcaveSpec& c = concave_specs()[size_t(sh.mesh)];
            const uint32 n = uint32(c.vertices.size() / 3), m = uint32(c.indices.size() / 3);
            std::unique_ptr<TriangleVertexArray> tva;
            if (c.normals.empty())
                tva.reset(new TriangleVertexArray(n, c.vertices.data(), 3 * sizeof(float), m, c.indices.data(),
                                                  3 * sizeof(uint32_t),
                                                  TriangleVertexArray::VertexDataType::VERTEX_FLOAT_TYPE,
                                                  TriangleVertexArray::IndexDataType::INDEX_INTEGER_TYPE));
            else
                tva.reset(new TriangleVertexArray(n, c.vertices.data(), 3 * sizeof(float), c.normals.data(),
                                                  3 * sizeof(float), m, c.indices.data(), 3 * sizeof(uint32_t),
                                                  TriangleVertexArray::VertexDataType::VERTEX_FLOAT_TYPE,
                                                  TriangleVertexArray::NormalDataType::NORMAL_FLOAT_TYPE,
                                                  TriangleVertexArray::IndexDataType::INDEX_INTEGER_TYPE));
            std::vector<Message> messages;
            TriangleMesh* mesh = W->common.createTriangleMesh(*tva, messages);
            if (!mesh) return -1;
            cs[i] = W->common.createConcaveMeshShape(mesh, Vector3(c.scale[0], c.scale[1], c.scale[2]));
        }
        else if (sh.kind == RP3DG_SHAPE_CONVEX_MESH) {
            if (sh.mesh < 0 || size_t(sh.mesh) >= convex_specs().size()) return -1;
            ConvexSpec& c = convex_specs()[size_t(sh.mesh)];
            PolygonVertexArray pva(uint32(c.vertices.size() / 3), c.vertices.data(), 3 * sizeof(float),
                                   c.indices.data(), sizeof(uint32_t), uint32(c.faces.size()), c.faces.data(),
                                   PolygonVertexArray::VertexDataType::VERTEX_FLOAT_TYPE,
                                   PolygonVertexArray::IndexDataType::INDEX_INTEGER_TYPE);
            std::vector<Message> messages;
            ConvexMesh* mesh = W->common.createConvexMesh(pva, messages);
            if (!mesh) return -1;
            cs[i] = W->common.createConvexMeshShape(mesh, Vector3(c.scale[0], c.scale[1], c.scale[2]));
        }
        else return -1;
    }
    uint32_t ci = 0;
    for (uint32_t b = 0; b < nb; b++) {
        const rp3dg_body_desc& d = bd[b];
        RigidBody* body = W->world->createRigidBody(
            Transform(Vector3(d.position[0], d.position[1], d.position[2]),
                      Quaternion(d.orientation[0], d.orientation[1], d.orientation[2], d.orientation[3])));
        while (ci < nc && uint32_t(cd[ci].body) == b) {
            const rp3dg_collider_desc& c = cd[ci];
            Collider* col = body->addCollider(cs[size_t(c.shape)],
                Transform(Vector3(c.position[0], c.position[1], c.position[2]),
                          Quaternion(c.orientation[0], c.orientation[1], c.orientation[2], c.orientation[3])));
            col->getMaterial().setFrictionCoefficient(c.friction);
            col->getMaterial().setBounciness(c.bounciness);
            col->getMaterial().setMassDensity(c.mass_density);
            col->setCollisionCategoryBits(c.category);
            col->setCollideWithMaskBits(c.mask);
            if (c.flags & RP3DG_COLLIDER_TRIGGER) col->setIsTrigger(true);
            W->colliders.push_back(col);
            ci++;
        }
        if (d.type == RP3DG_BODY_DYNAMIC) body->updateMassPropertiesFromColliders();
        else body->setType(d.type == RP3DG_BODY_STATIC ? BodyType::STATIC : BodyType::KINEMATIC);
        body->setLinearDamping(d.linear_damping);
        body->setAngularDamping(d.angular_damping);
        body->setLinearLockAxisFactor(Vector3(d.linear_lock[0], d.linear_lock[1], d.linear_lock[2]));
        body->setAngularLockAxisFactor(Vector3(d.angular_lock[0], d.angular_lock[1], d.angular_lock[2]));
        body->enableGravity(d.gravity_enabled != 0);
        body->setIsAllowedToSleep(d.allowed_to_sleep != 0);
        if (d.type != RP3DG_BODY_STATIC) {
            body->setLinearVelocity(Vector3(d.linear_velocity[0], d.linear_velocity[1], d.linear_velocity[2]));
            body->setAngularVelocity(Vector3(d.angular_velocity[0], d.angular_velocity[1], d.angular_velocity[2]));
        }
        W->bodies.push_back(body);
    }
    worlds().push_back(std::move(W));
    return int(worlds().size()) - 1;
}

// createJoint for each description, in order (rp3dg_world_add_joints).
int ref_scene_add_joints(int id, const rp3dg_joint_desc* jd, uint32_t n) {
    World& W = *worlds().at(size_t(id));
    for (uint32_t i = 0; i < n; i++) {
        const rp3dg_joint_desc& d = jd[i];
        RigidBody* b1 = W.bodies.at(size_t(d.body1));
        RigidBody* b2 = W.bodies.at(size_t(d.body2));
        const Vector3 anchor(d.anchor[0], d.anchor[1], d.anchor[2]);
        if (d.type == RP3DG_JOINT_BALL_AND_SOCKET) {
            BallAndSocketJointInfo info(b1, b2, anchor);
            info.isCollisionEnabled = d.collision_enabled != 0;
            auto* j = static_cast<BallAndSocketJoint*>(W.world->createJoint(info));
            W.joints.push_back(j);
            if (d.cone_limit_enabled) {
                j->enableConeLimit(true);
                j->setConeLimitHalfAngle(d.cone_half_angle);
            }
        } else if (d.type == RP3DG_JOINT_FIXED) {
            FixedJointInfo info(b1, b2, anchor);
            info.isCollisionEnabled = d.collision_enabled != 0;
            W.joints.push_back(W.world->createJoint(info));
        } else if (d.type == RP3DG_JOINT_SLIDER) {
            SliderJointInfo info(b1, b2, anchor, Vector3(d.axis[0], d.axis[1], d.axis[2]));
            info.isCollisionEnabled = d.collision_enabled != 0;
            info.isLimitEnabled = d.limit_enabled != 0;
            info.minTranslationLimit = d.min_angle;
            info.maxTranslationLimit = d.max_angle;
            info.isMotorEnabled = d.motor_enabled != 0;
            info.motorSpeed = d.motor_speed;
            info.maxMotorForce = d.max_motor_torque;
            W.joints.push_back(W.world->createJoint(info));
        } else {
            HingeJointInfo info(b1, b2, anchor, Vector3(d.axis[0], d.axis[1], d.axis[2]));
            info.isCollisionEnabled = d.collision_enabled != 0;
            info.isLimitEnabled = d.limit_enabled != 0;
            info.minAngleLimit = d.min_angle;
            info.maxAngleLimit = d.max_angle;
            info.isMotorEnabled = d.motor_enabled != 0;
            info.motorSpeed = d.motor_speed;
            info.maxMotorTorque = d.max_motor_torque;
            W.joints.push_back(W.world->createJoint(info));
        }
    }
    return 0;
}

// PhysicsWorld::raycast for each ray with a RaycastCallback that keeps the
// last hit and returns its hitFraction (mode 0), returns 0 after the first
// hit (mode 1) or records every hit and returns 1 (mode 2); hits as
// rp3dg_raycast_hit (flags 0), max_hits records per ray, counts per ray.
struct RayRecorder : public RaycastCallback {
    int mode = 0;
    uint32_t max_hits = 1, count = 0;
    rp3dg_raycast_hit* out = nullptr;
    const std::unordered_map<const void*, int32_t>* bindex = nullptr;
    const std::unordered_map<const void*, int32_t>* cindex = nullptr;
    decimal notifyRaycastHit(const RaycastInfo& info) override {
        rp3dg_raycast_hit h{};
        h.world_point[0] = float(info.worldPoint.x); h.world_point[1] = float(info.worldPoint.y);
        h.world_point[2] = float(info.worldPoint.z);
        h.world_normal[0] = float(info.worldNormal.x); h.world_normal[1] = float(info.worldNormal.y);
        h.world_normal[2] = float(info.worldNormal.z);
        h.hit_fraction = float(info.hitFraction);
        h.body = bindex->at(static_cast<const void*>(info.body));
        h.collider = cindex->at(static_cast<const void*>(info.collider));
        if (mode == 2) {
            if (count < max_hits) out[count] = h;
        } else if (max_hits) {
            out[0] = h;
        }
        count++;
        return mode == 0 ? info.hitFraction : (mode == 1 ? decimal(0.0) : decimal(1.0));
    }
};
int ref_scene_raycast(int id, const rp3dg_ray* rays, uint32_t n, int mode, uint32_t max_hits, rp3dg_raycast_hit* hits,
                      uint32_t* counts) {
    World& W = *worlds().at(size_t(id));
    std::unordered_map<const void*, int32_t> bindex, cindex;
    for (size_t i = 0; i < W.bodies.size(); i++) bindex[static_cast<const void*>(static_cast<Body*>(W.bodies[i]))] = int32_t(i);
    for (size_t i = 0; i < W.colliders.size(); i++) cindex[static_cast<const void*>(W.colliders[i])] = int32_t(i);
    RayRecorder cb;
    cb.mode = mode;
    cb.max_hits = max_hits;
    cb.bindex = &bindex;
    cb.cindex = &cindex;
    for (uint32_t i = 0; i < n; i++) {
        const rp3dg_ray& r = rays[i];
        cb.count = 0;
        cb.out = hits + size_t(i) * max_hits;
        Ray ray(Vector3(r.point1[0], r.point1[1], r.point1[2]), Vector3(r.point2[0], r.point2[1], r.point2[2]),
                r.max_fraction);
        W.world->raycast(ray, &cb, static_cast<unsigned short>(r.category_mask));
        counts[i] = cb.count;
    }
    return 0;
}

// HingeJoint::setMotorSpeed / SliderJoint::setMotorSpeed on joint k.
int ref_scene_set_motor_speed(int id, uint32_t k, float speed) {
    World& W = *worlds().at(size_t(id));
    Joint* j = W.joints.at(size_t(k));
    if (auto* h = dynamic_cast<HingeJoint*>(j)) {
        h->setMotorSpeed(speed);
        return 0;
    }
    if (auto* sl = dynamic_cast<SliderJoint*>(j)) {
        sl->setMotorSpeed(speed);
        return 0;
    }
    return -1;
}

// Body state in creation order.
int ref_scene_bodies(int id, float* pos, float* ori, float* lv, float* av, uint8_t* sleeping) {
    World& W = *worlds().at(size_t(id));
    for (size_t i = 0; i < W.bodies.size(); i++) {
        RigidBody* b = W.bodies[i];
        const Transform& t = b->getTransform();
        const Vector3 p = t.getPosition();
        const Quaternion q = t.getOrientation();
        const Vector3 v = b->getLinearVelocity(), a = b->getAngularVelocity();
        if (pos) { pos[3 * i] = float(p.x); pos[3 * i + 1] = float(p.y); pos[3 * i + 2] = float(p.z); }
        if (ori) { ori[4 * i] = float(q.x); ori[4 * i + 1] = float(q.y); ori[4 * i + 2] = float(q.z); ori[4 * i + 3] = float(q.w); }
        if (lv) { lv[3 * i] = float(v.x); lv[3 * i + 1] = float(v.y); lv[3 * i + 2] = float(v.z); }
        if (av) { av[3 * i] = float(a.x); av[3 * i + 1] = float(a.y); av[3 * i + 2] = float(a.z); }
        if (sleeping) sleeping[i] = b->isSleeping() ? 1 : 0;
    }
    return int(W.bodies.size());
}

// Overlapping-pair ids in array order (enabled convex pairs, then disabled).
long ref_scene_pairs(int id, uint64_t* out, long cap) {
    World& W = *worlds().at(size_t(id));
    OverlappingPairs& op = W.world->mCollisionDetection.mOverlappingPairs;
    long k = 0;
    for (uint64 i = 0; i < op.mConvexPairs.size(); i++, k++)
        if (out && k < cap) out[k] = op.mConvexPairs[i].pairID;
    for (uint64 i = 0; i < op.mDisabledConvexPairs.size(); i++, k++)
        if (out && k < cap) out[k] = op.mDisabledConvexPairs[i].pairID;
    for (uint64 i = 0; i < op.mConcavePairs.size(); i++, k++)
        if (out && k < cap) out[k] = op.mConcavePairs[i].pairID;
    for (uint64 i = 0; i < op.mDisabledConcavePairs.size(); i++, k++)
        if (out && k < cap) out[k] = op.mDisabledConcavePairs[i].pairID;
    return k;
}

// Contact manifolds of the last step in the solver's order: body creation
// indices, point counts and the points (normal + depth, local points).
long ref_scene_contacts(int id, int32_t* body1, int32_t* body2, uint8_t* npts, long cap, float* nd, float* l1,
                        float* l2, long cap_points, long* nb_points) {
    World& W = *worlds().at(size_t(id));
    PhysicsWorld& w = *W.world;
    std::unordered_map<uint32_t, int32_t> index;
    for (size_t i = 0; i < W.bodies.size(); i++) index[W.bodies[i]->getEntity().id] = int32_t(i);
    Array<ContactManifold>& mans = *w.mCollisionDetection.mCurrentContactManifolds;
    Array<ContactPoint>& pts = *w.mCollisionDetection.mCurrentContactPoints;
    long k = 0, p = 0;
    for (uint64 m = 0; m < mans.size(); m++, k++) {
        const ContactManifold& M = mans[m];
        if (k < cap) {
            if (body1) body1[k] = index[M.bodyEntity1.id];
            if (body2) body2[k] = index[M.bodyEntity2.id];
            if (npts) npts[k] = uint8_t(M.nbContactPoints);
        }
        for (uint32 c = M.contactPointsIndex; c < M.contactPointsIndex + M.nbContactPoints; c++, p++) {
            if (p >= cap_points) continue;
            const ContactPoint& P = pts[c];
            const Vector3 n = P.getNormal(), a = P.getLocalPointOnShape1(), b = P.getLocalPointOnShape2();
            if (nd) { nd[4 * p] = float(n.x); nd[4 * p + 1] = float(n.y); nd[4 * p + 2] = float(n.z); nd[4 * p + 3] = float(P.getPenetrationDepth()); }
            if (l1) { l1[4 * p] = float(a.x); l1[4 * p + 1] = float(a.y); l1[4 * p + 2] = float(a.z); l1[4 * p + 3] = 0.0f; }
            if (l2) { l2[4 * p] = float(b.x); l2[4 * p + 1] = float(b.y); l2[4 * p + 2] = float(b.z); l2[4 * p + 3] = 0.0f; }
        }
    }
    if (nb_points) *nb_points = p;
    return k;
}

void ref_world_destroy_all(void) { worlds().clear(); }

}  // extern "C"
