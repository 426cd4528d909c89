/*
 * pe_b200_collision_system.h -- pe's collision system with the whole time step on a B200.
 *
 * Two specialisations of pe's CollisionSystem class template, selected by the coarse-detector
 * policy pe::detection::coarse::B200Detection (pe_b200_pe_config.h):
 *   CollisionSystem< C<B200Detection,FD,BG,response::DEMSolver> >
 *       the interface of pe/core/collisionsystem/DEMSolver.h:112-313;
 *   CollisionSystem< C<B200Detection,FD,BG,response::HardContactSemiImplicitTimesteppingSolvers> >
 *       the interface of pe/core/collisionsystem/HardContactSemiImplicitTimesteppingSolvers.h:
 *       186-283, with pe's RelaxationModel names and setters.
 * pe's World (src/core/World.cpp:262-306, 330-357) adds and removes bodies and calls
 * simulationStep through theCollisionSystem() exactly as with pe's own systems.  The bodies stay
 * pe's objects, owned by the World; the collision system keeps a device copy (libpe_b200,
 * include/pe_b200.h):
 *   - when bodies were added or removed since the last step, it uploads the materials in use
 *     (Material::get*), the planes and fixed boxes as walls, the spheres in system-id order (so
 *     body 1 of every sphere pair is pe's, MaxContacts.h:550-551) and the moving boxes;
 *   - otherwise it compares every sphere's position, velocities and orientation with what it
 *     last wrote, and uploads the state again if a program changed any (setPosition etc.);
 *   - it advances the device state by one step (gravity and drag from Settings, as pe's move()
 *     reads them) and writes positions, orientations and velocities back into the bodies with
 *     pe's setters, so every getter a program calls afterwards sees the new state.
 * Limits (reported as std::invalid_argument before the step): spheres, planes and boxes only
 * (no capsules, cylinders, unions, meshes); no fixed spheres; no force generators, springs or
 * joints; one process (no MPI domain decomposition).  Errors of the library become
 * std::invalid_argument (PE_B200_ERR_ARG) or std::runtime_error, as pe reports its own.
 */
#ifndef PE_B200_COLLISION_SYSTEM_H
#define PE_B200_COLLISION_SYSTEM_H

#include <pe_b200.h>

#include <algorithm>
#include <cstring>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <pe/core/attachable/AttachableStorage.h>
#include <pe/core/domaindecomp/Domain.h>
#include <pe/core/domaindecomp/ProcessStorage.h>
#include <pe/core/joint/JointStorage.h>
#include <pe/core/Materials.h>
#include <pe/core/rigidbody/BodyCast.h>
#include <pe/core/rigidbody/BodyStorage.h>
#include <pe/core/rigidbody/Box.h>
#include <pe/core/rigidbody/Plane.h>
#include <pe/core/rigidbody/Sphere.h>
#include <pe/core/Settings.h>
#include <pe/core/contact/ContactVector.h>
#include <pe/util/logging/Logger.h>
#include <pe/util/policies/NoDelete.h>
#include <pe/util/singleton/Singleton.h>

namespace pe {

namespace b200 {

// Status of a libpe_b200 call as pe reports errors: exceptions.
inline void check(int rc, pe_b200_ctx *ctx, const char *what) {
    if (rc == PE_B200_OK) return;
    std::ostringstream m;
    m << "pe_b200: " << what << " failed (status " << rc << ")";
    if (ctx && *pe_b200_last_error(ctx)) m << ": " << pe_b200_last_error(ctx);
    if (rc == PE_B200_ERR_ARG) throw std::invalid_argument(m.str());
    throw std::runtime_error(m.str());
}

// The device side of one collision system: a libpe_b200 context, the body lists in the order
// the device knows them, and the state last exchanged with the bodies.
class Bridge {
public:
    explicit Bridge(int32_t solver) : ctx_(NULL), dirty_(true), g_{0, 0, 0}, damping_(1.0) {
        pe_b200_params p;
        pe_b200_default_params(&p);
        p.solver = solver;
#ifdef PE_B200_MIXED_PRECISION
        p.precision = PE_B200_MIXED;
#endif
        p.track_orientation = 1;   // pe's spheres carry an orientation (Default.h:190-193)
        check(pe_b200_create(&p, &ctx_), NULL, "pe_b200_create");
    }
    ~Bridge() {
        if (ctx_) pe_b200_destroy(ctx_);
    }

    pe_b200_ctx *context() { return ctx_; }
    void markDirty() { dirty_ = true; }

    // HCSITS settings (HardContactSemiImplicitTimesteppingSolvers.h:770-850)
    void setMaxIterations(size_t n) {
        check(pe_b200_set_max_iterations(ctx_, (int32_t)std::min<size_t>(n, 0x7fffffff)), ctx_,
              "setMaxIterations");
    }
    void setRelaxationModel(int model) {
        check(pe_b200_set_relaxation_model(ctx_, model), ctx_, "setRelaxationModel");
    }
    void setErrorReductionParameter(real erp) {
        check(pe_b200_set_error_reduction(ctx_, erp), ctx_, "setErrorReductionParameter");
    }
    size_t numberOfContacts() {
        int64_t nc = 0;
        int32_t ncol = 0;
        double dmax = 0, res = 0;
        if (pe_b200_last_step_stats(ctx_, &nc, &ncol, &dmax, &res) != PE_B200_OK) return 0;
        return (size_t)nc;
    }

    // One time step of every body of `bodies`.
    template <typename BS>
    void step(BS &bodies, real dt) {
        if (dirty_) upload(bodies);
        else push();
        const Vec3 &g = Settings::gravity();
        if (g[0] != g_[0] || g[1] != g_[1] || g[2] != g_[2]) {
            g_[0] = g[0]; g_[1] = g[1]; g_[2] = g[2];
            check(pe_b200_set_gravity(ctx_, g_), ctx_, "setGravity");
        }
        if (Settings::damping() != damping_) {
            damping_ = Settings::damping();
            check(pe_b200_set_damping(ctx_, damping_), ctx_, "setDamping");
        }
        check(pe_b200_step(ctx_, 1, dt), ctx_, "simulationStep");
        pull();
    }

    // pe's contacts of the current state (detection only), as pe's coarse + fine detection
    // would report them, in the device's (b1, b2) order.
    template <typename BS, typename Contacts>
    void findContacts(BS &bodies, Contacts &contacts) {
        if (dirty_) upload(bodies);
        else push();
        int64_t nc = 0;
        check(pe_b200_find_contacts(ctx_, 0, NULL, NULL, &nc), ctx_, "findContacts");
        std::vector<int64_t> ids(2 * (size_t)nc + 2);
        std::vector<double> geom(7 * (size_t)nc + 7);
        check(pe_b200_find_contacts(ctx_, nc, ids.data(), geom.data(), &nc), ctx_, "findContacts");
        for (int64_t k = 0; k < nc; ++k) {
            const double *q = &geom[7 * (size_t)k];
            contacts.addVertexFaceContact(body(ids[2 * k]), body(ids[2 * k + 1]),
                                          Vec3(q[0], q[1], q[2]), Vec3(q[3], q[4], q[5]), q[6]);
        }
    }

private:
    Bridge(const Bridge &);
    Bridge &operator=(const Bridge &);

    // the pe body of a device contact id: spheres, then planes, fixed boxes, moving boxes
    GeomID body(int64_t id) const {
        size_t k = (size_t)id;
        if (k < spheres_.size()) return spheres_[k];
        k -= spheres_.size();
        if (k < planes_.size()) return planes_[k];
        k -= planes_.size();
        if (k < fixed_.size()) return fixed_[k];
        k -= fixed_.size();
        if (k < moving_.size()) return moving_[k];
        throw std::runtime_error("pe_b200: contact id out of range");
    }

    struct LessSystemID {
        bool operator()(const RigidBody *a, const RigidBody *b) const {
            return a->getSystemID() < b->getSystemID();
        }
    };

    template <typename BS>
    void upload(BS &bodies) {
        spheres_.clear();
        planes_.clear();
        fixed_.clear();
        moving_.clear();
        for (typename BS::Iterator it = bodies.begin(); it != bodies.end(); ++it) {
            RigidBody *b = *it;
            switch (b->getType()) {
                case sphereType:
                    if (b->isFixed())
                        throw std::invalid_argument(
                            "pe_b200: fixed spheres are not supported by the B200 collision system");
                    spheres_.push_back(static_body_cast<Sphere>(b));
                    break;
                case planeType: planes_.push_back(static_body_cast<Plane>(b)); break;
                case boxType:
                    (b->isFixed() ? fixed_ : moving_).push_back(static_body_cast<Box>(b));
                    break;
                default:
                    throw std::invalid_argument(
                        "pe_b200: only spheres, planes and boxes are supported by the B200 "
                        "collision system");
            }
        }
        // system-id order: body 1 of a pair is the sphere with the smaller id
        std::stable_sort(spheres_.begin(), spheres_.end(), LessSystemID());
        std::stable_sort(planes_.begin(), planes_.end(), LessSystemID());
        std::stable_sort(fixed_.begin(), fixed_.end(), LessSystemID());
        std::stable_sort(moving_.begin(), moving_.end(), LessSystemID());
        // the materials in use, in a dense table
        std::vector<MaterialID> used;
        std::vector<int32_t> smat(spheres_.size()), pmat(planes_.size()), fmat(fixed_.size()),
            mmat(moving_.size());
        index_materials(spheres_, smat, used);
        index_materials(planes_, pmat, used);
        index_materials(fixed_, fmat, used);
        index_materials(moving_, mmat, used);
        std::vector<pe_b200_material> mt(std::max<size_t>(used.size(), 1));
        for (size_t k = 0; k < used.size(); ++k) {
            const MaterialID m = used[k];
            pe_b200_material &o = mt[k];
            o.density = Material::getDensity(m);
            o.cor = Material::getRestitution(m);
            o.csf = Material::getStaticFriction(m);
            o.cdf = Material::getDynamicFriction(m);
            o.poisson = Material::getPoissonRatio(m);
            o.young = Material::getYoungModulus(m);
            o.stiffness = Material::getStiffness(m);
            o.dampingN = Material::getDampingN(m);
            o.dampingT = Material::getDampingT(m);
        }
        if (used.empty()) {   // no bodies: any valid material
            pe_b200_material &o = mt[0];
            o.density = 1; o.cor = 0; o.csf = o.cdf = 0; o.poisson = 0.25; o.young = 1;
            o.stiffness = 1; o.dampingN = o.dampingT = 0;
        }
        check(pe_b200_set_materials(ctx_, (int32_t)mt.size(), mt.data()), ctx_, "materials");
        // walls: planes (n, d with n.x = d on the plane), fixed boxes (centre, sides, rotation)
        std::vector<double> pl(4 * planes_.size()), bx(15 * fixed_.size());
        for (size_t k = 0; k < planes_.size(); ++k) {
            const Vec3 &n = planes_[k]->getNormal();
            pl[4 * k] = n[0]; pl[4 * k + 1] = n[1]; pl[4 * k + 2] = n[2];
            pl[4 * k + 3] = planes_[k]->getDisplacement();
        }
        for (size_t k = 0; k < fixed_.size(); ++k) {
            const Vec3 &c = fixed_[k]->getPosition(), &l = fixed_[k]->getLengths();
            const Rot3 &R = fixed_[k]->getRotation();
            double *o = &bx[15 * k];
            for (int a = 0; a < 3; ++a) { o[a] = c[a]; o[3 + a] = l[a]; }
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) o[6 + 3 * i + j] = R(i, j);
        }
        check(pe_b200_set_walls(ctx_, 0, (int32_t)planes_.size(), pl.data(), pmat.data(),
                                (int32_t)fixed_.size(), bx.data(), fmat.data()),
              ctx_, "walls");
        const size_t n = spheres_.size();
        std::vector<double> r(n);
        gather(x_, v_, w_, q_);
        for (size_t i = 0; i < n; ++i) r[i] = spheres_[i]->getRadius();
        check(pe_b200_upload_bodies(ctx_, (int64_t)n, x_.data(), v_.data(), w_.data(), r.data(),
                                    smat.data(), NULL, 1),
              ctx_, "upload");
        if (n) check(pe_b200_set_orientations(ctx_, q_.data()), ctx_, "orientations");
        if (!moving_.empty()) {
            const size_t m = moving_.size();
            std::vector<double> len(3 * m);
            gather_boxes(bx_, bq_, bv_, bw_);
            for (size_t k = 0; k < m; ++k) {
                const Vec3 &l = moving_[k]->getLengths();
                for (int a = 0; a < 3; ++a) len[3 * k + a] = l[a];
            }
            check(pe_b200_upload_boxes(ctx_, (int32_t)m, bx_.data(), bq_.data(), bv_.data(),
                                       bw_.data(), len.data(), mmat.data(), NULL),
                  ctx_, "boxes");
        }
        dirty_ = false;
    }

    template <typename V>
    static void index_materials(const V &bodies, std::vector<int32_t> &idx,
                                std::vector<MaterialID> &used) {
        for (size_t k = 0; k < bodies.size(); ++k) {
            const MaterialID m = bodies[k]->getMaterial();
            std::vector<MaterialID>::iterator f = std::find(used.begin(), used.end(), m);
            if (f == used.end()) {
                used.push_back(m);
                f = used.end() - 1;
            }
            idx[k] = (int32_t)(f - used.begin());
        }
    }

    void gather(std::vector<double> &x, std::vector<double> &v, std::vector<double> &w,
                std::vector<double> &q) const {
        const size_t n = spheres_.size();
        x.resize(3 * n); v.resize(3 * n); w.resize(3 * n); q.resize(4 * n);
        for (size_t i = 0; i < n; ++i) {
            const Sphere *s = spheres_[i];
            const Vec3 &p = s->getPosition(), &lv = s->getLinearVel(), &av = s->getAngularVel();
            const Quat &o = s->getQuaternion();
            for (int a = 0; a < 3; ++a) {
                x[3 * i + a] = p[a];
                v[3 * i + a] = lv[a];
                w[3 * i + a] = av[a];
            }
            for (int a = 0; a < 4; ++a) q[4 * i + a] = o[a];
        }
    }

    void gather_boxes(std::vector<double> &x, std::vector<double> &q, std::vector<double> &v,
                      std::vector<double> &w) const {
        const size_t m = moving_.size();
        x.resize(3 * m); q.resize(4 * m); v.resize(3 * m); w.resize(3 * m);
        for (size_t k = 0; k < m; ++k) {
            const Box *b = moving_[k];
            const Vec3 &p = b->getPosition(), &lv = b->getLinearVel(), &av = b->getAngularVel();
            const Quat &o = b->getQuaternion();
            for (int a = 0; a < 3; ++a) {
                x[3 * k + a] = p[a];
                v[3 * k + a] = lv[a];
                w[3 * k + a] = av[a];
            }
            for (int a = 0; a < 4; ++a) q[4 * k + a] = o[a];
        }
    }

    static bool same(const std::vector<double> &a, const std::vector<double> &b) {
        return a.size() == b.size() &&
               (a.empty() || std::memcmp(a.data(), b.data(), a.size() * sizeof(double)) == 0);
    }

    // state changed on the host since the last exchange (a program's setPosition, ...) goes to
    // the device before the step
    void push() {
        std::vector<double> x, v, w, q;
        gather(x, v, w, q);
        if (!same(x, x_) || !same(v, v_) || !same(w, w_)) {
            check(pe_b200_set_state(ctx_, x.data(), v.data(), w.data()), ctx_, "setState");
            x_.swap(x); v_.swap(v); w_.swap(w);
        }
        if (!same(q, q_)) {
            if (!q.empty()) check(pe_b200_set_orientations(ctx_, q.data()), ctx_, "orientations");
            q_.swap(q);
        }
        if (!moving_.empty()) {
            std::vector<double> bx, bq, bv, bw;
            gather_boxes(bx, bq, bv, bw);
            // a moving box changed on the host: upload everything again
            if (!same(bx, bx_) || !same(bq, bq_) || !same(bv, bv_) || !same(bw, bw_))
                dirty_ = true;
        }
    }

    // the device state after the step, written into pe's bodies through their setters
    void pull() {
        const size_t n = spheres_.size();
        x_.resize(3 * n); v_.resize(3 * n); w_.resize(3 * n); q_.resize(4 * n);
        check(pe_b200_download_bodies(ctx_, x_.data(), v_.data(), w_.data(), q_.data()), ctx_,
              "download");
        for (size_t i = 0; i < n; ++i) {
            Sphere *s = spheres_[i];
            s->setPosition(x_[3 * i], x_[3 * i + 1], x_[3 * i + 2]);
            s->setOrientation(q_[4 * i], q_[4 * i + 1], q_[4 * i + 2], q_[4 * i + 3]);
            s->setLinearVel(v_[3 * i], v_[3 * i + 1], v_[3 * i + 2]);
            s->setAngularVel(w_[3 * i], w_[3 * i + 1], w_[3 * i + 2]);
        }
        if (!moving_.empty()) {
            const size_t m = moving_.size();
            bx_.resize(3 * m); bq_.resize(4 * m); bv_.resize(3 * m); bw_.resize(3 * m);
            check(pe_b200_download_boxes(ctx_, bx_.data(), bq_.data(), bv_.data(), bw_.data()),
                  ctx_, "download boxes");
            for (size_t k = 0; k < m; ++k) {
                Box *b = moving_[k];
                b->setPosition(bx_[3 * k], bx_[3 * k + 1], bx_[3 * k + 2]);
                b->setOrientation(bq_[4 * k], bq_[4 * k + 1], bq_[4 * k + 2], bq_[4 * k + 3]);
                b->setLinearVel(bv_[3 * k], bv_[3 * k + 1], bv_[3 * k + 2]);
                b->setAngularVel(bw_[3 * k], bw_[3 * k + 1], bw_[3 * k + 2]);
            }
        }
    }

    pe_b200_ctx *ctx_;
    bool dirty_;
    double g_[3], damping_;
    std::vector<Sphere *> spheres_;
    std::vector<Plane *> planes_;
    std::vector<Box *> fixed_, moving_;
    std::vector<double> x_, v_, w_, q_, bx_, bq_, bv_, bw_;
};

}  // namespace b200

namespace detection {
namespace coarse {

// The coarse-detector policy of the B200 collision system.  Detection runs on the device inside
// the step; this class only gives pe's configuration its CoarseDetector type and answers
// findContacts (HashGrids::findContacts, HashGrids.h:1121) through the device.
template <typename C>
class B200Detection {
public:
    typedef BodyStorage<C> BS;
    typedef typename C::BodyID BodyID;

    B200Detection(BS &bodies, BS & /*shadow copies: none without MPI*/)
        : bodies_(bodies), bridge_(NULL) {}
    void bind(b200::Bridge *bridge) { bridge_ = bridge; }
    void add(BodyID) {}
    void remove(BodyID) {}
    void clear() {}
    template <typename Contacts>
    void findContacts(Contacts &contacts) {
        if (!bridge_) throw std::runtime_error("pe_b200: detector without a collision system");
        bridge_->findContacts(bodies_, contacts);
    }

private:
    BS &bodies_;
    b200::Bridge *bridge_;
};

}  // namespace coarse
}  // namespace detection

// ---------------------------------------------------------------------------------------------
// The parts both specialisations share: storages, add/remove (DEMSolver.h:988-1130), clear
// (:2115-2149), and the step through the bridge.  pe's World and MPISystem reach the storages
// as friends; with one process there are no shadow copies and no synchronisation.
// ---------------------------------------------------------------------------------------------
#define PE_B200_COLLISION_SYSTEM_COMMON(SELF)                                                   \
public:                                                                                        \
    typedef BodyStorage<Config> BS;                                                            \
    typedef typename BS::Iterator BodyIterator;                                                \
    typedef typename Config::BodyType BodyType;                                                \
    typedef typename Config::BodyID BodyID;                                                    \
    typedef typename Config::ConstBodyID ConstBodyID;                                          \
    typedef AttachableStorage<Config> AS;                                                      \
    typedef typename Config::AttachableType AttachableType;                                    \
    typedef typename Config::AttachableID AttachableID;                                        \
    typedef typename Config::ConstAttachableID ConstAttachableID;                              \
    typedef JointStorage<Config> JS;                                                           \
    typedef typename Config::JointType JointType;                                              \
    typedef typename Config::JointID JointID;                                                  \
    typedef typename Config::ConstJointID ConstJointID;                                        \
    typedef typename Config::ContactType ContactType;                                          \
    typedef typename Config::ContactID ContactID;                                              \
    typedef typename Config::ConstContactID ConstContactID;                                    \
    typedef ContactVector<ContactType, NoDelete> Contacts;                                     \
    typedef ProcessStorage<Config> PS;                                                         \
    typedef typename PS::Iterator ProcessIterator;                                             \
    typedef typename Config::ProcessType ProcessType;                                          \
    typedef typename Config::ProcessID ProcessID;                                              \
    typedef typename Config::ConstProcessID ConstProcessID;                                    \
    typedef detection::coarse::B200Detection<Config> CoarseDetector;                           \
    typedef FD FineDetector;                                                                   \
    typedef BG<Config> BatchGenerator;                                                         \
                                                                                               \
    ~SELF() { clear(); }                                                                       \
    inline CoarseDetector &getCoarseDetector() { return detector_; }                           \
    inline BS &getBodyStorage() { return bodystorage_; }                                       \
    inline BS &getBodyShadowCopyStorage() { return bodystorageShadowCopies_; }                 \
    inline const PS &getProcessStorage() const { return processstorage_; }                     \
    inline const AS &getAttachableStorage() const { return attachablestorage_; }               \
    inline const Domain &getDomain() const { return domain_; }                                 \
    inline bool isSyncRequired() const { return false; }                                       \
    inline bool isSyncRequiredLocally() const { return false; }                                \
    /* stage times are kept by the library (pe_b200_set_profiling / pe_b200_profile) */       \
    inline void logProfilingSummary() const {}                                                 \
    /* the library context, e.g. for pe_b200_set_profiling or pe_b200_autotune */             \
    inline pe_b200_ctx *getB200Context() { return bridge_.context(); }                         \
                                                                                               \
private:                                                                                       \
    inline void add(BodyID body) {                                                             \
        bodystorage_.add(body);                                                                \
        bridge_.markDirty();                                                                   \
    }                                                                                          \
    inline void remove(BodyID body) {                                                          \
        bodystorage_.remove(body);                                                             \
        bridge_.markDirty();                                                                   \
    }                                                                                          \
    inline BodyIterator remove(BodyIterator body) {                                            \
        bridge_.markDirty();                                                                   \
        return bodystorage_.remove(body);                                                      \
    }                                                                                          \
    inline void removeFromCollisionDetector(BodyID) { bridge_.markDirty(); }                   \
    void simulationStep(real dt) {                                                             \
        if (!attachablestorage_.isEmpty() || !jointstorage_.isEmpty())                         \
            throw std::invalid_argument("pe_b200: attachables and joints are not supported "   \
                                        "by the B200 collision system");                       \
        bridge_.step(bodystorage_, dt);                                                        \
    }                                                                                          \
    void synchronize() {}                                                                      \
    inline void clear() {                                                                      \
        for (BodyIterator body = bodystorage_.begin(); body != bodystorage_.end(); ++body)     \
            delete *body;                                                                      \
        bodystorage_.clear();                                                                  \
        bridge_.markDirty();                                                                   \
    }                                                                                          \
    inline void clearContacts() {}                                                             \
                                                                                               \
    BS bodystorage_;                                                                           \
    BS bodystorageShadowCopies_;                                                               \
    PS processstorage_;                                                                        \
    Domain domain_;                                                                            \
    AS attachablestorage_;                                                                     \
    JS jointstorage_;                                                                          \
    b200::Bridge bridge_;                                                                      \
    CoarseDetector detector_;                                                                  \
                                                                                               \
    friend class World;                                                                        \
    friend class MPISystem;                                                                    \
    template <typename Geometry>                                                               \
    friend void defineLocalDomain(const Geometry &geometry);                                   \
    friend GravityID instantiateGravity(id_t sid, pe::BodyID body, const Vec3 &gravity);       \
    friend GravityID attachGravity(pe::BodyID body, const Vec3 &gravity);                      \
    friend SpringID instantiateSpring(id_t sid, pe::BodyID body1, const Vec3 &anchor1,         \
                                      pe::BodyID body2, const Vec3 &anchor2, real stiffness,   \
                                      real damping, real length, bool visible);                \
    friend SpringID attachSpring(pe::BodyID body1, const Vec3 &anchor1, pe::BodyID body2,      \
                                 const Vec3 &anchor2, real stiffness, real damping,            \
                                 real length, bool visible);                                   \
    friend void detach(pe::AttachableID attachable);                                           \
    friend FixedJointID attachFixedJoint(pe::BodyID body1, const Vec3 &anchor1,                \
                                         pe::BodyID body2, const Vec3 &anchor2, real scale);   \
    friend void detach(pe::JointID joint);                                                     \
    friend CollisionSystemID theCollisionSystem();                                             \
    pe_BEFRIEND_SINGLETON;

// ---- DEM: CollisionSystem< C<B200Detection,FD,BG,response::DEMSolver> > ----------------------
template <typename FD, template <typename> class BG,
          template <template <typename> class, typename, template <typename> class,
                    template <typename, typename, typename> class> class C>
class CollisionSystem<C<detection::coarse::B200Detection, FD, BG, response::DEMSolver> >
    : public Singleton<CollisionSystem<C<detection::coarse::B200Detection, FD, BG,
                                         response::DEMSolver> >,
                       logging::Logger> {
public:
    typedef C<detection::coarse::B200Detection, FD, BG, response::DEMSolver> Config;
    // pe's response type, for pe's ContactSolver typedef (the device runs the response)
    typedef response::DEMSolver<Config> ContactSolver;
    PE_B200_COLLISION_SYSTEM_COMMON(CollisionSystem)

private:
    // replaces DEMSolver.h:335-437: the device context instead of pe's detector and solver
    explicit CollisionSystem()
        : Singleton<CollisionSystem, logging::Logger>(),
          bodystorage_(), bodystorageShadowCopies_(), processstorage_(),
          domain_(processstorage_), attachablestorage_(), jointstorage_(),
          bridge_(PE_B200_DEM), detector_(bodystorage_, bodystorageShadowCopies_) {
        detector_.bind(&bridge_);
    }
};

// ---- hard contacts: CollisionSystem< C<B200Detection,FD,BG,response::HCSITS> > -------------
template <typename FD, template <typename> class BG,
          template <template <typename> class, typename, template <typename> class,
                    template <typename, typename, typename> class> class C>
class CollisionSystem<C<detection::coarse::B200Detection, FD, BG,
                        response::HardContactSemiImplicitTimesteppingSolvers> >
    : public Singleton<CollisionSystem<C<detection::coarse::B200Detection, FD, BG,
                                         response::HardContactSemiImplicitTimesteppingSolvers> >,
                       logging::Logger> {
public:
    typedef C<detection::coarse::B200Detection, FD, BG,
              response::HardContactSemiImplicitTimesteppingSolvers> Config;
    typedef response::HardContactSemiImplicitTimesteppingSolvers<Config> ContactSolver;
    PE_B200_COLLISION_SYSTEM_COMMON(CollisionSystem)

public:
    // pe's relaxation models, HardContactSemiImplicitTimesteppingSolvers.h:172-179
    enum RelaxationModel {
        InelasticFrictionlessContact,
        ApproximateInelasticCoulombContactByDecoupling,
        ApproximateInelasticCoulombContactByOrthogonalProjections,
        InelasticCoulombContactByDecoupling,
        InelasticCoulombContactByOrthogonalProjections,
        InelasticGeneralizedMaximumDissipationContact
    };

    inline size_t getNumberOfContacts() { return bridge_.numberOfContacts(); }
    // HardContactSemiImplicitTimesteppingSolvers.h:770-850.  The relaxation parameter scales the
    // corrections of bodies shared with other processes (:3832-3833); with one process it has
    // no effect and is only stored.
    inline void setRelaxationParameter(real f) { relaxationParam_ = f; }
    inline void setMaxIterations(size_t n) { bridge_.setMaxIterations(n); }
    inline void setRelaxationModel(RelaxationModel m) { bridge_.setRelaxationModel((int)m); }
    inline void setErrorReductionParameter(real erp) { bridge_.setErrorReductionParameter(erp); }
    inline void clearShadowCopies() {}

private:
    // replaces HardContactSemiImplicitTimesteppingSolvers.h:408-460
    explicit CollisionSystem()
        : Singleton<CollisionSystem, logging::Logger>(),
          bodystorage_(), bodystorageShadowCopies_(), processstorage_(),
          domain_(processstorage_), attachablestorage_(), jointstorage_(),
          bridge_(PE_B200_HCSITS), detector_(bodystorage_, bodystorageShadowCopies_),
          relaxationParam_(0.9) {
        detector_.bind(&bridge_);
        // pe's defaults (:420-425: erp 0.7, 100 sweeps, approximate Coulomb friction by
        // decoupling) are the library's defaults (pe_b200_default_params)
    }

    real relaxationParam_;
};

#undef PE_B200_COLLISION_SYSTEM_COMMON

}  // namespace pe

#endif
