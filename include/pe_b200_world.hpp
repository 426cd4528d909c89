/* pe_b200_world.hpp -- pe's World / body-creation API on top of the C ABI of pe_b200.h.
 *
 * Header-only C++17.  A program written against pe's single-domain API
 *
 *     WorldID world = theWorld();
 *     world->setGravity(0.0, 0.0, -9.81);
 *     MaterialID m = createMaterial("granite2", 1.0, 0.0, 0.15, 0.15, 0.25, 1e9, 2e5, 100, 100);
 *     createPlane(100, 0.0, 0.0, 1.0, 0.0, m);
 *     SphereID s = createSphere(1, 0.0, 0.0, 0.5, 0.5, m);
 *     world->run(1000, 1e-4);
 *     Vec3 x = s->getPosition();
 *
 * compiles against this header with `namespace pe = pe_b200;` (or `using namespace pe_b200;`)
 * and runs its time steps on the GPU.  It follows
 *   - World (pe/core/World.h:159-295, src/core/World.cpp:262-357): setGravity, setDamping,
 *     simulationStep, run, size, destroy;
 *   - createMaterial and the predefined materials iron, copper, granite, oak, fir
 *     (src/core/Materials.cpp:175-290, pe/core/Materials.h:831-1176);
 *   - createSphere (src/core/rigidbody/Sphere.cpp:1187-1200), createPlane
 *     (src/core/rigidbody/Plane.cpp:1202-1225), createBox (src/core/rigidbody/Box.cpp:1312-1330);
 *   - the HCSITS setters of the collision system (HardContactSemiImplicitTimesteppingSolvers.h:
 *     172-179 for the model names, 793-850 for the setters);
 * with pe's exceptions: std::invalid_argument for invalid arguments, std::runtime_error for
 * unsupported configurations and device errors.
 *
 * Differences from pe, all checked at the call that hits them:
 *   - spheres and boxes move, planes are fixed; fixed boxes are walls; moving boxes need FP64
 *     precision (setPrecision(PE_B200_MIXED) with a moving box fails at the next step);
 *   - the solver is chosen at run time (theCollisionSystem()->setSolver) instead of by the
 *     compile-time pe_CONSTRAINT_SOLVER; the default is PE_B200_CONSTRAINT_SOLVER
 *     (PE_B200_DEM unless defined before including this header);
 *   - state lives on the GPU: setters upload before the next step, getters download once after
 *     each step (or batch of steps).
 */
#ifndef PE_B200_WORLD_HPP
#define PE_B200_WORLD_HPP

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "pe_b200.h"

#ifndef PE_B200_CONSTRAINT_SOLVER
#define PE_B200_CONSTRAINT_SOLVER PE_B200_DEM
#endif

namespace pe_b200 {

typedef double real;
typedef std::size_t id_t;

// ---- vectors -----------------------------------------------------------------------------------
class Vec3 {
  public:
    Vec3() : v_{0.0, 0.0, 0.0} {}
    Vec3(real x, real y, real z) : v_{x, y, z} {}
    real operator[](std::size_t i) const { return v_[i]; }
    real &operator[](std::size_t i) { return v_[i]; }
    Vec3 operator+(const Vec3 &b) const { return Vec3(v_[0] + b[0], v_[1] + b[1], v_[2] + b[2]); }
    Vec3 operator-(const Vec3 &b) const { return Vec3(v_[0] - b[0], v_[1] - b[1], v_[2] - b[2]); }
    Vec3 operator*(real s) const { return Vec3(v_[0] * s, v_[1] * s, v_[2] * s); }
    real operator*(const Vec3 &b) const { return v_[0] * b[0] + v_[1] * b[1] + v_[2] * b[2]; }
    real sqrLength() const { return (*this) * (*this); }
    real length() const { return std::sqrt(sqrLength()); }
    Vec3 getNormalized() const {
        const real l = length();
        return l > 0.0 ? (*this) * (1.0 / l) : *this;
    }

  private:
    real v_[3];
};

// ---- materials ---------------------------------------------------------------------------------
typedef std::size_t MaterialID;
const MaterialID iron = 0;
const MaterialID copper = 1;
const MaterialID granite = 2;
const MaterialID oak = 3;
const MaterialID fir = 4;
const MaterialID invalid_material = static_cast<MaterialID>(-1);

class Material {
  public:
    Material(const std::string &name, const pe_b200_material &m) : name_(name), m_(m) {}
    const std::string &getName() const { return name_; }
    real getDensity() const { return m_.density; }
    real getRestitution() const { return m_.cor; }
    real getStaticFriction() const { return m_.csf; }
    real getDynamicFriction() const { return m_.cdf; }
    real getPoissonRatio() const { return m_.poisson; }
    real getYoungModulus() const { return m_.young; }
    real getStiffness() const { return m_.stiffness; }
    real getDampingN() const { return m_.dampingN; }
    real getDampingT() const { return m_.dampingT; }
    const pe_b200_material &record() const { return m_; }

  private:
    std::string name_;
    pe_b200_material m_;
};

namespace detail {
inline std::vector<Material> &materials() {
    // pe's predefined materials, in pe's order (pe/core/Materials.h:831, 896, 961, 1026, 1091)
    static std::vector<Material> table = {
        Material("iron", {7874, 0.5, 0.1, 0.1, 0.24, 200, 200, 0, 0}),
        Material("copper", {8920, 0.5, 0.1, 0.1, 0.33, 117, 117, 0, 0}),
        Material("granite", {2800, 0.5, 0.1, 0.1, 0.25, 55, 55, 0, 0}),
        Material("oak", {800, 0.5, 0.1, 0.1, 0.35, 11, 11, 0, 0}),
        Material("fir", {500, 0.5, 0.1, 0.1, 0.34, 13, 13, 0, 0}),
    };
    return table;
}
inline unsigned long &anonymous_materials() {
    static unsigned long count = 0;
    return count;
}
}  // namespace detail

inline const Material &getMaterial(MaterialID id) {
    if (id >= detail::materials().size()) throw std::invalid_argument("Invalid material ID");
    return detail::materials()[id];
}

/* Material::find (src/core/Materials.cpp:302) */
inline MaterialID findMaterial(const std::string &name) {
    const std::vector<Material> &t = detail::materials();
    for (std::size_t i = 0; i < t.size(); ++i)
        if (t[i].getName() == name) return i;
    return invalid_material;
}

inline void markMaterialsChanged();

/* createMaterial with pe's argument checks and messages (src/core/Materials.cpp:175-223) */
inline MaterialID createMaterial(const std::string &name, real density, real cor, real csf,
                                 real cdf, real poisson, real young, real stiffness,
                                 real dampingN, real dampingT) {
    if (findMaterial(name) != invalid_material)
        throw std::invalid_argument("Material of that name already exists!");
    if (density <= 0.0) throw std::invalid_argument("Invalid material density!");
    if (cor < 0.0 || cor > 1.0) throw std::invalid_argument("Invalid coefficient of restitution!");
    if (csf < 0.0) throw std::invalid_argument("Invalid coefficient of static friction!");
    if (cdf < 0.0) throw std::invalid_argument("Invalid coefficient of dynamic friction!");
    if (poisson < -1.0 || poisson > 0.5) throw std::invalid_argument("Invalid Poisson's ratio");
    if (young <= 0.0) throw std::invalid_argument("Invalid Young's modulus");
    if (stiffness <= 0.0) throw std::invalid_argument("Invalid stiffness");
    if (dampingN < 0.0 || dampingT < 0.0)
        throw std::invalid_argument("Invalid damping coefficients");
    detail::materials().emplace_back(
        name, pe_b200_material{density, cor, csf, cdf, poisson, young, stiffness, dampingN, dampingT});
    markMaterialsChanged();
    return detail::materials().size() - 1;
}

/* anonymous material "Material<k>" (src/core/Materials.cpp:275-290) */
inline MaterialID createMaterial(real density, real cor, real csf, real cdf, real poisson,
                                 real young, real stiffness, real dampingN, real dampingT) {
    std::string name;
    do {
        if (detail::anonymous_materials() + 1 == 0)
            throw std::runtime_error("Index overflow for anonymous materials");
        name = "Material" + std::to_string(++detail::anonymous_materials());
    } while (findMaterial(name) != invalid_material);
    return createMaterial(name, density, cor, csf, cdf, poisson, young, stiffness, dampingN,
                          dampingT);
}

// ---- bodies ------------------------------------------------------------------------------------
class World;
namespace detail {
inline void rot_of(const real q[4], real R[9]);
}

class RigidBody {
  public:
    virtual ~RigidBody() {}
    id_t getID() const { return uid_; }
    id_t getSystemID() const { return sid_; }
    MaterialID getMaterial() const { return mat_; }
    bool isVisible() const { return visible_; }

  protected:
    RigidBody(World *w, id_t sid, id_t uid, MaterialID mat, bool visible)
        : world_(w), sid_(sid), uid_(uid), mat_(mat), visible_(visible) {}
    World *world_;
    id_t sid_, uid_;
    MaterialID mat_;
    bool visible_;
    friend class World;
};

class Sphere : public RigidBody {
  public:
    real getRadius() const { return r_; }
    /* SphereBase::calcMass (pe/core/rigidbody/SphereBase.h:169-171) */
    real getMass() const {
        return 4.0 / 3.0 * M_PI * r_ * r_ * r_ * getMaterial_().getDensity();
    }
    Vec3 getPosition() const;
    Vec3 getLinearVel() const;
    Vec3 getAngularVel() const;
    void setPosition(real x, real y, real z);
    void setPosition(const Vec3 &p) { setPosition(p[0], p[1], p[2]); }
    void setLinearVel(real x, real y, real z);
    void setLinearVel(const Vec3 &v) { setLinearVel(v[0], v[1], v[2]); }
    void setAngularVel(real x, real y, real z);
    void setAngularVel(const Vec3 &w) { setAngularVel(w[0], w[1], w[2]); }

  private:
    Sphere(World *w, id_t sid, id_t uid, const Vec3 &x, real r, MaterialID m, bool visible)
        : RigidBody(w, sid, uid, m, visible), x_(x), r_(r) {}
    const Material &getMaterial_() const { return pe_b200::getMaterial(mat_); }
    Vec3 x_, v_, w_;
    real r_;
    friend class World;
};

class Plane : public RigidBody {
  public:
    const Vec3 &getNormal() const { return n_; }
    real getDisplacement() const { return d_; }

  private:
    Plane(World *w, id_t sid, id_t uid, const Vec3 &n, real d, MaterialID m, bool visible)
        : RigidBody(w, sid, uid, m, visible), n_(n), d_(d) {}
    Vec3 n_;
    real d_;
    friend class World;
};

/* A box: fixed boxes are walls, the others move (BoxTrait::move for DEM, box bodies in the
 * hard-contact solver).  Contacts between a fixed and a moving box are computed with the fixed
 * box as pe's lower system id, as when fixed boxes are created first. */
class Box : public RigidBody {
  public:
    Vec3 getPosition() const;
    const Vec3 &getLengths() const { return l_; }
    bool isFixed() const { return fixed_; }
    void setFixed(bool fixed);
    /* BoxBase::calcMass (pe/core/rigidbody/BoxBase.h:186-189) */
    real getMass() const { return l_[0] * l_[1] * l_[2] * pe_b200::getMaterial(mat_).getDensity(); }
    /* rotation matrix, row-major (Quaternion::toRotationMatrix of the orientation) */
    const real *getRotation() const;
    /* orientation (w, x, y, z) */
    std::array<real, 4> getQuaternion() const;
    Vec3 getLinearVel() const;
    Vec3 getAngularVel() const;
    void setPosition(real x, real y, real z);
    void setPosition(const Vec3 &p) { setPosition(p[0], p[1], p[2]); }
    void setLinearVel(real x, real y, real z);
    void setLinearVel(const Vec3 &v) { setLinearVel(v[0], v[1], v[2]); }
    void setAngularVel(real x, real y, real z);
    void setAngularVel(const Vec3 &w) { setAngularVel(w[0], w[1], w[2]); }
    /* Box::setOrientation (src/core/rigidbody/Box.cpp:289-300) */
    void setOrientation(real r, real i, real j, real k);
    /* Box::rotate (src/core/rigidbody/Box.cpp:489-500): q = Quat(axis, angle) * q */
    void rotate(const Vec3 &axis, real angle);
    void rotate(real x, real y, real z, real angle) { rotate(Vec3(x, y, z), angle); }

  private:
    Box(World *w, id_t sid, id_t uid, const Vec3 &x, const Vec3 &l, MaterialID m, bool visible)
        : RigidBody(w, sid, uid, m, visible), x_(x), l_(l), q_{1, 0, 0, 0},
          R_{1, 0, 0, 0, 1, 0, 0, 0, 1} {}
    void changed();
    Vec3 x_, l_, v_, w_;
    real q_[4];
    real R_[9];
    bool fixed_ = false;
    friend class World;
};

typedef Sphere *SphereID;
typedef Plane *PlaneID;
typedef Box *BoxID;
typedef RigidBody *BodyID;

// ---- collision system (solver settings) --------------------------------------------------------
class CollisionSystem {
  public:
    /* HardContactSemiImplicitTimesteppingSolvers.h:172-179 */
    enum RelaxationModel {
        InelasticFrictionlessContact,
        ApproximateInelasticCoulombContactByDecoupling,
        ApproximateInelasticCoulombContactByOrthogonalProjections,
        InelasticCoulombContactByDecoupling,
        InelasticCoulombContactByOrthogonalProjections,
        InelasticGeneralizedMaximumDissipationContact
    };
    /* HCSITS.h:793-850 */
    void setMaxIterations(std::size_t n);
    void setRelaxationModel(RelaxationModel m);
    void setErrorReductionParameter(real erp);
    /* pe stores it but none of its relaxation models reads it (they use w = 1) */
    void setRelaxationParameter(real omega) { omega_ = omega; }
    real getRelaxationParameter() const { return omega_; }
    std::size_t getMaxIterations() const { return (std::size_t)p_.max_iterations; }
    RelaxationModel getRelaxationModel() const { return model_; }
    /* run-time replacement of the compile-time pe_CONSTRAINT_SOLVER */
    void setSolver(int solver);   /* PE_B200_DEM or PE_B200_HCSITS */
    void setPrecision(int prec);  /* PE_B200_FP64 or PE_B200_MIXED */
    void setDevice(int device);
    /* pe's compile-time DEMConfig forceModel at run time: 0 linear ('basic'), 1 Hertz */
    void setForceModel(int model);
    int getSolver() const { return p_.solver; }
    int getPrecision() const { return p_.precision; }
    /* number of contacts and NBGS colours of the last step */
    void lastStepStats(int64_t *ncontacts, int32_t *ncolors) const;

  private:
    CollisionSystem() {
        pe_b200_default_params(&p_);
        p_.solver = PE_B200_CONSTRAINT_SOLVER;
    }
    pe_b200_params p_;
    RelaxationModel model_ = ApproximateInelasticCoulombContactByDecoupling;
    real omega_ = 0.75;
    World *world_ = nullptr;
    friend class World;
};

// ---- world -------------------------------------------------------------------------------------
class World {
  public:
    typedef std::size_t SizeType;

    static World &instance() {
        static World w;
        return w;
    }
    ~World() { release(); }

    void setGravity(real gx, real gy, real gz) { setGravity(Vec3(gx, gy, gz)); }
    void setGravity(const Vec3 &g) {
        g_ = g;
        if (ctx_) check(pe_b200_set_gravity(ctx_, gravity_array()));
    }
    const Vec3 &getGravity() const { return g_; }
    void setDamping(real damping) {
        if (damping < 0.0 || damping > 1.0) throw std::invalid_argument("Invalid damping factor");
        damping_ = damping;
        if (ctx_) check(pe_b200_set_damping(ctx_, damping_));
    }
    real getDamping() const { return damping_; }

    SizeType size() const { return spheres_.size() + planes_.size() + boxes_.size(); }
    SizeType numSpheres() const { return spheres_.size(); }
    SizeType numPlanes() const { return planes_.size(); }
    SizeType numBoxes() const { return boxes_.size(); }
    SphereID sphere(SizeType i) const { return spheres_.at(i).get(); }

    /* World::simulationStep (src/core/World.cpp:330-357) */
    void simulationStep(real timestep) { run(1, timestep); }
    /* World::run: `steps` time steps in one call into the library */
    void run(unsigned int steps, real timestep) {
        if (!(timestep > 0.0)) throw std::invalid_argument("Invalid time step size");
        prepare();
        if (!spheres_.empty()) check(pe_b200_step(ctx_, (int32_t)steps, timestep));
        host_stale_ = !spheres_.empty();
    }

    /* destroy(BodyID): removes and deletes a body */
    void destroy(BodyID b) {
        pull();
        if (erase(spheres_, b) || erase(planes_, b) || erase(boxes_, b)) {
            structure_dirty_ = true;
            return;
        }
        throw std::invalid_argument("Body does not belong to this world");
    }
    /* removes every body (pe's World::destroy of all bodies / a fresh world) */
    void clear() {
        spheres_.clear();
        planes_.clear();
        boxes_.clear();
        structure_dirty_ = true;
        host_stale_ = false;
    }

    CollisionSystem &collisionSystem() { return cs_; }
    pe_b200_ctx *context() { return ctx_; }

    /* pe's binary checkpoint (BodyBinaryWriter::writeFile, src/core/BodyBinaryWriter.cpp:47-245)
     * for one process: spheres and boxes in the local chunk, planes (which pe writes only when
     * global) left out; big-endian as pe's network-order buffers.  Sphere orientations are not
     * tracked here and are written as the identity. */
    void writeCheckpoint(const char *filename) const;
    /* BodyBinaryReader::readFile (src/core/BodyBinaryReader.cpp:57-300): every body of the world
     * is replaced by the file's; material ids refer to the material table as it is now */
    void readCheckpoint(const char *filename);

    // -- used by the free functions and the body classes ----------------------------------------
    SphereID addSphere(id_t uid, const Vec3 &x, real r, MaterialID m, bool visible) {
        pull();
        if (!(r > 0.0)) throw std::invalid_argument("Invalid sphere radius");
        getMaterial(m);
        spheres_.emplace_back(new Sphere(this, next_sid_++, uid, x, r, m, visible));
        structure_dirty_ = true;
        return spheres_.back().get();
    }
    PlaneID addPlane(id_t uid, Vec3 n, real d, MaterialID m, bool visible) {
        if (n.sqrLength() == 0.0) throw std::invalid_argument("Invalid plane normal!");
        getMaterial(m);
        pull();
        planes_.emplace_back(new Plane(this, next_sid_++, uid, n.getNormalized(), d, m, visible));
        structure_dirty_ = true;
        return planes_.back().get();
    }
    BoxID addBox(id_t uid, const Vec3 &x, const Vec3 &l, MaterialID m, bool visible) {
        if (l[0] <= 0.0 || l[1] <= 0.0 || l[2] <= 0.0)
            throw std::invalid_argument("Invalid side length");
        getMaterial(m);
        pull();
        boxes_.emplace_back(new Box(this, next_sid_++, uid, x, l, m, visible));
        structure_dirty_ = true;
        return boxes_.back().get();
    }
    void pull() const {
        if (!host_stale_ || !ctx_) return;
        const std::size_t n = spheres_.size();
        std::vector<double> x(3 * n), v(3 * n), w(3 * n);
        if (n) check(pe_b200_download_bodies(ctx_, x.data(), v.data(), w.data(), nullptr));
        for (std::size_t i = 0; i < n; ++i) {
            Sphere &s = *spheres_[i];
            s.x_ = Vec3(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
            s.v_ = Vec3(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
            s.w_ = Vec3(w[3 * i], w[3 * i + 1], w[3 * i + 2]);
        }
        std::vector<Box *> mv;
        for (const auto &b : boxes_)
            if (!b->fixed_) mv.push_back(b.get());
        if (!mv.empty()) {
            const std::size_t m = mv.size();
            std::vector<double> bx(3 * m), bq(4 * m), bv(3 * m), bw(3 * m);
            check(pe_b200_download_boxes(ctx_, bx.data(), bq.data(), bv.data(), bw.data()));
            for (std::size_t k = 0; k < m; ++k) {
                Box &b = *mv[k];
                b.x_ = Vec3(bx[3 * k], bx[3 * k + 1], bx[3 * k + 2]);
                for (int a = 0; a < 4; ++a) b.q_[a] = bq[4 * k + a];
                detail::rot_of(b.q_, b.R_);
                b.v_ = Vec3(bv[3 * k], bv[3 * k + 1], bv[3 * k + 2]);
                b.w_ = Vec3(bw[3 * k], bw[3 * k + 1], bw[3 * k + 2]);
            }
        }
        host_stale_ = false;
    }
    void markStateDirty() { state_dirty_ = true; }
    void markBoxesDirty() { boxes_dirty_ = true; }
    void markStructureDirty() { structure_dirty_ = true; }
    void markParamsDirty() { params_dirty_ = true; }
    void check(int rc) const {
        if (rc == PE_B200_OK) return;
        const std::string msg = ctx_ ? pe_b200_last_error(ctx_) : "pe_b200 error";
        if (rc == PE_B200_ERR_ARG) throw std::invalid_argument(msg);
        throw std::runtime_error(msg + " (status " + std::to_string(rc) + ")");
    }

  private:
    World() { cs_.world_ = this; }
    World(const World &) = delete;
    World &operator=(const World &) = delete;

    template <typename T>
    static bool erase(std::vector<std::unique_ptr<T>> &v, BodyID b) {
        for (auto it = v.begin(); it != v.end(); ++it)
            if (it->get() == b) {
                v.erase(it);
                return true;
            }
        return false;
    }
    const double *gravity_array() {
        ga_[0] = g_[0];
        ga_[1] = g_[1];
        ga_[2] = g_[2];
        return ga_;
    }
    void release() {
        if (ctx_) pe_b200_destroy(ctx_);
        ctx_ = nullptr;
    }
    // brings the device up to date with the host-side world before a step
    void prepare() {
        if (params_dirty_ || !ctx_) {
            pull();
            release();
            pe_b200_params p = cs_.p_;
            for (int k = 0; k < 3; ++k) p.gravity[k] = g_[k];
            p.damping = damping_;
            int rc = pe_b200_create(&p, &ctx_);
            if (rc != PE_B200_OK) {
                ctx_ = nullptr;
                throw std::runtime_error("pe_b200_create failed (status " + std::to_string(rc) + ")");
            }
            params_dirty_ = false;
            structure_dirty_ = true;
        }
        if (structure_dirty_) {
            std::vector<pe_b200_material> mats;
            for (const Material &m : detail::materials()) mats.push_back(m.record());
            check(pe_b200_set_materials(ctx_, (int32_t)mats.size(), mats.data()));
            std::vector<double> planes, boxes;
            std::vector<int32_t> pm, bm;
            for (const auto &p : planes_) {
                planes.insert(planes.end(), {p->n_[0], p->n_[1], p->n_[2], p->d_});
                pm.push_back((int32_t)p->mat_);
            }
            int32_t nfixed = 0;
            for (const auto &b : boxes_) {
                if (!b->fixed_) continue;
                boxes.insert(boxes.end(), {b->x_[0], b->x_[1], b->x_[2], b->l_[0], b->l_[1], b->l_[2]});
                boxes.insert(boxes.end(), b->R_, b->R_ + 9);
                bm.push_back((int32_t)b->mat_);
                ++nfixed;
            }
            check(pe_b200_set_walls(ctx_, 0, (int32_t)planes_.size(), planes.data(), pm.data(),
                                    nfixed, boxes.data(), bm.data()));
            const std::size_t n = spheres_.size();
            std::vector<double> x, v, w, r;
            std::vector<int32_t> mat;
            for (const auto &s : spheres_) {
                x.insert(x.end(), {s->x_[0], s->x_[1], s->x_[2]});
                v.insert(v.end(), {s->v_[0], s->v_[1], s->v_[2]});
                w.insert(w.end(), {s->w_[0], s->w_[1], s->w_[2]});
                r.push_back(s->r_);
                mat.push_back((int32_t)s->mat_);
            }
            check(pe_b200_upload_bodies(ctx_, (int64_t)n, x.data(), v.data(), w.data(), r.data(),
                                        mat.data(), nullptr, 1));
            upload_boxes();
            structure_dirty_ = false;
            state_dirty_ = false;
            boxes_dirty_ = false;
        } else if (state_dirty_ || boxes_dirty_) {
            const std::size_t n = spheres_.size();
            std::vector<double> x(3 * n), v(3 * n), w(3 * n);
            for (std::size_t i = 0; i < n; ++i)
                for (int a = 0; a < 3; ++a) {
                    x[3 * i + a] = spheres_[i]->x_[a];
                    v[3 * i + a] = spheres_[i]->v_[a];
                    w[3 * i + a] = spheres_[i]->w_[a];
                }
            if (n && state_dirty_) check(pe_b200_set_state(ctx_, x.data(), v.data(), w.data()));
            if (boxes_dirty_) upload_boxes();
            state_dirty_ = false;
            boxes_dirty_ = false;
        }
        check(pe_b200_set_gravity(ctx_, gravity_array()));
        check(pe_b200_set_damping(ctx_, damping_));
    }

    // the moving boxes, in system-id order
    void upload_boxes() {
        std::vector<double> x, q, v, w, l;
        std::vector<int32_t> mat;
        for (const auto &b : boxes_) {
            if (b->fixed_) continue;
            x.insert(x.end(), {b->x_[0], b->x_[1], b->x_[2]});
            q.insert(q.end(), b->q_, b->q_ + 4);
            v.insert(v.end(), {b->v_[0], b->v_[1], b->v_[2]});
            w.insert(w.end(), {b->w_[0], b->w_[1], b->w_[2]});
            l.insert(l.end(), {b->l_[0], b->l_[1], b->l_[2]});
            mat.push_back((int32_t)b->mat_);
        }
        check(pe_b200_upload_boxes(ctx_, (int32_t)mat.size(), x.data(), q.data(), v.data(),
                                   w.data(), l.data(), mat.data(), nullptr));
    }

    friend class BodyBinaryWriter;
    friend class BodyBinaryReader;
    friend class Box;
    CollisionSystem cs_;
    pe_b200_ctx *ctx_ = nullptr;
    std::vector<std::unique_ptr<Sphere>> spheres_;
    std::vector<std::unique_ptr<Plane>> planes_;
    std::vector<std::unique_ptr<Box>> boxes_;
    Vec3 g_;
    double ga_[3] = {0.0, 0.0, 0.0};
    real damping_ = 1.0;
    id_t next_sid_ = 0;
    bool structure_dirty_ = true, state_dirty_ = false, params_dirty_ = true, boxes_dirty_ = false;
    mutable bool host_stale_ = false;
};

typedef World *WorldID;

/* pe's checkpoint writer and reader (pe/core/BodyBinaryWriter.h:96, BodyBinaryReader.h:61) */
class BodyBinaryWriter {
  public:
    void writeFile(const char *filename) { World::instance().writeCheckpoint(filename); }
};
class BodyBinaryReader {
  public:
    void readFile(const char *filename) { World::instance().readCheckpoint(filename); }
};

namespace detail {
// big-endian encoding of pe's send buffers (pe/core/BodyBinaryWriter.h:68)
inline void put_be(std::string &out, const void *p, size_t n) {
    const unsigned char *b = static_cast<const unsigned char *>(p);
    for (size_t k = 0; k < n; ++k) out.push_back((char)b[n - 1 - k]);
}
template <typename T>
inline void put(std::string &out, T v) { put_be(out, &v, sizeof(T)); }
inline void put_vec(std::string &out, const Vec3 &v) {
    for (int a = 0; a < 3; ++a) put<double>(out, v[a]);
}
template <typename T>
inline T get(const std::string &in, size_t &p) {
    if (p + sizeof(T) > in.size()) throw std::runtime_error("Invalid body data chunk size.");
    T v;
    unsigned char *b = reinterpret_cast<unsigned char *>(&v);
    for (size_t k = 0; k < sizeof(T); ++k) b[sizeof(T) - 1 - k] = (unsigned char)in[p + k];
    p += sizeof(T);
    return v;
}
inline Vec3 get_vec(const std::string &in, size_t &p) {
    const double x = get<double>(in, p), y = get<double>(in, p), z = get<double>(in, p);
    return Vec3(x, y, z);
}
// Quaternion::toRotationMatrix, in pe's operation order (pe/math/Quaternion.h:591-602)
inline void rot_of(const real q[4], real R[9]) {
    R[0] = 1.0 - 2.0 * q[2] * q[2] - 2.0 * q[3] * q[3];
    R[1] = 2.0 * (q[1] * q[2] - q[0] * q[3]);
    R[2] = 2.0 * (q[1] * q[3] + q[0] * q[2]);
    R[3] = 2.0 * (q[1] * q[2] + q[0] * q[3]);
    R[4] = 1.0 - 2.0 * q[1] * q[1] - 2.0 * q[3] * q[3];
    R[5] = 2.0 * (q[2] * q[3] - q[0] * q[1]);
    R[6] = 2.0 * (q[1] * q[3] - q[0] * q[2]);
    R[7] = 2.0 * (q[2] * q[3] + q[0] * q[1]);
    R[8] = 1.0 - 2.0 * q[1] * q[1] - 2.0 * q[2] * q[2];
}
}  // namespace detail

inline void World::writeCheckpoint(const char *filename) const {
    using namespace detail;
    pull();
    auto rigid = [](std::string &out, const RigidBody &b, bool fixed, const Vec3 &x, const real q[4],
                    const Vec3 &v, const Vec3 &w) {
        put<uint64_t>(out, b.sid_);
        put<uint64_t>(out, b.uid_);
        put<uint8_t>(out, b.visible_ ? 1 : 0);
        put<uint8_t>(out, fixed ? 1 : 0);
        put_vec(out, x);
        for (int k = 0; k < 4; ++k) put<double>(out, q[k]);
        put_vec(out, v);
        put_vec(out, w);
        put<uint64_t>(out, b.mat_);
    };
    std::string glob, loc;
    put<uint64_t>(glob, 0);
    for (uint8_t t = 1; t <= 7; ++t) {
        put<uint8_t>(glob, t);
        put<uint32_t>(glob, 0);
    }
    put<uint64_t>(loc, next_sid_);
    const real ident[4] = {1, 0, 0, 0};
    for (uint8_t t : {1, 2, 3, 4, 6, 7}) {
        put<uint8_t>(loc, t);
        if (t == 1) {
            put<uint32_t>(loc, (uint32_t)spheres_.size());
            for (const auto &s : spheres_) {
                rigid(loc, *s, false, s->x_, ident, s->v_, s->w_);
                put<double>(loc, s->r_);
            }
        } else if (t == 2) {
            put<uint32_t>(loc, (uint32_t)boxes_.size());
            for (const auto &b : boxes_) {
                rigid(loc, *b, b->fixed_, b->x_, b->q_, b->fixed_ ? Vec3() : b->v_,
                      b->fixed_ ? Vec3() : b->w_);
                put_vec(loc, b->l_);
            }
        } else {
            put<uint32_t>(loc, 0);
        }
    }
    std::string head = std::string("PE") + std::string("\x00\x01\x08\x04\x08\x08\x01", 7);
    put<uint32_t>(head, 1);
    const uint32_t header_size = (uint32_t)head.size() + 3 * 4;
    const uint32_t offset = header_size + (uint32_t)glob.size();
    put<uint32_t>(head, header_size);
    put<uint32_t>(head, offset);
    put<uint32_t>(head, offset + (uint32_t)loc.size());
    std::ofstream f(filename, std::ios::binary);
    if (!f) throw std::runtime_error("Cannot open file.");
    f << head << glob << loc;
    if (!f) throw std::runtime_error("Cannot write file.");
}

inline void World::readCheckpoint(const char *filename) {
    using namespace detail;
    std::ifstream f(filename, std::ios::binary);
    if (!f) throw std::runtime_error("Cannot open file.");
    const std::string in((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    // the header checks of BodyBinaryReader.cpp:100-162
    if (in.size() < 25 || in[0] != 'P' || in[1] != 'E') throw std::runtime_error("Invalid file format.");
    if (in[2] != 0 || in[3] != 1) throw std::runtime_error("Unsupported file format version.");
    if (in[4] != 8) throw std::runtime_error("Invalid size of floating point data.");
    if (in[5] != 4 || in[6] != 8 || in[7] != 8 || in[8] != 1)
        throw std::runtime_error("Size of a data type does not match the data type used to produce the file.");
    size_t p = 9;
    if (get<uint32_t>(in, p) != 1)
        throw std::runtime_error("Number of processes differ from the number of processes used to produce the file.");
    const uint32_t goff = get<uint32_t>(in, p), loff = get<uint32_t>(in, p), lend = get<uint32_t>(in, p);
    if (loff < goff || lend < loff || lend > in.size()) throw std::runtime_error("Invalid body data offset.");
    clear();
    id_t counter = 0;
    auto chunk = [&](size_t q, size_t end) {
        const id_t c = (id_t)get<uint64_t>(in, q);
        while (q < end) {
            const uint8_t t = get<uint8_t>(in, q);
            const uint32_t cnt = get<uint32_t>(in, q);
            for (uint32_t k = 0; k < cnt; ++k) {
                const id_t sid = (id_t)get<uint64_t>(in, q), uid = (id_t)get<uint64_t>(in, q);
                const bool vis = get<uint8_t>(in, q) != 0, fixed = get<uint8_t>(in, q) != 0;
                const Vec3 x = get_vec(in, q);
                real qq[4];
                for (int a = 0; a < 4; ++a) qq[a] = get<double>(in, q);
                const Vec3 v = get_vec(in, q), w = get_vec(in, q);
                const MaterialID m = (MaterialID)get<uint64_t>(in, q);
                getMaterial(m);
                if (t == 1) {
                    const real r = get<double>(in, q);
                    spheres_.emplace_back(new Sphere(this, sid, uid, x, r, m, vis));
                    spheres_.back()->v_ = v;
                    spheres_.back()->w_ = w;
                } else if (t == 2) {
                    const Vec3 l = get_vec(in, q);
                    boxes_.emplace_back(new Box(this, sid, uid, x, l, m, vis));
                    Box &bx = *boxes_.back();
                    for (int a = 0; a < 4; ++a) bx.q_[a] = qq[a];
                    rot_of(qq, bx.R_);
                    bx.fixed_ = fixed;
                    bx.v_ = v;
                    bx.w_ = w;
                } else if (t == 5) {
                    real R[9];
                    rot_of(qq, R);
                    const Vec3 nrm(R[2], R[5], R[8]);
                    planes_.emplace_back(new Plane(this, sid, uid, nrm, nrm * x, m, vis));
                } else {
                    throw std::runtime_error("Unsupported geometry type in checkpoint.");
                }
            }
        }
        return c;
    };
    chunk(goff, loff);
    counter = chunk(loff, lend);
    // bodies in system-id order, as pe's storage holds them after creation
    auto by_sid = [](const auto &a, const auto &b) { return a->sid_ < b->sid_; };
    std::stable_sort(spheres_.begin(), spheres_.end(), by_sid);
    std::stable_sort(boxes_.begin(), boxes_.end(), by_sid);
    next_sid_ = counter;
    structure_dirty_ = true;
    host_stale_ = false;
}

/* theWorld() (pe/core/World.h:333) */
inline WorldID theWorld() { return &World::instance(); }
/* theCollisionSystem() */
inline CollisionSystem *theCollisionSystem() { return &World::instance().collisionSystem(); }

inline void markMaterialsChanged() { World::instance().markStructureDirty(); }

// ---- body creation (pe's free functions) -------------------------------------------------------
inline SphereID createSphere(id_t uid, const Vec3 &gpos, real radius, MaterialID material,
                             bool visible = true) {
    return World::instance().addSphere(uid, gpos, radius, material, visible);
}
inline SphereID createSphere(id_t uid, real x, real y, real z, real radius, MaterialID material,
                             bool visible = true) {
    return createSphere(uid, Vec3(x, y, z), radius, material, visible);
}
inline PlaneID createPlane(id_t uid, const Vec3 &normal, real d, MaterialID material,
                           bool visible = true) {
    return World::instance().addPlane(uid, normal, d, material, visible);
}
inline PlaneID createPlane(id_t uid, real a, real b, real c, real d, MaterialID material,
                           bool visible = true) {
    return createPlane(uid, Vec3(a, b, c), d, material, visible);
}
/* plane through gpos: d = normalised normal . gpos (Plane.cpp:1260-1320) */
inline PlaneID createPlane(id_t uid, const Vec3 &normal, const Vec3 &gpos, MaterialID material,
                           bool visible = true) {
    if (normal.sqrLength() == 0.0) throw std::invalid_argument("Invalid plane normal!");
    const Vec3 n = normal.getNormalized();
    return createPlane(uid, n, n * gpos, material, visible);
}
inline BoxID createBox(id_t uid, const Vec3 &gpos, const Vec3 &lengths, MaterialID material,
                       bool visible = true) {
    return World::instance().addBox(uid, gpos, lengths, material, visible);
}
inline BoxID createBox(id_t uid, real x, real y, real z, real lx, real ly, real lz,
                       MaterialID material, bool visible = true) {
    return createBox(uid, Vec3(x, y, z), Vec3(lx, ly, lz), material, visible);
}
inline void destroy(BodyID body) { World::instance().destroy(body); }

// ---- out-of-line members -----------------------------------------------------------------------
inline Vec3 Sphere::getPosition() const { world_->pull(); return x_; }
inline Vec3 Sphere::getLinearVel() const { world_->pull(); return v_; }
inline Vec3 Sphere::getAngularVel() const { world_->pull(); return w_; }
inline void Sphere::setPosition(real x, real y, real z) {
    world_->pull();
    x_ = Vec3(x, y, z);
    world_->markStateDirty();
}
inline void Sphere::setLinearVel(real x, real y, real z) {
    world_->pull();
    v_ = Vec3(x, y, z);
    world_->markStateDirty();
}
inline void Sphere::setAngularVel(real x, real y, real z) {
    world_->pull();
    w_ = Vec3(x, y, z);
    world_->markStateDirty();
}
inline void Box::setFixed(bool fixed) {
    world_->pull();
    fixed_ = fixed;
    if (fixed) v_ = w_ = Vec3();
    world_->markStructureDirty();
}
// a state change: a fixed box is part of the walls, a moving one of the box upload
inline void Box::changed() {
    if (fixed_) world_->markStructureDirty();
    else world_->markBoxesDirty();
}
inline Vec3 Box::getPosition() const { world_->pull(); return x_; }
inline const real *Box::getRotation() const { world_->pull(); return R_; }
inline std::array<real, 4> Box::getQuaternion() const {
    world_->pull();
    return {q_[0], q_[1], q_[2], q_[3]};
}
inline Vec3 Box::getLinearVel() const { world_->pull(); return v_; }
inline Vec3 Box::getAngularVel() const { world_->pull(); return w_; }
inline void Box::setPosition(real x, real y, real z) {
    world_->pull();
    x_ = Vec3(x, y, z);
    changed();
}
inline void Box::setLinearVel(real x, real y, real z) {
    world_->pull();
    if (!fixed_) v_ = Vec3(x, y, z);   // RigidBody::setLinearVel: no effect on fixed bodies
    changed();
}
inline void Box::setAngularVel(real x, real y, real z) {
    world_->pull();
    if (!fixed_) w_ = Vec3(x, y, z);
    changed();
}
inline void Box::setOrientation(real r, real i, real j, real k) {
    world_->pull();
    q_[0] = r; q_[1] = i; q_[2] = j; q_[3] = k;
    detail::rot_of(q_, R_);
    changed();
}
inline void Box::rotate(const Vec3 &axis, real angle) {
    if (axis.sqrLength() == 0.0) throw std::invalid_argument("Invalid rotation axis");
    world_->pull();
    // Quaternion(axis, angle) (pe/math/Quaternion.h:274-294) times q (Quaternion.h:1146-1153)
    real d[4] = {1.0, 0.0, 0.0, 0.0};
    if (!(std::fabs(angle) < 1e-15)) {
        const real sina = std::sin(angle * 0.5), cosa = std::cos(angle * 0.5);
        const Vec3 u = axis.getNormalized();
        d[0] = cosa; d[1] = sina * u[0]; d[2] = sina * u[1]; d[3] = sina * u[2];
    }
    const real *q = q_;
    const real r0 = d[0] * q[0] - d[1] * q[1] - d[2] * q[2] - d[3] * q[3];
    const real r1 = d[0] * q[1] + d[1] * q[0] + d[2] * q[3] - d[3] * q[2];
    const real r2 = d[0] * q[2] + d[2] * q[0] + d[3] * q[1] - d[1] * q[3];
    const real r3 = d[0] * q[3] + d[3] * q[0] + d[1] * q[2] - d[2] * q[1];
    q_[0] = r0; q_[1] = r1; q_[2] = r2; q_[3] = r3;
    detail::rot_of(q_, R_);
    changed();
}

inline void CollisionSystem::setMaxIterations(std::size_t n) {
    if (n > (std::size_t)INT32_MAX) throw std::invalid_argument("Invalid number of iterations");
    p_.max_iterations = (int32_t)n;
    if (world_->context()) world_->check(pe_b200_set_max_iterations(world_->context(), p_.max_iterations));
}
inline void CollisionSystem::setRelaxationModel(RelaxationModel m) {
    model_ = m;
    p_.relaxation_model = (int32_t)m;
    if (world_->context())
        world_->check(pe_b200_set_relaxation_model(world_->context(), p_.relaxation_model));
}
inline void CollisionSystem::setErrorReductionParameter(real erp) {
    p_.erp = erp;
    if (world_->context()) world_->check(pe_b200_set_error_reduction(world_->context(), erp));
}
inline void CollisionSystem::setSolver(int solver) {
    if (solver != PE_B200_DEM && solver != PE_B200_HCSITS) throw std::invalid_argument("Invalid solver");
    p_.solver = solver;
    world_->markParamsDirty();
}
inline void CollisionSystem::setPrecision(int prec) {
    if (prec != PE_B200_FP64 && prec != PE_B200_MIXED) throw std::invalid_argument("Invalid precision");
    p_.precision = prec;
    world_->markParamsDirty();
}
inline void CollisionSystem::setForceModel(int model) {
    if (model != 0 && model != 1) throw std::invalid_argument("Invalid force model");
    p_.force_model = model;
    world_->markParamsDirty();
}
inline void CollisionSystem::setDevice(int device) {
    p_.device = device;
    world_->markParamsDirty();
}
inline void CollisionSystem::lastStepStats(int64_t *ncontacts, int32_t *ncolors) const {
    double dm, res;
    if (!world_->context()) {
        *ncontacts = 0;
        *ncolors = 0;
        return;
    }
    world_->check(pe_b200_last_step_stats(world_->context(), ncontacts, ncolors, &dm, &res));
}

}  // namespace pe_b200

#endif  // PE_B200_WORLD_HPP
