// Test driver of include/pe_b200_world.hpp: a program written against pe's World and
// body-creation API.
//
//   world_driver errors                      argument checks, no GPU needed; prints "ok"
//   world_driver run <scene> <dem|hcsits> <fp64|mixed> <steps> <out>
//       builds the scene of a scene file (pe_b200.scenes binary format) with createMaterial /
//       createPlane / createBox / createSphere, runs `steps` time steps in two calls (reading
//       the positions in between, as a user would) and writes the final x, v, w (3n doubles each)
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <vector>

#include "pe_b200_world.hpp"

namespace pe = pe_b200;

static int expect_throw(const char *what, const std::function<void()> &f, bool invalid_arg) {
    try {
        f();
    } catch (const std::invalid_argument &) {
        if (invalid_arg) return 0;
        std::fprintf(stderr, "%s: std::invalid_argument, expected std::runtime_error\n", what);
        return 1;
    } catch (const std::runtime_error &) {
        if (!invalid_arg) return 0;
        std::fprintf(stderr, "%s: std::runtime_error, expected std::invalid_argument\n", what);
        return 1;
    }
    std::fprintf(stderr, "%s: no exception\n", what);
    return 1;
}

static int errors() {
    using namespace pe;
    int bad = 0;
    WorldID world = theWorld();
    bad += expect_throw("duplicate material", [] { createMaterial("iron", 1, 0, 0.1, 0.1, 0.2, 1, 1, 0, 0); }, true);
    bad += expect_throw("density", [] { createMaterial("m1", 0.0, 0, 0.1, 0.1, 0.2, 1, 1, 0, 0); }, true);
    bad += expect_throw("restitution", [] { createMaterial("m2", 1.0, 1.5, 0.1, 0.1, 0.2, 1, 1, 0, 0); }, true);
    bad += expect_throw("poisson", [] { createMaterial("m3", 1.0, 0.5, 0.1, 0.1, 0.7, 1, 1, 0, 0); }, true);
    bad += expect_throw("stiffness", [] { createMaterial("m4", 1.0, 0.5, 0.1, 0.1, 0.2, 1, 0, 0, 0); }, true);
    bad += expect_throw("damping", [] { createMaterial("m5", 1.0, 0.5, 0.1, 0.1, 0.2, 1, 1, -1, 0); }, true);
    const MaterialID a = createMaterial(1.0, 0.0, 0.15, 0.15, 0.25, 1e9, 2e5, 100, 80);
    if (getMaterial(a).getName() != "Material1" || a != 5) {
        std::fprintf(stderr, "anonymous material: %s id %zu\n", getMaterial(a).getName().c_str(), a);
        ++bad;
    }
    if (findMaterial("granite") != granite || findMaterial("none") != invalid_material) ++bad;
    bad += expect_throw("radius", [a] { createSphere(1, 0, 0, 0, 0.0, a); }, true);
    bad += expect_throw("material id", [] { createSphere(1, 0, 0, 0, 1.0, 99); }, true);
    bad += expect_throw("plane normal", [a] { createPlane(2, 0, 0, 0, 1.0, a); }, true);
    bad += expect_throw("box sides", [a] { createBox(3, 0, 0, 0, 1.0, 0.0, 1.0, a); }, true);
    bad += expect_throw("time step", [world] { world->simulationStep(0.0); }, true);
    bad += expect_throw("damping factor", [world] { world->setDamping(1.5); }, true);
    // createPlane normalises the normal and keeps d (Plane.cpp:1218-1223)
    PlaneID p = createPlane(4, 0.0, 0.0, 2.0, 3.0, a);
    if (p->getNormal()[2] != 1.0 || p->getDisplacement() != 3.0) ++bad;
    PlaneID q = createPlane(5, Vec3(0, 2, 0), Vec3(7, 4, 1), a);
    if (q->getNormal()[1] != 1.0 || q->getDisplacement() != 4.0) ++bad;
    SphereID s = createSphere(6, 1.0, 2.0, 3.0, 0.5, a);
    s->setLinearVel(1.0, 0.0, 0.0);
    if (s->getLinearVel()[0] != 1.0 || s->getPosition()[2] != 3.0 || s->getSystemID() != 2) ++bad;
    if (world->size() != 3) ++bad;
    destroy(q);
    if (world->size() != 2 || world->numPlanes() != 1) ++bad;
    world->clear();
    std::printf(bad ? "failed %d\n" : "ok\n", bad);
    return bad ? 1 : 0;
}

struct SceneFile {
    std::vector<double> mats, planes, boxes, x, v, w, r;
    std::vector<int32_t> plane_mat, box_mat, mat;
    double g[3], dt, damping;
    uint64_t n;
    // scene version 2: moving boxes
    uint32_t nmb = 0;
    std::vector<double> mb_x, mb_q, mb_v, mb_w, mb_len;
    std::vector<int32_t> mb_mat;
};

static bool read_scene(const char *path, SceneFile &s) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    char magic[8];
    uint32_t ver, nm, npl, nbx, steps;
    f.read(magic, 8);
    f.read((char *)&ver, 4);
    f.read((char *)&nm, 4);
    f.read((char *)&s.n, 8);
    f.read((char *)&npl, 4);
    f.read((char *)&nbx, 4);
    f.read((char *)s.g, 24);
    f.read((char *)&s.dt, 8);
    f.read((char *)&s.damping, 8);
    f.read((char *)&steps, 4);
    auto rd = [&f](auto &vec, size_t count) {
        vec.resize(count);
        f.read((char *)vec.data(), count * sizeof(vec[0]));
    };
    rd(s.mats, 9 * (size_t)nm);
    rd(s.planes, 4 * (size_t)npl);
    rd(s.plane_mat, npl);
    rd(s.boxes, 15 * (size_t)nbx);
    rd(s.box_mat, nbx);
    rd(s.x, 3 * s.n);
    rd(s.v, 3 * s.n);
    rd(s.w, 3 * s.n);
    rd(s.r, s.n);
    rd(s.mat, s.n);
    if (ver >= 2) {
        f.read((char *)&s.nmb, 4);
        rd(s.mb_x, 3 * (size_t)s.nmb);
        rd(s.mb_q, 4 * (size_t)s.nmb);
        rd(s.mb_v, 3 * (size_t)s.nmb);
        rd(s.mb_w, 3 * (size_t)s.nmb);
        rd(s.mb_len, 3 * (size_t)s.nmb);
        rd(s.mb_mat, s.nmb);
    }
    return (bool)f;
}

static int run(const char *scene, const char *solver, const char *prec, int steps, const char *out) {
    using namespace pe;
    SceneFile sf;
    if (!read_scene(scene, sf)) {
        std::fprintf(stderr, "cannot read %s\n", scene);
        return 2;
    }
    WorldID world = theWorld();
    CollisionSystem *cs = theCollisionSystem();
    cs->setSolver(std::strcmp(solver, "hcsits") == 0 ? PE_B200_HCSITS : PE_B200_DEM);
    cs->setPrecision(std::strcmp(prec, "mixed") == 0 ? PE_B200_MIXED : PE_B200_FP64);
    cs->setRelaxationModel(CollisionSystem::ApproximateInelasticCoulombContactByDecoupling);
    cs->setMaxIterations(100);
    world->setGravity(sf.g[0], sf.g[1], sf.g[2]);
    world->setDamping(sf.damping);
    std::vector<MaterialID> mid;
    for (size_t k = 0; k < sf.mats.size() / 9; ++k) {
        const double *m = &sf.mats[9 * k];
        mid.push_back(createMaterial(m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8]));
    }
    pe::id_t uid = 1000;
    for (size_t k = 0; k < sf.plane_mat.size(); ++k) {
        const double *p = &sf.planes[4 * k];
        createPlane(uid++, p[0], p[1], p[2], p[3], mid[sf.plane_mat[k]]);
    }
    for (size_t k = 0; k < sf.box_mat.size(); ++k) {
        const double *b = &sf.boxes[15 * k];
        BoxID box = createBox(uid++, b[0], b[1], b[2], b[3], b[4], b[5], mid[sf.box_mat[k]]);
        for (int e = 0; e < 9; ++e)
            if (b[6 + e] != (e % 4 == 0 ? 1.0 : 0.0)) {
                std::fprintf(stderr, "the driver takes axis-aligned boxes only\n");
                return 2;
            }
        box->setFixed(true);
    }
    std::vector<BoxID> moving;
    for (uint32_t k = 0; k < sf.nmb; ++k) {
        const double *x = &sf.mb_x[3 * k], *q = &sf.mb_q[4 * k], *l = &sf.mb_len[3 * k];
        BoxID box = createBox(uid++, x[0], x[1], x[2], l[0], l[1], l[2], mid[sf.mb_mat[k]]);
        box->setOrientation(q[0], q[1], q[2], q[3]);
        box->setLinearVel(sf.mb_v[3 * k], sf.mb_v[3 * k + 1], sf.mb_v[3 * k + 2]);
        box->setAngularVel(sf.mb_w[3 * k], sf.mb_w[3 * k + 1], sf.mb_w[3 * k + 2]);
        moving.push_back(box);
    }
    std::vector<SphereID> spheres;
    for (uint64_t i = 0; i < sf.n; ++i) {
        SphereID s = createSphere(uid++, sf.x[3 * i], sf.x[3 * i + 1], sf.x[3 * i + 2], sf.r[i],
                                  mid[sf.mat[i]]);
        s->setLinearVel(sf.v[3 * i], sf.v[3 * i + 1], sf.v[3 * i + 2]);
        s->setAngularVel(sf.w[3 * i], sf.w[3 * i + 1], sf.w[3 * i + 2]);
        spheres.push_back(s);
    }
    const int first = steps / 2;
    try {
        world->run(first, sf.dt);
        double zsum = 0.0;
        for (SphereID s : spheres) zsum += s->getPosition()[2];
        for (BoxID b : moving) zsum += b->getPosition()[2];
        std::printf("mean z after %d steps: %.17g\n", first,
                    zsum / (double)std::max<size_t>(1, sf.n + sf.nmb));
        for (int k = first; k < steps; ++k) world->simulationStep(sf.dt);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "step failed: %s\n", e.what());
        return 3;
    }
    std::vector<double> res;
    for (int f = 0; f < 3; ++f)
        for (SphereID s : spheres) {
            const Vec3 a = f == 0 ? s->getPosition() : f == 1 ? s->getLinearVel() : s->getAngularVel();
            res.insert(res.end(), {a[0], a[1], a[2]});
        }
    // moving boxes: x, v, w (3 per box each), q (4 per box)
    for (int f = 0; f < 3; ++f)
        for (BoxID b : moving) {
            const Vec3 a = f == 0 ? b->getPosition() : f == 1 ? b->getLinearVel() : b->getAngularVel();
            res.insert(res.end(), {a[0], a[1], a[2]});
        }
    for (BoxID b : moving) {
        const std::array<double, 4> q = b->getQuaternion();
        res.insert(res.end(), q.begin(), q.end());
    }
    std::ofstream o(out, std::ios::binary);
    o.write((const char *)res.data(), res.size() * sizeof(double));
    std::printf("ok\n");
    return o ? 0 : 4;
}

// the compiled reference's body creation order: spheres (user id = index), planes, boxes
static void build_like_reference(const SceneFile &sf) {
    using namespace pe;
    std::vector<MaterialID> mid;
    for (size_t k = 0; k < sf.mats.size() / 9; ++k) {
        const double *m = &sf.mats[9 * k];
        mid.push_back(createMaterial("scene_material_" + std::to_string(k), m[0], m[1], m[2], m[3],
                                     m[4], m[5], m[6], m[7], m[8]));
    }
    for (uint64_t i = 0; i < sf.n; ++i) {
        SphereID s = createSphere(i, sf.x[3 * i], sf.x[3 * i + 1], sf.x[3 * i + 2], sf.r[i],
                                  mid[sf.mat[i]]);
        s->setLinearVel(sf.v[3 * i], sf.v[3 * i + 1], sf.v[3 * i + 2]);
        s->setAngularVel(sf.w[3 * i], sf.w[3 * i + 1], sf.w[3 * i + 2]);
    }
    const size_t np = sf.plane_mat.size();
    for (size_t k = 0; k < np; ++k) {
        const double *p = &sf.planes[4 * k];
        createPlane(sf.n + k, Vec3(p[0], p[1], p[2]), p[3], mid[sf.plane_mat[k]]);
    }
    for (size_t k = 0; k < sf.box_mat.size(); ++k) {
        const double *b = &sf.boxes[15 * k];
        createBox(sf.n + np + k, Vec3(b[0], b[1], b[2]), Vec3(b[3], b[4], b[5]), mid[sf.box_mat[k]])
            ->setFixed(true);
    }
}

// peb_write <scene> <out.peb>: the scene's bodies as pe's checkpoint writer would store them
static int peb_write(const char *scene, const char *out) {
    SceneFile sf;
    if (!read_scene(scene, sf)) return 2;
    build_like_reference(sf);
    pe::BodyBinaryWriter().writeFile(out);
    std::printf("ok\n");
    return 0;
}

// peb_resume <scene> <in.peb> <steps> <out>: the scene's materials, the checkpoint's bodies, the
// scene's planes again (pe writes only global planes), then `steps` FP64 DEM steps on the GPU
static int peb_resume(const char *scene, const char *in, int steps, const char *out) {
    using namespace pe;
    SceneFile sf;
    if (!read_scene(scene, sf)) return 2;
    build_like_reference(sf);
    BodyBinaryReader().readFile(in);
    for (size_t k = 0; k < sf.plane_mat.size(); ++k) {
        const double *p = &sf.planes[4 * k];
        createPlane(sf.n + k, Vec3(p[0], p[1], p[2]), p[3], 5 + sf.plane_mat[k]);
    }
    WorldID world = theWorld();
    world->setGravity(sf.g[0], sf.g[1], sf.g[2]);
    world->setDamping(sf.damping);
    theCollisionSystem()->setSolver(PE_B200_DEM);
    theCollisionSystem()->setPrecision(PE_B200_FP64);
    try {
        world->run(steps, sf.dt);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "step failed: %s\n", e.what());
        return 3;
    }
    std::vector<double> res;
    for (int f = 0; f < 3; ++f)
        for (size_t i = 0; i < world->numSpheres(); ++i) {
            SphereID s = world->sphere(i);
            const Vec3 a = f == 0 ? s->getPosition() : f == 1 ? s->getLinearVel() : s->getAngularVel();
            res.insert(res.end(), {a[0], a[1], a[2]});
        }
    std::ofstream o(out, std::ios::binary);
    o.write((const char *)res.data(), res.size() * sizeof(double));
    std::printf("ok\n");
    return o ? 0 : 4;
}

int main(int argc, char **argv) {
    if (argc == 4 && std::strcmp(argv[1], "peb_write") == 0) return peb_write(argv[2], argv[3]);
    if (argc == 6 && std::strcmp(argv[1], "peb_resume") == 0)
        return peb_resume(argv[2], argv[3], std::atoi(argv[4]), argv[5]);
    if (argc >= 2 && std::strcmp(argv[1], "errors") == 0) return errors();
    if (argc == 7 && std::strcmp(argv[1], "run") == 0)
        return run(argv[2], argv[3], argv[4], std::atoi(argv[5]), argv[6]);
    std::fprintf(stderr, "usage: world_driver errors | run <scene> <dem|hcsits> <fp64|mixed> <steps> <out>\n");
    return 2;
}
