// ref_driver.cpp -- drives the compiled pe reference through its own public API.
//
// TEST INFRASTRUCTURE ONLY (oracle).  Built twice by oracle/ref/Makefile from pe's own,
// unmodified sources: once with pe_CONSTRAINT_SOLVER = response::DEMSolver (linear force law
// via the DEMConfig overlay) and once with HardContactSemiImplicitTimesteppingSolvers.
//
// Usage:
//   ref_<solver> step  <scene> <steps> <out.bin> [model] [max_iter]
//       runs <steps> World::simulationStep calls; writes x, v, w (3n doubles each), q (4n),
//       then for the moving boxes x, v, w (3M each) and q (4M)
//   ref_<solver> pairs <scene> <out.bin>
//       runs pe's coarse+fine detection once and writes the contacts in pe's detection order:
//       int64 count, then per contact b1, b2 (int64 user ids), gpos[3], normal[3], dist
//   ref_<solver> time  <scene> <warmup> <steps> [model] [max_iter]
//       times <steps> steps after <warmup> untimed steps, prints one JSON line
//
// Body user ids: spheres 0..n-1 (created first, in order, so pe's system-id order is the index
// order), planes n..n+P-1, fixed boxes n+P..n+P+B-1, moving boxes n+P+B..n+P+B+M-1.  Scene file
// layout: pe_b200/scenes.py.
#include <pe/core.h>

#include <chrono>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

using namespace pe;

namespace {

struct SceneFile {
    uint32_t nmat = 0, nplanes = 0, nboxes = 0;
    uint64_t n = 0;
    double g[3] = {0, 0, 0}, dt = 0, damping = 1;
    uint32_t steps = 0;
    std::vector<double> mats, planes, boxes, x, v, w, r;
    std::vector<int32_t> plane_mat, box_mat, mat;
    // scene version 2: moving boxes (created after the fixed boxes)
    uint32_t nmb = 0;
    std::vector<double> mb_x, mb_q, mb_v, mb_w, mb_len;
    std::vector<int32_t> mb_mat;
};

template <typename T>
void rd(std::ifstream& f, T* p, size_t count) {
    f.read(reinterpret_cast<char*>(p), static_cast<std::streamsize>(count * sizeof(T)));
    if (!f) throw std::runtime_error("truncated scene file");
}

SceneFile load(const char* path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open scene file");
    char magic[8];
    uint32_t ver;
    SceneFile s;
    rd(f, magic, 8);
    if (std::memcmp(magic, "PEB2SCN", 8) != 0) throw std::runtime_error("bad scene magic");
    rd(f, &ver, 1);
    rd(f, &s.nmat, 1);
    rd(f, &s.n, 1);
    rd(f, &s.nplanes, 1);
    rd(f, &s.nboxes, 1);
    rd(f, s.g, 3);
    rd(f, &s.dt, 1);
    rd(f, &s.damping, 1);
    rd(f, &s.steps, 1);
    s.mats.resize(9 * s.nmat);            rd(f, s.mats.data(), s.mats.size());
    s.planes.resize(4 * s.nplanes);       rd(f, s.planes.data(), s.planes.size());
    s.plane_mat.resize(s.nplanes);        rd(f, s.plane_mat.data(), s.plane_mat.size());
    s.boxes.resize(15 * s.nboxes);        rd(f, s.boxes.data(), s.boxes.size());
    s.box_mat.resize(s.nboxes);           rd(f, s.box_mat.data(), s.box_mat.size());
    s.x.resize(3 * s.n);                  rd(f, s.x.data(), s.x.size());
    s.v.resize(3 * s.n);                  rd(f, s.v.data(), s.v.size());
    s.w.resize(3 * s.n);                  rd(f, s.w.data(), s.w.size());
    s.r.resize(s.n);                      rd(f, s.r.data(), s.r.size());
    s.mat.resize(s.n);                    rd(f, s.mat.data(), s.mat.size());
    if (ver >= 2) {
        rd(f, &s.nmb, 1);
        s.mb_x.resize(3 * s.nmb);         rd(f, s.mb_x.data(), s.mb_x.size());
        s.mb_q.resize(4 * s.nmb);         rd(f, s.mb_q.data(), s.mb_q.size());
        s.mb_v.resize(3 * s.nmb);         rd(f, s.mb_v.data(), s.mb_v.size());
        s.mb_w.resize(3 * s.nmb);         rd(f, s.mb_w.data(), s.mb_w.size());
        s.mb_len.resize(3 * s.nmb);       rd(f, s.mb_len.data(), s.mb_len.size());
        s.mb_mat.resize(s.nmb);           rd(f, s.mb_mat.data(), s.mb_mat.size());
    }
    return s;
}

std::vector<BoxID> g_mboxes;   // the moving boxes of the loaded scene, in scene order

std::vector<SphereID> build_world(const SceneFile& s) {
    WorldID world = theWorld();
    world->setGravity(s.g[0], s.g[1], s.g[2]);
    world->setDamping(s.damping);
    std::vector<MaterialID> mids;
    for (uint32_t m = 0; m < s.nmat; ++m) {
        const double* a = &s.mats[9 * m];
        std::ostringstream name;
        name << "scene_material_" << m;
        mids.push_back(createMaterial(name.str(), a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7],
                                      a[8]));
    }
    std::vector<SphereID> spheres;
    spheres.reserve(s.n);
    for (uint64_t i = 0; i < s.n; ++i) {
        SphereID sp = createSphere(static_cast<pe::id_t>(i),
                                   Vec3(s.x[3 * i], s.x[3 * i + 1], s.x[3 * i + 2]), s.r[i],
                                   mids[s.mat[i]]);
        sp->setLinearVel(s.v[3 * i], s.v[3 * i + 1], s.v[3 * i + 2]);
        sp->setAngularVel(s.w[3 * i], s.w[3 * i + 1], s.w[3 * i + 2]);
        spheres.push_back(sp);
    }
    for (uint32_t p = 0; p < s.nplanes; ++p) {
        const double* a = &s.planes[4 * p];
        createPlane(static_cast<pe::id_t>(s.n + p), Vec3(a[0], a[1], a[2]), a[3],
                    mids[s.plane_mat[p]]);
    }
    for (uint32_t b = 0; b < s.nboxes; ++b) {
        const double* a = &s.boxes[15 * b];
        for (int k = 0; k < 9; ++k)
            if (a[6 + k] != ((k % 4 == 0) ? 1.0 : 0.0))
                throw std::runtime_error("the driver supports axis-aligned boxes only");
        BoxID box = createBox(static_cast<pe::id_t>(s.n + s.nplanes + b), Vec3(a[0], a[1], a[2]),
                              Vec3(a[3], a[4], a[5]), mids[s.box_mat[b]]);
        box->setFixed(true);
    }
    g_mboxes.clear();
    for (uint32_t m = 0; m < s.nmb; ++m) {
        const double *x = &s.mb_x[3 * m], *q = &s.mb_q[4 * m], *l = &s.mb_len[3 * m];
        BoxID box = createBox(static_cast<pe::id_t>(s.n + s.nplanes + s.nboxes + m),
                              Vec3(x[0], x[1], x[2]), Vec3(l[0], l[1], l[2]), mids[s.mb_mat[m]]);
        box->setOrientation(Quat(q[0], q[1], q[2], q[3]));
        box->setLinearVel(s.mb_v[3 * m], s.mb_v[3 * m + 1], s.mb_v[3 * m + 2]);
        box->setAngularVel(s.mb_w[3 * m], s.mb_w[3 * m + 1], s.mb_w[3 * m + 2]);
        g_mboxes.push_back(box);
    }
    return spheres;
}

void configure_solver(int argc, char** argv, int first) {
#if defined(PE_REF_HCSITS)
    int model = argc > first ? std::atoi(argv[first]) : 0;
    int maxit = argc > first + 1 ? std::atoi(argv[first + 1]) : 100;
    typedef CollisionSystem<Config> CS;
    // pe's RelaxationModel values 0-5 (HardContactSemiImplicitTimesteppingSolvers.h:172-179)
    theCollisionSystem()->setRelaxationModel(static_cast<typename CS::RelaxationModel>(model));
    theCollisionSystem()->setMaxIterations(static_cast<size_t>(maxit));
#else
    (void)argc; (void)argv; (void)first;
#endif
}

void write_state(const char* path, const std::vector<SphereID>& sp) {
    std::ofstream f(path, std::ios::binary);
    std::vector<double> out;
    out.reserve(sp.size() * 13);
    for (size_t i = 0; i < sp.size(); ++i) { const Vec3& a = sp[i]->getPosition(); out.push_back(a[0]); out.push_back(a[1]); out.push_back(a[2]); }
    for (size_t i = 0; i < sp.size(); ++i) { const Vec3& a = sp[i]->getLinearVel(); out.push_back(a[0]); out.push_back(a[1]); out.push_back(a[2]); }
    for (size_t i = 0; i < sp.size(); ++i) { const Vec3& a = sp[i]->getAngularVel(); out.push_back(a[0]); out.push_back(a[1]); out.push_back(a[2]); }
    for (size_t i = 0; i < sp.size(); ++i) { const Quat& q = sp[i]->getQuaternion(); for (int k = 0; k < 4; ++k) out.push_back(q[k]); }
    // moving boxes: x, v, w (3 each per box), then q (4 per box)
    const std::vector<BoxID>& mb = g_mboxes;
    for (size_t i = 0; i < mb.size(); ++i) { const Vec3& a = mb[i]->getPosition(); out.push_back(a[0]); out.push_back(a[1]); out.push_back(a[2]); }
    for (size_t i = 0; i < mb.size(); ++i) { const Vec3& a = mb[i]->getLinearVel(); out.push_back(a[0]); out.push_back(a[1]); out.push_back(a[2]); }
    for (size_t i = 0; i < mb.size(); ++i) { const Vec3& a = mb[i]->getAngularVel(); out.push_back(a[0]); out.push_back(a[1]); out.push_back(a[2]); }
    for (size_t i = 0; i < mb.size(); ++i) { const Quat& q = mb[i]->getQuaternion(); for (int k = 0; k < 4; ++k) out.push_back(q[k]); }
    f.write(reinterpret_cast<const char*>(out.data()),
            static_cast<std::streamsize>(out.size() * sizeof(double)));
}

void write_pairs(const char* path) {
    typedef CollisionSystem<Config> CS;
    CS::Contacts contacts;
    theCollisionSystem()->getCoarseDetector().findContacts(contacts);
    std::ofstream f(path, std::ios::binary);
    const int64_t nc = static_cast<int64_t>(contacts.size());
    f.write(reinterpret_cast<const char*>(&nc), sizeof nc);
    for (CS::Contacts::Iterator c = contacts.begin(); c != contacts.end(); ++c) {
        int64_t ids[2] = {static_cast<int64_t>(c->getBody1()->getID()),
                          static_cast<int64_t>(c->getBody2()->getID())};
        double rec[7];
        const Vec3& g = c->getPosition();
        const Vec3& n = c->getNormal();
        rec[0] = g[0]; rec[1] = g[1]; rec[2] = g[2];
        rec[3] = n[0]; rec[4] = n[1]; rec[5] = n[2];
        rec[6] = c->getDistance();
        f.write(reinterpret_cast<const char*>(ids), sizeof ids);
        f.write(reinterpret_cast<const char*>(rec), sizeof rec);
    }
}

}  // namespace

int main(int argc, char** argv) {
    try {
        if (argc < 3) {
            std::cerr << "usage: step|pairs|time <scene> ...\n";
            return 2;
        }
        const std::string mode(argv[1]);
        SceneFile s = load(argv[2]);
        std::vector<SphereID> sp = build_world(s);
        WorldID world = theWorld();
        if (mode == "step" && argc >= 5) {
            configure_solver(argc, argv, 5);
            const int steps = std::atoi(argv[3]);
            for (int k = 0; k < steps; ++k) world->simulationStep(s.dt);
            write_state(argv[4], sp);
        } else if (mode == "peb_write" && argc >= 5) {
            // pe's own checkpoint writer (src/core/BodyBinaryWriter.cpp) after `steps` steps
            const int steps = std::atoi(argv[3]);
            for (int k = 0; k < steps; ++k) world->simulationStep(s.dt);
            BodyBinaryWriter writer;
            writer.writeFile(argv[4]);
        } else if (mode == "peb_read" && argc >= 6) {
            // pe's own checkpoint reader (src/core/BodyBinaryReader.cpp): it replaces every body
            // of the world by the file's; the scene's planes (which pe does not write unless
            // global) are created again, then `steps` steps run and the spheres' state is written
            BodyBinaryReader reader;
            reader.readFile(argv[3]);
            std::vector<MaterialID> mids;
            for (uint32_t m = 0; m < s.nmat; ++m) mids.push_back(static_cast<MaterialID>(5 + m));
            for (uint32_t p = 0; p < s.nplanes; ++p) {
                const double* a = &s.planes[4 * p];
                createPlane(static_cast<pe::id_t>(s.n + p), Vec3(a[0], a[1], a[2]), a[3],
                            mids[s.plane_mat[p]]);
            }
            std::vector<SphereID> read;
            for (World::Bodies::CastIterator<Sphere> it = world->begin<Sphere>();
                 it != world->end<Sphere>(); ++it)
                read.push_back(*it);
            g_mboxes.clear();
            for (World::Bodies::CastIterator<Box> it = world->begin<Box>();
                 it != world->end<Box>(); ++it)
                if (!(*it)->isFixed()) g_mboxes.push_back(*it);
            const int steps = std::atoi(argv[4]);
            for (int k = 0; k < steps; ++k) world->simulationStep(s.dt);
            write_state(argv[5], read);
        } else if (mode == "pairs" && argc >= 4) {
            write_pairs(argv[3]);
        } else if (mode == "time" && argc >= 5) {
            configure_solver(argc, argv, 5);
            const int warm = std::atoi(argv[3]), steps = std::atoi(argv[4]);
            for (int k = 0; k < warm; ++k) world->simulationStep(s.dt);
            const auto t0 = std::chrono::steady_clock::now();
            for (int k = 0; k < steps; ++k) world->simulationStep(s.dt);
            const auto t1 = std::chrono::steady_clock::now();
            const double sec = std::chrono::duration<double>(t1 - t0).count();
            std::printf("{\"spheres\": %llu, \"steps\": %d, \"seconds\": %.9g, "
                        "\"sphere_steps_per_s\": %.9g}\n",
                        static_cast<unsigned long long>(s.n), steps, sec,
                        static_cast<double>(s.n) * steps / sec);
        } else {
            std::cerr << "bad arguments\n";
            return 2;
        }
    } catch (std::exception& e) {
        std::cerr << "ref_driver error: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
