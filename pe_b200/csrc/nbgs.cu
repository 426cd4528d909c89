// nbgs.cu -- hard-contact step (pe's HardContactSemiImplicitTimesteppingSolvers, "HCSITS") and
// the explicit contact list behind pe_b200_find_contacts.
//
// Step (HCSITS.h:1472-2019), one sorted pass per stage:
//   permute + body cache    state to cell-sorted slot order; v' = v + g dt,
//                           w' = w + dt I^-1 ((I w) x w), dv = dw = 0 (HCSITS.h:1834-1880, 4094-4110)
//   detect                  per-body count, exclusive scan, write (deterministic order)
//   colour                  body-conflict-free edge colouring of the contact graph: rounds of
//                           speculative greedy colouring (propose the smallest colour free at
//                           both bodies, keep the highest-priority proposal of every clash;
//                           walls never conflict: infinite mass)
//   contact cache           frame n,t,o; ERP-scaled distance; Delassus block D, D^-1, 1/D_nn,
//                           (D_to)^-1 (HCSITS.h:1741-1820), stored in colour-sorted order
//   sweeps                  max_iterations x colours: each colour is a conflict-free parallel
//                           Gauss-Seidel sweep (relaxInelasticFrictionlessContacts :2039-2105,
//                           relaxApproximateInelasticCoulombContactsByDecoupling :2129-2304)
//   integrate               x += (v'+dv) dt, quaternion, drag, store v, w (HCSITS.h:4135-4190)
// Colour order replaces pe's detection order; only converged frictionless velocities are
// order-independent, which is what the parity tests compare.
#include <algorithm>
#include <type_traits>
#include <vector>

#include <cooperative_groups.h>

#include "contacts.cuh"

namespace peb {

namespace {

constexpr int kBlk = 256;
constexpr int kMaxColors = 256;   // colours of one step (8 bits in the packed colour)
constexpr size_t kBlockSmemMax = 200 * 1024;   // shared memory of the single-block sweep form
// contacts coloured by one thread in one launch: scenes with moving boxes (where it saves many
// colours), and sphere scenes with the bodies' colour masks in shared memory or in global memory
// (every contact's mask update is then an L2 round trip)
constexpr int64_t kSerialColourMax = 8192;
constexpr int64_t kSerialColourMaxSpheres = 512;
constexpr int64_t kSerialColourMaxGlobal = 128;
constexpr int kMaxRounds = 4096;                // rounds of the parallel colouring
// device counters of a step (NbgsBuf.dd)
enum : int {
    kDdAbort = 0,    // the contacts exceeded the capacity: the rest of the call does nothing
    kDdNeed = 1,     // the largest contact count seen
    kDdNcolors = 2,  // colours of the step
    kDdMaxcol = 3,   // contacts of the largest colour
    kDdSteps = 4,    // steps completed (not aborted) since the host reset it
    kDdNc = 5,       // contact count written by the host (scenes with moving boxes)
    kDdSink = 6,     // error bits nobody reads (a capacity overflow that aborts instead)
    kDdSeen = 7,     // the largest contact count of the call's steps (reset per call)
    kDdRounds = 8,   // the step colours by the parallel rounds (more contacts than one thread takes)
    kDdCount = 10
};

struct CountF {
    int n = 0;
    __device__ void operator()(const ContactGeom &) { ++n; }
};

// --------------------------------------------------------------------------------------------
// contact list for pe_b200_find_contacts (uses the sort of the current state, no permutation)
// --------------------------------------------------------------------------------------------
__global__ void k_count(int64_t n, VisitArgs a, int32_t *cnt) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    CountF f;
    visit_contacts(a, a.sorted ? a.sorted[t] : (int32_t)t, f);
    cnt[t] = f.n;
}

struct ListF {
    int64_t pos;
    int64_t cap;
    int64_t n_total;
    int32_t uid_self;
    int64_t *ids;
    double *geom;
    const int32_t *uid;
    __device__ void operator()(const ContactGeom &g) {
        if (pos < cap) {
            ids[2 * pos] = uid_self;
            ids[2 * pos + 1] = g.other >= 0 ? (int64_t)uid[g.other] : n_total + g.wall;
            double *o = geom + 7 * pos;
            o[0] = g.gx; o[1] = g.gy; o[2] = g.gz;
            o[3] = g.nx; o[4] = g.ny; o[5] = g.nz;
            o[6] = g.dist;
        }
        ++pos;
    }
};

__global__ void k_list(int64_t n, VisitArgs a, const int32_t *off, int64_t cap, int64_t *ids,
                       double *geom) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int32_t b = a.sorted ? a.sorted[t] : (int32_t)t;
    ListF f;
    f.pos = off[t];
    f.cap = cap;
    f.n_total = n;
    f.uid_self = a.uid[b];
    f.ids = ids;
    f.geom = geom;
    f.uid = a.uid;
    visit_contacts(a, b, f);
}

VisitArgs visit_args(Ctx *c, const int32_t *sorted) {
    VisitArgs a;
    a.sorted = sorted;
    a.cell_start = c->cell_start;
    a.scenes = c->d_scenes;
    a.planes = c->d_planes;
    a.boxes = c->d_boxes;
    a.pr = c->cur.pr;
    a.tag = c->cur.tag;
    a.uid = c->cur.uid;
    a.total_planes = (int32_t)(c->planes.size() / 4);
    return a;
}

// --------------------------------------------------------------------------------------------
// hard-contact step
// --------------------------------------------------------------------------------------------
template <typename T>
struct Raw {  // detection output, detection order
    int32_t *b1, *b2;
    T *r1, *r2, *n;   // 3 x cap each, component-major
    T *dist, *mu;
};

// 4-vectors of the arithmetic type: the sweep reads whole 16/32-byte records
template <typename T> struct Vec4;
template <> struct Vec4<float> { typedef float4 type; };
template <> struct Vec4<double> { typedef double4 type; };
template <typename T> using T4 = typename Vec4<T>::type;

template <typename T>
__device__ __forceinline__ T4<T> mk4(T x, T y, T z, T w) {
    T4<T> r;
    r.x = x; r.y = y; r.z = z; r.w = w;
    return r;
}
template <typename T>
__device__ __forceinline__ V3<T> xyz(const T4<T> &a) { return v3(a.x, a.y, a.z); }

// loads that bypass L1: in the persistent sweeps, other SMs update these between colours
__device__ __forceinline__ float4 ldcg4(const float4 *p) { return __ldcg(p); }
__device__ __forceinline__ double4 ldcg4(const double4 *p) {
    const double2 a = __ldcg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldcg(reinterpret_cast<const double2 *>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// Colour-sorted solver records, one per contact.  rec holds kRec 4-vectors per contact, the
// frictionless sweep reading only the first three:
//   [n, dist] [r1, 1/D_nn] [r2, D_nn] [t, mu] [o, Dto^-1_tt] [D^-1 xx xy xz yy]
//   [D^-1 yz zz, Dto^-1_to, Dto^-1_oo]
constexpr int kRec = 7;
template <typename T>
struct Cache {
    int2 *ids;    // body 1, body 2 (-1: wall)
    T4<T> *rec;   // kRec per contact
    T4<T> *p;     // impulse in the contact frame (n, t, o, -)
    T4<T> *dc;    // 2 per contact: Delassus block in the contact frame [xy xz yy yz] [zz - - -]
                  // (its xx is rec[2].w), read by relaxation models 2-5 only
    // the sweeps' accessors
    __device__ __forceinline__ int2 get_ids(int64_t k) const { return ids[k]; }
    __device__ __forceinline__ const T4<T> *rec_of(int64_t k) const { return rec + (int64_t)kRec * k; }
    template <bool COH>
    __device__ __forceinline__ T4<T> get_p(int64_t k) const { return COH ? ldcg4(p + k) : p[k]; }
    __device__ __forceinline__ void put_p(int64_t k, const T4<T> &v) const { p[k] = v; }
    __device__ __forceinline__ const T4<T> *dc_of(int64_t k) const { return dc + 2 * k; }
};

// A block's own copy of the records of the contacts it sweeps, in shared memory, indexed by the
// block's local slot: the first NREC records of each contact (3 for the frictionless sweep, 7
// with friction; relaxation models 0 and 1 only).
template <typename T, int NREC>
struct SmemContacts {
    int2 *ids;
    T4<T> *rec;
    T4<T> *p;
    __device__ __forceinline__ int2 get_ids(int64_t k) const { return ids[k]; }
    __device__ __forceinline__ const T4<T> *rec_of(int64_t k) const { return rec + (int64_t)NREC * k; }
    template <bool COH>
    __device__ __forceinline__ T4<T> get_p(int64_t k) const { return p[k]; }
    __device__ __forceinline__ void put_p(int64_t k, const T4<T> &v) const { p[k] = v; }
    __device__ __forceinline__ const T4<T> *dc_of(int64_t) const { return nullptr; }
};

// The contacts of the compact single-block sweep: each contact's two bodies as slots of the
// block's shared body records (sids, -1 for a wall); the solver records stay in global memory.
template <typename T>
struct CompactContacts {
    const int2 *sids;
    const T4<T> *rec;
    T4<T> *p;
    const T4<T> *dc;
    __device__ __forceinline__ int2 get_ids(int64_t k) const { return sids[k]; }
    __device__ __forceinline__ const T4<T> *rec_of(int64_t k) const { return rec + (int64_t)kRec * k; }
    template <bool COH>
    __device__ __forceinline__ T4<T> get_p(int64_t k) const { return p[k]; }
    __device__ __forceinline__ void put_p(int64_t k, const T4<T> &v) const { p[k] = v; }
    __device__ __forceinline__ const T4<T> *dc_of(int64_t k) const { return dc + 2 * k; }
};

// Per body, slot order: velocities after the predictor with 1/m, 1/I (read-only in the sweeps)
// and the velocity corrections (read and written by the sweeps).
template <typename T>
struct BodyV {
    T4<T> *vr;    // v, 1/m
    T4<T> *wr;    // w, 1/I
    T4<T> *dv;    // dv, -
    T4<T> *dw;    // dw, -
    // scenes with moving boxes: the rows of every body's world-frame inverse inertia
    // R I^-1 R^T (RigidBody.h:866-869; a sphere's is 1/I on the diagonal), else null
    T4<T> *ia = nullptr, *ib = nullptr, *ic = nullptr;
    // the sweeps' accessors (COH: bypass L1, for records other SMs update between colours)
    __device__ __forceinline__ T4<T> get_vr(int32_t b) const { return vr[b]; }
    __device__ __forceinline__ T4<T> get_wr(int32_t b) const { return wr[b]; }
    template <bool COH>
    __device__ __forceinline__ T4<T> get_dv(int32_t b) const { return COH ? ldcg4(dv + b) : dv[b]; }
    template <bool COH>
    __device__ __forceinline__ T4<T> get_dw(int32_t b) const { return COH ? ldcg4(dw + b) : dw[b]; }
    __device__ __forceinline__ void put_dv(int32_t b, const T4<T> &v) const { dv[b] = v; }
    __device__ __forceinline__ void put_dw(int32_t b, const T4<T> &v) const { dw[b] = v; }
};

// The body records of a sweep kept in the shared memory of one thread-block cluster: body b
// lives in CTA b mod C (C = 2^shift, the cluster size) at row slot b / C, and is reached
// through distributed shared memory from every CTA of the cluster.  Rows: vr, wr, dv, dw, each
// `per` records long.
// loads and stores of a 4-vector at a shared::cluster address (mapa of a shared::cta address)
__device__ __forceinline__ float4 ld_dsm(uint32_t a, float) {
    float4 v;
    asm volatile("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ double4 ld_dsm(uint32_t a, double) {
    double4 v;
    asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a) : "memory");
    asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(v.z), "=d"(v.w) : "r"(a + 16) : "memory");
    return v;
}
__device__ __forceinline__ void st_dsm(uint32_t a, const float4 &v) {
    asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};"
                 :: "r"(a), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w) : "memory");
}
__device__ __forceinline__ void st_dsm(uint32_t a, const double4 &v) {
    asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" :: "r"(a), "d"(v.x), "d"(v.y) : "memory");
    asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" :: "r"(a + 16), "d"(v.z), "d"(v.w) : "memory");
}

template <typename T>
struct ClusterBodies {
    uint32_t base;   // shared::cta address of this CTA's rows (the same offset in every CTA)
    int per, shift;
    __device__ __forceinline__ uint32_t at(int row, int32_t b) const {
        const uint32_t a = base + (uint32_t)(((int64_t)row * per + (b >> shift)) * sizeof(T4<T>));
        uint32_t r;
        asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"((uint32_t)(b & ((1 << shift) - 1))));
        return r;
    }
    __device__ __forceinline__ T4<T> get_vr(int32_t b) const { return ld_dsm(at(0, b), T(0)); }
    __device__ __forceinline__ T4<T> get_wr(int32_t b) const { return ld_dsm(at(1, b), T(0)); }
    template <bool COH>
    __device__ __forceinline__ T4<T> get_dv(int32_t b) const { return ld_dsm(at(2, b), T(0)); }
    template <bool COH>
    __device__ __forceinline__ T4<T> get_dw(int32_t b) const { return ld_dsm(at(3, b), T(0)); }
    __device__ __forceinline__ void put_dv(int32_t b, const T4<T> &v) const { st_dsm(at(2, b), v); }
    __device__ __forceinline__ void put_dw(int32_t b, const T4<T> &v) const { st_dsm(at(3, b), v); }
};

// a body's inverse inertia applied to a vector: the scalar of a sphere, or (GEN) the full
// world-frame matrix of any body
template <typename T, bool GEN>
struct InvI;
template <typename T>
struct InvI<T, false> {
    T s;
    __device__ __forceinline__ V3<T> operator()(V3<T> a) const { return s * a; }
};
template <typename T>
struct InvI<T, true> {
    T4<T> a, b, c;
    __device__ __forceinline__ V3<T> operator()(V3<T> v) const {
        return v3(a.x * v.x + a.y * v.y + a.z * v.z, b.x * v.x + b.y * v.y + b.z * v.z,
                  c.x * v.x + c.y * v.y + c.z * v.z);
    }
};
template <typename T, bool GEN, typename BV>
__device__ __forceinline__ InvI<T, GEN> load_invi(const BV &bv, int32_t b, T ii) {
    if constexpr (GEN) {
        InvI<T, true> r;
        if (b >= 0) {
            r.a = bv.ia[b];
            r.b = bv.ib[b];
            r.c = bv.ic[b];
        } else {
            r.a = r.b = r.c = mk4<T>(T(0), T(0), T(0), T(0));
        }
        return r;
    } else {
        return InvI<T, false>{ii};
    }
}

template <typename T>
__device__ __forceinline__ V3<T> ld3c(const T *a, int64_t i, int64_t s) {
    return v3(a[i], a[i + s], a[i + 2 * s]);
}
template <typename T>
__device__ __forceinline__ void st3c(T *a, int64_t i, int64_t s, V3<T> v) {
    a[i] = v.x; a[i + s] = v.y; a[i + 2 * s] = v.z;
}

// permute to slot order and fill the body cache
template <typename VT, bool TRACKQ>
__global__ void k_permute_cache(int64_t n, const int32_t *sorted, const double4 *pr,
                                const VT *vw, const uint32_t *tag, const int32_t *uid,
                                const double4 *q, double4 *pr_o, VT *vw_o, uint32_t *tag_o,
                                int32_t *uid_o, double4 *q_o, const MatDev *mats, double gx,
                                double gy, double gz, double dt, BodyV<VT> bv) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int32_t b = sorted[t];
    const double4 p = pr[b];
    const uint32_t tg = tag[b];
    pr_o[t] = p;
    tag_o[t] = tg;
    uid_o[t] = uid[b];
    if (TRACKQ) q_o[t] = q[b];
    V3<VT> v = ld_vw(vw, n, b, 0), w = ld_vw(vw, n, b, 1);
    st_vw(vw_o, n, t, v, w);
    double im, ii, I;
    sphere_mass(p.w, mats[tg & 0xffffu].density, im, ii, I);
    const V3<VT> vp = v + v3(VT(gx), VT(gy), VT(gz)) * VT(dt);
    const V3<VT> Iw = VT(I) * w;
    const V3<VT> wp = w + VT(dt) * (VT(ii) * cross(Iw, w));
    bv.vr[t] = mk4<VT>(vp.x, vp.y, vp.z, VT(im));
    bv.wr[t] = mk4<VT>(wp.x, wp.y, wp.z, VT(ii));
    bv.dv[t] = mk4<VT>(VT(0), VT(0), VT(0), VT(0));
    bv.dw[t] = mk4<VT>(VT(0), VT(0), VT(0), VT(0));
    if (bv.ia) {
        bv.ia[t] = mk4<VT>(VT(ii), VT(0), VT(0), VT(0));
        bv.ib[t] = mk4<VT>(VT(0), VT(ii), VT(0), VT(0));
        bv.ic[t] = mk4<VT>(VT(0), VT(0), VT(ii), VT(0));
    }
}

template <typename T>
struct RawF {
    int64_t pos, cap, n;
    int32_t self;
    double4 ps;
    V3<double> vs, ws;
    const MatDev *mats;
    uint32_t tag_self;
    const uint32_t *tag;
    const int32_t *plane_mat, *box_mat;
    int32_t total_planes;
    const double4 *pr;
    const T *vw;
    double erp;
    Raw<T> raw;
    __device__ void operator()(const ContactGeom &g) {
        if (pos >= cap) { ++pos; return; }
        // relative velocity at the contact point for the friction pick (Contact.cpp:82-105)
        const V3<double> gp = v3(g.gx, g.gy, g.gz);
        const V3<double> r1 = gp - v3(ps.x, ps.y, ps.z);
        V3<double> rvel = vs + cross(ws, r1);
        V3<double> r2 = v3(0.0, 0.0, 0.0);
        int32_t m2;
        if (g.other >= 0) {
            const double4 pj = pr[g.other];
            r2 = gp - v3(pj.x, pj.y, pj.z);
            const V3<T> vt = ld_vw(vw, n, g.other, 0), wt = ld_vw(vw, n, g.other, 1);
            const V3<double> vj = v3(double(vt.x), double(vt.y), double(vt.z));
            const V3<double> wj = v3(double(wt.x), double(wt.y), double(wt.z));
            rvel = rvel - (vj + cross(wj, r2));
            m2 = (int32_t)(tag[g.other] & 0xffffu);
        } else {
            m2 = g.wall < total_planes ? plane_mat[g.wall] : box_mat[g.wall - total_planes];
        }
        const V3<double> n = v3(g.nx, g.ny, g.nz);
        const double nvel = dot(n, rvel);
        const double tvel = dot(n, rvel - n * nvel);
        const MatDev &a = mats[tag_self & 0xffffu], &b = mats[m2];
        const double mu = (fabs(tvel) > kFrictionThreshold) ? a.cdf + b.cdf : a.csf + b.csf;
        double dist = g.dist;
        if (dist < 0.0) dist *= erp;   // HCSITS.h:1797-1800
        raw.b1[pos] = self;
        raw.b2[pos] = g.other;
        st3c(raw.r1, pos, cap, v3(T(r1.x), T(r1.y), T(r1.z)));
        st3c(raw.r2, pos, cap, v3(T(r2.x), T(r2.y), T(r2.z)));
        st3c(raw.n, pos, cap, v3(T(n.x), T(n.y), T(n.z)));
        raw.dist[pos] = T(dist);
        raw.mu[pos] = T(mu);
        ++pos;
    }
};

template <typename T>
__global__ void k_raw(int64_t n, VisitArgs a, const int32_t *off, int64_t cap, const T *vw,
                      const MatDev *mats, const int32_t *plane_mat, const int32_t *box_mat,
                      double erp, Raw<T> raw, int32_t *err) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    RawF<T> f;
    f.pos = off[t];
    f.cap = cap;
    f.n = n;
    f.self = (int32_t)t;
    f.ps = a.pr[t];
    const V3<T> vt = ld_vw(vw, n, t, 0), wt = ld_vw(vw, n, t, 1);
    f.vs = v3(double(vt.x), double(vt.y), double(vt.z));
    f.ws = v3(double(wt.x), double(wt.y), double(wt.z));
    f.mats = mats;
    f.tag_self = a.tag[t];
    f.tag = a.tag;
    f.plane_mat = plane_mat;
    f.box_mat = box_mat;
    f.total_planes = a.total_planes;
    f.pr = a.pr;
    f.vw = vw;
    f.erp = erp;
    f.raw = raw;
    visit_contacts(a, (int32_t)t, f);
    if (f.pos > cap) atomicOr(err, DERR_CAPACITY);
}

// ---- colouring --------------------------------------------------------------------------------
// Kernels over the contacts read their count from device memory (ncp) and loop with a grid
// stride, so a step can be queued without the host knowing the count; none runs when the
// step was aborted for capacity (dd[kDdAbort]).
// (cond, may be null: the step needs the body -> contacts adjacency, i.e. the parallel rounds)
__global__ void k_degree(const int32_t *ncp, const int32_t *dd, const int32_t *cond,
                         const int32_t *b1, const int32_t *b2, int32_t *deg) {
    if (dd[kDdAbort] || (cond && !*cond)) return;
    const int64_t nc = *ncp;
    GRID_STRIDE(c, nc) {
        atomicAdd(&deg[b1[c]], 1);
        if (b2[c] >= 0) atomicAdd(&deg[b2[c]], 1);
    }
}

__global__ void k_adj_fill(const int32_t *ncp, const int32_t *dd, const int32_t *cond,
                           const int32_t *b1, const int32_t *b2, int32_t *fill, int32_t *adj) {
    if (dd[kDdAbort] || (cond && !*cond)) return;
    const int64_t nc = *ncp;
    GRID_STRIDE(c, nc) {
        adj[atomicAdd(&fill[b1[c]], 1)] = (int32_t)c;
        if (b2[c] >= 0) adj[atomicAdd(&fill[b2[c]], 1)] = (int32_t)c;
    }
}

// the guard of a step queued without the host: more contacts than the step was planned for
// (the buffers' capacity, or none for a step planned without contacts) abort the rest of the
// call (its steps leave the state as it is); the largest count is recorded
// the same for a step planned without contacts, in one launch instead of count, scan and
// guard: a sphere with any contact aborts the call's remaining steps (they are repeated with
// the contact stages, which record the counts).  dd[kDdNc] stays 0 from the last step that
// counted (it found none, or this plan would not have been chosen).
__global__ void k_any_contact(int64_t n, VisitArgs a, int32_t *dd) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || dd[kDdAbort]) return;
    CountF f;
    visit_contacts(a, a.sorted ? a.sorted[t] : (int32_t)t, f);
    if (f.n > 0) {
        dd[kDdAbort] = 1;
        atomicMax(&dd[kDdSeen], f.n);
    }
}

__global__ void k_guard(const int32_t *total, int64_t limit, int64_t serial_max, int32_t *dd) {
    const int32_t t = *total;
    dd[kDdRounds] = t > serial_max ? 1 : 0;
    if (t > limit) dd[kDdAbort] = 1;
    if (t > dd[kDdNeed]) dd[kDdNeed] = t;
    if (t > dd[kDdSeen]) dd[kDdSeen] = t;
}

__device__ __forceinline__ uint32_t prio(uint32_t c) {
    uint32_t h = c * 0x9E3779B1u;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

__device__ __forceinline__ bool beats(uint32_t c, uint32_t e) {
    const uint32_t pc = prio(c), pe_ = prio(e);
    return pc > pe_ || (pc == pe_ && c > e);
}

// Speculative greedy colouring, one round = propose + settle.  Propose: every uncoloured
// contact takes the smallest colour free at both of its bodies among the colours settled in
// earlier rounds.  Settle: a proposal stands unless a contact sharing one of its dynamic bodies
// proposed the same colour with a higher priority (a fixed hash of the contact index).  The
// highest-priority proposal of every clash stands, so each round colours a large share of the
// remaining contacts -- a few rounds even where a box carries dozens of contact points, against
// a round per priority level when only local priority maxima take colours.  The result depends
// only on the contact order, not on scheduling.  W 64-bit words of settled colours per body
// (64 W colours: 64 for spheres, whose contacts are few, 256 for scenes with boxes).
template <int W>
__device__ __forceinline__ void color_propose(int64_t c, const int32_t *b1, const int32_t *b2,
                                              const int32_t *color, const uint64_t *used,
                                              int32_t *tent, int32_t *err) {
    if (color[c] >= 0) {
        tent[c] = -1;
        return;
    }
    const int32_t a = b1[c], b = b2[c];
    int col = -1;
#pragma unroll
    for (int wd = 0; wd < W && col < 0; ++wd) {
        const uint64_t u = used[(int64_t)a * W + wd] | (b >= 0 ? used[(int64_t)b * W + wd] : 0ull);
        const int f = __ffsll((long long)~u) - 1;
        if (f >= 0) col = 64 * wd + f;
    }
    if (col < 0) atomicOr(err, DERR_COLORS);   // stays uncoloured; the step reports the error
    tent[c] = col;
}

template <int W>
__device__ __forceinline__ void color_settle(int64_t c, int round, const int32_t *b1,
                                             const int32_t *b2, const int32_t *adj_start,
                                             const int32_t *adj, const int32_t *tent,
                                             int32_t *color, uint64_t *used, int32_t *remaining) {
    const int32_t t = tent[c];
    if (t < 0) return;
    const int32_t bodies[2] = {b1[c], b2[c]};
    for (int k = 0; k < 2; ++k) {
        const int32_t b = bodies[k];
        if (b < 0) continue;
        for (int s = adj_start[b]; s < adj_start[b + 1]; ++s) {
            const int32_t e = adj[s];
            if (e != c && tent[e] == t && beats((uint32_t)e, (uint32_t)c)) {
                atomicAdd(remaining, 1);
                return;
            }
        }
    }
    // colour and round packed: low 8 bits colour, upper bits the round it was settled in
    color[c] = (round << 8) | t;
    atomicOr((unsigned long long *)&used[(int64_t)bodies[0] * W + (t >> 6)], 1ull << (t & 63));
    if (bodies[1] >= 0)
        atomicOr((unsigned long long *)&used[(int64_t)bodies[1] * W + (t >> 6)], 1ull << (t & 63));
}

template <int W>
__global__ void k_color_propose(const int32_t *ncp, const int32_t *b1, const int32_t *b2,
                                const int32_t *color, const uint64_t *used, int32_t *tent,
                                int32_t *err) {
    const int64_t nc = *ncp;
    GRID_STRIDE(c, nc) color_propose<W>(c, b1, b2, color, used, tent, err);
}

template <int W>
__global__ void k_color_settle(const int32_t *ncp, int round, const int32_t *b1,
                               const int32_t *b2, const int32_t *adj_start, const int32_t *adj,
                               const int32_t *tent, int32_t *color, uint64_t *used,
                               int32_t *remaining) {
    const int64_t nc = *ncp;
    GRID_STRIDE(c, nc)
        color_settle<W>(c, round, b1, b2, adj_start, adj, tent, color, used, remaining);
}

// All rounds of the parallel colouring in one cooperative launch, for steps queued without
// the host: rounds separated by bounded grid barriers until a round leaves no contact
// uncoloured (rem: one counter per round, zeroed before the launch).  Does nothing when the
// one-thread colouring handles the step (at most serial_max contacts).
template <int W>
__global__ void k_color_rounds(const int32_t *ncp, const int32_t *dd, int64_t serial_max,
                               const int32_t *b1, const int32_t *b2, const int32_t *adj_start,
                               const int32_t *adj, int32_t *tent, int32_t *color, uint64_t *used,
                               int32_t *rem, unsigned int *bar, int32_t *err) {
    if (dd[kDdAbort]) return;
    const int64_t nc = *ncp;
    if (nc <= serial_max) return;
    for (int round = 0; round < kMaxRounds; ++round) {
        GRID_STRIDE(c, nc) color_propose<W>(c, b1, b2, color, used, tent, err);
        if (!grid_sync(bar, err)) return;
        GRID_STRIDE(c, nc)
            color_settle<W>(c, round, b1, b2, adj_start, adj, tent, color, used, rem + round);
        if (!grid_sync(bar, err)) return;
        if (*(volatile int32_t *)(rem + round) == 0) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(err, DERR_COLORS);
}

// Few contacts: one thread colours them greedily in contact order (the smallest colour free at
// both bodies), in one launch.  Where a body carries dozens of contacts (box stacks) this needs
// about as many colours as the busiest body has contacts, the least possible, where the parallel
// rounds need a launch pair per round and end with more colours.
// The used-colour masks live in shared memory when they fit (used_global == null), else in
// the zeroed global array.
template <int W>
__global__ void k_color_serial(const int32_t *ncp, const int32_t *dd, int64_t serial_max,
                               const int32_t *__restrict__ b1, const int32_t *__restrict__ b2,
                               int32_t *__restrict__ color, int64_t nbod, uint64_t *used_global,
                               int32_t *err) {
    if (dd[kDdAbort]) return;
    const int64_t nc = *ncp;
    if (nc > serial_max) return;   // the parallel rounds colour this step
    extern __shared__ uint64_t used_shared[];
    uint64_t *used = used_global ? used_global : used_shared;
    if (!used_global)
        for (int64_t i = threadIdx.x; i < nbod * W; i += blockDim.x) used_shared[i] = 0ull;
    __syncthreads();
    if (threadIdx.x != 0) return;
    // the bodies of the next contacts are loaded ahead, off the chain of mask updates
    constexpr int kAhead = 8;
    int32_t qa[kAhead], qb[kAhead];
#pragma unroll
    for (int k = 0; k < kAhead; ++k) {
        qa[k] = k < nc ? __ldg(b1 + k) : 0;
        qb[k] = k < nc ? __ldg(b2 + k) : -1;
    }
    for (int64_t c = 0; c < nc; ++c) {
        const int32_t a = qa[0], b = qb[0];
#pragma unroll
        for (int k = 0; k + 1 < kAhead; ++k) {
            qa[k] = qa[k + 1];
            qb[k] = qb[k + 1];
        }
        qa[kAhead - 1] = c + kAhead < nc ? __ldg(b1 + c + kAhead) : 0;
        qb[kAhead - 1] = c + kAhead < nc ? __ldg(b2 + c + kAhead) : -1;
        int col = -1;
#pragma unroll
        for (int wd = 0; wd < W && col < 0; ++wd) {
            const uint64_t u = used[(int64_t)a * W + wd] | (b >= 0 ? used[(int64_t)b * W + wd] : 0ull);
            const int f = __ffsll((long long)~u) - 1;
            if (f >= 0) col = 64 * wd + f;
        }
        if (col < 0) {
            atomicOr(err, DERR_COLORS);
            color[c] = 0;
            continue;
        }
        color[c] = col;
        used[(int64_t)a * W + (col >> 6)] |= 1ull << (col & 63);
        if (b >= 0) used[(int64_t)b * W + (col >> 6)] |= 1ull << (col & 63);
    }
}

__global__ void k_color_hist(const int32_t *ncp, const int32_t *dd, int32_t *color,
                             int32_t *hist, int32_t *ncolors) {
    if (dd[kDdAbort]) return;
    const int64_t nc = *ncp;
    GRID_STRIDE(c, nc) {
        const int col = color[c] & 0xff;
        color[c] = col;
        atomicAdd(&hist[col], 1);
        atomicMax(ncolors, col + 1);
    }
}

// colour offsets from the histogram (one block of kMaxColors threads): cstart[0..ncolors] and
// a copy as the fill counters of k_color_pos; the colour count and the largest colour in dd
__global__ void __launch_bounds__(kMaxColors) k_color_scan(const int32_t *hist,
                                                           const int32_t *nco, int32_t *cstart,
                                                           int32_t *fill, int32_t *dd) {
    __shared__ int32_t s[kMaxColors];
    const int ncol = *nco;
    const int i = threadIdx.x;
    const int32_t h = i < ncol ? hist[i] : 0;
    s[i] = h;
    __syncthreads();
    // Hillis-Steele inclusive scan (256 entries)
    for (int o = 1; o < kMaxColors; o <<= 1) {
        const int32_t v = i >= o ? s[i - o] : 0;
        __syncthreads();
        s[i] += v;
        __syncthreads();
    }
    const int32_t excl = s[i] - h;
    if (i <= ncol) {
        const int32_t start = (i == ncol) ? (ncol > 0 ? s[ncol - 1] : 0) : excl;
        cstart[i] = start;
        fill[i] = start;
    }
    __syncthreads();
    // largest colour
    s[i] = h;
    __syncthreads();
    for (int o = kMaxColors / 2; o > 0; o >>= 1) {
        if (i < o) s[i] = max(s[i], s[i + o]);
        __syncthreads();
    }
    if (i == 0) {
        dd[kDdNcolors] = ncol;
        dd[kDdMaxcol] = s[0];
    }
}

__global__ void k_color_pos(const int32_t *ncp, const int32_t *dd, const int32_t *color,
                            int32_t *fill, int32_t *pos) {
    if (dd[kDdAbort]) return;
    const int64_t nc = *ncp;
    GRID_STRIDE(c, nc) pos[c] = atomicAdd(&fill[color[c]], 1);
}

// ---- contact cache (HCSITS.h:1767-1815) --------------------------------------------------------
template <typename T, bool GEN>
__global__ void k_cache(const int32_t *ncp, const int32_t *dd, int64_t cap, Raw<T> raw,
                        const int32_t *pos, BodyV<T> bv, int64_t nb, Cache<T> cc) {
    if (dd[kDdAbort]) return;
    const int64_t nc = *ncp;
    GRID_STRIDE(c, nc) {
    const int64_t k = pos[c];
    const int32_t b1 = raw.b1[c], b2 = raw.b2[c];
    const V3<T> r1 = ld3c(raw.r1, c, cap), r2 = ld3c(raw.r2, c, cap), n = ld3c(raw.n, c, cap);
    V3<T> t;
    if (fabs(n.x) < fabs(n.y)) {
        if (fabs(n.x) < fabs(n.z)) t = v3(T(0), n.z, -n.y);
        else t = v3(n.y, -n.x, T(0));
    } else {
        if (fabs(n.y) < fabs(n.z)) t = v3(-n.z, T(0), n.x);
        else t = v3(n.y, -n.x, T(0));
    }
    t = normalized(t);
    const V3<T> o = cross(n, t);
    const T im1 = bv.vr[b1].w, ii1 = bv.wr[b1].w;
    const T im2 = b2 >= 0 ? bv.vr[b2].w : T(0), ii2 = b2 >= 0 ? bv.wr[b2].w : T(0);
    // D = -(r1^x I1^-1 r1^x + r2^x I2^-1 r2^x) + (1/m1 + 1/m2) 1 with scalar sphere inertia:
    // -r^x r^x = |r|^2 1 - r r^T
    T D[9];
    if constexpr (GEN) {
        // -(r1^x I1 r1^x + r2^x I2 r2^x) + (1/m1 + 1/m2) 1 with the full world-frame inverse
        // inertias, in pe's operation order (Matrix3x3.h:2355-2365, 2419-2432; HCSITS.h:1802)
        T A[9], B[9];
        const InvI<T, true> I1 = load_invi<T, true>(bv, b1, ii1), I2 = load_invi<T, true>(bv, b2, ii2);
        auto rmr = [](const InvI<T, true> &I, V3<T> r, T *out) {
            const T m[9] = {I.a.x, I.a.y, I.a.z, I.b.x, I.b.y, I.b.z, I.c.x, I.c.y, I.c.z};
            T x[9];   // r^x * M
            x[0] = r.y * m[6] - r.z * m[3]; x[1] = r.y * m[7] - r.z * m[4]; x[2] = r.y * m[8] - r.z * m[5];
            x[3] = r.z * m[0] - r.x * m[6]; x[4] = r.z * m[1] - r.x * m[7]; x[5] = r.z * m[2] - r.x * m[8];
            x[6] = r.x * m[3] - r.y * m[0]; x[7] = r.x * m[4] - r.y * m[1]; x[8] = r.x * m[5] - r.y * m[2];
            // (r^x M) * r^x
            out[0] = x[1] * r.z - x[2] * r.y; out[1] = x[2] * r.x - x[0] * r.z; out[2] = x[0] * r.y - x[1] * r.x;
            out[3] = x[4] * r.z - x[5] * r.y; out[4] = x[5] * r.x - x[3] * r.z; out[5] = x[3] * r.y - x[4] * r.x;
            out[6] = x[7] * r.z - x[8] * r.y; out[7] = x[8] * r.x - x[6] * r.z; out[8] = x[6] * r.y - x[7] * r.x;
        };
        rmr(I1, r1, A);
        rmr(I2, r2, B);
        const T ims = im1 + im2;
#pragma unroll
        for (int k = 0; k < 9; ++k) D[k] = -(A[k] + B[k]);
        D[0] += ims; D[4] += ims; D[8] += ims;
    } else {
        const T a1 = dot(r1, r1), a2 = dot(r2, r2);
        const T rr1[3] = {r1.x, r1.y, r1.z}, rr2[3] = {r2.x, r2.y, r2.z};
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const T d1 = (i == j ? a1 : T(0)) - rr1[i] * rr1[j];
                const T d2 = (i == j ? a2 : T(0)) - rr2[i] * rr2[j];
                D[3 * i + j] = ii1 * d1 + ii2 * d2 + (i == j ? im1 + im2 : T(0));
            }
    }
    // rotate into the contact frame: Dc = C^T D C with C = [n t o]
    const V3<T> C[3] = {n, t, o};
    T Dc[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const V3<T> DCi = v3(D[0] * C[i].x + D[1] * C[i].y + D[2] * C[i].z,
                             D[3] * C[i].x + D[4] * C[i].y + D[5] * C[i].z,
                             D[6] * C[i].x + D[7] * C[i].y + D[8] * C[i].z);
#pragma unroll
        for (int j = 0; j < 3; ++j) Dc[j][i] = dot(C[j], DCi);
    }
    // symmetric inverse
    const T xx = Dc[0][0], xy = Dc[0][1], xz = Dc[0][2], yy = Dc[1][1], yz = Dc[1][2],
            zz = Dc[2][2];
    const T c00 = yy * zz - yz * yz, c01 = xz * yz - xy * zz, c02 = xy * yz - xz * yy;
    const T det = xx * c00 + xy * c01 + xz * c02;
    const T id = T(1) / det;
    const T d2 = yy * zz - yz * yz;
    const T id2 = T(1) / d2;
    T4<T> *R = cc.rec + (int64_t)kRec * k;
    R[0] = mk4<T>(n.x, n.y, n.z, raw.dist[c]);
    R[1] = mk4<T>(r1.x, r1.y, r1.z, T(1) / xx);
    R[2] = mk4<T>(r2.x, r2.y, r2.z, xx);
    R[3] = mk4<T>(t.x, t.y, t.z, raw.mu[c]);
    R[4] = mk4<T>(o.x, o.y, o.z, zz * id2);
    R[5] = mk4<T>(c00 * id, c01 * id, c02 * id, (xx * zz - xz * xz) * id);
    R[6] = mk4<T>((xy * xz - xx * yz) * id, (xx * yy - xy * xy) * id, -yz * id2, yy * id2);
    cc.dc[2 * k] = mk4<T>(xy, xz, yy, yz);
    cc.dc[2 * k + 1] = mk4<T>(zz, T(0), T(0), T(0));
    cc.ids[k] = make_int2(b1, b2);
    cc.p[k] = mk4<T>(T(0), T(0), T(0), T(0));
    }
    (void)nb;
}

// ---- one colour of one sweep ----------------------------------------------------------------
// ---- one-contact solvers of pe's relaxation models 2-5, in the contact frame --------------
// g: relative velocity in the contact frame with the ERP-scaled penetration term on its normal
// component; D: the Delassus block (symmetric); pc: the contact's impulse before this update.

// projection onto the friction cone of the orthogonal-projection models (HCSITS.h:2680-2700)
template <typename T>
__device__ __forceinline__ V3<T> cone_projection(V3<T> p, T mu) {
    const T flimit = mu * p.x;
    const T fsq = p.y * p.y + p.z * p.z;
    if (p.x > T(0) && fsq < flimit * flimit) return p;
    if (p.x < T(0) && fsq < p.x / (mu * mu)) return v3(T(0), T(0), T(0));
    const T f = sqrt(fsq);
    p.x = (f * mu + p.x) / (mu * mu + T(1));
    const T factor = mu * p.x / f;
    p.y *= factor;
    p.z *= factor;
    return p;
}

// models 2 and 4 (HCSITS.h:2631-2723): one step of relaxation w = 1 on D p + g, the exact form
// raising its normal part by mu |(D p + g)_to|, then the cone projection
template <typename T, bool EXACT>
__device__ __forceinline__ V3<T> solve_orthogonal(V3<T> pc, V3<T> g, const T D[6], T mu) {
    V3<T> tmp = v3(D[0] * pc.x + D[1] * pc.y + D[2] * pc.z + g.x,
                   D[1] * pc.x + D[3] * pc.y + D[4] * pc.z + g.y,
                   D[2] * pc.x + D[4] * pc.y + D[5] * pc.z + g.z);
    if (EXACT) tmp.x += sqrt(tmp.y * tmp.y + tmp.z * tmp.z) * mu;
    return cone_projection<T>(pc - tmp, mu);
}

// 0.5 x^T A x - x^T b for the golden-section searches (A symmetric 2x2)
template <typename T>
__device__ __forceinline__ T quad2(T a00, T a01, T a11, T x0, T x1, T b0, T b1) {
    const T y0 = a00 * x0 + a01 * x1, y1 = a01 * x0 + a11 * x1;
    return ((T(0.5) * x0) * y0 + (T(0.5) * x1) * y1) - (x0 * b0 + x1 * b1);
}

// golden-section search over the angle of the friction circle (radius(alpha)), keeping the
// smallest energy found (HCSITS.h:2440-2500, 2895-2945); 20 sub-iterations (HCSITS.h:423)
template <typename T, typename R>
__device__ __forceinline__ void golden_angle(T alpha_left, T alpha_right, R radius, T a00, T a01,
                                             T a11, T b0, T b1, T &x0, T &x1, T &fmid) {
    const T phi = T(0.5) * (T(1) + sqrt(T(5)));
    T alpha_mid = (alpha_right + alpha_left * phi) / (T(1) + phi);
    T r = radius(alpha_mid);
    x0 = r * cos(alpha_mid);
    x1 = r * sin(alpha_mid);
    fmid = quad2<T>(a00, a01, a11, x0, x1, b0, b1);
    bool leftlarger = false;
    for (int k = 0; k < 20; ++k) {
        const T alpha_next = alpha_left + (alpha_right - alpha_mid);
        r = radius(alpha_next);
        const T n0 = r * cos(alpha_next), n1 = r * sin(alpha_next);
        const T fnext = quad2<T>(a00, a01, a11, n0, n1, b0, b1);
        if (leftlarger) {
            if (fnext < fmid) {
                alpha_right = alpha_mid; alpha_mid = alpha_next;
                x0 = n0; x1 = n1; fmid = fnext; leftlarger = true;
            } else {
                alpha_left = alpha_next; leftlarger = false;
            }
        } else {
            if (fnext < fmid) {
                alpha_left = alpha_mid; alpha_mid = alpha_next;
                x0 = n0; x1 = n1; fmid = fnext; leftlarger = false;
            } else {
                alpha_right = alpha_next; leftlarger = true;
            }
        }
    }
}

// model 3 (HCSITS.h:2330-2595): exact Coulomb friction by 20 rounds of a normal solve for the
// current tangential impulse and a tangential solve for the new normal one; a tangential solve
// outside the cone is replaced by the energy minimiser on the cone's circle.  corr(p) is the
// change of the relative velocity an impulse p (world frame) causes through the bodies'
// rotational inertia alone, as pe writes it.
template <typename T, typename Corr>
__device__ __forceinline__ V3<T> solve_coulomb_decoupling(V3<T> pcf, const V3<T> &gdot,
                                                          const V3<T> &n, const V3<T> &t,
                                                          const V3<T> &o, T dist_dtinv,
                                                          T dn_inv, T tt, T to, T oo,
                                                          const T D[6], T mu, Corr corr) {
    for (int j = 0; j < 20; ++j) {
        pcf.x = T(0);
        V3<T> gc = gdot + corr(t * pcf.y + o * pcf.z);
        const T gcn = dot(n, gc) + dist_dtinv;
        pcf.x = -(dn_inv * gcn);
        pcf.x = pcf.x > T(0) ? pcf.x : T(0);
        gc = gdot + corr(n * pcf.x);
        const T gt = dot(t, gc), go = dot(o, gc);
        pcf.y = -(tt * gt + to * go);
        pcf.z = -(to * gt + oo * go);
        const T flimit = mu * pcf.x;
        const T fsq = pcf.y * pcf.y + pcf.z * pcf.z;
        if (fsq > flimit * flimit) {
            const T f = flimit / sqrt(fsq);
            const T shift = atan2(-pcf.z, pcf.y);
            const T acos_f = acos(f);
            T x0, x1, fm;
            golden_angle<T>(-acos_f - shift, acos_f - shift, [flimit](T) { return flimit; },
                            D[3], D[4], D[5], -gt, -go, x0, x1, fm);
            pcf.y = x0;
            pcf.z = x1;
        }
    }
    return pcf;
}

// model 5 (HCSITS.h:2745-3055): generalized maximum dissipation: the tangential impulse of
// least kinetic energy on the intersection of the plane of maximum compression with the
// friction cone, by a golden-section search over the angle; pcf enters as -D^-1 g.
template <typename T>
__device__ __forceinline__ V3<T> solve_gmd(V3<T> pcf, const V3<T> &g, const T D[6], T mu,
                                           T fsq) {
    const T twopi = T(6.283185307179586476925286766559);
    const T invA_nn = T(1) / D[0];
    const T offdiag = D[4] - invA_nn * D[1] * D[2];
    const T a00 = D[3] - invA_nn * (D[1] * D[1]), a11 = D[5] - invA_nn * (D[2] * D[2]);
    const T b0 = -g.y + invA_nn * D[1] * g.x, b1 = -g.z + invA_nn * D[2] * g.x;
    const T shiftI = atan2(-D[2], D[1]);
    const T shiftJ = atan2(-pcf.z, pcf.y);
    const T a3 = sqrt(D[1] * D[1] + D[2] * D[2]);
    const T fractionI = -D[0] / (mu * a3);
    T fractionJ = invA_nn * mu * ((-g.x) / sqrt(fsq) - a3 * cos(shiftI - shiftJ));
    fractionJ = fractionJ < T(1) ? fractionJ : T(1);
    T alpha_left, alpha_right;
    if (fractionJ < T(-1)) {
        const T angleI = acos(fractionI);
        alpha_left = -angleI - shiftI;
        alpha_right = +angleI - shiftI;
        if (alpha_left < T(0)) { alpha_left += twopi; alpha_right += twopi; }
    } else if (D[0] > mu * a3) {
        const T angleJ = acos(fractionJ);
        alpha_left = -angleJ - shiftJ;
        alpha_right = +angleJ - shiftJ;
        if (alpha_left < T(0)) { alpha_left += twopi; alpha_right += twopi; }
    } else {
        const T angleJ = acos(fractionJ);
        T a1l = -angleJ - shiftJ, a1r = +angleJ - shiftJ;
        if (a1l < T(0)) { a1l += twopi; a1r += twopi; }
        const T angleI = acos(fractionI);
        T a2l = -angleI - shiftI, a2r = +angleI - shiftI;
        if (a2l < T(0)) { a2l += twopi; a2r += twopi; }
        if (a1l > a2l) {
            T u = a1l; a1l = a2l; a2l = u;
            u = a1r; a1r = a2r; a2r = u;
        }
        if (a2l > a1r) {
            a2r -= twopi;
            if (!(a2r > a1r)) a1r = a2r;
        } else {
            a1l = a2l;
            if (!(a2r > a1r)) a1r = a2r;
        }
        alpha_left = a1l;
        alpha_right = a1r;
    }
    auto radius = [&](T alpha) {
        T r = mu * (-g.x) / (D[0] + mu * a3 * cos(alpha + shiftI));
        return r < T(0) ? T(INFINITY) : r;
    };
    T x0, x1, fm;
    golden_angle<T>(alpha_left, alpha_right, radius, a00, offdiag, a11, b0, b1, x0, x1, fm);
    {
        const T alpha_init = atan2(pcf.z, pcf.y);
        const T r = radius(alpha_init);
        const T i0 = r * cos(alpha_init), i1 = r * sin(alpha_init);
        if (quad2<T>(a00, offdiag, a11, i0, i1, b0, b1) < fm) {
            x0 = i0;
            x1 = i1;
        }
    }
    return v3(invA_nn * (-g.x - D[1] * x0 - D[2] * x1), x0, x1);
}

// one contact of one sweep of relaxation model MODEL (pe's RelaxationModel, HCSITS.h:172-179);
// COHERENT: read the velocity corrections and the impulse from L2
template <typename T, int MODEL, bool COHERENT, bool GEN = false, typename BV = BodyV<T>,
          typename CC = Cache<T>>
__device__ __forceinline__ void sweep_contact(int64_t k, T dtinv, const CC &cc,
                                              const BV &bv, int track_delta,
                                              unsigned long long *delta) {
    constexpr bool FRICTION = MODEL != 0;
    const int2 ids = cc.get_ids(k);
    const int32_t b1 = ids.x, b2 = ids.y;
    const T4<T> *R = cc.rec_of(k);
    const T4<T> q0 = R[0], q1 = R[1], q2 = R[2];
    const V3<T> n = xyz<T>(q0), r1 = xyz<T>(q1), r2 = xyz<T>(q2);
    const T dist = q0.w, dn_inv = q1.w;
    const T4<T> pc4 = cc.template get_p<COHERENT>(k);
    const V3<T> pc = xyz<T>(pc4);  // contact frame
    const T4<T> vr1 = bv.get_vr(b1), wr1 = bv.get_wr(b1);
    const T im1 = vr1.w, ii1 = wr1.w;
    V3<T> dv1 = xyz<T>(bv.template get_dv<COHERENT>(b1));
    V3<T> dw1 = xyz<T>(bv.template get_dw<COHERENT>(b1));
    const V3<T> v1 = xyz<T>(vr1), w1 = xyz<T>(wr1);
    V3<T> dv2 = v3(T(0), T(0), T(0)), dw2 = dv2, v2 = dv2, w2 = dv2;
    T im2 = T(0), ii2 = T(0);
    if (b2 >= 0) {
        const T4<T> vr2 = bv.get_vr(b2), wr2 = bv.get_wr(b2);
        im2 = vr2.w;
        ii2 = wr2.w;
        dv2 = xyz<T>(bv.template get_dv<COHERENT>(b2));
        dw2 = xyz<T>(bv.template get_dw<COHERENT>(b2));
        v2 = xyz<T>(vr2);
        w2 = xyz<T>(wr2);
    }
    const InvI<T, GEN> I1 = load_invi<T, GEN>(bv, b1, ii1), I2 = load_invi<T, GEN>(bv, b2, ii2);
    static_assert(!GEN || std::is_same<BV, BodyV<T>>::value, "full inverse inertias: BodyV only");
    V3<T> t, o;
    V3<T> pold;
    T4<T> q3, q4;
    if (FRICTION) {
        q3 = R[3];
        q4 = R[4];
        t = xyz<T>(q3);
        o = xyz<T>(q4);
        pold = n * pc.x + t * pc.y + o * pc.z;
    } else {
        pold = n * pc.x;
    }
    // remove this contact's impulse (HCSITS.h:2050-2053)
    dv1 = dv1 - im1 * pold;
    dw1 = dw1 - I1(cross(r1, pold));
    if (b2 >= 0) {
        dv2 = dv2 + im2 * pold;
        dw2 = dw2 + I2(cross(r2, pold));
    }
    const V3<T> gdot = ((v1 + dv1) - (v2 + dv2) + cross(w1 + dw1, r1)) - cross(w2 + dw2, r2);
    T gn = dot(n, gdot) + dist * dtinv;
    V3<T> pnew = v3(T(0), T(0), T(0));
    V3<T> pcf = pnew;
    bool apply = false;
    if (MODEL == 0 || MODEL == 1) {
        if (gn < T(0)) {
            apply = true;
            if (!FRICTION) {
                pcf.x = -dn_inv * gn;
                pnew = n * pcf.x;
            } else {
                const T gt = dot(t, gdot), go = dot(o, gdot);
                const T4<T> q5 = R[5], q6 = R[6];
                const T dxx = q5.x, dxy = q5.y, dxz = q5.z, dyy = q5.w, dyz = q6.x, dzz = q6.y;
                pcf = v3(-(dxx * gn + dxy * gt + dxz * go), -(dxy * gn + dyy * gt + dyz * go),
                         -(dxz * gn + dyz * gt + dzz * go));
                const T mu = q3.w;
                T flimit = mu * pcf.x;
                T fsq = pcf.y * pcf.y + pcf.z * pcf.z;
                if (fsq > flimit * flimit || pcf.x < T(0)) {
                    // decoupled relaxation (HCSITS.h:2187-2228)
                    V3<T> ptmp = t * pc.y + o * pc.z;
                    const V3<T> e1 = cross(I1(cross(r1, ptmp)), r1);
                    const V3<T> e2 = (b2 >= 0) ? cross(I2(cross(r2, ptmp)), r2) : v3(T(0), T(0), T(0));
                    const T gdot_n = gn + dot(n, e1 + e2);
                    pcf.x = -(dn_inv * gdot_n);
                    pcf.x = pcf.x > T(0) ? pcf.x : T(0);
                    ptmp = n * pcf.x;
                    const V3<T> f1 = cross(I1(cross(r1, ptmp)), r1);
                    const V3<T> f2 = (b2 >= 0) ? cross(I2(cross(r2, ptmp)), r2) : v3(T(0), T(0), T(0));
                    const V3<T> gdot2 = (gdot + f1) + f2;
                    const T g2t = dot(t, gdot2), g2o = dot(o, gdot2);
                    const T ttt = q4.w, tto = q6.z, too = q6.w;
                    pcf.y = -(ttt * g2t + tto * g2o);
                    pcf.z = -(tto * g2t + too * g2o);
                    flimit = mu * pcf.x;
                    fsq = pcf.y * pcf.y + pcf.z * pcf.z;
                    if (fsq > flimit * flimit) {
                        const T f = flimit / sqrt(fsq);
                        pcf.y *= f;
                        pcf.z *= f;
                    }
                }
                pnew = n * pcf.x + t * pcf.y + o * pcf.z;
            }
        }
    } else {
        const T mu = q3.w;
        const V3<T> g = v3(gn, dot(t, gdot), dot(o, gdot));
        const T4<T> *dck = cc.dc_of(k);
        const T4<T> d0 = dck[0], d1 = dck[1];
        const T D[6] = {q2.w, d0.x, d0.y, d0.z, d0.w, d1.x};   // xx xy xz yy yz zz
        if (MODEL == 2 || MODEL == 4) {
            pcf = solve_orthogonal<T, MODEL == 4>(pc, g, D, mu);
            apply = true;
        } else if (gn < T(0)) {
            apply = true;
            const T4<T> q5 = R[5], q6 = R[6];
            pcf = v3(-(q5.x * g.x + q5.y * g.y + q5.z * g.z), -(q5.y * g.x + q5.w * g.y + q6.x * g.z),
                     -(q5.z * g.x + q6.x * g.y + q6.y * g.z));
            const T flimit = mu * pcf.x;
            const T fsq = pcf.y * pcf.y + pcf.z * pcf.z;
            if (fsq > flimit * flimit || pcf.x < T(0)) {
                if (MODEL == 3) {
                    auto corr = [&](const V3<T> &pp) {
                        const V3<T> e1 = cross(I1(cross(r1, pp)), r1);
                        const V3<T> e2 = (b2 >= 0) ? cross(I2(cross(r2, pp)), r2) : v3(T(0), T(0), T(0));
                        return e1 + e2;
                    };
                    pcf = solve_coulomb_decoupling<T>(pcf, gdot, n, t, o, dist * dtinv, dn_inv, q4.w,
                                                      q6.z, q6.w, D, mu, corr);
                } else {
                    pcf = solve_gmd<T>(pcf, g, D, mu, fsq);
                }
            }
        }
        if (apply) pnew = n * pcf.x + t * pcf.y + o * pcf.z;
    }
    if (apply) {
        dv1 = dv1 + im1 * pnew;
        dw1 = dw1 + I1(cross(r1, pnew));
        if (b2 >= 0) {
            dv2 = dv2 - im2 * pnew;
            dw2 = dw2 - I2(cross(r2, pnew));
        }
    }
    cc.put_p(k, mk4<T>(pcf.x, pcf.y, pcf.z, T(0)));
    bv.put_dv(b1, mk4<T>(dv1.x, dv1.y, dv1.z, T(0)));
    bv.put_dw(b1, mk4<T>(dw1.x, dw1.y, dw1.z, T(0)));
    if (b2 >= 0) {
        bv.put_dv(b2, mk4<T>(dv2.x, dv2.y, dv2.z, T(0)));
        bv.put_dw(b2, mk4<T>(dw2.x, dw2.y, dw2.z, T(0)));
    }
    if (track_delta) {
        const V3<T> dp = pold - pnew;
        const double m = fmax(fabs(double(dp.x)), fmax(fabs(double(dp.y)), fabs(double(dp.z))));
        atomicMax(delta, (unsigned long long)__double_as_longlong(m));
    }
}

// Whether a sweep form runs for this step (decided on the device, so that a step can be queued
// without the host knowing its colours): not after a capacity abort; gate 1 (one block) only
// when every colour fits one block, gate 2 (the grid) only when one does not, gate 0 always.
// Gates 4 and 5 split gate 1 by the contact count: 4 when the compact single-block form holds
// them all (kCompactMax), 5 when it does not.  Gate 3 (the cluster form) runs for colours beyond
// one block up to kDsmemMaxcol, and gate 6 (the grid, when the cluster form is launched beside
// it) for larger ones.
constexpr int kCompactMax = 768;      // contacts of the compact single-block form
constexpr int kDsmemMaxcol = 3072;    // largest colour the cluster form takes in automatic mode
__device__ __forceinline__ bool sweeps_gate(const int32_t *dd, int gate) {
    if (dd[kDdAbort]) return false;
    const int maxcol = dd[kDdMaxcol];
    const int nc = dd[kDdNc];
    if ((gate == 1 || gate == 4 || gate == 5) && maxcol > kBlk) return false;
    if (gate == 4 && nc > kCompactMax) return false;
    if (gate == 5 && nc <= kCompactMax) return false;
    if ((gate == 2 || gate == 3 || gate == 6) && maxcol <= kBlk) return false;
    if (gate == 3 && maxcol > kDsmemMaxcol) return false;
    if (gate == 6 && maxcol <= kDsmemMaxcol) return false;
    return true;
}

template <typename T, int MODEL, bool GEN = false>
__global__ void __launch_bounds__(kBlk) k_sweep(int64_t begin, int64_t end, int64_t cap, T dtinv,
                                                Cache<T> cc, BodyV<T> bv, int64_t nb,
                                                int track_delta, unsigned long long *delta) {
    const int64_t k = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= end) return;
    sweep_contact<T, MODEL, false, GEN>(k, dtinv, cc, bv, track_delta, delta);
}

// All sweeps of a step in one cooperative launch: colour after colour, separated by bounded
// grid barriers (each colour is conflict-free, so its contacts run in parallel).
template <typename T, int MODEL, bool GEN = false>
__global__ void __launch_bounds__(kBlk) k_sweeps_persistent(int iters, const int32_t *dd,
                                                            int gate,
                                                            const int32_t *color_start,
                                                            int64_t cap, T dtinv, Cache<T> cc,
                                                            BodyV<T> bv, int64_t nb,
                                                            int track_last,
                                                            unsigned long long *delta,
                                                            unsigned int *bar, int32_t *err) {
    if (!sweeps_gate(dd, gate)) return;
    const int ncolors = dd[kDdNcolors];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t g0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned int episode = 0;   // bar[0] was zeroed before the launch
    for (int it = 0; it < iters; ++it) {
        const int track = (track_last && it == iters - 1) ? 1 : 0;
        for (int col = 0; col < ncolors; ++col) {
            const int64_t e = color_start[col + 1];
            for (int64_t k = color_start[col] + g0; k < e; k += stride)
                sweep_contact<T, MODEL, true, GEN>(k, dtinv, cc, bv, track, delta);
            if (!grid_sync_counted(bar, episode, err)) return;
        }
    }
}

// The grid form with each block's contacts staged in its shared memory (relaxation models 0 and
// 1, sphere scenes): block b sweeps the b-th of G equal chunks of every colour, so it handles
// the same contacts in every sweep, and their records (ids, the solver records the model reads,
// the impulse) are copied into its shared memory before the sweeps (as many as fit, scap; the
// rest are read from global memory) and the impulses written back after.  A colour's contact
// then starts with its bodies' loads instead of first loading its own record from L2.
template <typename T, int MODEL>
__global__ void __launch_bounds__(kBlk) k_sweeps_grid_staged(int iters, const int32_t *dd,
                                                             int gate, const int32_t *color_start,
                                                             T dtinv, Cache<T> cc, BodyV<T> bv,
                                                             int scap, int track_last,
                                                             unsigned long long *delta,
                                                             unsigned int *bar, int32_t *err) {
    static_assert(MODEL <= 1, "staged records: relaxation models 0 and 1");
    constexpr int NREC = MODEL == 0 ? 3 : 7;
    if (!sweeps_gate(dd, gate)) return;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int32_t lo_s[kMaxColors], n_s[kMaxColors], off_s[kMaxColors];
    const int ncolors = dd[kDdNcolors];
    const int G = gridDim.x, r = blockIdx.x;
    if (threadIdx.x == 0) {
        int off = 0;
        for (int col = 0; col < ncolors; ++col) {
            const int64_t b0 = color_start[col], len = color_start[col + 1] - b0;
            const int lo = (int)(b0 + len * r / G), hi = (int)(b0 + len * (r + 1) / G);
            lo_s[col] = lo;
            n_s[col] = hi - lo;
            off_s[col] = off;
            off += hi - lo;
        }
    }
    SmemContacts<T, NREC> sc;
    sc.rec = (T4<T> *)smem;
    sc.p = sc.rec + (int64_t)NREC * scap;
    sc.ids = (int2 *)(sc.p + scap);
    __syncthreads();
    for (int col = 0; col < ncolors; ++col)
        for (int i = threadIdx.x; i < n_s[col]; i += blockDim.x) {
            const int local = off_s[col] + i;
            if (local >= scap) break;
            const int64_t k = lo_s[col] + i;
            sc.ids[local] = cc.ids[k];
            for (int q = 0; q < NREC; ++q) sc.rec[(int64_t)NREC * local + q] = cc.rec[(int64_t)kRec * k + q];
            sc.p[local] = cc.p[k];
        }
    __syncthreads();
    unsigned int episode = 0;   // bar[0] was zeroed before the launch
    for (int it = 0; it < iters; ++it) {
        const int track = (track_last && it == iters - 1) ? 1 : 0;
        for (int col = 0; col < ncolors; ++col) {
            const int n = n_s[col], lo = lo_s[col], off = off_s[col];
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                if (off + i < scap)
                    sweep_contact<T, MODEL, true, false, BodyV<T>, SmemContacts<T, NREC>>(
                        off + i, dtinv, sc, bv, track, delta);
                else
                    sweep_contact<T, MODEL, true, false>(lo + i, dtinv, cc, bv, track, delta);
            }
            if (!grid_sync_counted(bar, episode, err)) return;
        }
    }
    for (int col = 0; col < ncolors; ++col)
        for (int i = threadIdx.x; i < n_s[col]; i += blockDim.x) {
            const int local = off_s[col] + i;
            if (local >= scap) break;
            cc.p[lo_s[col] + i] = sc.p[local];
        }
}

// All sweeps of a step in one thread block, when every colour fits the block: the colours are
// separated by __syncthreads, and the body and impulse updates of a colour, made on this SM,
// are read back through its L1 by the next.  Scenes whose contacts crowd on few bodies (box
// stacks: dozens of contact points per box, so many colours of a few dozen contacts) spend most
// of a sweep on the barriers; this form makes a barrier cost a few dozen cycles.
template <typename T, int MODEL, bool GEN = false>
__global__ void __launch_bounds__(kBlk) k_sweeps_block(int iters, const int32_t *dd, int gate,
                                                       const int32_t *color_start, int64_t cap,
                                                       T dtinv, Cache<T> cc, BodyV<T> bv,
                                                       int64_t nb, int track_last,
                                                       unsigned long long *delta) {
    if (!sweeps_gate(dd, gate)) return;
    const int ncolors = dd[kDdNcolors];
    for (int it = 0; it < iters; ++it) {
        const int track = (track_last && it == iters - 1) ? 1 : 0;
        for (int col = 0; col < ncolors; ++col) {
            const int64_t e = color_start[col + 1];
            for (int64_t k = color_start[col] + threadIdx.x; k < e; k += blockDim.x)
                sweep_contact<T, MODEL, false, GEN>(k, dtinv, cc, bv, track, delta);
            __syncthreads();
        }
    }
}

// The single-block form with the bodies' velocity records in shared memory (when they fit):
// the updates of one colour reach the next colour's reads at shared-memory latency.  A
// contact's impulse is read and written by one thread only, so it stays in global memory.
template <typename T, int MODEL, bool GEN = false>
__global__ void __launch_bounds__(kBlk) k_sweeps_block_smem(int iters, const int32_t *dd,
                                                            int gate,
                                                            const int32_t *color_start,
                                                            int64_t cap, T dtinv, Cache<T> cc,
                                                            BodyV<T> bv, int64_t nbod,
                                                            int track_last,
                                                            unsigned long long *delta) {
    if (!sweeps_gate(dd, gate)) return;
    const int ncolors = dd[kDdNcolors];
    extern __shared__ __align__(16) unsigned char smem[];
    T4<T> *sh = (T4<T> *)smem;
    const int nrow = GEN ? 7 : 4;   // vr wr dv dw (ia ib ic)
    BodyV<T> sb;
    sb.vr = sh;
    sb.wr = sh + nbod;
    sb.dv = sh + 2 * nbod;
    sb.dw = sh + 3 * nbod;
    if (GEN) {
        sb.ia = sh + 4 * nbod;
        sb.ib = sh + 5 * nbod;
        sb.ic = sh + 6 * nbod;
    }
    (void)nrow;
    for (int64_t i = threadIdx.x; i < nbod; i += blockDim.x) {
        sb.vr[i] = bv.vr[i];
        sb.wr[i] = bv.wr[i];
        sb.dv[i] = bv.dv[i];
        sb.dw[i] = bv.dw[i];
        if (GEN) {
            sb.ia[i] = bv.ia[i];
            sb.ib[i] = bv.ib[i];
            sb.ic[i] = bv.ic[i];
        }
    }
    __syncthreads();
    for (int it = 0; it < iters; ++it) {
        const int track = (track_last && it == iters - 1) ? 1 : 0;
        for (int col = 0; col < ncolors; ++col) {
            const int64_t e = color_start[col + 1];
            for (int64_t k = color_start[col] + threadIdx.x; k < e; k += blockDim.x)
                sweep_contact<T, MODEL, false, GEN>(k, dtinv, cc, sb, track, delta);
            __syncthreads();
        }
    }
    for (int64_t i = threadIdx.x; i < nbod; i += blockDim.x) {
        bv.dv[i] = sb.dv[i];
        bv.dw[i] = sb.dw[i];
    }
}

// All sweeps of a step in one thread block with only the bodies that have contacts in shared
// memory (sphere scenes with at most kCompactMax contacts, every colour within the block): a
// scene of thousands of bodies and a few contacts sweeps at shared-memory latency, where the
// whole-scene form cannot hold its bodies.  Each body gets a slot: the first of its contacts to
// claim it (atomic compare-and-swap on slot_of, which holds -1 for every body outside this
// kernel) loads its records; the claims are undone at the end.
template <typename T, int MODEL>
__global__ void __launch_bounds__(kBlk) k_sweeps_compact(int iters, const int32_t *dd, int gate,
                                                         const int32_t *color_start, T dtinv,
                                                         Cache<T> cc, BodyV<T> bv,
                                                         int32_t *slot_of, int track_last,
                                                         unsigned long long *delta) {
    if (!sweeps_gate(dd, gate)) return;
    const int nc = dd[kDdNc];
    if (nc > kCompactMax) return;   // the gate of the host-driven launch (0) does not check it
    const int ncolors = dd[kDdNcolors];
    constexpr int bcap = 2 * kCompactMax;
    extern __shared__ __align__(16) unsigned char smem[];
    T4<T> *sh = (T4<T> *)smem;
    int32_t *sbody = (int32_t *)(sh + 4 * bcap);     // slot -> body
    int2 *sids = (int2 *)(sbody + bcap);              // contact -> its bodies' slots
    int32_t *claim = (int32_t *)(sids + kCompactMax); // claim (2 k + side) -> slot
    __shared__ int32_t cs[kMaxColors + 1];
    __shared__ int nslots;
    if (threadIdx.x == 0) nslots = 0;
    for (int i = threadIdx.x; i <= ncolors; i += blockDim.x) cs[i] = color_start[i];
    __syncthreads();
    for (int k = threadIdx.x; k < nc; k += blockDim.x) {
        const int2 id = cc.ids[k];
        if (atomicCAS(&slot_of[id.x], -1, 2 * k) == -1) {
            const int sl = atomicAdd(&nslots, 1);
            claim[2 * k] = sl;
            sbody[sl] = id.x;
        }
        if (id.y >= 0 && atomicCAS(&slot_of[id.y], -1, 2 * k + 1) == -1) {
            const int sl = atomicAdd(&nslots, 1);
            claim[2 * k + 1] = sl;
            sbody[sl] = id.y;
        }
    }
    __syncthreads();
    const int ns = nslots;
    for (int sl = threadIdx.x; sl < ns; sl += blockDim.x) {
        const int32_t b = sbody[sl];
        sh[sl] = bv.vr[b];
        sh[bcap + sl] = bv.wr[b];
        sh[2 * bcap + sl] = bv.dv[b];
        sh[3 * bcap + sl] = bv.dw[b];
    }
    for (int k = threadIdx.x; k < nc; k += blockDim.x) {
        const int2 id = cc.ids[k];
        const int s1 = claim[__ldcg(slot_of + id.x)];
        const int s2 = id.y >= 0 ? claim[__ldcg(slot_of + id.y)] : -1;
        sids[k] = make_int2(s1, s2);
    }
    __syncthreads();
    BodyV<T> sb;
    sb.vr = sh;
    sb.wr = sh + bcap;
    sb.dv = sh + 2 * bcap;
    sb.dw = sh + 3 * bcap;
    const CompactContacts<T> ccs{sids, cc.rec, cc.p, cc.dc};
    for (int it = 0; it < iters; ++it) {
        const int track = (track_last && it == iters - 1) ? 1 : 0;
        for (int col = 0; col < ncolors; ++col) {
            const int e = cs[col + 1];
            for (int k = cs[col] + threadIdx.x; k < e; k += blockDim.x)
                sweep_contact<T, MODEL, false, false, BodyV<T>, CompactContacts<T>>(k, dtinv, ccs, sb,
                                                                                    track, delta);
            __syncthreads();
        }
    }
    for (int sl = threadIdx.x; sl < ns; sl += blockDim.x) {
        const int32_t b = sbody[sl];
        bv.dv[b] = sh[2 * bcap + sl];
        bv.dw[b] = sh[3 * bcap + sl];
        slot_of[b] = -1;
    }
}

template <typename T>
constexpr size_t compact_smem() {
    return (size_t)4 * 2 * kCompactMax * sizeof(T4<T>) + (size_t)2 * kCompactMax * 4 +
           (size_t)kCompactMax * 8 + (size_t)2 * kCompactMax * 4;
}

// All sweeps of a step inside one thread-block cluster: the colours are separated by the
// cluster's hardware barrier (release/acquire at cluster scope) instead of a barrier through
// global atomics, which costs a few microseconds per colour.  Used while the largest colour
// fits the cluster's threads a few times over; no thread waits on anything but the barrier.
constexpr int kClusterBlk = 512;
constexpr int kClusterPerThread = 4;

template <typename T, int MODEL>
__global__ void __launch_bounds__(kClusterBlk) k_sweeps_cluster(int iters, int ncolors,
                                                                const int32_t *color_start,
                                                                int64_t cap, T dtinv, Cache<T> cc,
                                                                BodyV<T> bv, int64_t nb,
                                                                int track_last,
                                                                unsigned long long *delta) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;   // the grid is one cluster
    const int64_t g0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int it = 0; it < iters; ++it) {
        const int track = (track_last && it == iters - 1) ? 1 : 0;
        for (int col = 0; col < ncolors; ++col) {
            const int64_t e = color_start[col + 1];
            for (int64_t k = color_start[col] + g0; k < e; k += stride)
                sweep_contact<T, MODEL, true>(k, dtinv, cc, bv, track, delta);
            cluster.sync();
        }
    }
}

// All sweeps of a step inside one thread-block cluster with the bodies' records in the
// cluster's distributed shared memory (ClusterBodies: body b in CTA b mod C), so that a
// colour's body loads and stores take a shared-memory round trip across the cluster instead of
// an L2 round trip, and the colours are separated by the cluster's hardware barrier.  CTA r
// sweeps the r-th of C equal chunks of every colour.  STAGE (relaxation models 0 and 1): the
// records of the CTA's contacts are copied into its shared memory before the sweeps (as many as
// fit, scap; the rest are read from global memory) and their impulses written back after, so a
// colour touches no global memory.  Every CTA reaches the same barriers (the colour loop is
// uniform across the cluster), and the gate is read from device memory that no kernel of this
// launch writes, so all CTAs agree on it.
constexpr int kDsBlk = 512;

template <typename T, int MODEL, bool STAGE>
__global__ void __launch_bounds__(kDsBlk) k_sweeps_dsmem(int iters, const int32_t *dd, int gate,
                                                         const int32_t *color_start, int64_t cap,
                                                         T dtinv, Cache<T> cc, BodyV<T> bv,
                                                         int64_t nbod, int per, int shift,
                                                         int scap, int track_last,
                                                         unsigned long long *delta) {
    namespace cg = cooperative_groups;
    static_assert(!STAGE || MODEL <= 1, "staged records: relaxation models 0 and 1");
    constexpr int NREC = MODEL == 0 ? 3 : 7;
    if (!sweeps_gate(dd, gate)) return;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int32_t lo_s[kMaxColors], n_s[kMaxColors], off_s[kMaxColors];
    T4<T> *sh = (T4<T> *)smem;
    const int ncolors = dd[kDdNcolors];
    const int rank = (int)cluster.block_rank();
    const int C = 1 << shift;
    if (threadIdx.x == 0) {
        int off = 0;
        for (int col = 0; col < ncolors; ++col) {
            const int64_t b0 = color_start[col], len = color_start[col + 1] - b0;
            const int lo = (int)(b0 + len * rank / C), hi = (int)(b0 + len * (rank + 1) / C);
            lo_s[col] = lo;
            n_s[col] = hi - lo;
            off_s[col] = off;
            off += hi - lo;
        }
    }
    for (int j = threadIdx.x; j < per; j += blockDim.x) {
        const int64_t b = ((int64_t)j << shift) + rank;
        if (b < nbod) {
            sh[j] = bv.vr[b];
            sh[per + j] = bv.wr[b];
            sh[2 * per + j] = bv.dv[b];
            sh[3 * per + j] = bv.dw[b];
        }
    }
    SmemContacts<T, NREC> sc;
    sc.rec = sh + 4 * (int64_t)per;
    sc.p = sc.rec + (int64_t)NREC * scap;
    sc.ids = (int2 *)(sc.p + scap);
    __syncthreads();
    if (STAGE) {
        for (int col = 0; col < ncolors; ++col)
            for (int i = threadIdx.x; i < n_s[col]; i += blockDim.x) {
                const int local = off_s[col] + i;
                if (local >= scap) break;
                const int64_t k = lo_s[col] + i;
                sc.ids[local] = cc.ids[k];
                for (int q = 0; q < NREC; ++q) sc.rec[(int64_t)NREC * local + q] = cc.rec[(int64_t)kRec * k + q];
                sc.p[local] = cc.p[k];
            }
    }
    cluster.sync();
    ClusterBodies<T> cb{(uint32_t)__cvta_generic_to_shared(sh), per, shift};
    for (int it = 0; it < iters; ++it) {
        const int track = (track_last && it == iters - 1) ? 1 : 0;
        for (int col = 0; col < ncolors; ++col) {
            const int n = n_s[col], lo = lo_s[col], off = off_s[col];
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                if (STAGE && off + i < scap)
                    sweep_contact<T, MODEL, false, false, ClusterBodies<T>, SmemContacts<T, NREC>>(
                        off + i, dtinv, sc, cb, track, delta);
                else
                    sweep_contact<T, MODEL, false, false, ClusterBodies<T>>(lo + i, dtinv, cc, cb,
                                                                           track, delta);
            }
            cluster.sync();
        }
    }
    for (int j = threadIdx.x; j < per; j += blockDim.x) {
        const int64_t b = ((int64_t)j << shift) + rank;
        if (b < nbod) {
            bv.dv[b] = sh[2 * per + j];
            bv.dw[b] = sh[3 * per + j];
        }
    }
    if (STAGE) {
        for (int col = 0; col < ncolors; ++col)
            for (int i = threadIdx.x; i < n_s[col]; i += blockDim.x) {
                const int local = off_s[col] + i;
                if (local >= scap) break;
                cc.p[lo_s[col] + i] = sc.p[local];
            }
    }
}

// complementarity residual of the final impulses (same definition as the oracle), in FP64
template <typename T, bool FRICTION>
__global__ void k_residual(const int32_t *ncp, int64_t cap, double dtinv, Cache<T> cc,
                           BodyV<T> bv, int64_t nb, unsigned long long *res) {
    const int64_t nc = *ncp;
    GRID_STRIDE(k, nc) {
    const int2 ids = cc.ids[k];
    const int32_t b1 = ids.x, b2 = ids.y;
    auto D3 = [](const T4<T> &q) { return v3(double(q.x), double(q.y), double(q.z)); };
    const T4<T> *R = cc.rec + (int64_t)kRec * k;
    const V3<double> n = D3(R[0]), r1 = D3(R[1]), r2 = D3(R[2]), t = D3(R[3]), o = D3(R[4]);
    V3<double> a = D3(bv.vr[b1]) + D3(bv.dv[b1]), wa = D3(bv.wr[b1]) + D3(bv.dw[b1]);
    V3<double> b = v3(0.0, 0.0, 0.0), wb = b;
    if (b2 >= 0) {
        b = D3(bv.vr[b2]) + D3(bv.dv[b2]);
        wb = D3(bv.wr[b2]) + D3(bv.dw[b2]);
    }
    const V3<double> gdot = ((a - b) + cross(wa, r1)) - cross(wb, r2);
    const double gn = dot(n, gdot) + double(R[0].w) * dtinv;
    const V3<double> pc = D3(cc.p[k]);
    const double pn = pc.x, Dnn = double(R[2].w);
    double r = fabs(fmin(pn * Dnn, gn));
    if (FRICTION) {
        const double pt = pc.y, po = pc.z, gt = dot(t, gdot), go = dot(o, gdot);
        const double pto = sqrt(pt * pt + po * po), gto = sqrt(gt * gt + go * go);
        const double mu = double(R[3].w);
        r = fmax(r, fmax(0.0, pto - mu * pn) * Dnn);
        // an impulse projected onto the cone lands on it up to the rounding of the impulse's
        // own type: FP32 impulses within 1e-5 of mu p_n count as on the cone (sliding)
        const double on_cone = sizeof(T) == 4 ? 1e-5 : 1e-9;
        if (pn > 0.0) {
            if (pto < mu * pn * (1.0 - on_cone)) r = fmax(r, gto);
            else if (pto > 0.0) r = fmax(r, gto + (pt * gt + po * go) / pto);
        }
    }
    atomicMax(res, (unsigned long long)__double_as_longlong(r));
    }
}

// After a capacity abort (dd[kDdAbort]) the state is copied unchanged instead (the step does
// nothing and is run again); otherwise thread 0 counts the step in dd[kDdSteps].
template <typename VT, bool TRACKQ>
__global__ void k_integrate(int64_t n, double dt, double drag, int has_drag, BodyV<VT> bv,
                            const SceneInfo *scenes, const double4 *pr, const VT *vw,
                            const uint32_t *tag, const int32_t *uid, const double4 *q,
                            double4 *pr_o, VT *vw_o, uint32_t *tag_o, int32_t *uid_o,
                            double4 *q_o, int32_t *key, int32_t *rank, int32_t *cell_count,
                            int32_t *dd, int32_t *err) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    if (dd[kDdAbort]) {
        const double4 p = pr[t];
        pr_o[t] = p;
        cp_vw(vw_o, t, vw, t, n);
        const uint32_t tg = tag[t];
        tag_o[t] = tg;
        uid_o[t] = uid[t];
        if (TRACKQ) q_o[t] = q[t];
        const SceneInfo &s = scenes[tg >> 16];
        int cx, cy, cz;
        cell_coords(s, p.x, p.y, p.z, cx, cy, cz);
        const int32_t kk = (int32_t)cell_key(s, cx, cy, cz);
        key[t] = kk;
        rank[t] = atomicAdd(&cell_count[kk], 1);
        return;
    }
    if (t == 0) dd[kDdSteps] += 1;
    V3<VT> v = xyz<VT>(bv.vr[t]) + xyz<VT>(bv.dv[t]);
    V3<VT> w = xyz<VT>(bv.wr[t]) + xyz<VT>(bv.dw[t]);
    const double4 p = pr[t];
    const double nx = p.x + double(v.x) * dt, ny = p.y + double(v.y) * dt, nz = p.z + double(v.z) * dt;
    if (TRACKQ) {
        const double phx = double(w.x) * dt, phy = double(w.y) * dt, phz = double(w.z) * dt;
        const double ang = sqrt(phx * phx + phy * phy + phz * phz);
        double d0 = 1.0, d1 = 0.0, d2 = 0.0, d3 = 0.0;
        if (!(fabs(ang) < 1e-15)) {
            double sa, ca;
            sincos(ang * 0.5, &sa, &ca);
            const double il = 1.0 / ang;
            d0 = ca; d1 = sa * (phx * il); d2 = sa * (phy * il); d3 = sa * (phz * il);
        }
        const double4 qq = q[t];
        double4 r;
        r.x = d0 * qq.x - d1 * qq.y - d2 * qq.z - d3 * qq.w;
        r.y = d0 * qq.y + d1 * qq.x + d2 * qq.w - d3 * qq.z;
        r.z = d0 * qq.z + d2 * qq.x + d3 * qq.y - d1 * qq.w;
        r.w = d0 * qq.w + d3 * qq.x + d1 * qq.z - d2 * qq.y;
        q_o[t] = r;
    }
    if (has_drag) {
        v = v * VT(drag);
        w = w * VT(drag);
    }
    pr_o[t] = make_double4(nx, ny, nz, p.w);
    st_vw(vw_o, n, t, v, w);
    const uint32_t tg = tag[t];
    tag_o[t] = tg;
    uid_o[t] = uid[t];
    if (!isfinite(nx) || !isfinite(ny) || !isfinite(nz)) atomicOr(err, DERR_NAN);
    const SceneInfo &s = scenes[tg >> 16];
    int cx, cy, cz;
    cell_coords(s, nx, ny, nz, cx, cy, cz);
    const int32_t kk = (int32_t)cell_key(s, cx, cy, cz);
    key[t] = kk;
    rank[t] = atomicAdd(&cell_count[kk], 1);
}

// ---- buffers -------------------------------------------------------------------------------
int nbgs_alloc(Ctx *c, int64_t cap) {
    NbgsBuf &b = c->nb;
    const size_t es = (c->p.precision == PE_B200_FP64) ? 8 : 4;
    const int64_t n = std::max<int64_t>(c->n, 1);
    const bool gen = c->mb.m > 0;
    const int64_t nbod = n + c->mb.m;
    // graphs captured on the buffers replaced below are never launched again
    if (b.cap < cap || (b.cnt && (b.nbod != nbod || b.gen != gen))) nbgs_graph_free(c);
    if (b.cap < cap) {
        dfree(c, b.cache);
        b.cache = nullptr;
        dfree(c, b.order);
        b.order = nullptr;
        dfree(c, b.color);
        b.color = nullptr;
        dfree(c, b.body_adj);
        b.body_adj = nullptr;
        // raw: 2 int + 11 T; cache: 2 int + (kRec + 3) x 4 T  (per contact)
        const size_t bytes = (size_t)cap * (4 * sizeof(int32_t) + (11 + 4 * (kRec + 3)) * es) + 64 * 256;
        PEB_CUDA(c, dmalloc(c, &b.cache, bytes));
        PEB_CUDA(c, dmalloc(c, &b.order, (size_t)cap * sizeof(int32_t)));
        PEB_CUDA(c, dmalloc(c, &b.color, (size_t)cap * sizeof(int32_t)));
        PEB_CUDA(c, dmalloc(c, &b.body_adj, (size_t)2 * cap * sizeof(int32_t)));
        b.cap = cap;
    }
    // per-body buffers: spheres, then moving boxes (with inverse inertia rows, GEN)
    if (b.cnt && (b.nbod != nbod || b.gen != gen)) {
        dfree(c, b.cnt);
        dfree(c, b.body_cnt);
        dfree(c, b.used);
        dfree(c, b.vel);
        b.cnt = b.body_cnt = nullptr;
        b.used = nullptr;
        b.vel = nullptr;
        dfree(c, b.flags);
        dfree(c, b.red);
        dfree(c, b.cstart_dev);
        dfree(c, b.bar);
        dfree(c, b.dd);
        dfree(c, b.rem);
        dfree(c, b.bar2);
        dfree(c, b.slot_of);
        b.slot_of = nullptr;
        if (b.color_start) cudaFreeHost(b.color_start);
        if (b.h_dd) cudaFreeHost(b.h_dd);
        b.flags = nullptr;
        b.red = nullptr;
        b.cstart_dev = nullptr;
        b.bar = nullptr;
        b.dd = b.rem = nullptr;
        b.bar2 = nullptr;
        b.color_start = nullptr;
        b.h_dd = nullptr;
    }
    if (!b.cnt) {
        b.nbod = nbod;
        b.gen = gen;
        PEB_CUDA(c, dmalloc(c, &b.cnt, ((size_t)nbod + 2) * sizeof(int32_t)));
        PEB_CUDA(c, dmalloc(c, &b.body_cnt, ((size_t)nbod + 2) * sizeof(int32_t)));
        PEB_CUDA(c, dmalloc(c, &b.used, (size_t)nbod * (gen ? 4 : 1) * sizeof(uint64_t)));
        PEB_CUDA(c, dmalloc(c, &b.vel, (size_t)nbod * (gen ? 28 : 16) * es));
        PEB_CUDA(c, dmalloc(c, &b.flags, (3 * kMaxColors + 8) * sizeof(int32_t)));
        PEB_CUDA(c, cudaMallocHost(&b.color_start, (2 * kMaxColors + 8) * sizeof(int32_t)));
        PEB_CUDA(c, dmalloc(c, &b.red, 4 * sizeof(double)));
        PEB_CUDA(c, dmalloc(c, &b.cstart_dev, (kMaxColors + 2) * sizeof(int32_t)));
        PEB_CUDA(c, dmalloc(c, &b.bar, 2 * sizeof(unsigned int)));
        PEB_CUDA(c, cudaMemsetAsync(b.bar, 0, 2 * sizeof(unsigned int), c->stream));
        PEB_CUDA(c, dmalloc(c, &b.dd, kDdCount * sizeof(int32_t)));
        PEB_CUDA(c, cudaMemsetAsync(b.dd, 0, kDdCount * sizeof(int32_t), c->stream));
        PEB_CUDA(c, cudaMallocHost(&b.h_dd, kDdCount * sizeof(int32_t)));
        memset(b.h_dd, 0, kDdCount * sizeof(int32_t));
        PEB_CUDA(c, dmalloc(c, &b.rem, kMaxRounds * sizeof(int32_t)));
        PEB_CUDA(c, dmalloc(c, &b.slot_of, (size_t)nbod * sizeof(int32_t)));
        PEB_CUDA(c, cudaMemsetAsync(b.slot_of, 0xff, (size_t)nbod * sizeof(int32_t), c->stream));
        PEB_CUDA(c, dmalloc(c, &b.bar2, 2 * sizeof(unsigned int)));
        PEB_CUDA(c, cudaMemsetAsync(b.bar2, 0, 2 * sizeof(unsigned int), c->stream));
    }
    return PE_B200_OK;
}

template <typename T>
void layout(Ctx *c, Raw<T> &raw, Cache<T> &cc, BodyV<T> &bv) {
    NbgsBuf &b = c->nb;
    const int64_t cap = b.cap;
    char *p = (char *)b.cache;
    auto take = [&](size_t bytes) {
        char *q = p;
        p += (bytes + 255) & ~(size_t)255;
        return q;
    };
    raw.b1 = (int32_t *)take(cap * 4);
    raw.b2 = (int32_t *)take(cap * 4);
    raw.r1 = (T *)take(3 * cap * sizeof(T));
    raw.r2 = (T *)take(3 * cap * sizeof(T));
    raw.n = (T *)take(3 * cap * sizeof(T));
    raw.dist = (T *)take(cap * sizeof(T));
    raw.mu = (T *)take(cap * sizeof(T));
    cc.ids = (int2 *)take(cap * sizeof(int2));
    cc.rec = (T4<T> *)take(kRec * cap * sizeof(T4<T>));
    cc.p = (T4<T> *)take(cap * sizeof(T4<T>));
    cc.dc = (T4<T> *)take(2 * cap * sizeof(T4<T>));
    const int64_t n = b.nbod;
    T4<T> *v = (T4<T> *)b.vel;
    bv.vr = v;
    bv.wr = v + n;
    bv.dv = v + 2 * n;
    bv.dw = v + 3 * n;
    if (b.gen) {
        bv.ia = v + 4 * n;
        bv.ib = v + 5 * n;
        bv.ic = v + 6 * n;
    } else {
        bv.ia = bv.ib = bv.ic = nullptr;
    }
}

// the sweep kernels of relaxation model m (pe's RelaxationModel 0-5)
template <typename VT>
auto cluster_kernel(int m) -> decltype(&k_sweeps_cluster<VT, 0>) {
    switch (m) {
        case 1: return k_sweeps_cluster<VT, 1>;
        case 2: return k_sweeps_cluster<VT, 2>;
        case 3: return k_sweeps_cluster<VT, 3>;
        case 4: return k_sweeps_cluster<VT, 4>;
        case 5: return k_sweeps_cluster<VT, 5>;
        default: return k_sweeps_cluster<VT, 0>;
    }
}
template <typename VT, bool GEN>
auto persistent_kernel_g(int m) -> decltype(&k_sweeps_persistent<VT, 0, GEN>) {
    switch (m) {
        case 1: return k_sweeps_persistent<VT, 1, GEN>;
        case 2: return k_sweeps_persistent<VT, 2, GEN>;
        case 3: return k_sweeps_persistent<VT, 3, GEN>;
        case 4: return k_sweeps_persistent<VT, 4, GEN>;
        case 5: return k_sweeps_persistent<VT, 5, GEN>;
        default: return k_sweeps_persistent<VT, 0, GEN>;
    }
}
// gen: bodies with a full inverse inertia (moving boxes; FP64 only)
template <typename VT>
auto persistent_kernel(int m, bool gen) -> decltype(&k_sweeps_persistent<VT, 0, false>) {
    if constexpr (std::is_same<VT, double>::value) {
        if (gen) return persistent_kernel_g<VT, true>(m);
    }
    return persistent_kernel_g<VT, false>(m);
}
template <typename VT, bool GEN>
auto block_kernel_g(int m) -> decltype(&k_sweeps_block<VT, 0, GEN>) {
    switch (m) {
        case 1: return k_sweeps_block<VT, 1, GEN>;
        case 2: return k_sweeps_block<VT, 2, GEN>;
        case 3: return k_sweeps_block<VT, 3, GEN>;
        case 4: return k_sweeps_block<VT, 4, GEN>;
        case 5: return k_sweeps_block<VT, 5, GEN>;
        default: return k_sweeps_block<VT, 0, GEN>;
    }
}
template <typename VT>
auto block_kernel(int m, bool gen) -> decltype(&k_sweeps_block<VT, 0, false>) {
    if constexpr (std::is_same<VT, double>::value) {
        if (gen) return block_kernel_g<VT, true>(m);
    }
    return block_kernel_g<VT, false>(m);
}
template <typename VT, bool GEN>
auto block_smem_kernel_g(int m) -> decltype(&k_sweeps_block_smem<VT, 0, GEN>) {
    switch (m) {
        case 1: return k_sweeps_block_smem<VT, 1, GEN>;
        case 2: return k_sweeps_block_smem<VT, 2, GEN>;
        case 3: return k_sweeps_block_smem<VT, 3, GEN>;
        case 4: return k_sweeps_block_smem<VT, 4, GEN>;
        case 5: return k_sweeps_block_smem<VT, 5, GEN>;
        default: return k_sweeps_block_smem<VT, 0, GEN>;
    }
}
template <typename VT>
auto block_smem_kernel(int m, bool gen) -> decltype(&k_sweeps_block_smem<VT, 0, false>) {
    if constexpr (std::is_same<VT, double>::value) {
        if (gen) return block_smem_kernel_g<VT, true>(m);
    }
    return block_smem_kernel_g<VT, false>(m);
}
template <typename VT, bool GEN>
auto colour_kernel_g(int m) -> decltype(&k_sweep<VT, 0, GEN>) {
    switch (m) {
        case 1: return k_sweep<VT, 1, GEN>;
        case 2: return k_sweep<VT, 2, GEN>;
        case 3: return k_sweep<VT, 3, GEN>;
        case 4: return k_sweep<VT, 4, GEN>;
        case 5: return k_sweep<VT, 5, GEN>;
        default: return k_sweep<VT, 0, GEN>;
    }
}
template <typename VT>
auto colour_kernel(int m, bool gen) -> decltype(&k_sweep<VT, 0, false>) {
    if constexpr (std::is_same<VT, double>::value) {
        if (gen) return colour_kernel_g<VT, true>(m);
    }
    return colour_kernel_g<VT, false>(m);
}

// Runs all sweeps in one cluster when the largest colour is small enough; *done reports it.
// The cluster size (16 CTAs if the GPU schedules such clusters, else 8) is probed once.
template <typename VT>
int sweeps_in_cluster(Ctx *c, int model, int iters, int ncolors, int maxcol, int64_t cap, VT dtinv,
                      const Cache<VT> &cc, const BodyV<VT> &bv, int64_t n,
                      unsigned long long *dl, bool *done) {
    NbgsBuf &nb = c->nb;
    auto kern = cluster_kernel<VT>(model);
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    cfg.blockDim = dim3(kClusterBlk);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = c->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (nb.cluster < 0) {
        nb.cluster = 0;
        for (int size : {16, 8}) {
            auto probe = cluster_kernel<VT>(model);
            if (size > 8 &&
                cudaFuncSetAttribute((const void *)probe, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            if (size > 8) {
                cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
                cudaGetLastError();
            }
            cfg.gridDim = dim3(size);
            attr[0].val.clusterDim.x = size;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, (const void *)probe, &cfg) == cudaSuccess &&
                nclusters >= 1) {
                nb.cluster = size;
                break;
            }
            cudaGetLastError();
        }
    }
    if (nb.cluster == 0 || maxcol > (int64_t)nb.cluster * kClusterBlk * kClusterPerThread)
        return PE_B200_OK;
    PEB_CUDA(c, cudaMemcpyAsync(nb.cstart_dev, nb.color_start, (ncolors + 1) * sizeof(int32_t),
                                cudaMemcpyHostToDevice, c->stream));
    if (nb.cluster > 8) {
        cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        cudaGetLastError();
    }
    cfg.gridDim = dim3(nb.cluster);
    attr[0].val.clusterDim.x = nb.cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, iters, ncolors, (const int32_t *)nb.cstart_dev,
                                             cap, dtinv, cc, bv, n, c->want_residual ? 1 : 0, dl);
    if (e != cudaSuccess) {
        cudaGetLastError();
        nb.cluster = 0;
        return PE_B200_OK;
    }
    c->launches++;
    *done = true;
    return PE_B200_OK;
}

// Launches k_sweeps_grid_staged (sphere scenes, relaxation models 0 and 1) as one cooperative
// grid of `blocks` blocks (at most one per SM: each holds as many staged contacts as its shared
// memory takes); *done reports it.
template <typename VT>
int launch_sweeps_grid_staged(Ctx *c, int model, int iters, int gate, VT dtinv,
                              const Cache<VT> &cc, const BodyV<VT> &bv, int track,
                              unsigned long long *dl, int64_t blocks, bool *done) {
    NbgsBuf &nb = c->nb;
    *done = false;
    if (nb.gen || model > 1 || nb.staged_off || nb.coop_disabled) return PE_B200_OK;
    auto kern = model == 0 ? k_sweeps_grid_staged<VT, 0> : k_sweeps_grid_staged<VT, 1>;
    const int64_t rec_bytes = (model == 0 ? 3 : 7) * (int64_t)sizeof(T4<VT>) +
                              (int64_t)sizeof(T4<VT>) + (int64_t)sizeof(int2);
    if (nb.ds_optin == 0) cudaDeviceGetAttribute(&nb.ds_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    const int64_t room = (int64_t)nb.ds_optin - (3 * kMaxColors * 4 + 1024);
    const int64_t scap = room / rec_bytes;
    const size_t bytes = (size_t)(scap * rec_bytes);
    if (scap < 256 || cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)bytes) != cudaSuccess) {
        cudaGetLastError();
        nb.staged_off = true;
        return PE_B200_OK;
    }
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kBlk, bytes) != cudaSuccess || occ < 1) {
        cudaGetLastError();
        nb.staged_off = true;
        return PE_B200_OK;
    }
    // the barrier counter counts iters x colours x blocks arrivals: past 2^32 the grid shrinks
    const int64_t g = std::max<int64_t>(
        1, std::min<int64_t>(std::min<int64_t>(blocks, (int64_t)occ * c->sm_count),
                             (int64_t)(4.0e9 / ((double)std::max(iters, 1) * kMaxColors))));
    PEB_CUDA(c, cudaMemsetAsync(nb.bar, 0, sizeof(unsigned int), c->stream));
    int iters_a = iters, gate_a = gate, scap_a = (int)scap, track_a = track;
    VT dtinv_a = dtinv;
    const int32_t *dd = nb.dd, *cs = nb.cstart_dev;
    Cache<VT> cc_a = cc;
    BodyV<VT> bv_a = bv;
    void *args[] = {&iters_a, &dd, &gate_a, &cs, &dtinv_a, &cc_a, &bv_a, &scap_a, &track_a, &dl,
                    &nb.bar, &c->d_err};
    const cudaError_t e = cudaLaunchCooperativeKernel((const void *)kern, dim3((unsigned)g),
                                                      dim3(kBlk), args, bytes, c->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        nb.staged_off = true;
        return PE_B200_OK;
    }
    c->launches++;
    *done = true;
    return PE_B200_OK;
}

template <typename VT>
auto compact_kernel(int m) -> decltype(&k_sweeps_compact<VT, 0>) {
    switch (m) {
        case 1: return k_sweeps_compact<VT, 1>;
        case 2: return k_sweeps_compact<VT, 2>;
        case 3: return k_sweeps_compact<VT, 3>;
        case 4: return k_sweeps_compact<VT, 4>;
        case 5: return k_sweeps_compact<VT, 5>;
        default: return k_sweeps_compact<VT, 0>;
    }
}

// Launches k_sweeps_compact (sphere scenes); *done reports it.
template <typename VT>
int launch_sweeps_compact(Ctx *c, int model, int iters, int gate, VT dtinv, const Cache<VT> &cc,
                          const BodyV<VT> &bv, int track, unsigned long long *dl, bool *done) {
    NbgsBuf &nb = c->nb;
    *done = false;
    if (nb.gen || !nb.slot_of || nb.compact_off) return PE_B200_OK;
    auto kern = compact_kernel<VT>(model);
    constexpr size_t bytes = compact_smem<VT>();
    if (cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)bytes) != cudaSuccess) {
        cudaGetLastError();
        nb.compact_off = true;
        return PE_B200_OK;
    }
    kern<<<1, kBlk, bytes, c->stream>>>(iters, nb.dd, gate, nb.cstart_dev, dtinv, cc, bv,
                                         nb.slot_of, track, dl);
    PEB_LAUNCHED(c);
    *done = true;
    return PE_B200_OK;
}

template <typename VT>
auto dsmem_kernel(int m, bool stage) -> decltype(&k_sweeps_dsmem<VT, 0, false>) {
    if (stage && m == 0) return k_sweeps_dsmem<VT, 0, true>;
    if (stage && m == 1) return k_sweeps_dsmem<VT, 1, true>;
    switch (m) {
        case 1: return k_sweeps_dsmem<VT, 1, false>;
        case 2: return k_sweeps_dsmem<VT, 2, false>;
        case 3: return k_sweeps_dsmem<VT, 3, false>;
        case 4: return k_sweeps_dsmem<VT, 4, false>;
        case 5: return k_sweeps_dsmem<VT, 5, false>;
        default: return k_sweeps_dsmem<VT, 0, false>;
    }
}

// Launches k_sweeps_dsmem when the bodies' records fit the shared memory of one cluster (16
// CTAs where the GPU schedules such clusters, else 8), with as many of its contacts' records
// staged beside them as fit; *done reports it.  The plan for a (model, precision, body count)
// is probed once and kept.
template <typename VT>
int launch_sweeps_dsmem(Ctx *c, int model, int iters, int gate, int64_t cap, VT dtinv,
                        const Cache<VT> &cc, const BodyV<VT> &bv, int track,
                        unsigned long long *dl, bool *done) {
    NbgsBuf &nb = c->nb;
    *done = false;
    if (nb.gen) return PE_B200_OK;
    const int key = model * 2 + (sizeof(VT) == 8 ? 1 : 0);
    const bool can_stage = model <= 1;
    const int64_t rec_bytes = (model == 0 ? 3 : 7) * (int64_t)sizeof(T4<VT>) + (int64_t)sizeof(T4<VT>) +
                              (int64_t)sizeof(int2);
    constexpr int64_t kStatic = 3 * kMaxColors * 4 + 1024;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(kDsBlk);
    cfg.stream = c->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    auto plan = [&](int size, int64_t &per, int64_t &scap, int64_t &bytes, int optin) {
        per = (nb.nbod + size - 1) / size;
        const int64_t body_bytes = 4 * per * (int64_t)sizeof(T4<VT>);
        const int64_t room = (int64_t)optin - kStatic - body_bytes;
        scap = can_stage && room > 0 ? room / rec_bytes : 0;
        if (scap < 64) scap = 0;
        bytes = body_bytes + scap * rec_bytes;
        return room >= 0;
    };
    if (nb.ds_nbod != nb.nbod || nb.ds_key != key) {
        nb.ds_nbod = nb.nbod;
        nb.ds_key = key;
        nb.ds_size = 0;
        int optin = 0;
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
        nb.ds_optin = optin;
        for (int size : {16, 8}) {
            int64_t per, scap, bytes;
            if (!plan(size, per, scap, bytes, optin)) continue;
            auto kern = dsmem_kernel<VT>(model, scap > 0);
            if (size > 8 && cudaFuncSetAttribute((const void *)kern,
                                                 cudaFuncAttributeNonPortableClusterSizeAllowed,
                                                 1) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            if (cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)bytes) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            cfg.gridDim = dim3(size);
            cfg.dynamicSmemBytes = (size_t)bytes;
            attr[0].val.clusterDim.x = size;
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, (const void *)kern, &cfg) == cudaSuccess &&
                nclusters >= 1) {
                nb.ds_size = size;
                break;
            }
            cudaGetLastError();
        }
    }
    if (nb.ds_size == 0) return PE_B200_OK;
    const int size = nb.ds_size;
    const int shift = size == 16 ? 4 : 3;
    int64_t per, scap, bytes;
    plan(size, per, scap, bytes, nb.ds_optin);
    auto kern = dsmem_kernel<VT>(model, scap > 0);
    // the attributes are per kernel: set again, since another body count may have set them
    if (size > 8)
        cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    cudaGetLastError();
    cfg.gridDim = dim3(size);
    cfg.dynamicSmemBytes = (size_t)bytes;
    attr[0].val.clusterDim.x = size;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, iters, (const int32_t *)nb.dd, gate,
                                             (const int32_t *)nb.cstart_dev, cap, dtinv, cc, bv,
                                             nb.nbod, (int)per, shift, (int)scap, track, dl);
    if (e != cudaSuccess) {
        cudaGetLastError();
        nb.ds_size = 0;
        return PE_B200_OK;
    }
    c->launches++;
    *done = true;
    return PE_B200_OK;
}

// The colouring rounds of a queued step in one cooperative launch (k_color_rounds); a grid of
// as many blocks as fit, at most one thread per contact of the capacity.
template <typename VT>
int launch_color_rounds(Ctx *c, const int32_t *ncp, int32_t *dd, const Raw<VT> &raw,
                        int64_t cap, int64_t serial_max) {
    NbgsBuf &nb = c->nb;
    static int occ = 0;
    if (occ == 0 && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_color_rounds<1>, kBlk,
                                                                  0) != cudaSuccess)
        occ = 1;
    const unsigned grid = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>((int64_t)std::max(occ, 1) * c->sm_count, (cap + kBlk - 1) / kBlk));
    int32_t *tent = nb.order;   // free until the colour sort
    const int32_t *b1 = raw.b1, *b2 = raw.b2, *adj_start = nb.body_cnt, *adj = nb.body_adj;
    int32_t *color = nb.color, *rem = nb.rem, *err = c->d_err;
    uint64_t *used = nb.used;
    unsigned int *bar = nb.bar2;
    void *args[] = {&ncp, &dd, &serial_max, &b1, &b2, &adj_start, &adj, &tent, &color, &used,
                    &rem, &bar, &err};
    PEB_CUDA(c, cudaLaunchCooperativeKernel((const void *)k_color_rounds<1>, dim3(grid),
                                            dim3(kBlk), args, 0, c->stream));
    c->launches++;
    return PE_B200_OK;
}

// Blocks of the grid sweep form of queued steps: enough for the largest colour of the last step
// whose counts reached the host (one block per 4096 contacts of the capacity before any did),
// rounded up to a power of two so that a captured graph of steps stays valid while that colour
// changes little.
inline int64_t queued_sweep_blocks(const Ctx *c) {
    const NbgsBuf &nb = c->nb;
    const int64_t maxcol = nb.h_dd && nb.h_dd[kDdMaxcol] > 0 ? nb.h_dd[kDdMaxcol] : nb.cap / 16;
    int64_t b = 1;
    while (b * kBlk < maxcol) b <<= 1;
    return b;
}

// The sweeps of a queued step: the single-block form and the grid form are both launched and
// each runs only for the case it serves (sweeps_gate: every colour fits one block, or not).
// The grid form's size follows the largest colour of an earlier step (any size is correct:
// its blocks stride over a colour's contacts).
template <typename VT>
int launch_sweeps_queued(Ctx *c, int model, bool gen, int iters, int64_t cap, VT dtinv,
                         const Cache<VT> &cc, const BodyV<VT> &bv, int64_t n,
                         unsigned long long *dl) {
    NbgsBuf &nb = c->nb;
    int32_t *dd = nb.dd;
    const int mode = c->tune.nbgs_sweeps;
    // every colour within one block: the compact form for a few contacts, else the whole-scene
    // single-block form
    bool compact = false;
    if (!gen && mode != 2) {
        int rc = launch_sweeps_compact<VT>(c, model, iters, 4, dtinv, cc, bv, 0, dl, &compact);
        if (rc) return rc;
    }
    const int block_gate = compact ? 5 : 1;
    const size_t smem = (size_t)(gen ? 7 : 4) * nb.nbod * sizeof(T4<VT>);
    bool smem_ok = smem <= kBlockSmemMax;
    if (smem_ok) {
        auto kern = block_smem_kernel<VT>(model, gen);
        smem_ok = cudaFuncSetAttribute((const void *)kern,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kBlockSmemMax) == cudaSuccess;
        if (smem_ok) {
            kern<<<1, kBlk, smem, c->stream>>>(iters, dd, block_gate, nb.cstart_dev, cap, dtinv, cc,
                                               bv, nb.nbod, 0, dl);
            PEB_LAUNCHED(c);
        } else {
            cudaGetLastError();
        }
    }
    if (!smem_ok) {
        block_kernel<VT>(model, gen)<<<1, kBlk, 0, c->stream>>>(iters, dd, block_gate,
                                                                nb.cstart_dev, cap, dtinv, cc, bv,
                                                                n, 0, dl);
        PEB_LAUNCHED(c);
    }
    int grid_gate = 2;
    if (mode == 0 || mode == 5) {
        // the colours beyond one block: in one cluster's shared memory, if the bodies fit there
        // (automatic: up to kDsmemMaxcol contacts per colour, the grid form beyond)
        bool done = false;
        int rc = launch_sweeps_dsmem<VT>(c, model, iters, mode == 5 ? 2 : 3, cap, dtinv, cc, bv, 0,
                                         dl, &done);
        if (rc) return rc;
        if (done && mode == 5) return PE_B200_OK;
        if (done) grid_gate = 6;
    }
    if (!gen && model <= 1) {
        bool done = false;
        int rc = launch_sweeps_grid_staged<VT>(c, model, iters, grid_gate, dtinv, cc, bv, 0, dl,
                                               queued_sweep_blocks(c), &done);
        if (rc) return rc;
        if (done) return PE_B200_OK;
    }
    auto kern = persistent_kernel<VT>(model, gen);
    int occ = 0;
    PEB_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kBlk, 0));
    // the largest colour of the last step whose counts reached the host, else one block per
    // 4096 contacts of the capacity
    const unsigned grid = (unsigned)std::min<int64_t>((int64_t)std::max(occ, 1) * c->sm_count,
                                                      queued_sweep_blocks(c));
    // the barrier counter counts iters x colours x blocks arrivals: past 2^32 (kMaxColors
    // colours at most) the grid shrinks
    const unsigned g = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>(grid, (int64_t)(4.0e9 / ((double)std::max(iters, 1) * kMaxColors))));
    PEB_CUDA(c, cudaMemsetAsync(nb.bar, 0, sizeof(unsigned int), c->stream));
    int iters_a = iters, gate_a = grid_gate, track_a = 0;
    int64_t cap_a = cap, n_a = n;
    VT dtinv_a = dtinv;
    int32_t *cs = nb.cstart_dev;
    Cache<VT> cc_a = cc;
    BodyV<VT> bv_a = bv;
    void *args[] = {&iters_a, &dd, &gate_a, &cs, &cap_a, &dtinv_a, &cc_a, &bv_a, &n_a, &track_a,
                    &dl, &nb.bar, &c->d_err};
    PEB_CUDA(c, cudaLaunchCooperativeKernel((const void *)kern, dim3(g), dim3(kBlk), args, 0,
                                            c->stream));
    c->launches++;
    return PE_B200_OK;
}

// contacts one thread colours (more take the parallel rounds): scenes with moving boxes, or
// sphere scenes with the colour masks in shared memory or in global memory
inline int64_t colour_serial_max(const Ctx *c) {
    const bool gen = c->mb.m > 0;
    const size_t masks = (size_t)(c->n + c->mb.m) * (gen ? 4 : 1) * sizeof(uint64_t);
    return gen ? kSerialColourMax
               : (masks <= 48 * 1024 ? kSerialColourMaxSpheres : kSerialColourMaxGlobal);
}

// One hard-contact step: sort, permute, detect, colour, cache, sweep, integrate.
// queued: the step is queued without the host waiting on the device (sphere scenes without a
// residual request, automatic/grid/single-block sweep forms): the contact count stays on the
// device (a count beyond the capacity aborts the rest of the call, which nbgs_run repeats after
// growing the buffers), the colouring runs its rounds in one cooperative launch, and the sweep
// form is chosen on the device from the largest colour.  Otherwise the host reads the counts
// (moving boxes need them for their own kernels; per-colour launches need the colour offsets).
template <typename VT>
int nbgs_step_t(Ctx *c, double dt, bool queued) {
    NbgsBuf &nb = c->nb;
    const int64_t n = c->n;
    // moving boxes: bodies n .. n+m-1 with full inverse inertias (FP64 only, checked by the
    // caller)
    const bool gen = c->mb.m > 0;
    const int64_t nbod = n + c->mb.m;
    const int64_t auto_cap = c->p.max_contacts > 0 ? c->p.max_contacts : std::max<int64_t>(8 * nbod, 1024);
    int rc = nbgs_alloc(c, auto_cap);
    if (rc) return rc;
    nb.on_device = queued;
    // 1. sort, permute to slot order, body cache
    if (n > 0) {
        if (!c->binned) {
            rc = grid_bin_current(c);
            if (rc) return rc;
        }
        rc = grid_sort(c);
        if (rc) return rc;
    }
    Raw<VT> raw;
    Cache<VT> cc;
    BodyV<VT> bv;
    layout(c, raw, cc, bv);
    auto body_cache_d = [&]() {
        BodyCacheD d{};
        if constexpr (std::is_same<VT, double>::value)
            d = BodyCacheD{bv.vr, bv.wr, bv.dv, bv.dw, bv.ia, bv.ib, bv.ic};
        return d;
    };
    if (gen) {
        rc = mbox_hc_bodycache(c, body_cache_d(), dt);
        if (rc) return rc;
    }
    if (n > 0) {
        prof_begin(c, ST_PERMUTE);
        const bool tq = c->p.track_orientation != 0;
        auto kern = tq ? k_permute_cache<VT, true> : k_permute_cache<VT, false>;
        kern<<<grid_for(n, kBlk), kBlk, 0, c->stream>>>(
            n, c->sorted, c->cur.pr, (const VT *)c->cur.vw, c->cur.tag, c->cur.uid, c->cur.q,
            c->nxt.pr, (VT *)c->nxt.vw, c->nxt.tag, c->nxt.uid, c->nxt.q, c->d_mats,
            c->p.gravity[0], c->p.gravity[1], c->p.gravity[2], dt, bv);
        PEB_LAUNCHED(c);
        prof_end(c, ST_PERMUTE);
        std::swap(c->cur, c->nxt);
    }
    // 2. detection: count, scan, write (state is in slot order now: sorted == identity);
    // the contacts of the moving boxes follow the spheres' contacts
    VisitArgs va = visit_args(c, nullptr);
    prof_begin(c, ST_DETECT);
    int64_t nc = 0;                 // the count (host-known steps only)
    int32_t total_s = 0;            // sphere contacts (host-known steps only)
    int32_t *dd = nb.dd;
    const int32_t *ncp = dd + kDdNc;   // the count on the device
    if (queued && nb.plan_none) {
        if (n > 0) {
            k_any_contact<<<grid_for(n, kBlk), kBlk, 0, c->stream>>>(n, va, dd);
            PEB_LAUNCHED(c);
        }
    } else if (queued) {
        if (n > 0) {
            k_count<<<grid_for(n, kBlk), kBlk, 0, c->stream>>>(n, va, nb.cnt);
            PEB_LAUNCHED(c);
            rc = scan_exclusive(c, nb.cnt, nb.cnt, n);
            if (rc) return rc;
            PEB_CUDA(c, cudaMemcpyAsync(dd + kDdNc, nb.cnt + n, sizeof(int32_t),
                                        cudaMemcpyDeviceToDevice, c->stream));
        } else {
            PEB_CUDA(c, cudaMemsetAsync(dd + kDdNc, 0, sizeof(int32_t), c->stream));
        }
        k_guard<<<1, 1, 0, c->stream>>>(ncp, nb.cap, colour_serial_max(c), dd);
        PEB_LAUNCHED(c);
    } else {
        int32_t total_b = 0;
        if (n > 0) {
            k_count<<<grid_for(n, kBlk), kBlk, 0, c->stream>>>(n, va, nb.cnt);
            PEB_LAUNCHED(c);
            rc = scan_exclusive(c, nb.cnt, nb.cnt, n);
            if (rc) return rc;
            PEB_CUDA(c, cudaMemcpyAsync(&total_s, nb.cnt + n, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
            PEB_CUDA(c, cudaStreamSynchronize(c->stream));
        }
        if (gen) {
            rc = mbox_hc_count(c, &total_b);
            if (rc) return rc;
        }
        if ((int64_t)total_s + total_b > INT32_MAX)
            return set_err(c, PE_B200_ERR_CAPACITY, "contact count exceeds int32");
        const int32_t total = total_s + total_b;
        if (total > nb.cap) {
            if (c->p.max_contacts > 0)
                return set_err(c, PE_B200_ERR_CAPACITY, "contact capacity exceeded");
            rc = nbgs_alloc(c, (int64_t)total * 5 / 4 + 1024);
            if (rc) return rc;
            layout(c, raw, cc, bv);
            dd = nb.dd;
        }
        nc = total;
        // the kernels read the count from the device
        nb.h_dd[kDdNc] = total;
        PEB_CUDA(c, cudaMemcpyAsync(dd + kDdNc, nb.h_dd + kDdNc, sizeof(int32_t),
                                    cudaMemcpyHostToDevice, c->stream));
        c->last_ncontacts = nc;
    }
    const int64_t cap = nb.cap;
    // a step planned without contacts aborts if it finds any: it writes no records
    if (n > 0 && !(queued && nb.plan_none)) {
        // a queued step's overflow aborts it instead of reporting an error
        k_raw<VT><<<grid_for(n, kBlk), kBlk, 0, c->stream>>>(n, va, nb.cnt, cap, (const VT *)c->cur.vw,
                                                             c->d_mats, c->d_plane_mat, c->d_box_mat,
                                                             c->p.erp, raw, queued ? dd + kDdSink : c->d_err);
        PEB_LAUNCHED(c);
    }
    if constexpr (std::is_same<VT, double>::value) {
        if (gen) {
            rc = mbox_hc_raw(c, total_s, cap, raw.b1, raw.b2, raw.r1, raw.r2, raw.n, raw.dist,
                             raw.mu);
            if (rc) return rc;
        }
    }
    prof_end(c, ST_DETECT);
    const unsigned cgrid = capped_grid(c, cap, kBlk);   // kernels over the contacts
    // 3. colouring
    int32_t ncolors = 0;
    const bool any = queued ? !nb.plan_none : nc > 0;
    if (any) {
        prof_begin(c, ST_COLOR);
        const size_t masks = (size_t)nbod * (gen ? 4 : 1) * sizeof(uint64_t);
        const bool in_smem = masks <= 48 * 1024;
        const int64_t serial_max = colour_serial_max(c);
        // the body -> contacts adjacency of the parallel rounds (skipped on the device, or by the
        // host, when one thread colours the step)
        const int32_t *rounds = queued ? dd + kDdRounds : nullptr;
        if (queued || nc > serial_max) {
            PEB_CUDA(c, cudaMemsetAsync(nb.body_cnt, 0, ((size_t)nbod + 1) * sizeof(int32_t), c->stream));
            k_degree<<<cgrid, kBlk, 0, c->stream>>>(ncp, dd, rounds, raw.b1, raw.b2, nb.body_cnt);
            PEB_LAUNCHED(c);
            rc = scan_exclusive_cond(c, nb.body_cnt, nb.body_cnt, nbod, rounds);
            if (rc) return rc;
            int32_t *fill = nb.cnt;  // reuse: counts are consumed
            PEB_CUDA(c, cudaMemcpyAsync(fill, nb.body_cnt, ((size_t)nbod + 1) * sizeof(int32_t),
                                        cudaMemcpyDeviceToDevice, c->stream));
            k_adj_fill<<<cgrid, kBlk, 0, c->stream>>>(ncp, dd, rounds, raw.b1, raw.b2, fill,
                                                      nb.body_adj);
            PEB_LAUNCHED(c);
        }
        PEB_CUDA(c, cudaMemsetAsync(nb.color, 0xff, (size_t)(queued ? cap : nc) * sizeof(int32_t), c->stream));
        const int words = gen ? 4 : 1;
        PEB_CUDA(c, cudaMemsetAsync(nb.used, 0, (size_t)nbod * words * sizeof(uint64_t), c->stream));
        if (queued) {
            // one thread for a few contacts; otherwise every round in one cooperative launch
            k_color_serial<1><<<1, 256, in_smem ? masks : 0, c->stream>>>(
                ncp, dd, serial_max, raw.b1, raw.b2, nb.color, nbod, in_smem ? nullptr : nb.used,
                c->d_err);
            PEB_LAUNCHED(c);
            PEB_CUDA(c, cudaMemsetAsync(nb.rem, 0, kMaxRounds * sizeof(int32_t), c->stream));
            rc = launch_color_rounds(c, ncp, dd, raw, cap, serial_max);
            if (rc) return rc;
        } else {
            int round = 0;
            if (nc <= serial_max) {
                (gen ? k_color_serial<4> : k_color_serial<1>)<<<1, 256, in_smem ? masks : 0, c->stream>>>(
                    ncp, dd, serial_max, raw.b1, raw.b2, nb.color, nbod, in_smem ? nullptr : nb.used,
                    c->d_err);
                PEB_LAUNCHED(c);
            }
            for (; nc > serial_max;) {
                const int batch = 8;
                PEB_CUDA(c, cudaMemsetAsync(nb.flags, 0, batch * sizeof(int32_t), c->stream));
                int32_t *tent = nb.order;   // free until the colour sort below
                for (int k = 0; k < batch; ++k, ++round) {
                    (gen ? k_color_propose<4> : k_color_propose<1>)<<<cgrid, kBlk, 0, c->stream>>>(
                        ncp, raw.b1, raw.b2, nb.color, nb.used, tent, c->d_err);
                    PEB_LAUNCHED(c);
                    (gen ? k_color_settle<4> : k_color_settle<1>)<<<cgrid, kBlk, 0, c->stream>>>(
                        ncp, round, raw.b1, raw.b2, nb.body_cnt, nb.body_adj, tent, nb.color, nb.used,
                        nb.flags + k);
                    PEB_LAUNCHED(c);
                }
                int32_t rem[8];
                PEB_CUDA(c, cudaMemcpyAsync(rem, nb.flags, sizeof rem, cudaMemcpyDeviceToHost, c->stream));
                PEB_CUDA(c, cudaStreamSynchronize(c->stream));
                if (rem[batch - 1] == 0) break;
                if (round > kMaxRounds) return set_err(c, PE_B200_ERR_TIMEOUT, "colouring did not finish");
            }
        }
        // counting sort by colour: histogram, offsets on the device
        PEB_CUDA(c, cudaMemsetAsync(nb.flags, 0, 2 * kMaxColors * sizeof(int32_t), c->stream));
        int32_t *hist = nb.flags, *nco = nb.flags + kMaxColors;
        k_color_hist<<<cgrid, kBlk, 0, c->stream>>>(ncp, dd, nb.color, hist, nco);
        PEB_LAUNCHED(c);
        int32_t *cfill = nb.flags + 2 * kMaxColors;   // the colour offsets as fill counters
        k_color_scan<<<1, kMaxColors, 0, c->stream>>>(hist, nco, nb.cstart_dev, cfill, dd);
        PEB_LAUNCHED(c);
        if (!queued) {
            // the host-driven forms need the offsets on the host
            PEB_CUDA(c, cudaMemcpyAsync(nb.color_start, nb.cstart_dev, (kMaxColors + 1) * sizeof(int32_t),
                                        cudaMemcpyDeviceToHost, c->stream));
            PEB_CUDA(c, cudaMemcpyAsync(nb.h_dd, dd, kDdCount * sizeof(int32_t),
                                        cudaMemcpyDeviceToHost, c->stream));
            PEB_CUDA(c, cudaStreamSynchronize(c->stream));
            ncolors = nb.h_dd[kDdNcolors];
        }
        k_color_pos<<<cgrid, kBlk, 0, c->stream>>>(ncp, dd, nb.color, cfill, nb.order);
        PEB_LAUNCHED(c);
        prof_end(c, ST_COLOR);
        prof_begin(c, ST_CACHE);
        // 4. contact cache in colour-sorted order
        if constexpr (std::is_same<VT, double>::value) {
            if (gen) k_cache<VT, true><<<cgrid, kBlk, 0, c->stream>>>(ncp, dd, cap, raw, nb.order, bv, n, cc);
            else k_cache<VT, false><<<cgrid, kBlk, 0, c->stream>>>(ncp, dd, cap, raw, nb.order, bv, n, cc);
        } else {
            k_cache<VT, false><<<cgrid, kBlk, 0, c->stream>>>(ncp, dd, cap, raw, nb.order, bv, n, cc);
        }
        PEB_LAUNCHED(c);
        prof_end(c, ST_CACHE);
    }
    c->last_ncolors = ncolors;
    // 5. sweeps
    const int model = c->p.relaxation_model;
    const bool fr = model != PE_B200_INELASTIC_FRICTIONLESS;
    const int iters = c->p.max_iterations;
    unsigned long long *dl = (unsigned long long *)nb.red;
    if (c->want_residual) PEB_CUDA(c, cudaMemsetAsync(nb.red, 0, 2 * sizeof(double), c->stream));
    if (queued && any && iters > 0) {
        prof_begin(c, ST_SWEEP);
        rc = launch_sweeps_queued<VT>(c, model, gen, iters, cap, VT(1.0 / dt), cc, bv, n, dl);
        if (rc) return rc;
        prof_end(c, ST_SWEEP);
    } else if (!queued && nc > 0) {
        prof_begin(c, ST_SWEEP);
        bool done = iters == 0;
        int maxcol = 1;
        for (int col = 0; col < ncolors; ++col)
            maxcol = std::max(maxcol, nb.color_start[col + 1] - nb.color_start[col]);
        const int mode = c->tune.nbgs_sweeps;
        // the one-cluster form has the cheaper barrier but only a few SMs' load bandwidth; on
        // B200 the grid form is faster for every scene measured, so it is the automatic choice
        if (!done && nb.cluster != 0 && mode == 1 && !gen) {
            int rc = sweeps_in_cluster<VT>(c, model, iters, ncolors, maxcol, cap, VT(1.0 / dt), cc,
                                           bv, n, dl, &done);
            if (rc) return rc;
        }
        if (!done && mode == 5) {
            int rc = launch_sweeps_dsmem<VT>(c, model, iters, 0, cap, VT(1.0 / dt), cc, bv,
                                            c->want_residual ? 1 : 0, dl, &done);
            if (rc) return rc;
        }
        if (!done && (mode == 0 || mode == 4) && maxcol <= kBlk && !gen && nc <= kCompactMax) {
            // a few contacts: one block with their bodies in shared memory
            int rc = launch_sweeps_compact<VT>(c, model, iters, 0, VT(1.0 / dt), cc, bv,
                                              c->want_residual ? 1 : 0, dl, &done);
            if (rc) return rc;
        }
        if (!done && mode == 0 && maxcol > kBlk && maxcol <= kDsmemMaxcol) {
            int rc = launch_sweeps_dsmem<VT>(c, model, iters, 0, cap, VT(1.0 / dt), cc, bv,
                                            c->want_residual ? 1 : 0, dl, &done);
            if (rc) return rc;
        }
        if (!done && (mode == 0 || mode == 4) && maxcol <= kBlk) {
            // every colour fits one block: all sweeps in one block, colours separated by
            // __syncthreads (automatic, or asked for with 4)
            const size_t smem = (size_t)(gen ? 7 : 4) * nb.nbod * sizeof(T4<VT>);
            bool smem_ok = smem <= kBlockSmemMax;
            if (smem_ok) {
                auto kern = block_smem_kernel<VT>(model, gen);
                // opt in to the large shared-memory carve-out (per kernel; cheap to repeat)
                smem_ok = cudaFuncSetAttribute((const void *)kern,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)kBlockSmemMax) == cudaSuccess;
                if (smem_ok) {
                    kern<<<1, kBlk, smem, c->stream>>>(iters, dd, 0, nb.cstart_dev, cap,
                                                       VT(1.0 / dt), cc, bv, nb.nbod,
                                                       c->want_residual ? 1 : 0, dl);
                    PEB_LAUNCHED(c);
                } else {
                    cudaGetLastError();
                }
            }
            if (!smem_ok) {
                block_kernel<VT>(model, gen)<<<1, kBlk, 0, c->stream>>>(
                    iters, dd, 0, nb.cstart_dev, cap, VT(1.0 / dt), cc, bv, n,
                    c->want_residual ? 1 : 0, dl);
                PEB_LAUNCHED(c);
            }
            done = true;
        }
        if (!done && mode != 3 && !gen && model <= 1) {
            // the grid form with each block's contacts staged in its shared memory
            int rc = launch_sweeps_grid_staged<VT>(c, model, iters, 0, VT(1.0 / dt), cc, bv,
                                                  c->want_residual ? 1 : 0, dl,
                                                  std::max<int64_t>(1, (maxcol + kBlk - 1) / kBlk),
                                                  &done);
            if (rc) return rc;
        }
        if (!done && !nb.coop_disabled && mode != 3) {
            // all sweeps in one cooperative launch (colours separated by grid barriers); as few
            // blocks as the largest colour needs, so the barriers stay short
            auto kern = persistent_kernel<VT>(model, gen);
            int occ = 0;
            cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kBlk, 0);
            const unsigned grid = (unsigned)std::min<int64_t>(
                (int64_t)std::max(occ, 1) * c->sm_count, std::max<int64_t>(1, (maxcol + kBlk - 1) / kBlk));
            // the barrier counter of one launch counts iters x colours x blocks arrivals; past
            // 2^32 the colours are launched one by one instead
            const bool fits = (double)iters * ncolors * grid < 4.0e9;
            if (e == cudaSuccess && occ > 0 && fits) {
                // the barrier counter of this launch starts at zero (its episodes count up)
                PEB_CUDA(c, cudaMemsetAsync(nb.bar, 0, sizeof(unsigned int), c->stream));
                int iters_a = iters, gate_a = 0, track_a = c->want_residual ? 1 : 0;
                int64_t cap_a = cap, n_a = n;
                VT dtinv_a = VT(1.0 / dt);
                int32_t *cs = nb.cstart_dev;
                int32_t *dd_a = dd;
                void *args[] = {&iters_a, &dd_a, &gate_a, &cs, &cap_a, &dtinv_a, &cc, &bv, &n_a,
                                &track_a, &dl, &nb.bar, &c->d_err};
                e = cudaLaunchCooperativeKernel((const void *)kern, dim3(grid), dim3(kBlk), args, 0,
                                                c->stream);
            }
            if (e == cudaSuccess && occ > 0 && fits) {
                done = true;
                c->launches++;
            } else if (e != cudaSuccess) {
                cudaGetLastError();
                nb.coop_disabled = true;
            }
        }
        for (int it = 0; !done && it < iters; ++it) {
            const int track = (c->want_residual && it == iters - 1) ? 1 : 0;
            for (int col = 0; col < ncolors; ++col) {
                const int64_t b = nb.color_start[col], e = nb.color_start[col + 1];
                if (e <= b) continue;
                colour_kernel<VT>(model, gen)<<<grid_for(e - b, kBlk), kBlk, 0, c->stream>>>(
                    b, e, cap, VT(1.0 / dt), cc, bv, n, track, dl);
                PEB_LAUNCHED(c);
            }
        }
        prof_end(c, ST_SWEEP);
    }
    if (c->want_residual && any) {
        if (fr)
            k_residual<VT, true><<<cgrid, kBlk, 0, c->stream>>>(ncp, cap, 1.0 / dt, cc, bv, n, dl + 1);
        else
            k_residual<VT, false><<<cgrid, kBlk, 0, c->stream>>>(ncp, cap, 1.0 / dt, cc, bv, n, dl + 1);
        PEB_LAUNCHED(c);
    }
    // 6. integrate into the other buffer and bin for the next step
    {
        prof_begin(c, ST_INTEGRATE);
        const bool tq = c->p.track_orientation != 0;
        const int has_drag = c->p.damping < 1.0;
        const double drag = has_drag ? pow(c->p.damping, dt) : 1.0;
        auto kern = tq ? k_integrate<VT, true> : k_integrate<VT, false>;
        if (n > 0) {
            kern<<<grid_for(n, kBlk), kBlk, 0, c->stream>>>(
                n, dt, drag, has_drag, bv, c->d_scenes, c->cur.pr, (const VT *)c->cur.vw,
                c->cur.tag, c->cur.uid, c->cur.q, c->nxt.pr, (VT *)c->nxt.vw, c->nxt.tag,
                c->nxt.uid, c->nxt.q, c->key, c->rank, c->cell_count, dd, c->d_err);
            PEB_LAUNCHED(c);
        }
        if (gen) {
            rc = mbox_hc_integrate(c, body_cache_d(), dt);
            if (rc) return rc;
        }
        prof_end(c, ST_INTEGRATE);
        if (n > 0) std::swap(c->cur, c->nxt);
    }
    if (c->want_residual) {
        double r[2];
        PEB_CUDA(c, cudaMemcpyAsync(r, nb.red, sizeof r, cudaMemcpyDeviceToHost, c->stream));
        PEB_CUDA(c, cudaStreamSynchronize(c->stream));
        c->last_delta = nc > 0 ? r[0] : 0.0;
        c->last_residual = nc > 0 ? r[1] : 0.0;
    } else {
        c->last_delta = -1.0;
        c->last_residual = -1.0;
    }
    return PE_B200_OK;
}

}  // namespace

void nbgs_free(Ctx *c) {
    NbgsBuf &b = c->nb;
    dfree(c, b.cache);
    dfree(c, b.order);
    dfree(c, b.color);
    dfree(c, b.body_adj);
    dfree(c, b.cnt);
    dfree(c, b.body_cnt);
    dfree(c, b.used);
    dfree(c, b.vel);
    dfree(c, b.flags);
    dfree(c, b.red);
    dfree(c, b.cstart_dev);
    dfree(c, b.bar);
    dfree(c, b.dd);
    dfree(c, b.rem);
    dfree(c, b.bar2);
    dfree(c, b.slot_of);
    if (b.color_start) cudaFreeHost(b.color_start);
    if (b.h_dd) cudaFreeHost(b.h_dd);
    nbgs_graph_free(c);
    b = NbgsBuf();
}

void nbgs_graph_free(Ctx *c) {
    for (NbgsBuf::GraphSlot &s : c->nb.gslot) {
        if (s.exec) cudaGraphExecDestroy(s.exec);
        s = NbgsBuf::GraphSlot();
    }
}

namespace {

// whether the hard-contact steps of this context are queued without host waits
bool nbgs_queued(const Ctx *c) {
    const int mode = c->tune.nbgs_sweeps;
    return c->mb.m == 0 && !c->want_residual && (mode == 0 || mode == 2 || mode == 4 || mode == 5);
}

}  // namespace

int nbgs_step(Ctx *c, double dt) {
    if (c->n == 0 && c->mb.m == 0) return PE_B200_OK;
    const bool q = nbgs_queued(c);
    return (c->p.precision == PE_B200_FP64) ? nbgs_step_t<double>(c, dt, q)
                                            : nbgs_step_t<float>(c, dt, q);
}

// Replays of a captured graph of c->graph_steps queued steps (even, so that the buffer swaps
// cancel) while they fit in nsteps; *ran receives the steps run (0: graphs are off, not
// possible, or the buffers are fresh).  A graph is kept per key (buffers, the settings it bakes
// in, the plan with or without contacts, the sweep grid), so a scene whose plan or largest
// colour alternates replays graphs captured before.  Nothing runs on the device during a
// capture, so a failed capture only switches graphs off.
int nbgs_graph_run(Ctx *c, int32_t nsteps, double dt, int32_t *ran) {
    NbgsBuf &nb = c->nb;
    *ran = 0;
    const int32_t gs = c->graph_steps & ~1;
    if (gs < 2 || nsteps < gs || nb.gfailed || c->prof || !nb.warm) return PE_B200_OK;
    union {
        double d;
        uint64_t u;
    } dtu;
    dtu.d = dt;
    union {
        double d;
        uint64_t u;
    } erpu;
    erpu.d = c->p.erp;
    const uint64_t key[12] = {(uint64_t)(uintptr_t)c->cur.pr, (uint64_t)(uintptr_t)c->nxt.pr,
                              (uint64_t)(uintptr_t)nb.cache, (uint64_t)nb.cap, c->epoch,
                              (uint64_t)c->p.max_iterations, (uint64_t)c->p.relaxation_model,
                              erpu.u, dtu.u, (uint64_t)nb.plan_none,
                              (uint64_t)queued_sweep_blocks(c), (uint64_t)gs};
    NbgsBuf::GraphSlot *hit = nullptr, *lru = &nb.gslot[0];
    for (NbgsBuf::GraphSlot &s : nb.gslot) {
        bool match = s.exec != nullptr;
        for (int i = 0; i < 12 && match; ++i) match = s.key[i] == key[i];
        if (match) hit = &s;
        if (!s.exec || (lru->exec && s.used < lru->used)) lru = &s;
    }
    if (!hit) {
        hit = lru;
        if (hit->exec) cudaGraphExecDestroy(hit->exec);
        hit->exec = nullptr;
        const BodyBuf cur0 = c->cur, nxt0 = c->nxt;
        const int64_t l0 = c->launches;
        cudaGraph_t g = nullptr;
        int rc = PE_B200_OK;
        cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            for (int32_t k = 0; k < gs && rc == PE_B200_OK; ++k) rc = nbgs_step(c, dt);
            const cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
            if (e == cudaSuccess) e = e2;
        }
        const int64_t per = c->launches - l0;
        c->launches = l0;
        bool ok = e == cudaSuccess && rc == PE_B200_OK && g != nullptr && c->cur.pr == cur0.pr;
        if (ok) ok = cudaGraphInstantiate(&hit->exec, g, 0) == cudaSuccess;
        if (g) cudaGraphDestroy(g);
        if (!ok) {
            nbgs_graph_free(c);
            nb.gfailed = true;
            c->cur = cur0;
            c->nxt = nxt0;
            cudaGetLastError();
            c->err.clear();
            return PE_B200_OK;
        }
        for (int i = 0; i < 12; ++i) hit->key[i] = key[i];
        hit->launches = per;
        c->graph_captures++;
    }
    hit->used = ++nb.gclock;
    PEB_CUDA(c, cudaGraphLaunch(hit->exec, c->stream));
    c->launches += hit->launches;
    c->graph_replays++;
    *ran = gs;
    return PE_B200_OK;
}

// nsteps hard-contact steps.  Queued steps are checked once at the end: if some step found
// more contacts than the buffers hold, it and every later step of the call left the state as
// it was; the buffers grow to the count seen and those steps run again.
int nbgs_run(Ctx *c, int32_t nsteps, double dt) {
    if (c->n == 0 && c->mb.m == 0) return PE_B200_OK;
    if (!nbgs_queued(c)) {
        for (int32_t k = 0; k < nsteps; ++k) {
            const int rc = nbgs_step(c, dt);
            if (rc) return rc;
        }
        return PE_B200_OK;
    }
    int32_t left = nsteps;
    for (int attempt = 0; left > 0; ++attempt) {
        if (c->nb.dd) {
            PEB_CUDA(c, cudaMemsetAsync(c->nb.dd + kDdSteps, 0, sizeof(int32_t), c->stream));
            PEB_CUDA(c, cudaMemsetAsync(c->nb.dd + kDdSeen, 0, sizeof(int32_t), c->stream));
        }
        int32_t k = 0;
        while (k < left) {
            int32_t ran = 0;
            int rc = nbgs_graph_run(c, left - k, dt, &ran);
            if (rc) return rc;
            if (ran == 0) {
                rc = nbgs_step(c, dt);
                if (rc) return rc;
                c->nb.warm = true;
                ran = 1;
            }
            k += ran;
        }
        NbgsBuf &nb = c->nb;
        PEB_CUDA(c, cudaMemcpyAsync(nb.h_dd, nb.dd, kDdCount * sizeof(int32_t),
                                    cudaMemcpyDeviceToHost, c->stream));
        PEB_CUDA(c, cudaStreamSynchronize(c->stream));
        c->last_ncontacts = nb.h_dd[kDdNc];
        c->last_ncolors = nb.h_dd[kDdNc] > 0 ? nb.h_dd[kDdNcolors] : 0;
        if (!nb.h_dd[kDdAbort]) {
            // the next call's steps skip the contact stages while the scene has no contacts:
            // none in any step of this call
            nb.plan_none = nb.h_dd[kDdSeen] == 0;
            break;
        }
        const int32_t done = nb.h_dd[kDdSteps];
        const int64_t need = nb.h_dd[kDdNeed];
        if (attempt >= 8) return set_err(c, PE_B200_ERR_CAPACITY, "contact buffers kept overflowing");
        if (need > nb.cap) {
            if (c->p.max_contacts > 0)
                return set_err(c, PE_B200_ERR_CAPACITY, "contact capacity exceeded");
            int rc = nbgs_alloc(c, need + need / 4 + 1024);
            if (rc) return rc;
        }
        nb.plan_none = false;
        PEB_CUDA(c, cudaMemsetAsync(nb.dd + kDdAbort, 0, sizeof(int32_t), c->stream));
        nb.h_dd[kDdAbort] = 0;
        left -= done;
    }
    return PE_B200_OK;
}

const int2 *nbgs_ids_ptr(Ctx *c) {
    if (c->p.precision == PE_B200_FP64) {
        Raw<double> raw;
        Cache<double> cc;
        BodyV<double> bv;
        layout(c, raw, cc, bv);
        return cc.ids;
    }
    Raw<float> raw;
    Cache<float> cc;
    BodyV<float> bv;
    layout(c, raw, cc, bv);
    return cc.ids;
}

int find_contacts(Ctx *c, int64_t cap, int64_t *ids, double *geom, int64_t *n_out) {
    const int64_t n = c->n;
    *n_out = 0;
    if (n == 0) {
        // moving boxes only
        std::vector<int64_t> bid;
        std::vector<double> bg;
        int rc = mbox_find_contacts(c, bid, bg);
        if (rc) return rc;
        const int64_t nb_ = (int64_t)bid.size() / 3;
        std::vector<int64_t> idx(nb_);
        for (int64_t k = 0; k < nb_; ++k) idx[k] = k;
        std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) {
            if (bid[3 * a] != bid[3 * b]) return bid[3 * a] < bid[3 * b];
            return bid[3 * a + 1] < bid[3 * b + 1];
        });
        for (int64_t k = 0; k < std::min<int64_t>(cap, nb_); ++k) {
            ids[2 * k] = bid[3 * idx[k]];
            ids[2 * k + 1] = bid[3 * idx[k] + 1];
            for (int a = 0; a < 7; ++a) geom[7 * k + a] = bg[7 * idx[k] + a];
        }
        *n_out = nb_;
        return PE_B200_OK;
    }
    // make the sort describe the current state (keeps key/rank/counts valid for the next step)
    if (!c->binned) {
        int rc = grid_bin_current(c);
        if (rc) return rc;
    }
    // the sort consumes cell_count; rebuild it afterwards from the same state
    int rc = grid_sort(c);
    if (rc) return rc;
    int32_t *cnt = nullptr;
    PEB_CUDA(c, dmalloc(c, &cnt, ((size_t)n + 2) * sizeof(int32_t)));
    VisitArgs va = visit_args(c, c->sorted);
    k_count<<<grid_for(n, kBlk), kBlk, 0, c->stream>>>(n, va, cnt);
    PEB_LAUNCHED(c);
    rc = scan_exclusive(c, cnt, cnt, n);
    if (rc) { dfree(c, cnt); return rc; }
    int32_t total = 0;
    PEB_CUDA(c, cudaMemcpyAsync(&total, cnt + n, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    std::vector<int64_t> hid(2 * (size_t)std::max(total, 1));
    std::vector<double> hg(7 * (size_t)std::max(total, 1));
    int64_t *d_ids = nullptr;
    double *d_geom = nullptr;
    cudaError_t e = dmalloc(c, &d_ids, hid.size() * sizeof(int64_t));
    if (e == cudaSuccess) e = dmalloc(c, &d_geom, hg.size() * sizeof(double));
    if (e != cudaSuccess) {
        dfree(c, cnt); dfree(c, d_ids); dfree(c, d_geom);
        return cuda_err(c, e, "find_contacts alloc");
    }
    k_list<<<grid_for(n, kBlk), kBlk, 0, c->stream>>>(n, va, cnt, total, d_ids, d_geom);
    c->launches++;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(hid.data(), d_ids, hid.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hg.data(), d_geom, hg.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    dfree(c, cnt);
    dfree(c, d_ids);
    dfree(c, d_geom);
    if (e != cudaSuccess) return cuda_err(c, e, "find_contacts");
    // the contacts of the moving boxes (pe's orientation and ids) follow
    {
        std::vector<int64_t> bid;
        std::vector<double> bg;
        rc = mbox_find_contacts(c, bid, bg);
        if (rc) return rc;
        const int64_t nb_ = (int64_t)bid.size() / 3;
        hid.resize(2 * (size_t)total);
        hg.resize(7 * (size_t)total);
        for (int64_t k = 0; k < nb_; ++k) {
            hid.push_back(bid[3 * k]);
            hid.push_back(bid[3 * k + 1]);
            for (int a = 0; a < 7; ++a) hg.push_back(bg[7 * k + a]);
        }
        total += (int32_t)nb_;
    }
    // canonical order (b1, b2); the several contacts of a box pair keep their order
    std::vector<int64_t> idx(total);
    for (int64_t k = 0; k < total; ++k) idx[k] = k;
    std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) {
        if (hid[2 * a] != hid[2 * b]) return hid[2 * a] < hid[2 * b];
        return hid[2 * a + 1] < hid[2 * b + 1];
    });
    const int64_t m = std::min<int64_t>(cap, total);
    for (int64_t k = 0; k < m; ++k) {
        ids[2 * k] = hid[2 * idx[k]];
        ids[2 * k + 1] = hid[2 * idx[k] + 1];
        for (int a = 0; a < 7; ++a) geom[7 * k + a] = hg[7 * idx[k] + a];
    }
    *n_out = total;
    // restore the binning of the current state for the next step
    return grid_bin_current(c);
}

}  // namespace peb
