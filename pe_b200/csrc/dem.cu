// dem.cu -- the DEM step: neighbour search, contact law, force accumulation and integration.
//
// Restates, per body:
//   detection    HashGrids::findContacts + MaxContacts::collideSphere{Sphere,Plane,Box}
//                (pe/core/detection/coarse/HashGrids.h:1121-1314,
//                 pe/core/detection/fine/MaxContacts.h:547-569, 777-790, 589-668)
//   contact law  response::DEMSolver::resolveContact, linear spring-dashpot + damping-limited
//                Coulomb friction (pe/core/response/DEMSolver.h:328-379)
//   forces       RigidBody::addForceAtPos (pe/core/rigidbody/RigidBody.h:1775-1803)
//   integration  SphereTrait::move, semi-implicit Euler + quaternion update
//                (pe/core/rigidbody/spheretrait/Default.h:149-220)
// pe has no tangential contact history, so a contact's force depends only on the two bodies'
// current state: every thread gathers the forces on its own sphere (each pair is evaluated by
// both partners, in pe's orientation -- body 1 = smaller id -- so both see bitwise-opposite
// forces) and no atomics or contact list are needed.
//
// Two neighbour sources:
//   grid   (k_dem_step) every step: the counting-sorted uniform grid, 27 cells per sphere; the
//          thread owning sorted slot t writes its body to slot t of the other buffer, so the
//          state is re-sorted by cell as a side effect, and it bins the result for the next sort.
//   lists  (k_dem_contacts + k_dem_move) Verlet lists: all pairs closer than r_i + r_j + skin
//          when the list was built.  A sphere's accumulated path length is tracked; once any
//          sphere has moved skin/2 the device requests a rebuild, which the next step performs
//          (sort, gather into cell order, count/scan/write the lists, mark the spheres that can
//          feel a force) before its force kernels.  Every pair that can come within the contact
//          threshold is therefore in the list, and the pair set is the grid's, exactly.  The
//          rebuild kernel runs every step and returns at once unless requested, so the host
//          never waits on the device to decide.  If a rebuild overflows the list capacity, that
//          step's contact kernel searches the fresh grid instead (exact) and the host grows the
//          capacity at its next check.
#include <math_constants.h>

#include <algorithm>
#include <climits>

#include "internal.cuh"
#include "rebuild.cuh"

namespace peb {

namespace {

#ifndef PEB_DEM_BLOCK
#define PEB_DEM_BLOCK 128
#endif
#ifndef PEB_LIST_MIN_BLOCKS_F32
#define PEB_LIST_MIN_BLOCKS_F32 7
#endif
constexpr int kDemBlock = PEB_DEM_BLOCK;

template <typename T>
struct Acc {
    V3<T> F, T_;
};

template <typename T>
__device__ __forceinline__ T tmin(T a, T b) { return a < b ? a : b; }

// The linear spring-dashpot law of response/DEMSolver.h:328-379 for one contact, in pe's
// orientation (n from body 2 to body 1).  r1/r2: contact point relative to the two centres
// (pe evaluates (gpos - gpos_) for velFromWF and addForceAtPos alike); w2 may be zero (walls).
// Adds the force on body `self` (1 or 2) to acc.
// reff > 0 selects the extended Hertz law (sphere-sphere contacts with forceModel == hertz,
// response/DEMSolver.h:343-357); reff = r1 r2 / (r1 + r2) (contacttrait/DEMSolver.h:152-159)
template <typename T>
__device__ __forceinline__ void dem_contact(V3<T> n, T dist, V3<T> r1, V3<T> r2, V3<T> v1,
                                            V3<T> w1, V3<T> v2, V3<T> w2, const MatDev &m1,
                                            const MatDev &m2, bool self_is_1, Acc<T> &acc,
                                            T reff = T(0)) {
    // velFromWF, RigidBody.h:1080-1085
    const V3<T> rvel = (v1 + cross(w1, r1)) - (v2 + cross(w2, r2));
    // Contact.cpp:86-105: composed coefficients and the static/dynamic friction pick
    const T k = T(1) / (T(m1.rk) + T(m2.rk));
    const T cn = T(1) / (T(m1.rcn) + T(m2.rcn));
    const T ct = T(1) / (T(m1.rct) + T(m2.rct));
    const T nvel = dot(n, rvel);
    const T tvel = dot(n, rvel - n * nvel);
    const T mu = (fabs(tvel) > T(kFrictionThreshold)) ? T(m1.cdf) + T(m2.cdf)
                                                      : T(m1.csf) + T(m2.csf);
    const T delta = -dist;
    const T relVelN = -nvel;
    const V3<T> relVel = -rvel;
    const V3<T> relVelT = relVel - n * relVelN;
    T fNabs;
    if (reff > T(0)) {
        // Materials.h:586-600, pe's operation order
        const T tmp1 = T(m2.young) * (T(1) - T(m1.poisson) * T(m1.poisson));
        const T tmp2 = T(m1.young) * (T(1) - T(m2.poisson) * T(m2.poisson));
        const T eeff = (T(m1.young) * T(m2.young)) / (tmp1 + tmp2);
        const T kh = (T(4) / T(3)) * eeff * sqrt(reff);
        fNabs = kh * pow(delta, T(1.5)) + cn * relVelN * pow(delta, T(0.5));
    } else {
        fNabs = k * delta + cn * relVelN;
    }
    if (fNabs < T(0)) fNabs = T(0);
    const V3<T> fN = fNabs * n;
    const T fTabs = tmin(ct * length(relVelT), mu * fNabs);
    const V3<T> fT = fTabs * normalized(relVelT);
    if (self_is_1) {
        acc.F = acc.F + fN;
        acc.T_ = acc.T_ + cross(r1, fN);
        acc.F = acc.F + fT;
        acc.T_ = acc.T_ + cross(r1, fT);
    } else {
        const V3<T> mfN = -fN, mfT = -fT;
        acc.F = acc.F + mfN;
        acc.T_ = acc.T_ + cross(r2, mfN);
        acc.F = acc.F + mfT;
        acc.T_ = acc.T_ + cross(r2, mfT);
    }
}

template <typename VT>
struct DemArgs {
    int64_t n;
    double dt;
    double g[3];
    double drag;      // damping^dt
    int has_drag;
    const int32_t *sorted;   // grid kernel: slot -> body; nullptr: identity
    const int32_t *cell_start;
    const SceneInfo *scenes;
    const MatDev *mats;
    const double4 *planes;
    const float4 *planes_f;   // FP32 copy of planes (may be null: converted on the fly)
    const int32_t *plane_mat;
    const double *boxes;
    const int32_t *box_mat;
    const double4 *pr;
    const VT *vw;
    const uint32_t *tag;
    const int32_t *uid;
    const double4 *q;
    double4 *pr_out;
    VT *vw_out;
    uint32_t *tag_out;
    int32_t *uid_out;
    double4 *q_out;
    int32_t *key;
    int32_t *rank;
    int32_t *cell_count;
    int32_t *err;
    // lists
    const int32_t *nl_start;
    const int32_t *nl_idx;
    float *disp;
    int32_t *nl_flags;
    float half_skin;
    int hertz;        // extended Hertz law for sphere pairs (force_model 1)
    const double *ext = nullptr;   // moving boxes: their force and torque on body b (6 per body)
    // one scene and one material: their records as launch parameters (read from the constant
    // bank instead of through the body's tag)
    SceneInfo s0;
    MatDev m0;
    // list step: the spheres marked at the last rebuild and their forces
    const int32_t *act = nullptr;     // exclusive offsets of the marks (n + 1)
    const int32_t *alist = nullptr;   // the marked spheres
    VT *facc = nullptr;               // their force and torque, component-major (6 x n)
    // list step: the rebuild's copy of the state in cell order, read instead of pr/vw/tag/uid/q
    // by the force kernels of a step that rebuilt (nl_flags[4]); tag_out/uid_out then receive
    // the reordered tags and ids in place
    const double4 *alt_pr = nullptr;
    const VT *alt_vw = nullptr;
    const uint32_t *alt_tag = nullptr;
    const int32_t *alt_uid = nullptr;
    const double4 *alt_q = nullptr;
};

// The state a list step's force kernels read: the current buffers, or the copy in cell order
// when the step rebuilt the lists (the copy is not moved back: the integration writes the next
// state from it).  Read after the rebuild kernel has finished.
template <typename VT>
__device__ __forceinline__ DemArgs<VT> list_view(const DemArgs<VT> &a0) {
    DemArgs<VT> a = a0;
    if (a0.nl_flags[4]) {
        a.pr = a0.alt_pr;
        a.vw = a0.alt_vw;
        a.tag = a0.alt_tag;
        a.uid = a0.alt_uid;
        a.q = a0.alt_q;
    }
    return a;
}

// one sphere pair (this body and neighbour j), both in the buffers of `a`; self1: this body is
// pe's body 1, i.e. has the smaller system id (MaxContacts.h:550-551).  ONE: a single material
// (a.m0), so the neighbour's tag is not read.
template <typename T, typename VT, bool HERTZ, bool ONE = false>
__device__ __forceinline__ void pair_force_o(const DemArgs<VT> &a, const double4 &pi, V3<T> vi,
                                             V3<T> wi, const MatDev &mi, int32_t j,
                                             const double4 &pj, bool self1, Acc<T> &acc) {
    const double4 p1 = self1 ? pi : pj;
    const double4 p2 = self1 ? pj : pi;
    const double nx = p1.x - p2.x, ny = p1.y - p2.y, nz = p1.z - p2.z;
    const double len = length_rn(nx, ny, nz);
    const double dist = __dsub_rn(__dsub_rn(len, p1.w), p2.w);
    // only penetrating contacts produce a force (ContactBase.h:307-310)
    if (!(dist < -kContactThreshold)) return;
    const MatDev &mj = ONE ? a.m0 : a.mats[a.tag[j] & 0xffffu];
    const V3<T> vj = ld_vw(a.vw, a.n, j, 0), wj = ld_vw(a.vw, a.n, j, 1);
    V3<T> n, r1, r2;
    if (sizeof(T) == 8) {
        // FP64: the contact point in absolute coordinates, as pe computes it
        const double il = 1.0 / len;
        const double nnx = nx * il, nny = ny * il, nnz = nz * il;
        const double k = p2.w + 0.5 * dist;
        const double gx = p2.x + nnx * k, gy = p2.y + nny * k, gz = p2.z + nnz * k;
        n = v3(T(nnx), T(nny), T(nnz));
        r1 = v3(T(gx - p1.x), T(gy - p1.y), T(gz - p1.z));
        r2 = v3(T(gx - p2.x), T(gy - p2.y), T(gz - p2.z));
    } else {
        // mixed: relative vectors only (the absolute point needs FP64)
        const V3<T> d = v3(T(nx), T(ny), T(nz));
        const T il = T(1) / T(len);
        n = d * il;
        const T k = T(p2.w) + T(0.5) * T(dist);
        r2 = n * k;
        r1 = r2 - d;
    }
    const T reff = HERTZ ? (T(p1.w) * T(p2.w)) / (T(p1.w) + T(p2.w)) : T(0);
    if (self1)
        dem_contact<T>(n, T(dist), r1, r2, vi, wi, vj, wj, mi, mj, true, acc, reff);
    else
        dem_contact<T>(n, T(dist), r1, r2, vj, wj, vi, wi, mj, mi, false, acc, reff);
}

template <typename T, typename VT, bool HERTZ>
__device__ __forceinline__ void pair_force(const DemArgs<VT> &a, const double4 &pi, V3<T> vi,
                                           V3<T> wi, int32_t uidi, const MatDev &mi,
                                           int32_t j, const double4 &pj, Acc<T> &acc) {
    pair_force_o<T, VT, HERTZ>(a, pi, vi, wi, mi, j, pj, uidi < a.uid[j], acc);
}

// walls of the sphere's scene: planes (MaxContacts.h:777-790), then boxes
// (MaxContacts.h:589-668); the sphere is body 1 and the fixed wall has zero velocity
template <typename T, typename VT>
__device__ __forceinline__ void wall_forces(const DemArgs<VT> &a, const SceneInfo &s,
                                            const double4 &pi, V3<T> vi, V3<T> wi,
                                            const MatDev &mi, Acc<T> &acc) {
    const V3<T> zero = v3(T(0), T(0), T(0));
    // a sphere clear of every (axis-aligned) plane tests none of them
    const bool clear = pi.x - pi.w > s.wall_lo[0] && pi.x + pi.w < s.wall_hi[0] &&
                       pi.y - pi.w > s.wall_lo[1] && pi.y + pi.w < s.wall_hi[1] &&
                       pi.z - pi.w > s.wall_lo[2] && pi.z + pi.w < s.wall_hi[2];
    const float pxf = float(pi.x), pyf = float(pi.y), pzf = float(pi.z), prf = float(pi.w);
    const float tol = 1e-3f * (1.0f + fabsf(pxf) + fabsf(pyf) + fabsf(pzf));
    for (int p = 0; p < (clear ? 0 : s.nplanes); ++p) {
        float4 pf;
        if (a.planes_f) {
            pf = a.planes_f[s.plane_begin + p];
        } else {
            const double4 q = a.planes[s.plane_begin + p];
            pf = make_float4(float(q.x), float(q.y), float(q.z), float(q.w));
        }
        // FP32 estimate first: spheres clearly off the plane skip the exact FP64 test (the
        // estimate's error is far below the 1e-3 margin for coordinates up to ~1e4)
        const float est = pf.x * pxf + pf.y * pyf + pf.z * pzf - prf - pf.w;
        if (est > tol + 1e-3f * fabsf(pf.w)) continue;
        const double4 pl = a.planes[s.plane_begin + p];
        const double kk = dot_rn(pl.x, pl.y, pl.z, pi.x, pi.y, pi.z);
        const double dist = __dsub_rn(__dsub_rn(kk, pi.w), pl.w);
        if (!(dist < -kContactThreshold)) continue;
        const MatDev &mw = a.mats[a.plane_mat[s.plane_begin + p]];
        const V3<T> n = v3(T(pl.x), T(pl.y), T(pl.z));
        V3<T> r1;
        if (sizeof(T) == 8) {
            const double f = pi.w + dist;
            const double gx = pi.x - f * pl.x, gy = pi.y - f * pl.y, gz = pi.z - f * pl.z;
            r1 = v3(T(gx - pi.x), T(gy - pi.y), T(gz - pi.z));
        } else {
            r1 = n * (-(T(pi.w) + T(dist)));
        }
        dem_contact<T>(n, T(dist), r1, zero, vi, wi, zero, zero, mi, mw, true, acc);
    }
    for (int k = 0; k < s.nboxes; ++k) {
        const double *B = a.boxes + 15 * (int64_t)(s.box_begin + k);
        const double l0 = 0.5 * B[3], l1 = 0.5 * B[4], l2 = 0.5 * B[5];
        const double *R = B + 6;
        const double dx = pi.x - B[0], dy = pi.y - B[1], dz = pi.z - B[2];
        double p0 = dx * R[0] + dy * R[3] + dz * R[6];
        double p1 = dx * R[1] + dy * R[4] + dz * R[7];
        double p2 = dx * R[2] + dy * R[5] + dz * R[8];
        bool outside = false;
        if (p0 < -l0) { p0 = -l0; outside = true; } else if (p0 > l0) { p0 = l0; outside = true; }
        if (p1 < -l1) { p1 = -l1; outside = true; } else if (p1 > l1) { p1 = l1; outside = true; }
        if (p2 < -l2) { p2 = -l2; outside = true; } else if (p2 > l2) { p2 = l2; outside = true; }
        double nx, ny, nz, dist, gx, gy, gz;
        if (!outside) {
            dist = fabs(p0) - l0;
            int face = 0;
            double pf = p0;
            const double t1 = fabs(p1) - l1;
            if (dist < t1) { dist = t1; face = 1; pf = p1; }
            const double t2 = fabs(p2) - l2;
            if (dist < t2) { dist = t2; face = 2; pf = p2; }
            const double sg = (pf > 0.0) ? 1.0 : -1.0;
            nx = R[face] * sg; ny = R[3 + face] * sg; nz = R[6 + face] * sg;
            dist -= pi.w;
            gx = pi.x; gy = pi.y; gz = pi.z;
        } else {
            const double qx = R[0] * p0 + R[1] * p1 + R[2] * p2;
            const double qy = R[3] * p0 + R[4] * p1 + R[5] * p2;
            const double qz = R[6] * p0 + R[7] * p1 + R[8] * p2;
            const double mx = dx - qx, my = dy - qy, mz = dz - qz;
            const double len = length_rn(mx, my, mz);
            dist = len - pi.w;
            const double il = 1.0 / len;
            nx = mx * il; ny = my * il; nz = mz * il;
            gx = B[0] + qx; gy = B[1] + qy; gz = B[2] + qz;
        }
        if (!(dist < -kContactThreshold)) continue;
        const MatDev &mw = a.mats[a.box_mat[s.box_begin + k]];
        const V3<T> n = v3(T(nx), T(ny), T(nz));
        const V3<T> r1 = v3(T(gx - pi.x), T(gy - pi.y), T(gz - pi.z));
        dem_contact<T>(n, T(dist), r1, zero, vi, wi, zero, zero, mi, mw, true, acc);
    }
}

// SphereTrait::move, Default.h:166-216: new position (radius kept), v and w; writes q.
// Mixed precision: ext carries the linear velocity's extension bytes in and out (internal.cuh);
// the velocity is updated and the position advanced in FP64, then split again.
template <typename VT, bool TRACKQ>
__device__ __forceinline__ double4 integrate_core(const DemArgs<VT> &a, int64_t b, int64_t t,
                                                  const double4 &pi, V3<VT> vi, V3<VT> wi,
                                                  const MatDev &mi, const Acc<VT> &acc,
                                                  V3<VT> &v, V3<VT> &w, uint32_t &ext) {
    using T = VT;
    T im, ii;
    if (sizeof(T) == 8) {
        double dim, dii, I;
        sphere_mass(pi.w, mi.density, dim, dii, I);
        im = T(dim);
        ii = T(dii);
    } else {
        // mixed precision: the same formulas in FP32 (SphereBase.h:169-171, 230-234)
        const float r = float(pi.w);
        const float m = 4.0f / 3.0f * 3.14159265f * r * r * r * float(mi.density);
        im = T(__frcp_rn(m));
        ii = T(__frcp_rn(0.4f * m * r * r));
    }
    const V3<T> gg = v3(T(a.g[0]), T(a.g[1]), T(a.g[2]));
    const V3<T> vdot = acc.F * T(im) + gg;
    const V3<T> wdot = T(ii) * acc.T_;
    w = wi + wdot * T(a.dt);
    double nxp, nyp, nzp;
    double vx = 0.0, vy = 0.0, vz = 0.0;   // mixed: the FP64 linear velocity
    if constexpr (sizeof(T) == 8) {
        v = vi + vdot * T(a.dt);
        nxp = pi.x + double(v.x) * a.dt;
        nyp = pi.y + double(v.y) * a.dt;
        nzp = pi.z + double(v.z) * a.dt;
    } else {
        vx = vext_value(vi.x, ext, 0) + double(vdot.x) * a.dt;
        vy = vext_value(vi.y, ext, 1) + double(vdot.y) * a.dt;
        vz = vext_value(vi.z, ext, 2) + double(vdot.z) * a.dt;
        nxp = pi.x + vx * a.dt;
        nyp = pi.y + vy * a.dt;
        nzp = pi.z + vz * a.dt;
    }
    if (TRACKQ) {
        // q = Quat(phi, |phi|) * q (Quaternion.h:274-294, 1146-1153)
        const double phx = double(w.x) * a.dt, phy = double(w.y) * a.dt, phz = double(w.z) * a.dt;
        const double ang = sqrt(phx * phx + phy * phy + phz * phz);
        double d0 = 1.0, d1 = 0.0, d2 = 0.0, d3 = 0.0;
        if (!(fabs(ang) < 1e-15)) {
            double sa, ca;
            sincos(ang * 0.5, &sa, &ca);
            const double il = 1.0 / ang;
            d0 = ca; d1 = sa * (phx * il); d2 = sa * (phy * il); d3 = sa * (phz * il);
        }
        const double4 q = a.q[b];
        double4 r;
        r.x = d0 * q.x - d1 * q.y - d2 * q.z - d3 * q.w;
        r.y = d0 * q.y + d1 * q.x + d2 * q.w - d3 * q.z;
        r.z = d0 * q.z + d2 * q.x + d3 * q.y - d1 * q.w;
        r.w = d0 * q.w + d3 * q.x + d1 * q.z - d2 * q.y;
        a.q_out[t] = r;
    }
    if constexpr (sizeof(T) == 8) {
        if (a.has_drag) {
            v = v * T(a.drag);
            w = w * T(a.drag);
        }
    } else {
        if (a.has_drag) {
            vx *= a.drag;
            vy *= a.drag;
            vz *= a.drag;
            w = w * T(a.drag);
        }
        ext = 0u;
        v.x = vext_split(vx, ext, 0);
        v.y = vext_split(vy, ext, 1);
        v.z = vext_split(vz, ext, 2);
    }
    if (!isfinite(nxp) || !isfinite(nyp) || !isfinite(nzp)) atomicOr(a.err, DERR_NAN);
    return make_double4(nxp, nyp, nzp, pi.w);
}

// the extension bytes of body i's velocity (zero in FP64)
template <typename VT>
__device__ __forceinline__ uint32_t ld_ext(const VT *vw, int64_t n, int64_t i) {
    if constexpr (sizeof(VT) == 4) return ld_vext(vw, n, i);
    else return 0u;
}

// the same loads through L2 only (data another kernel, still running, has made visible)
__device__ __forceinline__ double4 ld_cg(const double4 *p) {
    const double2 lo = __ldcg(reinterpret_cast<const double2 *>(p));
    const double2 hi = __ldcg(reinterpret_cast<const double2 *>(p) + 1);
    return make_double4(lo.x, lo.y, hi.x, hi.y);
}
template <typename T>
__device__ __forceinline__ V3<T> ld_vw_cg(const T *vw, int64_t n, int64_t i, int which) {
    const T *p = vw + 3 * which * n + i;
    return v3(__ldcg(p), __ldcg(p + n), __ldcg(p + 2 * n));
}
template <typename VT>
__device__ __forceinline__ uint32_t ld_ext_cg(const VT *vw, int64_t n, int64_t i) {
    if constexpr (sizeof(VT) == 4) return __ldcg(reinterpret_cast<const uint32_t *>(vw + 6 * n) + i);
    else return 0u;
}

template <typename VT, bool TRACKQ>
__device__ __forceinline__ double4 integrate(const DemArgs<VT> &a, int64_t b, int64_t t,
                                             const double4 &pi, V3<VT> vi, V3<VT> wi,
                                             const MatDev &mi, const Acc<VT> &acc, V3<VT> &v) {
    V3<VT> w;
    uint32_t ext = ld_ext(a.vw, a.n, b);
    const double4 out = integrate_core<VT, TRACKQ>(a, b, t, pi, vi, wi, mi, acc, v, w, ext);
    a.pr_out[t] = out;
    st_vw(a.vw_out, a.n, t, v, w, ext);
    return out;
}

// all grid neighbours of body b (slot cells of the sphere's scene); the bound is conservative
// for penetrating contacts
template <typename T, typename VT, bool HERTZ>
__device__ __forceinline__ void grid_forces(const DemArgs<VT> &a, const SceneInfo &s, int32_t b,
                                            const double4 &pi, V3<T> vi, V3<T> wi, int32_t uidi,
                                            const MatDev &mi, Acc<T> &acc) {
    int cx, cy, cz;
    cell_coords(s, pi.x, pi.y, pi.z, cx, cy, cz);
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, s.dim[0] - 1);
    for (int dz = -1; dz <= 1; ++dz) {
        const int z = cz + dz;
        if (z < 0 || z >= s.dim[2]) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            const int y = cy + dy;
            if (y < 0 || y >= s.dim[1]) continue;
            const int64_t c0 = cell_key(s, x0, y, z);
            const int64_t c1 = c0 + (x1 - x0) + 1;
            const int e = a.cell_start[c1];
            for (int slot = a.cell_start[c0]; slot < e; ++slot) {
                const int32_t j = a.sorted ? a.sorted[slot] : slot;
                if (j == b) continue;
                const double4 pj = a.pr[j];
                const double ddx = pi.x - pj.x, ddy = pi.y - pj.y, ddz = pi.z - pj.z;
                const double rs = pi.w + pj.w;
                if (ddx * ddx + ddy * ddy + ddz * ddz >= rs * rs) continue;
                pair_force<T, VT, HERTZ>(a, pi, vi, wi, uidi, mi, j, pj, acc);
            }
        }
    }
}

template <typename VT, bool TRACKQ, bool HERTZ>
__global__ void __launch_bounds__(kDemBlock) k_dem_step(DemArgs<VT> a) {
    using T = VT;  // arithmetic type of the contact law (double or float)
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    const int32_t b = a.sorted[t];
    const double4 pi = a.pr[b];
    const uint32_t tagi = a.tag[b];
    const int32_t uidi = a.uid[b];
    const SceneInfo &s = a.scenes[tagi >> 16];
    const MatDev &mi = a.mats[tagi & 0xffffu];
    const V3<T> vi = ld_vw(a.vw, a.n, b, 0), wi = ld_vw(a.vw, a.n, b, 1);
    Acc<T> acc;
    acc.F = v3(T(0), T(0), T(0));
    acc.T_ = acc.F;
    grid_forces<T, VT, HERTZ>(a, s, b, pi, vi, wi, uidi, mi, acc);
    wall_forces<T, VT>(a, s, pi, vi, wi, mi, acc);
    if (a.ext) {
        const double *e = a.ext + 6 * (int64_t)b;
        acc.F = acc.F + v3(T(e[0]), T(e[1]), T(e[2]));
        acc.T_ = acc.T_ + v3(T(e[3]), T(e[4]), T(e[5]));
    }
    V3<T> v;
    const double4 o = integrate<VT, TRACKQ>(a, b, t, pi, vi, wi, mi, acc, v);
    a.tag_out[t] = tagi;
    a.uid_out[t] = uidi;
    // bin for the next step's counting sort
    int ncx, ncy, ncz;
    cell_coords(s, o.x, o.y, o.z, ncx, ncy, ncz);
    const int32_t kk = (int32_t)cell_key(s, ncx, ncy, ncz);
    a.key[t] = kk;
    a.rank[t] = atomicAdd(&a.cell_count[kk], 1);
}

// ---- grid step with a sorted FP32 copy of the positions ---------------------------------------
// The same step as k_dem_step with the 27-cell search reading, per candidate, one 16-byte record
// of the sort's FP32 position copy (posf, slot order: consecutive candidates are consecutive
// records, and no load waits on another) instead of the slot's body index and then its FP64
// record.  Far candidates are rejected by an FP32 test whose margin covers its rounding; the
// survivors take k_dem_step's exact FP64 test and pair force in k_dem_step's order, so the
// results are bitwise those of k_dem_step.
// slots [b, e) of the row of cells (z, y), x0 .. x1 (empty outside the grid)
__device__ __forceinline__ void row_slots(const int32_t *__restrict__ cell_start,
                                          const SceneInfo &s, int x0, int x1, int y, int z,
                                          int &b, int &e) {
    b = e = 0;
    if (z < 0 || z >= s.dim[2] || y < 0 || y >= s.dim[1]) return;
    const int64_t c0 = cell_key(s, x0, y, z);
    b = cell_start[c0];
    e = cell_start[c0 + (x1 - x0) + 1];
}

template <typename T, typename VT, bool HERTZ>
__device__ __forceinline__ void grid_forces_sorted(const DemArgs<VT> &a, const SceneInfo &s,
                                                   const float4 *__restrict__ posf, int64_t self,
                                                   int32_t b,
                                                   const double4 &pi, V3<T> vi, V3<T> wi,
                                                   int32_t uidi, const MatDev &mi, Acc<T> &acc) {
    int cx, cy, cz;
    cell_coords(s, pi.x, pi.y, pi.z, cx, cy, cz);
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, s.dim[0] - 1);
    // coordinates relative to the grid origin, as the sort wrote them
    const float pxf = float(pi.x - s.lo[0]), pyf = float(pi.y - s.lo[1]),
                pzf = float(pi.z - s.lo[2]);
    // |d_fp32 - d| stays below ~1e-7 (|x| + |y| + |z| + 2 r + d) for any partner closer than
    // r_i + r_j; the margin is 100 times that
    const float tol = 1e-5f * (1.0f + fabsf(pxf) + fabsf(pyf) + fabsf(pzf) + 4.0f * float(pi.w));
    const float prf = float(pi.w) + tol;
    // one candidate that passed the FP32 test: k_dem_step's exact test and pair force (the body's
    // own slot is the one candidate k_dem_step skips as j == b)
    auto exact = [&](int slot) {
        if (slot == self) return;
        const int32_t j = a.sorted[slot];
        const double4 pj = a.pr[j];
        const double ddx = pi.x - pj.x, ddy = pi.y - pj.y, ddz = pi.z - pj.z;
        const double rsd = pi.w + pj.w;
        if (ddx * ddx + ddy * ddy + ddz * ddz >= rsd * rsd) return;
        pair_force<T, VT, HERTZ>(a, pi, vi, wi, uidi, mi, j, pj, acc);
    };
    auto near = [&](const float4 &q) {
        const float dx = pxf - q.x, dy = pyf - q.y, dz = pzf - q.z;
        const float rs = prf + q.w;
        return dx * dx + dy * dy + dz * dz < rs * rs;
    };
    // rows (z, y) in k_dem_step's order; the next row's bounds load while this one runs
    int nb, ne;
    row_slots(a.cell_start, s, x0, x1, cy - 1, cz - 1, nb, ne);
#pragma unroll 1
    for (int r = 0; r < 9; ++r) {
        int slot = nb;
        const int e = ne;
        if (r < 8) row_slots(a.cell_start, s, x0, x1, cy + (r + 1) % 3 - 1, cz + (r + 1) / 3 - 1,
                             nb, ne);
        // eight candidate records in flight at a time; the hits keep their slot order
        for (; slot + 8 <= e; slot += 8) {
            unsigned hit = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) hit |= near(posf[slot + k]) ? (1u << k) : 0u;
            while (hit) {
                const int k = __ffs(hit) - 1;
                hit &= hit - 1u;
                exact(slot + k);
            }
        }
        if (slot + 4 <= e) {
            unsigned hit = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) hit |= near(posf[slot + k]) ? (1u << k) : 0u;
            while (hit) {
                const int k = __ffs(hit) - 1;
                hit &= hit - 1u;
                exact(slot + k);
            }
            slot += 4;
        }
        for (; slot < e; ++slot)
            if (near(posf[slot])) exact(slot);
    }
}

// The grid step in two kernels.  k_grid_near (few registers, so many warps hide the candidate
// loads) runs the FP32 test over half of each sphere's 27-cell neighbourhood: the candidates
// in a later slot (in cell order, the rows of the neighbourhood come in increasing cell key, so
// these are the own row's later slots and the whole of the later rows).  Every pair within
// reach is so tested once, by its lower slot, and a pair that passes is recorded for both
// spheres (atomic counters, up to kNear slots each; the counters start at zero).  k_dem_near
// sorts a sphere's recorded slots, which puts them in the order in which k_dem_step's 27-cell
// scan visits them (ascending slot), takes each through k_dem_step's exact test and pair force
// (or, for a sphere with more than kNear, searches its cells again), then the walls and the
// integration.  Same terms in the same order: bitwise the results of k_dem_step.
constexpr int kNear = 16;
constexpr int kNearBlock = 256;

__global__ void __launch_bounds__(kNearBlock, 5) k_grid_near(
    int64_t n, const int32_t *__restrict__ sorted, const double4 *__restrict__ pr,
    const uint32_t *__restrict__ tag, const SceneInfo *__restrict__ scenes,
    const int32_t *__restrict__ cell_start, const float4 *__restrict__ posf,
    int32_t *__restrict__ near_cnt, int32_t *__restrict__ near_idx) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int32_t b = sorted[t];
    const double4 pi = pr[b];
    const SceneInfo &s = scenes[tag[b] >> 16];
    int cx, cy, cz;
    cell_coords(s, pi.x, pi.y, pi.z, cx, cy, cz);
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, s.dim[0] - 1);
    // the values and margin of grid_forces_sorted
    const float pxf = float(pi.x - s.lo[0]), pyf = float(pi.y - s.lo[1]),
                pzf = float(pi.z - s.lo[2]);
    const float tol = 1e-5f * (1.0f + fabsf(pxf) + fabsf(pyf) + fabsf(pzf) + 4.0f * float(pi.w));
    const float prf = float(pi.w) + tol;
    auto near = [&](const float4 &q, float rq) {
        const float dx = pxf - q.x, dy = pyf - q.y, dz = pzf - q.z;
        const float rs = prf + rq;
        return dx * dx + dy * dy + dz * dz < rs * rs;
    };
    // a pair passes for one sphere's margin or the other's (each sphere's test in k_dem_near's
    // fallback uses its own); the larger margin covers both
    auto keep = [&](int slot) {
        const int32_t p = atomicAdd(&near_cnt[t], 1);
        if (p < kNear) near_idx[(int64_t)p * n + t] = slot;
        const int32_t q = atomicAdd(&near_cnt[slot], 1);
        if (q < kNear) near_idx[(int64_t)q * n + slot] = (int32_t)t;
    };
    auto test = [&](int slot) {
        const float4 q = posf[slot];
        // the partner's margin, as its own thread computes it
        const float tq = 1e-5f * (1.0f + fabsf(q.x) + fabsf(q.y) + fabsf(q.z) + 4.0f * q.w);
        return near(q, q.w + fmaxf(tq - tol, 0.0f));
    };
    // the own row's later slots, then the later rows (z, y) of the neighbourhood
#pragma unroll 1
    for (int r = 4; r < 9; ++r) {
        int slot, e;
        row_slots(cell_start, s, x0, x1, cy + r % 3 - 1, cz + r / 3 - 1, slot, e);
        if (r == 4) slot = (int)t + 1;
        for (; slot + 8 <= e; slot += 8) {
            unsigned hit = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) hit |= test(slot + k) ? (1u << k) : 0u;
            while (hit) {
                const int k = __ffs(hit) - 1;
                hit &= hit - 1u;
                keep(slot + k);
            }
        }
        for (; slot < e; ++slot)
            if (test(slot)) keep(slot);
    }
}

template <typename VT, bool TRACKQ, bool HERTZ>
__global__ void __launch_bounds__(kDemBlock) k_dem_near(DemArgs<VT> a,
                                                        const float4 *__restrict__ posf,
                                                        const int32_t *__restrict__ near_cnt,
                                                        const int32_t *__restrict__ near_idx) {
    using T = VT;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    const int32_t b = a.sorted[t];
    const double4 pi = a.pr[b];
    const uint32_t tagi = a.tag[b];
    const int32_t uidi = a.uid[b];
    const int cnt = near_cnt[t];
    const SceneInfo &s = a.scenes[tagi >> 16];
    const MatDev &mi = a.mats[tagi & 0xffffu];
    const V3<T> vi = ld_vw(a.vw, a.n, b, 0), wi = ld_vw(a.vw, a.n, b, 1);
    Acc<T> acc;
    acc.F = v3(T(0), T(0), T(0));
    acc.T_ = acc.F;
    if (cnt > kNear) {
        grid_forces_sorted<T, VT, HERTZ>(a, s, posf, t, b, pi, vi, wi, uidi, mi, acc);
    } else if (cnt > 0) {
        // the recorded slots in ascending order (a sorting network over registers; empty
        // places hold INT_MAX and sort last)
        int32_t sl[kNear];
#pragma unroll
        for (int k = 0; k < kNear; ++k) sl[k] = k < cnt ? near_idx[(int64_t)k * a.n + t] : INT_MAX;
        if (cnt > 1) {
#pragma unroll
            for (int kk = 2; kk <= kNear; kk <<= 1)
#pragma unroll
                for (int j = kk >> 1; j > 0; j >>= 1)
#pragma unroll
                    for (int i = 0; i < kNear; ++i) {
                        const int l = i ^ j;
                        if (l > i) {
                            const int32_t x = sl[i], y = sl[l];
                            const bool up = (i & kk) == 0;
                            if ((x > y) == up) {
                                sl[i] = y;
                                sl[l] = x;
                            }
                        }
                    }
        }
#pragma unroll
        for (int k = 0; k < kNear; ++k) {
            if (k >= cnt) break;
            const int32_t j = a.sorted[sl[k]];
            const double4 pj = a.pr[j];
            const double ddx = pi.x - pj.x, ddy = pi.y - pj.y, ddz = pi.z - pj.z;
            const double rsd = pi.w + pj.w;
            if (ddx * ddx + ddy * ddy + ddz * ddz >= rsd * rsd) continue;
            pair_force<T, VT, HERTZ>(a, pi, vi, wi, uidi, mi, j, pj, acc);
        }
    }
    wall_forces<T, VT>(a, s, pi, vi, wi, mi, acc);
    if (a.ext) {
        const double *e = a.ext + 6 * (int64_t)b;
        acc.F = acc.F + v3(T(e[0]), T(e[1]), T(e[2]));
        acc.T_ = acc.T_ + v3(T(e[3]), T(e[4]), T(e[5]));
    }
    V3<T> v;
    const double4 o = integrate<VT, TRACKQ>(a, b, t, pi, vi, wi, mi, acc, v);
    a.tag_out[t] = tagi;
    a.uid_out[t] = uidi;
    int ncx, ncy, ncz;
    cell_coords(s, o.x, o.y, o.z, ncx, ncy, ncz);
    const int32_t kk = (int32_t)cell_key(s, ncx, ncy, ncz);
    a.key[t] = kk;
    a.rank[t] = atomicAdd(&a.cell_count[kk], 1);
}

// launch shapes of the list step kernel: threads per block and the resident blocks per SM the
// register allocation must allow, for FP32 and FP64 velocities (pe_b200_autotune picks one)
struct DemShape {
    int block, minb_f32, minb_f64;
};
constexpr DemShape kDemShapes[] = {{kDemBlock, PEB_LIST_MIN_BLOCKS_F32, 5},
                                   {256, 3, 2},
                                   {64, 14, 10},
                                   {128, 8, 6},
                                   {128, 6, 4},
                                   {256, 4, 3}};
constexpr int kDemShapeCount = (int)(sizeof(kDemShapes) / sizeof(kDemShapes[0]));

// List step, in two kernels; body t stays at index t (the order changes only at rebuilds).
// The rebuild marks the spheres that can feel a force before the next rebuild -- those with list
// entries, and those within reach of a wall (not inside the box of the scene's planes by
// skin/2, or near a fixed box) -- and lists them in ascending order (act: exclusive offsets of
// the marks, act[n] the count; alist: the marked spheres).  k_dem_contacts sums the pair and
// wall forces of the marked spheres only, in the order of the single-kernel form, into facc;
// k_dem_move then integrates every sphere, reading facc for the marked ones, so the common
// sphere of a sparse scene runs a short kernel without the contact code's registers.

// Forces on the marked spheres m = first, first + stride, ... (a grid-stride loop over the
// marked list), the state read through `a` (the rebuild's copy when the step rebuilt).  SPLIT:
// they are integrated too, on a second stream beside k_dem_move, which then leaves them out;
// else their forces are stored for k_dem_move, which runs after.
template <typename VT, bool HERTZ, bool ONE, bool SPLIT, bool TRACKQ>
__device__ __forceinline__ void contacts_loop(const DemArgs<VT> &a, bool rebuilt, int64_t first,
                                              int64_t stride) {
    using T = VT;
    const int32_t na = a.act[a.n];
    for (int32_t m = (int32_t)first; m < na; m += (int32_t)stride) {
        const int64_t t = a.alist[m];
        const double4 pi = a.pr[t];
        const uint32_t tagi = a.tag[t];
        const V3<T> vi = ld_vw(a.vw, a.n, t, 0), wi = ld_vw(a.vw, a.n, t, 1);
        int k = a.nl_start[t];
        const int e = a.nl_start[t + 1];
        const SceneInfo &s = ONE ? a.s0 : a.scenes[tagi >> 16];
        const MatDev &mi = ONE ? a.m0 : a.mats[tagi & 0xffffu];
        Acc<T> acc;
        acc.F = v3(T(0), T(0), T(0));
        acc.T_ = acc.F;
        // a body without candidates at the last rebuild has no contact partner before the
        // next one, lists or not; the others read whether that rebuild's lists fit
        if (k < e && a.nl_flags[1] != 0) {
            grid_forces<T, VT, HERTZ>(a, s, (int32_t)t, pi, vi, wi, a.uid[t], mi, acc);
        } else if (k < e) {
            // entries: neighbour index, top bit set when this body is pe's body 1; two at a
            // time so their loads overlap
            for (; k + 1 < e; k += 2) {
                const uint32_t e0 = (uint32_t)a.nl_idx[k], e1 = (uint32_t)a.nl_idx[k + 1];
                const int32_t j0 = (int32_t)(e0 & 0x7fffffffu), j1 = (int32_t)(e1 & 0x7fffffffu);
                const double4 p0 = a.pr[j0], p1 = a.pr[j1];
                pair_force_o<T, VT, HERTZ, ONE>(a, pi, vi, wi, mi, j0, p0, (e0 >> 31) != 0u, acc);
                pair_force_o<T, VT, HERTZ, ONE>(a, pi, vi, wi, mi, j1, p1, (e1 >> 31) != 0u, acc);
            }
            if (k < e) {
                const uint32_t e0 = (uint32_t)a.nl_idx[k];
                const int32_t j0 = (int32_t)(e0 & 0x7fffffffu);
                pair_force_o<T, VT, HERTZ, ONE>(a, pi, vi, wi, mi, j0, a.pr[j0], (e0 >> 31) != 0u, acc);
            }
        }
        wall_forces<T, VT>(a, s, pi, vi, wi, mi, acc);
        if constexpr (SPLIT) {
            // the integration of k_dem_move for this sphere
            uint32_t ext = ld_ext(a.vw, a.n, t);
            V3<T> v, w;
            const double4 o = integrate_core<VT, TRACKQ>(a, t, t, pi, vi, wi, mi, acc, v, w, ext);
            a.pr_out[t] = o;
            st_vw(a.vw_out, a.n, t, v, w, ext);
            if (rebuilt) {
                a.tag_out[t] = tagi;
                a.uid_out[t] = a.uid[t];
            }
            const float vx = float(v.x), vy = float(v.y), vz = float(v.z);
            const float d = a.disp[t] + sqrtf(vx * vx + vy * vy + vz * vz) * float(a.dt) * 1.0001f;
            a.disp[t] = d;
            if (!(d < a.half_skin)) atomicOr(&a.nl_flags[0], 1);
        } else {
            const int64_t cap = a.n;
            a.facc[m] = acc.F.x;
            a.facc[cap + m] = acc.F.y;
            a.facc[2 * cap + m] = acc.F.z;
            a.facc[3 * cap + m] = acc.T_.x;
            a.facc[4 * cap + m] = acc.T_.y;
            a.facc[5 * cap + m] = acc.T_.z;
        }
    }
}

template <typename VT, bool HERTZ, bool ONE = false, bool SPLIT = false, bool TRACKQ = false>
__global__ void __launch_bounds__(128) k_dem_contacts(DemArgs<VT> a0) {
    // launched early behind the rebuild kernel: nothing is read before it has finished
    pdl_wait();
    pdl_trigger();
    const bool rebuilt = a0.nl_flags[4] != 0;
    const DemArgs<VT> a = list_view(a0);
    contacts_loop<VT, HERTZ, ONE, SPLIT, TRACKQ>(a, rebuilt, (int64_t)blockIdx.x * blockDim.x + threadIdx.x,
                                                 (int64_t)gridDim.x * blockDim.x);
}

// The list step's rebuild check (and, when requested, the rebuild) and the forces on the marked
// spheres in one cooperative kernel: a step without a rebuild goes straight from the flag to
// the forces, without a kernel boundary between them.  The flag is read by every thread before
// any block writes it; after a rebuild a grid barrier makes the lists and marks visible first.
// SPLIT (the overlapped form): the kernel also integrates the marked spheres, and k_dem_move,
// released at the trigger below, integrates the others meanwhile; it reads the rebuild flag
// and the marks without waiting for this kernel, so they are made visible before the trigger.
// resident blocks per SM the registers of the overlapped form's mixed-precision linear-law
// kernels must allow: 4 (64 registers) took the contact-dense 1M step from 134 to 109 us (more
// warps on the neighbours' loads); 5 and 6 spill too much (118, 147 us); the sparse step is the
// same at all four.  The FP64 and Hertz kernels would spill kilobytes at 64 and keep their own.
#ifndef PEB_FUSED_MINB
#define PEB_FUSED_MINB 4
#endif
template <typename VT, bool HERTZ, bool ONE, bool SPLIT = false>
__global__ void __launch_bounds__(kRbBlock,
                                  (SPLIT && sizeof(VT) == 4 && !HERTZ) ? PEB_FUSED_MINB : 1)
    k_rebuild_contacts(RebuildArgs<VT> ra, DemArgs<VT> da) {
    pdl_wait();
    const bool rebuilt = ra.flags[0] != 0;
    if (rebuilt) {
        if (!rebuild_stages(ra)) return;
        if (!grid_sync(ra.bar, ra.err)) return;
    } else if (blockIdx.x == 0 && threadIdx.x == 0) {
        ra.flags[4] = 0;   // the integration reads the current state
    }
    if constexpr (SPLIT) {
        // after a rebuild the grid barrier has ordered every write of it; without one only the
        // flag written just above is new: block 0 fences it before any of its threads triggers
        if (blockIdx.x == 0) {
            if (threadIdx.x == 0) __threadfence();
            __syncthreads();
        }
    }
    pdl_trigger();
    DemArgs<VT> a = da;
    if (rebuilt) {
        a.pr = da.alt_pr;
        a.vw = da.alt_vw;
        a.tag = da.alt_tag;
        a.uid = da.alt_uid;
        a.q = da.alt_q;
    }
    contacts_loop<VT, HERTZ, ONE, SPLIT, false>(a, rebuilt, (int64_t)blockIdx.x * blockDim.x + threadIdx.x,
                                                (int64_t)gridDim.x * blockDim.x);
}

// integration of every sphere with the forces of k_dem_contacts (SPLIT: of the unmarked ones;
// the contact kernel integrates the marked ones).  SPLIT does not wait for the kernel before it
// (the contact kernel of the overlapped form, which lets it start once the rebuild flag and
// the marks are final): the flag, the marks and, after a rebuild, the copy in cell order are
// read through L2, and one block waits for the contact kernel before it exits, so that the
// next step, which waits for this kernel, also finds the marked spheres integrated.
// Launched after a finished kernel (the two-stream form), the waits return at once.
template <typename VT, bool TRACKQ, int BLOCK, int MINB, bool ONE = false, bool SPLIT = false>
__global__ void __launch_bounds__(BLOCK, MINB) k_dem_move(DemArgs<VT> a0) {
    using T = VT;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    // This body's records of the current state are loaded before waiting for the kernel before
    // this one (launched early behind it): the previous step's integration wrote them and had
    // completed before that kernel could let this one start, and that kernel does not write
    // them.  The first wave's loads so overlap the contact kernel.  After a rebuild they are
    // read again from the copy in cell order, and the path length (zeroed by the rebuild)
    // starts from zero.
    const bool in = t < a0.n;
    double4 pi = make_double4(0.0, 0.0, 0.0, 0.0);
    uint32_t tagi = 0u, ext = 0u;
    V3<T> vi = v3(T(0), T(0), T(0)), wi = vi;
    float disp0 = 0.f;
    if (in) {
        pi = a0.pr[t];
        tagi = ONE ? 0u : a0.tag[t];
        vi = ld_vw(a0.vw, a0.n, t, 0);
        wi = ld_vw(a0.vw, a0.n, t, 1);
        ext = ld_ext(a0.vw, a0.n, t);
        disp0 = a0.disp[t];
    }
    // the next step's rebuild may be scheduled from here on (it waits for this kernel in turn)
    if constexpr (!SPLIT) pdl_wait();
    pdl_trigger();
    // whether this step rebuilt the lists (its state is then the copy in cell order)
    const bool rebuilt = (SPLIT ? __ldcg(&a0.nl_flags[4]) : a0.nl_flags[4]) != 0;
    DemArgs<VT> a = a0;
    bool moved = false;
    if (in) {
        const int32_t m = SPLIT ? __ldcg(&a.act[t]) : a.act[t];
        const bool marked = (SPLIT ? __ldcg(&a.act[t + 1]) : a.act[t + 1]) > m;
        Acc<T> acc;
        acc.F = v3(T(0), T(0), T(0));
        acc.T_ = acc.F;
        if (!(SPLIT && marked)) {
        if (marked) {
            const int64_t cap = a.n;
            acc.F = v3(a.facc[m], a.facc[cap + m], a.facc[2 * cap + m]);
            acc.T_ = v3(a.facc[3 * cap + m], a.facc[4 * cap + m], a.facc[5 * cap + m]);
        }
        if (rebuilt) {
            if constexpr (SPLIT) {
                pi = ld_cg(&a0.alt_pr[t]);
                tagi = __ldcg(&a0.alt_tag[t]);
                vi = ld_vw_cg(a0.alt_vw, a.n, t, 0);
                wi = ld_vw_cg(a0.alt_vw, a.n, t, 1);
                ext = ld_ext_cg(a0.alt_vw, a.n, t);
                a.uid_out[t] = __ldcg(&a0.alt_uid[t]);
            } else {
                pi = a0.alt_pr[t];
                tagi = a0.alt_tag[t];
                vi = ld_vw(a0.alt_vw, a.n, t, 0);
                wi = ld_vw(a0.alt_vw, a.n, t, 1);
                ext = ld_ext(a0.alt_vw, a.n, t);
                a.uid_out[t] = a0.alt_uid[t];
            }
            disp0 = 0.f;
            a.q = a0.alt_q;
            // the reordered tags replace the current ones (the ids just above)
            a.tag_out[t] = tagi;
        }
        const MatDev &mi = ONE ? a.m0 : a.mats[tagi & 0xffffu];
        V3<T> v, w;
        const double4 o = integrate_core<VT, TRACKQ>(a, t, t, pi, vi, wi, mi, acc, v, w, ext);
        // whole 32-byte records: a partial sector write would make L2 fetch the sector first
        a.pr_out[t] = o;
        st_vw(a.vw_out, a.n, t, v, w, ext);
        const float vx = float(v.x), vy = float(v.y), vz = float(v.z);
        const float d = disp0 + sqrtf(vx * vx + vy * vy + vz * vz) * float(a.dt) * 1.0001f;
        a.disp[t] = d;
        moved = !(d < a.half_skin);   // also catches NaN
        }
    }
    if (__any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0) atomicOr(&a.nl_flags[0], 1);
    // after an overflow every step rebuilds until the host has grown the list buffer
    if (t == 0 && (SPLIT ? __ldcg(&a.nl_flags[1]) : a.nl_flags[1]) != 0) atomicOr(&a.nl_flags[0], 1);
    // a grid completes when its last block exits: one block waiting for the contact kernel is
    // enough (the last one, which starts last, so the others do not hold their SM slots)
    if constexpr (SPLIT) {
        if (blockIdx.x == gridDim.x - 1) pdl_wait();
    }
}

template <typename VT>
DemArgs<VT> dem_args(Ctx *c, double dt) {
    DemArgs<VT> a;
    a.n = c->n;
    a.dt = dt;
    for (int k = 0; k < 3; ++k) a.g[k] = c->p.gravity[k];
    a.has_drag = c->p.damping < 1.0;
    a.drag = a.has_drag ? pow(c->p.damping, dt) : 1.0;
    a.sorted = c->sorted;
    a.cell_start = c->cell_start;
    a.scenes = c->d_scenes;
    a.mats = c->d_mats;
    a.planes = c->d_planes;
    a.planes_f = c->d_planes_f;
    a.plane_mat = c->d_plane_mat;
    a.boxes = c->d_boxes;
    a.box_mat = c->d_box_mat;
    a.pr = c->cur.pr;
    a.vw = (const VT *)c->cur.vw;
    a.tag = c->cur.tag;
    a.uid = c->cur.uid;
    a.q = c->cur.q;
    a.pr_out = c->nxt.pr;
    a.vw_out = (VT *)c->nxt.vw;
    a.tag_out = c->nxt.tag;
    a.uid_out = c->nxt.uid;
    a.q_out = c->nxt.q;
    a.key = c->key;
    a.rank = c->rank;
    a.cell_count = c->cell_count;
    a.err = c->d_err;
    a.nl_start = c->nl.start;
    a.nl_idx = c->nl.idx;
    a.disp = c->nl.disp;
    a.nl_flags = c->nl.flags;
    a.half_skin = float(0.5 * c->nl.skin * (1.0 - 1e-5));
    a.hertz = c->p.force_model == 1 ? 1 : 0;
    a.ext = c->mb.m > 0 ? c->mb.ext : nullptr;
    a.act = c->nl.act;
    a.alist = c->nl.alist;
    a.facc = (VT *)c->nl.facc;
    return a;
}

template <typename VT>
int launch_dem(Ctx *c, double dt) {
    DemArgs<VT> a = dem_args<VT>(c, dt);
    prof_begin(c, ST_DEM);
    const unsigned g = grid_for(c->n, kDemBlock);
    if (c->tune.dem_grid == 1) {
        // one thread per sphere, candidates through the sorted order and their FP64 records
        if (a.hertz) {
            if (c->p.track_orientation) k_dem_step<VT, true, true><<<g, kDemBlock, 0, c->stream>>>(a);
            else k_dem_step<VT, false, true><<<g, kDemBlock, 0, c->stream>>>(a);
        } else {
            if (c->p.track_orientation) k_dem_step<VT, true, false><<<g, kDemBlock, 0, c->stream>>>(a);
            else k_dem_step<VT, false, false><<<g, kDemBlock, 0, c->stream>>>(a);
        }
    } else {
        const float4 *pf = c->posf;
        const int32_t *nc = c->near, *ni = c->near + c->n;
        PEB_CUDA(c, cudaMemsetAsync(c->near, 0, (size_t)c->n * sizeof(int32_t), c->stream));
        k_grid_near<<<grid_for(c->n, kNearBlock), kNearBlock, 0, c->stream>>>(
            c->n, c->sorted, c->cur.pr, c->cur.tag, c->d_scenes, c->cell_start, pf, c->near,
            c->near + c->n);
        PEB_LAUNCHED(c);
        if (a.hertz) {
            if (c->p.track_orientation) k_dem_near<VT, true, true><<<g, kDemBlock, 0, c->stream>>>(a, pf, nc, ni);
            else k_dem_near<VT, false, true><<<g, kDemBlock, 0, c->stream>>>(a, pf, nc, ni);
        } else {
            if (c->p.track_orientation) k_dem_near<VT, true, false><<<g, kDemBlock, 0, c->stream>>>(a, pf, nc, ni);
            else k_dem_near<VT, false, false><<<g, kDemBlock, 0, c->stream>>>(a, pf, nc, ni);
        }
    }
    PEB_LAUNCHED(c);
    prof_end(c, ST_DEM);
    return PE_B200_OK;
}

// ---- list rebuild (every kernel returns at once unless a rebuild was requested) -------------
__global__ void k_zero_c(int32_t *p, int64_t n, const int32_t *cond) {
    if (!*cond) return;
    GRID_STRIDE(i, n) p[i] = 0;
}

__global__ void k_bin_c(int64_t n, const double4 *pr, const uint32_t *tag,
                        const SceneInfo *scenes, int32_t *key, int32_t *rank,
                        int32_t *cell_count, const int32_t *cond) {
    if (!*cond) return;
    GRID_STRIDE(i, n) {
        const double4 p = pr[i];
        const SceneInfo &s = scenes[tag[i] >> 16];
        int cx, cy, cz;
        cell_coords(s, p.x, p.y, p.z, cx, cy, cz);
        const int32_t k = (int32_t)cell_key(s, cx, cy, cz);
        key[i] = k;
        rank[i] = atomicAdd(&cell_count[k], 1);
    }
}

__global__ void k_scatter_c(int64_t n, const int32_t *key, const int32_t *rank,
                            const int32_t *start, int32_t *sorted, const int32_t *cond) {
    if (!*cond) return;
    GRID_STRIDE(i, n) sorted[start[key[i]] + rank[i]] = (int32_t)i;
}

__global__ void k_fixup_c(int64_t ncell, const int32_t *start, int32_t *sorted,
                          const int32_t *cond) {
    if (!*cond) return;
    GRID_STRIDE(c, ncell) {
        const int b = start[c], e = start[c + 1];
        for (int i = b + 1; i < e; ++i) {
            const int32_t v = sorted[i];
            int j = i - 1;
            while (j >= b && sorted[j] > v) {
                sorted[j + 1] = sorted[j];
                --j;
            }
            sorted[j + 1] = v;
        }
    }
}

// gather into cell order (tmp), resetting the path lengths
template <typename VT>
__global__ void k_permute_c(int64_t n, const int32_t *sorted, BodyBuf src, BodyBuf dst,
                            float *disp, const int32_t *cond) {
    if (!*cond) return;
    GRID_STRIDE(t, n) {
        const int32_t b = sorted[t];
        dst.pr[t] = src.pr[b];
        cp_vw((VT *)dst.vw, t, (const VT *)src.vw, b, n);
        dst.tag[t] = src.tag[b];
        dst.uid[t] = src.uid[b];
        if (src.q) dst.q[t] = src.q[b];
        disp[t] = 0.f;
    }
}

// neighbours of body t (state in cell order, so slot == index): pairs closer than
// r_i + r_j + skin.  mode 0 counts, mode 1 writes.
template <int MODE>
__global__ void k_list(int64_t n, const double4 *pr, const uint32_t *tag, const int32_t *uid,
                       const SceneInfo *scenes, const int32_t *cell_start, double skin,
                       int32_t *cnt, const int32_t *start, int64_t cap, int32_t *idx,
                       const int32_t *cond) {
    if (!*cond) return;
    if (MODE == 1 && start[n] > cap) return;  // overflow: the force kernel searches the grid
    GRID_STRIDE(t, n) {
    const double4 pi = pr[t];
    const SceneInfo &s = scenes[tag[t] >> 16];
    int cx, cy, cz;
    cell_coords(s, pi.x, pi.y, pi.z, cx, cy, cz);
    // only the cells within reach of the sphere (a partner is at most r_max + skin further)
    const double reach = (pi.w + s.rmax + skin) * (1.0 + 1e-12) + 1e-12;
    int x0, x1, y0, y1, z0, z1;
    search_range(s, 0, pi.x, reach, cx, x0, x1);
    search_range(s, 1, pi.y, reach, cy, y0, y1);
    search_range(s, 2, pi.z, reach, cz, z0, z1);
    int pos = (MODE == 1) ? start[t] : 0;
    int count = 0;
    for (int z = z0; z <= z1; ++z) {
        for (int y = y0; y <= y1; ++y) {
            const int64_t c0 = cell_key(s, x0, y, z);
            const int64_t c1 = c0 + (x1 - x0) + 1;
            const int e = cell_start[c1];
            for (int j = cell_start[c0]; j < e; ++j) {
                if (j == t) continue;
                const double4 pj = pr[j];
                const double dx = pi.x - pj.x, dy2 = pi.y - pj.y, dz2 = pi.z - pj.z;
                const double rc = pi.w + pj.w + skin;
                if (dx * dx + dy2 * dy2 + dz2 * dz2 < rc * rc) {
                    if (MODE == 1)
                        idx[pos++] = (int32_t)((uint32_t)j | (uid[t] < uid[j] ? 0x80000000u : 0u));
                    ++count;
                }
            }
        }
    }
    if (MODE == 0) cnt[t] = count;
    }
}

// the list step's marks (internal.cuh list_marked) from the neighbour counts
__global__ void k_mark_c(int64_t n, const double4 *pr, const uint32_t *tag, const SceneInfo *scenes,
                         const double *boxes, double margin, const int32_t *cnt, int32_t *act,
                         const int32_t *cond) {
    if (!*cond) return;
    GRID_STRIDE(t, n) act[t] = list_marked(scenes[tag[t] >> 16], pr[t], boxes, margin, cnt[t]) ? 1 : 0;
}

__global__ void k_alist_c(int64_t n, const int32_t *act, int32_t *alist, const int32_t *cond) {
    if (!*cond) return;
    GRID_STRIDE(t, n) if (act[t + 1] > act[t]) alist[act[t]] = (int32_t)t;
}

__global__ void k_rebuild_done(int64_t n, const int32_t *start, int64_t cap, int32_t *flags) {
    flags[4] = flags[0] ? 1 : 0;   // the force kernels read the copy in cell order
    if (!flags[0]) return;
    flags[0] = 0;
    flags[1] = start[n] > cap ? 1 : 0;
    flags[2] = start[n];
    flags[3] += 1;
}

template <typename VT>
int list_rebuild(Ctx *c) {
    ListBuf &L = c->nl;
    const int64_t n = c->n;
    const int32_t *cond = L.flags;
    prof_begin(c, ST_REBUILD);
    k_zero_c<<<capped_grid(c, c->ncell + 1, 256), 256, 0, c->stream>>>(c->cell_count, c->ncell + 1, cond);
    PEB_LAUNCHED(c);
    k_bin_c<<<capped_grid(c, n, 256), 256, 0, c->stream>>>(n, c->cur.pr, c->cur.tag, c->d_scenes,
                                                     c->key, c->rank, c->cell_count, cond);
    PEB_LAUNCHED(c);
    int rc = scan_exclusive_cond(c, c->cell_count, c->cell_start, c->ncell, cond);
    if (rc) return rc;
    k_scatter_c<<<capped_grid(c, n, 256), 256, 0, c->stream>>>(n, c->key, c->rank, c->cell_start,
                                                         c->sorted, cond);
    PEB_LAUNCHED(c);
    k_fixup_c<<<capped_grid(c, c->ncell, 256), 256, 0, c->stream>>>(c->ncell, c->cell_start, c->sorted,
                                                             cond);
    PEB_LAUNCHED(c);
    k_permute_c<VT><<<capped_grid(c, n, 256), 256, 0, c->stream>>>(n, c->sorted, c->cur, L.tmp, L.disp,
                                                             cond);
    PEB_LAUNCHED(c);
    k_list<0><<<capped_grid(c, n, 128), 128, 0, c->stream>>>(n, L.tmp.pr, L.tmp.tag, L.tmp.uid, c->d_scenes,
                                                       c->cell_start, L.skin, L.cnt, nullptr, 0,
                                                       nullptr, cond);
    PEB_LAUNCHED(c);
    k_mark_c<<<capped_grid(c, n, 256), 256, 0, c->stream>>>(n, L.tmp.pr, L.tmp.tag, c->d_scenes,
                                                          c->d_boxes, 0.5 * L.skin * (1.0 + 1e-9),
                                                          L.cnt, L.act, cond);
    PEB_LAUNCHED(c);
    rc = scan_exclusive_cond(c, L.cnt, L.start, n, cond);
    if (rc) return rc;
    rc = scan_exclusive_cond(c, L.act, L.act, n, cond);
    if (rc) return rc;
    k_alist_c<<<capped_grid(c, n, 256), 256, 0, c->stream>>>(n, L.act, L.alist, cond);
    PEB_LAUNCHED(c);
    k_list<1><<<capped_grid(c, n, 128), 128, 0, c->stream>>>(n, L.tmp.pr, L.tmp.tag, L.tmp.uid, c->d_scenes,
                                                       c->cell_start, L.skin, nullptr, L.start,
                                                       L.cap, L.idx, cond);
    PEB_LAUNCHED(c);
    k_rebuild_done<<<1, 1, 0, c->stream>>>(n, L.start, L.cap, L.flags);
    PEB_LAUNCHED(c);
    prof_end(c, ST_REBUILD);
    return PE_B200_OK;
}

// the second stream and the two events of the split list step, created on first use
bool split_streams(Ctx *c) {
    if (c->side) return true;
    if (c->split_failed) return false;
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    if (cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, hi) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        c->split_failed = true;
        return false;
    }
    return true;
}

// contacts_done: the fused rebuild-and-contacts kernel has run (1: it stored the marked spheres'
// forces; 2: the overlapped form, it integrates them too)
template <typename VT, bool TRACKQ, int V, bool HERTZ>
void launch_list_shape(Ctx *c, const DemArgs<VT> &a, int contacts_done) {
    static_assert(V >= 0 && V < kDemShapeCount, "launch shape index");
    constexpr int B = kDemShapes[V].block;
    constexpr int M = sizeof(VT) == 4 ? kDemShapes[V].minb_f32 : kDemShapes[V].minb_f64;
    const bool one = c->nscenes == 1 && c->mats_dev.size() == 1 && !TRACKQ && !HERTZ;
    if (c->tune.dem_split == 1 && !contacts_done && split_streams(c)) {
        // the marked spheres (forces and integration) on the second stream, beside the
        // integration of the others: both start once the rebuild kernel has finished, and the
        // next step waits for both
        const unsigned gc = (unsigned)std::min<int64_t>(grid_for(c->n, 128), 8 * (int64_t)c->sm_count);
        const unsigned gm = (unsigned)grid_for(c->n, B);
        cudaEventRecord(c->ev_fork, c->stream);
        cudaStreamWaitEvent(c->side, c->ev_fork, 0);
        DemArgs<VT> b = a;
        if (one) {
            b.s0 = c->scenes[0];
            b.m0 = c->mats_dev[0];
            k_dem_contacts<VT, HERTZ, true, true, TRACKQ><<<gc, 128, 0, c->side>>>(b);
            k_dem_move<VT, TRACKQ, B, M, true, true><<<gm, B, 0, c->stream>>>(b);
        } else {
            k_dem_contacts<VT, HERTZ, false, true, TRACKQ><<<gc, 128, 0, c->side>>>(b);
            k_dem_move<VT, TRACKQ, B, M, false, true><<<gm, B, 0, c->stream>>>(b);
        }
        c->launches++;
        cudaEventRecord(c->ev_join, c->side);
        cudaStreamWaitEvent(c->stream, c->ev_join, 0);
        return;
    }
    // each kernel is scheduled while the one before it finishes (a rebuild that has nothing to
    // do lets the contact kernel start at once)
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    // the contact kernel strides over the marked spheres, whose count only the device knows:
    // as many blocks as stay resident (all spheres may be marked in a contact-dense scene)
    static int occ[2] = {0, 0};
    int &oc = occ[one ? 1 : 0];
    if (oc == 0) {
        const void *kc = one ? (const void *)k_dem_contacts<VT, HERTZ, true>
                             : (const void *)k_dem_contacts<VT, HERTZ, false>;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&oc, kc, 128, 0) != cudaSuccess || oc < 1) {
            cudaGetLastError();
            oc = 4;
        }
    }
    cudaLaunchConfig_t cc = {};
    cc.gridDim = dim3((unsigned)std::min<int64_t>(grid_for(c->n, 128), (int64_t)oc * c->sm_count));
    cc.blockDim = dim3(128);
    cc.stream = c->stream;
    cc.attrs = at;
    cc.numAttrs = 1;
    cudaLaunchConfig_t cm = cc;
    cm.gridDim = dim3((unsigned)grid_for(c->n, B));
    cm.blockDim = dim3(B);
    if (one) {
        DemArgs<VT> b = a;
        b.s0 = c->scenes[0];
        b.m0 = c->mats_dev[0];
        if (!contacts_done) {
            cudaLaunchKernelEx(&cc, k_dem_contacts<VT, HERTZ, true>, b);
            c->launches++;
        }
        if (contacts_done == 2) cudaLaunchKernelEx(&cm, k_dem_move<VT, TRACKQ, B, M, true, true>, b);
        else cudaLaunchKernelEx(&cm, k_dem_move<VT, TRACKQ, B, M, true>, b);
    } else {
        if (!contacts_done) {
            cudaLaunchKernelEx(&cc, k_dem_contacts<VT, HERTZ, false>, a);
            c->launches++;
        }
        if (contacts_done == 2) cudaLaunchKernelEx(&cm, k_dem_move<VT, TRACKQ, B, M, false, true>, a);
        else cudaLaunchKernelEx(&cm, k_dem_move<VT, TRACKQ, B, M, false>, a);
    }
}

// The fused rebuild-and-contacts kernel for one law and record source: cooperative, and
// scheduled while the force kernel before it finishes.  *fused 0: not launched (the kernel
// cannot be resident, or the driver refused it), the step runs the separate kernels; 1 or 2
// (SPLIT, the overlapped form): launched.
template <typename VT, bool HERTZ, bool ONE, bool SPLIT>
int launch_rebuild_contacts_t(Ctx *c, const DemArgs<VT> &a, int *fused) {
    ListBuf &L = c->nl;
    static int occ = 0;
    if (occ == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_rebuild_contacts<VT, HERTZ, ONE, SPLIT>,
                                                          kRbBlock, 0) != cudaSuccess || occ < 1) {
            cudaGetLastError();
            occ = 0;
            L.fuse_off = true;
            return PE_B200_OK;
        }
    }
    RebuildArgs<VT> ra;
    unsigned grid = 0;
    int rc = rebuild_setup<VT>(c, occ, ra, &grid);
    if (rc) return rc;
    DemArgs<VT> b = a;
    if (ONE) {
        b.s0 = c->scenes[0];
        b.m0 = c->mats_dev[0];
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kRbBlock);
    cfg.stream = c->stream;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = L.rebuild_pdl_off ? 1 : 2;
    if (cudaLaunchKernelEx(&cfg, k_rebuild_contacts<VT, HERTZ, ONE, SPLIT>, ra, b) != cudaSuccess) {
        cudaGetLastError();
        L.fuse_off = true;
        return PE_B200_OK;
    }
    c->launches++;
    *fused = SPLIT ? 2 : 1;
    return PE_B200_OK;
}

// ovl: the overlapped form (sphere orientations not tracked)
template <typename VT>
int launch_rebuild_contacts(Ctx *c, const DemArgs<VT> &a, bool ovl, int *fused) {
    *fused = 0;
    const bool track = c->p.track_orientation != 0;
    const bool one = c->nscenes == 1 && c->mats_dev.size() == 1 && !track && !a.hertz;
    if (ovl && !track) {
        if (a.hertz) return launch_rebuild_contacts_t<VT, true, false, true>(c, a, fused);
        return one ? launch_rebuild_contacts_t<VT, false, true, true>(c, a, fused)
                   : launch_rebuild_contacts_t<VT, false, false, true>(c, a, fused);
    }
    if (a.hertz) return launch_rebuild_contacts_t<VT, true, false, false>(c, a, fused);
    return one ? launch_rebuild_contacts_t<VT, false, true, false>(c, a, fused)
               : launch_rebuild_contacts_t<VT, false, false, false>(c, a, fused);
}

template <typename VT>
int list_step(Ctx *c, double dt) {
    ListBuf &L = c->nl;
    DemArgs<VT> a = dem_args<VT>(c, dt);
    a.sorted = nullptr;   // the grid fallback sees the state in cell order
    a.alt_pr = L.tmp.pr;
    a.alt_vw = (const VT *)L.tmp.vw;
    a.alt_tag = L.tmp.tag;
    a.alt_uid = L.tmp.uid;
    a.alt_q = L.tmp.q;
    a.tag_out = c->cur.tag;   // tags and ids stay in place (reordered there after a rebuild)
    a.uid_out = c->cur.uid;
    prof_begin(c, ST_REBUILD);
    int rc = PE_B200_OK;
    // the rebuild check and the contact forces in one kernel (not while profiling, whose stage
    // timers keep the two apart, nor in the two-stream form)
    int fused = 0;
    if (!L.coop_disabled && c->tune.rebuild_per_sm >= 0 && c->tune.dem_split != 1 && !c->prof &&
        !L.fuse_off) {
        rc = launch_rebuild_contacts<VT>(c, a, c->tune.dem_split == 2, &fused);
        if (rc) return rc;
    }
    if (fused) {
    } else if (!L.coop_disabled && c->tune.rebuild_per_sm >= 0) {
        rc = dem_list_rebuild_persistent(c);
        if (rc != PE_B200_OK) {
            // no cooperative launch here: the rebuild kernels run one by one and return at
            // once unless a rebuild was requested
            L.coop_disabled = true;
            cudaGetLastError();
            c->err.clear();
            rc = list_rebuild<VT>(c);
        }
    } else {
        rc = list_rebuild<VT>(c);
    }
    prof_end(c, ST_REBUILD);
    if (rc) return rc;
    prof_begin(c, ST_DEM);
    // the Hertz law and orientation tracking run the default launch shape
    if (a.hertz)
        c->p.track_orientation ? launch_list_shape<VT, true, 0, true>(c, a, fused)
                               : launch_list_shape<VT, false, 0, true>(c, a, fused);
    else if (c->p.track_orientation)
        launch_list_shape<VT, true, 0, false>(c, a, fused);
    else
        switch (c->tune.dem_variant) {
            case 1: launch_list_shape<VT, false, 1, false>(c, a, fused); break;
            case 2: launch_list_shape<VT, false, 2, false>(c, a, fused); break;
            case 3: launch_list_shape<VT, false, 3, false>(c, a, fused); break;
            case 4: launch_list_shape<VT, false, 4, false>(c, a, fused); break;
            case 5: launch_list_shape<VT, false, 5, false>(c, a, fused); break;
            default: launch_list_shape<VT, false, 0, false>(c, a, fused); break;
        }
    PEB_LAUNCHED(c);
    prof_end(c, ST_DEM);
    // positions/velocities/orientations double-buffered; tag and uid stay where they are
    std::swap(c->cur.pr, c->nxt.pr);
    std::swap(c->cur.vw, c->nxt.vw);
    std::swap(c->cur.q, c->nxt.q);
    return PE_B200_OK;
}

__global__ void k_set_one(int32_t *p) { *p = 1; }

}  // namespace

int dem_step(Ctx *c, double dt) {
    int rc;
    if (c->n > 0) {
        if (!c->binned) {
            rc = grid_bin_current(c);
            if (rc) return rc;
        }
        // the sorted FP32 position copy of the default grid form
        const bool with_pos = c->tune.dem_grid != 1;
        if (with_pos && !c->posf) {
            PEB_CUDA(c, dmalloc(c, &c->posf, (size_t)c->n * sizeof(float4)));
            PEB_CUDA(c, dmalloc(c, &c->near, (size_t)c->n * (1 + kNear) * sizeof(int32_t)));
        }
        rc = grid_sort(c, with_pos);
        if (rc) return rc;
    }
    // moving boxes: their forces on the spheres and their own step, from the current state
    rc = mbox_dem(c, dt);
    if (rc) return rc;
    if (c->n > 0) {
        rc = (c->p.precision == PE_B200_FP64) ? launch_dem<double>(c, dt) : launch_dem<float>(c, dt);
        if (rc) return rc;
        std::swap(c->cur, c->nxt);
    }
    if (c->mb.m > 0) mbox_swap(c);
    return PE_B200_OK;
}

// ---- list mode: buffers, rebuild requests, the capacity check ------------------------------
int dem_list_alloc(Ctx *c) {
    ListBuf &L = c->nl;
    const size_t n = (size_t)std::max<int64_t>(c->n, 1);
    L.cap = c->p.max_contacts > 0 ? c->p.max_contacts : std::max<int64_t>(16 * c->n, 1024);
    PEB_CUDA(c, dmalloc(c, &L.start, (n + 2) * sizeof(int32_t)));
    PEB_CUDA(c, dmalloc(c, &L.cnt, (n + 2) * sizeof(int32_t)));
    PEB_CUDA(c, dmalloc(c, &L.idx, (size_t)L.cap * sizeof(int32_t)));
    PEB_CUDA(c, dmalloc(c, &L.disp, n * sizeof(float)));
    PEB_CUDA(c, dmalloc(c, &L.flags, 8 * sizeof(int32_t)));
    PEB_CUDA(c, cudaMemsetAsync(L.flags, 0, 8 * sizeof(int32_t), c->stream));
    PEB_CUDA(c, cudaMemsetAsync(L.disp, 0, n * sizeof(float), c->stream));
    if (!L.h_flags) PEB_CUDA(c, cudaMallocHost(&L.h_flags, 8 * sizeof(int32_t)));
    if (!L.ev) PEB_CUDA(c, cudaEventCreateWithFlags(&L.ev, cudaEventDisableTiming));
    PEB_CUDA(c, dmalloc(c, &L.rb_bar, 2 * sizeof(unsigned int)));
    PEB_CUDA(c, cudaMemsetAsync(L.rb_bar, 0, 2 * sizeof(unsigned int), c->stream));
    // the per-block partial sums of every rebuild kernel (fused or not, any CTAs per SM), sized
    // once for the largest cooperative grid of kRbBlock threads: a step never allocates, so a
    // step captured into a graph never frees or allocates a buffer (a stream-ordered free in a
    // capture must name a graph allocation)
    {
        int tpsm = 2048;
        if (cudaDeviceGetAttribute(&tpsm, cudaDevAttrMaxThreadsPerMultiProcessor, c->device) !=
            cudaSuccess || tpsm < kRbBlock) {
            cudaGetLastError();
            tpsm = 2048;
        }
        const int64_t blk = (int64_t)(tpsm / kRbBlock) * std::max(c->sm_count, 1) + 1;
        PEB_CUDA(c, dmalloc(c, &L.rb_blk, (size_t)blk * sizeof(int32_t)));
        L.rb_blk_cap = blk;
    }
    PEB_CUDA(c, dmalloc(c, &L.tmp.pr, n * sizeof(double4)));
    PEB_CUDA(c, dmalloc(c, &L.tmp.vw, n * (size_t)c->vw_bytes));
    PEB_CUDA(c, dmalloc(c, &L.tmp.tag, n * sizeof(uint32_t)));
    PEB_CUDA(c, dmalloc(c, &L.tmp.uid, n * sizeof(int32_t)));
    PEB_CUDA(c, dmalloc(c, &L.stash, (size_t)kListStash * n * sizeof(int32_t)));
    PEB_CUDA(c, dmalloc(c, &L.act, (n + 2) * sizeof(int32_t)));
    PEB_CUDA(c, cudaMemsetAsync(L.act, 0, (n + 2) * sizeof(int32_t), c->stream));
    PEB_CUDA(c, dmalloc(c, &L.alist, n * sizeof(int32_t)));
    PEB_CUDA(c, dmalloc(c, &L.facc, 6 * n * (c->p.precision == PE_B200_FP64 ? 8 : 4)));
    if (c->p.track_orientation) PEB_CUDA(c, dmalloc(c, &L.tmp.q, n * sizeof(double4)));
    L.enabled = true;
    L.check_pending = false;
    L.warm = false;
    return dem_list_request_rebuild(c);
}

void dem_list_free(Ctx *c) {
    ListBuf &L = c->nl;
    dem_graph_free(c);
    if (L.check_pending && L.ev) cudaEventSynchronize(L.ev);
    dfree(c, L.rb_bar);
    dfree(c, L.rb_blk);
    dfree(c, L.start);
    dfree(c, L.cnt);
    dfree(c, L.idx);
    dfree(c, L.disp);
    dfree(c, L.flags);
    dfree(c, L.tmp.pr);
    dfree(c, L.tmp.vw);
    dfree(c, L.tmp.tag);
    dfree(c, L.tmp.uid);
    dfree(c, L.tmp.q);
    dfree(c, L.stash);
    dfree(c, L.act);
    dfree(c, L.alist);
    dfree(c, L.facc);
    if (L.h_flags) cudaFreeHost(L.h_flags);
    if (L.ev) cudaEventDestroy(L.ev);
    const double skin = L.skin;
    L = ListBuf();
    L.skin = skin;
}

int dem_list_request_rebuild(Ctx *c) {
    k_set_one<<<1, 1, 0, c->stream>>>(c->nl.flags);
    PEB_LAUNCHED(c);
    return PE_B200_OK;
}

namespace {

// capacity check of an earlier step, without waiting for the device: a rebuild whose lists did
// not fit (the step then searched the grid) grows the list buffer and asks for a new rebuild
int list_capacity_check(Ctx *c) {
    ListBuf &L = c->nl;
    if (L.check_pending && cudaEventQuery(L.ev) == cudaSuccess) {
        L.check_pending = false;
        if (L.h_flags[1]) {
            PEB_CUDA(c, cudaStreamSynchronize(c->stream));
            const int64_t need = std::max<int64_t>(L.h_flags[2], 0);
            const int64_t cap = std::max<int64_t>(2 * L.cap, need + need / 4 + 1024);
            dfree(c, L.idx);
            L.idx = nullptr;
            PEB_CUDA(c, dmalloc(c, &L.idx, (size_t)cap * sizeof(int32_t)));
            L.cap = cap;
            c->epoch++;
            int rc = dem_list_request_rebuild(c);
            if (rc) return rc;
        }
    }
    return PE_B200_OK;
}

// queues the read-back of the rebuild flags that list_capacity_check looks at
// A read-back is a copy in the stream between two kernels, so it is queued once every
// kCheckEvery steps: a list overflow (which only a rebuild can cause) is noticed that much later,
// and the steps in between search the grid for the spheres that have candidates.
constexpr int kCheckEvery = 8;

int list_queue_check(Ctx *c, int steps = 1) {
    ListBuf &L = c->nl;
    L.since_check += steps;
    if (L.since_check < kCheckEvery) return PE_B200_OK;
    if (!L.check_pending) {
        L.since_check = 0;
        PEB_CUDA(c, cudaMemcpyAsync(L.h_flags, L.flags, 4 * sizeof(int32_t),
                                    cudaMemcpyDeviceToHost, c->stream));
        PEB_CUDA(c, cudaEventRecord(L.ev, c->stream));
        L.check_pending = true;
    }
    return PE_B200_OK;
}

int list_step_any(Ctx *c, double dt) {
    return (c->p.precision == PE_B200_FP64) ? list_step<double>(c, dt) : list_step<float>(c, dt);
}

void graph_key(const Ctx *c, const void *key[12]) {
    const void *k[12] = {c->cur.pr, c->cur.vw, c->cur.q, c->cur.tag, c->cur.uid, c->nxt.pr,
                         c->nxt.vw, c->nxt.q, c->nl.idx, (const void *)(intptr_t)c->nl.cap,
                         (const void *)(intptr_t)c->n, c->nl.rb_blk};
    for (int i = 0; i < 12; ++i) key[i] = k[i];
}

// Captures steps list steps into c->sg.  Nothing runs on the device during a capture, so a
// failed capture leaves the context exactly as it was and only switches graphs off.
int capture_steps(Ctx *c, int32_t steps, double dt) {
    StepGraph &G = c->sg;
    dem_graph_free(c);
    const BodyBuf cur0 = c->cur, nxt0 = c->nxt;
    const bool coop0 = c->nl.coop_disabled;
    const int64_t l0 = c->launches;
    const void *key[12];
    graph_key(c, key);
    cudaGraph_t g = nullptr;
    int rc = PE_B200_OK;
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        for (int32_t k = 0; k < steps && rc == PE_B200_OK; ++k) rc = list_step_any(c, dt);
        const cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
        if (e == cudaSuccess) e = e2;
    }
    const int64_t per_replay = c->launches - l0;
    c->launches = l0;
    bool ok = e == cudaSuccess && rc == PE_B200_OK && g != nullptr &&
              c->nl.coop_disabled == coop0 && c->cur.pr == cur0.pr && c->cur.vw == cur0.vw;
    if (ok) ok = cudaGraphInstantiate(&G.exec, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    if (!ok) {
        if (G.exec) cudaGraphExecDestroy(G.exec);
        G.exec = nullptr;
        G.failed = true;
        c->cur = cur0;
        c->nxt = nxt0;
        c->nl.coop_disabled = coop0;
        cudaGetLastError();
        c->err.clear();
        return PE_B200_OK;
    }
    G.steps = steps;
    G.dt = dt;
    G.epoch = c->epoch;
    for (int i = 0; i < 12; ++i) G.key[i] = key[i];
    G.launches = per_replay;
    c->graph_captures++;
    return PE_B200_OK;
}

}  // namespace

int dem_list_step(Ctx *c, double dt) {
    if (c->n == 0) return PE_B200_OK;
    int rc = list_capacity_check(c);
    if (rc) return rc;
    rc = list_step_any(c, dt);
    if (rc) return rc;
    c->nl.warm = true;
    return list_queue_check(c);
}

void dem_graph_free(Ctx *c) {
    if (c->sg.exec) cudaGraphExecDestroy(c->sg.exec);
    c->sg.exec = nullptr;
    c->sg.steps = 0;
}

int dem_list_graph_run(Ctx *c, int32_t nsteps, double dt, int32_t *done) {
    *done = 0;
    StepGraph &G = c->sg;
    // an even count: the buffer swaps of one replay cancel, so every replay starts on the
    // buffers the graph was captured on
    const int32_t gs = c->graph_steps & ~1;
    if (c->n == 0 || gs < 2 || G.failed) return PE_B200_OK;
    while (nsteps - *done >= gs) {
        int rc = list_capacity_check(c);
        if (rc) return rc;
        if (!c->nl.warm) {
            // first step on fresh buffers: allocations happen outside any capture
            rc = dem_list_step(c, dt);
            if (rc) return rc;
            ++*done;
            continue;
        }
        const void *key[12];
        graph_key(c, key);
        bool match = G.exec && G.steps == gs && G.dt == dt && G.epoch == c->epoch;
        for (int i = 0; i < 12 && match; ++i) match = G.key[i] == key[i];
        if (!match) {
            rc = capture_steps(c, gs, dt);
            if (rc) return rc;
            if (G.failed) return PE_B200_OK;
        }
        PEB_CUDA(c, cudaGraphLaunch(G.exec, c->stream));
        c->launches += G.launches;
        c->graph_replays++;
        *done += gs;
        rc = list_queue_check(c, gs);
        if (rc) return rc;
    }
    return PE_B200_OK;
}

int dem_variant_count() { return kDemShapeCount; }

// Launches the FP64 step kernel on caller-provided buffers (used by the allocation-free entry
// point in noalloc.cu); every pointer is device memory the caller owns.
cudaError_t dem_launch_fp64_raw(const DemRawArgs &r, cudaStream_t stream) {
    DemArgs<double> a;
    a.n = r.n;
    a.dt = r.dt;
    for (int k = 0; k < 3; ++k) a.g[k] = r.g[k];
    a.has_drag = r.damping < 1.0;
    a.drag = a.has_drag ? pow(r.damping, r.dt) : 1.0;
    a.sorted = r.sorted;
    a.cell_start = r.cell_start;
    a.scenes = r.scenes;
    a.mats = r.mats;
    a.planes = r.planes;
    a.planes_f = nullptr;
    a.plane_mat = r.plane_mat;
    a.boxes = r.boxes;
    a.box_mat = r.box_mat;
    a.pr = r.pr;
    a.vw = r.vw;
    a.tag = r.tag;
    a.uid = r.uid;
    a.q = nullptr;
    a.pr_out = r.pr_out;
    a.vw_out = r.vw_out;
    a.tag_out = r.tag_out;
    a.uid_out = r.uid_out;
    a.q_out = nullptr;
    a.key = r.key;
    a.rank = r.rank;
    a.cell_count = r.cell_count;
    a.err = r.err;
    a.nl_start = nullptr;
    a.nl_idx = nullptr;
    a.disp = nullptr;
    a.nl_flags = nullptr;
    a.half_skin = 0.f;
    a.hertz = 0;
    a.ext = nullptr;
    if (r.n > 0)
        k_dem_step<double, false, false><<<grid_for(r.n, kDemBlock), kDemBlock, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace peb
