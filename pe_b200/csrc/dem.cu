// dem.cu -- fused DEM step: neighbour search, contact law, force accumulation and integration
// in one kernel per step.
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
// Each thread owns one slot of the cell-sorted order and writes the integrated body to that
// slot of the other buffer, so the state is re-sorted by cell as a side effect; it also bins
// the integrated position for the next step's counting sort.
#include <math_constants.h>

#include "internal.cuh"

namespace peb {

namespace {

constexpr int kDemBlock = 128;

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
template <typename T>
__device__ __forceinline__ void dem_contact(V3<T> n, T dist, V3<T> r1, V3<T> r2, V3<T> v1,
                                            V3<T> w1, V3<T> v2, V3<T> w2, const MatDev &m1,
                                            const MatDev &m2, bool self_is_1, Acc<T> &acc) {
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
    T fNabs = k * delta + cn * relVelN;
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
    const int32_t *sorted;
    const int32_t *cell_start;
    const SceneInfo *scenes;
    const MatDev *mats;
    const double4 *planes;
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
};

template <typename VT, bool TRACKQ>
__global__ void __launch_bounds__(kDemBlock) k_dem_step(DemArgs<VT> a) {
    using T = VT;  // arithmetic type of the contact law (double or float)
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    const int32_t b = a.sorted[t];
    const double4 pi = a.pr[b];
    const uint32_t tagi = a.tag[b];
    const int32_t uidi = a.uid[b];
    const SceneInfo &s = a.scenes[tagi >> 16];
    const MatDev mi = a.mats[tagi & 0xffffu];
    const V3<T> vi = ld_vw(a.vw, b, 0), wi = ld_vw(a.vw, b, 1);
    Acc<T> acc;
    acc.F = v3(T(0), T(0), T(0));
    acc.T_ = acc.F;

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
                const int32_t j = a.sorted[slot];
                if (j == b) continue;
                const double4 pj = a.pr[j];
                const double ddx = pi.x - pj.x, ddy = pi.y - pj.y, ddz = pi.z - pj.z;
                const double rs = pi.w + pj.w;
                // only penetrating contacts (dist < -contactThreshold) produce a force
                // (ContactBase.h:307-310); this bound is conservative for them
                if (ddx * ddx + ddy * ddy + ddz * ddz >= rs * rs) continue;
                const int32_t uidj = a.uid[j];
                const bool self1 = uidi < uidj;
                // pe orientation: body 1 = smaller system id (MaxContacts.h:550-551)
                const double4 p1 = self1 ? pi : pj;
                const double4 p2 = self1 ? pj : pi;
                const double nx = p1.x - p2.x, ny = p1.y - p2.y, nz = p1.z - p2.z;
                const double len = length_rn(nx, ny, nz);
                const double dist = __dsub_rn(__dsub_rn(len, p1.w), p2.w);
                if (!(dist < -kContactThreshold)) continue;
                const MatDev mj = a.mats[a.tag[j] & 0xffffu];
                const V3<T> vj = ld_vw(a.vw, j, 0), wj = ld_vw(a.vw, j, 1);
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
                if (self1)
                    dem_contact<T>(n, T(dist), r1, r2, vi, wi, vj, wj, mi, mj, true, acc);
                else
                    dem_contact<T>(n, T(dist), r1, r2, vj, wj, vi, wi, mj, mi, false, acc);
            }
        }
    }
    // walls: planes (MaxContacts.h:777-790), then boxes (MaxContacts.h:589-668); the sphere is
    // body 1 and the fixed wall has zero velocity
    const V3<T> zero = v3(T(0), T(0), T(0));
    for (int p = 0; p < s.nplanes; ++p) {
        const double4 pl = a.planes[s.plane_begin + p];
        const double kk = dot_rn(pl.x, pl.y, pl.z, pi.x, pi.y, pi.z);
        const double dist = __dsub_rn(__dsub_rn(kk, pi.w), pl.w);
        if (!(dist < -kContactThreshold)) continue;
        const MatDev mw = a.mats[a.plane_mat[s.plane_begin + p]];
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
        const double l[3] = {0.5 * B[3], 0.5 * B[4], 0.5 * B[5]};
        const double *R = B + 6;
        const double dx = pi.x - B[0], dy = pi.y - B[1], dz = pi.z - B[2];
        double p[3] = {dx * R[0] + dy * R[3] + dz * R[6], dx * R[1] + dy * R[4] + dz * R[7],
                       dx * R[2] + dy * R[5] + dz * R[8]};
        bool outside = false;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            if (p[ax] < -l[ax]) { p[ax] = -l[ax]; outside = true; }
            else if (p[ax] > l[ax]) { p[ax] = l[ax]; outside = true; }
        }
        double nx, ny, nz, dist, gx, gy, gz;
        if (!outside) {
            dist = fabs(p[0]) - l[0];
            int face = 0;
            for (int ax = 1; ax < 3; ++ax) {
                const double tmp = fabs(p[ax]) - l[ax];
                if (dist < tmp) { dist = tmp; face = ax; }
            }
            const double sg = (p[face] > 0.0) ? 1.0 : -1.0;
            nx = R[face] * sg; ny = R[3 + face] * sg; nz = R[6 + face] * sg;
            dist -= pi.w;
            gx = pi.x; gy = pi.y; gz = pi.z;
        } else {
            const double qx = R[0] * p[0] + R[1] * p[1] + R[2] * p[2];
            const double qy = R[3] * p[0] + R[4] * p[1] + R[5] * p[2];
            const double qz = R[6] * p[0] + R[7] * p[1] + R[8] * p[2];
            const double mx = dx - qx, my = dy - qy, mz = dz - qz;
            const double len = length_rn(mx, my, mz);
            dist = len - pi.w;
            const double il = 1.0 / len;
            nx = mx * il; ny = my * il; nz = mz * il;
            gx = B[0] + qx; gy = B[1] + qy; gz = B[2] + qz;
        }
        if (!(dist < -kContactThreshold)) continue;
        const MatDev mw = a.mats[a.box_mat[s.box_begin + k]];
        const V3<T> n = v3(T(nx), T(ny), T(nz));
        const V3<T> r1 = v3(T(gx - pi.x), T(gy - pi.y), T(gz - pi.z));
        dem_contact<T>(n, T(dist), r1, zero, vi, wi, zero, zero, mi, mw, true, acc);
    }

    // SphereTrait::move, Default.h:166-216
    double im, ii, I;
    sphere_mass(pi.w, mi.density, im, ii, I);
    (void)I;
    const V3<T> gg = v3(T(a.g[0]), T(a.g[1]), T(a.g[2]));
    const V3<T> vdot = acc.F * T(im) + gg;
    const V3<T> wdot = T(ii) * acc.T_;
    V3<T> v = vi + vdot * T(a.dt);
    V3<T> w = wi + wdot * T(a.dt);
    const double nxp = pi.x + double(v.x) * a.dt;
    const double nyp = pi.y + double(v.y) * a.dt;
    const double nzp = pi.z + double(v.z) * a.dt;
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
    if (a.has_drag) {
        v = v * T(a.drag);
        w = w * T(a.drag);
    }
    a.pr_out[t] = make_double4(nxp, nyp, nzp, pi.w);
    VT *o = a.vw_out + 6 * t;
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = w.x; o[4] = w.y; o[5] = w.z;
    a.tag_out[t] = tagi;
    a.uid_out[t] = uidi;
    if (!isfinite(nxp) || !isfinite(nyp) || !isfinite(nzp)) atomicOr(a.err, DERR_NAN);
    // bin for the next step's counting sort
    int ncx, ncy, ncz;
    cell_coords(s, nxp, nyp, nzp, ncx, ncy, ncz);
    const int32_t kk = (int32_t)cell_key(s, ncx, ncy, ncz);
    a.key[t] = kk;
    a.rank[t] = atomicAdd(&a.cell_count[kk], 1);
}

template <typename VT>
int launch_dem(Ctx *c, double dt) {
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
    prof_begin(c, ST_DEM);
    if (c->p.track_orientation)
        k_dem_step<VT, true><<<grid_for(c->n, kDemBlock), kDemBlock, 0, c->stream>>>(a);
    else
        k_dem_step<VT, false><<<grid_for(c->n, kDemBlock), kDemBlock, 0, c->stream>>>(a);
    PEB_LAUNCHED(c);
    prof_end(c, ST_DEM);
    return PE_B200_OK;
}

}  // namespace

int dem_step(Ctx *c, double dt) {
    if (!c->binned) {
        int rc = grid_bin_current(c);
        if (rc) return rc;
    }
    int rc = grid_sort(c);
    if (rc) return rc;
    if (c->n > 0) {
        rc = (c->p.precision == PE_B200_FP64) ? launch_dem<double>(c, dt) : launch_dem<float>(c, dt);
        if (rc) return rc;
        std::swap(c->cur, c->nxt);
    }
    return PE_B200_OK;
}

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
    if (r.n > 0)
        k_dem_step<double, false><<<grid_for(r.n, kDemBlock), kDemBlock, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace peb
