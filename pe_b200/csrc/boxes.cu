// boxes.cu -- moving (non-fixed) boxes: pe's box fine detection, the linear DEM law on box
// contacts, BoxTrait::move, and the box side of the hard-contact step.
//
// Fine detection (pe/core/detection/fine/MaxContacts.h):
//   sphere/box  :589-668   one contact, normal from the box to the sphere
//   box/box     :867-2250  separating-axis test over 15 axes; the deepest face axis gives the
//                          vertex/face contacts of the incident face clipped against the
//                          reference face, the deepest edge/edge axis one edge/edge contact
//   box/plane   :2380-2528 every corner below the plane
// Bounding boxes are tested first as HashGrids::collide does (HashGrids.h:1351-1358).
//
// This file is compiled without fused multiply-adds (build.py): the separating-axis test picks
// the contact case by comparing depths that tie for aligned boxes (stacks), and pe's choice is
// reproduced only when every product and sum rounds as in pe's FP64 code.
//
// Work layout.  Each step first computes every box's rotation and bounding box and sorts the
// boxes into a small uniform grid (one block; cells wide enough that bodies whose bounding
// boxes overlap a box's sit in a neighbouring cell of the box's centre cell).  Each box is one
// thread block that walks its candidates with its threads: the spheres in the cells of the
// spheres' own grid that its bounding box covers, the scene's planes and fixed boxes, and the
// moving boxes of the neighbouring box-grid cells.  The DEM force of the boxes on a sphere is
// gathered by one warp per sphere over the neighbouring box-grid cells, for the spheres whose
// cell has a box nearby.  Every thread or lane visits a fixed subset in a fixed order and sums
// reduce in fixed trees, so results do not depend on scheduling.
//
// Contact ids inside this file: spheres 0..n-1 (index in the current buffers), moving box m
// n + m, walls -(1 + global wall index) (planes first, then fixed boxes).
#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.cuh"

namespace peb {

namespace {

constexpr int kBoxBlk = 128;
constexpr int kRowBatch = 256;       // rows of sphere-grid cells a box block stages at a time
constexpr int kGridBlk = 1024;
constexpr int kMaxBoxCells = 1 << 16;
using V = V3<double>;

struct BoxArgs {
    int64_t n;          // spheres
    int32_t m;          // moving boxes
    const double4 *pr;
    const double *vw;   // FP64 velocities, component-major
    const uint32_t *tag;
    const int32_t *uid;
    const SceneInfo *scenes;
    const MatDev *mats;
    const double4 *planes;
    const int32_t *plane_mat;
    int32_t total_planes;
    const double *boxes;
    const int32_t *box_mat;
    const double *bx, *bq, *bv, *bw, *blen, *bprops;
    const int32_t *bmat, *bscene;
    // the spheres' cell grid of the current step (slot -> body through sorted, or identity)
    const int32_t *cell_start;
    const int32_t *sorted;
    // per-box rotation (9) and bounding box (6) of this step, and the box grid (k_box_grid)
    const double *bR, *bbb;
    const double *gparm;     // lo xyz, 1/h, then the three dims as doubles
    const int32_t *gstart;   // cell -> first entry in gids
    const int32_t *gids;     // boxes by cell, ascending index within a cell
    const int32_t *gcell;    // box -> its cell
    const uint32_t *gnear;   // bit per cell: a box in this cell or a neighbouring one
};

// an oriented box as the fine detection sees it
struct OBox {
    V x;
    double R[9];
    double len[3], hl[3];
    int64_t key;    // pe's system-id order (fixed boxes before moving boxes)
    int32_t ref;    // contact id
};

__device__ __forceinline__ V ld3(const double *p) { return v3(p[0], p[1], p[2]); }

// Quaternion.h:591-602 (toRotationMatrix)
__device__ __forceinline__ void quat_to_rot(const double *q, double *R) {
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

// R^T v and R v for row-major R (RotationMatrix.h:1318-1324 with trans())
__device__ __forceinline__ V rt_mulv(const double *R, V v) {
    return v3(R[0] * v.x + R[3] * v.y + R[6] * v.z, R[1] * v.x + R[4] * v.y + R[7] * v.z,
              R[2] * v.x + R[5] * v.y + R[8] * v.z);
}
__device__ __forceinline__ V r_mulv(const double *R, V v) {
    return v3(R[0] * v.x + R[1] * v.y + R[2] * v.z, R[3] * v.x + R[4] * v.y + R[5] * v.z,
              R[6] * v.x + R[7] * v.y + R[8] * v.z);
}
__device__ __forceinline__ double comp(V a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

__device__ OBox moving_box(const BoxArgs &a, int32_t m) {
    OBox b;
    b.x = ld3(a.bx + 3 * m);
    for (int k = 0; k < 9; ++k) b.R[k] = a.bR[9 * m + k];
    for (int k = 0; k < 3; ++k) {
        b.len[k] = a.blen[3 * m + k];
        b.hl[k] = 0.5 * b.len[k];
    }
    b.key = (int64_t(1) << 40) + m;
    b.ref = (int32_t)(a.n + m);
    return b;
}

__device__ OBox fixed_box(const BoxArgs &a, int32_t gk) {
    const double *B = a.boxes + 15 * (int64_t)gk;
    OBox b;
    b.x = ld3(B);
    for (int k = 0; k < 9; ++k) b.R[k] = B[6 + k];
    for (int k = 0; k < 3; ++k) {
        b.len[k] = B[3 + k];
        b.hl[k] = 0.5 * B[3 + k];
    }
    b.key = gk;
    b.ref = -(1 + a.total_planes + gk);
    return b;
}

// BoxBase.cpp:100-115 (calcBoundingBox): lo[0..2], hi[3..5]
__device__ void box_aabb(const OBox &b, double *bb) {
    const double *R = b.R, *L = b.len;
    const double e0 = 0.5 * (fabs(R[0] * L[0]) + fabs(R[1] * L[1]) + fabs(R[2] * L[2])) + kContactThreshold;
    const double e1 = 0.5 * (fabs(R[3] * L[0]) + fabs(R[4] * L[1]) + fabs(R[5] * L[2])) + kContactThreshold;
    const double e2 = 0.5 * (fabs(R[6] * L[0]) + fabs(R[7] * L[1]) + fabs(R[8] * L[2])) + kContactThreshold;
    bb[0] = b.x.x - e0; bb[1] = b.x.y - e1; bb[2] = b.x.z - e2;
    bb[3] = b.x.x + e0; bb[4] = b.x.y + e1; bb[5] = b.x.z + e2;
}

// BoundingBox.h:487-497
__device__ __forceinline__ bool aabb_overlap(const double *a, const double *b) {
    return !(b[0] > a[3] || b[1] > a[4] || b[2] > a[5] || b[3] < a[0] || b[4] < a[1] ||
             b[5] < a[2]);
}

// Contact sinks are called as f(b1, b2, gpos, normal, dist, kind): pe's body order (normal
// from body 2 to body 1); kind 1 marks an edge/edge contact.

// MaxContacts.h:589-668 (sphere s with centre p.xyz and radius p.w against box b)
template <typename F>
__device__ void collide_sphere_box(int32_t sref, const double4 &p, const OBox &b, F &f) {
    const double *R = b.R;
    const double l3[3] = {b.hl[0], b.hl[1], b.hl[2]};
    const V d = v3(p.x, p.y, p.z) - b.x;
    double q[3] = {d.x * R[0] + d.y * R[3] + d.z * R[6], d.x * R[1] + d.y * R[4] + d.z * R[7],
                   d.x * R[2] + d.y * R[5] + d.z * R[8]};
    bool outside = false;
    for (int k = 0; k < 3; ++k) {
        if (q[k] < -l3[k]) { q[k] = -l3[k]; outside = true; }
        else if (q[k] > l3[k]) { q[k] = l3[k]; outside = true; }
    }
    if (!outside) {
        double dist = fabs(q[0]) - l3[0];
        int face = 0;
        for (int k = 1; k < 3; ++k) {
            const double tmp = fabs(q[k]) - l3[k];
            if (dist < tmp) { dist = tmp; face = k; }
        }
        double nl[3] = {0.0, 0.0, 0.0};
        nl[face] = (q[face] > 0.0) ? 1.0 : -1.0;
        const V n = r_mulv(R, v3(nl[0], nl[1], nl[2]));
        dist -= p.w;
        f(sref, b.ref, v3(p.x, p.y, p.z), n, dist, 0);
        return;
    }
    const V qw = r_mulv(R, v3(q[0], q[1], q[2]));
    const V n = d - qw;
    const double dist = length(n) - p.w;
    if (dist < kContactThreshold) f(sref, b.ref, b.x + qw, normalized(n), dist, 0);
}

// MaxContacts.h:2380-2528: the corners in pe's order (lower face, then upper face)
template <typename F>
__device__ void collide_box_plane(const OBox &b, const double4 &pl, int32_t pref, F &f) {
    const V pn = v3(pl.x, pl.y, pl.z);
    const double *R = b.R;
    const double range[3] = {0.5 * b.len[0], 0.5 * b.len[1], 0.5 * b.len[2]};
    const V nr = rt_mulv(R, pn);
    const double nrel[3] = {nr.x, nr.y, nr.z};
    double mn = range[0];
    if (range[1] < mn) mn = range[1];
    if (range[2] < mn) mn = range[2];
    const double minlength = -0.99 * mn;
    const int sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
    const int sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    const int sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    for (int k = 0; k < 8; ++k) {
        const double a0 = sx[k] > 0 ? range[0] * nrel[0] : -(range[0] * nrel[0]);
        const double a1 = sy[k] > 0 ? range[1] * nrel[1] : -(range[1] * nrel[1]);
        const double a2 = sz[k] > 0 ? range[2] * nrel[2] : -(range[2] * nrel[2]);
        if (!((a0 + a1) + a2 < minlength)) continue;
        const V corner = v3(sx[k] * range[0], sy[k] * range[1], sz[k] * range[2]);
        const V pos = b.x + r_mulv(R, corner);
        const double kk = pos.x * pn.x + pos.y * pn.y + pos.z * pn.z;
        const double dist = kk - pl.w;
        if (dist < kContactThreshold) f(b.ref, pref, pos, pn, dist, 0);
    }
}

// GeomTools.cpp:387-408
__device__ void intersect_lines(V o1, V d1, V o2, V d2, double &s, double &t) {
    const V c = cross(d1, d2);
    const double sqrlen = c.x * c.x + c.y * c.y + c.z * c.z;
    if (sqrlen < 1e-8) {   // parallelThreshold, Thresholds.h:170
        s = 0.0;
        t = 0.0;
        return;
    }
    const double isqrlen = 1.0 / sqrlen;
    const V p = o2 - o1;
    const double dd = dot(d1, d2);
    const double a = dot(d1, p);
    const double b = dot(-d2, p);
    s = (a * dot(d2, d2) + dd * b) * isqrlen;
    t = (b * dot(d1, d1) + dd * a) * isqrlen;
}

// component i of (a, b, c) and the vector with component ix = vx, iy = vy and the remaining
// one vz, both by selects: runtime axis indices then need no indexed local arrays
__device__ __forceinline__ double sel3(int i, double a, double b, double c) {
    return i == 0 ? a : (i == 1 ? b : c);
}
__device__ __forceinline__ double sel3(int i, V v) { return sel3(i, v.x, v.y, v.z); }
__device__ __forceinline__ V perm3(int ix, double vx, int iy, double vy, double vz) {
    return v3(ix == 0 ? vx : (iy == 0 ? vy : vz), ix == 1 ? vx : (iy == 1 ? vy : vz),
              ix == 2 ? vx : (iy == 2 ? vy : vz));
}

// MaxContacts.h:867-2250
template <typename F>
__device__ void collide_box_box(const OBox &p1, const OBox &p2, F &f) {
    const bool swp = p2.key < p1.key;
    const OBox b1 = swp ? p2 : p1;
    const OBox b2 = swp ? p1 : p2;
    double maxDepth = -1.79769313486231570815e308;
    bool invertNormal = false;
    int contactCase = 0;
    V contactNormal = v3(0.0, 0.0, 0.0), normal_c = contactNormal;
    const double *R1 = b1.R, *R2 = b2.R;
    double rR[9], rQ[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            rR[3 * i + j] = R1[i] * R2[j] + R1[3 + i] * R2[3 + j] + R1[6 + i] * R2[6 + j];
#pragma unroll
    for (int k = 0; k < 9; ++k) rQ[k] = fabs(rR[k]);
    const V rp = rt_mulv(R1, b2.x - b1.x);
    const double rPos[3] = {rp.x, rp.y, rp.z};
    const double *hl1 = b1.hl, *hl2 = b2.hl;
    // the face axes of box 1 (MaxContacts.h:905-970)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const double term1 = fabs(rPos[i]) - (hl1[i] + hl2[0] * rQ[3 * i] + hl2[1] * rQ[3 * i + 1] +
                                               hl2[2] * rQ[3 * i + 2]);
        if (term1 > kContactThreshold) return;
        if (i == 0 || term1 > maxDepth) {
            maxDepth = term1;
            contactNormal = v3(R1[i], R1[3 + i], R1[6 + i]);
            contactCase = 1 + i;
            invertNormal = rPos[i] < 0.0;
        }
    }
    // the face axes of box 2
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const double term1 = rPos[0] * rR[j] + rPos[1] * rR[3 + j] + rPos[2] * rR[6 + j];
        const double term2 =
            fabs(term1) - (hl1[0] * rQ[j] + hl1[1] * rQ[3 + j] + hl1[2] * rQ[6 + j] + hl2[j]);
        if (term2 > kContactThreshold) return;
        if (term2 > maxDepth) {
            maxDepth = term2;
            contactNormal = v3(R2[j], R2[3 + j], R2[6 + j]);
            contactCase = 4 + j;
            invertNormal = term1 < 0.0;
        }
    }
    // the nine edge/edge axes in pe's order (au x bu, au x bv, ..., aw x bw): term1 =
    // rPos[p0]*rR[p1] - rPos[p2]*rR[p3], term2 = hl1[h0]*rQ[q0] + hl1[h1]*rQ[q1], term3 =
    // hl2[h2]*rQ[q2] + hl2[h3]*rQ[q3], axis length from rR[s0], rR[s1], zero axis component
    constexpr int8_t E[9][15] = {
        {2, 3, 1, 6, 1, 6, 2, 3, 2, 1, 1, 2, 6, 3, 0}, {2, 4, 1, 7, 1, 7, 2, 4, 0, 2, 2, 0, 7, 4, 0},
        {2, 5, 1, 8, 1, 8, 2, 5, 1, 0, 0, 1, 8, 5, 0}, {0, 6, 2, 0, 2, 0, 0, 6, 2, 4, 1, 5, 6, 0, 1},
        {0, 7, 2, 1, 2, 1, 0, 7, 0, 5, 2, 3, 7, 1, 1}, {0, 8, 2, 2, 2, 2, 0, 8, 1, 3, 0, 4, 8, 2, 1},
        {1, 0, 0, 3, 0, 3, 1, 0, 2, 7, 1, 8, 3, 0, 2}, {1, 1, 0, 4, 0, 4, 1, 1, 0, 8, 2, 6, 4, 1, 2},
        {1, 2, 0, 5, 0, 5, 1, 2, 1, 6, 0, 7, 5, 2, 2}};
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        const int8_t *c = E[e];
        const double term1 = rPos[c[0]] * rR[c[1]] - rPos[c[2]] * rR[c[3]];
        const double term2 = hl1[c[4]] * rQ[c[5]] + hl1[c[6]] * rQ[c[7]];
        const double term3 = hl2[c[8]] * rQ[c[9]] + hl2[c[10]] * rQ[c[11]];
        double sum = fabs(term1) - (term2 + term3);
        if (fabs(term1) > term2 + term3 + kContactThreshold) return;
        const double a = rR[c[12]], b = rR[c[13]];
        const double length = sqrt(a * a + b * b);
        if (length > 2.2204460492503131e-16) {   // epsilon (Limits.h:381)
            sum /= length;
            if (sum > maxDepth && fabs(sum - maxDepth) > 1e-8) {   // accuracy (Limits.h:385)
                maxDepth = sum;
                if (c[14] == 0) normal_c = v3(0.0, -a / length, b / length);
                else if (c[14] == 1) normal_c = v3(a / length, 0.0, -b / length);
                else normal_c = v3(-a / length, b / length, 0.0);
                contactCase = 7 + e;
                invertNormal = term1 < 0.0;
            }
        }
    }
    if (contactCase == 0) return;
    if (contactCase > 6) contactNormal = r_mulv(R1, normal_c);
    if (invertNormal) contactNormal = -contactNormal;

    if (contactCase > 6) {   // edge/edge, MaxContacts.h:1343-1417
        V sg = rt_mulv(R1, contactNormal);
        V sv = v3(sg.x > 0.0 ? hl1[0] : -hl1[0], sg.y > 0.0 ? hl1[1] : -hl1[1],
                  sg.z > 0.0 ? hl1[2] : -hl1[2]);
        V pB1 = b1.x + r_mulv(R1, sv);
        sg = rt_mulv(R2, contactNormal);
        sv = v3(sg.x > 0.0 ? -hl2[0] : hl2[0], sg.y > 0.0 ? -hl2[1] : hl2[1],
                sg.z > 0.0 ? -hl2[2] : hl2[2]);
        V pB2 = b2.x + r_mulv(R2, sv);
        const int ia = (contactCase - 7) / 3, ib = (contactCase - 7) % 3;
        const V ua = v3(sel3(ia, R1[0], R1[1], R1[2]), sel3(ia, R1[3], R1[4], R1[5]),
                        sel3(ia, R1[6], R1[7], R1[8]));
        const V ub = v3(sel3(ib, R2[0], R2[1], R2[2]), sel3(ib, R2[3], R2[4], R2[5]),
                        sel3(ib, R2[6], R2[7], R2[8]));
        double s, t;
        intersect_lines(pB1, ua, pB2, ub, s, t);
        pB1 = pB1 + s * ua;
        pB2 = pB2 + t * ub;
        const V gpos = 0.5 * (pB1 + pB2);
        f(b2.ref, b1.ref, gpos, contactNormal, maxDepth, 1);
        return;
    }

    // vertex/face, MaxContacts.h:1419-2250: A owns the reference face.  Points of A's frame are
    // kept with their components in the order (xa, ya, za): the reference face's normal axis
    // first, so the clipping below reads fixed components.
    const bool sw = contactCase > 3;
    const OBox A = sw ? b2 : b1;
    const OBox B = sw ? b1 : b2;
    if (sw) contactNormal = -contactNormal;
    const double *Ra = A.R, *Rb = B.R;
    const V na = rt_mulv(Ra, contactNormal), nb = rt_mulv(Rb, contactNormal);
    int xb, yb, zb;
    if (fabs(nb.x) > fabs(nb.y)) {
        if (fabs(nb.x) > fabs(nb.z)) { xb = 0; yb = 1; zb = 2; }
        else { xb = 2; yb = 0; zb = 1; }
    } else if (fabs(nb.y) > fabs(nb.z)) { xb = 1; yb = 2; zb = 0; }
    else { xb = 2; yb = 0; zb = 1; }
    const int xa = contactCase < 4 ? contactCase - 1 : contactCase - 4;
    const int ya = xa == 0 ? 1 : (xa == 1 ? 2 : 0);
    const int za = xa == 0 ? 2 : (xa == 1 ? 0 : 1);
    const double hxa = sel3(xa, A.hl[0], A.hl[1], A.hl[2]), hya = sel3(ya, A.hl[0], A.hl[1], A.hl[2]),
                 hza = sel3(za, A.hl[0], A.hl[1], A.hl[2]);
    const double hxb = sel3(xb, B.hl[0], B.hl[1], B.hl[2]), hyb = sel3(yb, B.hl[0], B.hl[1], B.hl[2]),
                 hzb = sel3(zb, B.hl[0], B.hl[1], B.hl[2]);
    const double nax = sel3(xa, na), nbx = sel3(xb, nb);
    // the incident face of B in A's frame: T in A's axes, P the same with (xa, ya, za) order
    V T[4], P[4];
    const V ab = B.x - A.x;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const V vb = perm3(xb, nbx > 0.0 ? -hxb : hxb, yb, (k & 1) ? hyb : -hyb,
                           (k & 2) ? hzb : -hzb);
        T[k] = rt_mulv(Ra, ab + r_mulv(Rb, vb));
        P[k] = v3(sel3(xa, T[k]), sel3(ya, T[k]), sel3(za, T[k]));
    }
    const double offseta = nax > 0.0 ? hxa : -hxa;
    // the incident face's edges v0-v1, v0-v2, v3-v1, v3-v2 against the reference face's side
    // lines y = +h, y = -h, z = +h, z = -h (MaxContacts.h:1546-2065)
    constexpr int EP[4] = {0, 0, 3, 3}, EQ[4] = {1, 2, 1, 2};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const V Pe = P[EP[e]], Qe = P[EQ[e]];
#pragma unroll
        for (int side = 0; side < 4; ++side) {
            const bool ys = side < 2;   // the side lines y = +-h, else z = +-h
            const double hc = ys ? hya : hza, ho = ys ? hza : hya;
            const double h = (side & 1) ? -hc : hc;
            const double pc = ys ? Pe.y : Pe.z, qc = ys ? Qe.y : Qe.z;
            if (!((pc > h) ^ (qc > h))) continue;
            const double s = (h - pc) / (qc - pc);
            if (!(s > 0.0 && s < 1.0)) continue;
            const double po = ys ? Pe.z : Pe.y, qo = ys ? Qe.z : Qe.y;
            const double tmp = po + s * (qo - po);
            if (!(fabs(tmp) < ho)) continue;
            const double dist = fabs(Pe.x + s * (Qe.x - Pe.x)) - hxa;
            if (!(dist < kContactThreshold)) continue;
            const V posa = perm3(xa, offseta, ya, ys ? h : tmp, ys ? tmp : h);
            f(B.ref, A.ref, A.x + r_mulv(Ra, posa), contactNormal, dist, 0);
        }
    }
    // vertices of B inside the reference face (MaxContacts.h:2067-2118)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (fabs(P[k].y) <= hya && fabs(P[k].z) <= hza) {
            const double dist = fabs(P[k].x) - hxa;
            if (dist < kContactThreshold)
                f(B.ref, A.ref, A.x + r_mulv(Ra, T[k]), contactNormal, dist, 0);
        }
    }
    // vertices of A's reference face inside B's incident face, a vertex on B's vertex counted
    // once (MaxContacts.h:2179-2250)
    const V ba = A.x - B.x;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const V va = perm3(xa, offseta, ya, (k & 1) ? hya : -hya, (k & 2) ? hza : -hza);
        const V t = rt_mulv(Rb, ba + r_mulv(Ra, va));
        const double ay = fabs(sel3(yb, t)), az = fabs(sel3(zb, t));
        if ((ay <= hyb && az < hzb) || (ay < hyb && az <= hzb)) {
            const double dist = fabs(sel3(xb, t)) - hxb;
            if (dist < kContactThreshold) f(B.ref, A.ref, B.x + r_mulv(Rb, t), contactNormal, dist, 0);
        }
    }
}

// the box grid cell of a point, clamped
__device__ __forceinline__ void box_cell(const double *gp, double x, double y, double z, int &cx,
                                         int &cy, int &cz) {
    cx = clampi((int)floor((x - gp[0]) * gp[3]), 0, (int)gp[4] - 1);
    cy = clampi((int)floor((y - gp[1]) * gp[3]), 0, (int)gp[5] - 1);
    cz = clampi((int)floor((z - gp[2]) * gp[3]), 0, (int)gp[6] - 1);
}

// Every contact of moving box m, visited by thread tid of the nthr threads of a block (all of
// them call it): the spheres in the cells of the spheres' grid that the box's bounding box,
// grown by the largest radius, covers; the scene's planes and fixed boxes; and (all_pairs:
// every other / else: the later) moving boxes of the scene in the neighbouring box-grid cells.
template <typename F>
__device__ void visit_box(const BoxArgs &a, int32_t m, int tid, int nthr, bool all_pairs, F &f) {
    const OBox B = moving_box(a, m);
    const double *bb = a.bbb + 6 * m;
    const int32_t sc = a.bscene[m];
    const SceneInfo &s = a.scenes[sc];
    if (a.n > 0 && a.cell_start) {
        // the covered cells come as rows along x (contiguous slots); the rows of a batch are
        // laid end to end so that the threads share the spheres evenly
        __shared__ int32_t rbeg[kRowBatch], rcnt[kRowBatch];
        const double reach = s.rmax + kContactThreshold;
        int x0, y0, z0, x1, y1, z1;
        cell_coords(s, bb[0] - reach, bb[1] - reach, bb[2] - reach, x0, y0, z0);
        cell_coords(s, bb[3] + reach, bb[4] + reach, bb[5] + reach, x1, y1, z1);
        const int ny = y1 - y0 + 1, nrows = ny * (z1 - z0 + 1);
        for (int r0 = 0; r0 < nrows; r0 += kRowBatch) {
            const int nr = min(kRowBatch, nrows - r0);
            __syncthreads();
            for (int r = tid; r < nr; r += nthr) {
                const int y = y0 + (r0 + r) % ny, z = z0 + (r0 + r) / ny;
                const int64_t c0 = cell_key(s, x0, y, z), c1 = cell_key(s, x1, y, z) + 1;
                rbeg[r] = a.cell_start[c0];
                rcnt[r] = a.cell_start[c1] - rbeg[r];
            }
            __syncthreads();
            if (tid == 0)
                for (int r = 1; r < nr; ++r) rcnt[r] += rcnt[r - 1];   // inclusive prefix
            __syncthreads();
            const int total = rcnt[nr - 1];
            for (int k = tid; k < total; k += nthr) {
                int lo = 0, hi = nr - 1;   // the first row whose prefix exceeds k
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (rcnt[mid] > k) hi = mid;
                    else lo = mid + 1;
                }
                const int slot = rbeg[lo] + k - (lo > 0 ? rcnt[lo - 1] : 0);
                const int32_t i = a.sorted ? a.sorted[slot] : slot;
                const double4 p = a.pr[i];
                const double r = p.w + kContactThreshold;   // SphereBase.h:208-218
                const double sb[6] = {p.x - r, p.y - r, p.z - r, p.x + r, p.y + r, p.z + r};
                if (aabb_overlap(sb, bb)) collide_sphere_box(i, p, B, f);
            }
        }
    }
    for (int p = tid; p < s.nplanes; p += nthr)
        collide_box_plane(B, a.planes[s.plane_begin + p], -(1 + s.plane_begin + p), f);
    for (int k = tid; k < s.nboxes; k += nthr) {
        const OBox W = fixed_box(a, s.box_begin + k);
        double wb[6];
        box_aabb(W, wb);
        if (aabb_overlap(bb, wb)) collide_box_box(B, W, f);
    }
    // the 27 neighbouring box-grid cells (z, then y, then x) staged at once; candidate g of
    // their concatenation goes to thread g mod nthr
    __shared__ int32_t nb_beg[27], nb_pre[27];
    __syncthreads();
    if (tid < 27) {
        const double *gp = a.gparm;
        const int gx = (int)gp[4], gy = (int)gp[5], gz = (int)gp[6];
        const int32_t cm = a.gcell[m];
        const int x = cm % gx + tid % 3 - 1, y = (cm / gx) % gy + (tid / 3) % 3 - 1,
                  z = cm / (gx * gy) + tid / 9 - 1;
        int32_t b0 = 0, cnt = 0;
        if (x >= 0 && y >= 0 && z >= 0 && x < gx && y < gy && z < gz) {
            const int32_t c = (z * gy + y) * gx + x;
            b0 = a.gstart[c];
            cnt = a.gstart[c + 1] - b0;
        }
        nb_beg[tid] = b0;
        nb_pre[tid] = cnt;
    }
    __syncthreads();
    if (tid == 0)
        for (int i = 1; i < 27; ++i) nb_pre[i] += nb_pre[i - 1];   // inclusive prefix
    __syncthreads();
    const int total = nb_pre[26];
    for (int g = tid; g < total; g += nthr) {
        int i = 0;
        while (nb_pre[i] <= g) ++i;
        const int32_t j = a.gids[nb_beg[i] + g - (i > 0 ? nb_pre[i - 1] : 0)];
        if (j == m || (!all_pairs && j < m) || a.bscene[j] != sc) continue;
        if (!aabb_overlap(bb, a.bbb + 6 * j)) continue;
        collide_box_box(B, moving_box(a, j), f);
    }
}

// ---- body access by contact id ---------------------------------------------------------------
__device__ __forceinline__ int32_t body_mat(const BoxArgs &a, int32_t ref) {
    if (ref >= 0) return ref < a.n ? (int32_t)(a.tag[ref] & 0xffffu) : a.bmat[ref - a.n];
    const int32_t w = -ref - 1;
    return w < a.total_planes ? a.plane_mat[w] : a.box_mat[w - a.total_planes];
}
__device__ __forceinline__ V body_x(const BoxArgs &a, int32_t ref) {
    if (ref < a.n) {
        const double4 p = a.pr[ref];
        return v3(p.x, p.y, p.z);
    }
    return ld3(a.bx + 3 * (ref - a.n));
}
// RigidBody.h:1080-1085 (walls: zero)
__device__ __forceinline__ V vel_at(const BoxArgs &a, int32_t ref, V gpos) {
    if (ref < 0) return v3(0.0, 0.0, 0.0);
    V v, w;
    if (ref < a.n) {
        v = ld_vw(a.vw, a.n, ref, 0);
        w = ld_vw(a.vw, a.n, ref, 1);
    } else {
        v = ld3(a.bv + 3 * (ref - a.n));
        w = ld3(a.bw + 3 * (ref - a.n));
    }
    return v + cross(w, gpos - body_x(a, ref));
}

// response/DEMSolver.h:328-379, linear law, with Contact.cpp:72-115's composition; pe's
// edge/edge contacts keep zero stiffness and damping (Contact.cpp:131-175, ContactBase.h:
// 253-255), so they exert no force.  Returns false when the contact does not penetrate.
__device__ bool dem_force(const BoxArgs &a, int32_t b1, int32_t b2, V gpos, V n, double dist,
                          int kind, V &fN, V &fT) {
    if (!(dist < -kContactThreshold)) return false;   // ContactBase.h:307-310
    const V rvel = vel_at(a, b1, gpos) - vel_at(a, b2, gpos);
    const MatDev &m1 = a.mats[body_mat(a, b1)], &m2 = a.mats[body_mat(a, b2)];
    double k = 1.0 / (m1.rk + m2.rk), cn = 1.0 / (m1.rcn + m2.rcn), ct = 1.0 / (m1.rct + m2.rct);
    const double nvel = dot(n, rvel);
    const double tvel = dot(n, rvel - n * nvel);
    const double mu = (fabs(tvel) > kFrictionThreshold) ? m1.cdf + m2.cdf : m1.csf + m2.csf;
    if (kind == 1) k = cn = ct = 0.0;
    const double delta = -dist;
    const double relVelN = -dot(n, rvel);
    const V relVel = -rvel;
    const V relVelT = relVel - n * relVelN;
    double fNabs = k * delta + cn * relVelN;
    if (fNabs < 0.0) fNabs = 0.0;
    fN = fNabs * n;
    const double ft1 = ct * length(relVelT), ft2 = mu * fNabs;
    fT = (ft1 < ft2 ? ft1 : ft2) * normalized(relVelT);
    return true;
}

// ---- DEM ---------------------------------------------------------------------------------------
// spheres in a box-grid cell with a box nearby go to the list; the others get zero force
__global__ void k_sphere_box_near(BoxArgs a, double *ext, int32_t *list, int32_t *count) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= a.n) return;
    const double4 p = a.pr[b];
    const SceneInfo &s = a.scenes[a.tag[b] >> 16];
    const double *gp = a.gparm;
    // a sphere more than one cell outside the box grid touches no box (boxes' centres lie in
    // the grid and the cells are wider than any box plus a sphere)
    const double ux = floor((p.x - gp[0]) * gp[3]), uy = floor((p.y - gp[1]) * gp[3]),
                 uz = floor((p.z - gp[2]) * gp[3]);
    const bool inside = ux >= -1.0 && ux <= gp[4] && uy >= -1.0 && uy <= gp[5] && uz >= -1.0 &&
                        uz <= gp[6];
    int cx, cy, cz;
    box_cell(gp, p.x, p.y, p.z, cx, cy, cz);
    const int32_t own = (cz * (int)gp[5] + cy) * (int)gp[4] + cx;
    if (s.nmbox > 0 && inside && ((a.gnear[own >> 5] >> (own & 31)) & 1u)) {
        list[atomicAdd(count, 1)] = (int32_t)b;
    } else {
        double *e = ext + 6 * b;
        for (int k = 0; k < 6; ++k) e[k] = 0.0;
    }
}

// The boxes' forces on the listed spheres (each sphere is body 1 of its sphere/box contacts),
// one warp per sphere: lane l takes the candidates l, l + 32, ... of the neighbouring box-grid
// cells (cell by cell, ascending box index within a cell) and a fixed butterfly sums the lanes,
// so the result depends neither on scheduling nor on the list's order.
__global__ void k_sphere_box_forces(BoxArgs a, double *ext, const int32_t *list,
                                    const int32_t *count) {
    __shared__ int32_t nb_beg[8][32], nb_pre[8][32];   // per warp of the 256-thread block
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int32_t nl = *count;
    for (int64_t li = warp0; li < nl; li += nwarps) {
        __syncwarp();
        const int32_t b = list[li];
        const double4 p = a.pr[b];
        V F = v3(0.0, 0.0, 0.0), T = F;
        const V x = v3(p.x, p.y, p.z);
        const double r = p.w + kContactThreshold;
        const double sb[6] = {p.x - r, p.y - r, p.z - r, p.x + r, p.y + r, p.z + r};
        auto f = [&](int32_t b1, int32_t b2, V gpos, V n, double dist, int kind) {
            V fN, fT;
            if (!dem_force(a, b1, b2, gpos, n, dist, kind, fN, fT)) return;
            const V r1 = gpos - x;
            F = F + fN;
            T = T + cross(r1, fN);
            F = F + fT;
            T = T + cross(r1, fT);
        };
        const int32_t sc = (int32_t)(a.tag[b] >> 16);
        const double *gp = a.gparm;
        const int gx = (int)gp[4], gy = (int)gp[5], gz = (int)gp[6];
        int cx, cy, cz;
        box_cell(gp, p.x, p.y, p.z, cx, cy, cz);
        // lanes 0..26 load the 27 neighbouring cells (z, then y, then x); candidate g of their
        // concatenation goes to lane g mod 32
        int32_t b0 = 0, cnt = 0;
        if (lane < 27) {
            const int xx = cx + lane % 3 - 1, y = cy + (lane / 3) % 3 - 1, z = cz + lane / 9 - 1;
            if (xx >= 0 && y >= 0 && z >= 0 && xx < gx && y < gy && z < gz) {
                const int32_t c = (z * gy + y) * gx + xx;
                b0 = a.gstart[c];
                cnt = a.gstart[c + 1] - b0;
            }
        }
        int32_t pre = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t u = __shfl_up_sync(0xffffffffu, pre, o);
            if (lane >= o) pre += u;
        }
        nb_beg[wib][lane] = b0;
        nb_pre[wib][lane] = pre;
        __syncwarp();
        const int32_t total = nb_pre[wib][26];
        for (int g = lane; g < total; g += 32) {
            int i = 0;
            while (nb_pre[wib][i] <= g) ++i;
            const int32_t m = a.gids[nb_beg[wib][i] + g - (i > 0 ? nb_pre[wib][i - 1] : 0)];
            if (a.bscene[m] != sc || !aabb_overlap(sb, a.bbb + 6 * m)) continue;
            collide_sphere_box(b, p, moving_box(a, m), f);
        }
        double v[6] = {F.x, F.y, F.z, T.x, T.y, T.z};
        for (int o = 16; o > 0; o >>= 1)
            for (int q = 0; q < 6; ++q) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
        if (lane == 0) {
            double *e = ext + 6 * (int64_t)b;
            for (int q = 0; q < 6; ++q) e[q] = v[q];
        }
    }
}

__device__ void block_sum6(double *v, double (*sh)[6]) {
    const int t = threadIdx.x;
    for (int k = 0; k < 6; ++k) sh[t][k] = v[k];
    __syncthreads();
    for (int half = kBoxBlk / 2; half > 0; half >>= 1) {
        if (t < half)
            for (int k = 0; k < 6; ++k) sh[t][k] += sh[t + half][k];
        __syncthreads();
    }
    for (int k = 0; k < 6; ++k) v[k] = sh[0][k];
}

// Quaternion(phi, |phi|) * q (Quaternion.h:274-294, 1146-1153)
__device__ void quat_rotate(const double *q, V phi, double *out) {
    const double angle = sqrt(phi.x * phi.x + phi.y * phi.y + phi.z * phi.z);
    double d0 = 1.0, d1 = 0.0, d2 = 0.0, d3 = 0.0;
    if (!(fabs(angle) < 1e-15)) {
        const double sina = sin(angle * 0.5), cosa = cos(angle * 0.5);
        const V ax = normalized(phi);
        d0 = cosa; d1 = sina * ax.x; d2 = sina * ax.y; d3 = sina * ax.z;
    }
    out[0] = d0 * q[0] - d1 * q[1] - d2 * q[2] - d3 * q[3];
    out[1] = d0 * q[1] + d1 * q[0] + d2 * q[3] - d3 * q[2];
    out[2] = d0 * q[2] + d2 * q[0] + d3 * q[1] - d1 * q[3];
    out[3] = d0 * q[3] + d3 * q[0] + d1 * q[2] - d2 * q[1];
}

// new position and orientation of box m from velocities v, w; writes the next buffers
__device__ void box_advance(const BoxArgs &a, int32_t m, V v, V w, double dt, double drag,
                            int has_drag, double *xo, double *qo, double *vo, double *wo) {
    const V x = ld3(a.bx + 3 * m) + v * dt;
    double q[4];
    quat_rotate(a.bq + 4 * m, w * dt, q);
    if (has_drag) {
        v = v * drag;
        w = w * drag;
    }
    xo[3 * m] = x.x; xo[3 * m + 1] = x.y; xo[3 * m + 2] = x.z;
    for (int k = 0; k < 4; ++k) qo[4 * m + k] = q[k];
    vo[3 * m] = v.x; vo[3 * m + 1] = v.y; vo[3 * m + 2] = v.z;
    wo[3 * m] = w.x; wo[3 * m + 1] = w.y; wo[3 * m + 2] = w.z;
}

// one block per moving box: its contact forces, then BoxTrait::move (boxtrait/Default.h:149-220)
__global__ void __launch_bounds__(kBoxBlk) k_box_dem(BoxArgs a, double gx, double gy, double gz,
                                                     double dt, double drag, int has_drag,
                                                     double *xo, double *qo, double *vo,
                                                     double *wo, int32_t *err) {
    __shared__ double sh[kBoxBlk][6];
    const int32_t m = blockIdx.x;
    const V xb = ld3(a.bx + 3 * m);
    const int32_t self = (int32_t)(a.n + m);
    V F = v3(0.0, 0.0, 0.0), T = F;
    auto f = [&](int32_t b1, int32_t b2, V gpos, V n, double dist, int kind) {
        V fN, fT;
        if (!dem_force(a, b1, b2, gpos, n, dist, kind, fN, fT)) return;
        if (b2 == self) {
            fN = -fN;
            fT = -fT;
        }
        const V r = gpos - xb;
        F = F + fN;
        T = T + cross(r, fN);
        F = F + fT;
        T = T + cross(r, fT);
    };
    visit_box(a, m, threadIdx.x, blockDim.x, true, f);
    double acc[6] = {F.x, F.y, F.z, T.x, T.y, T.z};
    block_sum6(acc, sh);
    if (threadIdx.x != 0) return;
    F = v3(acc[0], acc[1], acc[2]);
    T = v3(acc[3], acc[4], acc[5]);
    const double *pp = a.bprops + 8 * m;
    double R[9];
    quat_to_rot(a.bq + 4 * m, R);
    const V vdot = F * pp[0] + v3(gx, gy, gz);
    const V t1 = rt_mulv(R, T);
    const V wdot = r_mulv(R, v3(pp[1] * t1.x, pp[2] * t1.y, pp[3] * t1.z));
    const V v = ld3(a.bv + 3 * m) + vdot * dt;
    const V w = ld3(a.bw + 3 * m) + wdot * dt;
    box_advance(a, m, v, w, dt, drag, has_drag, xo, qo, vo, wo);
    if (!isfinite(xo[3 * m]) || !isfinite(xo[3 * m + 1]) || !isfinite(xo[3 * m + 2]))
        atomicOr(err, DERR_NAN);
}

// ---- hard contacts -------------------------------------------------------------------------
// R D R^T for diagonal D, as ((R * D) * trans(R)) (RotationMatrix.h:1370-1429)
__device__ void rot_diag_rt(const double *R, const double *d, double *out) {
    double RD[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            RD[3 * i + j] = R[3 * i] * (j == 0 ? d[0] : 0.0) + R[3 * i + 1] * (j == 1 ? d[1] : 0.0) +
                            R[3 * i + 2] * (j == 2 ? d[2] : 0.0);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            out[3 * i + j] = RD[3 * i] * R[3 * j] + RD[3 * i + 1] * R[3 * j + 1] +
                             RD[3 * i + 2] * R[3 * j + 2];
}

// body cache of box m at slot n + m (HCSITS.h:1834-1880): v + g dt and
// w + dt I^-1 ((I w) x w) in the world frame, and the world-frame inverse inertia
__global__ void k_box_bodycache(BoxArgs a, BodyCacheD bc, double gx, double gy, double gz,
                                double dt) {
    const int32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= a.m) return;
    const double *pp = a.bprops + 8 * m;
    double R[9], Iinv[9], I[9];
    quat_to_rot(a.bq + 4 * m, R);
    rot_diag_rt(R, pp + 1, Iinv);
    rot_diag_rt(R, pp + 4, I);
    const V v = ld3(a.bv + 3 * m), w = ld3(a.bw + 3 * m);
    const V vp = v + v3(gx, gy, gz) * dt;
    const V Iw = v3(I[0] * w.x + I[1] * w.y + I[2] * w.z, I[3] * w.x + I[4] * w.y + I[5] * w.z,
                    I[6] * w.x + I[7] * w.y + I[8] * w.z);
    const V c = cross(Iw, w);
    const V g = v3(Iinv[0] * c.x + Iinv[1] * c.y + Iinv[2] * c.z,
                   Iinv[3] * c.x + Iinv[4] * c.y + Iinv[5] * c.z,
                   Iinv[6] * c.x + Iinv[7] * c.y + Iinv[8] * c.z);
    const V wp = w + dt * g;
    const int64_t t = a.n + m;
    bc.vr[t] = make_double4(vp.x, vp.y, vp.z, pp[0]);
    bc.wr[t] = make_double4(wp.x, wp.y, wp.z, 0.0);
    bc.dv[t] = make_double4(0.0, 0.0, 0.0, 0.0);
    bc.dw[t] = make_double4(0.0, 0.0, 0.0, 0.0);
    bc.ia[t] = make_double4(Iinv[0], Iinv[1], Iinv[2], 0.0);
    bc.ib[t] = make_double4(Iinv[3], Iinv[4], Iinv[5], 0.0);
    bc.ic[t] = make_double4(Iinv[6], Iinv[7], Iinv[8], 0.0);
}

// per-thread contact counts of box m, scanned across the block; *total (thread 0) the sum
__device__ int block_excl_scan(int v, int *total) {
    __shared__ int sh[kBoxBlk];
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int o = 1; o < kBoxBlk; o <<= 1) {
        const int u = t >= o ? sh[t - o] : 0;
        __syncthreads();
        sh[t] += u;
        __syncthreads();
    }
    const int incl = sh[t];
    *total = sh[kBoxBlk - 1];
    __syncthreads();
    return incl - v;
}

__global__ void __launch_bounds__(kBoxBlk) k_box_count(BoxArgs a, int32_t *cnt) {
    const int32_t m = blockIdx.x;
    int c = 0;
    auto f = [&](int32_t, int32_t, V, V, double, int) { ++c; };
    visit_box(a, m, threadIdx.x, blockDim.x, false, f);
    int total;
    block_excl_scan(c, &total);
    if (threadIdx.x == 0) cnt[m] = total;
}

struct RawOut {
    int32_t *b1, *b2;
    double *r1, *r2, *n, *dist, *mu;
    int64_t cap;
    double erp;
};

// writes the contacts of box m after the sphere contacts (base) at the box's offset: bodies as
// body slots (walls -1, always body 2), contact frame vectors relative to both centres,
// the ERP-scaled distance and the friction coefficient the Contact ctor picks
__global__ void __launch_bounds__(kBoxBlk) k_box_raw(BoxArgs a, const int32_t *off, int64_t base,
                                                     RawOut o, int32_t *err) {
    const int32_t m = blockIdx.x;
    int c = 0;
    auto count = [&](int32_t, int32_t, V, V, double, int) { ++c; };
    visit_box(a, m, threadIdx.x, blockDim.x, false, count);
    int total;
    int64_t pos = base + off[m] + block_excl_scan(c, &total);
    auto write = [&](int32_t b1, int32_t b2, V gpos, V n, double dist, int) {
        if (pos >= o.cap) {
            atomicOr(err, DERR_CAPACITY);
            ++pos;
            return;
        }
        const V rvel = vel_at(a, b1, gpos) - vel_at(a, b2, gpos);
        const MatDev &m1 = a.mats[body_mat(a, b1)], &m2 = a.mats[body_mat(a, b2)];
        const double nvel = dot(n, rvel);
        const double tvel = dot(n, rvel - n * nvel);
        const double mu = (fabs(tvel) > kFrictionThreshold) ? m1.cdf + m2.cdf : m1.csf + m2.csf;
        if (b1 < 0) {   // a wall as body 1 (box/fixed-box): the same contact seen from the box
            const int32_t t = b1;
            b1 = b2;
            b2 = t;
            n = -n;
        }
        const V r1 = gpos - body_x(a, b1);
        const V r2 = b2 >= 0 ? gpos - body_x(a, b2) : v3(0.0, 0.0, 0.0);
        if (dist < 0.0) dist *= o.erp;   // HCSITS.h:1797-1800
        o.b1[pos] = b1;
        o.b2[pos] = b2 >= 0 ? b2 : -1;
        const int64_t cp = o.cap;
        o.r1[pos] = r1.x; o.r1[pos + cp] = r1.y; o.r1[pos + 2 * cp] = r1.z;
        o.r2[pos] = r2.x; o.r2[pos + cp] = r2.y; o.r2[pos + 2 * cp] = r2.z;
        o.n[pos] = n.x; o.n[pos + cp] = n.y; o.n[pos + 2 * cp] = n.z;
        o.dist[pos] = dist;
        o.mu[pos] = mu;
        ++pos;
    };
    visit_box(a, m, threadIdx.x, blockDim.x, false, write);
}

// integratePositions (HCSITS.h:4135-4190) of box m from the slot n + m of the body cache
__global__ void k_box_integrate(BoxArgs a, BodyCacheD bc, double dt, double drag, int has_drag,
                                double *xo, double *qo, double *vo, double *wo, int32_t *err) {
    const int32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= a.m) return;
    const int64_t t = a.n + m;
    const double4 vr = bc.vr[t], wr = bc.wr[t], dv = bc.dv[t], dw = bc.dw[t];
    const V v = v3(vr.x, vr.y, vr.z) + v3(dv.x, dv.y, dv.z);
    const V w = v3(wr.x, wr.y, wr.z) + v3(dw.x, dw.y, dw.z);
    box_advance(a, m, v, w, dt, drag, has_drag, xo, qo, vo, wo);
    if (!isfinite(xo[3 * m]) || !isfinite(xo[3 * m + 1]) || !isfinite(xo[3 * m + 2]))
        atomicOr(err, DERR_NAN);
}

// ---- contact list for pe_b200_find_contacts ------------------------------------------------
__global__ void __launch_bounds__(kBoxBlk) k_box_list(BoxArgs a, const int32_t *off, int64_t cap,
                                                      int64_t n_ids, int64_t total_walls,
                                                      int64_t *ids, double *geom) {
    const int32_t m = blockIdx.x;
    int c = 0;
    auto count = [&](int32_t, int32_t, V, V, double, int) { ++c; };
    visit_box(a, m, threadIdx.x, blockDim.x, false, count);
    int total;
    int64_t pos = off[m] + block_excl_scan(c, &total);
    auto uid_of = [&](int32_t ref) -> int64_t {
        if (ref < 0) return n_ids + (-ref - 1);
        if (ref < a.n) return a.uid[ref];
        return n_ids + total_walls + (ref - a.n);
    };
    auto write = [&](int32_t b1, int32_t b2, V gpos, V n, double dist, int kind) {
        if (pos < cap) {
            ids[3 * pos] = uid_of(b1);
            ids[3 * pos + 1] = uid_of(b2);
            ids[3 * pos + 2] = kind;
            double *g = geom + 7 * pos;
            g[0] = gpos.x; g[1] = gpos.y; g[2] = gpos.z;
            g[3] = n.x; g[4] = n.y; g[5] = n.z;
            g[6] = dist;
        }
        ++pos;
    };
    visit_box(a, m, threadIdx.x, blockDim.x, false, write);
}

// per-box rotation and bounding box of this step
__global__ void k_box_geom(int32_t m, const double *x, const double *q, const double *len,
                           double *R, double *bbb) {
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    OBox b;
    b.x = ld3(x + 3 * k);
    quat_to_rot(q + 4 * k, b.R);
    for (int a = 0; a < 3; ++a) b.len[a] = len[3 * k + a];
    for (int a = 0; a < 9; ++a) R[9 * k + a] = b.R[a];
    box_aabb(b, bbb + 6 * k);
}

// The box grid, built by one block: cells at least two box half-extents and one half-extent
// plus the largest sphere radius wide, so a sphere or a box whose bounding box overlaps a box's
// lies in a neighbouring cell of that box's centre cell; at most a few cells per box.  Boxes are
// counted, scanned and filled into their cells, each cell is put in ascending box order, and a
// bit per cell marks the cells with a box in or next to them.
__global__ void __launch_bounds__(kGridBlk) k_box_grid(int32_t m, const double *bbb, double rmax,
                                                       double *gp, int32_t *gcell,
                                                       int32_t *gstart, int32_t *gfill,
                                                       int32_t *gids, uint32_t *gnear) {
    __shared__ double rlo[3][kGridBlk / 32], rhi[3][kGridBlk / 32], rext[kGridBlk / 32];
    __shared__ int32_t part[kGridBlk];
    __shared__ int32_t s_ncell;
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    const int64_t want = 8 * (int64_t)m > 512 ? 8 * (int64_t)m : 512;
    const int64_t max_cells = want < kMaxBoxCells ? want : kMaxBoxCells;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    double ext = 0.0;
    for (int32_t k = t; k < m; k += kGridBlk) {
        const double *b = bbb + 6 * k;
        for (int a = 0; a < 3; ++a) {
            const double c = 0.5 * (b[a] + b[3 + a]);
            lo[a] = fmin(lo[a], c);
            hi[a] = fmax(hi[a], c);
            ext = fmax(ext, 0.5 * (b[3 + a] - b[a]));
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = fmin(lo[a], __shfl_down_sync(0xffffffffu, lo[a], o));
            hi[a] = fmax(hi[a], __shfl_down_sync(0xffffffffu, hi[a], o));
        }
        ext = fmax(ext, __shfl_down_sync(0xffffffffu, ext, o));
    }
    if (lane == 0) {
        for (int a = 0; a < 3; ++a) {
            rlo[a][wid] = lo[a];
            rhi[a][wid] = hi[a];
        }
        rext[wid] = ext;
    }
    __syncthreads();
    if (t == 0) {
        for (int w = 1; w < kGridBlk / 32; ++w) {
            for (int a = 0; a < 3; ++a) {
                rlo[a][0] = fmin(rlo[a][0], rlo[a][w]);
                rhi[a][0] = fmax(rhi[a][0], rhi[a][w]);
            }
            rext[0] = fmax(rext[0], rext[w]);
        }
        double h = fmax(2.0 * rext[0], rext[0] + rmax) + 4.0 * kContactThreshold;
        if (!(h > 0.0 && h < 1e300)) h = 1.0;
        double span[3];
        for (int a = 0; a < 3; ++a) {
            const double sp = rhi[a][0] - rlo[a][0];
            span[a] = (sp >= 0.0 && sp < 1e300) ? sp : 0.0;   // non-finite states: one cell
        }
        int dim[3] = {1, 1, 1};
        int64_t ncell = 1;
        for (int it = 0; it < 256; ++it) {
            ncell = 1;
            for (int a = 0; a < 3; ++a) {
                dim[a] = (int)fmin(fmax(floor(span[a] / h) + 1.0, 1.0), 4096.0);
                ncell *= dim[a];
            }
            if (ncell <= max_cells) break;
            h *= 1.26;
        }
        if (ncell > max_cells) {   // spans beyond any grid: every box in one cell
            dim[0] = dim[1] = dim[2] = 1;
            ncell = 1;
        }
        for (int a = 0; a < 3; ++a) gp[a] = rlo[a][0];
        gp[3] = 1.0 / h;
        for (int a = 0; a < 3; ++a) gp[4 + a] = dim[a];
        s_ncell = (int32_t)ncell;
    }
    __syncthreads();
    const int32_t ncell = s_ncell;
    for (int32_t c = t; c <= ncell; c += kGridBlk) gstart[c] = 0;
    for (int32_t w = t; w <= (ncell >> 5); w += kGridBlk) gnear[w] = 0u;
    __syncthreads();
    const int gx = (int)gp[4], gy = (int)gp[5], gz = (int)gp[6];
    for (int32_t k = t; k < m; k += kGridBlk) {
        const double *b = bbb + 6 * k;
        int cx, cy, cz;
        box_cell(gp, 0.5 * (b[0] + b[3]), 0.5 * (b[1] + b[4]), 0.5 * (b[2] + b[5]), cx, cy, cz);
        const int32_t c = (cz * gy + cy) * gx + cx;
        gcell[k] = c;
        atomicAdd(&gstart[c + 1], 1);
        for (int z = max(cz - 1, 0); z <= min(cz + 1, gz - 1); ++z)
            for (int y = max(cy - 1, 0); y <= min(cy + 1, gy - 1); ++y)
                for (int x = max(cx - 1, 0); x <= min(cx + 1, gx - 1); ++x) {
                    const int32_t nc = (z * gy + y) * gx + x;
                    atomicOr(&gnear[nc >> 5], 1u << (nc & 31));
                }
    }
    __syncthreads();
    // exclusive scan of the counts: each thread a contiguous chunk, then the chunk totals
    const int32_t chunk = (ncell + kGridBlk) / kGridBlk;
    const int32_t b0 = t * chunk + 1, b1 = min(b0 + chunk, ncell + 1);
    int32_t sum = 0;
    for (int32_t c = b0; c < b1; ++c) sum += gstart[c];
    part[t] = sum;
    __syncthreads();
    for (int o = 1; o < kGridBlk; o <<= 1) {
        const int32_t u = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += u;
        __syncthreads();
    }
    int32_t run = t > 0 ? part[t - 1] : 0;
    for (int32_t c = b0; c < b1; ++c) {
        run += gstart[c];
        gstart[c] = run;
    }
    __syncthreads();
    for (int32_t c = t; c < ncell; c += kGridBlk) gfill[c] = gstart[c];
    __syncthreads();
    for (int32_t k = t; k < m; k += kGridBlk) gids[atomicAdd(&gfill[gcell[k]], 1)] = k;
    __syncthreads();
    for (int32_t c = t; c < ncell; c += kGridBlk) {   // ascending box order in each cell
        const int32_t e0 = gstart[c], e1 = gstart[c + 1];
        for (int32_t i = e0 + 1; i < e1; ++i) {
            const int32_t v = gids[i];
            int32_t j = i - 1;
            while (j >= e0 && gids[j] > v) {
                gids[j + 1] = gids[j];
                --j;
            }
            gids[j + 1] = v;
        }
    }
}

BoxArgs box_args(Ctx *c) {
    BoxArgs a;
    a.n = c->n;
    a.m = c->mb.m;
    a.pr = c->cur.pr;
    a.vw = (const double *)c->cur.vw;
    a.tag = c->cur.tag;
    a.uid = c->cur.uid;
    a.scenes = c->d_scenes;
    a.mats = c->d_mats;
    a.planes = c->d_planes;
    a.plane_mat = c->d_plane_mat;
    a.total_planes = (int32_t)(c->planes.size() / 4);
    a.boxes = c->d_boxes;
    a.box_mat = c->d_box_mat;
    a.bx = c->mb.x;
    a.bq = c->mb.q;
    a.bv = c->mb.v;
    a.bw = c->mb.w;
    a.blen = c->mb.len;
    a.bprops = c->mb.props;
    a.bmat = c->mb.mat;
    a.bscene = c->mb.scene;
    a.cell_start = c->cell_start;
    a.sorted = nullptr;
    a.bR = c->mb.R;
    a.bbb = c->mb.aabb;
    a.gparm = c->mb.gparm;
    a.gstart = c->mb.gstart;
    a.gids = c->mb.gids;
    a.gcell = c->mb.gcell;
    a.gnear = c->mb.gnear;
    return a;
}

// this step's box rotations, bounding boxes and box grid
int box_geometry(Ctx *c) {
    MBoxBuf &b = c->mb;
    k_box_geom<<<grid_for(b.m, 128), 128, 0, c->stream>>>(b.m, b.x, b.q, b.len, b.R, b.aabb);
    PEB_LAUNCHED(c);
    double rmax = 0.0;
    for (const SceneInfo &s : c->scenes) rmax = std::max(rmax, s.rmax);
    k_box_grid<<<1, kGridBlk, 0, c->stream>>>(b.m, b.aabb, c->n > 0 ? rmax : 0.0, b.gparm, b.gcell,
                                              b.gstart, b.gfill, b.gids, b.gnear);
    PEB_LAUNCHED(c);
    return PE_B200_OK;
}

// exclusive scan of cnt[0..m) into cnt[0..m], small m, on the host (the counts come back for
// the capacity check anyway)
int scan_counts(Ctx *c, int32_t m, int32_t *total) {
    std::vector<int32_t> h(m + 1, 0);
    PEB_CUDA(c, cudaMemcpyAsync(h.data(), c->mb.cnt, m * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                c->stream));
    PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    int64_t s = 0;
    for (int32_t k = 0; k < m; ++k) {
        const int64_t v = h[k];
        h[k] = (int32_t)s;
        s += v;
    }
    if (s > INT32_MAX) return set_err(c, PE_B200_ERR_CAPACITY, "too many box contacts");
    h[m] = (int32_t)s;
    PEB_CUDA(c, cudaMemcpyAsync(c->mb.cnt, h.data(), (m + 1) * sizeof(int32_t),
                                cudaMemcpyHostToDevice, c->stream));
    PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    *total = (int32_t)s;
    return PE_B200_OK;
}

}  // namespace

// ---- host side ---------------------------------------------------------------------------------
// BoxBase.h:186-189 (mass), BoxBase.cpp:152-158 (inertia, inverted by Matrix3x3::getInverse,
// Matrix3x3.h:1084-1105, reduced to the diagonal)
static void box_props(const double *len, double density, double *out) {
    const double mass = len[0] * len[1] * len[2] * density;
    double I[3];
    I[0] = mass / 12.0 * (len[1] * len[1] + len[2] * len[2]);
    I[1] = mass / 12.0 * (len[0] * len[0] + len[2] * len[2]);
    I[2] = mass / 12.0 * (len[0] * len[0] + len[1] * len[1]);
    double det = I[0] * ((I[1] * I[2]) - (0.0 * 0.0)) + 0.0 * ((0.0 * 0.0) - (I[2] * 0.0)) +
                 0.0 * ((0.0 * 0.0) - (I[1] * 0.0));
    det = 1.0 / det;
    out[0] = 1.0 / mass;
    out[1] = det * ((I[1] * I[2]) - (0.0 * 0.0));
    out[2] = det * ((I[2] * I[0]) - (0.0 * 0.0));
    out[3] = det * ((I[0] * I[1]) - (0.0 * 0.0));
    out[4] = I[0];
    out[5] = I[1];
    out[6] = I[2];
    out[7] = 0.0;
}

void mbox_free(Ctx *c) {
    MBoxBuf &b = c->mb;
    dfree(c, b.x);
    dfree(c, b.x2);
    dfree(c, b.len);
    dfree(c, b.mat);
    dfree(c, b.cnt);
    dfree(c, b.ext);
    dfree(c, b.R);
    dfree(c, b.gstart);
    b = MBoxBuf();
}

int mbox_upload(Ctx *c, int32_t m, const double *x, const double *q, const double *v,
                const double *w, const double *len, const int32_t *mat, const int32_t *scene) {
    mbox_free(c);
    for (SceneInfo &s : c->scenes) s.mbox_begin = s.nmbox = 0;
    if (m > 0) {
        MBoxBuf &b = c->mb;
        const size_t nm = (size_t)m;
        // one allocation per buffer set: x q v w (13 per box), twice; len + props (11); ints
        PEB_CUDA(c, dmalloc(c, &b.x, 13 * nm * sizeof(double)));
        PEB_CUDA(c, dmalloc(c, &b.x2, 13 * nm * sizeof(double)));
        PEB_CUDA(c, dmalloc(c, &b.len, 11 * nm * sizeof(double)));
        PEB_CUDA(c, dmalloc(c, &b.mat, 2 * nm * sizeof(int32_t)));
        PEB_CUDA(c, dmalloc(c, &b.cnt, (nm + 2) * sizeof(int32_t)));
        // rotations, bounding boxes, grid parameters; grid cells, box lists, neighbour bits
        PEB_CUDA(c, dmalloc(c, &b.R, (15 * nm + 8) * sizeof(double)));
        b.aabb = b.R + 9 * nm;
        b.gparm = b.aabb + 6 * nm;
        const size_t cells = (size_t)kMaxBoxCells + 2;
        PEB_CUDA(c, dmalloc(c, &b.gstart, (2 * cells + 2 * nm + cells / 32 + 2) * sizeof(int32_t)));
        b.gfill = b.gstart + cells;
        b.gids = b.gfill + cells;
        b.gcell = b.gids + nm;
        b.gnear = (uint32_t *)(b.gcell + nm);
        b.q = b.x + 3 * nm;
        b.v = b.q + 4 * nm;
        b.w = b.v + 3 * nm;
        b.q2 = b.x2 + 3 * nm;
        b.v2 = b.q2 + 4 * nm;
        b.w2 = b.v2 + 3 * nm;
        b.props = b.len + 3 * nm;
        b.scene = b.mat + nm;
        b.m = m;
        std::vector<double> props(8 * nm);
        std::vector<int32_t> ints(2 * nm);
        for (int32_t k = 0; k < m; ++k) {
            box_props(len + 3 * k, c->mats[mat[k]].density, &props[8 * k]);
            ints[k] = mat[k];
            ints[nm + k] = scene ? scene[k] : 0;
        }
        PEB_CUDA(c, cudaMemcpyAsync(b.x, x, 3 * nm * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        PEB_CUDA(c, cudaMemcpyAsync(b.q, q, 4 * nm * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        PEB_CUDA(c, cudaMemcpyAsync(b.v, v, 3 * nm * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        PEB_CUDA(c, cudaMemcpyAsync(b.w, w, 3 * nm * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        PEB_CUDA(c, cudaMemcpyAsync(b.len, len, 3 * nm * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        PEB_CUDA(c, cudaMemcpyAsync(b.props, props.data(), 8 * nm * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        PEB_CUDA(c, cudaMemcpyAsync(b.mat, ints.data(), 2 * nm * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
        for (int32_t k = 0; k < m; ++k) {
            SceneInfo &s = c->scenes[ints[nm + k]];
            if (s.nmbox == 0) s.mbox_begin = k;
            s.nmbox++;
        }
    }
    PEB_CUDA(c, cudaMemcpyAsync(c->d_scenes, c->scenes.data(), c->scenes.size() * sizeof(SceneInfo),
                           cudaMemcpyHostToDevice, c->stream));
    c->epoch++;
    return PE_B200_OK;
}

int mbox_download(Ctx *c, double *x, double *q, double *v, double *w) {
    const MBoxBuf &b = c->mb;
    const size_t nm = (size_t)b.m;
    if (nm == 0) return PE_B200_OK;
    PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    if (x) PEB_CUDA(c, cudaMemcpyAsync(x, b.x, 3 * nm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (q) PEB_CUDA(c, cudaMemcpyAsync(q, b.q, 4 * nm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (v) PEB_CUDA(c, cudaMemcpyAsync(v, b.v, 3 * nm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (w) PEB_CUDA(c, cudaMemcpyAsync(w, b.w, 3 * nm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    return PE_B200_OK;
}

void mbox_swap(Ctx *c) {
    MBoxBuf &b = c->mb;
    std::swap(b.x, b.x2);
    std::swap(b.q, b.q2);
    std::swap(b.v, b.v2);
    std::swap(b.w, b.w2);
}

int mbox_dem(Ctx *c, double dt) {
    MBoxBuf &b = c->mb;
    if (b.m == 0) return PE_B200_OK;
    const int64_t n = c->n;
    const size_t nn = (size_t)std::max<int64_t>(n, 1);
    if (b.ext_cap < n || !b.ext) {
        dfree(c, b.ext);
        b.ext = nullptr;
        PEB_CUDA(c, dmalloc(c, &b.ext, nn * 6 * sizeof(double) + (nn + 2) * sizeof(int32_t)));
        b.ext_cap = n;
    }
    int32_t *near_list = (int32_t *)(b.ext + 6 * nn);
    int32_t *near_count = near_list + nn;
    int rc = box_geometry(c);
    if (rc) return rc;
    BoxArgs a = box_args(c);
    a.sorted = c->sorted;   // the grid step leaves the state in body order
    if (n > 0) {
        PEB_CUDA(c, cudaMemsetAsync(near_count, 0, sizeof(int32_t), c->stream));
        k_sphere_box_near<<<grid_for(n, 256), 256, 0, c->stream>>>(a, b.ext, near_list, near_count);
        PEB_LAUNCHED(c);
        const int64_t warps = std::min<int64_t>(n, (int64_t)c->sm_count * 64);
        k_sphere_box_forces<<<(unsigned)((warps + 7) / 8), 256, 0, c->stream>>>(a, b.ext, near_list,
                                                                              near_count);
        PEB_LAUNCHED(c);
    }
    const int has_drag = c->p.damping < 1.0;
    const double drag = has_drag ? pow(c->p.damping, dt) : 1.0;
    k_box_dem<<<b.m, kBoxBlk, 0, c->stream>>>(a, c->p.gravity[0], c->p.gravity[1],
                                              c->p.gravity[2], dt, drag, has_drag, b.x2, b.q2,
                                              b.v2, b.w2, c->d_err);
    PEB_LAUNCHED(c);
    return PE_B200_OK;
}

int mbox_hc_bodycache(Ctx *c, const BodyCacheD &bv, double dt) {
    const MBoxBuf &b = c->mb;
    if (b.m == 0) return PE_B200_OK;
    k_box_bodycache<<<grid_for(b.m, 128), 128, 0, c->stream>>>(
        box_args(c), bv, c->p.gravity[0], c->p.gravity[1], c->p.gravity[2], dt);
    PEB_LAUNCHED(c);
    return PE_B200_OK;
}

int mbox_hc_count(Ctx *c, int32_t *total) {
    *total = 0;
    const MBoxBuf &b = c->mb;
    if (b.m == 0) return PE_B200_OK;
    int rc = box_geometry(c);   // the state is in slot order here: sorted is the identity
    if (rc) return rc;
    k_box_count<<<b.m, kBoxBlk, 0, c->stream>>>(box_args(c), b.cnt);
    PEB_LAUNCHED(c);
    return scan_counts(c, b.m, total);
}

int mbox_hc_raw(Ctx *c, int64_t base, int64_t cap, int32_t *b1, int32_t *b2, double *r1,
                double *r2, double *nrm, double *dist, double *mu) {
    const MBoxBuf &b = c->mb;
    if (b.m == 0) return PE_B200_OK;
    RawOut o{b1, b2, r1, r2, nrm, dist, mu, cap, c->p.erp};
    k_box_raw<<<b.m, kBoxBlk, 0, c->stream>>>(box_args(c), b.cnt, base, o, c->d_err);
    PEB_LAUNCHED(c);
    return PE_B200_OK;
}

int mbox_hc_integrate(Ctx *c, const BodyCacheD &bv, double dt) {
    MBoxBuf &b = c->mb;
    if (b.m == 0) return PE_B200_OK;
    const int has_drag = c->p.damping < 1.0;
    const double drag = has_drag ? pow(c->p.damping, dt) : 1.0;
    k_box_integrate<<<grid_for(b.m, 128), 128, 0, c->stream>>>(box_args(c), bv, dt, drag, has_drag,
                                                                b.x2, b.q2, b.v2, b.w2, c->d_err);
    PEB_LAUNCHED(c);
    mbox_swap(c);
    return PE_B200_OK;
}

int mbox_find_contacts(Ctx *c, std::vector<int64_t> &ids, std::vector<double> &geom) {
    const MBoxBuf &b = c->mb;
    ids.clear();
    geom.clear();
    if (b.m == 0) return PE_B200_OK;
    int rc = box_geometry(c);
    if (rc) return rc;
    BoxArgs a = box_args(c);
    a.sorted = c->sorted;   // the current state, binned by the grid just sorted
    k_box_count<<<b.m, kBoxBlk, 0, c->stream>>>(a, b.cnt);
    PEB_LAUNCHED(c);
    int32_t total = 0;
    rc = scan_counts(c, b.m, &total);
    if (rc) return rc;
    if (total == 0) return PE_B200_OK;
    int64_t *d_ids = nullptr;
    double *d_geom = nullptr;
    cudaError_t e = dmalloc(c, &d_ids, (size_t)total * 3 * sizeof(int64_t));
    if (e == cudaSuccess) e = dmalloc(c, &d_geom, (size_t)total * 7 * sizeof(double));
    const int64_t total_walls = (int64_t)(c->planes.size() / 4 + c->boxes.size() / 15);
    if (e == cudaSuccess) {
        k_box_list<<<b.m, kBoxBlk, 0, c->stream>>>(a, b.cnt, total, c->n, total_walls, d_ids,
                                                   d_geom);
        c->launches++;
        e = cudaGetLastError();
    }
    ids.resize((size_t)total * 3);
    geom.resize((size_t)total * 7);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ids.data(), d_ids, ids.size() * sizeof(int64_t), cudaMemcpyDeviceToHost,
                            c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(geom.data(), d_geom, geom.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    dfree(c, d_ids);
    dfree(c, d_geom);
    if (e != cudaSuccess) return cuda_err(c, e, "box contacts");
    return PE_B200_OK;
}

}  // namespace peb
