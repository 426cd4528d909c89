/*
 * pe_oracle.c -- CPU restatement (FP64, scalar C99) of pe's single-domain rigid-body time step.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product path.  Only tests/, the smoke
 * check and the CPU-baseline leg of bench.py load this library; the product never does.
 *
 * Each function cites the pe source it restates (paths relative to the pe project root).
 * Arithmetic is written in the same operation order as pe so that a step agrees with the
 * compiled reference to a few ulps; the pin against that build lives in tests/test_oracle_*.py.
 */
#include "pe_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define THR PE_OR_CONTACT_THRESHOLD

/* ------------------------------------------------------------------------------------------ */
/* small vector helpers, same operation order as pe/math/Vector3.h                            */
/* ------------------------------------------------------------------------------------------ */
typedef struct { double x, y, z; } v3;

static inline v3 mk(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 ld3(const double *p) { return mk(p[0], p[1], p[2]); }
static inline void st3(double *p, v3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul(v3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline v3 smul(double s, v3 a) { return mk(s * a.x, s * a.y, s * a.z); }
static inline v3 neg(v3 a) { return mk(-a.x, -a.y, -a.z); }
/* Vector3.h:2098 */
static inline double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* Vector3.h:2342-2344 */
static inline v3 cross(v3 a, v3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
/* Vector3.h:958 */
static inline double length(v3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
/* Vector3.h:994-1010 / 1025-1037 */
static inline v3 normalized(v3 a) {
    const double len = sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
    if (len == 0.0) return a;
    const double il = 1.0 / len;
    return mk(a.x * il, a.y * il, a.z * il);
}

/* 3x3 row-major matrices (pe/math/Matrix3x3.h) */
typedef struct { double m[9]; } m3;

static m3 m3_scaled_identity(double s) {
    m3 r; memset(&r, 0, sizeof r); r.m[0] = r.m[4] = r.m[8] = s; return r;
}
/* Matrix3x3.h:351-358: columns c1, c2, c3 */
static m3 m3_cols(v3 a, v3 b, v3 c) {
    m3 r;
    r.m[0] = a.x; r.m[1] = b.x; r.m[2] = c.x;
    r.m[3] = a.y; r.m[4] = b.y; r.m[5] = c.y;
    r.m[6] = a.z; r.m[7] = b.z; r.m[8] = c.z;
    return r;
}
static m3 m3_trans(m3 a) {
    m3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[3 * i + j] = a.m[3 * j + i];
    return r;
}
static v3 m3_mulv(m3 a, v3 v) {
    return mk(a.m[0] * v.x + a.m[1] * v.y + a.m[2] * v.z,
              a.m[3] * v.x + a.m[4] * v.y + a.m[5] * v.z,
              a.m[6] * v.x + a.m[7] * v.y + a.m[8] * v.z);
}
static m3 m3_mul(m3 a, m3 b) {
    m3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            r.m[3 * i + j] = a.m[3 * i + 0] * b.m[0 + j] + a.m[3 * i + 1] * b.m[3 + j] +
                             a.m[3 * i + 2] * b.m[6 + j];
    return r;
}
/* Matrix3x3.h:2419-2432: vec % mat = r^x * M */
static m3 v3_cross_m3(v3 v, m3 a) {
    m3 r;
    r.m[0] = v.y * a.m[6] - v.z * a.m[3];
    r.m[1] = v.y * a.m[7] - v.z * a.m[4];
    r.m[2] = v.y * a.m[8] - v.z * a.m[5];
    r.m[3] = v.z * a.m[0] - v.x * a.m[6];
    r.m[4] = v.z * a.m[1] - v.x * a.m[7];
    r.m[5] = v.z * a.m[2] - v.x * a.m[8];
    r.m[6] = v.x * a.m[3] - v.y * a.m[0];
    r.m[7] = v.x * a.m[4] - v.y * a.m[1];
    r.m[8] = v.x * a.m[5] - v.y * a.m[2];
    return r;
}
/* Matrix3x3.h:2355-2365: mat % vec = M * r^x */
static m3 m3_cross_v3(m3 a, v3 v) {
    m3 r;
    r.m[0] = a.m[1] * v.z - a.m[2] * v.y;
    r.m[1] = a.m[2] * v.x - a.m[0] * v.z;
    r.m[2] = a.m[0] * v.y - a.m[1] * v.x;
    r.m[3] = a.m[4] * v.z - a.m[5] * v.y;
    r.m[4] = a.m[5] * v.x - a.m[3] * v.z;
    r.m[5] = a.m[3] * v.y - a.m[4] * v.x;
    r.m[6] = a.m[7] * v.z - a.m[8] * v.y;
    r.m[7] = a.m[8] * v.x - a.m[6] * v.z;
    r.m[8] = a.m[6] * v.y - a.m[7] * v.x;
    return r;
}
/* Matrix3x3.h:1084-1105 */
static m3 m3_inv(m3 a) {
    const double *v = a.m;
    double det = v[0] * ((v[4] * v[8]) - (v[7] * v[5])) + v[1] * ((v[5] * v[6]) - (v[8] * v[3])) +
                 v[2] * ((v[3] * v[7]) - (v[4] * v[6]));
    det = 1.0 / det;
    m3 r;
    r.m[0] = det * ((v[4] * v[8]) - (v[5] * v[7]));
    r.m[1] = det * ((v[7] * v[2]) - (v[8] * v[1]));
    r.m[2] = det * ((v[1] * v[5]) - (v[2] * v[4]));
    r.m[3] = det * ((v[5] * v[6]) - (v[3] * v[8]));
    r.m[4] = det * ((v[8] * v[0]) - (v[6] * v[2]));
    r.m[5] = det * ((v[2] * v[3]) - (v[0] * v[5]));
    r.m[6] = det * ((v[3] * v[7]) - (v[4] * v[6]));
    r.m[7] = det * ((v[6] * v[1]) - (v[7] * v[0]));
    r.m[8] = det * ((v[0] * v[4]) - (v[1] * v[3]));
    return r;
}

/* Quaternion (w, x, y, z): axis-angle ctor Quaternion.h:274-294, product Quaternion.h:1146-1153 */
static void quat_update(double *q, v3 phi) {
    const double angle = length(phi);
    double d[4];
    if (fabs(angle) < 1e-15) {
        d[0] = 1.0; d[1] = d[2] = d[3] = 0.0;
    } else {
        const double sina = sin(angle * 0.5), cosa = cos(angle * 0.5);
        const v3 ax = normalized(phi);
        d[0] = cosa; d[1] = sina * ax.x; d[2] = sina * ax.y; d[3] = sina * ax.z;
    }
    const double r = d[0] * q[0] - d[1] * q[1] - d[2] * q[2] - d[3] * q[3];
    const double i = d[0] * q[1] + d[1] * q[0] + d[2] * q[3] - d[3] * q[2];
    const double j = d[0] * q[2] + d[2] * q[0] + d[3] * q[1] - d[1] * q[3];
    const double k = d[0] * q[3] + d[3] * q[0] + d[1] * q[2] - d[2] * q[1];
    q[0] = r; q[1] = i; q[2] = j; q[3] = k;
}

/* ------------------------------------------------------------------------------------------ */
/* bodies and materials                                                                        */
/* ------------------------------------------------------------------------------------------ */

/* SphereBase.h:169-171 (mass), SphereBase.cpp:79-80 (1/m), SphereBase.h:230-234 (inertia,
 * inverted by Matrix3x3::getInverse, Matrix3x3.h:1084-1105, reduced here to the diagonal). */
void pe_or_sphere_mass(double r, double density, double *inv_mass, double *inv_inertia,
                       double *inertia) {
    const double mass = 4.0 / 3.0 * M_PI * r * r * r * density;
    const double I = 0.4 * mass * r * r;
    double det = I * ((I * I) - (0.0 * 0.0)) + 0.0 * ((0.0 * 0.0) - (I * 0.0)) +
                 0.0 * ((0.0 * 0.0) - (I * 0.0));
    det = 1.0 / det;
    if (inv_mass) *inv_mass = 1.0 / mass;
    if (inv_inertia) *inv_inertia = det * ((I * I) - (0.0 * 0.0));
    if (inertia) *inertia = I;
}

/* Quaternion.h:591-602 (toRotationMatrix) */
static void quat_to_rot(const double *q, double *R) {
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

/* BoxBase.h:186-189 (mass), BoxBase.cpp:152-158 (inertia, inverted by Matrix3x3::getInverse,
 * Matrix3x3.h:1084-1105, reduced here to the diagonal): im, I[3], Iinv[3] in the body frame */
static void box_mass(const double *len, double density, double *im, double *I, double *Iinv) {
    const double mass = len[0] * len[1] * len[2] * density;
    *im = 1.0 / mass;
    I[0] = mass / 12.0 * (len[1] * len[1] + len[2] * len[2]);
    I[1] = mass / 12.0 * (len[0] * len[0] + len[2] * len[2]);
    I[2] = mass / 12.0 * (len[0] * len[0] + len[1] * len[1]);
    double det = I[0] * ((I[1] * I[2]) - (0.0 * 0.0)) + 0.0 * ((0.0 * 0.0) - (I[2] * 0.0)) +
                 0.0 * ((0.0 * 0.0) - (I[1] * 0.0));
    det = 1.0 / det;
    Iinv[0] = det * ((I[1] * I[2]) - (0.0 * 0.0));
    Iinv[1] = det * ((I[2] * I[0]) - (0.0 * 0.0));
    Iinv[2] = det * ((I[0] * I[1]) - (0.0 * 0.0));
}

/* R * diag(d) * R^T in pe's operation order ((R * D) * trans(R), RotationMatrix.h:1370-1429) */
static m3 rot_diag_rt(const double *R, const double *d) {
    m3 D;
    memset(&D, 0, sizeof D);
    D.m[0] = d[0]; D.m[4] = d[1]; D.m[8] = d[2];
    m3 Rm, Rt;
    memcpy(Rm.m, R, sizeof Rm.m);
    Rt = m3_trans(Rm);
    return m3_mul(m3_mul(Rm, D), Rt);
}

typedef struct {
    int64_t n, nb;   /* spheres, all bodies */
    double *im;      /* inverse mass per body (walls 0) */
    double *ii;      /* inverse inertia (scalar) per body (walls 0) */
    double *I;       /* inertia (scalar) per body (walls 0) */
    int32_t *bmat;   /* material per body */
    double *bpos;    /* 3 per body: centre (planes: anchor point normal*d) */
    int64_t mbase;   /* id of the first moving box */
    m3 *Iinv_w;      /* moving boxes: inverse inertia in the world frame (RigidBody.h:866-869) */
    m3 *I_w;         /* moving boxes: inertia in the world frame (RigidBody.h:842-845) */
} body_props;

static int body_props_init(const pe_or_world *w, body_props *bp) {
    const int64_t nw = (int64_t)w->nplanes + w->nboxes;
    bp->n = w->n;
    bp->nb = w->n + nw + w->nmboxes;
    bp->mbase = w->n + nw;
    bp->Iinv_w = (m3 *)calloc((size_t)(w->nmboxes > 0 ? w->nmboxes : 1), sizeof(m3));
    bp->I_w = (m3 *)calloc((size_t)(w->nmboxes > 0 ? w->nmboxes : 1), sizeof(m3));
    bp->im = (double *)calloc((size_t)bp->nb, sizeof(double));
    bp->ii = (double *)calloc((size_t)bp->nb, sizeof(double));
    bp->I = (double *)calloc((size_t)bp->nb, sizeof(double));
    bp->bmat = (int32_t *)calloc((size_t)bp->nb, sizeof(int32_t));
    bp->bpos = (double *)calloc((size_t)bp->nb * 3, sizeof(double));
    if (!bp->im || !bp->ii || !bp->I || !bp->bmat || !bp->bpos || !bp->Iinv_w || !bp->I_w)
        return -1;
    for (int64_t i = 0; i < w->n; ++i) {
        pe_or_sphere_mass(w->r[i], w->mats[w->mat[i]].density, &bp->im[i], &bp->ii[i], &bp->I[i]);
        bp->bmat[i] = w->mat[i];
        st3(bp->bpos + 3 * i, ld3(w->x + 3 * i));
    }
    for (int32_t p = 0; p < w->nplanes; ++p) {
        const int64_t b = w->n + p;
        bp->bmat[b] = w->plane_mat[p];
        /* Plane.cpp:1202-1207: anchor point normal*d */
        st3(bp->bpos + 3 * b, mul(ld3(w->planes + 4 * p), w->planes[4 * p + 3]));
    }
    for (int32_t k = 0; k < w->nboxes; ++k) {
        const int64_t b = w->n + w->nplanes + k;
        bp->bmat[b] = w->box_mat[k];
        st3(bp->bpos + 3 * b, ld3(w->boxes + 15 * k));
    }
    for (int32_t m = 0; m < w->nmboxes; ++m) {
        const int64_t b = bp->mbase + m;
        double I[3], Iinv[3], R[9];
        box_mass(w->mb_len + 3 * m, w->mats[w->mb_mat[m]].density, &bp->im[b], I, Iinv);
        quat_to_rot(w->mb_q + 4 * m, R);
        bp->Iinv_w[m] = rot_diag_rt(R, Iinv);
        bp->I_w[m] = rot_diag_rt(R, I);
        bp->bmat[b] = w->mb_mat[m];
        st3(bp->bpos + 3 * b, ld3(w->mb_x + 3 * m));
    }
    return 0;
}

static void body_props_free(body_props *bp) {
    free(bp->im); free(bp->ii); free(bp->I); free(bp->bmat); free(bp->bpos);
    free(bp->Iinv_w); free(bp->I_w);
}

/* Materials.h:633-639, 671-677, 709-715: harmonic composition inv(inv(a)+inv(b)) */
static inline double harmonic(double a, double b) { return 1.0 / (1.0 / a + 1.0 / b); }

typedef struct { double k, cn, ct, mu; } contact_params;

/* Contact.cpp:72-115: composed stiffness/damping and the static-vs-dynamic friction pick. */
static contact_params compose(const pe_or_world *w, int32_t m1, int32_t m2, v3 n, v3 rvel) {
    const pe_or_material *a = &w->mats[m1], *b = &w->mats[m2];
    contact_params c;
    c.k = harmonic(a->stiffness, b->stiffness);
    c.cn = harmonic(a->dampingN, b->dampingN);
    c.ct = harmonic(a->dampingT, b->dampingT);
    const double nvel = dot(n, rvel);
    const double tvel = dot(n, sub(rvel, mul(n, nvel)));
    /* Materials.cpp:238-243: csf/cdf tables hold the sum of both materials' coefficients */
    if (fabs(tvel) > PE_OR_FRICTION_THRESHOLD)
        c.mu = (m1 == m2) ? a->cdf + a->cdf : a->cdf + b->cdf;
    else
        c.mu = (m1 == m2) ? a->csf + a->csf : a->csf + b->csf;
    return c;
}

/* ------------------------------------------------------------------------------------------ */
/* fine detection: MaxContacts.h                                                               */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
    pe_or_contact *c;
    int64_t n, cap;
    int oom;
} clist;

static void cpush(clist *l, int64_t b1, int64_t b2, v3 gpos, v3 n, double dist) {
    if (l->n == l->cap) {
        int64_t nc = l->cap ? 2 * l->cap : 1024;
        pe_or_contact *p = (pe_or_contact *)realloc(l->c, (size_t)nc * sizeof(pe_or_contact));
        if (!p) { l->oom = 1; return; }
        l->c = p; l->cap = nc;
    }
    pe_or_contact *c = &l->c[l->n++];
    c->b1 = b1; c->b2 = b2;
    st3(c->gpos, gpos); st3(c->n, n); c->dist = dist;
    c->kind = 0;
}

/* MaxContacts.h:547-569 (i < j: body 1 is the sphere with the smaller system id) */
static void collide_sphere_sphere(const pe_or_world *w, int64_t i, int64_t j, clist *l) {
    const v3 x1 = ld3(w->x + 3 * i), x2 = ld3(w->x + 3 * j);
    v3 normal = sub(x1, x2);
    const double dist = length(normal) - w->r[i] - w->r[j];
    if (dist < THR) {
        normal = normalized(normal);
        const double k = w->r[j] + 0.5 * dist;
        const v3 gpos = add(x2, mul(normal, k));
        cpush(l, i, j, gpos, normal, dist);
    }
}

/* MaxContacts.h:777-790 */
static void collide_sphere_plane(const pe_or_world *w, int64_t i, int32_t p, clist *l) {
    const v3 pn = ld3(w->planes + 4 * p);
    const double pd = w->planes[4 * p + 3];
    const v3 x = ld3(w->x + 3 * i);
    const double k = dot(pn, x);
    const double dist = k - w->r[i] - pd;
    if (dist < THR) {
        const v3 gpos = sub(x, smul(w->r[i] + dist, pn));
        cpush(l, i, w->n + p, gpos, pn, dist);
    }
}

/* A box as the fine detection sees it: centre, rotation (row-major), side lengths, half
 * lengths (real(0.5) * length, as MaxContacts.h and BoxBase.cpp compute them) and body id. */
typedef struct {
    v3 x;
    double R[9];
    double len[3], hl[3];
    int64_t id;
    int fixed;
} obox;


static int64_t mbox_base(const pe_or_world *w) { return w->n + w->nplanes + w->nboxes; }

static obox fixed_box(const pe_or_world *w, int32_t k) {
    const double *B = w->boxes + 15 * k;
    obox b;
    b.x = ld3(B);
    memcpy(b.R, B + 6, sizeof b.R);
    for (int a = 0; a < 3; ++a) { b.len[a] = B[3 + a]; b.hl[a] = 0.5 * B[3 + a]; }
    b.id = w->n + w->nplanes + k;
    b.fixed = 1;
    return b;
}

static obox moving_box(const pe_or_world *w, int32_t m) {
    obox b;
    b.x = ld3(w->mb_x + 3 * m);
    quat_to_rot(w->mb_q + 4 * m, b.R);
    for (int a = 0; a < 3; ++a) { b.len[a] = w->mb_len[3 * m + a]; b.hl[a] = 0.5 * b.len[a]; }
    b.id = mbox_base(w) + m;
    b.fixed = 0;
    return b;
}

/* BoxBase.cpp:100-115 (calcBoundingBox): lo[0..2], hi[3..5] */
static void box_aabb(const obox *b, double *bb) {
    const double *R = b->R, *L = b->len;
    const double e[3] = {
        0.5 * (fabs(R[0] * L[0]) + fabs(R[1] * L[1]) + fabs(R[2] * L[2])) + THR,
        0.5 * (fabs(R[3] * L[0]) + fabs(R[4] * L[1]) + fabs(R[5] * L[2])) + THR,
        0.5 * (fabs(R[6] * L[0]) + fabs(R[7] * L[1]) + fabs(R[8] * L[2])) + THR};
    const double c[3] = {b->x.x, b->x.y, b->x.z};
    for (int a = 0; a < 3; ++a) { bb[a] = c[a] - e[a]; bb[3 + a] = c[a] + e[a]; }
}

/* SphereBase.h:208-218 */
static void sphere_aabb(const pe_or_world *w, int64_t i, double *bb) {
    const double r = w->r[i] + THR;
    for (int a = 0; a < 3; ++a) { bb[a] = w->x[3 * i + a] - r; bb[3 + a] = w->x[3 * i + a] + r; }
}

/* BoundingBox.h:487-497 */
static int aabb_overlap(const double *a, const double *b) {
    return !(b[0] > a[3] || b[1] > a[4] || b[2] > a[5] || b[3] < a[0] || b[4] < a[1] ||
             b[5] < a[2]);
}

/* MaxContacts.h:589-668 (sphere i against a box, fixed or moving) */
static void collide_sphere_obox(const pe_or_world *w, int64_t i, const obox *bx, clist *l) {
    const v3 L = mk(bx->hl[0], bx->hl[1], bx->hl[2]);
    const double *R = bx->R;
    const v3 spos = ld3(w->x + 3 * i), bpos = bx->x;
    const int64_t bid = bx->id;
    int outside = 0;
    const v3 d = sub(spos, bpos);
    double p[3] = {d.x * R[0] + d.y * R[3] + d.z * R[6], d.x * R[1] + d.y * R[4] + d.z * R[7],
                   d.x * R[2] + d.y * R[5] + d.z * R[8]};
    const double l3[3] = {L.x, L.y, L.z};
    for (int a = 0; a < 3; ++a) {
        if (p[a] < -l3[a]) { p[a] = -l3[a]; outside = 1; }
        else if (p[a] > l3[a]) { p[a] = l3[a]; outside = 1; }
    }
    if (!outside) {
        double dist = fabs(p[0]) - l3[0];
        int face = 0;
        for (int a = 1; a < 3; ++a) {
            const double tmp = fabs(p[a]) - l3[a];
            if (dist < tmp) { dist = tmp; face = a; }
        }
        double nl[3] = {0.0, 0.0, 0.0};
        nl[face] = (p[face] > 0.0) ? 1.0 : -1.0;
        const v3 n = mk(R[0] * nl[0] + R[1] * nl[1] + R[2] * nl[2],
                        R[3] * nl[0] + R[4] * nl[1] + R[5] * nl[2],
                        R[6] * nl[0] + R[7] * nl[1] + R[8] * nl[2]);
        dist -= w->r[i];
        cpush(l, i, bid, spos, n, dist);
        return;
    }
    const v3 q = mk(R[0] * p[0] + R[1] * p[1] + R[2] * p[2], R[3] * p[0] + R[4] * p[1] + R[5] * p[2],
                    R[6] * p[0] + R[7] * p[1] + R[8] * p[2]);
    const v3 n = sub(d, q);
    const double dist = length(n) - w->r[i];
    if (dist < THR) cpush(l, i, bid, add(bpos, q), normalized(n), dist);
}

/* MaxContacts.h:2380-2528: every corner of the box on the plane's side is tested */
static void collide_box_plane(const pe_or_world *w, const obox *b, int32_t p, clist *l) {
    const v3 pn = ld3(w->planes + 4 * p);
    const double pd = w->planes[4 * p + 3];
    const double *R = b->R;
    const double range[3] = {0.5 * b->len[0], 0.5 * b->len[1], 0.5 * b->len[2]};
    const double nrel[3] = {R[0] * pn.x + R[3] * pn.y + R[6] * pn.z,
                            R[1] * pn.x + R[4] * pn.y + R[7] * pn.z,
                            R[2] * pn.x + R[5] * pn.y + R[8] * pn.z};
    double mn = range[0];
    if (range[1] < mn) mn = range[1];
    if (range[2] < mn) mn = range[2];
    const double minlength = -0.99 * mn;
    /* corner order of pe: lower-left-front, lower-right-front, lower-right-back,
     * lower-left-back, then the same four on the upper face */
    static const int sg[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                 {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
    for (int k = 0; k < 8; ++k) {
        const double a = sg[k][0] > 0 ? range[0] * nrel[0] : -(range[0] * nrel[0]);
        const double bb = sg[k][1] > 0 ? range[1] * nrel[1] : -(range[1] * nrel[1]);
        const double c = sg[k][2] > 0 ? range[2] * nrel[2] : -(range[2] * nrel[2]);
        if (!((a + bb) + c < minlength)) continue;
        const double cl[3] = {sg[k][0] * range[0], sg[k][1] * range[1], sg[k][2] * range[2]};
        const v3 pos = add(b->x, mk(R[0] * cl[0] + R[1] * cl[1] + R[2] * cl[2],
                                    R[3] * cl[0] + R[4] * cl[1] + R[5] * cl[2],
                                    R[6] * cl[0] + R[7] * cl[1] + R[8] * cl[2]));
        const double kk = pos.x * pn.x + pos.y * pn.y + pos.z * pn.z;
        const double dist = kk - pd;
        if (dist < THR) cpush(l, b->id, w->n + p, pos, pn, dist);
    }
}

/* R^T v and R v for row-major R (RotationMatrix.h:1318-1324 with trans()) */
static v3 rt_mulv(const double *R, v3 v) {
    return mk(R[0] * v.x + R[3] * v.y + R[6] * v.z, R[1] * v.x + R[4] * v.y + R[7] * v.z,
              R[2] * v.x + R[5] * v.y + R[8] * v.z);
}
static v3 r_mulv(const double *R, v3 v) {
    return mk(R[0] * v.x + R[1] * v.y + R[2] * v.z, R[3] * v.x + R[4] * v.y + R[5] * v.z,
              R[6] * v.x + R[7] * v.y + R[8] * v.z);
}
static inline double v3_get(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static inline void v3_set(v3 *a, int i, double s) {
    if (i == 0) a->x = s; else if (i == 1) a->y = s; else a->z = s;
}

/* GeomTools.cpp:387-408 */
static void intersect_lines(v3 o1, v3 d1, v3 o2, v3 d2, double *s, double *t) {
    const v3 c = cross(d1, d2);
    const double sqrlen = c.x * c.x + c.y * c.y + c.z * c.z;
    if (sqrlen < 1e-8) { /* parallelThreshold, Thresholds.h:170 */
        *s = 0.0;
        *t = 0.0;
        return;
    }
    const double isqrlen = 1.0 / sqrlen;
    const v3 p = sub(o2, o1);
    const double dd = dot(d1, d2);
    const double a = dot(d1, p);
    const double b = dot(neg(d2), p);
    *s = (a * dot(d2, d2) + dd * b) * isqrlen;
    *t = (b * dot(d1, d1) + dd * a) * isqrlen;
}

/* one contact point of the vertex/face case (MaxContacts.h:1419-2250): body 1 is B, body 2 A */
static void bb_push(clist *l, const obox *A, const obox *B, v3 gpos, v3 n, double dist) {
    cpush(l, B->id, A->id, gpos, n, dist);
}

/* MaxContacts.h:867-2250: separating-axis test over the 15 axes of the two boxes, then one
 * contact at the closest points of the two edges (edge/edge case) or the contact points of
 * the incident face clipped against the reference face (vertex/face case). */
static void collide_box_box(const obox *p1, const obox *p2, clist *l) {
    const obox *b1 = p1, *b2 = p2;
    if (b2->id < b1->id) { const obox *t = b1; b1 = b2; b2 = t; }
    double maxDepth = -1.79769313486231570815e308;
    int invertNormal = 0;
    int contactCase = 0;
    v3 contactNormal = mk(0.0, 0.0, 0.0), normal_c = mk(0.0, 0.0, 0.0);
    const double *R1 = b1->R, *R2 = b2->R;
    double rR[9], rQ[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            rR[3 * i + j] = R1[i] * R2[j] + R1[3 + i] * R2[3 + j] + R1[6 + i] * R2[6 + j];
    for (int k = 0; k < 9; ++k) rQ[k] = fabs(rR[k]);
    const v3 rPv = rt_mulv(R1, sub(b2->x, b1->x));
    const double rPos[3] = {rPv.x, rPv.y, rPv.z};
    const double *hl1 = b1->hl, *hl2 = b2->hl;
    /* the three face axes of box 1 */
    for (int i = 0; i < 3; ++i) {
        const double term1 =
            fabs(rPos[i]) - (hl1[i] + hl2[0] * rQ[3 * i] + hl2[1] * rQ[3 * i + 1] + hl2[2] * rQ[3 * i + 2]);
        if (term1 > THR) return;
        if (i == 0 || term1 > maxDepth) {
            maxDepth = term1;
            contactNormal = mk(R1[i], R1[3 + i], R1[6 + i]);
            contactCase = 1 + i;
            invertNormal = rPos[i] < 0.0;
        }
    }
    /* the three face axes of box 2 */
    for (int j = 0; j < 3; ++j) {
        const double term1 = rPos[0] * rR[j] + rPos[1] * rR[3 + j] + rPos[2] * rR[6 + j];
        const double term2 =
            fabs(term1) - (hl1[0] * rQ[j] + hl1[1] * rQ[3 + j] + hl1[2] * rQ[6 + j] + hl2[j]);
        if (term2 > THR) return;
        if (term2 > maxDepth) {
            maxDepth = term2;
            contactNormal = mk(R2[j], R2[3 + j], R2[6 + j]);
            contactCase = 4 + j;
            invertNormal = term1 < 0.0;
        }
    }
    /* the nine edge-edge axes, in pe's order (au x bu, au x bv, ... aw x bw); per case: the
     * indices of term1 = rPos[p0]*rR[p1] - rPos[p2]*rR[p3], term2 = hl1[h0]*rQ[q0] +
     * hl1[h1]*rQ[q1], term3 = hl2[h2]*rQ[q2] + hl2[h3]*rQ[q3], length from rR[s0], rR[s1] and
     * the axis in box 1's frame */
    static const int E[9][16] = {
        /* p0 p1 p2 p3  h0 q0 h1 q1  h2 q2 h3 q3  s0 s1 axis(zero component) */
        {2, 3, 1, 6, 1, 6, 2, 3, 2, 1, 1, 2, 6, 3, 0, 0},
        {2, 4, 1, 7, 1, 7, 2, 4, 0, 2, 2, 0, 7, 4, 0, 0},
        {2, 5, 1, 8, 1, 8, 2, 5, 1, 0, 0, 1, 8, 5, 0, 0},
        {0, 6, 2, 0, 2, 0, 0, 6, 2, 4, 1, 5, 6, 0, 1, 0},
        {0, 7, 2, 1, 2, 1, 0, 7, 0, 5, 2, 3, 7, 1, 1, 0},
        {0, 8, 2, 2, 2, 2, 0, 8, 1, 3, 0, 4, 8, 2, 1, 0},
        {1, 0, 0, 3, 0, 3, 1, 0, 2, 7, 1, 8, 3, 0, 2, 0},
        {1, 1, 0, 4, 0, 4, 1, 1, 0, 8, 2, 6, 4, 1, 2, 0},
        {1, 2, 0, 5, 0, 5, 1, 2, 1, 6, 0, 7, 5, 2, 2, 0}};
    for (int e = 0; e < 9; ++e) {
        const int *c = E[e];
        const double term1 = rPos[c[0]] * rR[c[1]] - rPos[c[2]] * rR[c[3]];
        const double term2 = hl1[c[4]] * rQ[c[5]] + hl1[c[6]] * rQ[c[7]];
        const double term3 = hl2[c[8]] * rQ[c[9]] + hl2[c[10]] * rQ[c[11]];
        double sum = fabs(term1) - (term2 + term3);
        if (fabs(term1) > term2 + term3 + THR) return;
        const double a = rR[c[12]], b = rR[c[13]];
        const double length = sqrt(a * a + b * b);
        if (length > 2.2204460492503131e-16) { /* epsilon */
            sum /= length;
            if (sum > maxDepth && fabs(sum - maxDepth) > 1e-8) { /* accuracy */
                maxDepth = sum;
                /* au x b*: (0, -s0, s1); av x b*: (s0, 0, -s1); aw x b*: (-s0, s1, 0) */
                if (c[14] == 0) normal_c = mk(0.0, -a / length, b / length);
                else if (c[14] == 1) normal_c = mk(a / length, 0.0, -b / length);
                else normal_c = mk(-a / length, b / length, 0.0);
                contactCase = 7 + e;
                invertNormal = term1 < 0.0;
            }
        }
    }
    if (contactCase == 0) return;
    if (contactCase > 6) contactNormal = r_mulv(R1, normal_c);
    if (invertNormal) contactNormal = neg(contactNormal);

    if (contactCase > 6) { /* edge/edge, MaxContacts.h:1343-1417 */
        v3 pB1 = b1->x;
        v3 sg = rt_mulv(R1, contactNormal);
        v3 sv;
        for (int i = 0; i < 3; ++i) v3_set(&sv, i, v3_get(sg, i) > 0.0 ? hl1[i] : -hl1[i]);
        pB1 = add(pB1, r_mulv(R1, sv));
        v3 pB2 = b2->x;
        sg = rt_mulv(R2, contactNormal);
        for (int i = 0; i < 3; ++i) v3_set(&sv, i, v3_get(sg, i) > 0.0 ? -hl2[i] : hl2[i]);
        pB2 = add(pB2, r_mulv(R2, sv));
        v3 ua, ub;
        for (int i = 0; i < 3; ++i) {
            v3_set(&ua, i, R1[(contactCase - 7) / 3 + i * 3]);
            v3_set(&ub, i, R2[(contactCase - 7) % 3 + i * 3]);
        }
        double s, t;
        intersect_lines(pB1, ua, pB2, ub, &s, &t);
        pB1 = add(pB1, smul(s, ua));
        pB2 = add(pB2, smul(t, ub));
        const v3 gpos = smul(0.5, add(pB1, pB2));
        cpush(l, b2->id, b1->id, gpos, contactNormal, maxDepth);
        if (!l->oom) l->c[l->n - 1].kind = 1;
        return;
    }

    /* vertex/face: A owns the reference face */
    const obox *A = b1, *B = b2;
    const double *hla = hl1, *hlb = hl2;
    if (contactCase > 3) {
        A = b2; B = b1;
        hla = hl2; hlb = hl1;
        contactNormal = neg(contactNormal);
    }
    const double *Ra = A->R, *Rb = B->R;
    const v3 na = rt_mulv(Ra, contactNormal), nb = rt_mulv(Rb, contactNormal);
    const double normala[3] = {na.x, na.y, na.z}, normalb[3] = {nb.x, nb.y, nb.z};
    int xb, yb, zb;
    if (fabs(normalb[0]) > fabs(normalb[1])) {
        if (fabs(normalb[0]) > fabs(normalb[2])) { xb = 0; yb = 1; zb = 2; }
        else { xb = 2; yb = 0; zb = 1; }
    } else if (fabs(normalb[1]) > fabs(normalb[2])) { xb = 1; yb = 2; zb = 0; }
    else { xb = 2; yb = 0; zb = 1; }
    const int xa = contactCase < 4 ? contactCase - 1 : contactCase - 4;
    const int ya = xa == 0 ? 1 : (xa == 1 ? 2 : 0);
    const int za = xa == 0 ? 2 : (xa == 1 ? 0 : 1);
    /* the incident face of B in B's frame, then in A's frame */
    double vb[4][3];
    for (int k = 0; k < 4; ++k) {
        vb[k][xb] = normalb[xb] > 0.0 ? -hlb[xb] : hlb[xb];
        vb[k][yb] = (k & 1) ? hlb[yb] : -hlb[yb];
        vb[k][zb] = (k & 2) ? hlb[zb] : -hlb[zb];
    }
    const v3 ab = sub(B->x, A->x);
    double vba[4][3];
    for (int k = 0; k < 4; ++k) {
        const v3 t = rt_mulv(Ra, add(ab, r_mulv(Rb, mk(vb[k][0], vb[k][1], vb[k][2]))));
        vba[k][0] = t.x; vba[k][1] = t.y; vba[k][2] = t.z;
    }
    const double offseta = normala[xa] > 0.0 ? hla[xa] : -hla[xa];
    /* the incident face's edges (v0-v1, v0-v2, v3-v1, v3-v2) against the four side lines of
     * the reference face (y = +h, y = -h, z = +h, z = -h in A's frame), MaxContacts.h:1546 */
    static const int EDGE[4][2] = {{0, 1}, {0, 2}, {3, 1}, {3, 2}};
    for (int e = 0; e < 4; ++e) {
        const double *P = vba[EDGE[e][0]], *Q = vba[EDGE[e][1]];
        for (int side = 0; side < 4; ++side) {
            const int cc = side < 2 ? ya : za, o = side < 2 ? za : ya;
            const double h = (side & 1) ? -hla[cc] : hla[cc];
            if (!((P[cc] > h) ^ (Q[cc] > h))) continue;
            const double s = (h - P[cc]) / (Q[cc] - P[cc]);
            if (!(s > 0.0 && s < 1.0)) continue;
            const double tmp = P[o] + s * (Q[o] - P[o]);
            if (!(fabs(tmp) < hla[o])) continue;
            const double dist = fabs(P[xa] + s * (Q[xa] - P[xa])) - hla[xa];
            if (!(dist < THR)) continue;
            double posa[3];
            posa[xa] = offseta;
            posa[cc] = h;
            posa[o] = tmp;
            const v3 gpos = add(A->x, r_mulv(Ra, mk(posa[0], posa[1], posa[2])));
            bb_push(l, A, B, gpos, contactNormal, dist);
        }
    }
    /* vertices of B inside the reference face */
    for (int k = 0; k < 4; ++k) {
        if (fabs(vba[k][ya]) <= hla[ya] && fabs(vba[k][za]) <= hla[za]) {
            const double dist = fabs(vba[k][xa]) - hla[xa];
            if (dist < THR) {
                const v3 gpos = add(A->x, r_mulv(Ra, mk(vba[k][0], vba[k][1], vba[k][2])));
                bb_push(l, A, B, gpos, contactNormal, dist);
            }
        }
    }
    /* vertices of A's reference face inside B's incident face (a vertex on B's vertex is
     * counted once, MaxContacts.h:2179-2185) */
    double va[4][3];
    for (int k = 0; k < 4; ++k) {
        va[k][xa] = normala[xa] > 0.0 ? hla[xa] : -hla[xa];
        va[k][ya] = (k & 1) ? hla[ya] : -hla[ya];
        va[k][za] = (k & 2) ? hla[za] : -hla[za];
    }
    const v3 ba = sub(A->x, B->x);
    for (int k = 0; k < 4; ++k) {
        const v3 t = rt_mulv(Rb, add(ba, r_mulv(Ra, mk(va[k][0], va[k][1], va[k][2]))));
        const double vab[3] = {t.x, t.y, t.z};
        const double ay = fabs(vab[yb]), az = fabs(vab[zb]);
        if (((ay <= hlb[yb] && az < hlb[zb]) || (ay < hlb[yb] && az <= hlb[zb]))) {
            const double dist = fabs(vab[xb]) - hlb[xb];
            if (dist < THR) {
                const v3 gpos = add(B->x, r_mulv(Rb, t));
                bb_push(l, A, B, gpos, contactNormal, dist);
            }
        }
    }
}

static int cmp_contact(const pe_or_contact *x, const pe_or_contact *y) {
    if (x->b1 != y->b1) return x->b1 < y->b1 ? -1 : 1;
    if (x->b2 != y->b2) return x->b2 < y->b2 ? -1 : 1;
    return 0;
}

/* merge sort by (b1, b2), stable so that the contacts of one box pair keep their order */
static int stable_sort_contacts(pe_or_contact *c, int64_t n) {
    pe_or_contact *tmp = (pe_or_contact *)malloc((size_t)n * sizeof(pe_or_contact));
    if (!tmp) return -1;
    for (int64_t width = 1; width < n; width *= 2) {
        for (int64_t lo = 0; lo < n; lo += 2 * width) {
            const int64_t mid = lo + width < n ? lo + width : n;
            const int64_t hi = lo + 2 * width < n ? lo + 2 * width : n;
            int64_t a = lo, b = mid, k = lo;
            while (a < mid && b < hi) tmp[k++] = (cmp_contact(&c[b], &c[a]) < 0) ? c[b++] : c[a++];
            while (a < mid) tmp[k++] = c[a++];
            while (b < hi) tmp[k++] = c[b++];
        }
        memcpy(c, tmp, (size_t)n * sizeof(pe_or_contact));
    }
    free(tmp);
    return 0;
}

/* Broadphase: a uniform cell list whose cell is at least the largest AABB extent, so every pair
 * with overlapping AABBs (pe/core/detection/coarse/HashGrids.h:1351-1358) lies in neighbouring
 * cells.  The resulting contact set equals pe's (its hash grids are exact broadphases), and is
 * sorted canonically by (b1, b2). */
static int find_contacts_list(const pe_or_world *w, clist *l) {
    memset(l, 0, sizeof *l);
    const int64_t n = w->n;
    if (n > 0) {
        double rmax = 0.0, lo[3] = {INFINITY, INFINITY, INFINITY},
               hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int64_t i = 0; i < n; ++i) {
            if (w->r[i] > rmax) rmax = w->r[i];
            for (int a = 0; a < 3; ++a) {
                const double c = w->x[3 * i + a];
                if (c < lo[a]) lo[a] = c;
                if (c > hi[a]) hi[a] = c;
            }
        }
        double h = 2.0 * (rmax + THR) * (1.0 + 1e-9);
        int64_t dim[3], ncell;
        for (;;) {
            ncell = 1;
            for (int a = 0; a < 3; ++a) {
                dim[a] = (int64_t)floor((hi[a] - lo[a]) / h) + 1;
                ncell *= dim[a];
            }
            if (ncell <= 8 * n + 4096) break;
            h *= 1.26;
        }
        int64_t *cell = (int64_t *)malloc((size_t)n * sizeof(int64_t));
        int64_t *start = (int64_t *)calloc((size_t)ncell + 1, sizeof(int64_t));
        int64_t *order = (int64_t *)malloc((size_t)n * sizeof(int64_t));
        if (!cell || !start || !order) { free(cell); free(start); free(order); return -1; }
        for (int64_t i = 0; i < n; ++i) {
            int64_t c[3];
            for (int a = 0; a < 3; ++a) {
                c[a] = (int64_t)floor((w->x[3 * i + a] - lo[a]) / h);
                if (c[a] < 0) c[a] = 0;
                if (c[a] >= dim[a]) c[a] = dim[a] - 1;
            }
            cell[i] = (c[2] * dim[1] + c[1]) * dim[0] + c[0];
            start[cell[i] + 1]++;
        }
        for (int64_t c = 0; c < ncell; ++c) start[c + 1] += start[c];
        {
            int64_t *fill = (int64_t *)malloc((size_t)ncell * sizeof(int64_t));
            if (!fill) { free(cell); free(start); free(order); return -1; }
            memcpy(fill, start, (size_t)ncell * sizeof(int64_t));
            for (int64_t i = 0; i < n; ++i) order[fill[cell[i]]++] = i;
            free(fill);
        }
        for (int64_t i = 0; i < n; ++i) {
            const int64_t c = cell[i];
            const int64_t cx = c % dim[0], cy = (c / dim[0]) % dim[1], cz = c / (dim[0] * dim[1]);
            for (int64_t dz = -1; dz <= 1; ++dz) {
                const int64_t z = cz + dz;
                if (z < 0 || z >= dim[2]) continue;
                for (int64_t dy = -1; dy <= 1; ++dy) {
                    const int64_t y = cy + dy;
                    if (y < 0 || y >= dim[1]) continue;
                    for (int64_t dx = -1; dx <= 1; ++dx) {
                        const int64_t x = cx + dx;
                        if (x < 0 || x >= dim[0]) continue;
                        const int64_t nc = (z * dim[1] + y) * dim[0] + x;
                        for (int64_t s = start[nc]; s < start[nc + 1]; ++s) {
                            const int64_t j = order[s];
                            if (j > i) collide_sphere_sphere(w, i, j, l);
                        }
                    }
                }
            }
        }
        free(cell); free(start); free(order);
    }
    /* HashGrids.h:1278-1285: every gridded body against every infinite body (planes); boxes are
     * finite bodies in the grids, tested here directly */
    for (int64_t i = 0; i < n; ++i) {
        for (int32_t p = 0; p < w->nplanes; ++p) collide_sphere_plane(w, i, p, l);
        for (int32_t b = 0; b < w->nboxes; ++b) {
            const obox fb = fixed_box(w, b);
            collide_sphere_obox(w, i, &fb, l);
        }
    }
    /* moving boxes: HashGrids::collide (HashGrids.h:1351-1358) tests the bounding boxes before
     * the fine detection; planes are infinite bodies and always tested (HashGrids.h:1278-1285);
     * fixed boxes are finite bodies in the grids */
    const int32_t M = w->nmboxes;
    if (M > 0) {
        obox *mb = (obox *)malloc((size_t)M * sizeof(obox));
        double *bb = (double *)malloc((size_t)M * 6 * sizeof(double));
        if (!mb || !bb) { free(mb); free(bb); free(l->c); return -1; }
        for (int32_t m = 0; m < M; ++m) {
            mb[m] = moving_box(w, m);
            box_aabb(&mb[m], bb + 6 * m);
        }
        for (int64_t i = 0; i < n; ++i) {
            double sb[6];
            sphere_aabb(w, i, sb);
            for (int32_t m = 0; m < M; ++m)
                if (aabb_overlap(sb, bb + 6 * m)) collide_sphere_obox(w, i, &mb[m], l);
        }
        for (int32_t m = 0; m < M; ++m) {
            for (int32_t p = 0; p < w->nplanes; ++p) collide_box_plane(w, &mb[m], p, l);
            for (int32_t k = 0; k < w->nboxes; ++k) {
                const obox fb = fixed_box(w, k);
                double fbb[6];
                box_aabb(&fb, fbb);
                if (aabb_overlap(bb + 6 * m, fbb)) collide_box_box(&mb[m], &fb, l);
            }
            for (int32_t m2 = m + 1; m2 < M; ++m2)
                if (aabb_overlap(bb + 6 * m, bb + 6 * m2)) collide_box_box(&mb[m], &mb[m2], l);
        }
        free(mb);
        free(bb);
    }
    if (l->oom) { free(l->c); return -1; }
    if (l->n > 1 && stable_sort_contacts(l->c, l->n) != 0) { free(l->c); return -1; }
    return 0;
}

int64_t pe_or_find_contacts(const pe_or_world *w, pe_or_contact *out, int64_t cap) {
    clist l;
    if (find_contacts_list(w, &l) != 0) return -1;
    const int64_t m = l.n < cap ? l.n : cap;
    if (m > 0 && out) memcpy(out, l.c, (size_t)m * sizeof(pe_or_contact));
    free(l.c);
    return l.n;
}

/* ------------------------------------------------------------------------------------------ */
/* DEM step                                                                                    */
/* ------------------------------------------------------------------------------------------ */

/* RigidBody.h:1080-1085 */
static inline v3 vel_from_wf(const pe_or_world *w, int64_t b, v3 gpos) {
    const int64_t mb = mbox_base(w);
    if (b >= w->n && b < mb) return mk(0.0, 0.0, 0.0);
    const double *vv = b < w->n ? w->v + 3 * b : w->mb_v + 3 * (b - mb);
    const double *ww = b < w->n ? w->w + 3 * b : w->mb_w + 3 * (b - mb);
    const double *xx = b < w->n ? w->x + 3 * b : w->mb_x + 3 * (b - mb);
    const v3 v = ld3(vv), om = ld3(ww), x = ld3(xx);
    return add(v, cross(om, sub(gpos, x)));
}

/* index of a dynamic body in the force accumulators (spheres, then moving boxes); -1: wall */
static inline int64_t dyn_index(const pe_or_world *w, int64_t b) {
    if (b < w->n) return b;
    const int64_t mb = mbox_base(w);
    return b >= mb ? w->n + (b - mb) : -1;
}

static inline const double *body_x(const pe_or_world *w, int64_t b) {
    return b < w->n ? w->x + 3 * b : w->mb_x + 3 * (b - mbox_base(w));
}

/* RigidBody.h:1775-1803 */
static inline void add_force_at_pos(const pe_or_world *w, double *F, double *T, int64_t b, v3 f,
                                    v3 gpos) {
    const int64_t d = dyn_index(w, b);
    if (d < 0) return; /* walls are fixed: their accumulated force is never used */
    st3(F + 3 * d, add(ld3(F + 3 * d), f));
    st3(T + 3 * d, add(ld3(T + 3 * d), cross(sub(gpos, ld3(body_x(w, b))), f)));
}

static int32_t body_mat(const pe_or_world *w, int64_t b) {
    if (b < w->n) return w->mat[b];
    if (b < w->n + w->nplanes) return w->plane_mat[b - w->n];
    if (b < mbox_base(w)) return w->box_mat[b - w->n - w->nplanes];
    return w->mb_mat[b - mbox_base(w)];
}




/* Materials.h:586-600: effective Young's modulus 1/E = (1-nu1^2)/E1 + (1-nu2^2)/E2, in pe's
 * operation order */
static double effective_young(const pe_or_material *a, const pe_or_material *b) {
    const double tmp1 = b->young * (1.0 - a->poisson * a->poisson);
    const double tmp2 = a->young * (1.0 - b->poisson * b->poisson);
    return (a->young * b->young) / (tmp1 + tmp2);
}

/* response/DEMSolver.h:176-380 (single-process branch): the extended Hertz law for sphere-sphere
 * contacts when forceModel == hertz (:343-357; contacttrait/DEMSolver.h:143-160 for the
 * effective radius and modulus; other contacts have no effective radius), else the linear
 * spring-dashpot law (:360-366) */
static void dem_resolve(const pe_or_world *w, const pe_or_contact *c, double *F, double *T) {
    if (!(c->dist < -THR)) return; /* ContactBase.h:307-310 isPenetrating */
    const v3 gpos = ld3(c->gpos), n = ld3(c->n);
    const v3 rvel = sub(vel_from_wf(w, c->b1, gpos), vel_from_wf(w, c->b2, gpos));
    contact_params cp = compose(w, body_mat(w, c->b1), body_mat(w, c->b2), n, rvel);
    if (c->kind == 1) cp.k = cp.cn = cp.ct = 0.0;
    const double delta = -c->dist;
    const double relVelN = -dot(n, rvel);
    const v3 relVel = neg(rvel);
    const v3 relVelT = sub(relVel, mul(n, relVelN));
    double fNabs;
    if (w->force_model == 1 && c->b2 < w->n) {
        const double r1 = w->r[c->b1], r2 = w->r[c->b2];
        const double Reff = (r1 * r2) / (r1 + r2);
        const double Eeff = effective_young(&w->mats[w->mat[c->b1]], &w->mats[w->mat[c->b2]]);
        const double k = (4.0 / 3.0) * Eeff * sqrt(Reff);
        fNabs = k * pow(delta, 1.5) + cp.cn * relVelN * pow(delta, 0.5);
    } else {
        fNabs = cp.k * delta + cp.cn * relVelN;
    }
    if (fNabs < 0.0) fNabs = 0.0;
    const v3 fN = smul(fNabs, n);
    const double ft1 = cp.ct * length(relVelT), ft2 = cp.mu * fNabs;
    const double fTabs = ft1 < ft2 ? ft1 : ft2;
    const v3 fT = smul(fTabs, normalized(relVelT));
    add_force_at_pos(w, F, T, c->b1, fN, gpos);
    add_force_at_pos(w, F, T, c->b2, neg(fN), gpos);
    add_force_at_pos(w, F, T, c->b1, fT, gpos);
    add_force_at_pos(w, F, T, c->b2, neg(fT), gpos);
}

/* boxtrait/Default.h:149-220 (BoxTrait::move) for moving box m, force F and torque T */
static void box_move(pe_or_world *w, int32_t m, v3 F, v3 T, double dt) {
    const pe_or_material *mt = &w->mats[w->mb_mat[m]];
    double im, I[3], Iinv[3], R[9];
    box_mass(w->mb_len + 3 * m, mt->density, &im, I, Iinv);
    quat_to_rot(w->mb_q + 4 * m, R);
    const v3 g = mk(w->gravity[0], w->gravity[1], w->gravity[2]);
    const v3 vdot = add(mul(F, im), g);
    const v3 tmp1 = rt_mulv(R, T);
    const v3 tmp2 = mk(Iinv[0] * tmp1.x, Iinv[1] * tmp1.y, Iinv[2] * tmp1.z);
    const v3 wdot = r_mulv(R, tmp2);
    v3 v = add(ld3(w->mb_v + 3 * m), mul(vdot, dt));
    v3 om = add(ld3(w->mb_w + 3 * m), mul(wdot, dt));
    st3(w->mb_x + 3 * m, add(ld3(w->mb_x + 3 * m), mul(v, dt)));
    quat_update(w->mb_q + 4 * m, mul(om, dt));
    if (w->damping < 1.0) {
        const double drag = pow(w->damping, dt);
        v = mul(v, drag);
        om = mul(om, drag);
    }
    st3(w->mb_v + 3 * m, v);
    st3(w->mb_w + 3 * m, om);
}

/* collisionsystem/DEMSolver.h:1155-1262 + spheretrait/Default.h:149-220 */
int64_t pe_or_dem_step(pe_or_world *w, double dt) {
    clist l;
    if (find_contacts_list(w, &l) != 0) return -1;
    const int64_t n = w->n, nd = w->n + w->nmboxes;
    double *F = (double *)calloc((size_t)(3 * nd + 3), sizeof(double));
    double *T = (double *)calloc((size_t)(3 * nd + 3), sizeof(double));
    if (!F || !T) { free(F); free(T); free(l.c); return -1; }
    for (int64_t k = 0; k < l.n; ++k) dem_resolve(w, &l.c[k], F, T);
    const v3 g = mk(w->gravity[0], w->gravity[1], w->gravity[2]);
    for (int64_t i = 0; i < n; ++i) {
        double im, ii;
        pe_or_sphere_mass(w->r[i], w->mats[w->mat[i]].density, &im, &ii, NULL);
        const v3 vdot = add(mul(ld3(F + 3 * i), im), g);
        const v3 wdot = smul(ii, ld3(T + 3 * i));
        v3 v = add(ld3(w->v + 3 * i), mul(vdot, dt));
        v3 om = add(ld3(w->w + 3 * i), mul(wdot, dt));
        st3(w->x + 3 * i, add(ld3(w->x + 3 * i), mul(v, dt)));
        if (w->q) quat_update(w->q + 4 * i, mul(om, dt));
        if (w->damping < 1.0) {
            const double drag = pow(w->damping, dt);
            v = mul(v, drag);
            om = mul(om, drag);
        }
        st3(w->v + 3 * i, v);
        st3(w->w + 3 * i, om);
    }
    for (int32_t m = 0; m < w->nmboxes; ++m)
        box_move(w, m, ld3(F + 3 * (n + m)), ld3(T + 3 * (n + m)), dt);
    free(F); free(T);
    const int64_t nc = l.n;
    free(l.c);
    return nc;
}

/* ------------------------------------------------------------------------------------------ */
/* hard-contact step (HCSITS)                                                                  */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
    int64_t b1, b2;
    v3 r1, r2, n, t, o;
    double dist, mu;
    m3 D, Dinv;
    double Dn_inv;
    double Dto_inv[4];
    v3 p;
} hc_contact;

/* HardContactSemiImplicitTimesteppingSolvers.h:1767-1815 */
static void hc_cache(const pe_or_world *w, const body_props *bp, const pe_or_contact *c,
                     double erp, hc_contact *h) {
    h->b1 = c->b1; h->b2 = c->b2;
    const v3 gpos = ld3(c->gpos);
    h->r1 = sub(gpos, ld3(bp->bpos + 3 * c->b1));
    h->r2 = sub(gpos, ld3(bp->bpos + 3 * c->b2));
    const v3 n = ld3(c->n);
    h->n = n;
    v3 t;
    if (fabs(n.x) < fabs(n.y)) {
        if (fabs(n.x) < fabs(n.z)) t = mk(0.0, n.z, -n.y);
        else t = mk(n.y, -n.x, 0.0);
    } else {
        if (fabs(n.y) < fabs(n.z)) t = mk(-n.z, 0.0, n.x);
        else t = mk(n.y, -n.x, 0.0);
    }
    h->t = normalized(t);
    h->o = cross(n, h->t);
    const m3 cf = m3_cols(h->n, h->t, h->o);
    h->dist = c->dist;
    if (h->dist < 0.0) h->dist *= erp;
    /* the friction coefficient is the one the Contact ctor chose (Contact.cpp:102-105) */
    {
        const v3 rv = sub(vel_from_wf(w, c->b1, gpos), vel_from_wf(w, c->b2, gpos));
        h->mu = compose(w, body_mat(w, c->b1), body_mat(w, c->b2), n, rv).mu;
    }
    const m3 I1 = c->b1 >= bp->mbase ? bp->Iinv_w[c->b1 - bp->mbase]
                                     : m3_scaled_identity(bp->ii[c->b1]);
    const m3 I2 = c->b2 >= bp->mbase ? bp->Iinv_w[c->b2 - bp->mbase]
                                     : m3_scaled_identity(bp->ii[c->b2]);
    const m3 a = m3_cross_v3(v3_cross_m3(h->r1, I1), h->r1);
    const m3 b = m3_cross_v3(v3_cross_m3(h->r2, I2), h->r2);
    m3 D;
    for (int k = 0; k < 9; ++k) D.m[k] = -(a.m[k] + b.m[k]);
    const double ims = bp->im[c->b1] + bp->im[c->b2];
    D.m[0] += ims; D.m[4] += ims; D.m[8] += ims;
    D = m3_mul(m3_mul(m3_trans(cf), D), cf);
    h->D = D;
    h->Dinv = m3_inv(D);
    h->Dn_inv = 1.0 / D.m[0];
    /* inverse of the 2x2 block (D[4] D[5]; D[7] D[8]) */
    const double det = D.m[4] * D.m[8] - D.m[5] * D.m[7];
    const double idet = 1.0 / det;
    h->Dto_inv[0] = idet * D.m[8];
    h->Dto_inv[1] = -idet * D.m[5];
    h->Dto_inv[2] = -idet * D.m[7];
    h->Dto_inv[3] = idet * D.m[4];
    h->p = mk(0.0, 0.0, 0.0);
}

typedef struct {
    v3 *v, *w, *dv, *dw;
} hc_bodies;

static inline v3 wf_imp(const body_props *bp, int64_t b, v3 r, v3 p) {
    if (b >= bp->mbase) return m3_mulv(bp->Iinv_w[b - bp->mbase], cross(r, p));
    return smul(bp->ii[b], cross(r, p));
}

static inline void hc_apply(const body_props *bp, hc_bodies *B, const hc_contact *h, v3 p,
                            double sign) {
    /* dv1 += sign*im1*p; dw1 += sign*Iinv1*(r1 x p); body 2 with the opposite sign.  Walls
     * carry zero inverse mass and inertia, so their corrections stay zero as in pe -- unless an
     * impulse is not finite, which pe then spreads through the wall as well. */
    B->dv[h->b1] = add(B->dv[h->b1], smul(sign, smul(bp->im[h->b1], p)));
    B->dw[h->b1] = add(B->dw[h->b1], smul(sign, wf_imp(bp, h->b1, h->r1, p)));
    B->dv[h->b2] = sub(B->dv[h->b2], smul(sign, smul(bp->im[h->b2], p)));
    B->dw[h->b2] = sub(B->dw[h->b2], smul(sign, wf_imp(bp, h->b2, h->r2, p)));
}

static inline v3 hc_gdot(const hc_bodies *B, const hc_contact *h) {
    const v3 a = add(B->v[h->b1], B->dv[h->b1]);
    const v3 b = add(B->v[h->b2], B->dv[h->b2]);
    const v3 c = cross(add(B->w[h->b1], B->dw[h->b1]), h->r1);
    const v3 d = cross(add(B->w[h->b2], B->dw[h->b2]), h->r2);
    return sub(add(sub(a, b), c), d);
}

static inline double maxabs3(v3 a) {
    return fmax(fabs(a.x), fmax(fabs(a.y), fabs(a.z)));
}

/* HardContactSemiImplicitTimesteppingSolvers.h:2039-2105 */
static double relax_frictionless(const body_props *bp, hc_bodies *B, hc_contact *C, int64_t nc,
                                 double dtinv) {
    double delta_max = 0.0;
    for (int64_t i = 0; i < nc; ++i) {
        hc_contact *h = &C[i];
        hc_apply(bp, B, h, h->p, -1.0);
        const v3 gdot = hc_gdot(B, h);
        double gn = dot(h->n, gdot);
        gn += h->dist * dtinv;
        if (gn >= 0.0) {
            delta_max = fmax(delta_max, maxabs3(h->p));
            h->p = mk(0.0, 0.0, 0.0);
        } else {
            const v3 p_wf = mul(h->n, -h->Dn_inv * gn);
            delta_max = fmax(delta_max, maxabs3(sub(h->p, p_wf)));
            h->p = p_wf;
            hc_apply(bp, B, h, h->p, 1.0);
        }
    }
    return delta_max;
}

/* HardContactSemiImplicitTimesteppingSolvers.h:2129-2304 */
static double relax_approx_coulomb(const body_props *bp, hc_bodies *B, hc_contact *C, int64_t nc,
                                   double dtinv) {
    double delta_max = 0.0;
    for (int64_t i = 0; i < nc; ++i) {
        hc_contact *h = &C[i];
        hc_apply(bp, B, h, h->p, -1.0);
        const v3 gdot = hc_gdot(B, h);
        const m3 cf = m3_cols(h->n, h->t, h->o);
        v3 g = m3_mulv(m3_trans(cf), gdot);
        g.x += h->dist * dtinv;
        if (g.x >= 0.0) {
            delta_max = fmax(delta_max, maxabs3(h->p));
            h->p = mk(0.0, 0.0, 0.0);
            continue;
        }
        v3 pcf = neg(m3_mulv(h->Dinv, g));
        double flimit = h->mu * pcf.x;
        double fsq = pcf.y * pcf.y + pcf.z * pcf.z;
        if (fsq > flimit * flimit || pcf.x < 0.0) {
            v3 ptmp = add(mul(h->t, dot(h->t, h->p)), mul(h->o, dot(h->o, h->p)));
            const double gdot_n =
                g.x + dot(h->n, add(cross(wf_imp(bp, h->b1, h->r1, ptmp), h->r1),
                                    cross(wf_imp(bp, h->b2, h->r2, ptmp), h->r2)));
            pcf.x = -(h->Dn_inv * gdot_n);
            pcf.x = fmax(0.0, pcf.x);
            ptmp = mul(h->n, pcf.x);
            const v3 gdot2 = add(add(gdot, cross(wf_imp(bp, h->b1, h->r1, ptmp), h->r1)),
                                 cross(wf_imp(bp, h->b2, h->r2, ptmp), h->r2));
            const double gt = dot(h->t, gdot2), go = dot(h->o, gdot2);
            pcf.y = -(h->Dto_inv[0] * gt + h->Dto_inv[1] * go);
            pcf.z = -(h->Dto_inv[2] * gt + h->Dto_inv[3] * go);
            flimit = h->mu * pcf.x;
            fsq = pcf.y * pcf.y + pcf.z * pcf.z;
            if (fsq > flimit * flimit) {
                const double f = flimit / sqrt(fsq);
                pcf.y *= f;
                pcf.z *= f;
            }
        }
        const v3 p_wf = m3_mulv(cf, pcf);
        delta_max = fmax(delta_max, maxabs3(sub(h->p, p_wf)));
        h->p = p_wf;
        hc_apply(bp, B, h, h->p, 1.0);
    }
    return delta_max;
}

/* HardContactSemiImplicitTimesteppingSolvers.h:2631-2723: one projected Jacobi-like update
 * per contact with relaxation w = 1, then the projection onto the friction cone (approximate:
 * the plain residual D p + gdot; exact: its normal part raised by mu |(D p + gdot)_to|) */
static double relax_orthogonal(const body_props *bp, hc_bodies *B, hc_contact *C, int64_t nc,
                               double dtinv, int approximate) {
    double delta_max = 0.0;
    for (int64_t i = 0; i < nc; ++i) {
        hc_contact *h = &C[i];
        hc_apply(bp, B, h, h->p, -1.0);
        const v3 gdot = hc_gdot(B, h);
        const m3 cf = m3_cols(h->n, h->t, h->o);
        v3 g = m3_mulv(m3_trans(cf), gdot);
        g.x += h->dist * dtinv;
        const double w = 1.0;
        v3 pcf = m3_mulv(m3_trans(cf), h->p);
        if (approximate) {
            pcf = sub(pcf, smul(w, add(m3_mulv(h->D, pcf), g)));
        } else {
            v3 tmp = add(m3_mulv(h->D, pcf), g);
            tmp.x += sqrt(tmp.y * tmp.y + tmp.z * tmp.z) * h->mu;
            pcf = sub(pcf, smul(w, tmp));
        }
        const double flimit = h->mu * pcf.x;
        const double fsq = pcf.y * pcf.y + pcf.z * pcf.z;
        if (pcf.x > 0.0 && fsq < flimit * flimit) {
            /* inside the cone */
        } else if (pcf.x < 0.0 && fsq < pcf.x / (h->mu * h->mu)) {
            pcf = mk(0.0, 0.0, 0.0);
        } else {
            const double f = sqrt(fsq);
            pcf.x = (f * h->mu + pcf.x) / (h->mu * h->mu + 1.0);
            const double factor = h->mu * pcf.x / f;
            pcf.y *= factor;
            pcf.z *= factor;
        }
        const v3 p_wf = m3_mulv(cf, pcf);
        delta_max = fmax(delta_max, maxabs3(sub(h->p, p_wf)));
        h->p = p_wf;
        hc_apply(bp, B, h, h->p, 1.0);
    }
    return delta_max;
}

/* 2x2 helpers in pe's evaluation order: Matrix2 * Vector2 and trans(a) * b */
static inline void m2_mulv(double a00, double a01, double a10, double a11, double x0, double x1,
                           double *y0, double *y1) {
    *y0 = a00 * x0 + a01 * x1;
    *y1 = a10 * x0 + a11 * x1;
}
/* real(0.5) * trans(x) * (A * x) - trans(x) * b, left to right */
static inline double quad2(double a00, double a01, double a10, double a11, double x0, double x1,
                           double b0, double b1) {
    double y0, y1;
    m2_mulv(a00, a01, a10, a11, x0, x1, &y0, &y1);
    return ((0.5 * x0) * y0 + (0.5 * x1) * y1) - (x0 * b0 + x1 * b1);
}

/* HardContactSemiImplicitTimesteppingSolvers.h:2330-2595: exact Coulomb friction by
 * alternating normal and tangential one-contact solves (20 rounds); a tangential solution
 * outside the cone is replaced by the minimiser of the tangential energy on the cone's circle,
 * found by a golden-section search over the angle (maxSubIterations = 20, HCSITS.h:423) */
static double relax_coulomb_decoupling(const body_props *bp, hc_bodies *B, hc_contact *C,
                                       int64_t nc, double dtinv) {
    double delta_max = 0.0;
    for (int64_t i = 0; i < nc; ++i) {
        hc_contact *h = &C[i];
        hc_apply(bp, B, h, h->p, -1.0);
        const v3 gdot = hc_gdot(B, h);
        const m3 cf = m3_cols(h->n, h->t, h->o);
        v3 g = m3_mulv(m3_trans(cf), gdot);
        g.x += h->dist * dtinv;
        if (g.x >= 0.0) {
            delta_max = fmax(delta_max, maxabs3(h->p));
            h->p = mk(0.0, 0.0, 0.0);
            continue;
        }
        v3 pcf = neg(m3_mulv(h->Dinv, g));
        double flimit = h->mu * pcf.x;
        double fsq = pcf.y * pcf.y + pcf.z * pcf.z;
        if (fsq > flimit * flimit || pcf.x < 0.0) {
            for (int j = 0; j < 20; ++j) {
                pcf.x = 0.0;
                const v3 pto = add(mul(h->t, pcf.y), mul(h->o, pcf.z));
                v3 gc = add(add(gdot, cross(wf_imp(bp, h->b1, h->r1, pto), h->r1)),
                            cross(wf_imp(bp, h->b2, h->r2, pto), h->r2));
                const double gc_n = dot(h->n, gc) + h->dist * dtinv;
                pcf.x = fmax(0.0, -(h->Dn_inv * gc_n));
                pcf.y = pcf.z = 0.0;
                const v3 pn = mul(h->n, pcf.x);
                gc = add(add(gdot, cross(wf_imp(bp, h->b1, h->r1, pn), h->r1)),
                         cross(wf_imp(bp, h->b2, h->r2, pn), h->r2));
                const double gt = dot(h->t, gc), go = dot(h->o, gc);
                double r0, r1;
                m2_mulv(h->Dto_inv[0], h->Dto_inv[1], h->Dto_inv[2], h->Dto_inv[3], gt, go, &r0, &r1);
                pcf.y = -r0;
                pcf.z = -r1;
                flimit = h->mu * pcf.x;
                fsq = pcf.y * pcf.y + pcf.z * pcf.z;
                if (fsq > flimit * flimit) {
                    const double a00 = h->D.m[4], a01 = h->D.m[5], a10 = h->D.m[7], a11 = h->D.m[8];
                    const double f = flimit / sqrt(fsq);
                    const double phi = 0.5 * (1.0 + sqrt(5.0));
                    const double shift = atan2(-pcf.z, pcf.y);
                    const double acos_f = acos(f);
                    double alpha_left = -acos_f - shift;
                    double alpha_right = acos_f - shift;
                    double alpha_mid = (alpha_right + alpha_left * phi) / (1.0 + phi);
                    double xm0 = flimit * cos(alpha_mid), xm1 = flimit * sin(alpha_mid);
                    double f_mid = quad2(a00, a01, a10, a11, xm0, xm1, -gt, -go);
                    int leftlarger = 0;
                    for (int k = 0; k < 20; ++k) {
                        const double alpha_next = alpha_left + (alpha_right - alpha_mid);
                        const double xn0 = flimit * cos(alpha_next), xn1 = flimit * sin(alpha_next);
                        const double f_next = quad2(a00, a01, a10, a11, xn0, xn1, -gt, -go);
                        if (leftlarger) {
                            if (f_next < f_mid) {
                                alpha_right = alpha_mid; alpha_mid = alpha_next;
                                xm0 = xn0; xm1 = xn1; f_mid = f_next; leftlarger = 1;
                            } else {
                                alpha_left = alpha_next; leftlarger = 0;
                            }
                        } else {
                            if (f_next < f_mid) {
                                alpha_left = alpha_mid; alpha_mid = alpha_next;
                                xm0 = xn0; xm1 = xn1; f_mid = f_next; leftlarger = 0;
                            } else {
                                alpha_right = alpha_next; leftlarger = 1;
                            }
                        }
                    }
                    pcf.y = xm0;
                    pcf.z = xm1;
                }
            }
        }
        const v3 p_wf = m3_mulv(cf, pcf);
        delta_max = fmax(delta_max, maxabs3(sub(h->p, p_wf)));
        h->p = p_wf;
        hc_apply(bp, B, h, h->p, 1.0);
    }
    return delta_max;
}

/* r_ub of the generalized maximum dissipation search (HCSITS.h:2890-2895) */
static inline double gmd_radius(const hc_contact *h, double gn, double a3, double alpha,
                                double shiftI) {
    double r = h->mu * (-gn) / (h->D.m[0] + h->mu * a3 * cos(alpha + shiftI));
    if (r < 0.0) r = INFINITY;
    return r;
}

/* HardContactSemiImplicitTimesteppingSolvers.h:2745-3055: friction by the generalized maximum
 * dissipation principle: the tangential impulse minimising the kinetic energy on the
 * intersection of the plane of maximum compression with the friction cone, by a golden-section
 * search over the angle */
static double relax_gmd(const body_props *bp, hc_bodies *B, hc_contact *C, int64_t nc,
                        double dtinv) {
    double delta_max = 0.0;
    for (int64_t i = 0; i < nc; ++i) {
        hc_contact *h = &C[i];
        hc_apply(bp, B, h, h->p, -1.0);
        const v3 gdot = hc_gdot(B, h);
        const m3 cf = m3_cols(h->n, h->t, h->o);
        v3 g = m3_mulv(m3_trans(cf), gdot);
        g.x += h->dist * dtinv;
        if (g.x >= 0.0) {
            delta_max = fmax(delta_max, maxabs3(h->p));
            h->p = mk(0.0, 0.0, 0.0);
            continue;
        }
        v3 pcf = neg(m3_mulv(h->Dinv, g));
        const double flimit = h->mu * pcf.x;
        const double fsq = pcf.y * pcf.y + pcf.z * pcf.z;
        if (fsq > flimit * flimit || pcf.x < 0.0) {
            const double *D = h->D.m;
            const double invA_nn = 1.0 / D[0];
            const double offdiag = D[5] - invA_nn * D[1] * D[2];
            const double A00 = D[4] - invA_nn * (D[1] * D[1]), A01 = offdiag, A10 = offdiag;
            const double A11 = D[8] - invA_nn * (D[2] * D[2]);
            const double bb0 = -g.y + invA_nn * D[1] * g.x, bb1 = -g.z + invA_nn * D[2] * g.x;
            const double shiftI = atan2(-D[2], D[1]);
            const double shiftJ = atan2(-pcf.z, pcf.y);
            const double a3 = sqrt(D[1] * D[1] + D[2] * D[2]);
            const double fractionI = -D[0] / (h->mu * a3);
            const double fractionJ =
                fmin(invA_nn * h->mu * ((-g.x) / sqrt(fsq) - a3 * cos(shiftI - shiftJ)), 1.0);
            double alpha_left, alpha_right;
            if (fractionJ < -1.0) {
                const double angleI = acos(fractionI);
                alpha_left = -angleI - shiftI;
                alpha_right = +angleI - shiftI;
                if (alpha_left < 0.0) {
                    alpha_left += 2 * M_PI;
                    alpha_right += 2 * M_PI;
                }
            } else if (D[0] > h->mu * a3) {
                const double angleJ = acos(fractionJ);
                alpha_left = -angleJ - shiftJ;
                alpha_right = +angleJ - shiftJ;
                if (alpha_left < 0.0) {
                    alpha_left += 2 * M_PI;
                    alpha_right += 2 * M_PI;
                }
            } else {
                const double angleJ = acos(fractionJ);
                double a1l = -angleJ - shiftJ, a1r = +angleJ - shiftJ;
                if (a1l < 0.0) { a1l += 2 * M_PI; a1r += 2 * M_PI; }
                const double angleI = acos(fractionI);
                double a2l = -angleI - shiftI, a2r = +angleI - shiftI;
                if (a2l < 0.0) { a2l += 2 * M_PI; a2r += 2 * M_PI; }
                if (a1l > a2l) {
                    double t0 = a1l; a1l = a2l; a2l = t0;
                    t0 = a1r; a1r = a2r; a2r = t0;
                }
                if (a2l > a1r) {
                    a2r -= 2 * M_PI;
                    if (!(a2r > a1r)) a1r = a2r;
                } else {
                    a1l = a2l;
                    if (!(a2r > a1r)) a1r = a2r;
                }
                alpha_left = a1l;
                alpha_right = a1r;
            }
            const double phi = 0.5 * (1.0 + sqrt(5.0));
            double alpha_mid = (alpha_right + alpha_left * phi) / (1.0 + phi);
            double r = gmd_radius(h, g.x, a3, alpha_mid, shiftI);
            double xm0 = r * cos(alpha_mid), xm1 = r * sin(alpha_mid);
            double f_mid = quad2(A00, A01, A10, A11, xm0, xm1, bb0, bb1);
            int leftlarger = 0;
            for (int k = 0; k < 20; ++k) {
                const double alpha_next = alpha_left + (alpha_right - alpha_mid);
                r = gmd_radius(h, g.x, a3, alpha_next, shiftI);
                const double xn0 = r * cos(alpha_next), xn1 = r * sin(alpha_next);
                const double f_next = quad2(A00, A01, A10, A11, xn0, xn1, bb0, bb1);
                if (leftlarger) {
                    if (f_next < f_mid) {
                        alpha_right = alpha_mid; alpha_mid = alpha_next;
                        xm0 = xn0; xm1 = xn1; f_mid = f_next; leftlarger = 1;
                    } else {
                        alpha_left = alpha_next; leftlarger = 0;
                    }
                } else {
                    if (f_next < f_mid) {
                        alpha_left = alpha_mid; alpha_mid = alpha_next;
                        xm0 = xn0; xm1 = xn1; f_mid = f_next; leftlarger = 0;
                    } else {
                        alpha_right = alpha_next; leftlarger = 1;
                    }
                }
            }
            {
                const double alpha_init = atan2(pcf.z, pcf.y);
                r = gmd_radius(h, g.x, a3, alpha_init, shiftI);
                const double xi0 = r * cos(alpha_init), xi1 = r * sin(alpha_init);
                const double f_init = quad2(A00, A01, A10, A11, xi0, xi1, bb0, bb1);
                if (f_init < f_mid) {
                    xm0 = xi0;
                    xm1 = xi1;
                }
            }
            pcf.x = invA_nn * (-g.x - D[1] * xm0 - D[2] * xm1);
            pcf.y = xm0;
            pcf.z = xm1;
        }
        const v3 p_wf = m3_mulv(cf, pcf);
        delta_max = fmax(delta_max, maxabs3(sub(h->p, p_wf)));
        h->p = p_wf;
        hc_apply(bp, B, h, h->p, 1.0);
    }
    return delta_max;
}

/* Complementarity residual of the final impulses, in velocity units (max over contacts):
 *   normal:   |min(p_n * D_nn, gdot_n)|                (0 <= p_n  _|_  gdot_n >= 0)
 *   cone:     max(0, |p_to| - mu p_n) * D_nn           (|p_to| <= mu p_n)
 *   friction: inside the cone the slip |gdot_to| must vanish; on the cone the impulse must
 *             oppose the slip: |gdot_to| + p_to.gdot_to/|p_to| = 0.
 * Frictionless contacts use the normal term only. */
static double hc_residual(const hc_bodies *B, const hc_contact *C, int64_t nc, double dtinv,
                          int friction) {
    double res = 0.0;
    for (int64_t i = 0; i < nc; ++i) {
        const hc_contact *h = &C[i];
        const v3 gdot = hc_gdot(B, h);
        const double gn = dot(h->n, gdot) + h->dist * dtinv;
        const double pn = dot(h->n, h->p);
        const double Dnn = h->D.m[0];
        res = fmax(res, fabs(fmin(pn * Dnn, gn)));
        if (!friction) continue;
        const double pt = dot(h->t, h->p), po = dot(h->o, h->p);
        const double gt = dot(h->t, gdot), go = dot(h->o, gdot);
        const double pto = sqrt(pt * pt + po * po), gto = sqrt(gt * gt + go * go);
        res = fmax(res, fmax(0.0, pto - h->mu * pn) * Dnn);
        if (pn <= 0.0) continue;
        if (pto < h->mu * pn * (1.0 - 1e-9)) res = fmax(res, gto);
        else if (pto > 0.0) res = fmax(res, gto + (pt * gt + po * go) / pto);
    }
    return res;
}

static int64_t hcsits_run(pe_or_world *w, double dt, int model, int max_iter, double erp,
                          const pe_or_contact *cl, int64_t nc, double *delta_out,
                          double *resid_out) {
    body_props bp;
    if (body_props_init(w, &bp) != 0) { body_props_free(&bp); return -1; }
    hc_contact *C = (hc_contact *)malloc((size_t)(nc > 0 ? nc : 1) * sizeof(hc_contact));
    hc_bodies B;
    B.v = (v3 *)calloc((size_t)bp.nb, sizeof(v3));
    B.w = (v3 *)calloc((size_t)bp.nb, sizeof(v3));
    B.dv = (v3 *)calloc((size_t)bp.nb, sizeof(v3));
    B.dw = (v3 *)calloc((size_t)bp.nb, sizeof(v3));
    if (!C || !B.v || !B.w || !B.dv || !B.dw) {
        free(C); free(B.v); free(B.w); free(B.dv); free(B.dw); body_props_free(&bp);
        return -1;
    }
    for (int64_t k = 0; k < nc; ++k) hc_cache(w, &bp, &cl[k], erp, &C[k]);
    /* body cache, HardContactSemiImplicitTimesteppingSolvers.h:1834-1880 and 4094-4110: the
     * force accumulators are zero in a step without force generators, so dv = dw = 0 */
    const v3 g = mk(w->gravity[0], w->gravity[1], w->gravity[2]);
    for (int64_t i = 0; i < w->n; ++i) {
        const v3 v = ld3(w->v + 3 * i), om = ld3(w->w + 3 * i);
        B.v[i] = add(v, mul(g, dt));
        const v3 Iw = smul(bp.I[i], om);
        B.w[i] = add(om, smul(dt, smul(bp.ii[i], cross(Iw, om))));
    }
    for (int32_t m = 0; m < w->nmboxes; ++m) {
        const int64_t b = bp.mbase + m;
        const v3 v = ld3(w->mb_v + 3 * m), om = ld3(w->mb_w + 3 * m);
        B.v[b] = add(v, mul(g, dt));
        B.w[b] = add(om, smul(dt, m3_mulv(bp.Iinv_w[m], cross(m3_mulv(bp.I_w[m], om), om))));
    }
    const double dtinv = 1.0 / dt;
    double delta = 0.0;
    for (int it = 0; it < max_iter; ++it) {
        /* the switch of HardContactSemiImplicitTimesteppingSolvers.h:1900-1926 */
        switch (model) {
            case PE_OR_FRICTIONLESS: delta = relax_frictionless(&bp, &B, C, nc, dtinv); break;
            case PE_OR_APPROX_COULOMB_DECOUPLING: delta = relax_approx_coulomb(&bp, &B, C, nc, dtinv); break;
            case PE_OR_APPROX_COULOMB_ORTHOGONAL: delta = relax_orthogonal(&bp, &B, C, nc, dtinv, 1); break;
            case PE_OR_COULOMB_DECOUPLING: delta = relax_coulomb_decoupling(&bp, &B, C, nc, dtinv); break;
            case PE_OR_COULOMB_ORTHOGONAL: delta = relax_orthogonal(&bp, &B, C, nc, dtinv, 0); break;
            default: delta = relax_gmd(&bp, &B, C, nc, dtinv); break;
        }
    }
    if (delta_out) *delta_out = delta;
    if (resid_out) *resid_out = hc_residual(&B, C, nc, dtinv, model != PE_OR_FRICTIONLESS);
    /* integratePositions, HardContactSemiImplicitTimesteppingSolvers.h:4135-4190 */
    for (int64_t i = 0; i < w->n; ++i) {
        v3 v = add(B.v[i], B.dv[i]), om = add(B.w[i], B.dw[i]);
        st3(w->x + 3 * i, add(ld3(w->x + 3 * i), mul(v, dt)));
        if (w->q) quat_update(w->q + 4 * i, mul(om, dt));
        if (w->damping < 1.0) {
            const double drag = pow(w->damping, dt);
            v = mul(v, drag);
            om = mul(om, drag);
        }
        st3(w->v + 3 * i, v);
        st3(w->w + 3 * i, om);
    }
    for (int32_t m = 0; m < w->nmboxes; ++m) {
        const int64_t b = bp.mbase + m;
        v3 v = add(B.v[b], B.dv[b]), om = add(B.w[b], B.dw[b]);
        st3(w->mb_x + 3 * m, add(ld3(w->mb_x + 3 * m), mul(v, dt)));
        quat_update(w->mb_q + 4 * m, mul(om, dt));
        if (w->damping < 1.0) {
            const double drag = pow(w->damping, dt);
            v = mul(v, drag);
            om = mul(om, drag);
        }
        st3(w->mb_v + 3 * m, v);
        st3(w->mb_w + 3 * m, om);
    }
    free(C); free(B.v); free(B.w); free(B.dv); free(B.dw); body_props_free(&bp);
    return nc;
}

int64_t pe_or_hcsits_step_contacts(pe_or_world *w, double dt, int model, int max_iter,
                                   double erp, const pe_or_contact *contacts, int64_t nc,
                                   double *delta_out, double *resid_out) {
    if (dt <= 0.0 || model < PE_OR_FRICTIONLESS || model > PE_OR_GENERALIZED_MAX_DISSIPATION)
        return -2;
    return hcsits_run(w, dt, model, max_iter, erp, contacts, nc, delta_out, resid_out);
}

int64_t pe_or_hcsits_step(pe_or_world *w, double dt, int model, int max_iter, double erp,
                          const int64_t *order, int64_t norder, double *delta_out,
                          double *resid_out) {
    if (dt <= 0.0 || model < PE_OR_FRICTIONLESS || model > PE_OR_GENERALIZED_MAX_DISSIPATION)
        return -2;
    clist l;
    if (find_contacts_list(w, &l) != 0) return -1;
    int64_t rc;
    if (order) {
        if (norder != l.n) { free(l.c); return -2; }
        pe_or_contact *perm = (pe_or_contact *)malloc((size_t)(l.n > 0 ? l.n : 1) *
                                                      sizeof(pe_or_contact));
        if (!perm) { free(l.c); return -1; }
        for (int64_t k = 0; k < l.n; ++k) {
            if (order[k] < 0 || order[k] >= l.n) { free(perm); free(l.c); return -2; }
            perm[k] = l.c[order[k]];
        }
        rc = hcsits_run(w, dt, model, max_iter, erp, perm, l.n, delta_out, resid_out);
        free(perm);
    } else {
        rc = hcsits_run(w, dt, model, max_iter, erp, l.c, l.n, delta_out, resid_out);
    }
    free(l.c);
    return rc;
}
