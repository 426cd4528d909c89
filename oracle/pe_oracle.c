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

typedef struct {
    int64_t n, nb;   /* spheres, all bodies */
    double *im;      /* inverse mass per body (walls 0) */
    double *ii;      /* inverse inertia (scalar) per body (walls 0) */
    double *I;       /* inertia (scalar) per body (walls 0) */
    int32_t *bmat;   /* material per body */
    double *bpos;    /* 3 per body: centre (planes: anchor point normal*d) */
} body_props;

static int body_props_init(const pe_or_world *w, body_props *bp) {
    const int64_t nw = (int64_t)w->nplanes + w->nboxes;
    bp->n = w->n;
    bp->nb = w->n + nw;
    bp->im = (double *)calloc((size_t)bp->nb, sizeof(double));
    bp->ii = (double *)calloc((size_t)bp->nb, sizeof(double));
    bp->I = (double *)calloc((size_t)bp->nb, sizeof(double));
    bp->bmat = (int32_t *)calloc((size_t)bp->nb, sizeof(int32_t));
    bp->bpos = (double *)calloc((size_t)bp->nb * 3, sizeof(double));
    if (!bp->im || !bp->ii || !bp->I || !bp->bmat || !bp->bpos) return -1;
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
    return 0;
}

static void body_props_free(body_props *bp) {
    free(bp->im); free(bp->ii); free(bp->I); free(bp->bmat); free(bp->bpos);
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

/* MaxContacts.h:589-668 */
static void collide_sphere_box(const pe_or_world *w, int64_t i, int32_t bi, clist *l) {
    const double *B = w->boxes + 15 * bi;
    const v3 L = mk(0.5 * B[3], 0.5 * B[4], 0.5 * B[5]);
    const double *R = B + 6;
    const v3 spos = ld3(w->x + 3 * i), bpos = ld3(B);
    const int64_t bid = w->n + w->nplanes + bi;
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

static int cmp_contact(const void *a, const void *b) {
    const pe_or_contact *x = (const pe_or_contact *)a, *y = (const pe_or_contact *)b;
    if (x->b1 != y->b1) return x->b1 < y->b1 ? -1 : 1;
    if (x->b2 != y->b2) return x->b2 < y->b2 ? -1 : 1;
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
        for (int32_t b = 0; b < w->nboxes; ++b) collide_sphere_box(w, i, b, l);
    }
    if (l->oom) { free(l->c); return -1; }
    if (l->n > 1) qsort(l->c, (size_t)l->n, sizeof(pe_or_contact), cmp_contact);
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
    if (b >= w->n) return mk(0.0, 0.0, 0.0);
    const v3 v = ld3(w->v + 3 * b), om = ld3(w->w + 3 * b), x = ld3(w->x + 3 * b);
    return add(v, cross(om, sub(gpos, x)));
}

/* RigidBody.h:1775-1803 */
static inline void add_force_at_pos(const pe_or_world *w, double *F, double *T, int64_t b, v3 f,
                                    v3 gpos) {
    if (b >= w->n) return; /* walls are fixed: their accumulated force is never used */
    st3(F + 3 * b, add(ld3(F + 3 * b), f));
    st3(T + 3 * b, add(ld3(T + 3 * b), cross(sub(gpos, ld3(w->x + 3 * b)), f)));
}

static int32_t body_mat(const pe_or_world *w, int64_t b) {
    if (b < w->n) return w->mat[b];
    if (b < w->n + w->nplanes) return w->plane_mat[b - w->n];
    return w->box_mat[b - w->n - w->nplanes];
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
    const contact_params cp = compose(w, body_mat(w, c->b1), body_mat(w, c->b2), n, rvel);
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

/* collisionsystem/DEMSolver.h:1155-1262 + spheretrait/Default.h:149-220 */
int64_t pe_or_dem_step(pe_or_world *w, double dt) {
    clist l;
    if (find_contacts_list(w, &l) != 0) return -1;
    const int64_t n = w->n;
    double *F = (double *)calloc((size_t)(3 * n + 3), sizeof(double));
    double *T = (double *)calloc((size_t)(3 * n + 3), sizeof(double));
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
    const m3 I1 = m3_scaled_identity(bp->ii[c->b1]), I2 = m3_scaled_identity(bp->ii[c->b2]);
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
