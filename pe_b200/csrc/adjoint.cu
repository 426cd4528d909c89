// adjoint.cu -- reverse-mode gradient of the FP64 DEM step (pe has no gradients; this extends the
// path): d loss / d (initial x, v, w) and d loss / d (k_n, c_n, c_t, mu).
//
// The forward map of one step is the grid-search DEM step of dem.cu (pe's linear law and
// semi-implicit Euler, DEMSolver.h:328-379, spheretrait/Default.h:149-220):
//     F_i = sum_c f_c(x, v, w; theta),  T_i = sum_c r_c x f_c
//     v+ = (v + (F/m + g) dt) drag,  x+ = x + (v + (F/m + g) dt) dt,  w+ = (w + I^-1 T dt) drag
// Its vector-Jacobian product, for post-step adjoints (lx+, lv+, lw+):
//     u = lv+ drag + lx+ dt                  (adjoint of the pre-drag velocity)
//     Fbar = u dt / m,  Tbar = lw+ drag I^-1 dt
//     lx = lx+ + sum_c d s_c / dx,  lv = u + sum_c d s_c / dv,  lw = lw+ drag + sum_c d s_c / dw
// with s_c = Fbar_1.f_1 + Tbar_1.tau_1 + Fbar_2.f_2 + Tbar_2.tau_2 for contact c.  Each thread
// owns one body and gathers d s_c over its contacts; the local derivatives of a contact are exact,
// evaluated with forward-mode dual numbers seeded on the body's own 9 state components and the 4
// contact parameters (the latter only once per contact).  Kinks of the law (max(0, .), the
// Coulomb min, contact onset) take the branch the forward step took.
//
// Memory: the forward run keeps a checkpoint every K steps; the backward pass recomputes each
// segment from its checkpoint, keeping the K pre-step states, and runs the adjoint steps in
// reverse.  Adjoints are stored by upload index, so the grid re-sorting of the state between
// steps does not matter.
#include <algorithm>
#include <vector>

#include "internal.cuh"

namespace peb {

namespace {

constexpr int ND = 13;  // x(3) v(3) w(3) k_n c_n c_t mu

struct Dual {
    double v;
    double d[ND];
    __device__ Dual() {}
    __device__ Dual(double a) : v(a) {
#pragma unroll
        for (int k = 0; k < ND; ++k) d[k] = 0.0;
    }
};

__device__ __forceinline__ Dual operator+(const Dual &a, const Dual &b) {
    Dual r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
__device__ __forceinline__ Dual operator-(const Dual &a, const Dual &b) {
    Dual r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
__device__ __forceinline__ Dual operator-(const Dual &a) {
    Dual r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < ND; ++k) r.d[k] = -a.d[k];
    return r;
}
__device__ __forceinline__ Dual operator*(const Dual &a, const Dual &b) {
    Dual r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
__device__ __forceinline__ Dual operator/(const Dual &a, const Dual &b) {
    Dual r;
    r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
#pragma unroll
    for (int k = 0; k < ND; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}
__device__ __forceinline__ Dual dsqrt(const Dual &a) {
    Dual r;
    r.v = sqrt(a.v);
    const double h = r.v > 0.0 ? 0.5 / r.v : 0.0;
#pragma unroll
    for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] * h;
    return r;
}

typedef V3<Dual> VD;

__device__ __forceinline__ VD vd(const V3<double> &a) { return v3(Dual(a.x), Dual(a.y), Dual(a.z)); }
__device__ __forceinline__ VD seeded(const V3<double> &a, int first) {
    VD r = vd(a);
    r.x.d[first] = 1.0;
    r.y.d[first + 1] = 1.0;
    r.z.d[first + 2] = 1.0;
    return r;
}
__device__ __forceinline__ Dual ddot(const VD &a, const VD &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ VD dcross(const VD &a, const VD &b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ VD dscale(const VD &a, const Dual &s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ VD dadd(const VD &a, const VD &b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ VD dsub(const VD &a, const VD &b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ Dual dvdot(const V3<double> &a, const VD &b) {
    return Dual(a.x) * b.x + Dual(a.y) * b.y + Dual(a.z) * b.z;
}

struct Params {
    Dual k, cn, ct, mu;
};

// pe's contact law (response/DEMSolver.h:328-379) on dual numbers: force on body 1
__device__ VD law(const VD &n, const Dual &dist, const VD &rvel, const Params &p) {
    const Dual delta = -dist;
    const Dual nvel = ddot(n, rvel);
    const Dual relVelN = -nvel;
    const VD relVelT = dadd(v3(-rvel.x, -rvel.y, -rvel.z), dscale(n, nvel));
    Dual fN = p.k * delta + p.cn * relVelN;
    if (fN.v < 0.0) fN = Dual(0.0);
    const VD fNv = dscale(n, fN);
    const Dual tl = dsqrt(ddot(relVelT, relVelT));
    if (tl.v == 0.0) return fNv;  // Vector3::getNormalized leaves a zero vector unchanged
    const Dual a = p.ct * tl, b = p.mu * fN;
    const Dual fT = (a.v < b.v) ? a : b;
    const VD tdir = v3(relVelT.x / tl, relVelT.y / tl, relVelT.z / tl);
    return dadd(fNv, dscale(tdir, fT));
}

struct AdjArgs {
    int64_t n;
    double dt, drag;
    const int32_t *sorted, *cell_start;
    const SceneInfo *scenes;
    const MatDev *mats;
    const double4 *planes;
    const int32_t *plane_mat;
    const double *boxes;
    const int32_t *box_mat;
    const double4 *pr;
    const double *vw;
    const uint32_t *tag;
    const int32_t *uid;
    const double *lx1, *lv1, *lw1;  // post-step adjoints by upload index (3n each)
    double *lx0, *lv0, *lw0;        // pre-step adjoints
    double *gpar;                   // per-block partial parameter gradients (4 per block)
};

__device__ __forceinline__ V3<double> ld3u(const double *a, int64_t u) {
    return v3(a[3 * u], a[3 * u + 1], a[3 * u + 2]);
}

// Fbar, Tbar of a body from its post-step adjoints
__device__ __forceinline__ void body_bars(const AdjArgs &a, int64_t u, double r, double density,
                                          V3<double> &Fb, V3<double> &Tb, V3<double> &uvel) {
    double im, ii, I;
    sphere_mass(r, density, im, ii, I);
    const V3<double> lx = ld3u(a.lx1, u), lv = ld3u(a.lv1, u), lw = ld3u(a.lw1, u);
    uvel = lv * a.drag + lx * a.dt;
    Fb = uvel * (a.dt * im);
    Tb = lw * (a.drag * ii * a.dt);
}

__global__ void __launch_bounds__(128) k_adjoint(AdjArgs a) {
    __shared__ double s_par[4][128];
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double gp[4] = {0.0, 0.0, 0.0, 0.0};
    if (t < a.n) {
        const int32_t b = a.sorted[t];
        const double4 pi = a.pr[b];
        const uint32_t tagi = a.tag[b];
        const int64_t ui = a.uid[b];
        const SceneInfo &s = a.scenes[tagi >> 16];
        const MatDev &mi = a.mats[tagi & 0xffffu];
        const V3<double> xi = v3(pi.x, pi.y, pi.z);
        const V3<double> vi = ld_vw(a.vw, a.n, b, 0), wi = ld_vw(a.vw, a.n, b, 1);
        V3<double> Fbi, Tbi, ui_vel;
        body_bars(a, ui, pi.w, mi.density, Fbi, Tbi, ui_vel);
        V3<double> gx = v3(0.0, 0.0, 0.0), gv = gx, gw = gx;
        const VD Xi = seeded(xi, 0), Vi = seeded(vi, 3), Wi = seeded(wi, 6);
        auto accumulate = [&](const Dual &sc, bool params) {
            gx = gx + v3(sc.d[0], sc.d[1], sc.d[2]);
            gv = gv + v3(sc.d[3], sc.d[4], sc.d[5]);
            gw = gw + v3(sc.d[6], sc.d[7], sc.d[8]);
            if (params)
                for (int k = 0; k < 4; ++k) gp[k] += sc.d[9 + k];
        };
        auto params_of = [&](const MatDev &m1, const MatDev &m2, bool seed, double tvel) {
            Params p;
            p.k = Dual(1.0 / (m1.rk + m2.rk));
            p.cn = Dual(1.0 / (m1.rcn + m2.rcn));
            p.ct = Dual(1.0 / (m1.rct + m2.rct));
            p.mu = Dual(fabs(tvel) > kFrictionThreshold ? m1.cdf + m2.cdf : m1.csf + m2.csf);
            if (seed) {
                p.k.d[9] = 1.0;
                p.cn.d[10] = 1.0;
                p.ct.d[11] = 1.0;
                p.mu.d[12] = 1.0;
            }
            return p;
        };
        // sphere pairs (grid neighbours, same predicate as the forward step)
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
                    const int64_t uj = a.uid[j];
                    const bool self1 = ui < uj;
                    const double4 p1 = self1 ? pi : pj, p2 = self1 ? pj : pi;
                    const double nx = p1.x - p2.x, ny = p1.y - p2.y, nz = p1.z - p2.z;
                    const double len = length_rn(nx, ny, nz);
                    const double dist = __dsub_rn(__dsub_rn(len, p1.w), p2.w);
                    if (!(dist < -kContactThreshold)) continue;
                    const MatDev &mj = a.mats[a.tag[j] & 0xffffu];
                    const V3<double> xj = v3(pj.x, pj.y, pj.z);
                    const V3<double> vj = ld_vw(a.vw, a.n, j, 0), wj = ld_vw(a.vw, a.n, j, 1);
                    V3<double> Fbj, Tbj, uj_vel;
                    body_bars(a, uj, pj.w, mj.density, Fbj, Tbj, uj_vel);
                    // pe orientation: 1 = smaller id; this body's state carries the seeds
                    const VD X1 = self1 ? Xi : vd(xj), X2 = self1 ? vd(xj) : Xi;
                    const VD V1 = self1 ? Vi : vd(vj), V2 = self1 ? vd(vj) : Vi;
                    const VD W1 = self1 ? Wi : vd(wj), W2 = self1 ? vd(wj) : Wi;
                    const double r1 = p1.w, r2 = p2.w;
                    const VD dd = dsub(X1, X2);
                    const Dual L = dsqrt(ddot(dd, dd));
                    const Dual Dist = (L - Dual(r1)) - Dual(r2);
                    const VD n = v3(dd.x / L, dd.y / L, dd.z / L);
                    const Dual kk = Dual(r2) + Dual(0.5) * Dist;
                    const VD gpos = dadd(X2, dscale(n, kk));
                    const VD R1 = dsub(gpos, X1), R2 = dsub(gpos, X2);
                    const VD rvel = dsub(dadd(V1, dcross(W1, R1)), dadd(V2, dcross(W2, R2)));
                    // friction pick on the forward values (Contact.cpp:102-105)
                    const V3<double> nv = v3(n.x.v, n.y.v, n.z.v), rv = v3(rvel.x.v, rvel.y.v, rvel.z.v);
                    const double tvel = dot(nv, rv - nv * dot(nv, rv));
                    const Params P = self1 ? params_of(mi, mj, true, tvel) : params_of(mj, mi, false, tvel);
                    const VD f1 = law(n, Dist, rvel, P);
                    const VD t1 = dcross(R1, f1), t2 = dcross(R2, v3(-f1.x, -f1.y, -f1.z));
                    const V3<double> Fb1 = self1 ? Fbi : Fbj, Tb1 = self1 ? Tbi : Tbj;
                    const V3<double> Fb2 = self1 ? Fbj : Fbi, Tb2 = self1 ? Tbj : Tbi;
                    const Dual sc = dvdot(Fb1, f1) + dvdot(Tb1, t1) - dvdot(Fb2, f1) + dvdot(Tb2, t2);
                    accumulate(sc, self1);
                }
            }
        }
        // walls: the sphere is body 1 and the wall does not move
        const VD zero = vd(v3(0.0, 0.0, 0.0));
        for (int p = 0; p < s.nplanes; ++p) {
            const double4 pl = a.planes[s.plane_begin + p];
            const double kd = dot_rn(pl.x, pl.y, pl.z, pi.x, pi.y, pi.z);
            const double dist = __dsub_rn(__dsub_rn(kd, pi.w), pl.w);
            if (!(dist < -kContactThreshold)) continue;
            const MatDev &mw = a.mats[a.plane_mat[s.plane_begin + p]];
            const VD n = vd(v3(pl.x, pl.y, pl.z));
            const Dual Dist = (ddot(n, Xi) - Dual(pi.w)) - Dual(pl.w);
            const VD gpos = dsub(Xi, dscale(n, Dual(pi.w) + Dist));
            const VD R1 = dsub(gpos, Xi);
            const VD rvel = dadd(Vi, dcross(Wi, R1));
            const V3<double> nv = v3(pl.x, pl.y, pl.z), rv = v3(rvel.x.v, rvel.y.v, rvel.z.v);
            const double tvel = dot(nv, rv - nv * dot(nv, rv));
            const Params P = params_of(mi, mw, true, tvel);
            const VD f1 = law(n, Dist, rvel, P);
            const Dual sc = dvdot(Fbi, f1) + dvdot(Tbi, dcross(R1, f1));
            accumulate(sc, true);
        }
        for (int k = 0; k < s.nboxes; ++k) {
            const double *B = a.boxes + 15 * (int64_t)(s.box_begin + k);
            const double *R = B + 6;
            const double l[3] = {0.5 * B[3], 0.5 * B[4], 0.5 * B[5]};
            const VD D = dsub(Xi, vd(v3(B[0], B[1], B[2])));
            Dual p[3] = {D.x * Dual(R[0]) + D.y * Dual(R[3]) + D.z * Dual(R[6]),
                         D.x * Dual(R[1]) + D.y * Dual(R[4]) + D.z * Dual(R[7]),
                         D.x * Dual(R[2]) + D.y * Dual(R[5]) + D.z * Dual(R[8])};
            bool outside = false;
            for (int ax = 0; ax < 3; ++ax) {
                if (p[ax].v < -l[ax]) { p[ax] = Dual(-l[ax]); outside = true; }
                else if (p[ax].v > l[ax]) { p[ax] = Dual(l[ax]); outside = true; }
            }
            VD n, gpos;
            Dual Dist;
            if (!outside) {
                double dmax = fabs(p[0].v) - l[0];
                int face = 0;
                for (int ax = 1; ax < 3; ++ax) {
                    const double tmp = fabs(p[ax].v) - l[ax];
                    if (dmax < tmp) { dmax = tmp; face = ax; }
                }
                const double sg = (p[face].v > 0.0) ? 1.0 : -1.0;
                n = vd(v3(R[face] * sg, R[3 + face] * sg, R[6 + face] * sg));
                Dist = (p[face] * Dual(sg) - Dual(l[face])) - Dual(pi.w);
                gpos = Xi;
            } else {
                const VD q = v3(Dual(R[0]) * p[0] + Dual(R[1]) * p[1] + Dual(R[2]) * p[2],
                                Dual(R[3]) * p[0] + Dual(R[4]) * p[1] + Dual(R[5]) * p[2],
                                Dual(R[6]) * p[0] + Dual(R[7]) * p[1] + Dual(R[8]) * p[2]);
                const VD m = dsub(D, q);
                const Dual L = dsqrt(ddot(m, m));
                Dist = L - Dual(pi.w);
                n = v3(m.x / L, m.y / L, m.z / L);
                gpos = dadd(vd(v3(B[0], B[1], B[2])), q);
            }
            if (!(Dist.v < -kContactThreshold)) continue;
            const MatDev &mw = a.mats[a.box_mat[s.box_begin + k]];
            const VD R1 = dsub(gpos, Xi);
            const VD rvel = dadd(Vi, dcross(Wi, R1));
            const V3<double> nv = v3(n.x.v, n.y.v, n.z.v), rv = v3(rvel.x.v, rvel.y.v, rvel.z.v);
            const double tvel = dot(nv, rv - nv * dot(nv, rv));
            const Params P = params_of(mi, mw, true, tvel);
            const VD f1 = law(n, Dist, rvel, P);
            const Dual sc = dvdot(Fbi, f1) + dvdot(Tbi, dcross(R1, f1));
            accumulate(sc, true);
        }
        (void)zero;
        const V3<double> lx = ld3u(a.lx1, ui), lw = ld3u(a.lw1, ui);
        const V3<double> ox = lx + gx, ov = ui_vel + gv, ow = lw * a.drag + gw;
        a.lx0[3 * ui] = ox.x; a.lx0[3 * ui + 1] = ox.y; a.lx0[3 * ui + 2] = ox.z;
        a.lv0[3 * ui] = ov.x; a.lv0[3 * ui + 1] = ov.y; a.lv0[3 * ui + 2] = ov.z;
        a.lw0[3 * ui] = ow.x; a.lw0[3 * ui + 1] = ow.y; a.lw0[3 * ui + 2] = ow.z;
    }
    // deterministic per-block parameter partials
    for (int k = 0; k < 4; ++k) s_par[k][threadIdx.x] = gp[k];
    __syncthreads();
    if (threadIdx.x < 4) {
        double acc = 0.0;
        for (int i = 0; i < blockDim.x; ++i) acc += s_par[threadIdx.x][i];
        a.gpar[4 * blockIdx.x + threadIdx.x] += acc;
    }
}

void free_ckpt(Ctx *c, BodyBuf &b) {
    dfree(c, b.pr);
    dfree(c, b.vw);
    dfree(c, b.tag);
    dfree(c, b.uid);
    b = BodyBuf();
}

int alloc_ckpt(Ctx *c, BodyBuf &b) {
    const size_t n = (size_t)std::max<int64_t>(c->n, 1);
    PEB_CUDA(c, dmalloc(c, &b.pr, n * sizeof(double4)));
    PEB_CUDA(c, dmalloc(c, &b.vw, n * (size_t)c->vw_bytes));
    PEB_CUDA(c, dmalloc(c, &b.tag, n * sizeof(uint32_t)));
    PEB_CUDA(c, dmalloc(c, &b.uid, n * sizeof(int32_t)));
    return PE_B200_OK;
}

int copy_state(Ctx *c, BodyBuf &dst, const BodyBuf &src) {
    const size_t n = (size_t)c->n;
    PEB_CUDA(c, cudaMemcpyAsync(dst.pr, src.pr, n * sizeof(double4), cudaMemcpyDeviceToDevice, c->stream));
    PEB_CUDA(c, cudaMemcpyAsync(dst.vw, src.vw, n * (size_t)c->vw_bytes, cudaMemcpyDeviceToDevice, c->stream));
    PEB_CUDA(c, cudaMemcpyAsync(dst.tag, src.tag, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, c->stream));
    PEB_CUDA(c, cudaMemcpyAsync(dst.uid, src.uid, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, c->stream));
    return PE_B200_OK;
}

// one grid-search FP64 step (the map the adjoint differentiates), from whatever state cur holds
int plain_step(Ctx *c, double dt) {
    c->binned = false;
    return dem_step(c, dt);
}

}  // namespace

void adjoint_free(Ctx *c) {
    for (auto &b : c->adj.ckpt) free_ckpt(c, b);
    for (auto &b : c->adj.seg) free_ckpt(c, b);
    c->adj.ckpt.clear();
    c->adj.seg.clear();
    c->adj.nsteps = 0;
}

int adjoint_forward(Ctx *c, int32_t nsteps, double dt, int32_t every) {
    if (c->p.solver != PE_B200_DEM || c->p.precision != PE_B200_FP64 || c->p.track_orientation ||
        c->p.force_model != 0)
        return set_err(c, PE_B200_ERR_UNSUPPORTED,
                       "the adjoint needs the linear DEM law in FP64 without orientation tracking");
    if (nsteps < 1 || every < 1 || !(dt > 0.0)) return PE_B200_ERR_ARG;
    adjoint_free(c);
    AdjState &A = c->adj;
    A.nsteps = nsteps;
    A.every = every;
    A.dt = dt;
    const int nck = (nsteps + every - 1) / every;
    A.ckpt.resize(nck);
    for (int k = 0; k < nck; ++k) {
        int rc = alloc_ckpt(c, A.ckpt[k]);
        if (rc) return rc;
    }
    for (int s = 0; s < nsteps; ++s) {
        if (s % every == 0) {
            int rc = copy_state(c, A.ckpt[s / every], c->cur);
            if (rc) return rc;
        }
        int rc = plain_step(c, dt);
        if (rc) return rc;
    }
    if (c->nl.enabled) return dem_list_request_rebuild(c);
    return PE_B200_OK;
}

int adjoint_backward(Ctx *c, const double *gx, const double *gv, const double *gw, double *ox,
                     double *ov, double *ow, double *gpar) {
    AdjState &A = c->adj;
    if (A.nsteps < 1 || A.ckpt.empty())
        return set_err(c, PE_B200_ERR_STATE, "run pe_b200_adjoint_forward first");
    const int64_t n = c->n;
    const size_t vb = 3 * (size_t)n * sizeof(double);
    double *l[6] = {};
    double *d_gpar = nullptr;
    const unsigned blocks = grid_for(n, 128);
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 6 && e == cudaSuccess; ++k) e = dmalloc(c, &l[k], vb);
    if (e == cudaSuccess) e = dmalloc(c, &d_gpar, 4 * sizeof(double) * blocks);
    auto cleanup = [&]() {
        for (int k = 0; k < 6; ++k) dfree(c, l[k]);
        dfree(c, d_gpar);
    };
    if (e != cudaSuccess) {
        cleanup();
        return cuda_err(c, e, "adjoint buffers");
    }
    // post-final adjoints (upload order)
    PEB_CUDA(c, cudaMemcpyAsync(l[0], gx, vb, cudaMemcpyHostToDevice, c->stream));
    PEB_CUDA(c, cudaMemcpyAsync(l[1], gv, vb, cudaMemcpyHostToDevice, c->stream));
    PEB_CUDA(c, cudaMemcpyAsync(l[2], gw, vb, cudaMemcpyHostToDevice, c->stream));
    PEB_CUDA(c, cudaMemsetAsync(d_gpar, 0, 4 * sizeof(double) * blocks, c->stream));
    // keep the final state: the backward pass overwrites cur while recomputing
    BodyBuf final_state;
    int rc = alloc_ckpt(c, final_state);
    if (!rc) rc = copy_state(c, final_state, c->cur);
    if (A.seg.size() < (size_t)A.every) {
        const size_t old = A.seg.size();
        A.seg.resize(A.every);
        for (size_t k = old; k < A.seg.size() && !rc; ++k) rc = alloc_ckpt(c, A.seg[k]);
    }
    int cur_l = 0;  // l[cur_l..cur_l+2] hold the post-step adjoints
    const int nck = (int)A.ckpt.size();
    for (int seg = nck - 1; seg >= 0 && !rc; --seg) {
        const int s0 = seg * A.every;
        const int s1 = std::min(A.nsteps, s0 + A.every);
        // recompute the segment, keeping every pre-step state
        rc = copy_state(c, c->cur, A.ckpt[seg]);
        for (int s = s0; s < s1 && !rc; ++s) {
            rc = copy_state(c, A.seg[s - s0], c->cur);
            if (!rc && s + 1 < s1) rc = plain_step(c, A.dt);
        }
        for (int s = s1 - 1; s >= s0 && !rc; --s) {
            rc = copy_state(c, c->cur, A.seg[s - s0]);
            if (!rc) rc = grid_bin_current(c);
            if (!rc) rc = grid_sort(c);
            if (rc) break;
            AdjArgs a;
            a.n = n;
            a.dt = A.dt;
            a.drag = c->p.damping < 1.0 ? pow(c->p.damping, A.dt) : 1.0;
            a.sorted = c->sorted;
            a.cell_start = c->cell_start;
            a.scenes = c->d_scenes;
            a.mats = c->d_mats;
            a.planes = c->d_planes;
            a.plane_mat = c->d_plane_mat;
            a.boxes = c->d_boxes;
            a.box_mat = c->d_box_mat;
            a.pr = c->cur.pr;
            a.vw = (const double *)c->cur.vw;
            a.tag = c->cur.tag;
            a.uid = c->cur.uid;
            a.lx1 = l[cur_l];
            a.lv1 = l[cur_l + 1];
            a.lw1 = l[cur_l + 2];
            a.lx0 = l[3 - cur_l];
            a.lv0 = l[4 - cur_l];
            a.lw0 = l[5 - cur_l];
            a.gpar = d_gpar;
            k_adjoint<<<blocks, 128, 0, c->stream>>>(a);
            c->launches++;
            e = cudaGetLastError();
            if (e != cudaSuccess) rc = cuda_err(c, e, "k_adjoint");
            cur_l = 3 - cur_l;
        }
    }
    if (!rc) {
        std::vector<double> hp(4 * (size_t)blocks);
        e = cudaMemcpyAsync(ox, l[cur_l], vb, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(ov, l[cur_l + 1], vb, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(ow, l[cur_l + 2], vb, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hp.data(), d_gpar, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) rc = cuda_err(c, e, "adjoint results");
        for (int k = 0; k < 4 && !rc; ++k) {
            double s = 0.0;
            for (unsigned b = 0; b < blocks; ++b) s += hp[4 * b + k];
            if (gpar) gpar[k] = s;
        }
    }
    // restore the final state
    if (!rc) rc = copy_state(c, c->cur, final_state);
    c->binned = false;
    if (!rc && c->nl.enabled) rc = dem_list_request_rebuild(c);
    cudaStreamSynchronize(c->stream);
    free_ckpt(c, final_state);
    cleanup();
    return rc;
}

}  // namespace peb
