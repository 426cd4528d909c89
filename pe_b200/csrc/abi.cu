// abi.cu -- the extern "C" entry points of libpe_b200.so (declared in include/pe_b200.h).
#include <nvtx3/nvToolsExt.h>

#include <cmath>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <new>

#include "internal.cuh"

namespace peb {

unsigned capped_grid(const Ctx *c, int64_t n, int block) {
    const int64_t g = (n + block - 1) / block;
    const int64_t cap = 8 * (int64_t)c->sm_count;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, cap));
}

namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pool[64] = {};
}  // namespace

// The library's pool on `dev`: device memory that contexts free stays reserved (release
// threshold: never) and serves the next allocations, on any of the library's streams.
static cudaError_t lib_pool(int dev, cudaMemPool_t *out) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!g_pool[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        cudaError_t e = cudaMemPoolCreate(&p, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = UINT64_MAX;
        e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(p);
            return e;
        }
        g_pool[dev] = p;
    }
    *out = g_pool[dev];
    return cudaSuccess;
}

cudaError_t dmalloc_bytes(Ctx *c, void **p, size_t bytes) {
    *p = nullptr;
    cudaMemPool_t pool = nullptr;
    cudaError_t e = lib_pool(c->device, &pool);
    if (e != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(p, std::max<size_t>(bytes, 1), pool, c->stream);
}

void dfree(Ctx *c, void *p) {
    if (p) cudaFreeAsync(p, c ? c->stream : nullptr);
}

int set_err(Ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_err(Ctx *c, cudaError_t e, const char *where) {
    char buf[512];
    snprintf(buf, sizeof buf, "CUDA error %d (%s) at %s", (int)e, cudaGetErrorString(e), where);
    // a failed allocation is not sticky: clear it, so the next launch check does not see it
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return set_err(c, PE_B200_ERR_NOMEM, buf);
    }
    return set_err(c, PE_B200_ERR_CUDA, buf);
}

const char *kStageNames[ST_COUNT] = {"sort", "dem_step", "permute", "detect", "color",
                                     "contact_cache", "sweeps", "integrate", "list_rebuild"};

static cudaEvent_t take_event(Ctx *c) {
    if (!c->ev_pool.empty()) {
        cudaEvent_t e = c->ev_pool.back();
        c->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

void prof_begin(Ctx *c, int stage) {
    // NVTX range per stage for timeline tools (host-side only; safe during graph capture)
    nvtxRangePushA(kStageNames[stage]);
    if (!c->prof) return;
    cudaEvent_t e = take_event(c);
    if (!e) return;
    cudaEventRecord(e, c->stream);
    c->ev_pending[stage] = e;
}

void prof_end(Ctx *c, int stage) {
    nvtxRangePop();
    if (!c->prof || !c->ev_pending[stage]) return;
    cudaEvent_t e = take_event(c);
    if (!e) return;
    cudaEventRecord(e, c->stream);
    c->ev_open[stage].push_back({c->ev_pending[stage], e});
    c->ev_pending[stage] = nullptr;
}

static void prof_collect(Ctx *c) {
    cudaStreamSynchronize(c->stream);
    for (int s = 0; s < ST_COUNT; ++s) {
        for (auto &pr : c->ev_open[s]) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) {
                c->prof_ms[s] += ms;
                c->prof_count[s] += 1;
            }
            c->ev_pool.push_back(pr.first);
            c->ev_pool.push_back(pr.second);
        }
        c->ev_open[s].clear();
    }
}

namespace {

void free_bodies(Ctx *c, BodyBuf &b) {
    dfree(c, b.pr);
    dfree(c, b.vw);
    dfree(c, b.tag);
    dfree(c, b.uid);
    dfree(c, b.q);
    b = BodyBuf();
}

void free_device(Ctx *c) {
    free_bodies(c, c->cur);
    free_bodies(c, c->nxt);
    dfree(c, c->key);
    dfree(c, c->rank);
    dfree(c, c->sorted);
    dfree(c, c->cell_count);
    dfree(c, c->cell_start);
    dfree(c, c->scan_tmp);
    dfree(c, c->gs_bar);
    dfree(c, c->gs_blk);
    c->gs_bar = nullptr;
    c->gs_blk = nullptr;
    c->gs_blk_cap = 0;
    dfree(c, c->posf);
    c->posf = nullptr;
    dfree(c, c->near);
    c->near = nullptr;
    dfree(c, c->d_scenes);
    dfree(c, c->d_mats);
    dfree(c, c->d_planes);
    dfree(c, c->d_plane_mat);
    dfree(c, c->d_boxes);
    dfree(c, c->d_box_mat);
    c->key = c->rank = c->sorted = c->cell_count = c->cell_start = c->scan_tmp = nullptr;
    c->scan_tmp_cap = 0;
    c->d_scenes = nullptr;
    c->d_mats = nullptr;
    c->d_planes = nullptr;
    c->d_plane_mat = nullptr;
    c->d_boxes = nullptr;
    c->d_box_mat = nullptr;
    nbgs_free(c);
    dem_list_free(c);
    adjoint_free(c);
    mbox_free(c);
    stage_free(c);
    c->uploaded = false;
    c->binned = false;
}

int alloc_bodies(Ctx *c, BodyBuf &b) {
    const size_t n = (size_t)std::max<int64_t>(c->n, 1);
    PEB_CUDA(c, dmalloc(c, &b.pr, n * sizeof(double4)));
    PEB_CUDA(c, dmalloc(c, &b.vw, n * (size_t)c->vw_bytes));
    PEB_CUDA(c, dmalloc(c, &b.tag, n * sizeof(uint32_t)));
    PEB_CUDA(c, dmalloc(c, &b.uid, n * sizeof(int32_t)));
    if (c->p.track_orientation) PEB_CUDA(c, dmalloc(c, &b.q, n * sizeof(double4)));
    return PE_B200_OK;
}

int check_material(const pe_b200_material &m, std::string &why) {
    // createMaterial argument checks, src/core/Materials.cpp:189-207
    if (!(m.density > 0)) { why = "Invalid material density!"; return 1; }
    if (m.cor < 0 || m.cor > 1) { why = "Invalid coefficient of restitution!"; return 1; }
    if (m.csf < 0) { why = "Invalid coefficient of static friction!"; return 1; }
    if (m.cdf < 0) { why = "Invalid coefficient of dynamic friction!"; return 1; }
    if (m.poisson < -1 || m.poisson > 0.5) { why = "Invalid Poisson's ratio"; return 1; }
    if (!(m.young > 0)) { why = "Invalid Young's modulus"; return 1; }
    if (!(m.stiffness > 0)) { why = "Invalid stiffness"; return 1; }
    if (m.dampingN < 0 || m.dampingT < 0) { why = "Invalid damping coefficients"; return 1; }
    return 0;
}

}  // namespace

int upload_tables(Ctx *c) {
    // materials
    std::vector<MatDev> md(c->mats.size());
    for (size_t k = 0; k < c->mats.size(); ++k) {
        const pe_b200_material &m = c->mats[k];
        md[k].density = m.density;
        md[k].rk = 1.0 / m.stiffness;
        md[k].rcn = 1.0 / m.dampingN;
        md[k].rct = 1.0 / m.dampingT;
        md[k].csf = m.csf;
        md[k].cdf = m.cdf;
        md[k].young = m.young;
        md[k].poisson = m.poisson;
    }
    dfree(c, c->d_mats);
    c->d_mats = nullptr;
    PEB_CUDA(c, dmalloc(c, &c->d_mats, std::max<size_t>(md.size(), 1) * sizeof(MatDev)));
    if (!md.empty())
        PEB_CUDA(c, cudaMemcpyAsync(c->d_mats, md.data(), md.size() * sizeof(MatDev),
                               cudaMemcpyHostToDevice, c->stream));
    c->mats_dev = md;
    // walls, concatenated per scene
    c->planes.clear();
    c->plane_mat.clear();
    c->boxes.clear();
    c->box_mat.clear();
    for (int s = 0; s < c->nscenes; ++s) {
        SceneInfo &si = c->scenes[s];
        si.plane_begin = (int32_t)(c->planes.size() / 4);
        si.nplanes = (int32_t)(c->scene_planes[s].size() / 4);
        si.box_begin = (int32_t)(c->boxes.size() / 15);
        si.nboxes = (int32_t)(c->scene_boxes[s].size() / 15);
        // the box inside every plane of the scene, 1e-6 inside each of them
        for (int a = 0; a < 3; ++a) {
            si.wall_lo[a] = -INFINITY;
            si.wall_hi[a] = INFINITY;
        }
        const std::vector<double> &sp = c->scene_planes[s];
        for (size_t q = 0; q + 3 < sp.size(); q += 4) {
            int axis = -1;
            for (int a = 0; a < 3; ++a)
                if (fabs(sp[q + a]) == 1.0 && sp[q + (a + 1) % 3] == 0.0 && sp[q + (a + 2) % 3] == 0.0)
                    axis = a;
            if (axis < 0) {
                for (int a = 0; a < 3; ++a) {
                    si.wall_lo[a] = INFINITY;
                    si.wall_hi[a] = -INFINITY;
                }
                break;
            }
            // n.x = d on the plane, body side n.x > d
            if (sp[q + axis] > 0) si.wall_lo[axis] = std::max(si.wall_lo[axis], sp[q + 3] + 1e-6);
            else si.wall_hi[axis] = std::min(si.wall_hi[axis], -sp[q + 3] - 1e-6);
        }
        c->planes.insert(c->planes.end(), c->scene_planes[s].begin(), c->scene_planes[s].end());
        c->plane_mat.insert(c->plane_mat.end(), c->scene_plane_mat[s].begin(),
                            c->scene_plane_mat[s].end());
        c->boxes.insert(c->boxes.end(), c->scene_boxes[s].begin(), c->scene_boxes[s].end());
        c->box_mat.insert(c->box_mat.end(), c->scene_box_mat[s].begin(),
                          c->scene_box_mat[s].end());
    }
    dfree(c, c->d_planes);
    dfree(c, c->d_plane_mat);
    dfree(c, c->d_boxes);
    dfree(c, c->d_box_mat);
    c->d_planes = nullptr;
    c->d_planes_f = nullptr;
    c->d_plane_mat = nullptr;
    c->d_boxes = nullptr;
    c->d_box_mat = nullptr;
    const size_t np = c->planes.size() / 4, nb = c->boxes.size() / 15;
    // FP64 planes followed by an FP32 copy for the kernels' quick rejection test
    PEB_CUDA(c, dmalloc(c, &c->d_planes, std::max<size_t>(np, 1) * (sizeof(double4) + sizeof(float4))));
    c->d_planes_f = reinterpret_cast<float4 *>(c->d_planes + std::max<size_t>(np, 1));
    PEB_CUDA(c, dmalloc(c, &c->d_plane_mat, std::max<size_t>(np, 1) * sizeof(int32_t)));
    PEB_CUDA(c, dmalloc(c, &c->d_boxes, std::max<size_t>(nb, 1) * 15 * sizeof(double)));
    PEB_CUDA(c, dmalloc(c, &c->d_box_mat, std::max<size_t>(nb, 1) * sizeof(int32_t)));
    if (np) {
        PEB_CUDA(c, cudaMemcpyAsync(c->d_planes, c->planes.data(), np * sizeof(double4),
                               cudaMemcpyHostToDevice, c->stream));
        std::vector<float> pf(4 * np);
        for (size_t k = 0; k < 4 * np; ++k) pf[k] = (float)c->planes[k];
        PEB_CUDA(c, cudaMemcpyAsync(c->d_planes_f, pf.data(), np * sizeof(float4),
                               cudaMemcpyHostToDevice, c->stream));
        PEB_CUDA(c, cudaMemcpyAsync(c->d_plane_mat, c->plane_mat.data(), np * sizeof(int32_t),
                               cudaMemcpyHostToDevice, c->stream));
    }
    if (nb) {
        PEB_CUDA(c, cudaMemcpyAsync(c->d_boxes, c->boxes.data(), nb * 15 * sizeof(double),
                               cudaMemcpyHostToDevice, c->stream));
        PEB_CUDA(c, cudaMemcpyAsync(c->d_box_mat, c->box_mat.data(), nb * sizeof(int32_t),
                               cudaMemcpyHostToDevice, c->stream));
    }
    dfree(c, c->d_scenes);
    c->d_scenes = nullptr;
    PEB_CUDA(c, dmalloc(c, &c->d_scenes, std::max<size_t>(c->scenes.size(), 1) * sizeof(SceneInfo)));
    if (!c->scenes.empty())
        PEB_CUDA(c, cudaMemcpyAsync(c->d_scenes, c->scenes.data(), c->scenes.size() * sizeof(SceneInfo),
                               cudaMemcpyHostToDevice, c->stream));
    return PE_B200_OK;
}

namespace {

// grid geometry of each scene: bounding box of its spheres, extended to axis-aligned planes
// that close the scene, with cells of the largest AABB extent (grown if the grid would be much
// larger than the body count; bodies that leave the grid are clamped into the border cells,
// which keeps the search exact and only costs speed)
void plan_grids(Ctx *c, const double *x, const double *r, const std::vector<int64_t> &order,
                const std::vector<int64_t> &begin, const std::vector<int64_t> &count,
                double skin) {
    c->plan_bounds.assign(6 * (size_t)c->nscenes, 0.0);
    c->plan_rmax.assign(c->nscenes, 0.0);
    c->plan_count.assign(c->nscenes, 0);
    for (int s = 0; s < c->nscenes; ++s) {
        double lo0 = INFINITY, lo1 = INFINITY, lo2 = INFINITY;
        double hi0 = -INFINITY, hi1 = -INFINITY, hi2 = -INFINITY, rmax = 0.0;
        const int64_t k0 = begin[s], k1 = begin[s] + count[s];
#pragma omp parallel for schedule(static) \
    reduction(min : lo0, lo1, lo2) reduction(max : hi0, hi1, hi2, rmax)
        for (int64_t k = k0; k < k1; ++k) {
            const int64_t i = order.empty() ? k : order[k];
            const double ri = r[i];
            rmax = std::max(rmax, ri);
            lo0 = std::min(lo0, x[3 * i] - ri);
            lo1 = std::min(lo1, x[3 * i + 1] - ri);
            lo2 = std::min(lo2, x[3 * i + 2] - ri);
            hi0 = std::max(hi0, x[3 * i] + ri);
            hi1 = std::max(hi1, x[3 * i + 1] + ri);
            hi2 = std::max(hi2, x[3 * i + 2] + ri);
        }
        double lo[3] = {lo0, lo1, lo2}, hi[3] = {hi0, hi1, hi2};
        if (count[s] == 0) {
            for (int a = 0; a < 3; ++a) { lo[a] = 0; hi[a] = 1; }
            rmax = 0.5;
        }
        const std::vector<double> &pl = c->scene_planes[s];
        for (size_t p = 0; p + 3 < pl.size(); p += 4) {
            for (int a = 0; a < 3; ++a) {
                const double na = pl[p + a];
                const bool axis = fabs(fabs(na) - 1.0) < 1e-12;
                if (!axis) continue;
                // n.x >= d: lower bound along +axis, or upper bound along -axis
                if (na > 0) lo[a] = std::min(lo[a], pl[p + 3]);
                else hi[a] = std::max(hi[a], -pl[p + 3]);
                // only extend towards the plane, never shrink below the bodies' extent
            }
        }
        for (int a = 0; a < 3; ++a) {
            c->plan_bounds[6 * s + a] = lo[a];
            c->plan_bounds[6 * s + 3 + a] = hi[a];
        }
        c->plan_rmax[s] = rmax;
        c->plan_count[s] = count[s];
        c->scenes[s].body_begin = begin[s];
        c->scenes[s].nbodies = count[s];
    }
    plan_cells(c, skin);
}

}  // namespace

// Cells of every scene for the bounds plan_grids recorded: edge 2 (r_max + contact threshold)
// plus the neighbour-list skin, so that the 27 cells around a body hold every body closer than
// r_i + r_j + skin; grown if the grid would be much larger than the body count.
void plan_cells(Ctx *c, double skin) {
    int64_t base = 0;
    for (int s = 0; s < c->nscenes; ++s) {
        SceneInfo &si = c->scenes[s];
        const double *lo = &c->plan_bounds[6 * s], *hi = &c->plan_bounds[6 * s + 3];
        double h = (2.0 * (c->plan_rmax[s] + kContactThreshold) + std::max(skin, 0.0)) * (1.0 + 1e-9);
        int64_t dim[3], nc;
        const int64_t cap = 8 * std::max<int64_t>(c->plan_count[s], 1) + 4096;
        for (;;) {
            nc = 1;
            for (int a = 0; a < 3; ++a) {
                dim[a] = (int64_t)floor((hi[a] - lo[a]) / h) + 1;
                nc *= dim[a];
            }
            if (nc <= cap) break;
            h *= 1.26;
        }
        for (int a = 0; a < 3; ++a) {
            si.lo[a] = lo[a];
            si.dim[a] = (int32_t)dim[a];
        }
        si.h = h;
        si.inv_h = 1.0 / h;
        si.rmax = c->plan_rmax[s];
        si.cell_base = base;
        base += nc;
    }
    c->ncell = base;
}


}  // namespace peb

namespace peb {

int run_steps(Ctx *c, int32_t nsteps, double dt) {
    int32_t k = 0;
    if (c->p.solver == PE_B200_DEM && c->mb.m > 0) {
        // moving boxes: the grid step (the neighbour lists and graphs cover spheres only)
        for (; k < nsteps; ++k) {
            const int rc = dem_step(c, dt);
            if (rc) return rc;
        }
        return PE_B200_OK;
    }
    if (c->p.solver == PE_B200_DEM && c->nl.enabled && !c->prof) {
        int rc = dem_list_graph_run(c, nsteps, dt, &k);
        if (rc) return rc;
    }
    if (c->p.solver != PE_B200_DEM) return nbgs_run(c, nsteps - k, dt);
    for (; k < nsteps; ++k) {
        const int rc = c->nl.enabled ? dem_list_step(c, dt) : dem_step(c, dt);
        if (rc) return rc;
    }
    return PE_B200_OK;
}

}  // namespace peb

using namespace peb;

extern "C" {

void pe_b200_default_params(pe_b200_params *p) {
    if (!p) return;
    memset(p, 0, sizeof *p);
    p->solver = PE_B200_DEM;
    p->precision = PE_B200_FP64;
    p->relaxation_model = PE_B200_APPROX_INELASTIC_COULOMB_DECOUPLING;
    p->max_iterations = 100;
    p->erp = 0.7;
    p->damping = 1.0;
    p->device = 0;
    p->track_orientation = 0;
    p->max_contacts = 0;
    p->skin = 0.0;
    p->neighbor_lists = 1;
    p->force_model = 0;
}

int pe_b200_create(const pe_b200_params *p, pe_b200_ctx **out) {
    if (!p || !out) return PE_B200_ERR_ARG;
    *out = nullptr;
    if (p->solver != PE_B200_DEM && p->solver != PE_B200_HCSITS) return PE_B200_ERR_ARG;
    if (p->precision != PE_B200_FP64 && p->precision != PE_B200_MIXED) return PE_B200_ERR_ARG;
    if (p->relaxation_model < PE_B200_INELASTIC_FRICTIONLESS ||
        p->relaxation_model > PE_B200_INELASTIC_GENERALIZED_MAX_DISSIPATION)
        return PE_B200_ERR_UNSUPPORTED;
    if (p->max_iterations < 0 || p->damping < 0 || p->damping > 1) return PE_B200_ERR_ARG;
    if (p->force_model != 0 && p->force_model != 1) return PE_B200_ERR_ARG;
    if (p->max_contacts < 0 || p->max_contacts > INT32_MAX) return PE_B200_ERR_ARG;   // int32 offsets
    Ctx *c = new (std::nothrow) Ctx();
    if (!c) return PE_B200_ERR_NOMEM;
    c->p = *p;
    c->device = p->device;
    // six FP64 components, or six FP32 components and the extension plane (internal.cuh)
    c->vw_bytes = p->precision == PE_B200_FP64 ? 6 * 8 : 7 * 4;
    cudaError_t e = cudaSetDevice(p->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = dmalloc(c, &c->d_err, sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_err, 0, sizeof(int32_t), c->stream);
    if (e == cudaSuccess) e = cudaMallocHost(&c->h_err, sizeof(int32_t));
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, p->device);
    if (e != cudaSuccess) {
        int rc = cuda_err(c, e, "pe_b200_create");
        if (c->stream) cudaStreamDestroy(c->stream);
        dfree(c, c->d_err);
        if (c->h_err) cudaFreeHost(c->h_err);
        delete c;
        return rc;
    }
    *out = reinterpret_cast<pe_b200_ctx *>(c);
    return PE_B200_OK;
}

int pe_b200_release_memory(int32_t device) {
    if (device < 0 || device >= 64) return PE_B200_ERR_ARG;
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        pool = g_pool[device];
    }
    if (!pool) return PE_B200_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return PE_B200_ERR_CUDA;
    const cudaError_t e = cudaMemPoolTrimTo(pool, 0);
    cudaSetDevice(prev);
    return e == cudaSuccess ? PE_B200_OK : PE_B200_ERR_CUDA;
}

int pe_b200_destroy(pe_b200_ctx *h) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c) return PE_B200_ERR_ARG;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    prof_collect(c);
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    c->ev_pool.clear();
    free_device(c);
    dfree(c, c->d_err);
    if (c->h_err) cudaFreeHost(c->h_err);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->dl) cudaStreamDestroy(c->dl);
    if (c->ev_dl0) cudaEventDestroy(c->ev_dl0);
    if (c->ev_dl1) cudaEventDestroy(c->ev_dl1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return PE_B200_OK;
}

const char *pe_b200_last_error(const pe_b200_ctx *h) {
    const Ctx *c = reinterpret_cast<const Ctx *>(h);
    return c ? c->err.c_str() : "null context";
}

int pe_b200_set_gravity(pe_b200_ctx *h, const double g[3]) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || !g) return PE_B200_ERR_ARG;
    for (int a = 0; a < 3; ++a) c->p.gravity[a] = g[a];
    c->epoch++;
    return PE_B200_OK;
}

int pe_b200_set_damping(pe_b200_ctx *h, double d) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c) return PE_B200_ERR_ARG;
    // World::setDamping, pe/core/World.h:767 (valid range [0, 1])
    if (d < 0.0 || d > 1.0) return set_err(c, PE_B200_ERR_ARG, "Invalid damping value");
    c->p.damping = d;
    c->epoch++;
    return PE_B200_OK;
}

int pe_b200_set_max_iterations(pe_b200_ctx *h, int32_t n) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || n < 0) return PE_B200_ERR_ARG;
    c->p.max_iterations = n;
    return PE_B200_OK;
}

int pe_b200_set_relaxation_model(pe_b200_ctx *h, int32_t m) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c) return PE_B200_ERR_ARG;
    // the models of HCSITS.h:172-179; others throw "Unsupported relaxation model." (:1926)
    if (m < PE_B200_INELASTIC_FRICTIONLESS || m > PE_B200_INELASTIC_GENERALIZED_MAX_DISSIPATION)
        return set_err(c, PE_B200_ERR_UNSUPPORTED, "Unsupported relaxation model.");
    c->p.relaxation_model = m;
    return PE_B200_OK;
}

int pe_b200_set_error_reduction(pe_b200_ctx *h, double erp) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || !(erp >= 0.0 && erp <= 1.0)) return PE_B200_ERR_ARG;
    c->p.erp = erp;
    return PE_B200_OK;
}

int pe_b200_set_residual(pe_b200_ctx *h, int32_t enabled) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c) return PE_B200_ERR_ARG;
    c->want_residual = enabled ? 1 : 0;
    return PE_B200_OK;
}

int pe_b200_set_materials(pe_b200_ctx *h, int32_t n, const pe_b200_material *m) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || n <= 0 || n > kMaxMaterials || !m) return PE_B200_ERR_ARG;
    std::string why;
    for (int32_t k = 0; k < n; ++k)
        if (check_material(m[k], why)) return set_err(c, PE_B200_ERR_ARG, why);
    c->mats.assign(m, m + n);
    c->epoch++;
    if (c->uploaded) {
        cudaSetDevice(c->device);
        return upload_tables(c);
    }
    return PE_B200_OK;
}

int pe_b200_set_walls(pe_b200_ctx *h, int32_t scene, int32_t nplanes, const double *planes,
                      const int32_t *plane_mat, int32_t nboxes, const double *boxes,
                      const int32_t *box_mat) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || scene < 0 || scene >= kMaxScenes || nplanes < 0 || nboxes < 0) return PE_B200_ERR_ARG;
    if ((nplanes > 0 && (!planes || !plane_mat)) || (nboxes > 0 && (!boxes || !box_mat)))
        return PE_B200_ERR_ARG;
    if ((size_t)scene >= c->scene_planes.size()) {
        c->scene_planes.resize(scene + 1);
        c->scene_plane_mat.resize(scene + 1);
        c->scene_boxes.resize(scene + 1);
        c->scene_box_mat.resize(scene + 1);
    }
    std::vector<double> pl(planes, planes + 4 * (size_t)nplanes);
    for (int32_t p = 0; p < nplanes; ++p) {
        double *q = &pl[4 * p];
        const double l2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
        // createPlane: zero normals are rejected, others normalised (Plane.cpp:1206-1219)
        if (!(l2 > 0.0)) return set_err(c, PE_B200_ERR_ARG, "Invalid plane normal!");
        const double len = sqrt(l2), il = 1.0 / len;
        q[0] *= il; q[1] *= il; q[2] *= il;
        if (plane_mat[p] < 0 || (size_t)plane_mat[p] >= c->mats.size())
            return set_err(c, PE_B200_ERR_ARG, "Invalid material ID");
    }
    for (int32_t b = 0; b < nboxes; ++b) {
        const double *q = boxes + 15 * b;
        // createBox: side lengths must be positive (Box.cpp:1316-1317)
        if (!(q[3] > 0 && q[4] > 0 && q[5] > 0))
            return set_err(c, PE_B200_ERR_ARG, "Invalid side length");
        if (box_mat[b] < 0 || (size_t)box_mat[b] >= c->mats.size())
            return set_err(c, PE_B200_ERR_ARG, "Invalid material ID");
    }
    c->scene_planes[scene] = pl;
    c->scene_plane_mat[scene].assign(plane_mat, plane_mat + nplanes);
    c->scene_boxes[scene].assign(boxes, boxes + 15 * (size_t)nboxes);
    c->scene_box_mat[scene].assign(box_mat, box_mat + nboxes);
    c->epoch++;
    if (c->uploaded) {
        cudaSetDevice(c->device);
        return upload_tables(c);
    }
    return PE_B200_OK;
}

int pe_b200_upload_bodies(pe_b200_ctx *h, int64_t n, const double *x, const double *v,
                          const double *w, const double *r, const int32_t *mat,
                          const int32_t *scene, int32_t nscenes) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || n < 0 || n > (int64_t)INT32_MAX / 2 || nscenes <= 0 || nscenes > kMaxScenes)
        return PE_B200_ERR_ARG;
    if (n > 0 && (!x || !v || !w || !r || !mat)) return PE_B200_ERR_ARG;
    if (c->mats.empty()) return set_err(c, PE_B200_ERR_STATE, "materials must be set before bodies");
    cudaSetDevice(c->device);
    // the first invalid sphere (in upload order) decides the error, as pe's createSphere calls
    // would have failed one at a time; the scan itself runs on all host threads
    int64_t first_bad = n;
    const int64_t nmat = (int64_t)c->mats.size();
#pragma omp parallel for reduction(min : first_bad) schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        bool ok = r[i] > 0.0 && mat[i] >= 0 && mat[i] < nmat &&
                  (!scene || (scene[i] >= 0 && scene[i] < nscenes));
        for (int a = 0; a < 3; ++a)
            ok = ok && isfinite(x[3 * i + a]) && isfinite(v[3 * i + a]) && isfinite(w[3 * i + a]);
        if (!ok && i < first_bad) first_bad = i;
    }
    if (first_bad < n) {
        const int64_t i = first_bad;
        // createSphere: the radius must be positive (Sphere.cpp:1193-1194)
        if (!(r[i] > 0.0)) return set_err(c, PE_B200_ERR_ARG, "Invalid sphere radius");
        if (mat[i] < 0 || mat[i] >= nmat) return set_err(c, PE_B200_ERR_ARG, "Invalid material ID");
        if (scene && (scene[i] < 0 || scene[i] >= nscenes))
            return set_err(c, PE_B200_ERR_ARG, "Invalid scene ID");
        return set_err(c, PE_B200_ERR_NAN, "non-finite body state");
    }
    free_device(c);
    c->epoch++;
    c->n = n;
    c->nscenes = nscenes;
    c->scenes.assign(nscenes, SceneInfo());
    c->scene_planes.resize(std::max<size_t>(c->scene_planes.size(), nscenes));
    c->scene_plane_mat.resize(c->scene_planes.size());
    c->scene_boxes.resize(c->scene_planes.size());
    c->scene_box_mat.resize(c->scene_planes.size());
    // group bodies by scene (stable) for the grid plan
    // (one scene: upload order itself, no permutation array)
    std::vector<int64_t> count(nscenes, 0), begin(nscenes, 0), order;
    if (!scene) {
        count[0] = n;
    } else {
        order.resize(n);
        for (int64_t i = 0; i < n; ++i) count[scene[i]]++;
        for (int s = 1; s < nscenes; ++s) begin[s] = begin[s - 1] + count[s - 1];
        std::vector<int64_t> fill(begin);
        for (int64_t i = 0; i < n; ++i) order[fill[scene[i]]++] = i;
    }
    const bool lists = c->p.solver == PE_B200_DEM && c->p.neighbor_lists && n > 0;
    if (lists) {
        double rmin = INFINITY;
#pragma omp parallel for schedule(static) reduction(min : rmin)
        for (int64_t i = 0; i < n; ++i) rmin = std::min(rmin, r[i]);
        c->nl.skin = c->p.skin > 0.0 ? c->p.skin : 0.1 * rmin;
    }
    plan_grids(c, x, r, order, begin, count, lists ? c->nl.skin : 0.0);
    if (c->ncell > (int64_t)INT32_MAX / 2) return set_err(c, PE_B200_ERR_CAPACITY, "grid too large");
    int rc = upload_tables(c);
    if (rc) return rc;
    rc = alloc_bodies(c, c->cur);
    if (rc) return rc;
    rc = alloc_bodies(c, c->nxt);
    if (rc) return rc;
    rc = grid_alloc(c);
    if (rc) return rc;
    // the caller's arrays go to the device as they are; a kernel packs them
    rc = pack_bodies(c, x, v, w, r, mat, scene);
    if (rc) return rc;
    c->uploaded = true;
    c->binned = false;
    if (lists) {
        rc = dem_list_alloc(c);
        if (rc) return rc;
    }
    return PE_B200_OK;
}

static int check_device_errors(Ctx *c);

int pe_b200_upload_boxes(pe_b200_ctx *h, int32_t m, const double *x, const double *q,
                         const double *v, const double *w, const double *lengths,
                         const int32_t *mat, const int32_t *scene) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || m < 0 || m > (1 << 24)) return PE_B200_ERR_ARG;
    if (m > 0 && (!x || !q || !v || !w || !lengths || !mat)) return PE_B200_ERR_ARG;
    if (!c->uploaded) return set_err(c, PE_B200_ERR_STATE, "spheres must be uploaded before boxes");
    if (m > 0 && c->p.precision != PE_B200_FP64)
        return set_err(c, PE_B200_ERR_UNSUPPORTED, "moving boxes need FP64 precision");
    const int64_t nmat = (int64_t)c->mats.size();
    for (int32_t k = 0; k < m; ++k) {
        // createBox: side lengths must be positive (src/core/rigidbody/Box.cpp:1316-1319)
        if (!(lengths[3 * k] > 0.0) || !(lengths[3 * k + 1] > 0.0) || !(lengths[3 * k + 2] > 0.0))
            return set_err(c, PE_B200_ERR_ARG, "Invalid side length");
        if (mat[k] < 0 || mat[k] >= nmat) return set_err(c, PE_B200_ERR_ARG, "Invalid material ID");
        if (scene && (scene[k] < 0 || scene[k] >= c->nscenes || (k > 0 && scene[k] < scene[k - 1])))
            return set_err(c, PE_B200_ERR_ARG, "Invalid scene ID (boxes must be grouped by scene)");
        bool ok = true;
        for (int a = 0; a < 3; ++a)
            ok = ok && std::isfinite(x[3 * k + a]) && std::isfinite(v[3 * k + a]) &&
                 std::isfinite(w[3 * k + a]);
        const double *qq = q + 4 * k;
        const double qn = qq[0] * qq[0] + qq[1] * qq[1] + qq[2] * qq[2] + qq[3] * qq[3];
        // Quaternion(r, i, j, k) wants a unit quaternion (Quaternion.h:251-255)
        if (!ok || !(std::fabs(qn - 1.0) < 1e-8)) return set_err(c, PE_B200_ERR_ARG, "Invalid box state");
    }
    cudaSetDevice(c->device);
    PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    return mbox_upload(c, m, x, q, v, w, lengths, mat, scene);
}

int pe_b200_download_boxes(pe_b200_ctx *h, double *x, double *q, double *v, double *w) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c) return PE_B200_ERR_ARG;
    cudaSetDevice(c->device);
    const int rc = mbox_download(c, x, q, v, w);
    if (rc) return rc;
    return check_device_errors(c);
}

int32_t pe_b200_box_count(const pe_b200_ctx *h) {
    const Ctx *c = reinterpret_cast<const Ctx *>(h);
    return c ? c->mb.m : -1;
}

int pe_b200_set_state(pe_b200_ctx *h, const double *x, const double *v, const double *w) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c) return PE_B200_ERR_ARG;
    if (!c->uploaded) return set_err(c, PE_B200_ERR_STATE, "no bodies uploaded");
    cudaSetDevice(c->device);
    const int64_t n = c->n;
    if (n == 0) return PE_B200_OK;
    // scattered by the body permutation on the device
    const int src = scatter_state(c, x, v, w);
    if (src) return src;
    c->binned = false;
    if (c->nl.enabled) {
        const int rc = dem_list_request_rebuild(c);
        if (rc) return rc;
    }
    return PE_B200_OK;
}

int pe_b200_set_orientations(pe_b200_ctx *h, const double *q) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || !q) return PE_B200_ERR_ARG;
    if (!c->uploaded) return set_err(c, PE_B200_ERR_STATE, "no bodies uploaded");
    if (!c->p.track_orientation)
        return set_err(c, PE_B200_ERR_STATE, "orientations are not tracked by this context");
    cudaSetDevice(c->device);
    return scatter_orientations(c, q);
}

int pe_b200_step(pe_b200_ctx *h, int32_t nsteps, double dt) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c) return PE_B200_ERR_ARG;
    // World::simulationStep rejects non-positive time steps (src/core/World.cpp:333-334)
    if (!(dt > 0.0)) return set_err(c, PE_B200_ERR_ARG, "Invalid time step size");
    if (nsteps < 0) return PE_B200_ERR_ARG;
    if (!c->uploaded) return set_err(c, PE_B200_ERR_STATE, "no bodies uploaded");
    cudaSetDevice(c->device);
    return run_steps(c, nsteps, dt);
}

int pe_b200_set_graph_steps(pe_b200_ctx *h, int32_t steps) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || steps < 0) return PE_B200_ERR_ARG;
    c->graph_steps = steps & ~1;
    c->sg.failed = false;
    c->nb.gfailed = false;
    dem_graph_free(c);
    nbgs_graph_free(c);
    return PE_B200_OK;
}

int pe_b200_graph_active(const pe_b200_ctx *h) {
    const Ctx *c = reinterpret_cast<const Ctx *>(h);
    if (!c) return 0;
    if (c->sg.exec && !c->sg.failed) return 1;
    if (c->nb.gfailed) return 0;
    for (const NbgsBuf::GraphSlot &s : c->nb.gslot)
        if (s.exec) return 1;
    return 0;
}

int pe_b200_graph_stats(const pe_b200_ctx *h, int64_t *captures, int64_t *replays) {
    const Ctx *c = reinterpret_cast<const Ctx *>(h);
    if (!c || !captures || !replays) return PE_B200_ERR_ARG;
    *captures = c->graph_captures;
    *replays = c->graph_replays;
    return PE_B200_OK;
}

int pe_b200_get_tuning(pe_b200_ctx *h, pe_b200_tuning *out) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || !out) return PE_B200_ERR_ARG;
    out->dem_variant = c->tune.dem_variant;
    out->rebuild_per_sm = c->tune.rebuild_per_sm;
    out->skin = c->nl.skin;
    out->ms_per_step = -1.0;
    out->variants = dem_variant_count();
    out->nbgs_sweeps = c->tune.nbgs_sweeps;
    out->dem_grid = c->tune.dem_grid;
    out->dem_split = c->tune.dem_split;
    return PE_B200_OK;
}

int pe_b200_set_tuning(pe_b200_ctx *h, const pe_b200_tuning *t) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || !t) return PE_B200_ERR_ARG;
    if (!c->uploaded) return set_err(c, PE_B200_ERR_STATE, "no bodies uploaded");
    cudaSetDevice(c->device);
    Tuning tu;
    tu.dem_variant = t->dem_variant;
    tu.rebuild_per_sm = t->rebuild_per_sm;
    tu.nbgs_sweeps = t->nbgs_sweeps;
    tu.dem_grid = t->dem_grid;
    tu.dem_split = t->dem_split;
    return set_tuning(c, tu, c->nl.enabled ? t->skin : c->nl.skin);
}

int pe_b200_autotune(pe_b200_ctx *h, double dt, int32_t trial_steps, pe_b200_tuning *out) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c) return PE_B200_ERR_ARG;
    if (!c->uploaded) return set_err(c, PE_B200_ERR_STATE, "no bodies uploaded");
    if (c->mb.m > 0)
        return set_err(c, PE_B200_ERR_UNSUPPORTED, "the tuner covers sphere scenes only");
    cudaSetDevice(c->device);
    return autotune(c, dt, trial_steps, out);
}

static int check_device_errors(Ctx *c) {
    PEB_CUDA(c, cudaMemcpyAsync(c->h_err, c->d_err, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                c->stream));
    PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    const int32_t e = *c->h_err;
    if (e) {
        PEB_CUDA(c, cudaMemsetAsync(c->d_err, 0, sizeof(int32_t), c->stream));
        if (e & DERR_NAN) return set_err(c, PE_B200_ERR_NAN, "non-finite body state after step");
        if (e & DERR_TIMEOUT) return set_err(c, PE_B200_ERR_TIMEOUT, "device wait timed out");
        return set_err(c, PE_B200_ERR_CAPACITY, "device capacity exceeded");
    }
    return PE_B200_OK;
}

int pe_b200_download_bodies(pe_b200_ctx *h, double *x, double *v, double *w, double *q) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c) return PE_B200_ERR_ARG;
    if (!c->uploaded) return set_err(c, PE_B200_ERR_STATE, "no bodies uploaded");
    if (q && !c->p.track_orientation)
        return set_err(c, PE_B200_ERR_STATE, "orientations are not tracked");
    cudaSetDevice(c->device);
    const int64_t n = c->n;
    if (n == 0) return PE_B200_OK;
    const int rc = check_device_errors(c);
    const int urc = unpack_bodies(c, x, v, w, q);
    if (urc) return urc;
    return rc;
}

int pe_b200_find_contacts(pe_b200_ctx *h, int64_t cap, int64_t *ids, double *geom,
                          int64_t *n_out) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || cap < 0 || !n_out || (cap > 0 && (!ids || !geom))) return PE_B200_ERR_ARG;
    if (!c->uploaded) return set_err(c, PE_B200_ERR_STATE, "no bodies uploaded");
    cudaSetDevice(c->device);
    return find_contacts(c, cap, ids, geom, n_out);
}

int pe_b200_last_step_stats(pe_b200_ctx *h, int64_t *ncontacts, int32_t *ncolors,
                            double *delta_max, double *residual) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c) return PE_B200_ERR_ARG;
    if (ncontacts) *ncontacts = c->last_ncontacts;
    if (ncolors) *ncolors = c->last_ncolors;
    if (delta_max) *delta_max = c->last_delta;
    if (residual) *residual = c->last_residual;
    return PE_B200_OK;
}

int pe_b200_adjoint_forward(pe_b200_ctx *h, int32_t nsteps, double dt, int32_t every) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c) return PE_B200_ERR_ARG;
    if (!c->uploaded) return set_err(c, PE_B200_ERR_STATE, "no bodies uploaded");
    if (c->mb.m > 0)
        return set_err(c, PE_B200_ERR_UNSUPPORTED, "the adjoint step covers sphere scenes only");
    cudaSetDevice(c->device);
    return adjoint_forward(c, nsteps, dt, every);
}

int pe_b200_adjoint_backward(pe_b200_ctx *h, const double *gx, const double *gv, const double *gw,
                             double *gx0, double *gv0, double *gw0, double *gparams) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || !gx || !gv || !gw || !gx0 || !gv0 || !gw0) return PE_B200_ERR_ARG;
    cudaSetDevice(c->device);
    return adjoint_backward(c, gx, gv, gw, gx0, gv0, gw0, gparams);
}

int pe_b200_neighbor_list_stats(pe_b200_ctx *h, int64_t *rebuilds, int64_t *entries,
                                int64_t *capacity, double *skin) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c) return PE_B200_ERR_ARG;
    int32_t f[4] = {0, 0, 0, 0};
    if (c->nl.enabled) {
        cudaSetDevice(c->device);
        PEB_CUDA(c, cudaMemcpyAsync(f, c->nl.flags, sizeof f, cudaMemcpyDeviceToHost, c->stream));
        PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    if (rebuilds) *rebuilds = f[3];
    if (entries) *entries = f[2];
    if (capacity) *capacity = c->nl.cap;
    if (skin) *skin = c->nl.skin;
    return PE_B200_OK;
}

int pe_b200_set_profiling(pe_b200_ctx *h, int32_t enabled) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c) return PE_B200_ERR_ARG;
    cudaSetDevice(c->device);
    prof_collect(c);
    c->prof = enabled != 0;
    for (int s = 0; s < ST_COUNT; ++s) {
        c->prof_ms[s] = 0.0;
        c->prof_count[s] = 0;
    }
    return PE_B200_OK;
}

int pe_b200_profile(pe_b200_ctx *h, int32_t cap, const char **names, double *total_ms,
                    int64_t *count, int32_t *n_out) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || cap < 0 || !n_out) return PE_B200_ERR_ARG;
    cudaSetDevice(c->device);
    prof_collect(c);
    const int m = cap < ST_COUNT ? cap : ST_COUNT;
    for (int s = 0; s < m; ++s) {
        if (names) names[s] = kStageNames[s];
        if (total_ms) total_ms[s] = c->prof_ms[s];
        if (count) count[s] = c->prof_count[s];
    }
    *n_out = ST_COUNT;
    return PE_B200_OK;
}

int pe_b200_validate(pe_b200_ctx *h, int64_t *problems) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || !problems) return PE_B200_ERR_ARG;
    *problems = 0;
    if (!c->uploaded) return PE_B200_OK;
    cudaSetDevice(c->device);
    int rc = validate_lists(c, problems);
    if (!rc) rc = validate_coloring(c, problems);
    return rc;
}

int pe_b200_selftest_timeout(pe_b200_ctx *h, int64_t polls) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || polls < 1 || polls > (int64_t(1) << 24)) return PE_B200_ERR_ARG;
    cudaSetDevice(c->device);
    int rc = check_device_errors(c);   // a pending device error belongs to an earlier call
    if (rc) return rc;
    rc = selftest_timeout(c, polls);
    if (rc) return rc;
    return check_device_errors(c);
}

int64_t pe_b200_kernel_launches(const pe_b200_ctx *h) {
    const Ctx *c = reinterpret_cast<const Ctx *>(h);
    return c ? c->launches : -1;
}

void *pe_b200_stream(pe_b200_ctx *h) {
    Ctx *c = reinterpret_cast<Ctx *>(h);
    return c ? (void *)c->stream : nullptr;
}

}  // extern "C"
