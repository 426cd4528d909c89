// noalloc.cu -- pe_b200_dem_step_static: one FP64 DEM step of a single scene that allocates
// no memory at all.
//
// Some callers cannot call cudaMalloc: a host application that owns every byte of device memory
// through its own arena or pool (a coupled fluid/particle code running inside a fixed memory
// budget, say), or a real-time loop that must not pay for an allocation's implicit device
// synchronisation.  For them this entry point runs the same step kernel as pe_b200_step, with
// its scratch (packed body records, grid keys, cell counts and offsets, the sorted order and the
// material/wall tables) in one file-scope __device__ array of fixed size, declared below.  The
// caller passes device pointers for the inputs and the outputs; materials and walls are small
// host arrays that are copied into the fixed array.
//
// Limits and sharing:
//   - at most PE_B200_STATIC_MAX_SPHERES spheres, 64 materials, 64 planes and 64 boxes; larger
//     inputs are rejected with PE_B200_ERR_ARG before anything runs.  The grid is coarsened
//     until it fits PE_B200_STATIC_MAX_CELLS cells (still exact, only slower);
//   - the array (kScratchBytes, about 7.3 MB) exists on every GPU that loads the library, from
//     module load until the process exits;
//   - every call on a device shares it and finds the previous call's contents; each call clears
//     what must start at zero.  Two calls whose work overlaps on the GPU (different streams or
//     host threads without ordering) race on the array and corrupt each other's results;
//   - in host code the array's name is only a host-side stand-in: its device address is looked
//     up with cudaGetSymbolAddress, with the device current, by the first call on each device
//     (again after cudaDeviceReset, which unloads the module: the cache is keyed on the CUDA
//     context's unique id, not on the device ordinal);
//   - a call is synchronous: it copies its small tables from host memory and waits for its
//     stream before returning.
#include <cuda.h>
#include <math.h>

#include <mutex>

#include "internal.cuh"
#include "static_grid.h"

namespace peb {

namespace {

constexpr int64_t kMaxSpheres = PE_B200_STATIC_MAX_SPHERES;
constexpr int64_t kMaxCells = PE_B200_STATIC_MAX_CELLS;
constexpr int kMaxMat = 64, kMaxPlanes = 64, kMaxBoxes = 64;

constexpr size_t al(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t OFF_PR_A = 0;
constexpr size_t OFF_PR_B = OFF_PR_A + al(kMaxSpheres * sizeof(double4));
constexpr size_t OFF_VW_A = OFF_PR_B + al(kMaxSpheres * sizeof(double4));
constexpr size_t OFF_VW_B = OFF_VW_A + al(kMaxSpheres * 6 * sizeof(double));
constexpr size_t OFF_TAG_A = OFF_VW_B + al(kMaxSpheres * 6 * sizeof(double));
constexpr size_t OFF_TAG_B = OFF_TAG_A + al(kMaxSpheres * sizeof(uint32_t));
constexpr size_t OFF_UID_A = OFF_TAG_B + al(kMaxSpheres * sizeof(uint32_t));
constexpr size_t OFF_UID_B = OFF_UID_A + al(kMaxSpheres * sizeof(int32_t));
constexpr size_t OFF_KEY = OFF_UID_B + al(kMaxSpheres * sizeof(int32_t));
constexpr size_t OFF_RANK = OFF_KEY + al(kMaxSpheres * sizeof(int32_t));
constexpr size_t OFF_SORTED = OFF_RANK + al(kMaxSpheres * sizeof(int32_t));
constexpr size_t OFF_COUNT = OFF_SORTED + al(kMaxSpheres * sizeof(int32_t));
constexpr size_t OFF_START = OFF_COUNT + al((kMaxCells + 1) * sizeof(int32_t));
constexpr size_t OFF_SCENE = OFF_START + al((kMaxCells + 2) * sizeof(int32_t));
constexpr size_t OFF_MATS = OFF_SCENE + al(sizeof(SceneInfo));
constexpr size_t OFF_PLANES = OFF_MATS + al(kMaxMat * sizeof(MatDev));
constexpr size_t OFF_PLANE_MAT = OFF_PLANES + al(kMaxPlanes * sizeof(double4));
constexpr size_t OFF_BOXES = OFF_PLANE_MAT + al(kMaxPlanes * sizeof(int32_t));
constexpr size_t OFF_BOX_MAT = OFF_BOXES + al(kMaxBoxes * 15 * sizeof(double));
constexpr size_t OFF_ERR = OFF_BOX_MAT + al(kMaxBoxes * sizeof(int32_t));
constexpr size_t kScratchBytes = OFF_ERR + al(sizeof(int32_t));

// error bits of this entry point (besides the step kernel's DERR_NAN)
constexpr int32_t SERR_RADIUS = 1 << 8;
constexpr int32_t SERR_MATERIAL = 1 << 9;

}  // namespace

// The scratch of pe_b200_dem_step_static (see the file comment for its rules).
static __device__ __align__(256) unsigned char g_static_scratch[kScratchBytes];

namespace {

std::mutex g_addr_mu;
struct ScratchAddr {
    unsigned long long ctx_id = 0;   // unique id of the context the address belongs to
    unsigned char *addr = nullptr;
};
ScratchAddr g_addr[128];

// The driver's context queries, fetched through the runtime (no link against libcuda).
typedef CUresult (*PfnCtxGetCurrent)(CUcontext *);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long *);

// Unique id of the current context (0 if none is current or the driver cannot say).
unsigned long long current_context_id() {
    static PfnCtxGetCurrent get_current = nullptr;
    static PfnCtxGetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<PfnCtxGetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PfnCtxGetId>(f);
        looked_up = true;
    }
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Set-up, once per device and context: the device address of g_static_scratch on `dev`, which
// must be current.  The lookup allocates nothing.
cudaError_t scratch_address(int dev, unsigned char **out) {
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (dev < 0 || dev >= 128) return cudaErrorInvalidDevice;
    ScratchAddr &s = g_addr[dev];
    unsigned long long id = current_context_id();
    if (!s.addr || id == 0 || id != s.ctx_id) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return e;
        s.addr = static_cast<unsigned char *>(p);
        // the lookup made the device's primary context current if none was
        if (id == 0) id = current_context_id();
        s.ctx_id = id;
    }
    *out = s.addr;
    return cudaSuccess;
}

__global__ void k_pack_bin(int64_t n, const double *x, const double *v, const double *w,
                           const double *r, const int32_t *mat, int32_t nmat, double max_radius,
                           const SceneInfo *scene, double4 *pr, double *vw, uint32_t *tag,
                           int32_t *uid, int32_t *key, int32_t *rank, int32_t *cell_count,
                           int32_t *err) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double px = x[3 * i], py = x[3 * i + 1], pz = x[3 * i + 2], ri = r[i];
    if (!(ri > 0.0 && ri <= max_radius)) atomicOr(err, SERR_RADIUS);
    int32_t m = mat[i];
    if (m < 0 || m >= nmat) {
        atomicOr(err, SERR_MATERIAL);
        m = 0;
    }
    pr[i] = make_double4(px, py, pz, ri);
    for (int a = 0; a < 3; ++a) {
        vw[a * n + i] = v[3 * i + a];
        vw[(3 + a) * n + i] = w[3 * i + a];
    }
    tag[i] = (uint32_t)m;
    uid[i] = (int32_t)i;
    int cx, cy, cz;
    cell_coords(*scene, px, py, pz, cx, cy, cz);
    const int32_t k = (int32_t)cell_key(*scene, cx, cy, cz);
    key[i] = k;
    rank[i] = atomicAdd(&cell_count[k], 1);
}

// exclusive scan of count[0, m) into start[0, m], one block of 1024 threads
__global__ void __launch_bounds__(1024) k_scan_one_block(const int32_t *count, int32_t *start,
                                                         int64_t m) {
    __shared__ int32_t warp_sum[32];
    const int t = threadIdx.x;
    const int64_t per = (m + 1023) / 1024;
    const int64_t b = t * per, e = (b + per < m) ? b + per : m;
    int32_t s = 0;
    for (int64_t i = b; i < e; ++i) s += count[i];
    int32_t incl = s;
    const int lane = t & 31, wid = t >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (lane == 31) warp_sum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int32_t ws = warp_sum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t u = __shfl_up_sync(0xffffffffu, ws, o);
            if (lane >= o) ws += u;
        }
        warp_sum[lane] = ws;
    }
    __syncthreads();
    int32_t run = incl - s + (wid > 0 ? warp_sum[wid - 1] : 0);
    for (int64_t i = b; i < e; ++i) {
        start[i] = run;
        run += count[i];
    }
    if (t == 1023) start[m] = warp_sum[31];
}

__global__ void k_scatter_s(int64_t n, const int32_t *key, const int32_t *rank,
                            const int32_t *start, int32_t *sorted) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    sorted[start[key[i]] + rank[i]] = (int32_t)i;
}

__global__ void k_fixup_s(int64_t ncell, const int32_t *start, int32_t *sorted) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
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

// the caller's outputs are written only when every radius and material index was valid
__global__ void k_unpack(int64_t n, const double4 *pr, const double *vw, const int32_t *uid,
                         const int32_t *err, double *x, double *v, double *w) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || (*err & (SERR_RADIUS | SERR_MATERIAL)) != 0) return;
    const int64_t i = uid[t];
    const double4 p = pr[t];
    x[3 * i] = p.x;
    x[3 * i + 1] = p.y;
    x[3 * i + 2] = p.z;
    for (int a = 0; a < 3; ++a) {
        v[3 * i + a] = vw[a * n + t];
        w[3 * i + a] = vw[(3 + a) * n + t];
    }
}

}  // namespace

}  // namespace peb

using namespace peb;

extern "C" int pe_b200_dem_step_static(int64_t n, const double *x, const double *v,
                                       const double *w, const double *r, const int32_t *mat,
                                       int32_t nmat, const pe_b200_material *mats,
                                       int32_t nplanes, const double *planes,
                                       const int32_t *plane_mat, int32_t nboxes,
                                       const double *boxes, const int32_t *box_mat,
                                       const double gravity[3], double damping, double dt,
                                       const double domain_lo[3], const double domain_hi[3],
                                       double max_radius, double *x_out, double *v_out,
                                       double *w_out, void *stream) {
    // ---- host-side checks (nothing has run on the GPU yet) ----
    if (n < 0 || n > kMaxSpheres) return PE_B200_ERR_ARG;
    if (nmat < 1 || nmat > kMaxMat || !mats) return PE_B200_ERR_ARG;
    if (nplanes < 0 || nplanes > kMaxPlanes || nboxes < 0 || nboxes > kMaxBoxes)
        return PE_B200_ERR_ARG;
    if ((nplanes > 0 && (!planes || !plane_mat)) || (nboxes > 0 && (!boxes || !box_mat)))
        return PE_B200_ERR_ARG;
    if (!gravity || !domain_lo || !domain_hi || !(dt > 0.0) || !(max_radius > 0.0) ||
        !isfinite(max_radius) ||
        !(damping >= 0.0 && damping <= 1.0))
        return PE_B200_ERR_ARG;
    if (n > 0 && (!x || !v || !w || !r || !mat || !x_out || !v_out || !w_out))
        return PE_B200_ERR_ARG;
    for (int a = 0; a < 3; ++a)
        if (!(domain_hi[a] >= domain_lo[a]) || !isfinite(domain_lo[a]) || !isfinite(domain_hi[a]))
            return PE_B200_ERR_ARG;
    // tables in fixed-size host arrays (createMaterial / createPlane / createBox checks)
    MatDev md[kMaxMat];
    for (int k = 0; k < nmat; ++k) {
        const pe_b200_material &m = mats[k];
        if (!(m.density > 0) || !(m.stiffness > 0) || m.dampingN < 0 || m.dampingT < 0 ||
            m.csf < 0 || m.cdf < 0)
            return PE_B200_ERR_ARG;
        md[k].density = m.density;
        md[k].rk = 1.0 / m.stiffness;
        md[k].rcn = 1.0 / m.dampingN;
        md[k].rct = 1.0 / m.dampingT;
        md[k].csf = m.csf;
        md[k].cdf = m.cdf;
    }
    double4 pl[kMaxPlanes];
    for (int p = 0; p < nplanes; ++p) {
        const double *q = planes + 4 * p;
        const double l2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
        if (!(l2 > 0.0) || plane_mat[p] < 0 || plane_mat[p] >= nmat) return PE_B200_ERR_ARG;
        const double il = 1.0 / sqrt(l2);
        pl[p] = make_double4(q[0] * il, q[1] * il, q[2] * il, q[3]);
    }
    for (int b = 0; b < nboxes; ++b) {
        const double *q = boxes + 15 * b;
        if (!(q[3] > 0 && q[4] > 0 && q[5] > 0) || box_mat[b] < 0 || box_mat[b] >= nmat)
            return PE_B200_ERR_ARG;
    }
    // grid: cells at least the largest AABB extent, coarsened to fit the fixed cell budget
    SceneInfo si = SceneInfo();
    StaticGrid grid;
    if (!static_grid_plan(domain_lo, domain_hi, 2.0 * (max_radius + kContactThreshold) * (1.0 + 1e-9),
                          kMaxCells, &grid))
        return PE_B200_ERR_ARG;
    const double h = grid.h;
    const int64_t nc = grid.ncell;
    const int64_t *dim = grid.dim;
    for (int a = 0; a < 3; ++a) {
        si.lo[a] = domain_lo[a];
        si.dim[a] = (int32_t)dim[a];
    }
    si.h = h;
    si.inv_h = 1.0 / h;
    si.cell_base = 0;
    si.plane_begin = 0;
    si.nplanes = nplanes;
    si.box_begin = 0;
    si.nboxes = nboxes;
    si.body_begin = 0;
    si.nbodies = n;

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return PE_B200_ERR_CUDA;
    unsigned char *base = nullptr;
    e = scratch_address(dev, &base);
    if (e != cudaSuccess) return PE_B200_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    double4 *pr_a = (double4 *)(base + OFF_PR_A), *pr_b = (double4 *)(base + OFF_PR_B);
    double *vw_a = (double *)(base + OFF_VW_A), *vw_b = (double *)(base + OFF_VW_B);
    uint32_t *tag_a = (uint32_t *)(base + OFF_TAG_A), *tag_b = (uint32_t *)(base + OFF_TAG_B);
    int32_t *uid_a = (int32_t *)(base + OFF_UID_A), *uid_b = (int32_t *)(base + OFF_UID_B);
    int32_t *key = (int32_t *)(base + OFF_KEY), *rank = (int32_t *)(base + OFF_RANK);
    int32_t *sorted = (int32_t *)(base + OFF_SORTED);
    int32_t *count = (int32_t *)(base + OFF_COUNT), *start = (int32_t *)(base + OFF_START);
    SceneInfo *d_scene = (SceneInfo *)(base + OFF_SCENE);
    MatDev *d_mats = (MatDev *)(base + OFF_MATS);
    double4 *d_planes = (double4 *)(base + OFF_PLANES);
    int32_t *d_plane_mat = (int32_t *)(base + OFF_PLANE_MAT);
    double *d_boxes = (double *)(base + OFF_BOXES);
    int32_t *d_box_mat = (int32_t *)(base + OFF_BOX_MAT);
    int32_t *d_err = (int32_t *)(base + OFF_ERR);

#define PEB_S(call)                                  \
    do {                                             \
        if ((e = (call)) != cudaSuccess) return PE_B200_ERR_CUDA; \
    } while (0)
    // tables and the zero-initialised parts (the array keeps the previous call's contents)
    PEB_S(cudaMemcpyAsync(d_scene, &si, sizeof si, cudaMemcpyHostToDevice, st));
    PEB_S(cudaMemcpyAsync(d_mats, md, nmat * sizeof(MatDev), cudaMemcpyHostToDevice, st));
    if (nplanes > 0) {
        PEB_S(cudaMemcpyAsync(d_planes, pl, nplanes * sizeof(double4), cudaMemcpyHostToDevice, st));
        PEB_S(cudaMemcpyAsync(d_plane_mat, plane_mat, nplanes * sizeof(int32_t),
                              cudaMemcpyHostToDevice, st));
    }
    if (nboxes > 0) {
        PEB_S(cudaMemcpyAsync(d_boxes, boxes, nboxes * 15 * sizeof(double), cudaMemcpyHostToDevice, st));
        PEB_S(cudaMemcpyAsync(d_box_mat, box_mat, nboxes * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    }
    PEB_S(cudaMemsetAsync(count, 0, (nc + 1) * sizeof(int32_t), st));
    PEB_S(cudaMemsetAsync(d_err, 0, sizeof(int32_t), st));
    if (n > 0) {
        k_pack_bin<<<grid_for(n, 256), 256, 0, st>>>(n, x, v, w, r, mat, nmat, max_radius,
                                                     d_scene, pr_a, vw_a, tag_a, uid_a, key,
                                                     rank, count, d_err);
        PEB_S(cudaGetLastError());
        k_scan_one_block<<<1, 1024, 0, st>>>(count, start, nc);
        PEB_S(cudaGetLastError());
        k_scatter_s<<<grid_for(n, 256), 256, 0, st>>>(n, key, rank, start, sorted);
        PEB_S(cudaGetLastError());
        k_fixup_s<<<grid_for(nc, 256), 256, 0, st>>>(nc, start, sorted);
        PEB_S(cudaGetLastError());
        DemRawArgs a;
        a.n = n;
        a.dt = dt;
        a.damping = damping;
        for (int k = 0; k < 3; ++k) a.g[k] = gravity[k];
        a.sorted = sorted;
        a.cell_start = start;
        a.scenes = d_scene;
        a.mats = d_mats;
        a.planes = d_planes;
        a.plane_mat = d_plane_mat;
        a.boxes = d_boxes;
        a.box_mat = d_box_mat;
        a.pr = pr_a;
        a.vw = vw_a;
        a.tag = tag_a;
        a.uid = uid_a;
        a.pr_out = pr_b;
        a.vw_out = vw_b;
        a.tag_out = tag_b;
        a.uid_out = uid_b;
        // the step kernel also bins its output for a next step; that count goes to the scratch
        // counters, which the next call clears
        a.key = key;
        a.rank = rank;
        a.cell_count = count;
        a.err = d_err;
        PEB_S(dem_launch_fp64_raw(a, st));
        k_unpack<<<grid_for(n, 256), 256, 0, st>>>(n, pr_b, vw_b, uid_b, d_err, x_out, v_out,
                                                   w_out);
        PEB_S(cudaGetLastError());
    }
    int32_t herr = 0;
    PEB_S(cudaMemcpyAsync(&herr, d_err, sizeof herr, cudaMemcpyDeviceToHost, st));
    PEB_S(cudaStreamSynchronize(st));
#undef PEB_S
    if (herr & (SERR_RADIUS | SERR_MATERIAL)) return PE_B200_ERR_ARG;
    if (herr & DERR_NAN) return PE_B200_ERR_NAN;
    return PE_B200_OK;
}
