// internal.cuh -- shared state, layouts and device helpers of libpe_b200.
//
// HBM layout (one context; all arrays in the internal body order, which is re-sorted by grid
// cell every step, so a CTA's bodies and their neighbours sit in a few cache lines):
//   pr   double4  (x, y, z, r)                        32 B / body, double-buffered
//   vw   VT[6]    (vx, vy, vz, wx, wy, wz)             48 B (FP64) or 24 B (mixed) / body
//   tag  uint32   material id | scene id << 16          4 B / body
//   uid  int32    upload index (pe creation order)      4 B / body
//   q    double4  orientation (only when tracked)      32 B / body
// Uniform grid per scene (cell >= largest AABB extent, pe/core/detection/coarse/HashGrids.h
// finds the same pair set): cell_count/cell_start are dense int32 arrays over all scenes' cells;
// key/rank hold every body's cell and its slot inside that cell for the next sort.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/pe_b200.h"

namespace peb {

constexpr double kContactThreshold = 1e-8;   // pe/core/Thresholds.h:151 (double)
constexpr float kContactThresholdF = 5e-7f;  // pe/core/Thresholds.h:103 (float)
constexpr double kFrictionThreshold = 1e-8;  // pe/core/Thresholds.h:161
constexpr int kMaxScenes = 65535;
constexpr int kMaxMaterials = 65535;
constexpr int kListStash = 8;   // neighbours per sphere the rebuild's counting pass keeps

struct SceneInfo {
    double lo[3];
    double h, inv_h;
    int32_t dim[3];
    int32_t pad0;
    int64_t cell_base;
    int32_t plane_begin, nplanes, box_begin, nboxes;
    int64_t body_begin, nbodies;   // in upload order
    // spheres whose extent lies inside [wall_lo, wall_hi] touch none of the scene's planes
    // (axis-aligned planes only; a scene with another plane has an empty box)
    double wall_lo[3], wall_hi[3];
    double rmax;                   // largest sphere radius of the scene at upload
    int32_t mbox_begin, nmbox;     // the scene's moving boxes (boxes.cu)
};

// per-material constants; reciprocals so a composed value is one division (Materials.h:633)
struct MatDev {
    double density;
    double rk, rcn, rct;   // 1/stiffness, 1/dampingN, 1/dampingT
    double csf, cdf;
    double young, poisson; // the extended Hertz law's effective modulus (Materials.h:586-600)
};

struct BodyBuf {
    double4 *pr = nullptr;
    void *vw = nullptr;
    uint32_t *tag = nullptr;
    int32_t *uid = nullptr;
    double4 *q = nullptr;
};

struct NbgsBuf {
    int64_t cap = 0;          // contact capacity
    // contact records (FP64 or FP32 by precision), struct-of-arrays in a single allocation
    void *cache = nullptr;
    int32_t *b1 = nullptr, *b2 = nullptr;     // internal slots; b2 < 0: wall
    int32_t *color = nullptr;                 // colour per contact
    int32_t *order = nullptr;                 // contacts sorted by colour
    int32_t *color_start = nullptr;           // host-visible after colouring
    int32_t *cnt = nullptr;                   // per-slot contact counts / offsets (N+1)
    int32_t *body_cnt = nullptr;              // per-body incident dynamic contacts (N+1)
    int32_t *body_adj = nullptr;              // body -> contacts CSR (2 * cap)
    uint64_t *used = nullptr;                 // colours used per body (bitmask)
    int32_t *flags = nullptr;                 // device counters (uncoloured, overflow, ...)
    int32_t *cstart_dev = nullptr;            // colour offsets on the device
    // device counters of a step the host does not wait on (nbgs.cu kDd*): capacity exceeded,
    // contacts needed, colours, largest colour, steps completed, ...
    int32_t *dd = nullptr;
    int32_t *h_dd = nullptr;                  // pinned mirror
    int32_t *rem = nullptr;                   // uncoloured contacts left after each colouring round
    unsigned int *bar2 = nullptr;             // grid barrier of the colouring rounds
    int32_t *slot_of = nullptr;               // per body: -1, or its claim in the compact sweep
    bool compact_off = false;                 // the compact sweep form cannot be launched
    bool staged_off = false;                  // nor the grid form with staged contacts
    bool on_device = false;                   // the last step's counts are only on the device
    bool plan_none = false;                   // queued steps planned without contacts
    bool warm = false;                        // a queued step has run on these buffers
    // captured CUDA graphs of queued steps, each valid for the buffers, settings, plan and
    // sweep grid in its key (nbgs.cu nbgs_graph_run); a miss replaces the least recently used
    struct GraphSlot {
        cudaGraphExec_t exec = nullptr;
        int64_t launches = 0;   // kernels per replay
        uint64_t used = 0;      // last use (gclock)
        uint64_t key[12] = {};
    };
    static constexpr int kGraphSlots = 4;
    GraphSlot gslot[kGraphSlots];
    uint64_t gclock = 0;
    bool gfailed = false;
    unsigned int *bar = nullptr;              // grid barrier of the persistent sweep
    bool coop_disabled = false;
    int cluster = -1;               // CTAs of the one-cluster sweep kernel (0: not available)
    // the sweep form with the bodies in one cluster's shared memory (nbgs.cu
    // launch_sweeps_dsmem): CTAs per cluster for the body count and kernel probed last (0: the
    // bodies do not fit)
    int64_t ds_nbod = -1;
    int ds_key = -1;
    int ds_size = 0;
    int ds_optin = 0;               // shared memory a block may opt in to
    void *vel = nullptr;                      // v', w', dv, dw per body (VT[12])
    int64_t nbod = 0;                         // bodies the per-body buffers hold
    bool gen = false;                         // they hold world-frame inverse inertias too
    double *red = nullptr;                    // reduction scratch
    int64_t red_cap = 0;
};

// Moving (non-fixed) boxes, FP64 (boxes.cu).  State arrays per box: x (3), q (4: w x y z),
// v (3), w (3), current and next step; props: 1/m, the body-frame inverse inertia diagonal (3),
// the body-frame inertia diagonal (3), unused (BoxBase.cpp:152-158, BoxBase.h:186-189).
struct MBoxBuf {
    int32_t m = 0;
    double *x = nullptr, *q = nullptr, *v = nullptr, *w = nullptr;
    double *x2 = nullptr, *q2 = nullptr, *v2 = nullptr, *w2 = nullptr;
    double *len = nullptr;     // side lengths, 3 per box
    double *props = nullptr;   // 8 per box
    int32_t *mat = nullptr, *scene = nullptr;
    int32_t *cnt = nullptr;    // contacts per box / offsets (m + 2)
    double *ext = nullptr;     // DEM: force and torque of the boxes on each sphere (6 per body),
                               // then the list of spheres near a box (n + 2 ints)
    int64_t ext_cap = 0;
    // per step: rotations (9 per box), bounding boxes (6 per box) and the box grid
    double *R = nullptr, *aabb = nullptr;
    double *gparm = nullptr;   // lo xyz, 1/h, dims
    int32_t *gstart = nullptr, *gfill = nullptr, *gids = nullptr, *gcell = nullptr;
    uint32_t *gnear = nullptr; // bit per cell: a box in it or in a neighbouring cell
};

// Verlet neighbour lists of the DEM step (dem_list.cu): every pair closer than r_i + r_j + skin
// at the last rebuild; valid while no sphere has moved more than skin/2 since then
struct ListBuf {
    bool enabled = false;
    double skin = 0.0;
    int64_t cap = 0;
    int32_t *start = nullptr;   // n + 1 (CSR offsets)
    int32_t *cnt = nullptr;     // n + 1
    int32_t *idx = nullptr;     // cap
    float *disp = nullptr;      // path length since the last rebuild
    int32_t *flags = nullptr;   // [0] rebuild requested, [1] list overflowed at this rebuild,
                                // [2] entries needed, [3] rebuild count
    int32_t *h_flags = nullptr; // pinned mirror
    cudaEvent_t ev = nullptr;
    bool check_pending = false;
    BodyBuf tmp;                // permutation target of a rebuild
    int32_t *stash = nullptr;   // kListStash x n, column-major: the first neighbours found by
                                // the counting pass of the persistent rebuild
    // spheres that can feel a force before the next rebuild (list entries, or near a wall):
    // exclusive offsets of the marks (n + 1; act[n] = count), the marked spheres in ascending
    // order, and their force and torque of the current step (6 x n of the precision's type)
    int32_t *act = nullptr;
    int32_t *alist = nullptr;
    void *facc = nullptr;
    // persistent rebuild kernel (rebuild.cu): grid barrier words and per-block partial sums
    unsigned int *rb_bar = nullptr;
    int32_t *rb_blk = nullptr;
    int64_t rb_blk_cap = 0;
    bool coop_disabled = false;
    bool fuse_off = false;   // the fused rebuild-and-contacts kernel cannot be launched here
    bool rebuild_pdl_off = false;  // the rebuild's cooperative launch without the early start
    bool warm = false;          // a list step has run since the buffers were (re)allocated
    int since_check = 1 << 20;  // steps since the last queued read-back of flags
};

// launch shapes of the DEM list step, picked by pe_b200_autotune (autotune.cu)
struct Tuning {
    int32_t dem_variant = 0;    // index into the k_dem_move launch shapes (dem.cu)
    int32_t rebuild_per_sm = 0; // persistent rebuild CTAs per SM; 0 = as many as fit
    int32_t nbgs_sweeps = 0;    // 0 automatic, 1 one cluster, 2 cooperative grid, 3 per colour,
                                // 4 one block, 5 bodies in one cluster's shared memory
    int32_t dem_grid = 0;       // grid step: 0 sorted FP32 candidate copy, 1 FP64 records only
    int32_t dem_split = 0;      // list step: 1 the marked spheres on a second stream (dem.cu)
};

// a captured CUDA graph of `steps` DEM list steps (dem.cu); valid while the buffers it was
// captured on and the context's parameter epoch are unchanged
struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    int32_t steps = 0;
    double dt = 0.0;
    uint64_t epoch = 0;
    const void *key[12] = {};
    int64_t launches = 0;       // kernels per replay
    bool failed = false;        // capture not possible here: plain launches from now on
};

// checkpoints of the adjoint's forward run (adjoint.cu)
struct AdjState {
    int32_t nsteps = 0, every = 1;
    double dt = 0.0;
    std::vector<BodyBuf> ckpt;   // state before steps 0, every, 2*every, ...
    std::vector<BodyBuf> seg;    // pre-step states of the segment being reversed
};

// stage timers (pe's profiling sections, e.g. DEMSolver.h:1159-1260): CUDA events around each
// stage on the context's stream, summed when queried
enum Stage : int {
    ST_SORT = 0, ST_DEM, ST_PERMUTE, ST_DETECT, ST_COLOR, ST_CACHE, ST_SWEEP, ST_INTEGRATE,
    ST_REBUILD, ST_COUNT
};
extern const char *kStageNames[ST_COUNT];

struct Ctx;
void prof_begin(Ctx *c, int stage);
void prof_end(Ctx *c, int stage);

struct Ctx {
    pe_b200_params p;
    std::string err;
    cudaStream_t stream = nullptr;
    // the split list step's second stream (higher priority: it runs the marked spheres' chain)
    // and its fork and join events
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool split_failed = false;
    // a second stream for the copies of a download (transfer.cu), created on first use
    cudaStream_t dl = nullptr;
    cudaEvent_t ev_dl0 = nullptr, ev_dl1 = nullptr;
    bool dl_failed = false;
    int device = 0;
    int sm_count = 148;
    int64_t launches = 0;

    // host copies
    std::vector<pe_b200_material> mats;
    std::vector<MatDev> mats_dev;   // host copy of d_mats
    std::vector<double> planes;     // 4 per plane, concatenated over scenes
    std::vector<int32_t> plane_mat;
    std::vector<double> boxes;      // 15 per box
    std::vector<int32_t> box_mat;
    std::vector<std::vector<double>> scene_planes, scene_boxes;
    std::vector<std::vector<int32_t>> scene_plane_mat, scene_box_mat;
    std::vector<SceneInfo> scenes;
    std::vector<double> plan_bounds;  // per scene: lo xyz, hi xyz of the grid (plan_grids)
    std::vector<double> plan_rmax;
    std::vector<int64_t> plan_count;

    // device
    int64_t n = 0;                  // bodies
    int32_t nscenes = 0;
    int64_t ncell = 0;              // total cells over scenes
    BodyBuf cur, nxt;
    int32_t *key = nullptr, *rank = nullptr, *sorted = nullptr;
    int32_t *cell_count = nullptr, *cell_start = nullptr;
    int32_t *scan_tmp = nullptr;
    int64_t scan_tmp_cap = 0;
    // the one-kernel grid sort (grid.cu): barrier counters, per-block partial sums for the
    // largest resident grid, and whether cooperative launches were refused here
    unsigned int *gs_bar = nullptr;
    int32_t *gs_blk = nullptr;
    int64_t gs_blk_cap = 0;
    bool gs_coop_off = false;
    float4 *posf = nullptr;         // grid step: FP32 positions relative to the grid origin and
                                    // radii, in the sort's slot order (grid_sort)
    int32_t *near = nullptr;        // grid step: per slot the count of candidates that passed
                                    // the FP32 test, then up to 16 of their slots (component-major)
    SceneInfo *d_scenes = nullptr;
    MatDev *d_mats = nullptr;
    double4 *d_planes = nullptr;    // (n, d)
    float4 *d_planes_f = nullptr;   // FP32 copy, inside the d_planes allocation
    int32_t *d_plane_mat = nullptr;
    double *d_boxes = nullptr;
    int32_t *d_box_mat = nullptr;
    int32_t *d_err = nullptr;       // device error word (bit flags)
    int32_t *h_err = nullptr;       // pinned mirror
    bool uploaded = false;
    bool binned = false;
    int64_t vw_bytes = 0;

    NbgsBuf nb;
    ListBuf nl;
    MBoxBuf mb;
    AdjState adj;
    Tuning tune;
    StepGraph sg;
    void *stage = nullptr;          // host-layout staging for uploads and downloads (transfer.cu)
    size_t stage_bytes = 0;
    int32_t graph_steps = 16;       // steps per graph replay; 0 = no graphs
    int64_t graph_captures = 0;     // graphs captured (DEM list and hard-contact steps)
    int64_t graph_replays = 0;      // graph launches
    uint64_t epoch = 1;             // bumped by every change that captured kernels bake in
    // profiling
    bool prof = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_open[ST_COUNT];
    cudaEvent_t ev_pending[ST_COUNT] = {};
    double prof_ms[ST_COUNT] = {};
    int64_t prof_count[ST_COUNT] = {};
    int64_t last_ncontacts = 0;
    int32_t last_ncolors = 0;
    double last_delta = -1.0, last_residual = -1.0;
    int32_t want_residual = 0;
};

// device error flags
enum : int32_t {
    DERR_CAPACITY = 1,
    DERR_NAN = 2,
    DERR_TIMEOUT = 4,
    DERR_CELL_OVERFLOW = 8,
    DERR_COLORS = 16,
};

// Device memory of a context comes from a stream-ordered pool per device that keeps what
// contexts free (abi.cu): a new context reuses the memory of the ones before it instead of
// mapping fresh pages.  dmalloc allocates on the context's stream, dfree frees there (nullptr
// allowed).
cudaError_t dmalloc_bytes(Ctx *c, void **p, size_t bytes);
void dfree(Ctx *c, void *p);
template <typename T>
inline cudaError_t dmalloc(Ctx *c, T **p, size_t bytes) {
    return dmalloc_bytes(c, reinterpret_cast<void **>(p), bytes);
}

int set_err(Ctx *c, int code, const std::string &msg);
int cuda_err(Ctx *c, cudaError_t e, const char *where);

#define PEB_CUDA(ctx, call)                                            \
    do {                                                               \
        cudaError_t e__ = (call);                                      \
        if (e__ != cudaSuccess) return ::peb::cuda_err(ctx, e__, #call); \
    } while (0)

#define PEB_LAUNCHED(ctx)                                                          \
    do {                                                                           \
        (ctx)->launches++;                                                         \
        cudaError_t e__ = cudaGetLastError();                                      \
        if (e__ != cudaSuccess) return ::peb::cuda_err(ctx, e__, "kernel launch"); \
    } while (0)

inline unsigned grid_for(int64_t n, int block) {
    return (unsigned)((n + block - 1) / block);
}

// grid-stride launches: at most 8 blocks per SM
unsigned capped_grid(const Ctx *c, int64_t n, int block);
#define GRID_STRIDE(i, n)                                                              \
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n);         \
         i += (int64_t)gridDim.x * blockDim.x)

// grid build: (re)bins bodies and sorts them by cell (grid.cu)
int grid_alloc(Ctx *c);
int grid_bin_current(Ctx *c);
// with_pos: also write posf (the FP32 positions in slot order) for the grid DEM step
int grid_sort(Ctx *c, bool with_pos = false);
int scan_exclusive(Ctx *c, const int32_t *in, int32_t *out, int64_t n);  // out[n] = total
int scan_exclusive_cond(Ctx *c, const int32_t *in, int32_t *out, int64_t n, const int32_t *cond);
int scan_reserve(Ctx *c, int64_t n);

// FP64 DEM step kernel on raw device buffers (layout as above; single launch, no allocation)
struct DemRawArgs {
    int64_t n;
    double dt, damping;
    double g[3];
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
    double4 *pr_out;
    double *vw_out;
    uint32_t *tag_out;
    int32_t *uid_out;
    int32_t *key, *rank, *cell_count, *err;
};
cudaError_t dem_launch_fp64_raw(const DemRawArgs &r, cudaStream_t stream);

// solvers
int dem_list_alloc(Ctx *c);
void dem_list_free(Ctx *c);
int dem_list_request_rebuild(Ctx *c);
int dem_list_rebuild_persistent(Ctx *c);
int dem_list_step(Ctx *c, double dt);
// runs whole graph replays of c->graph_steps list steps while they fit in nsteps; *done
// receives the steps run (0 when graphs are off or not possible)
int dem_list_graph_run(Ctx *c, int32_t nsteps, double dt, int32_t *done);
void dem_graph_free(Ctx *c);
int dem_variant_count();
// cells of every scene for neighbour-list skin `skin` (abi.cu)
void plan_cells(Ctx *c, double skin);
int upload_tables(Ctx *c);
// pe_b200_step's loop, shared with the autotuner
int run_steps(Ctx *c, int32_t nsteps, double dt);
// transfer.cu: the caller's arrays (upload order, interleaved xyz) <-> the device layout
int pack_bodies(Ctx *c, const double *x, const double *v, const double *w, const double *r,
                const int32_t *mat, const int32_t *scene);
int unpack_bodies(Ctx *c, double *x, double *v, double *w, double *q);
int scatter_state(Ctx *c, const double *x, const double *v, const double *w);
int scatter_orientations(Ctx *c, const double *q);
void stage_free(Ctx *c);
// autotune.cu
int set_list_skin(Ctx *c, double skin);
int set_tuning(Ctx *c, const Tuning &t, double skin);
int autotune(Ctx *c, double dt, int32_t trial, pe_b200_tuning *out);
int dem_step(Ctx *c, double dt);
int adjoint_forward(Ctx *c, int32_t nsteps, double dt, int32_t every);
int adjoint_backward(Ctx *c, const double *gx, const double *gv, const double *gw, double *ox,
                     double *ov, double *ow, double *gpar);
void adjoint_free(Ctx *c);
int nbgs_step(Ctx *c, double dt);
int nbgs_run(Ctx *c, int32_t nsteps, double dt);   // nsteps steps (retries aborted queued ones)
int find_contacts(Ctx *c, int64_t cap, int64_t *ids, double *geom, int64_t *n_out);
// boxes.cu: moving boxes
int mbox_upload(Ctx *c, int32_t m, const double *x, const double *q, const double *v,
                const double *w, const double *len, const int32_t *mat, const int32_t *scene);
int mbox_download(Ctx *c, double *x, double *q, double *v, double *w);
void mbox_free(Ctx *c);
// DEM: the boxes' forces on the spheres (mb.ext, by body index of the current buffers) and
// the boxes' own step into the next box buffers; the caller swaps them after the sphere step
int mbox_dem(Ctx *c, double dt);
void mbox_swap(Ctx *c);
// HCSITS (bodies n .. n+m-1 after the spheres): body cache, contacts (count, then write after
// the sphere contacts), integration
struct BodyCacheD {   // the FP64 body cache of the hard-contact step (slot order)
    double4 *vr, *wr, *dv, *dw, *ia, *ib, *ic;
};
int mbox_hc_bodycache(Ctx *c, const BodyCacheD &bv, double dt);
int mbox_hc_count(Ctx *c, int32_t *total);
int mbox_hc_raw(Ctx *c, int64_t base, int64_t cap, int32_t *b1, int32_t *b2, double *r1,
                double *r2, double *nrm, double *dist, double *mu);
int mbox_hc_integrate(Ctx *c, const BodyCacheD &bv, double dt);
// contacts involving moving boxes for pe_b200_find_contacts, in pe's orientation and ids
int mbox_find_contacts(Ctx *c, std::vector<int64_t> &ids, std::vector<double> &geom);

// body slots of the contacts of the last HCSITS step, in colour order (device memory)
const int2 *nbgs_ids_ptr(Ctx *c);
// validate.cu: host checks of the device state; each adds the problems it finds to *bad
int validate_coloring(Ctx *c, int64_t *bad);
int validate_lists(Ctx *c, int64_t *bad);
int selftest_timeout(Ctx *c, int64_t polls);
void nbgs_free(Ctx *c);
void nbgs_graph_free(Ctx *c);   // the captured hard-contact graphs

// ------------------------------------------------------------------------------------------
// device helpers
// ------------------------------------------------------------------------------------------
template <typename T>
struct V3 {
    T x, y, z;
};

template <typename T>
__host__ __device__ __forceinline__ V3<T> v3(T x, T y, T z) {
    return V3<T>{x, y, z};
}
template <typename T>
__host__ __device__ __forceinline__ V3<T> operator+(V3<T> a, V3<T> b) {
    return v3(a.x + b.x, a.y + b.y, a.z + b.z);
}
template <typename T>
__host__ __device__ __forceinline__ V3<T> operator-(V3<T> a, V3<T> b) {
    return v3(a.x - b.x, a.y - b.y, a.z - b.z);
}
template <typename T>
__host__ __device__ __forceinline__ V3<T> operator-(V3<T> a) {
    return v3(-a.x, -a.y, -a.z);
}
template <typename T>
__host__ __device__ __forceinline__ V3<T> operator*(V3<T> a, T s) {
    return v3(a.x * s, a.y * s, a.z * s);
}
template <typename T>
__host__ __device__ __forceinline__ V3<T> operator*(T s, V3<T> a) {
    return v3(s * a.x, s * a.y, s * a.z);
}
template <typename T>
__host__ __device__ __forceinline__ T dot(V3<T> a, V3<T> b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename T>
__host__ __device__ __forceinline__ V3<T> cross(V3<T> a, V3<T> b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <typename T>
__device__ __forceinline__ T vsqrt(T a);
template <>
__device__ __forceinline__ double vsqrt<double>(double a) { return sqrt(a); }
template <>
__device__ __forceinline__ float vsqrt<float>(float a) { return sqrtf(a); }

template <typename T>
__device__ __forceinline__ T length(V3<T> a) {
    return vsqrt<T>(a.x * a.x + a.y * a.y + a.z * a.z);
}
// Vector3::getNormalized (pe/math/Vector3.h:1025-1037)
template <typename T>
__device__ __forceinline__ V3<T> normalized(V3<T> a) {
    const T len = vsqrt<T>(a.x * a.x + a.y * a.y + a.z * a.z);
    if (len == T(0)) return a;
    const T il = T(1) / len;
    return v3(a.x * il, a.y * il, a.z * il);
}

// Length without fused multiply-adds, so a pair predicate evaluates exactly as pe's FP64 code
// (pe/math/Vector3.h:958) and the detected pair set matches bit for bit.
__device__ __forceinline__ double length_rn(double x, double y, double z) {
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
}
__device__ __forceinline__ double dot_rn(double ax, double ay, double az, double bx, double by,
                                         double bz) {
    return __dadd_rn(__dadd_rn(__dmul_rn(ax, bx), __dmul_rn(ay, by)), __dmul_rn(az, bz));
}

// velocities are component-major: component c (vx vy vz wx wy wz) of body i at vw[c * n + i].
// In mixed precision a seventh plane holds, per body, one extension byte for each linear
// component (bits 0-7 vx, 8-15 vy, 16-23 vz): the velocity is hi + e 2^-8 ulp(hi), hi the FP32
// component and e the signed byte.  A velocity that gains the same small increment every step
// (free flight: v += g dt) would round the same way step after step in 24 bits; with 32 bits
// the drift stays ~2^-33 per step.  Kernels that do not track the extension store it as zero.
constexpr int vw_planes(int bytes) { return bytes == 8 ? 6 : 7; }

template <typename T>
__device__ __forceinline__ V3<T> ld_vw(const T *vw, int64_t n, int64_t i, int which) {
    const T *p = vw + 3 * which * n + i;
    return v3(p[0], p[n], p[2 * n]);
}
__device__ __forceinline__ uint32_t ld_vext(const float *vw, int64_t n, int64_t i) {
    return reinterpret_cast<const uint32_t *>(vw + 6 * n)[i];
}
template <typename T>
__device__ __forceinline__ void st_vw(T *vw, int64_t n, int64_t i, V3<T> v, V3<T> w,
                                      uint32_t ext = 0u) {
    vw[i] = v.x;
    vw[n + i] = v.y;
    vw[2 * n + i] = v.z;
    vw[3 * n + i] = w.x;
    vw[4 * n + i] = w.y;
    vw[5 * n + i] = w.z;
    if constexpr (sizeof(T) == 4) reinterpret_cast<uint32_t *>(vw + 6 * n)[i] = ext;
}
template <typename T>
__device__ __forceinline__ void cp_vw(T *dst, int64_t i, const T *src, int64_t j, int64_t n) {
#pragma unroll
    for (int c = 0; c < 6; ++c) dst[c * n + i] = src[c * n + j];
    if constexpr (sizeof(T) == 4)
        reinterpret_cast<uint32_t *>(dst + 6 * n)[i] =
            reinterpret_cast<const uint32_t *>(src + 6 * n)[j];
}
// 2^-8 ulp(hi) as a double (zero and subnormal hi use the smallest normal exponent)
__device__ __forceinline__ double vext_unit(float hi) {
    const int ex = max((int)((__float_as_uint(hi) >> 23) & 0xffu), 1);
    return __longlong_as_double((long long)(ex - 158 + 1023) << 52);
}
// the FP64 value of component c of an extended velocity
__device__ __forceinline__ double vext_value(float hi, uint32_t ext, int c) {
    const int e = (int)(int8_t)(uint8_t)((ext >> (8 * c)) & 0xffu);
    return double(hi) + double(e) * vext_unit(hi);
}
// 2^8 / ulp(hi), the reciprocal of vext_unit (a power of two, so multiplying by it is exact)
__device__ __forceinline__ double vext_inv_unit(float hi) {
    const int ex = max((int)((__float_as_uint(hi) >> 23) & 0xffu), 1);
    return __longlong_as_double((long long)(158 - ex + 1023) << 52);
}
// FP64 velocity component -> FP32 component (round to nearest), its extension byte or-ed into
// ext at position c.  v - hi is exact, and so is the scaling by a power of two.
__device__ __forceinline__ float vext_split(double v, uint32_t &ext, int c) {
    const float hi = __double2float_rn(v);
    const double r = (v - double(hi)) * vext_inv_unit(hi);
    int e = isfinite(r) ? (int)rint(r) : 0;
    e = max(-127, min(127, e));
    ext |= ((uint32_t)(uint8_t)(int8_t)e) << (8 * c);
    return hi;
}

__device__ __forceinline__ void sphere_mass(double r, double density, double &im, double &ii,
                                            double &I) {
    // SphereBase.h:169-171, SphereBase.cpp:79-80, SphereBase.h:230-234 + Matrix3x3::getInverse
    const double mass = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(4.0 / 3.0, 3.14159265358979323846), r), r), r);
    const double m2 = __dmul_rn(mass, density);
    const double Iv = __dmul_rn(__dmul_rn(__dmul_rn(0.4, m2), r), r);
    const double I2 = __dmul_rn(Iv, Iv);
    const double det = __ddiv_rn(1.0, __dmul_rn(Iv, I2));
    im = __ddiv_rn(1.0, m2);
    ii = __dmul_rn(det, I2);
    I = Iv;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

__device__ __forceinline__ void cell_coords(const SceneInfo &s, double x, double y, double z,
                                            int &cx, int &cy, int &cz) {
    cx = clampi((int)floor((x - s.lo[0]) * s.inv_h), 0, s.dim[0] - 1);
    cy = clampi((int)floor((y - s.lo[1]) * s.inv_h), 0, s.dim[1] - 1);
    cz = clampi((int)floor((z - s.lo[2]) * s.inv_h), 0, s.dim[2] - 1);
}

// Cells along axis `a` that can hold a body closer than `reach` to coordinate p, whose own
// (clamped) cell is c: the clamped cells of p - reach and p + reach, never more than one cell
// either side of c since cell edges are at least 2 r_max + skin.
__device__ __forceinline__ void search_range(const SceneInfo &s, int a, double p, double reach,
                                             int c, int &lo, int &hi) {
    const int l = clampi((int)floor((p - reach - s.lo[a]) * s.inv_h), 0, s.dim[a] - 1);
    const int h = clampi((int)floor((p + reach - s.lo[a]) * s.inv_h), 0, s.dim[a] - 1);
    lo = max(l, c - 1);
    hi = min(h, c + 1);
}

__device__ __forceinline__ int64_t cell_key(const SceneInfo &s, int cx, int cy, int cz) {
    return s.cell_base + ((int64_t)cz * s.dim[1] + cy) * s.dim[0] + cx;
}

// Whether a sphere can feel a force before the next neighbour-list rebuild (the list step's
// marked spheres, dem.cu): it has list entries, or a wall may come within reach while it moves
// less than `margin` (half the skin) -- it is not inside the box of its scene's axis-aligned
// planes by r + margin (wall_forces then tests the planes), or it is within r + margin of the
// bounding sphere of one of the scene's fixed boxes (wall_forces tests every box).
__device__ __forceinline__ bool list_marked(const SceneInfo &s, const double4 &p,
                                            const double *boxes, double margin, int cnt) {
    if (cnt > 0) return true;
    const double r = p.w + margin;
    const bool clear = p.x - r > s.wall_lo[0] && p.x + r < s.wall_hi[0] &&
                       p.y - r > s.wall_lo[1] && p.y + r < s.wall_hi[1] &&
                       p.z - r > s.wall_lo[2] && p.z + r < s.wall_hi[2];
    if (!clear) return true;
    for (int k = 0; k < s.nboxes; ++k) {
        const double *B = boxes + 15 * (int64_t)(s.box_begin + k);
        const double hx = 0.5 * B[3], hy = 0.5 * B[4], hz = 0.5 * B[5];
        const double reach = (sqrt(hx * hx + hy * hy + hz * hz) + r) * (1.0 + 1e-9);
        const double dx = p.x - B[0], dy = p.y - B[1], dz = p.z - B[2];
        if (dx * dx + dy * dy + dz * dz < reach * reach) return true;
    }
    return false;
}

// Programmatic dependent launch: a kernel launched with the programmatic-serialization
// attribute may be scheduled while the kernel before it in the stream still runs; pdl_wait()
// returns once that kernel has completed and its writes are visible (at once when the launch
// had no such attribute), and pdl_trigger() lets the kernel after this one be scheduled early.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;"); }

// Grid-wide barrier for cooperative launches, with a bounded wait: a block that waits longer
// than ~2 s records DERR_TIMEOUT and every thread of it sees false.  bar[0] counts arrivals,
// bar[1] is the generation; both start at 0 and are left consistent after a completed barrier.
constexpr unsigned long long kSpinLimit = 1ull << 24;  // polls of ~100 ns each
__device__ __forceinline__ bool grid_sync(unsigned int *bar, int32_t *err) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int *vgen = bar + 1;
        const unsigned int gen = *vgen;
        __threadfence();
        const unsigned int arrived = atomicAdd(bar, 1u);
        int ok = 1;
        if (arrived == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            // poll hot for the first few thousand rounds (barriers between short stages end
            // within microseconds), then back off
            unsigned long long spins = 0;
            while (*vgen == gen) {
                if (++spins > 4096) __nanosleep(128);
                if (spins > kSpinLimit) {
                    ok = 0;
                    atomicOr(err, DERR_TIMEOUT);
                    break;
                }
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Grid-wide barrier on a counter that only grows within one launch (the caller zeroes it
// before the launch): a block's arrival is one release-add, and a block leaves once an
// acquire-load sees every block of this and all earlier episodes arrived.  Compared with
// grid_sync there is no reset and no second word the last block has to publish, so a barrier
// costs about one L2 round trip less.  *episode is the calling block's barrier count (thread 0
// keeps it).  The wait is bounded like grid_sync's.
__device__ __forceinline__ bool grid_sync_counted(unsigned int *count, unsigned int &episode,
                                                  int32_t *err) {
    __shared__ int s_ok2;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int target = (++episode) * gridDim.x;
        asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(count), "r"(1u) : "memory");
        unsigned int v = 0;
        unsigned long long spins = 0;
        int ok = 1;
        for (;;) {
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(count) : "memory");
            if (v >= target) break;
            if (++spins > 4096) __nanosleep(64);
            if (spins > kSpinLimit) {
                ok = 0;
                atomicOr(err, DERR_TIMEOUT);
                break;
            }
        }
        s_ok2 = ok;
    }
    __syncthreads();
    return s_ok2 != 0;
}

}  // namespace peb
