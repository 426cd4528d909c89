// grid.cu -- uniform-grid build as a counting sort of cell keys.
//
// pe's coarse detector (pe/core/detection/coarse/HashGrids.h:1121-1314) re-hashes every body
// into hierarchical hash grids and walks cell pairs with pointer-chasing.  Here the grid is a
// dense per-scene array of int32 cells with a cell at least the largest AABB extent, so every
// AABB-overlapping pair lies in neighbouring cells.  The sort is:
//   count  (atomic histogram; the producing step kernel already did this for the next step)
//   scan   (exclusive prefix sum over cells -> cell_start)
//   scatter(slot of body i = cell_start[key[i]] + rank[i])
//   fixup  (order each cell by body index, so the result is independent of atomic order)
// Outside graph captures the three run in one cooperative kernel (k_grid_sort) with bounded grid
// barriers between them, which also clears the counts for the next step; in a capture, and with
// rebuild_per_sm = -1 (no cooperative launches), they run as separate kernels.  Both give the
// same arrays.
#include "rebuild.cuh"

namespace peb {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int warp_incl_scan(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// exclusive scan of one tile; block total to tile_sums[blockIdx.x]
__global__ void __launch_bounds__(kScanThreads) k_scan_tile(const int32_t *__restrict__ in,
                                                            int32_t *__restrict__ out, int64_t n,
                                                            int32_t *__restrict__ tile_sums,
                                                            const int32_t *cond) {
    if (cond && !*cond) return;
    __shared__ int warp_tot[kScanThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + k;
        v[k] = (i < n) ? in[i] : 0;
        s += v[k];
    }
    const int incl = warp_incl_scan(s);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int t = (lane < kScanThreads / 32) ? warp_tot[lane] : 0;
        t = warp_incl_scan(t);
        if (lane < kScanThreads / 32) warp_tot[lane] = t;
    }
    __syncthreads();
    int run = incl - s + (warp > 0 ? warp_tot[warp - 1] : 0);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
    if (threadIdx.x == kScanThreads - 1) tile_sums[blockIdx.x] = run;
}

__global__ void k_scan_add(int32_t *__restrict__ out, int64_t n,
                           const int32_t *__restrict__ tile_off, const int32_t *cond) {
    if (cond && !*cond) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] += tile_off[i / kScanTile];
}

__global__ void k_set_total(int32_t *out, int64_t n, const int32_t *last_in,
                            const int32_t *last_out, const int32_t *cond) {
    if (cond && !*cond) return;
    out[n] = (n > 0) ? (*last_out + *last_in) : 0;
}

__global__ void k_bin(int64_t n, const double4 *__restrict__ pr, const uint32_t *__restrict__ tag,
                      const SceneInfo *__restrict__ scenes, int32_t *__restrict__ key,
                      int32_t *__restrict__ rank, int32_t *__restrict__ cell_count) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 p = pr[i];
    const SceneInfo &s = scenes[tag[i] >> 16];
    int cx, cy, cz;
    cell_coords(s, p.x, p.y, p.z, cx, cy, cz);
    const int32_t k = (int32_t)cell_key(s, cx, cy, cz);
    key[i] = k;
    rank[i] = atomicAdd(&cell_count[k], 1);
}

__global__ void k_scatter(int64_t n, const int32_t *__restrict__ key,
                          const int32_t *__restrict__ rank, const int32_t *__restrict__ start,
                          int32_t *__restrict__ sorted) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    sorted[start[key[i]] + rank[i]] = (int32_t)i;
}

// one cell's insertion sort by body index, and its FP32 position records (posf non-null)
__device__ __forceinline__ void fixup_cell(int64_t c, const int32_t *start, int32_t *sorted,
                                           const double4 *pr, const uint32_t *tag,
                                           const SceneInfo *scenes, float4 *posf) {
    const int b = start[c], e = start[c + 1];
    if (e == b) return;
    for (int i = b + 1; i < e; ++i) {
        const int32_t v = sorted[i];
        int j = i - 1;
        while (j >= b && sorted[j] > v) {
            sorted[j + 1] = sorted[j];
            --j;
        }
        sorted[j + 1] = v;
    }
    if (!posf) return;
    for (int i = b; i < e; ++i) {
        const int32_t j = sorted[i];
        const double4 p = pr[j];
        const SceneInfo &s = scenes[tag[j] >> 16];
        posf[i] = make_float4(float(p.x - s.lo[0]), float(p.y - s.lo[1]), float(p.z - s.lo[2]),
                              float(p.w));
    }
}

// insertion sort of each cell's slots by body index (cells hold a handful of bodies); with
// posf, the cell's bodies' positions relative to their scene's grid origin and radii in FP32,
// in slot order (the candidate records of the grid DEM step)
__global__ void k_fixup(int64_t ncell, const int32_t *__restrict__ start,
                        int32_t *__restrict__ sorted, const double4 *__restrict__ pr,
                        const uint32_t *__restrict__ tag, const SceneInfo *__restrict__ scenes,
                        float4 *__restrict__ posf) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    fixup_cell(c, start, sorted, pr, tag, scenes, posf);
}

struct GridSortArgs {
    int64_t n, ncell;
    int32_t *cell_count, *cell_start, *key, *rank, *sorted;
    const double4 *pr;
    const uint32_t *tag;
    const SceneInfo *scenes;
    float4 *posf;
    unsigned int *bar;
    int32_t *blk, *err;
};

// the whole sort in one cooperative grid: scan | scatter, clear the counts | per-cell order
__global__ void __launch_bounds__(kRbBlock) k_grid_sort(GridSortArgs g) {
    if (!grid_scan_raw(g.blk, g.bar, g.err, g.cell_count, g.cell_start, g.ncell)) return;
    if (!grid_sync(g.bar, g.err)) return;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t g0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int64_t i = g0; i < g.n; i += stride) g.sorted[g.cell_start[g.key[i]] + g.rank[i]] = (int32_t)i;
    // the scan has read every count: cleared for the step kernel, which bins for the next sort
    for (int64_t c = g0; c <= g.ncell; c += stride) g.cell_count[c] = 0;
    if (!grid_sync(g.bar, g.err)) return;
    for (int64_t c = g0; c < g.ncell; c += stride)
        fixup_cell(c, g.cell_start, g.sorted, g.pr, g.tag, g.scenes, g.posf);
}

}  // namespace

// sizes the scan scratch for inputs of up to n elements (so a later scan allocates nothing)
int scan_reserve(Ctx *c, int64_t n) {
    int64_t m = n, need = 0;
    while (true) {
        const int64_t tiles = (m + kScanTile - 1) / kScanTile;
        need += tiles + 1;
        if (tiles <= 1) break;
        m = tiles;
    }
    if (need + 1 > c->scan_tmp_cap) {
        if (c->scan_tmp) dfree(c, c->scan_tmp);
        c->scan_tmp = nullptr;
        PEB_CUDA(c, dmalloc(c, &c->scan_tmp, (size_t)(need + 1) * sizeof(int32_t)));
        c->scan_tmp_cap = need + 1;
    }
    return PE_B200_OK;
}

int scan_exclusive(Ctx *c, const int32_t *in, int32_t *out, int64_t n) {
    return scan_exclusive_cond(c, in, out, n, nullptr);
}

// cond (device int, may be null): when it holds 0 every kernel of the scan returns at once
int scan_exclusive_cond(Ctx *c, const int32_t *in, int32_t *out, int64_t n, const int32_t *cond) {
    // recursive reduce-then-scan; scratch holds every level's tile sums
    std::vector<int64_t> sizes;
    int64_t m = n;
    int64_t need = 0;
    while (true) {
        const int64_t tiles = (m + kScanTile - 1) / kScanTile;
        sizes.push_back(m);
        need += tiles + 1;
        if (tiles <= 1) break;
        m = tiles;
    }
    if (need + 1 > c->scan_tmp_cap) {
        if (c->scan_tmp) dfree(c, c->scan_tmp);
        c->scan_tmp = nullptr;
        PEB_CUDA(c, dmalloc(c, &c->scan_tmp, (size_t)(need + 1) * sizeof(int32_t)));
        c->scan_tmp_cap = need + 1;
    }
    // the last input element, kept for the total (the scan may run in place)
    int32_t *last_in = c->scan_tmp + need;
    if (n > 0)
        PEB_CUDA(c, cudaMemcpyAsync(last_in, in + n - 1, sizeof(int32_t), cudaMemcpyDeviceToDevice,
                                    c->stream));
    // level 0 ... L-1: scan, recording tile sums in scan_tmp
    std::vector<int32_t *> lvl_in, lvl_out, lvl_sums;
    const int32_t *cur_in = in;
    int32_t *cur_out = out;
    int32_t *tmp = c->scan_tmp;
    for (size_t l = 0; l < sizes.size(); ++l) {
        const int64_t len = sizes[l];
        const int64_t tiles = (len + kScanTile - 1) / kScanTile;
        int32_t *sums = tmp;
        tmp += tiles + 1;
        if (len > 0) {
            k_scan_tile<<<(unsigned)tiles, kScanThreads, 0, c->stream>>>(cur_in, cur_out, len, sums,
                                                                          cond);
            PEB_LAUNCHED(c);
        }
        lvl_out.push_back(cur_out);
        lvl_sums.push_back(sums);
        if (tiles <= 1) break;
        cur_in = sums;
        cur_out = sums;  // scanned in place at the next level (the tile kernel reads before writing)
    }
    // propagate offsets downwards
    for (int l = (int)lvl_out.size() - 2; l >= 0; --l) {
        const int64_t len = sizes[l];
        k_scan_add<<<capped_grid(c, len, 256), 256, 0, c->stream>>>(lvl_out[l], len, lvl_sums[l], cond);
        PEB_LAUNCHED(c);
    }
    k_set_total<<<1, 1, 0, c->stream>>>(out, n, last_in, out + (n > 0 ? n - 1 : 0), cond);
    PEB_LAUNCHED(c);
    return PE_B200_OK;
}

int grid_alloc(Ctx *c) {
    const size_t n = (size_t)c->n;
    if (!c->gs_bar) {
        PEB_CUDA(c, dmalloc(c, &c->gs_bar, 2 * sizeof(unsigned int)));
        PEB_CUDA(c, cudaMemsetAsync(c->gs_bar, 0, 2 * sizeof(unsigned int), c->stream));
        int tpsm = 2048;
        if (cudaDeviceGetAttribute(&tpsm, cudaDevAttrMaxThreadsPerMultiProcessor, c->device) !=
            cudaSuccess || tpsm < kRbBlock) {
            cudaGetLastError();
            tpsm = 2048;
        }
        c->gs_blk_cap = (int64_t)(tpsm / kRbBlock) * std::max(c->sm_count, 1) + 1;
        PEB_CUDA(c, dmalloc(c, &c->gs_blk, (size_t)c->gs_blk_cap * sizeof(int32_t)));
    }
    // the scan scratch of every scan a step runs (cells, bodies and moving boxes, list counts),
    // sized here so that no step allocates it inside a graph capture
    int rc = scan_reserve(c, std::max<int64_t>(c->ncell + 1, 2 * c->n + 1024));
    if (rc) return rc;
    PEB_CUDA(c, dmalloc(c, &c->key, n * sizeof(int32_t) + 16));
    PEB_CUDA(c, dmalloc(c, &c->rank, n * sizeof(int32_t) + 16));
    PEB_CUDA(c, dmalloc(c, &c->sorted, n * sizeof(int32_t) + 16));
    PEB_CUDA(c, dmalloc(c, &c->cell_count, ((size_t)c->ncell + 1) * sizeof(int32_t)));
    PEB_CUDA(c, dmalloc(c, &c->cell_start, ((size_t)c->ncell + 2) * sizeof(int32_t)));
    return PE_B200_OK;
}

int grid_bin_current(Ctx *c) {
    PEB_CUDA(c, cudaMemsetAsync(c->cell_count, 0, ((size_t)c->ncell + 1) * sizeof(int32_t),
                                c->stream));
    if (c->n > 0) {
        k_bin<<<grid_for(c->n, 256), 256, 0, c->stream>>>(c->n, c->cur.pr, c->cur.tag,
                                                          c->d_scenes, c->key, c->rank,
                                                          c->cell_count);
        PEB_LAUNCHED(c);
    }
    c->binned = true;
    return PE_B200_OK;
}

// cell_count/key/rank describe the current body order -> cell_start + sorted;
// cell_count is cleared for the producing kernel of this step.
int grid_sort(Ctx *c, bool with_pos) {
    prof_begin(c, ST_SORT);
    // one cooperative kernel for steps launched one by one; inside a graph capture the separate
    // kernels (cheap to launch from a graph) measured faster than the kernel's grid barriers
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(c->stream, &cap) != cudaSuccess) {
        cudaGetLastError();
        cap = cudaStreamCaptureStatusActive;
    }
    if (cap == cudaStreamCaptureStatusNone && !c->gs_coop_off && c->gs_blk &&
        c->tune.rebuild_per_sm >= 0 && c->ncell > 0) {
        static int occ = 0;
        if (occ == 0 &&
            (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_grid_sort, kRbBlock, 0) !=
                 cudaSuccess || occ < 1)) {
            cudaGetLastError();
            occ = 0;
            c->gs_coop_off = true;
        }
        if (occ > 0) {
            const int64_t work = std::max<int64_t>(c->ncell, c->n);
            const int64_t want = std::max<int64_t>(1, (work + kRbBlock - 1) / kRbBlock);
            const unsigned grid = (unsigned)std::min<int64_t>(
                std::min<int64_t>(want, (int64_t)occ * c->sm_count), c->gs_blk_cap - 1);
            GridSortArgs g;
            g.n = c->n;
            g.ncell = c->ncell;
            g.cell_count = c->cell_count;
            g.cell_start = c->cell_start;
            g.key = c->key;
            g.rank = c->rank;
            g.sorted = c->sorted;
            g.pr = c->cur.pr;
            g.tag = c->cur.tag;
            g.scenes = c->d_scenes;
            g.posf = with_pos ? c->posf : nullptr;
            g.bar = c->gs_bar;
            g.blk = c->gs_blk;
            g.err = c->d_err;
            void *args[] = {&g};
            if (cudaLaunchCooperativeKernel((const void *)k_grid_sort, dim3(grid), dim3(kRbBlock),
                                            args, 0, c->stream) == cudaSuccess) {
                c->launches++;
                prof_end(c, ST_SORT);
                return PE_B200_OK;
            }
            // refused (e.g. a shared device that allows no cooperative launches): the separate
            // kernels from now on
            cudaGetLastError();
            c->gs_coop_off = true;
        }
    }
    int rc = scan_exclusive(c, c->cell_count, c->cell_start, c->ncell);
    if (rc) return rc;
    if (c->n > 0) {
        k_scatter<<<grid_for(c->n, 256), 256, 0, c->stream>>>(c->n, c->key, c->rank,
                                                              c->cell_start, c->sorted);
        PEB_LAUNCHED(c);
        k_fixup<<<grid_for(c->ncell, 256), 256, 0, c->stream>>>(
            c->ncell, c->cell_start, c->sorted, c->cur.pr, c->cur.tag, c->d_scenes,
            with_pos ? c->posf : nullptr);
        PEB_LAUNCHED(c);
    }
    PEB_CUDA(c, cudaMemsetAsync(c->cell_count, 0, ((size_t)c->ncell + 1) * sizeof(int32_t),
                                c->stream));
    prof_end(c, ST_SORT);
    return PE_B200_OK;
}

}  // namespace peb
