// rebuild.cuh -- the stages of the DEM neighbour-list rebuild as device code, run by every block
// of a cooperative grid with bounded grid barriers between them (rebuild.cu's k_rebuild, and the
// rebuild-and-contacts kernel of the list step in dem.cu):
//   clear cell counts | bin (cell key + slot, atomic histogram) | scan counts -> cell offsets |
//   scatter | order each cell by body index | gather bodies into cell order (the list buffers'
//   copy of the state, which the force kernels of the step read instead of the current one) |
//   count neighbours closer than r_i + r_j + skin (keeping the first few), mark the spheres that
//   can feel a force before the next rebuild | scan counts -> list offsets | scan marks -> the
//   marked spheres | write lists
// Every barrier wait is bounded: a block that waits too long sets an error flag and returns.
#pragma once

#include <algorithm>

#include "internal.cuh"

namespace peb {

namespace {


constexpr int kRbBlock = 256;

template <typename VT>
struct RebuildArgs {
    int64_t n, ncell;
    const SceneInfo *scenes;
    BodyBuf cur, tmp;   // the state, and its copy in cell order (the lists index the copy)
    int32_t *key, *rank, *sorted, *cell_count, *cell_start;
    int32_t *cnt, *start, *idx, *stash;
    int64_t cap;
    double skin;
    const double *boxes;   // fixed boxes (15 doubles each), for the marks of the list step
    int32_t *act, *alist;  // marks -> exclusive offsets (n + 1), the marked spheres
    float *disp;
    int32_t *flags;
    unsigned int *bar;   // [0] arrivals, [1] generation
    int32_t *blk;        // per-block partial sums (gridDim.x + 1)
    int32_t *err;
};

__device__ int block_sum(int v) {
    __shared__ int ws[kRbBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    int t = 0;
    if (threadIdx.x == 0)
        for (int k = 0; k < kRbBlock / 32; ++k) t += ws[k];
    __syncthreads();
    return t;  // valid in thread 0
}

// inclusive scan across the block; *total receives the block total
__device__ int block_incl_scan(int v, int *total) {
    __shared__ int ws[kRbBlock / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) ws[w] = v;
    __syncthreads();
    if (w == 0) {
        int x = (lane < kRbBlock / 32) ? ws[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += u;
        }
        if (lane < kRbBlock / 32) ws[lane] = x;
    }
    __syncthreads();
    const int r = v + (w > 0 ? ws[w - 1] : 0);
    *total = ws[kRbBlock / 32 - 1];
    __syncthreads();
    return r;
}

// exclusive scan of in[0, m) into out[0, m], out[m] = total, by every block of a cooperative
// grid of kRbBlock threads; blocks own contiguous chunks, blk holds gridDim.x + 1 partial sums.
// The caller puts a grid barrier after it before reading out.
__device__ bool grid_scan_raw(int32_t *blk, unsigned int *bar, int32_t *err, const int32_t *in,
                              int32_t *out, int64_t m) {
    const int64_t per = (m + gridDim.x - 1) / gridDim.x;
    const int64_t b0 = (int64_t)blockIdx.x * per;
    const int64_t b1 = (b0 + per < m) ? b0 + per : m;
    int s = 0;
    for (int64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x) s += in[i];
    s = block_sum(s);
    if (threadIdx.x == 0) blk[blockIdx.x] = s;
    if (!grid_sync(bar, err)) return false;
    if (blockIdx.x == 0) {
        int run = 0;
        for (int64_t base = 0; base < gridDim.x; base += blockDim.x) {
            const int64_t i = base + threadIdx.x;
            const int v = (i < gridDim.x) ? blk[i] : 0;
            int tot;
            const int incl = block_incl_scan(v, &tot);
            if (i < gridDim.x) blk[i] = run + incl - v;
            run += tot;
        }
        if (threadIdx.x == 0) out[m] = run;
    }
    if (!grid_sync(bar, err)) return false;
    int run = blk[blockIdx.x];
    for (int64_t base = b0; base < b1; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const int v = (i < b1) ? in[i] : 0;
        int tot;
        const int incl = block_incl_scan(v, &tot);
        if (i < b1) out[i] = run + incl - v;
        run += tot;
    }
    return true;
}

template <typename VT>
__device__ __forceinline__ bool grid_scan(const RebuildArgs<VT> &a, const int32_t *in, int32_t *out,
                                          int64_t m) {
    return grid_scan_raw(a.blk, a.bar, a.err, in, out, m);
}

// The cells within reach of body t (state in cell order): at most 3 x 3 rows of at most 3
// cells, since a partner is at most r_max + skin further and cells are wider than that.
struct Reach {
    double4 p;
    int32_t uid;
    int x0, x1, y0, y1, z0, z1;
    const SceneInfo *s;
};

template <typename VT>
__device__ __forceinline__ Reach reach_of(const RebuildArgs<VT> &a, int64_t t) {
    Reach q;
    q.p = a.tmp.pr[t];
    q.uid = a.tmp.uid[t];
    q.s = &a.scenes[a.tmp.tag[t] >> 16];
    const SceneInfo &s = *q.s;
    int cx, cy, cz;
    cell_coords(s, q.p.x, q.p.y, q.p.z, cx, cy, cz);
    const double reach = (q.p.w + s.rmax + a.skin) * (1.0 + 1e-12) + 1e-12;
    search_range(s, 0, q.p.x, reach, cx, q.x0, q.x1);
    search_range(s, 1, q.p.y, reach, cy, q.y0, q.y1);
    search_range(s, 2, q.p.z, reach, cz, q.z0, q.z1);
    return q;
}

__device__ __forceinline__ bool within(const double4 &pi, const double4 &pj, double skin) {
    const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    const double rc = pi.w + pj.w + skin;
    return dx * dx + dy * dy + dz * dz < rc * rc;
}

// list entry: the partner's slot, top bit set when body t has the smaller uid
template <typename VT>
__device__ __forceinline__ int32_t entry(const RebuildArgs<VT> &a, int32_t uidt, int j) {
    return (int32_t)((uint32_t)j | (uidt < a.tmp.uid[j] ? 0x80000000u : 0u));
}

// Emits neighbour k of body t: MODE 0 keeps the first kListStash in the stash, MODE 1 writes
// the list at pos.
template <int MODE, typename VT>
__device__ __forceinline__ void emit(const RebuildArgs<VT> &a, int64_t t, int pos, int k,
                                     int32_t v) {
    if (MODE == 1) a.idx[pos + k] = v;
    else if (k < kListStash) a.stash[(int64_t)k * a.n + t] = v;
}

// Neighbours of body t, row by row, one candidate at a time: MODE 0 counts (and stashes), 1
// writes.  The form for rows longer than 32 candidates.
template <int MODE, typename VT>
__device__ int neighbours_serial(const RebuildArgs<VT> &a, int64_t t, int pos, const Reach &q) {
    const SceneInfo &s = *q.s;
    int count = 0;
    for (int z = q.z0; z <= q.z1; ++z) {
        for (int y = q.y0; y <= q.y1; ++y) {
            const int64_t c0 = cell_key(s, q.x0, y, z);
            const int e = a.cell_start[c0 + (q.x1 - q.x0) + 1];
            for (int j = a.cell_start[c0]; j < e; ++j) {
                if (j == t || !within(q.p, a.tmp.pr[j], a.skin)) continue;
                emit<MODE>(a, t, pos, count, entry(a, q.uid, j));
                ++count;
            }
        }
    }
    return count;
}

// Neighbours of body t with the bounds of all rows loaded together and the rows' candidates
// visited in lockstep (candidate i of every row, then i + 1), so that up to nine position
// loads are in flight at once.  Hits are bits of per-row masks and are emitted in (z, y, slot)
// order: the same list, entry for entry, as the row-by-row scan.
template <int MODE, typename VT>
__device__ int list_neighbours(const RebuildArgs<VT> &a, int64_t t, int pos) {
    const Reach q = reach_of(a, t);
    const SceneInfo &s = *q.s;
    const int nx = q.x1 - q.x0 + 1;
    int b[9], len[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        const int y = q.y0 + r % 3, z = q.z0 + r / 3;
        b[r] = 0;
        len[r] = 0;
        if (y <= q.y1 && z <= q.z1) {
            const int64_t c0 = cell_key(s, q.x0, y, z);
            b[r] = a.cell_start[c0];
            len[r] = a.cell_start[c0 + nx] - b[r];
        }
    }
    int longest = 0;
#pragma unroll
    for (int r = 0; r < 9; ++r) longest = max(longest, len[r]);
    if (longest > 32) return neighbours_serial<MODE>(a, t, pos, q);
    uint32_t hit[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) hit[r] = 0u;
    for (int i = 0; i < longest; ++i) {
#pragma unroll
        for (int r = 0; r < 9; ++r) {
            if (i < len[r]) {
                const int j = b[r] + i;
                if (j != t && within(q.p, a.tmp.pr[j], a.skin)) hit[r] |= 1u << i;
            }
        }
    }
    int count = 0;
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        for (uint32_t m = hit[r]; m; m &= m - 1) {
            if (MODE == 0 && count >= kListStash) {
                count += __popc(m);
                break;
            }
            emit<MODE>(a, t, pos, count, entry(a, q.uid, b[r] + __ffs(m) - 1));
            ++count;
        }
    }
    return count;
}

// The rebuild's stages (the kernel has found a rebuild requested); every block of the
// cooperative grid runs them.  false: a grid barrier gave up (DERR_TIMEOUT is set).
template <typename VT>
__device__ bool rebuild_stages(const RebuildArgs<VT> &a) {
    const int64_t n = a.n;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t g0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    // 1. clear the cell counts
    for (int64_t i = g0; i <= a.ncell; i += stride) a.cell_count[i] = 0;
    if (!grid_sync(a.bar, a.err)) return false;
    // 2. bin
    for (int64_t i = g0; i < n; i += stride) {
        const double4 p = a.cur.pr[i];
        const SceneInfo &s = a.scenes[a.cur.tag[i] >> 16];
        int cx, cy, cz;
        cell_coords(s, p.x, p.y, p.z, cx, cy, cz);
        const int32_t k = (int32_t)cell_key(s, cx, cy, cz);
        a.key[i] = k;
        a.rank[i] = atomicAdd(&a.cell_count[k], 1);
    }
    if (!grid_sync(a.bar, a.err)) return false;
    // 3. cell offsets
    if (!grid_scan(a, a.cell_count, a.cell_start, a.ncell)) return false;
    if (!grid_sync(a.bar, a.err)) return false;
    // 4. scatter
    for (int64_t i = g0; i < n; i += stride) a.sorted[a.cell_start[a.key[i]] + a.rank[i]] = (int32_t)i;
    if (!grid_sync(a.bar, a.err)) return false;
    // 5. order each cell by body index (independent of the atomics' order)
    for (int64_t c = g0; c < a.ncell; c += stride) {
        const int b = a.cell_start[c], e = a.cell_start[c + 1];
        for (int i = b + 1; i < e; ++i) {
            const int32_t v = a.sorted[i];
            int j = i - 1;
            while (j >= b && a.sorted[j] > v) {
                a.sorted[j + 1] = a.sorted[j];
                --j;
            }
            a.sorted[j + 1] = v;
        }
    }
    if (!grid_sync(a.bar, a.err)) return false;
    // 6. gather into cell order
    for (int64_t t = g0; t < n; t += stride) {
        const int32_t b = a.sorted[t];
        a.tmp.pr[t] = a.cur.pr[b];
        cp_vw((VT *)a.tmp.vw, t, (const VT *)a.cur.vw, b, n);
        a.tmp.tag[t] = a.cur.tag[b];
        a.tmp.uid[t] = a.cur.uid[b];
        if (a.cur.q) a.tmp.q[t] = a.cur.q[b];
        a.disp[t] = 0.f;
    }
    if (!grid_sync(a.bar, a.err)) return false;
    // 7. neighbour counts; the first kListStash neighbours of each body are kept; the mark of
    // every sphere that can feel a force before the next rebuild
    const double margin = 0.5 * a.skin * (1.0 + 1e-9);
    for (int64_t t = g0; t < n; t += stride) {
        const int k = list_neighbours<0, VT>(a, t, 0);
        a.cnt[t] = k;
        const double4 p = a.tmp.pr[t];
        a.act[t] = list_marked(a.scenes[a.tmp.tag[t] >> 16], p, a.boxes, margin, k) ? 1 : 0;
    }
    if (!grid_sync(a.bar, a.err)) return false;
    // 8. list offsets, and the marked spheres in ascending order
    if (!grid_scan(a, a.cnt, a.start, n)) return false;
    if (!grid_sync(a.bar, a.err)) return false;
    if (!grid_scan(a, a.act, a.act, n)) return false;
    if (!grid_sync(a.bar, a.err)) return false;
    for (int64_t t = g0; t < n; t += stride)
        if (a.act[t + 1] > a.act[t]) a.alist[a.act[t]] = (int32_t)t;
    const int64_t need = a.start[n];
    if (g0 == 0) {
        a.flags[1] = need > a.cap ? 1 : 0;
        a.flags[2] = (int32_t)need;
        a.flags[3] += 1;
        a.flags[4] = 1;
        a.flags[0] = 0;
    }
    // 9. write the lists (if they fit; otherwise the force kernel searches the fresh grid):
    // copied from the stash, or searched again for bodies with more neighbours than it holds
    if (need <= a.cap)
        for (int64_t t = g0; t < n; t += stride) {
            const int k = a.cnt[t];
            if (k == 0) continue;
            const int pos = a.start[t];
            if (k > kListStash) {
                list_neighbours<1, VT>(a, t, pos);
                continue;
            }
            for (int i = 0; i < k; ++i) a.idx[pos + i] = a.stash[(int64_t)i * n + t];
        }
    return true;
}

// The rebuild's arguments for the context's current state and list buffers, and the grid of a
// rebuild kernel with `occ` resident blocks per SM (at most the blocks the partial sums hold).
template <typename VT>
int rebuild_setup(Ctx *c, int occ, RebuildArgs<VT> &a, unsigned *grid_out) {
    ListBuf &L = c->nl;
    const int64_t want = std::max<int64_t>(1, (c->n + kRbBlock - 1) / kRbBlock);
    const int per_sm = c->tune.rebuild_per_sm > 0 ? std::min(occ, c->tune.rebuild_per_sm) : occ;
    // the partial-sum buffer is allocated with the list buffers for the largest resident grid;
    // a grid never outgrows it (nothing is allocated here, inside a graph capture or not)
    if (!L.rb_blk || L.rb_blk_cap < 2)
        return set_err(c, PE_B200_ERR_STATE, "rebuild buffers not allocated");
    const unsigned grid = (unsigned)std::min<int64_t>(
        std::min<int64_t>(want, (int64_t)per_sm * c->sm_count), L.rb_blk_cap - 1);
    a.n = c->n;
    a.ncell = c->ncell;
    a.scenes = c->d_scenes;
    a.cur = c->cur;
    a.tmp = L.tmp;
    a.key = c->key;
    a.rank = c->rank;
    a.sorted = c->sorted;
    a.cell_count = c->cell_count;
    a.cell_start = c->cell_start;
    a.cnt = L.cnt;
    a.start = L.start;
    a.idx = L.idx;
    a.stash = L.stash;
    a.cap = L.cap;
    a.skin = L.skin;
    a.boxes = c->d_boxes;
    a.act = L.act;
    a.alist = L.alist;
    a.disp = L.disp;
    a.flags = L.flags;
    a.bar = L.rb_bar;
    a.blk = L.rb_blk;
    a.err = c->d_err;
    *grid_out = grid;
    return PE_B200_OK;
}

}  // namespace

}  // namespace peb
