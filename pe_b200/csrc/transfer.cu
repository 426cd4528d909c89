// transfer.cu -- host <-> device body state in pe's creation order.
//
// The caller's arrays (interleaved xyz doubles per sphere, in upload order) are copied to a
// device staging area as they are, and kernels convert between that layout and the internal
// one (double4 position+radius, component-major velocities in the step's precision, bodies in
// the cell order of the last list rebuild).  The host then moves only the bytes the caller
// passes or asks for, in one copy per array, and no host loop touches every sphere.
#include <algorithm>

#include "internal.cuh"

namespace peb {

namespace {

// a body's velocities from a caller's FP64 linear velocity (3 doubles) and angular velocity;
// in mixed precision the linear one keeps its extension bytes
template <typename VT>
__device__ __forceinline__ void st_vw_in(VT *vw, int64_t n, int64_t i, const double *v,
                                         V3<VT> w) {
    if constexpr (sizeof(VT) == 4) {
        uint32_t ext = 0u;
        V3<float> a;
        a.x = vext_split(v[0], ext, 0);
        a.y = vext_split(v[1], ext, 1);
        a.z = vext_split(v[2], ext, 2);
        st_vw(vw, n, i, a, w, ext);
    } else {
        st_vw(vw, n, i, v3(v[0], v[1], v[2]), w);
    }
}

template <typename VT>
__global__ void k_pack(int64_t n, const double *x, const double *v, const double *w,
                       const double *r, const int32_t *mat, const int32_t *scene, double4 *pr,
                       VT *vw, uint32_t *tag, int32_t *uid, double4 *q) {
    GRID_STRIDE(i, n) {
        pr[i] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], r[i]);
        st_vw_in(vw, n, i, v + 3 * i, v3(VT(w[3 * i]), VT(w[3 * i + 1]), VT(w[3 * i + 2])));
        tag[i] = (uint32_t)mat[i] | ((uint32_t)(scene ? scene[i] : 0) << 16);
        uid[i] = (int32_t)i;
        if (q) q[i] = make_double4(1.0, 0.0, 0.0, 0.0);
    }
}

template <typename VT>
__global__ void k_unpack(int64_t n, const double4 *pr, const VT *vw, const int32_t *uid,
                         const double4 *q, double *x, double *v, double *w, double *qo) {
    GRID_STRIDE(t, n) {
        const int64_t i = uid[t];
        const double4 p = pr[t];
        x[3 * i] = p.x;
        x[3 * i + 1] = p.y;
        x[3 * i + 2] = p.z;
        const V3<VT> a = ld_vw(vw, n, t, 0), b = ld_vw(vw, n, t, 1);
        if constexpr (sizeof(VT) == 4) {
            const uint32_t ext = ld_vext(vw, n, t);
            v[3 * i] = vext_value(a.x, ext, 0);
            v[3 * i + 1] = vext_value(a.y, ext, 1);
            v[3 * i + 2] = vext_value(a.z, ext, 2);
        } else {
            v[3 * i] = a.x;
            v[3 * i + 1] = a.y;
            v[3 * i + 2] = a.z;
        }
        w[3 * i] = b.x;
        w[3 * i + 1] = b.y;
        w[3 * i + 2] = b.z;
        if (q) {
            const double4 o = q[t];
            qo[4 * i] = o.x;
            qo[4 * i + 1] = o.y;
            qo[4 * i + 2] = o.z;
            qo[4 * i + 3] = o.w;
        }
    }
}

// overwrite x, v, w (each may be absent) of the bodies from arrays in upload order
template <typename VT>
__global__ void k_scatter_state(int64_t n, const int32_t *uid, const double *x, const double *v,
                                const double *w, double4 *pr, VT *vw) {
    GRID_STRIDE(t, n) {
        const int64_t i = uid[t];
        if (x) {
            const double4 p = pr[t];
            pr[t] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], p.w);
        }
        const V3<VT> b = w ? v3(VT(w[3 * i]), VT(w[3 * i + 1]), VT(w[3 * i + 2])) : ld_vw(vw, n, t, 1);
        if (v) {
            st_vw_in(vw, n, t, v + 3 * i, b);
        } else {
            const V3<VT> a = ld_vw(vw, n, t, 0);
            if constexpr (sizeof(VT) == 4) st_vw(vw, n, t, a, b, ld_vext(vw, n, t));
            else st_vw(vw, n, t, a, b);
        }
    }
}

// overwrite the orientations (w x y z per body, upload order) of the bodies
__global__ void k_scatter_q(int64_t n, const int32_t *uid, const double *q, double4 *qd) {
    GRID_STRIDE(t, n) {
        const int64_t i = uid[t];
        qd[t] = make_double4(q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]);
    }
}

int stage_reserve(Ctx *c, size_t bytes) {
    if (c->stage_bytes >= bytes) return PE_B200_OK;
    dfree(c, c->stage);
    c->stage = nullptr;
    c->stage_bytes = 0;
    PEB_CUDA(c, dmalloc(c, &c->stage, bytes));
    c->stage_bytes = bytes;
    return PE_B200_OK;
}

// staging layout: x, v, w (3n doubles each), then r or q, then two int arrays
struct StageView {
    double *x, *v, *w, *r;
    int32_t *mat, *scene;
};

StageView stage_layout(Ctx *c) {
    const size_t n = (size_t)c->n;
    StageView s;
    s.x = (double *)c->stage;
    s.v = s.x + 3 * n;
    s.w = s.v + 3 * n;
    s.r = s.w + 3 * n;                 // n (upload) or 4n (orientations)
    s.mat = (int32_t *)(s.r + 4 * n);
    s.scene = s.mat + n;
    return s;
}

size_t stage_size(int64_t n) { return (size_t)std::max<int64_t>(n, 1) * (13 * sizeof(double) + 2 * sizeof(int32_t)); }

}  // namespace

int pack_bodies(Ctx *c, const double *x, const double *v, const double *w, const double *r,
                const int32_t *mat, const int32_t *scene) {
    const int64_t n = c->n;
    if (n == 0) return PE_B200_OK;
    int rc = stage_reserve(c, stage_size(n));
    if (rc) return rc;
    const StageView s = stage_layout(c);
    const size_t v3b = 3 * (size_t)n * sizeof(double);
    PEB_CUDA(c, cudaMemcpyAsync(s.x, x, v3b, cudaMemcpyHostToDevice, c->stream));
    PEB_CUDA(c, cudaMemcpyAsync(s.v, v, v3b, cudaMemcpyHostToDevice, c->stream));
    PEB_CUDA(c, cudaMemcpyAsync(s.w, w, v3b, cudaMemcpyHostToDevice, c->stream));
    PEB_CUDA(c, cudaMemcpyAsync(s.r, r, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    PEB_CUDA(c, cudaMemcpyAsync(s.mat, mat, n * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    if (scene)
        PEB_CUDA(c, cudaMemcpyAsync(s.scene, scene, n * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    const unsigned g = capped_grid(c, n, 256);
    if (c->p.precision == PE_B200_FP64)
        k_pack<double><<<g, 256, 0, c->stream>>>(n, s.x, s.v, s.w, s.r, s.mat, scene ? s.scene : nullptr,
                                                 c->cur.pr, (double *)c->cur.vw, c->cur.tag, c->cur.uid, c->cur.q);
    else
        k_pack<float><<<g, 256, 0, c->stream>>>(n, s.x, s.v, s.w, s.r, s.mat, scene ? s.scene : nullptr,
                                                c->cur.pr, (float *)c->cur.vw, c->cur.tag, c->cur.uid, c->cur.q);
    PEB_LAUNCHED(c);
    return PE_B200_OK;
}

// the download's second stream and its two events, created on first use (false: not
// available, the copies stay on the context's stream)
static bool download_streams(Ctx *c) {
    if (c->dl) return true;
    if (c->dl_failed) return false;
    if (cudaStreamCreateWithFlags(&c->dl, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_dl0, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_dl1, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (c->dl) cudaStreamDestroy(c->dl);
        if (c->ev_dl0) cudaEventDestroy(c->ev_dl0);
        if (c->ev_dl1) cudaEventDestroy(c->ev_dl1);
        c->dl = nullptr;
        c->ev_dl0 = c->ev_dl1 = nullptr;
        c->dl_failed = true;
        return false;
    }
    return true;
}

int unpack_bodies(Ctx *c, double *x, double *v, double *w, double *q) {
    const int64_t n = c->n;
    if (n == 0) return PE_B200_OK;
    int rc = stage_reserve(c, stage_size(n));
    if (rc) return rc;
    const StageView s = stage_layout(c);
    const unsigned g = capped_grid(c, n, 256);
    const double4 *cq = q ? c->cur.q : nullptr;
    if (c->p.precision == PE_B200_FP64)
        k_unpack<double><<<g, 256, 0, c->stream>>>(n, c->cur.pr, (const double *)c->cur.vw, c->cur.uid, cq,
                                                   s.x, s.v, s.w, s.r);
    else
        k_unpack<float><<<g, 256, 0, c->stream>>>(n, c->cur.pr, (const float *)c->cur.vw, c->cur.uid, cq,
                                                  s.x, s.v, s.w, s.r);
    PEB_LAUNCHED(c);
    const size_t v3b = 3 * (size_t)n * sizeof(double);
    struct Part {
        void *host;
        const void *dev;
        size_t bytes;
    };
    Part parts[4];
    int np = 0;
    if (x) parts[np++] = {x, s.x, v3b};
    if (v) parts[np++] = {v, s.v, v3b};
    if (w) parts[np++] = {w, s.w, v3b};
    if (q) parts[np++] = {q, s.r, 4 * (size_t)n * sizeof(double)};
    size_t total = 0;
    for (int k = 0; k < np; ++k) total += parts[k].bytes;
    if (total >= ((size_t)8 << 20) && download_streams(c)) {
        // large downloads: every array's second half on a second stream, so that two copy
        // engines move the halves at once; the context's stream waits for both
        PEB_CUDA(c, cudaEventRecord(c->ev_dl0, c->stream));
        PEB_CUDA(c, cudaStreamWaitEvent(c->dl, c->ev_dl0, 0));
        for (int k = 0; k < np; ++k) {
            const size_t half = (parts[k].bytes / 2) & ~(size_t)255;
            PEB_CUDA(c, cudaMemcpyAsync(parts[k].host, parts[k].dev, half, cudaMemcpyDeviceToHost,
                                        c->stream));
            PEB_CUDA(c, cudaMemcpyAsync((char *)parts[k].host + half,
                                        (const char *)parts[k].dev + half, parts[k].bytes - half,
                                        cudaMemcpyDeviceToHost, c->dl));
        }
        PEB_CUDA(c, cudaEventRecord(c->ev_dl1, c->dl));
        PEB_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_dl1, 0));
    } else {
        for (int k = 0; k < np; ++k)
            PEB_CUDA(c, cudaMemcpyAsync(parts[k].host, parts[k].dev, parts[k].bytes,
                                        cudaMemcpyDeviceToHost, c->stream));
    }
    PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    return PE_B200_OK;
}

int scatter_state(Ctx *c, const double *x, const double *v, const double *w) {
    const int64_t n = c->n;
    if (n == 0) return PE_B200_OK;
    int rc = stage_reserve(c, stage_size(n));
    if (rc) return rc;
    const StageView s = stage_layout(c);
    const size_t v3b = 3 * (size_t)n * sizeof(double);
    if (x) PEB_CUDA(c, cudaMemcpyAsync(s.x, x, v3b, cudaMemcpyHostToDevice, c->stream));
    if (v) PEB_CUDA(c, cudaMemcpyAsync(s.v, v, v3b, cudaMemcpyHostToDevice, c->stream));
    if (w) PEB_CUDA(c, cudaMemcpyAsync(s.w, w, v3b, cudaMemcpyHostToDevice, c->stream));
    const unsigned g = capped_grid(c, n, 256);
    if (c->p.precision == PE_B200_FP64)
        k_scatter_state<double><<<g, 256, 0, c->stream>>>(n, c->cur.uid, x ? s.x : nullptr, v ? s.v : nullptr,
                                                          w ? s.w : nullptr, c->cur.pr, (double *)c->cur.vw);
    else
        k_scatter_state<float><<<g, 256, 0, c->stream>>>(n, c->cur.uid, x ? s.x : nullptr, v ? s.v : nullptr,
                                                         w ? s.w : nullptr, c->cur.pr, (float *)c->cur.vw);
    PEB_LAUNCHED(c);
    return PE_B200_OK;
}

int scatter_orientations(Ctx *c, const double *q) {
    const int64_t n = c->n;
    if (n == 0) return PE_B200_OK;
    int rc = stage_reserve(c, stage_size(n));
    if (rc) return rc;
    const StageView s = stage_layout(c);
    PEB_CUDA(c, cudaMemcpyAsync(s.r, q, 4 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice,
                                c->stream));
    k_scatter_q<<<capped_grid(c, n, 256), 256, 0, c->stream>>>(n, c->cur.uid, s.r, c->cur.q);
    PEB_LAUNCHED(c);
    return PE_B200_OK;
}

void stage_free(Ctx *c) {
    dfree(c, c->stage);
    c->stage = nullptr;
    c->stage_bytes = 0;
}

}  // namespace peb
