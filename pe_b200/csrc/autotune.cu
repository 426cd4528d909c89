// autotune.cu -- launch-shape autotuner of the DEM list step (no pe counterpart: pe runs one
// fixed serial loop).
//
// The tunables change only how the work is laid out on the GPU, never which pairs a body sums
// or in which order, except for the skin, which changes when the state is re-sorted and so the
// last bits of the forces:
//   dem_variant     threads per block / resident blocks per SM of k_dem_move (dem.cu)
//   rebuild_per_sm  CTAs per SM of the persistent rebuild kernel (rebuild.cu); -1 rebuilds with
//                   one launch per stage instead (the same lists, entry for entry)
//   skin            neighbour-list skin (cells are re-planned to 2 r_max + skin)
//   dem_split       form of the list step: the contact forces before the integration, on a
//                   second stream beside it, or overlapped with it on one stream (dem.cu)
// Each trial restores the state saved at entry, forces a list rebuild, runs a few untimed steps
// (graph capture included), then times `trial` steps with CUDA events after forcing one more
// rebuild, so a trial's time charges at least one rebuild per `trial` steps.  Coordinate
// descent: skin first, then the force kernel's shape, then the rebuild grid.
#include <algorithm>
#include <cmath>

#include "internal.cuh"

namespace peb {

namespace {

void free_snap(Ctx *c, BodyBuf &b) {
    dfree(c, b.pr);
    dfree(c, b.vw);
    dfree(c, b.tag);
    dfree(c, b.uid);
    dfree(c, b.q);
    b = BodyBuf();
}

int copy_bodies(Ctx *c, BodyBuf &dst, const BodyBuf &src) {
    const size_t n = (size_t)c->n;
    PEB_CUDA(c, cudaMemcpyAsync(dst.pr, src.pr, n * sizeof(double4), cudaMemcpyDeviceToDevice, c->stream));
    PEB_CUDA(c, cudaMemcpyAsync(dst.vw, src.vw, n * (size_t)c->vw_bytes, cudaMemcpyDeviceToDevice, c->stream));
    PEB_CUDA(c, cudaMemcpyAsync(dst.tag, src.tag, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, c->stream));
    PEB_CUDA(c, cudaMemcpyAsync(dst.uid, src.uid, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, c->stream));
    if (src.q && dst.q)
        PEB_CUDA(c, cudaMemcpyAsync(dst.q, src.q, n * sizeof(double4), cudaMemcpyDeviceToDevice, c->stream));
    return PE_B200_OK;
}

}  // namespace

// New skin: re-plans the cells so the 27-cell search still covers r_i + r_j + skin, and asks
// for a list rebuild.
int set_list_skin(Ctx *c, double skin) {
    if (!(skin > 0.0) || !std::isfinite(skin)) return set_err(c, PE_B200_ERR_ARG, "invalid skin");
    if (skin == c->nl.skin) return PE_B200_OK;
    PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    c->nl.skin = skin;
    plan_cells(c, skin);
    dfree(c, c->cell_count);
    dfree(c, c->cell_start);
    c->cell_count = c->cell_start = nullptr;
    PEB_CUDA(c, dmalloc(c, &c->cell_count, ((size_t)c->ncell + 1) * sizeof(int32_t)));
    PEB_CUDA(c, dmalloc(c, &c->cell_start, ((size_t)c->ncell + 2) * sizeof(int32_t)));
    PEB_CUDA(c, cudaMemsetAsync(c->cell_count, 0, ((size_t)c->ncell + 1) * sizeof(int32_t), c->stream));
    int rc = scan_reserve(c, c->ncell + 1);
    if (rc) return rc;
    rc = upload_tables(c);
    if (rc) return rc;
    c->binned = false;
    c->epoch++;
    return dem_list_request_rebuild(c);
}

int set_tuning(Ctx *c, const Tuning &t, double skin) {
    if (t.dem_variant < 0 || t.dem_variant >= dem_variant_count() || t.rebuild_per_sm < -1 ||
        t.nbgs_sweeps < 0 || t.nbgs_sweeps > 5 || t.dem_grid < 0 || t.dem_grid > 1 ||
        t.dem_split < 0 || t.dem_split > 2)
        return set_err(c, PE_B200_ERR_ARG, "invalid tuning");
    // captured list-step graphs bake the form in; the new form's first step runs outside a
    // capture (the split form creates its second stream there)
    if (t.dem_split != c->tune.dem_split) {
        c->epoch++;
        c->nl.warm = false;
    }
    c->tune.dem_split = t.dem_split;
    // captured hard-contact graphs bake the sweep form in
    if (t.nbgs_sweeps != c->tune.nbgs_sweeps) c->epoch++;
    c->tune.nbgs_sweeps = t.nbgs_sweeps;
    c->tune.dem_grid = t.dem_grid;
    if (t.dem_variant != c->tune.dem_variant || t.rebuild_per_sm != c->tune.rebuild_per_sm) {
        c->tune = t;
        c->epoch++;
        // the rebuild grid may grow: its per-block buffer is allocated outside any capture
        c->nl.warm = false;
    }
    if (c->nl.enabled) return set_list_skin(c, skin);
    return PE_B200_OK;
}

int autotune(Ctx *c, double dt, int32_t trial, pe_b200_tuning *out) {
    if (c->p.solver != PE_B200_DEM || !c->nl.enabled || c->n == 0)
        return set_err(c, PE_B200_ERR_UNSUPPORTED, "the autotuner tunes the DEM neighbour-list step");
    if (!(dt > 0.0) || trial < 2) return PE_B200_ERR_ARG;
    BodyBuf snap;
    const size_t n = (size_t)c->n;
    cudaError_t e = dmalloc(c, &snap.pr, n * sizeof(double4));
    if (e == cudaSuccess) e = dmalloc(c, &snap.vw, n * (size_t)c->vw_bytes);
    if (e == cudaSuccess) e = dmalloc(c, &snap.tag, n * sizeof(uint32_t));
    if (e == cudaSuccess) e = dmalloc(c, &snap.uid, n * sizeof(int32_t));
    if (e == cudaSuccess && c->cur.q) e = dmalloc(c, &snap.q, n * sizeof(double4));
    if (e != cudaSuccess) {
        free_snap(c, snap);
        return cuda_err(c, e, "autotune snapshot");
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = copy_bodies(c, snap, c->cur);
    const Tuning t0 = c->tune;
    const double skin0 = c->nl.skin;
    const bool prof0 = c->prof;
    c->prof = false;
    const int32_t warm = std::max<int32_t>(2, trial / 4);

    auto measure = [&](const Tuning &t, double skin, double *ms) -> int {
        int r = copy_bodies(c, c->cur, snap);
        if (!r) r = set_tuning(c, t, skin);
        if (!r) r = dem_list_request_rebuild(c);
        if (!r) r = run_steps(c, warm, dt);
        if (!r) r = dem_list_request_rebuild(c);
        if (r) return r;
        PEB_CUDA(c, cudaEventRecord(e0, c->stream));
        r = run_steps(c, trial, dt);
        if (r) return r;
        PEB_CUDA(c, cudaEventRecord(e1, c->stream));
        PEB_CUDA(c, cudaEventSynchronize(e1));
        float f = 0.f;
        PEB_CUDA(c, cudaEventElapsedTime(&f, e0, e1));
        *ms = (double)f / trial;
        return PE_B200_OK;
    };

    Tuning best = t0;
    double best_skin = skin0, best_ms = INFINITY;
    auto consider = [&](const Tuning &t, double skin) -> int {
        double ms = INFINITY;
        int r = measure(t, skin, &ms);
        if (r) return r;
        if (ms < best_ms) {
            best_ms = ms;
            best = t;
            best_skin = skin;
        }
        return PE_B200_OK;
    };
    if (!rc) rc = consider(t0, skin0);
    for (double f : {0.5, 1.5, 2.0, 3.0})
        if (!rc) rc = consider(best, skin0 * f);
    for (int v = 0; v < dem_variant_count() && !rc; ++v) {
        if (v == best.dem_variant) continue;
        Tuning t = best;
        t.dem_variant = v;
        rc = consider(t, best_skin);
    }
    for (int r : {1, 2, 4, 0}) {
        if (rc || r == best.rebuild_per_sm) continue;
        Tuning t = best;
        t.rebuild_per_sm = r;
        rc = consider(t, best_skin);
    }
    const int32_t split0 = best.dem_split;
    for (int32_t f = 0; f <= 2; ++f) {
        if (rc || f == split0) continue;
        Tuning t = best;
        t.dem_split = f;
        rc = consider(t, best_skin);
    }
    // leave the state as it was at entry, with the winning shapes
    if (!rc) rc = copy_bodies(c, c->cur, snap);
    if (!rc) rc = set_tuning(c, best, best_skin);
    if (!rc) rc = dem_list_request_rebuild(c);
    cudaStreamSynchronize(c->stream);
    c->prof = prof0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    free_snap(c, snap);
    if (rc) return rc;
    if (out) {
        out->dem_variant = best.dem_variant;
        out->rebuild_per_sm = best.rebuild_per_sm;
        out->skin = best_skin;
        out->ms_per_step = best_ms;
        out->variants = dem_variant_count();
        out->nbgs_sweeps = best.nbgs_sweeps;
        out->dem_grid = c->tune.dem_grid;
        out->dem_split = best.dem_split;
    }
    return PE_B200_OK;
}

}  // namespace peb
