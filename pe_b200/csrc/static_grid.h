// static_grid.h -- the cell grid of the allocation-free DEM step (noalloc.cu), in plain C++ so
// that its size arithmetic is tested on the host (tests/cpp/static_grid_test.cpp).
//
// The grid covers the caller's domain [lo, hi] with cubic cells of edge h, starting at the
// smallest edge that keeps the 27-cell search exact (2 (r_max + contact threshold)).  When the
// cell count dim0 * dim1 * dim2 exceeds the fixed budget the edge grows by 1.26 per round (about
// 2x fewer cells) until it fits; a coarser grid is still exact, only slower.  Every per-axis count
// and their product are formed in double, where they are exact below 2^53, and compared with the
// budget before anything is converted to an integer, so a very wide domain or a tiny radius can
// neither overflow the product nor reach an out-of-range cast.
#pragma once

#include <math.h>
#include <stdint.h>

namespace peb {

struct StaticGrid {
    double h;         // cell edge
    int64_t dim[3];   // cells per axis
    int64_t ncell;    // dim0 * dim1 * dim2 <= the budget
    int rounds;       // coarsening rounds taken (0: the finest edge fitted)
};

// Returns false when no grid exists: a non-finite or inverted domain, a non-finite or
// non-positive starting edge, or a budget below one cell.
inline bool static_grid_plan(const double lo[3], const double hi[3], double h0,
                             int64_t max_cells, StaticGrid *g) {
    if (!(h0 > 0.0) || !isfinite(h0) || max_cells < 1) return false;
    double len[3];
    for (int a = 0; a < 3; ++a) {
        len[a] = hi[a] - lo[a];
        if (!isfinite(lo[a]) || !isfinite(hi[a]) || !isfinite(len[a]) || !(len[a] >= 0.0))
            return false;
    }
    const double budget = (double)max_cells;
    double h = h0;
    // each round divides the cell count by about 2; from the smallest edge (2e-8) over the widest
    // finite domain (1.8e308) about 3,100 rounds reach one cell, and an edge that overflows to
    // infinity gives one cell per axis
    for (int round = 0; round < 8192; ++round) {
        double d[3], prod = 1.0;
        bool fits = true;
        for (int a = 0; a < 3; ++a) {
            d[a] = floor(len[a] / h) + 1.0;
            if (!(d[a] <= budget)) fits = false;
        }
        if (fits) {
            // formed in double, so it cannot overflow; with factors of at most 2^17 (the
            // library's budget of 131,072 cells) it is exact
            prod = d[0] * d[1] * d[2];
            fits = prod <= budget;
        }
        if (fits) {
            g->h = h;
            g->ncell = 1;
            for (int a = 0; a < 3; ++a) {
                g->dim[a] = (int64_t)d[a];
                g->ncell *= g->dim[a];
            }
            g->rounds = round;
            return true;
        }
        h *= 1.26;
    }
    return false;
}

}  // namespace peb
