// static_grid_test.cpp -- host checks of the allocation-free step's grid planner
// (pe_b200/csrc/static_grid.h): wide domains and tiny radii coarsen the grid instead of
// overflowing the cell count, and impossible domains are refused.  Prints "ok" on success.
#include <math.h>
#include <stdio.h>

#include "static_grid.h"

static int failures = 0;
#define CHECK(c)                                                 \
    do {                                                         \
        if (!(c)) {                                              \
            printf("FAIL line %d: %s\n", __LINE__, #c);          \
            ++failures;                                          \
        }                                                        \
    } while (0)

static const int64_t kBudget = 131072;   // PE_B200_STATIC_MAX_CELLS

static double h0(double rmax) { return 2.0 * (rmax + 1e-8) * (1.0 + 1e-9); }

int main() {
    peb::StaticGrid g;
    // a small domain fits at the finest edge
    {
        const double lo[3] = {0, 0, 0}, hi[3] = {10, 10, 10};
        CHECK(peb::static_grid_plan(lo, hi, h0(0.5), kBudget, &g));
        CHECK(g.rounds == 0 && g.h == h0(0.5));
        CHECK(g.dim[0] == 10 && g.ncell == 1000);
    }
    // +-1e6 with r = 1e-3: about 5e8 cells per axis at the finest edge, whose product (1.25e26)
    // overflows int64; the planner coarsens until the product fits
    {
        const double lo[3] = {-1e6, -1e6, -1e6}, hi[3] = {1e6, 1e6, 1e6};
        CHECK(peb::static_grid_plan(lo, hi, h0(1e-3), kBudget, &g));
        CHECK(g.rounds > 0 && g.h > h0(1e-3));
        CHECK(g.ncell <= kBudget && g.ncell == g.dim[0] * g.dim[1] * g.dim[2]);
        for (int a = 0; a < 3; ++a) CHECK(g.dim[a] >= 1 && g.dim[a] <= kBudget);
        // every body of the domain lies in a cell: dim * h covers the extent
        for (int a = 0; a < 3; ++a) CHECK((double)g.dim[a] * g.h > hi[a] - lo[a]);
        // the previous, finer edge did not fit
        const double hf = g.h / 1.26;
        double prod = 1.0;
        for (int a = 0; a < 3; ++a) prod *= floor((hi[a] - lo[a]) / hf) + 1.0;
        CHECK(prod > (double)kBudget);
    }
    // one very long axis with thin others: each axis count alone exceeds the budget at first
    {
        const double lo[3] = {0, 0, 0}, hi[3] = {1e12, 1, 1};
        CHECK(peb::static_grid_plan(lo, hi, h0(0.5), kBudget, &g));
        CHECK(g.ncell <= kBudget && g.dim[0] <= kBudget);
    }
    // the widest finite domain still plans (the edge grows until a few cells remain)
    {
        const double lo[3] = {-8e307, -8e307, -8e307}, hi[3] = {8e307, 8e307, 8e307};
        CHECK(peb::static_grid_plan(lo, hi, h0(1e-300), kBudget, &g));
        CHECK(g.ncell >= 1 && g.ncell <= kBudget);
    }
    // refused: an extent that overflows to infinity, non-finite bounds, an inverted domain,
    // a non-finite or non-positive edge
    {
        const double lo[3] = {-1.7e308, 0, 0}, hi[3] = {1.7e308, 1, 1};
        CHECK(!peb::static_grid_plan(lo, hi, h0(0.5), kBudget, &g));
        const double lo2[3] = {0, 0, NAN}, hi2[3] = {1, 1, 1};
        CHECK(!peb::static_grid_plan(lo2, hi2, h0(0.5), kBudget, &g));
        const double lo3[3] = {0, 0, 2}, hi3[3] = {1, 1, 1};
        CHECK(!peb::static_grid_plan(lo3, hi3, h0(0.5), kBudget, &g));
        const double lo4[3] = {0, 0, 0}, hi4[3] = {1, 1, 1};
        CHECK(!peb::static_grid_plan(lo4, hi4, INFINITY, kBudget, &g));
        CHECK(!peb::static_grid_plan(lo4, hi4, 0.0, kBudget, &g));
        CHECK(!peb::static_grid_plan(lo4, hi4, 1.0, 0, &g));
    }
    if (failures == 0) printf("ok\n");
    return failures == 0 ? 0 : 1;
}
