// contacts.cuh -- contact enumeration for one sphere: every contact (dist < contactThreshold)
// in which the sphere is body 1 (the smaller id of a sphere pair, or the sphere of a sphere-wall
// pair), with pe's contact geometry:
//   sphere-sphere  MaxContacts.h:547-569   plane  MaxContacts.h:777-790   box  MaxContacts.h:589-668
#pragma once

#include "internal.cuh"

namespace peb {

struct ContactGeom {
    int32_t other;   // slot / body index of body 2, or -1 for a wall
    int32_t wall;    // global wall index (planes first, then boxes) when other < 0
    double gx, gy, gz;
    double nx, ny, nz;
    double dist;
};

struct VisitArgs {
    const int32_t *sorted;   // slot -> body index (nullptr: identity)
    const int32_t *cell_start;
    const SceneInfo *scenes;
    const double4 *planes;
    const double *boxes;
    const double4 *pr;
    const uint32_t *tag;
    const int32_t *uid;
    int32_t total_planes;
};

// f(const ContactGeom&) is called for each contact of body b (at cell-sorted slot t).
template <typename F>
__device__ __forceinline__ void visit_contacts(const VisitArgs &a, int32_t b, F &f) {
    const double4 pi = a.pr[b];
    const uint32_t tagi = a.tag[b];
    const int32_t uidi = a.uid[b];
    const SceneInfo &s = a.scenes[tagi >> 16];
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
            // one candidate, in slot order
            auto pair = [&](int32_t j, int32_t uidj, const double4 &pj) {
                if (j == b) return;
                if (!(uidi < uidj)) return;  // the pair belongs to body 1
                const double nx = pi.x - pj.x, ny = pi.y - pj.y, nz = pi.z - pj.z;
                const double rs = pi.w + pj.w + 2.0 * kContactThreshold;
                if (nx * nx + ny * ny + nz * nz > rs * rs * (1.0 + 1e-12)) return;
                const double len = length_rn(nx, ny, nz);
                const double dist = __dsub_rn(__dsub_rn(len, pi.w), pj.w);
                if (!(dist < kContactThreshold)) return;
                ContactGeom g;
                g.other = j;
                g.wall = -1;
                double ux = nx, uy = ny, uz = nz;
                if (len != 0.0) {
                    const double il = 1.0 / len;
                    ux = nx * il; uy = ny * il; uz = nz * il;
                }
                const double k = pj.w + 0.5 * dist;
                g.gx = pj.x + ux * k;
                g.gy = pj.y + uy * k;
                g.gz = pj.z + uz * k;
                g.nx = ux; g.ny = uy; g.nz = uz;
                g.dist = dist;
                f(g);
            };
            int slot = a.cell_start[c0];
            // four candidates' ids and records in flight at a time (visited in slot order)
            for (; slot + 4 <= e; slot += 4) {
                int32_t jj[4], uu[4];
                double4 pp[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) jj[q] = a.sorted ? a.sorted[slot + q] : slot + q;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    uu[q] = a.uid[jj[q]];
                    pp[q] = a.pr[jj[q]];
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) pair(jj[q], uu[q], pp[q]);
            }
            for (; slot < e; ++slot) {
                const int32_t j = a.sorted ? a.sorted[slot] : slot;
                pair(j, a.uid[j], a.pr[j]);
            }
        }
    }
    for (int p = 0; p < s.nplanes; ++p) {
        const double4 pl = a.planes[s.plane_begin + p];
        const double kk = dot_rn(pl.x, pl.y, pl.z, pi.x, pi.y, pi.z);
        const double dist = __dsub_rn(__dsub_rn(kk, pi.w), pl.w);
        if (!(dist < kContactThreshold)) continue;
        ContactGeom g;
        g.other = -1;
        g.wall = s.plane_begin + p;
        const double f2 = pi.w + dist;
        g.gx = pi.x - f2 * pl.x;
        g.gy = pi.y - f2 * pl.y;
        g.gz = pi.z - f2 * pl.z;
        g.nx = pl.x; g.ny = pl.y; g.nz = pl.z;
        g.dist = dist;
        f(g);
    }
    for (int k = 0; k < s.nboxes; ++k) {
        const double *B = a.boxes + 15 * (int64_t)(s.box_begin + k);
        const double l[3] = {0.5 * B[3], 0.5 * B[4], 0.5 * B[5]};
        const double *R = B + 6;
        const double dx = pi.x - B[0], dy = pi.y - B[1], dz = pi.z - B[2];
        double p[3] = {dx * R[0] + dy * R[3] + dz * R[6], dx * R[1] + dy * R[4] + dz * R[7],
                       dx * R[2] + dy * R[5] + dz * R[8]};
        bool outside = false;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            if (p[ax] < -l[ax]) { p[ax] = -l[ax]; outside = true; }
            else if (p[ax] > l[ax]) { p[ax] = l[ax]; outside = true; }
        }
        ContactGeom g;
        g.other = -1;
        g.wall = a.total_planes + s.box_begin + k;
        if (!outside) {
            double dist = fabs(p[0]) - l[0];
            int face = 0;
            for (int ax = 1; ax < 3; ++ax) {
                const double tmp = fabs(p[ax]) - l[ax];
                if (dist < tmp) { dist = tmp; face = ax; }
            }
            const double sg = (p[face] > 0.0) ? 1.0 : -1.0;
            g.nx = R[face] * sg; g.ny = R[3 + face] * sg; g.nz = R[6 + face] * sg;
            g.dist = dist - pi.w;
            g.gx = pi.x; g.gy = pi.y; g.gz = pi.z;
            f(g);
            continue;
        }
        const double qx = R[0] * p[0] + R[1] * p[1] + R[2] * p[2];
        const double qy = R[3] * p[0] + R[4] * p[1] + R[5] * p[2];
        const double qz = R[6] * p[0] + R[7] * p[1] + R[8] * p[2];
        const double mx = dx - qx, my = dy - qy, mz = dz - qz;
        const double len = length_rn(mx, my, mz);
        const double dist = __dsub_rn(len, pi.w);
        if (!(dist < kContactThreshold)) continue;
        const double il = 1.0 / len;
        g.nx = mx * il; g.ny = my * il; g.nz = mz * il;
        g.gx = B[0] + qx; g.gy = B[1] + qy; g.gz = B[2] + qz;
        g.dist = dist;
        f(g);
    }
}

}  // namespace peb
