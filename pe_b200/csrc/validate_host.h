// validate_host.h -- the host-side checks behind pe_b200_validate, on plain host arrays (no
// CUDA), so that they can be exercised on planted inconsistencies without a GPU.
#ifndef PE_B200_VALIDATE_HOST_H
#define PE_B200_VALIDATE_HOST_H

#include <algorithm>
#include <cstdint>
#include <utility>
#include <vector>

namespace peb {

// Contacts in colour order: ids2[2k], ids2[2k+1] are the body slots of contact k (< 0: a wall),
// colour c holds contacts [color_start[c], color_start[c+1]).  Counts every body met twice in
// one colour, every slot out of [0, n) and every malformed colour range.
inline int64_t coloring_problems(int64_t n, int64_t nc, const int32_t *ids2, int ncol,
                                 const int32_t *color_start) {
    int64_t bad = 0;
    std::vector<int> seen(std::max<int64_t>(n, 1), -1);
    for (int col = 0; col < ncol; ++col) {
        const int64_t b = color_start[col], e = color_start[col + 1];
        if (b < 0 || e < b || e > nc) {
            ++bad;
            continue;
        }
        for (int64_t k = b; k < e; ++k)
            for (int s = 0; s < 2; ++s) {
                const int32_t body = ids2[2 * k + s];
                if (body < 0) continue;
                if (body >= n || seen[body] == col) ++bad;
                else seen[body] = col;
            }
    }
    return bad;
}

// Verlet lists in CSR form: sphere t's entries are idx[start[t] .. start[t+1]), each the
// neighbour's slot in bits 0-30 and in bit 31 whether uid[t] < uid[neighbour] (pe's contact
// orientation).  Counts malformed offsets, entries out of range or pointing at the sphere itself,
// wrong orientation bits, and one problem if some pair is not listed from both sides.
inline int64_t list_problems(int64_t n, int64_t cap, const int32_t *start, const int32_t *idx,
                             const int32_t *uid) {
    int64_t bad = 0;
    const int64_t m = start[n];
    if (m < 0 || m > cap || start[0] != 0) return 1;
    std::vector<std::pair<int32_t, int32_t>> pairs, rev;
    pairs.reserve(m);
    for (int64_t t = 0; t < n; ++t) {
        if (start[t] > start[t + 1] || start[t + 1] > m) {
            ++bad;
            continue;
        }
        for (int32_t k = start[t]; k < start[t + 1]; ++k) {
            const uint32_t e = (uint32_t)idx[k];
            const int64_t j = (int64_t)(e & 0x7fffffffu);
            if (j >= n || j == t) {
                ++bad;
                continue;
            }
            if (((e >> 31) != 0u) != (uid[t] < uid[j])) ++bad;
            pairs.push_back({(int32_t)t, (int32_t)j});
        }
    }
    rev.reserve(pairs.size());
    for (const auto &p : pairs) rev.push_back({p.second, p.first});
    std::sort(pairs.begin(), pairs.end());
    std::sort(rev.begin(), rev.end());
    if (pairs != rev) ++bad;
    return bad;
}

}  // namespace peb

#endif
