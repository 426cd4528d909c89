// validate_test.cpp -- plants inconsistencies in host arrays and checks that the checks behind
// pe_b200_validate (pe_b200/csrc/validate_host.h) count them.  Prints "ok" on success.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "validate_host.h"

#define EXPECT(cond)                                                     \
    do {                                                                 \
        if (!(cond)) {                                                   \
            std::printf("failed at line %d: %s\n", __LINE__, #cond);     \
            return 1;                                                    \
        }                                                                \
    } while (0)

int main() {
    using peb::coloring_problems;
    using peb::list_problems;
    // four bodies, contacts (0,1) (2,3) | (1,2) (3,wall) | (0,3)
    std::vector<int32_t> ids = {0, 1, 2, 3, 1, 2, 3, -1, 0, 3};
    std::vector<int32_t> cs = {0, 2, 4, 5};
    EXPECT(coloring_problems(4, 5, ids.data(), 3, cs.data()) == 0);
    // body 2 twice in colour 1
    std::vector<int32_t> bad = ids;
    bad[6] = 2;
    EXPECT(coloring_problems(4, 5, bad.data(), 3, cs.data()) == 1);
    // slot out of range
    bad = ids;
    bad[9] = 4;
    EXPECT(coloring_problems(4, 5, bad.data(), 3, cs.data()) == 1);
    // colour range beyond the contacts
    std::vector<int32_t> cs_bad = {0, 2, 4, 6};
    EXPECT(coloring_problems(4, 5, ids.data(), 3, cs_bad.data()) == 1);
    // merging colours 0 and 1 puts bodies 1, 2, 3 twice in one colour
    std::vector<int32_t> cs_merged = {0, 4, 5};
    EXPECT(coloring_problems(4, 5, ids.data(), 2, cs_merged.data()) == 3);

    // lists of three spheres, uids 5 7 6: pairs (0,1) and (1,2)
    const uint32_t hi = 0x80000000u;
    std::vector<int32_t> uid = {5, 7, 6};
    std::vector<int32_t> start = {0, 1, 3, 4};
    std::vector<int32_t> idx = {(int32_t)(1u | hi), 0, 2, (int32_t)(1u | hi)};
    EXPECT(list_problems(3, 8, start.data(), idx.data(), uid.data()) == 0);
    // wrong orientation bit
    std::vector<int32_t> b2 = idx;
    b2[1] = (int32_t)(0u | hi);
    EXPECT(list_problems(3, 8, start.data(), b2.data(), uid.data()) == 1);
    // one-sided pair: sphere 2 lists 0 instead of 1
    b2 = idx;
    b2[3] = (int32_t)(0u | hi);
    EXPECT(list_problems(3, 8, start.data(), b2.data(), uid.data()) >= 1);
    // self entry
    b2 = idx;
    b2[0] = 0;
    EXPECT(list_problems(3, 8, start.data(), b2.data(), uid.data()) >= 1);
    // entry out of range
    b2 = idx;
    b2[2] = 3;
    EXPECT(list_problems(3, 8, start.data(), b2.data(), uid.data()) >= 1);
    // more entries than the capacity
    EXPECT(list_problems(3, 3, start.data(), idx.data(), uid.data()) == 1);
    // decreasing offsets
    std::vector<int32_t> s2 = {0, 3, 1, 4};
    EXPECT(list_problems(3, 8, s2.data(), idx.data(), uid.data()) >= 1);
    std::printf("ok\n");
    return 0;
}
