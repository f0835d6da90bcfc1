// select_sum_query.cpp -- the query of the reference's example
// (src/examples/select_sum_query.cpp:51-108) written for the device-resident
// C++ layer (morphstore_b200/morphstore.h), which keeps columns on the GPU
// between operators.  It differs from the reference's file: the base data
// come from a seeded splitmix64 generator instead of generate_with_distr,
// both columns are morphed to dynamic_vbp on the device first, and the
// program checks its sum instead of printing it.  The reference's own file,
// with only its processing style changed to gpu_b200, is built from the
// reference's sources through morphstore_b200/ve_gpu_b200.h by
// engine_b200/build.py.
//   SELECT SUM(baseCol2) WHERE baseCol1 = 150
// Base data: baseCol1 uniform in [100, 199], baseCol2 uniform in [0, 10]
// (seeded, counter-based splitmix64), compressed as dynamic_vbp on the device.
#include <morphstore_b200/morphstore.h>

#include <cinttypes>
#include <cstdio>
#include <vector>

using namespace morphstore;
using namespace vectorlib;

static uint64_t mix64(uint64_t seed, uint64_t i) {
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

int main(int argc, char **argv) {
    const size_t countValues = argc > 1 ? std::strtoull(argv[1], nullptr, 10) : 100 * 1000 * 1000;
    std::vector<uint64_t> v1(countValues), v2(countValues);
    for (size_t i = 0; i < countValues; i++) {
        v1[i] = 100 + mix64(1, i) % 100;
        v2[i] = mix64(2, i) % 11;
    }
    using ve = gpu_b200<v512<uint64_t>>;
    const column<uncompr_f> *baseCol1 = make_column(v1);
    const column<uncompr_f> *baseCol2 = make_column(v2);
    auto c1 = morph<ve, DEFAULT_DYNAMIC_VBP_F(ve)>(baseCol1);
    auto c2 = morph<ve, DEFAULT_DYNAMIC_VBP_F(ve)>(baseCol2);

    // Positions fulfilling "baseCol1 = 150"
    auto i1 = my_select_wit_t<equal, ve, uncompr_f, DEFAULT_DYNAMIC_VBP_F(ve)>::apply(c1, 150);
    // Data elements of "baseCol2" fulfilling "baseCol1 = 150"
    auto i2 = my_project_wit_t<ve, uncompr_f, DEFAULT_DYNAMIC_VBP_F(ve), uncompr_f>::apply(c2, i1);
    // Sum over the data elements of "baseCol2" fulfilling "baseCol1 = 150"
    auto i3 = agg_sum<ve, uncompr_f>(i2);

    uint64_t expect = 0;
    for (size_t i = 0; i < countValues; i++)
        if (v1[i] == 150) expect += v2[i];
    const uint64_t got = i3->to_host()[0];
    std::printf("SUM(baseCol2) = %" PRIu64 " (host check %" PRIu64 ", %s)\n", got, expect,
                got == expect ? "ok" : "MISMATCH");
    return got == expect ? 0 : 1;
}
