// kat_test.cpp -- the reference's operator known-answer tests
// (test/core/operators/{select,project,agg_sum_whole_column,
// agg_sum_group_based,group_unary,group_binary,intersect}_test.cpp) run
// through the drop-in C++ API on the GPU, plus compressed-format variants.
#include <morphstore_b200/morphstore.h>

#include <cstdio>
#include <vector>

using namespace morphstore;
using namespace vectorlib;
using ve = gpu_b200<v512<uint64_t>>;
using dv = DEFAULT_DYNAMIC_VBP_F(ve);

static int failures = 0;

template <class F>
static void expect(const char *name, const column<F> *c, const std::vector<uint64_t> &want) {
    const std::vector<uint64_t> got = c->to_host();
    const bool ok = got == want;
    std::printf("%-40s %s\n", name, ok ? "ok" : "not ok");
    failures += !ok;
}

int main() {
    expect("select(<100)", my_select_wit_t<less, ve, uncompr_f, uncompr_f>::apply(make_column({95, 102, 100, 87, 120}), 100),
           {0, 3});
    expect("project",
           my_project_wit_t<ve, uncompr_f, uncompr_f, uncompr_f>::apply(make_column({11, 44, 22, 33, 11}),
                                                                         make_column({1, 3, 4})),
           {44, 33, 11});
    expect("agg_sum (whole column)", agg_sum<ve, uncompr_f>(make_column({100, 150, 50, 500, 200, 100})), {1100});
    expect("agg_sum (group based)",
           agg_sum<ve, uncompr_f, uncompr_f, uncompr_f>(make_column({0, 0, 1, 0, 2, 1}),
                                                         make_column({100, 150, 50, 500, 200, 100}), 3),
           {750, 150, 200});
    auto g = group_vec<ve, uncompr_f, uncompr_f, uncompr_f>(make_column({333, 333, 111, 333, 222, 111}));
    expect("group (unary) ids", std::get<0>(g), {0, 0, 1, 0, 2, 1});
    expect("group (unary) extents", std::get<1>(g), {0, 2, 4});
    auto g2 = group<ve, uncompr_f, uncompr_f, uncompr_f, uncompr_f>(make_column({0, 0, 1, 0, 2, 1}),
                                                                      make_column({77, 88, 77, 77, 88, 88}));
    expect("group (binary) ids", std::get<0>(g2), {0, 1, 2, 0, 3, 4});
    expect("group (binary) extents", std::get<1>(g2), {0, 1, 2, 4, 5});
    expect("intersect_sorted",
           intersect_sorted<ve, uncompr_f, uncompr_f, uncompr_f>(make_column({1, 4, 5, 8, 9, 12}),
                                                                 make_column({1, 6, 8, 12, 15})),
           {1, 8, 12});
    // compressed variants: a 5000-value column in dynamic_vbp
    std::vector<uint64_t> big(5000), pos;
    uint64_t sum = 0;
    for (size_t i = 0; i < big.size(); i++) {
        big[i] = (i * 2654435761u) % 1000;
        if (big[i] < 100) pos.push_back(i), sum += big[i];
    }
    auto bc = morph<ve, dv>(make_column(big));
    expect("select on dynamic_vbp, dynamic_vbp out", my_select_wit_t<less, ve, dv, dv>::apply(bc, 100), pos);
    uint64_t total = 0;
    for (uint64_t x : big) total += x;
    expect("agg_sum on dynamic_vbp", agg_sum<ve, dv>(bc), {total});
    (void)sum;
    return failures ? 1 : 0;
}
