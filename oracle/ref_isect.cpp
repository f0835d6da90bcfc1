// ref_isect.cpp -- the reference's scalar intersect_sorted
// (include/core/operators/scalar/intersect_uncompr.h:41-86) behind a C ABI.
// TEST INFRASTRUCTURE ONLY (golden fixtures).  Kept in its own translation
// unit: the header defines a non-inline specialisation.
#include <core/memory/mm_glob.h>
#include <core/morphing/format.h>
#include <core/operators/scalar/intersect_uncompr.h>
#include <core/storage/column.h>

#include <cstdint>
#include <cstring>

using namespace morphstore;
using namespace vectorlib;

static const column<uncompr_f> *mk(const uint64_t *v, uint64_t n) {
    auto *c = new column<uncompr_f>(8 * n + 64);
    std::memcpy(c->get_data(), v, 8 * n);
    c->set_meta_data(n, 8 * n);
    return c;
}

extern "C" uint64_t ref_intersect_scalar(const uint64_t *l, uint64_t nl, const uint64_t *r, uint64_t nr,
                                         uint64_t *out) {
    const column<uncompr_f> *lc = mk(l, nl), *rc = mk(r, nr);
    const column<uncompr_f> *o = intersect_sorted<scalar<v64<uint64_t>>, uncompr_f, uncompr_f, uncompr_f>(lc, rc, 0);
    const uint64_t k = o->get_count_values();
    std::memcpy(out, o->get_data(), 8 * k);
    delete o;
    delete lc;
    delete rc;
    return k;
}
