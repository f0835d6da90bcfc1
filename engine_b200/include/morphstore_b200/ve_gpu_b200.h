// ve_gpu_b200.h -- the B200 processing style for MorphStore's own operator
// templates.
//
// MorphStore selects an operator implementation by its first template
// argument, the processing style (`ve`): select_t<…, scalar<v64<uint64_t>>,
// …> is the scalar code, my_select_wit_t<…, avx512<v512<uint64_t>>, …> the
// AVX-512 code.  This header adds one more style, vectorlib::gpu_b200<
// v512<uint64_t>>, and specialises the reference's operator structs for it
// (the mechanism of include/core/operators/scalar/select_uncompr.h:39-40),
// so a query written against the reference's headers runs on the GPU when
// only its `using ve = …` changes:
//
//   morph_t                  include/core/morphing/morph.h:81-241
//   my_select_wit_t          include/core/operators/general_vectorized/select_compr.h:92-260
//   select_t (interface)     include/core/operators/interfaces/select.h:38-95
//   my_project_wit_t         general_vectorized/project_compr.h:69-262
//   project_t (interface)    interfaces/project.h:36-100
//   agg_sum_t                general_vectorized/agg_sum_compr.h:73-153
//   grouped agg_sum          interfaces/agg_sum.h:95-106 (explicit specialisations)
//   semi_equi_join_t         general_vectorized/join_semi_equi_compr.h:99-300
//   natural_equi_join_t      general_vectorized/join_natural_equi_compr.h:116-300
//   my_intersect_wit_t       general_vectorized/intersect_compr.h:189-347
//   intersect_sorted         interfaces/intersect.h:52-63 (explicit specialisations)
//   group_wit_t / group_vec  general_vectorized/group_compr.h:93-300
//   group (unary, binary)    interfaces/group.h:58-112 (explicit specialisations)
//
// The columns stay the reference's host-resident column<F>: every call
// copies its input columns' bytes to the device (building the block index of
// dynamic_vbp-family inputs there), runs the C ABI (include/ms_gpu.h) and
// returns a new column<F> with the output bytes, allocated as the reference's
// operators allocate their outputs; the caller owns it.  The bytes are the
// reference's AVX-512 layouts (gpu_b200's vector_helper_t is the AVX-512
// one, so DEFAULT_*_F(ve) names them); other layouts do not compile.
// A failing call throws std::runtime_error, as the reference's host code
// does.  There is no CPU fallback.
//
// Use: put this header first (or pass it with `-include`), with the
// reference's include/ directory and this repository's include/ on the
// include path, and link libms_gpu.so.
//
// Tracing: when the environment variable MSV_GPU_B200_DUMP_DIR names a
// directory, every operator call also writes its input and output columns
// there in the reference's binary_io layout ([count][used bytes][bytes],
// include/core/persistence/binary_io.h:40-87) and appends one line per
// column to trace.txt: call number, operator, role, format code, bit width,
// count, used bytes, compressed bytes, file name.
#ifndef MORPHSTORE_B200_VE_GPU_B200_H
#define MORPHSTORE_B200_VE_GPU_B200_H

#include <core/memory/mm_glob.h>
#include <core/morphing/default_formats.h>
#include <core/morphing/format.h>
#include <core/morphing/uncompr.h>
#include <core/morphing/static_vbp.h>
#include <core/morphing/dynamic_vbp.h>
#include <core/morphing/delta.h>
#include <core/morphing/for.h>
#include <core/morphing/rle.h>
#include <core/morphing/morph.h>
#include <core/operators/interfaces/agg_sum.h>
#include <core/operators/interfaces/group.h>
#include <core/operators/interfaces/intersect.h>
#include <core/operators/interfaces/join.h>
#include <core/operators/interfaces/project.h>
#include <core/operators/interfaces/select.h>
#include <core/operators/general_vectorized/agg_sum_compr.h>
#include <core/operators/general_vectorized/group_compr.h>
#include <core/operators/general_vectorized/intersect_compr.h>
#include <core/operators/general_vectorized/join_natural_equi_compr.h>
#include <core/operators/general_vectorized/join_semi_equi_compr.h>
#include <core/operators/general_vectorized/project_compr.h>
#include <core/operators/general_vectorized/select_compr.h>
#include <core/storage/column.h>
#include <vector/vector_extension_structs.h>
#include <vector/vector_primitives.h>

#include <ms_gpu.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>

namespace vectorlib {

// The processing style.  Its vector_helper_t is v512<uint64_t>, so
// DEFAULT_DYNAMIC_VBP_F(ve) and friends (default_formats.h:35-82) name the
// AVX-512 layouts, which are the device's layouts.
template <class VectorReg> struct gpu_b200;
template <typename T> struct gpu_b200<v512<T>> {
    static_assert(std::is_same<T, uint64_t>::value, "gpu_b200: columns hold uint64_t values");
    using vector_helper_t = v512<T>;
    using base_t = typename vector_helper_t::base_t;
    struct vector_t {
        T e[8];
    };
    using size = std::integral_constant<size_t, 64>;
    using mask_t = uint8_t;
};

}  // namespace vectorlib

namespace morphstore {
namespace b200 {

using gpu_ve = vectorlib::gpu_b200<vectorlib::v512<uint64_t>>;

// ---------------------------------------------------------------------------
// formats with a device layout
// ---------------------------------------------------------------------------
template <class F> struct fmt {
    static_assert(!std::is_same<F, F>::value,
                  "gpu_b200: this format has no device layout (the AVX-512 defaults and rle_f do)");
};
template <> struct fmt<uncompr_f> {
    static const int code = MS_FMT_UNCOMPR;
    static const unsigned bw = 0;
};
template <unsigned t_bw> struct fmt<static_vbp_f<vbp_l<t_bw, 8>>> {
    static const int code = MS_FMT_STATIC_VBP;
    static const unsigned bw = t_bw;
};
template <> struct fmt<dynamic_vbp_f<512, 64, 8>> {
    static const int code = MS_FMT_DYNAMIC_VBP;
    static const unsigned bw = 0;
};
template <> struct fmt<delta_f<1024, 8, dynamic_vbp_f<512, 64, 8>>> {
    static const int code = MS_FMT_DELTA_DVBP;
    static const unsigned bw = 0;
};
template <> struct fmt<for_f<1024, 8, dynamic_vbp_f<512, 64, 8>>> {
    static const int code = MS_FMT_FOR_DVBP;
    static const unsigned bw = 0;
};
template <> struct fmt<rle_f> {
    static const int code = MS_FMT_RLE;
    static const unsigned bw = 0;
};

// comparisons: the vectorlib ones my_select_wit_t takes (primitives/
// compare.h) and the std functors the interface select_t takes
template <template <class, int> class C> struct cmp_code;
template <> struct cmp_code<vectorlib::equal> { static const int value = MS_CMP_EQ; };
template <> struct cmp_code<vectorlib::less> { static const int value = MS_CMP_LT; };
template <> struct cmp_code<vectorlib::lessequal> { static const int value = MS_CMP_LE; };
template <> struct cmp_code<vectorlib::greater> { static const int value = MS_CMP_GT; };
template <> struct cmp_code<vectorlib::greaterequal> { static const int value = MS_CMP_GE; };

template <template <typename> class Op> struct std_cmp_code;
template <> struct std_cmp_code<std::equal_to> { static const int value = MS_CMP_EQ; };
template <> struct std_cmp_code<std::less> { static const int value = MS_CMP_LT; };
template <> struct std_cmp_code<std::less_equal> { static const int value = MS_CMP_LE; };
template <> struct std_cmp_code<std::greater> { static const int value = MS_CMP_GT; };
template <> struct std_cmp_code<std::greater_equal> { static const int value = MS_CMP_GE; };

// ---------------------------------------------------------------------------
// device context: one arena per process, emptied after every call
// ---------------------------------------------------------------------------
// An arena that ran out (MS_ERR_NOMEM): with_arena grows it and re-runs.
struct out_of_device_memory : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void check(int status, const char *where) {
    if (status == MS_OK) return;
    const std::string msg = std::string("gpu_b200 ") + where + ": " + ms_gpu_status_string(status);
    if (status == MS_ERR_NOMEM) throw out_of_device_memory(msg);
    throw std::runtime_error(msg);
}

struct context {
    ms_arena *arena = nullptr;
    uint64_t capacity = 0;
    unsigned call = 0;

    static context &get() {
        static context c;
        return c;
    }
    void ensure(uint64_t need) {
        if (arena && capacity >= need) return;
        if (arena) ms_gpu_arena_destroy(arena);
        arena = nullptr;
        const char *env = std::getenv("MSV_GPU_ARENA_BYTES");
        uint64_t cap = env ? std::strtoull(env, nullptr, 10) : (uint64_t(1) << 30);
        while (cap < need) cap *= 2;
        check(ms_gpu_arena_create(cap, &arena), "arena_create");
        capacity = cap;
    }
    ~context() {
        if (arena) ms_gpu_arena_destroy(arena);
    }
};

// Run `body` (which uploads, computes and downloads) with an arena of at
// least `hint` bytes; an arena that runs out is doubled and the call re-run.
// The arena is emptied afterwards: nothing of a call stays on the device.
template <class Body> auto with_arena(uint64_t hint, Body body) -> decltype(body(static_cast<ms_arena *>(nullptr))) {
    context &cx = context::get();
    cx.ensure(hint);
    for (int attempt = 0;; attempt++) {
        try {
            auto r = body(cx.arena);
            check(ms_gpu_arena_reset(cx.arena), "arena_reset");
            return r;
        } catch (const out_of_device_memory &) {
            ms_gpu_arena_reset(cx.arena);
            if (attempt >= 6) throw;
            cx.ensure(cx.capacity * 2);
        } catch (...) {
            ms_gpu_arena_reset(cx.arena);
            throw;
        }
    }
}

inline uint64_t col_bytes(uint64_t used) { return used + 256; }

// ---------------------------------------------------------------------------
// tracing (MSV_GPU_B200_DUMP_DIR)
// ---------------------------------------------------------------------------
template <class F> void dump(const char *op, const char *role, const column<F> *c) {
    const char *dir = std::getenv("MSV_GPU_B200_DUMP_DIR");
    if (!dir || !c) return;
    const unsigned call = context::get().call;
    char name[128];
    std::snprintf(name, sizeof name, "%04u_%s_%s.col", call, op, role);
    const std::string path = std::string(dir) + "/" + name;
    if (FILE *f = std::fopen(path.c_str(), "wb")) {
        const uint64_t hdr[2] = {c->get_count_values(), c->get_size_used_byte()};
        std::fwrite(hdr, 8, 2, f);
        std::fwrite(c->get_data(), 1, c->get_size_used_byte(), f);
        std::fclose(f);
    }
    if (FILE *t = std::fopen((std::string(dir) + "/trace.txt").c_str(), "a")) {
        std::fprintf(t, "%u %s %s %d %u %llu %llu %llu %s\n", call, op, role, fmt<F>::code, fmt<F>::bw,
                     (unsigned long long)c->get_count_values(), (unsigned long long)c->get_size_used_byte(),
                     (unsigned long long)c->get_size_compr_byte(), name);
        std::fclose(t);
    }
}
inline void next_call() { context::get().call++; }

// ---------------------------------------------------------------------------
// host column <-> device column
// ---------------------------------------------------------------------------
template <class F> ms_col upload(const column<F> *c, ms_arena *a) {
    if (!c) throw std::runtime_error("gpu_b200: null input column");
    ms_col d{};
    d.format = uint32_t(fmt<F>::code);
    d.bw = fmt<F>::bw;
    d.count_values = c->get_count_values();
    d.size_used_byte = c->get_size_used_byte();
    d.size_compr_byte = fmt<F>::code == MS_FMT_UNCOMPR ? 0 : c->get_size_compr_byte();
    d.size_alloc_byte = d.size_used_byte + 64;
    check(ms_gpu_arena_alloc(a, d.size_alloc_byte, &d.data), "upload (arena)");
    if (d.size_used_byte) check(ms_gpu_memcpy(d.data, c->get_data(), d.size_used_byte, 0, 0, nullptr), "upload");
    if ((d.format == MS_FMT_DYNAMIC_VBP || d.format == MS_FMT_DELTA_DVBP || d.format == MS_FMT_FOR_DVBP) &&
        d.size_compr_byte)
        check(ms_gpu_build_index(&d, a, nullptr), "build_index");
    return d;
}

template <class F> column<F> *download(const ms_col &d) {
    // allocated as the reference's operators allocate an output in F
    // (get_size_max_byte_any_len, format.h:114-153), so that later reference
    // calls (prepare_for_random_access writes the gap) find the room they need
    const uint64_t worst = ms_size_max_byte_any_len(fmt<F>::code, fmt<F>::bw, d.count_values);
    auto *c = new column<F>(std::max<uint64_t>(std::max<uint64_t>(worst, d.size_used_byte), 8));
    if (d.size_used_byte) check(ms_gpu_memcpy(c->get_data(), d.data, d.size_used_byte, 1, 1, nullptr), "download");
    c->set_meta_data(d.count_values, d.size_used_byte, d.size_compr_byte);
    return c;
}

inline uint64_t out_hint(uint64_t n) { return 40 * n + (uint64_t(64) << 20); }

// ---------------------------------------------------------------------------
// the operators, once per signature
// ---------------------------------------------------------------------------
template <class D, class S> const column<D> *morph(const column<S> *in) {
    next_call();
    dump("morph", "in", in);
    const column<D> *out = with_arena(2 * col_bytes(in->get_size_used_byte()) + out_hint(in->get_count_values()),
                                      [&](ms_arena *a) {
                                          ms_col src = upload(in, a), dst{};
                                          check(ms_gpu_morph(&src, fmt<D>::code, fmt<D>::bw, &dst, a, nullptr),
                                                "morph");
                                          return download<D>(dst);
                                      });
    dump("morph", "out", out);
    return out;
}

template <class O, class I> const column<O> *select(int cmp, const column<I> *in, uint64_t val) {
    next_call();
    dump("select", "in", in);
    const column<O> *out = with_arena(col_bytes(in->get_size_used_byte()) + out_hint(in->get_count_values()),
                                      [&](ms_arena *a) {
                                          ms_col x = upload(in, a), o{};
                                          check(ms_gpu_select(cmp, val, &x, fmt<O>::code, fmt<O>::bw, &o, a, nullptr),
                                                "select");
                                          return download<O>(o);
                                      });
    dump("select", "out", out);
    return out;
}

template <class O, class D, class P> const column<O> *project(const column<D> *data, const column<P> *pos) {
    next_call();
    dump("project", "data", data);
    dump("project", "pos", pos);
    const column<O> *out =
        with_arena(col_bytes(data->get_size_used_byte()) + col_bytes(pos->get_size_used_byte()) +
                       out_hint(pos->get_count_values()),
                   [&](ms_arena *a) {
                       ms_col dd = upload(data, a), pp = upload(pos, a), o{};
                       check(ms_gpu_project(&dd, &pp, fmt<O>::code, fmt<O>::bw, &o, a, nullptr), "project");
                       return download<O>(o);
                   });
    dump("project", "out", out);
    return out;
}

template <class F> const column<uncompr_f> *agg_sum(const column<F> *in) {
    next_call();
    dump("agg_sum", "in", in);
    const column<uncompr_f> *out = with_arena(col_bytes(in->get_size_used_byte()) + (uint64_t(64) << 20),
                                              [&](ms_arena *a) {
                                                  ms_col x = upload(in, a);
                                                  void *d_sum = nullptr;
                                                  check(ms_gpu_arena_alloc(a, 8, &d_sum), "agg_sum (arena)");
                                                  check(ms_gpu_agg_sum(&x, static_cast<uint64_t *>(d_sum), a, nullptr),
                                                        "agg_sum");
                                                  check(ms_gpu_arena_check(a, nullptr), "agg_sum");
                                                  auto *c = new column<uncompr_f>(sizeof(uint64_t));
                                                  check(ms_gpu_memcpy(c->get_data(), d_sum, 8, 1, 1, nullptr),
                                                        "agg_sum");
                                                  // as agg_sum_compr.h:148-150 writes it
                                                  c->set_meta_data(1, sizeof(uint64_t), sizeof(uint64_t));
                                                  return c;
                                              });
    dump("agg_sum", "out", out);
    return out;
}

template <class O, class G, class D>
const column<O> *agg_sum_grouped(const column<G> *gr, const column<D> *data, uint64_t n_groups) {
    next_call();
    dump("agg_sum_grouped", "gr", gr);
    dump("agg_sum_grouped", "data", data);
    const column<O> *out =
        with_arena(col_bytes(gr->get_size_used_byte()) + col_bytes(data->get_size_used_byte()) + out_hint(n_groups),
                   [&](ms_arena *a) {
                       ms_col g = upload(gr, a), d = upload(data, a), o{};
                       check(ms_gpu_agg_sum_grouped(&g, &d, n_groups, &o, a, nullptr), "agg_sum_grouped");
                       return download<O>(o);
                   });
    dump("agg_sum_grouped", "out", out);
    return out;
}

template <class O, class L, class R> const column<O> *semi_join(const column<L> *l, const column<R> *r) {
    next_call();
    dump("semi_join", "l", l);
    dump("semi_join", "r", r);
    const column<O> *out =
        with_arena(col_bytes(l->get_size_used_byte()) + col_bytes(r->get_size_used_byte()) +
                       out_hint(r->get_count_values() + l->get_count_values()),
                   [&](ms_arena *a) {
                       ms_col ll = upload(l, a), rr = upload(r, a), o{};
                       check(ms_gpu_semi_join(&ll, &rr, fmt<O>::code, fmt<O>::bw, &o, a, nullptr), "semi_join");
                       return download<O>(o);
                   });
    dump("semi_join", "out", out);
    return out;
}

template <class OL, class OR, class L, class R>
std::tuple<const column<OL> *, const column<OR> *> natural_join(const column<L> *l, const column<R> *r) {
    next_call();
    dump("join", "l", l);
    dump("join", "r", r);
    auto out = with_arena(col_bytes(l->get_size_used_byte()) + col_bytes(r->get_size_used_byte()) +
                              2 * out_hint(r->get_count_values() + l->get_count_values()),
                          [&](ms_arena *a) {
                              ms_col ll = upload(l, a), rr = upload(r, a), ol{}, orr{};
                              check(ms_gpu_natural_join(&ll, &rr, fmt<OL>::code, fmt<OL>::bw, fmt<OR>::code,
                                                        fmt<OR>::bw, &ol, &orr, a, nullptr),
                                    "join");
                              column<OL> *cl = download<OL>(ol);
                              column<OR> *cr = nullptr;
                              try {
                                  cr = download<OR>(orr);
                              } catch (...) {
                                  delete cl;
                                  throw;
                              }
                              return std::make_tuple(static_cast<const column<OL> *>(cl),
                                                     static_cast<const column<OR> *>(cr));
                          });
    dump("join", "out_l", std::get<0>(out));
    dump("join", "out_r", std::get<1>(out));
    return out;
}

template <class O, class L, class R> const column<O> *intersect(const column<L> *l, const column<R> *r) {
    next_call();
    dump("intersect", "l", l);
    dump("intersect", "r", r);
    const column<O> *out =
        with_arena(col_bytes(l->get_size_used_byte()) + col_bytes(r->get_size_used_byte()) +
                       out_hint(std::min(l->get_count_values(), r->get_count_values())),
                   [&](ms_arena *a) {
                       ms_col ll = upload(l, a), rr = upload(r, a), o{};
                       check(ms_gpu_intersect_sorted(&ll, &rr, fmt<O>::code, fmt<O>::bw, &o, a, nullptr),
                             "intersect");
                       return download<O>(o);
                   });
    dump("intersect", "out", out);
    return out;
}

// group ids / extents; gr_in != nullptr for the binary group
template <class G, class E, class GI, class D>
std::tuple<const column<G> *, const column<E> *> group(const column<GI> *gr_in, const column<D> *in) {
    static_assert(fmt<G>::code != MS_FMT_STATIC_VBP && fmt<E>::code != MS_FMT_STATIC_VBP,
                  "gpu_b200: group outputs in static_vbp are not supported");
    next_call();
    if (gr_in) dump("group", "gr_in", gr_in);
    dump("group", "in", in);
    auto out = with_arena((gr_in ? col_bytes(gr_in->get_size_used_byte()) : 0) + col_bytes(in->get_size_used_byte()) +
                              2 * out_hint(in->get_count_values()),
                          [&](ms_arena *a) {
                              ms_col x = upload(in, a), og{}, oe{}, gi{};
                              if (gr_in) gi = upload(gr_in, a);
                              check(ms_gpu_group(gr_in ? &gi : nullptr, &x, fmt<G>::code, &og, fmt<E>::code, &oe, a,
                                                 nullptr),
                                    "group");
                              column<G> *cg = download<G>(og);
                              column<E> *ce = nullptr;
                              try {
                                  ce = download<E>(oe);
                              } catch (...) {
                                  delete cg;
                                  throw;
                              }
                              return std::make_tuple(static_cast<const column<G> *>(cg),
                                                     static_cast<const column<E> *>(ce));
                          });
    dump("group", "out_gr", std::get<0>(out));
    dump("group", "out_ext", std::get<1>(out));
    return out;
}

}  // namespace b200

// ===========================================================================
// specialisations of the reference's operator structs for gpu_b200
// ===========================================================================
using b200_ve = b200::gpu_ve;

// ---- morph (morph.h:81-241, rle.h:155-297) -------------------------------
// The reference has partial specialisations generic in the style for
// <F, F>, <uncompr, uncompr>, <D, uncompr>, <uncompr, S>, <rle, uncompr> and
// <uncompr, rle>; each gets a gpu_b200 counterpart that is more specialised
// than both it and the general <gpu_b200, D, S>.
template <class t_dst_f, class t_src_f> struct morph_t<b200_ve, t_dst_f, t_src_f> {
    static const column<t_dst_f> *apply(const column<t_src_f> *inCol) { return b200::morph<t_dst_f>(inCol); }
};
template <class t_f> struct morph_t<b200_ve, t_f, t_f> {
    static const column<t_f> *apply(const column<t_f> *inCol) { return inCol; }
};
template <> struct morph_t<b200_ve, uncompr_f, uncompr_f> {
    static const column<uncompr_f> *apply(const column<uncompr_f> *inCol) { return inCol; }
};
template <class t_dst_f> struct morph_t<b200_ve, t_dst_f, uncompr_f> {
    static const column<t_dst_f> *apply(const column<uncompr_f> *inCol) { return b200::morph<t_dst_f>(inCol); }
};
template <class t_src_f> struct morph_t<b200_ve, uncompr_f, t_src_f> {
    static const column<uncompr_f> *apply(const column<t_src_f> *inCol) { return b200::morph<uncompr_f>(inCol); }
};
template <> struct morph_t<b200_ve, rle_f, uncompr_f> {
    static const column<rle_f> *apply(const column<uncompr_f> *inCol) { return b200::morph<rle_f>(inCol); }
};
template <> struct morph_t<b200_ve, uncompr_f, rle_f> {
    static const column<uncompr_f> *apply(const column<rle_f> *inCol) { return b200::morph<uncompr_f>(inCol); }
};

// ---- select (select_compr.h:92-260; interfaces/select.h:38-95) ------------
// my_select_wit_t keeps the AVX-512 style's compare (signed before the
// scalar remainder, unsigned in it); the interface select_t, which the
// reference implements for the scalar style only, compares unsigned.
template <template <class, int> class t_compare, class t_out_pos_f, class t_in_data_f>
struct my_select_wit_t<t_compare, b200_ve, t_out_pos_f, t_in_data_f> {
    static const column<t_out_pos_f> *apply(const column<t_in_data_f> *const inDataCol, const uint64_t val,
                                            const size_t outPosCountEstimate = 0) {
        (void)outPosCountEstimate;
        return b200::select<t_out_pos_f>(b200::cmp_code<t_compare>::value, inDataCol, val);
    }
};
template <template <typename> class t_op, class t_out_pos_f, class t_in_data_f>
struct select_t<t_op, b200_ve, t_out_pos_f, t_in_data_f> {
    static const column<t_out_pos_f> *apply(const column<t_in_data_f> *const inDataCol, const uint64_t val,
                                            const size_t outPosCountEstimate = 0) {
        (void)outPosCountEstimate;
        return b200::select<t_out_pos_f>(b200::std_cmp_code<t_op>::value | MS_CMP_UNSIGNED, inDataCol, val);
    }
};

// ---- project (project_compr.h:69-262; interfaces/project.h:36-100) --------
// Unlike the reference, the data column may also be dynamic_vbp, delta_f or
// for_f (random access through the device block index).
template <class t_out_data_f, class t_in_data_f, class t_in_pos_f>
class my_project_wit_t<b200_ve, t_out_data_f, t_in_data_f, t_in_pos_f> {
public:
    static const column<t_out_data_f> *apply(const column<t_in_data_f> *const inDataCol,
                                             const column<t_in_pos_f> *const inPosCol) {
        return b200::project<t_out_data_f>(inDataCol, inPosCol);
    }
};
template <class t_out_data_f, class t_in_data_f, class t_in_pos_f>
struct project_t<b200_ve, t_out_data_f, t_in_data_f, t_in_pos_f> {
    static const column<t_out_data_f> *apply(const column<t_in_data_f> *const inDataCol,
                                             const column<t_in_pos_f> *const inPosCol) {
        return b200::project<t_out_data_f>(inDataCol, inPosCol);
    }
};
// beside the reference's style-generic project_t<ve, uncompr, uncompr,
// static_vbp positions> (scalar/project_compr.h:148-180)
template <unsigned t_bw, unsigned t_step>
struct project_t<b200_ve, uncompr_f, uncompr_f, static_vbp_f<vbp_l<t_bw, t_step>>> {
    static const column<uncompr_f> *apply(const column<uncompr_f> *const inDataCol,
                                          const column<static_vbp_f<vbp_l<t_bw, t_step>>> *const inPosCol) {
        return b200::project<uncompr_f>(inDataCol, inPosCol);
    }
};

// ---- whole-column agg_sum (agg_sum_compr.h:73-153, agg_sum_uncompr.h:103) -
template <class InFormatCol> struct agg_sum_t<b200_ve, InFormatCol> {
    static const column<uncompr_f> *apply(const column<InFormatCol> *const p_InDataCol) {
        return b200::agg_sum(p_InDataCol);
    }
};
template <> struct agg_sum_t<b200_ve, uncompr_f> {
    static const column<uncompr_f> *apply(const column<uncompr_f> *const p_InDataCol) {
        return b200::agg_sum(p_InDataCol);
    }
};

// ---- semi-join and natural join (join_semi_equi_compr.h:99-300,
// join_natural_equi_compr.h:116-300) ----------------------------------------
template <class DataStructure, class OutFormatCol, class InFormatLCol, class InFormatRCol>
struct semi_equi_join_t<b200_ve, DataStructure, OutFormatCol, InFormatLCol, InFormatRCol> {
    static const column<OutFormatCol> *apply(const column<InFormatLCol> *const p_InDataLCol,
                                             const column<InFormatRCol> *const p_InDataRCol,
                                             const size_t outCountEstimate = 0) {
        (void)outCountEstimate;
        return b200::semi_join<OutFormatCol>(p_InDataLCol, p_InDataRCol);
    }
};
template <class DataStructure, class OutFormatLCol, class OutFormatRCol, class InFormatLCol, class InFormatRCol>
struct natural_equi_join_t<b200_ve, DataStructure, OutFormatLCol, OutFormatRCol, InFormatLCol, InFormatRCol> {
    static const std::tuple<const column<OutFormatLCol> *, const column<OutFormatRCol> *> apply(
        const column<InFormatLCol> *const p_InDataLCol, const column<InFormatRCol> *const p_InDataRCol,
        const size_t outCountEstimate = 0) {
        (void)outCountEstimate;
        return b200::natural_join<OutFormatLCol, OutFormatRCol>(p_InDataLCol, p_InDataRCol);
    }
};

// ---- intersect (intersect_compr.h:189-347) ---------------------------------
template <class t_out_data_f, class t_in_pos_l_f, class t_in_pos_r_f>
class my_intersect_wit_t<b200_ve, t_out_data_f, t_in_pos_l_f, t_in_pos_r_f> {
public:
    static const column<t_out_data_f> *apply(const column<t_in_pos_l_f> *const p_Data1Column,
                                             const column<t_in_pos_r_f> *const p_Data2Column,
                                             const size_t p_OutPosCountEstimate = 0) {
        (void)p_OutPosCountEstimate;
        return b200::intersect<t_out_data_f>(p_Data1Column, p_Data2Column);
    }
};

// ---- group (group_compr.h:93-300) ------------------------------------------
template <class OutFormatGroupIds, class OutFormatGroupExtents, class InFormatData, class DataStructure>
struct group_wit_t<b200_ve, OutFormatGroupIds, OutFormatGroupExtents, InFormatData, DataStructure> {
    static const std::tuple<const column<OutFormatGroupIds> *, const column<OutFormatGroupExtents> *> apply(
        const column<InFormatData> *const p_InDataCol, const size_t outCountGroupExtentsEstimate = 0) {
        (void)outCountGroupExtentsEstimate;
        return b200::group<OutFormatGroupIds, OutFormatGroupExtents, uncompr_f>(
            static_cast<const column<uncompr_f> *>(nullptr), p_InDataCol);
    }
};

// ---- the interface function templates the reference defines only by
// explicit specialisation (scalar/agg_sum_uncompr.h, scalar/group_uncompr.h,
// scalar/intersect_uncompr.h): the same, for gpu_b200, over every pair of
// uncompr_f and the dynamic_vbp-family layouts -----------------------------
#define MSV_B200_DV dynamic_vbp_f<512, 64, 8>

template <>
inline const column<uncompr_f> *agg_sum<b200_ve, uncompr_f, uncompr_f, uncompr_f>(
    const column<uncompr_f> *const inGrCol, const column<uncompr_f> *const inDataCol, const size_t inExtCount) {
    return b200::agg_sum_grouped<uncompr_f>(inGrCol, inDataCol, inExtCount);
}
template <>
inline const column<uncompr_f> *agg_sum<b200_ve, uncompr_f, MSV_B200_DV, MSV_B200_DV>(
    const column<MSV_B200_DV> *const inGrCol, const column<MSV_B200_DV> *const inDataCol, const size_t inExtCount) {
    return b200::agg_sum_grouped<uncompr_f>(inGrCol, inDataCol, inExtCount);
}

template <>
inline const std::tuple<const column<uncompr_f> *, const column<uncompr_f> *>
group<b200_ve, uncompr_f, uncompr_f, uncompr_f>(const column<uncompr_f> *const inDataCol,
                                                 const size_t outExtCountEstimate) {
    (void)outExtCountEstimate;
    return b200::group<uncompr_f, uncompr_f, uncompr_f>(static_cast<const column<uncompr_f> *>(nullptr), inDataCol);
}
template <>
inline const std::tuple<const column<uncompr_f> *, const column<uncompr_f> *>
group<b200_ve, uncompr_f, uncompr_f, uncompr_f, uncompr_f>(const column<uncompr_f> *const inGrCol,
                                                            const column<uncompr_f> *const inDataCol,
                                                            const size_t outExtCountEstimate) {
    (void)outExtCountEstimate;
    return b200::group<uncompr_f, uncompr_f, uncompr_f>(inGrCol, inDataCol);
}

template <>
inline const column<uncompr_f> *intersect_sorted<b200_ve, uncompr_f, uncompr_f, uncompr_f>(
    const column<uncompr_f> *const inPosLCol, const column<uncompr_f> *const inPosRCol,
    const size_t outPosCountEstimate) {
    (void)outPosCountEstimate;
    return b200::intersect<uncompr_f>(inPosLCol, inPosRCol);
}

#undef MSV_B200_DV

}  // namespace morphstore

#endif  // MORPHSTORE_B200_VE_GPU_B200_H
