// ref_shim.cpp -- C-ABI over the MorphStore reference's own codecs and
// operators, compiled from the reference's headers where they lie (never
// copied).  TEST INFRASTRUCTURE ONLY: used to pin the C oracle (golden
// fixtures, direct differential tests) and as bench.py's CPU baseline.
//
// Built by oracle/Makefile into oracle/_ref/libmsref_<isa>.so.  VE selects
// the reference processing style (AVX-512 or AVX2 TVL back-end).
#include <core/memory/mm_glob.h>
#include <core/morphing/format.h>
#include <core/morphing/uncompr.h>
#include <core/morphing/static_vbp.h>
#include <core/morphing/dynamic_vbp.h>
#include <core/morphing/delta.h>
#include <core/morphing/for.h>
#include <core/morphing/rle.h>
#include <core/morphing/vbp.h>
#include <core/morphing/default_formats.h>
#include <core/operators/general_vectorized/select_compr.h>
#include <core/operators/general_vectorized/project_compr.h>
#include <core/operators/general_vectorized/agg_sum_compr.h>
#include <core/operators/general_vectorized/group_compr.h>
#include <core/operators/general_vectorized/join_semi_equi_compr.h>
#include <core/operators/general_vectorized/join_natural_equi_compr.h>
#include <core/operators/general_vectorized/intersect_compr.h>
#include <core/operators/interfaces/join.h>
#if defined(PART_OPS)
// defines non-inline specialisations: one translation unit only
#include <core/operators/scalar/agg_sum_uncompr.h>
#endif
#include <core/storage/column.h>
#include <vector/vector_primitives.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <tuple>
#include <type_traits>

using namespace morphstore;
using namespace vectorlib;

#ifndef VE
#define VE avx512<v512<uint64_t>>
#endif
using ve = VE;

using uf = uncompr_f;
using dv = DEFAULT_DYNAMIC_VBP_F(ve);
using dd = DEFAULT_DELTA_DYNAMIC_VBP_F(ve);
using fd = DEFAULT_FOR_DYNAMIC_VBP_F(ve);
template <unsigned bw> using sv = DEFAULT_STATIC_VBP_F(ve, bw);

enum { F_UNCOMPR = 0, F_STATIC = 1, F_DVBP = 2, F_DELTA = 3, F_FOR = 4, F_RLE = 5 };
enum { C_EQ = 0, C_LT = 1, C_LE = 2, C_GT = 3, C_GE = 4 };

extern "C" struct ref_meta {
    uint64_t count_values, size_used_byte, size_compr_byte;
};

template <class T> struct tag { using type = T; };

// Codec dispatch: every static_vbp bit width 1..64.
// Format codes of the C ABI, and dispatch over explicit lists of formats
// (bounds the number of template instances and thus the compile time).
template <class F> struct fcode;
template <> struct fcode<uf> { static const int code = F_UNCOMPR; static const unsigned bw = 0; };
template <unsigned B> struct fcode<sv<B>> { static const int code = F_STATIC; static const unsigned bw = B; };
template <> struct fcode<dv> { static const int code = F_DVBP; static const unsigned bw = 0; };
template <> struct fcode<dd> { static const int code = F_DELTA; static const unsigned bw = 0; };
template <> struct fcode<fd> { static const int code = F_FOR; static const unsigned bw = 0; };
template <> struct fcode<rle_f> { static const int code = F_RLE; static const unsigned bw = 0; };

template <class... Fs> struct flist {};
template <class Fn> int dispatch(int, unsigned, flist<>, Fn &) { return -12; }
template <class F, class... Rest, class Fn> int dispatch(int code, unsigned bw, flist<F, Rest...>, Fn &fn) {
    if (fcode<F>::code == code && (code != F_STATIC || fcode<F>::bw == bw)) return fn(tag<F>{});
    return dispatch(code, bw, flist<Rest...>{}, fn);
}
template <class L, class Fn> int with_formats(int code, unsigned bw, Fn fn) { return dispatch(code, bw, L{}, fn); }

using SelIn = flist<uf, sv<10>, dv, dd, fd>;
using SelOut = flist<uf, sv<32>, dv, dd, fd>;
using SelInCmp = flist<uf, dv>;
using SelOutCmp = flist<uf>;
using ProjData = flist<uf, sv<10>, sv<20>>;
using ProjPos = flist<uf, dv, dd>;
using ProjOut = flist<uf, dv>;
using SumIn = flist<uf, sv<10>, sv<20>, dv, dd, fd>;
using SjL = flist<uf, dd>;
using SjR = flist<uf, dv, fd>;
using SjOut = flist<uf, dv, dd>;
using IsL = flist<uf, dv, dd>;
using IsOut = flist<uf, dv>;
using GrIn = flist<uf, dv>;
using GrOut = flist<uf, dv>;
using JnL = flist<uf, dd>;
using JnR = flist<uf, dv, fd>;
using JnOut = flist<uf, dv>;

template <class F> static const column<F> *make_col(const uint8_t *bytes, const ref_meta *m, uint64_t alloc) {
    auto *c = new column<F>(alloc + 64);
    std::memcpy(c->get_data(), bytes, m->size_used_byte);
    c->set_meta_data(m->count_values, m->size_used_byte, m->size_compr_byte);
    return c;
}

static const column<uf> *make_ucol(const uint64_t *v, uint64_t n) {
    auto *c = new column<uf>(8 * n + 64);
    std::memcpy(c->get_data(), v, 8 * n);
    c->set_meta_data(n, 8 * n);
    return c;
}

template <class F> static int export_col(const column<F> *c, uint8_t *out, uint64_t cap, ref_meta *m) {
    m->count_values = c->get_count_values();
    m->size_used_byte = c->get_size_used_byte();
    m->size_compr_byte = c->get_size_compr_byte();
    if (m->size_used_byte > cap) return -2;
    std::memcpy(out, c->get_data(), m->size_used_byte);
    return 0;
}

template <class F> static uint64_t alloc_for(const ref_meta *m) {
    return m->size_used_byte + 64;
}

#if defined(PART_SELECT)
template <template <class, int> class CMP, class LIn, class LOut>
static int select_impl(uint64_t val, int in_fmt, unsigned in_bw, const uint8_t *in, const ref_meta *im, int out_fmt,
                       unsigned out_bw, uint8_t *out, uint64_t cap, ref_meta *om) {
    return with_formats<LIn>(in_fmt, in_bw, [&](auto ti) {
        using FI = typename decltype(ti)::type;
        const column<FI> *c = make_col<FI>(in, im, alloc_for<FI>(im));
        int r = with_formats<LOut>(out_fmt, out_bw, [&](auto to) {
            using FO = typename decltype(to)::type;
            const column<FO> *p = my_select_wit_t<CMP, ve, FO, FI>::apply(c, val);
            int rr = export_col(p, out, cap, om);
            delete p;
            return rr;
        });
        delete c;
        return r;
    });
}

#endif

extern "C" {


#if defined(PART_SV_LO)
// static_vbp codecs for bit widths PART_SV_LO..PART_SV_HI (one object file
// per range so the 64 instances compile in parallel).
#define MS_CAT2(a, b) a##b
#define MS_CAT(a, b) MS_CAT2(a, b)
extern "C++" {
template <class Fn, unsigned B> struct sv_part {
    static int go(unsigned bw, Fn &fn) {
        if (bw == B) return fn(tag<sv<B>>{});
        return sv_part<Fn, B + 1>::go(bw, fn);
    }
};
template <class Fn> struct sv_part<Fn, PART_SV_HI + 1> {
    static int go(unsigned, Fn &) { return -10; }
};
}

int MS_CAT(ref_sv_compress_, PART_SV_LO)(unsigned bw, const uint64_t *in, uint64_t n, uint8_t *out, uint64_t cap,
                                          ref_meta *m) {
    const column<uf> *u = make_ucol(in, n);
    auto fn = [&](auto t) {
        using F = typename decltype(t)::type;
        const column<F> *c = morph<ve, F>(u);
        int r = export_col(c, out, cap, m);
        delete c;
        return r;
    };
    int rc = sv_part<decltype(fn), PART_SV_LO>::go(bw, fn);
    delete u;
    return rc;
}

int MS_CAT(ref_sv_decompress_, PART_SV_LO)(unsigned bw, const uint8_t *in, const ref_meta *m, uint64_t *out) {
    auto fn = [&](auto t) {
        using F = typename decltype(t)::type;
        const column<F> *c = make_col<F>(in, m, alloc_for<F>(m));
        const column<uf> *u = morph<ve, uf>(c);
        std::memcpy(out, u->get_data(), 8 * u->get_count_values());
        delete u;
        delete c;
        return 0;
    };
    return sv_part<decltype(fn), PART_SV_LO>::go(bw, fn);
}
#endif

#if defined(PART_CODECS)
int ref_sv_compress_1(unsigned, const uint64_t *, uint64_t, uint8_t *, uint64_t, ref_meta *);
int ref_sv_compress_17(unsigned, const uint64_t *, uint64_t, uint8_t *, uint64_t, ref_meta *);
int ref_sv_compress_33(unsigned, const uint64_t *, uint64_t, uint8_t *, uint64_t, ref_meta *);
int ref_sv_compress_49(unsigned, const uint64_t *, uint64_t, uint8_t *, uint64_t, ref_meta *);
int ref_sv_decompress_1(unsigned, const uint8_t *, const ref_meta *, uint64_t *);
int ref_sv_decompress_17(unsigned, const uint8_t *, const ref_meta *, uint64_t *);
int ref_sv_decompress_33(unsigned, const uint8_t *, const ref_meta *, uint64_t *);
int ref_sv_decompress_49(unsigned, const uint8_t *, const ref_meta *, uint64_t *);

using CodecOther = flist<uf, dv, dd, fd, rle_f>;

// morph<ve, F>(uncompr column) -> compressed bytes + metadata.
int ref_compress(int fmt, unsigned bw, const uint64_t *in, uint64_t n, uint8_t *out, uint64_t cap, ref_meta *m) {
    if (fmt == F_STATIC) {
        if (bw < 1 || bw > 64) return -10;
        if (bw <= 16) return ref_sv_compress_1(bw, in, n, out, cap, m);
        if (bw <= 32) return ref_sv_compress_17(bw, in, n, out, cap, m);
        if (bw <= 48) return ref_sv_compress_33(bw, in, n, out, cap, m);
        return ref_sv_compress_49(bw, in, n, out, cap, m);
    }
    const column<uf> *u = make_ucol(in, n);
    int rc = with_formats<CodecOther>(fmt, bw, [&](auto t) {
        using F = typename decltype(t)::type;
        const column<F> *c = morph<ve, F>(u);
        int r = export_col(c, out, cap, m);
        if ((const void *)c != (const void *)u) delete c;
        return r;
    });
    delete u;
    return rc;
}

// morph<ve, uncompr_f>(compressed column) -> values.
int ref_decompress(int fmt, unsigned bw, const uint8_t *in, const ref_meta *m, uint64_t *out) {
    if (fmt == F_STATIC) {
        if (bw < 1 || bw > 64) return -10;
        if (bw <= 16) return ref_sv_decompress_1(bw, in, m, out);
        if (bw <= 32) return ref_sv_decompress_17(bw, in, m, out);
        if (bw <= 48) return ref_sv_decompress_33(bw, in, m, out);
        return ref_sv_decompress_49(bw, in, m, out);
    }
    return with_formats<CodecOther>(fmt, bw, [&](auto t) {
        using F = typename decltype(t)::type;
        const column<F> *c = make_col<F>(in, m, alloc_for<F>(m));
        const column<uf> *u = morph<ve, uf>(c);
        std::memcpy(out, u->get_data(), 8 * u->get_count_values());
        if ((const void *)u != (const void *)c) delete u;
        delete c;
        return 0;
    });
}
#endif

#if defined(PART_SELECT)
// my_select_wit_t<cmp, ve, out_f, in_f>::apply(in, val)
int ref_select(int cmp, uint64_t val, int in_fmt, unsigned in_bw, const uint8_t *in, const ref_meta *im, int out_fmt,
               unsigned out_bw, uint8_t *out, uint64_t cap, ref_meta *om) {
    switch (cmp) {
    case C_EQ: return select_impl<vectorlib::equal, SelInCmp, SelOutCmp>(val, in_fmt, in_bw, in, im, out_fmt, out_bw, out, cap, om);
    case C_LT: return select_impl<vectorlib::less, SelIn, SelOut>(val, in_fmt, in_bw, in, im, out_fmt, out_bw, out, cap, om);
    case C_LE: return select_impl<vectorlib::lessequal, SelInCmp, SelOutCmp>(val, in_fmt, in_bw, in, im, out_fmt, out_bw, out, cap, om);
    case C_GT: return select_impl<vectorlib::greater, SelInCmp, SelOutCmp>(val, in_fmt, in_bw, in, im, out_fmt, out_bw, out, cap, om);
    case C_GE: return select_impl<vectorlib::greaterequal, SelInCmp, SelOutCmp>(val, in_fmt, in_bw, in, im, out_fmt, out_bw, out, cap, om);
    }
    return -13;
}

#endif

#if defined(PART_OPS)
int ref_isa(void) {
#ifdef AVX512
    return 512;
#else
    return 256;
#endif
}

// my_project_wit_t<ve, out_f, data_f, pos_f>::apply(data, pos); data is
// uncompr_f or static_vbp_f (the only formats with random_read_access).
int ref_project(int data_fmt, unsigned data_bw, const uint8_t *data, const ref_meta *dm, int pos_fmt, unsigned pos_bw,
                const uint8_t *pos, const ref_meta *pm, int out_fmt, unsigned out_bw, uint8_t *out, uint64_t cap,
                ref_meta *om) {
    if (data_fmt != F_UNCOMPR && data_fmt != F_STATIC) return -14;
    return with_formats<ProjData>(data_fmt, data_bw, [&](auto td) {
        using FD = typename decltype(td)::type;
        const column<FD> *d = make_col<FD>(data, dm, alloc_for<FD>(dm) + 2 * 64 * 64 * 8);
        int r = with_formats<ProjPos>(pos_fmt, pos_bw, [&](auto tp) {
            using FP = typename decltype(tp)::type;
            const column<FP> *p = make_col<FP>(pos, pm, alloc_for<FP>(pm));
            int r2 = with_formats<ProjOut>(out_fmt, out_bw, [&](auto to) {
                using FO = typename decltype(to)::type;
                const column<FO> *o = my_project_wit_t<ve, FO, FD, FP>::apply(d, p);
                int r3 = export_col(o, out, cap, om);
                delete o;
                return r3;
            });
            delete p;
            return r2;
        });
        delete d;
        return r;
    });
}

// agg_sum<ve, F>(col)
int ref_agg_sum(int fmt, unsigned bw, const uint8_t *in, const ref_meta *m, uint64_t *sum) {
    return with_formats<SumIn>(fmt, bw, [&](auto t) {
        using F = typename decltype(t)::type;
        const column<F> *c = make_col<F>(in, m, alloc_for<F>(m));
        const column<uf> *s = agg_sum<ve, F>(c);
        *sum = *(const uint64_t *)s->get_data();
        delete s;
        delete c;
        return 0;
    });
}

// semi_join<ve, out_f, L_f, R_f>(L, R): positions of R whose value is in L.
int ref_semi_join(int l_fmt, const uint8_t *l, const ref_meta *lm, int r_fmt, const uint8_t *r, const ref_meta *rm,
                  int out_fmt, uint8_t *out, uint64_t cap, ref_meta *om) {
    return with_formats<SjL>(l_fmt, 0, [&](auto tl) {
        using FL = typename decltype(tl)::type;
        const column<FL> *lc = make_col<FL>(l, lm, alloc_for<FL>(lm));
        int res = with_formats<SjR>(r_fmt, 0, [&](auto tr) {
            using FR = typename decltype(tr)::type;
            const column<FR> *rc = make_col<FR>(r, rm, alloc_for<FR>(rm));
            int r2 = with_formats<SjOut>(out_fmt, 0, [&](auto to) {
                using FO = typename decltype(to)::type;
                const column<FO> *o = semi_join<ve, FO, FL, FR>(lc, rc);
                int r3 = export_col(o, out, cap, om);
                delete o;
                return r3;
            });
            delete rc;
            return r2;
        });
        delete lc;
        return res;
    });
}

// my_intersect_wit_t<ve, out_f, L_f, R_f>::apply(L, R); R uncompr_f.
int ref_intersect(int l_fmt, const uint8_t *l, const ref_meta *lm, const uint64_t *r, uint64_t nr, int out_fmt,
                  uint8_t *out, uint64_t cap, ref_meta *om) {
    const column<uf> *rc = make_ucol(r, nr);
    int res = with_formats<IsL>(l_fmt, 0, [&](auto tl) {
        using FL = typename decltype(tl)::type;
        const column<FL> *lc = make_col<FL>(l, lm, alloc_for<FL>(lm));
        int r2 = with_formats<IsOut>(out_fmt, 0, [&](auto to) {
            using FO = typename decltype(to)::type;
            const column<FO> *o = my_intersect_wit_t<ve, FO, FL, uf>::apply(lc, rc);
            int r3 = export_col(o, out, cap, om);
            delete o;
            return r3;
        });
        delete lc;
        return r2;
    });
    delete rc;
    return res;
}

// group_vec<ve, gr_f, ext_f, in_f>(col): group ids + extents.
int ref_group(int in_fmt, const uint8_t *in, const ref_meta *im, int gr_fmt, uint8_t *gr, uint64_t gr_cap,
              ref_meta *grm, int ext_fmt, uint8_t *ext, uint64_t ext_cap, ref_meta *extm) {
    return with_formats<GrIn>(in_fmt, 0, [&](auto ti) {
        using FI = typename decltype(ti)::type;
        const column<FI> *c = make_col<FI>(in, im, alloc_for<FI>(im));
        int r = with_formats<GrOut>(gr_fmt, 0, [&](auto tg) {
            using FG = typename decltype(tg)::type;
            return with_formats<GrOut>(ext_fmt, 0, [&](auto te) {
                using FE = typename decltype(te)::type;
                auto res = group_vec<ve, FG, FE, FI>(c);
                int a = export_col(std::get<0>(res), gr, gr_cap, grm);
                int b = export_col(std::get<1>(res), ext, ext_cap, extm);
                delete std::get<0>(res);
                delete std::get<1>(res);
                return a ? a : b;
            });
        });
        delete c;
        return r;
    });
}

// grouped agg_sum<scalar>(gr, data, n_groups) (scalar/agg_sum_uncompr.h:64-95).
int ref_agg_sum_grouped(const uint64_t *gr, const uint64_t *data, uint64_t n, uint64_t n_groups, uint64_t *out) {
    const column<uf> *g = make_ucol(gr, n);
    const column<uf> *d = make_ucol(data, n);
    const column<uf> *s = agg_sum<scalar<v64<uint64_t>>, uf, uf, uf>(g, d, n_groups);
    std::memcpy(out, s->get_data(), 8 * n_groups);
    delete s;
    delete g;
    delete d;
    return 0;
}

// CPU baseline: the select -> project -> sum query on the reference's own
// operators (select_sum_query.cpp:77-97).  x is compressed as dynamic_vbp,
// y as dynamic_vbp; the reference cannot project from dynamic_vbp, so y is
// decompressed first (part of the timed region).  Returns the sum; *secs =
// the operator time (compression outside the timed region).
uint64_t ref_bench_select_project_sum(const uint64_t *x, const uint64_t *y, uint64_t n, uint64_t c, double *secs,
                                      uint64_t *count, uint64_t *compr_bytes) {
    const column<uf> *xu = make_ucol(x, n);
    const column<uf> *yu = make_ucol(y, n);
    const column<dv> *xc = morph<ve, dv>(xu);
    const column<dv> *yc = morph<ve, dv>(yu);
    delete xu;
    delete yu;
    *compr_bytes = xc->get_size_used_byte() + yc->get_size_used_byte();
    auto t0 = std::chrono::steady_clock::now();
    const column<uf> *pos = my_select_wit_t<vectorlib::less, ve, uf, dv>::apply(xc, c);
    const column<uf> *yd = morph<ve, uf>(yc);
    const column<uf> *pr = my_project_wit_t<ve, uf, uf, uf>::apply(yd, pos);
    const column<uf> *s = agg_sum<ve, uf>(pr);
    auto t1 = std::chrono::steady_clock::now();
    *secs = std::chrono::duration<double>(t1 - t0).count();
    uint64_t sum = *(const uint64_t *)s->get_data();
    *count = pos->get_count_values();
    delete pos;
    delete yd;
    delete pr;
    delete s;
    delete xc;
    delete yc;
    return sum;
}


// The same query split into preparation and timed runs, so that a process
// which runs it step after step compresses its rows once: ref_sps_prepare
// compresses x and y (dynamic_vbp, as the GPU path stores them) and keeps
// them; ref_sps_run times select(x < c) -> morph(y) -> project -> agg_sum on
// them (the operators of select_sum_query.cpp:77-97) and returns the sum.
struct ref_sps {
    const column<dv> *x, *y;
};

void *ref_sps_prepare(const uint64_t *x, const uint64_t *y, uint64_t n, uint64_t *compr_bytes) {
    const column<uf> *xu = make_ucol(x, n);
    const column<uf> *yu = make_ucol(y, n);
    auto *h = new ref_sps{morph<ve, dv>(xu), morph<ve, dv>(yu)};
    delete xu;
    delete yu;
    *compr_bytes = h->x->get_size_used_byte() + h->y->get_size_used_byte();
    return h;
}

uint64_t ref_sps_run(void *handle, uint64_t c, double *secs, uint64_t *count) {
    const ref_sps *h = static_cast<const ref_sps *>(handle);
    auto t0 = std::chrono::steady_clock::now();
    const column<uf> *pos = my_select_wit_t<vectorlib::less, ve, uf, dv>::apply(h->x, c);
    const column<uf> *yd = morph<ve, uf>(h->y);
    const column<uf> *pr = my_project_wit_t<ve, uf, uf, uf>::apply(yd, pos);
    const column<uf> *s = agg_sum<ve, uf>(pr);
    auto t1 = std::chrono::steady_clock::now();
    *secs = std::chrono::duration<double>(t1 - t0).count();
    const uint64_t sum = *(const uint64_t *)s->get_data();
    *count = pos->get_count_values();
    delete pos;
    delete yd;
    delete pr;
    delete s;
    return sum;
}

void ref_sps_free(void *handle) {
    ref_sps *h = static_cast<ref_sps *>(handle);
    delete h->x;
    delete h->y;
    delete h;
}
#endif

#if defined(PART_JOIN)
// join<ve, outL_f, outR_f, L_f, R_f>(L, R) (join.h:158-187): the natural
// equi-join, (build position, probe position) pairs in probe order; both
// outputs in the same format.
int ref_natural_join(int l_fmt, const uint8_t *l, const ref_meta *lm, int r_fmt, const uint8_t *r, const ref_meta *rm,
                     int out_fmt, uint8_t *out_l, uint64_t cap_l, ref_meta *om_l, uint8_t *out_r, uint64_t cap_r,
                     ref_meta *om_r) {
    return with_formats<JnL>(l_fmt, 0, [&](auto tl) {
        using FL = typename decltype(tl)::type;
        const column<FL> *lc = make_col<FL>(l, lm, alloc_for<FL>(lm));
        int res = with_formats<JnR>(r_fmt, 0, [&](auto tr) {
            using FR = typename decltype(tr)::type;
            const column<FR> *rc = make_col<FR>(r, rm, alloc_for<FR>(rm));
            int r2 = with_formats<JnOut>(out_fmt, 0, [&](auto to) {
                using FO = typename decltype(to)::type;
                auto res2 = join<ve, FO, FO, FL, FR>(lc, rc);
                int r3 = export_col(std::get<0>(res2), out_l, cap_l, om_l);
                if (!r3) r3 = export_col(std::get<1>(res2), out_r, cap_r, om_r);
                delete std::get<0>(res2);
                delete std::get<1>(res2);
                return r3;
            });
            delete rc;
            return r2;
        });
        delete lc;
        return res;
    });
}
#endif

}  // extern "C"
