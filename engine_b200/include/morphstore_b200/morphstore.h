// morphstore.h -- the reference's column / format / operator API, backed by
// the B200 C ABI (include/ms_gpu.h).
//
// A query written against MorphStore's operator templates compiles against
// this header with the processing style `vectorlib::gpu_b200<v512<uint64_t>>`
// and runs on the GPU: morph<ve,F>(col), my_select_wit_t<cmp,ve,out,in>,
// my_project_wit_t<ve,out,data,pos>, agg_sum<ve,F>(col), grouped agg_sum,
// semi_join<ve,out,L,R>, intersect_sorted / my_intersect_wit_t, group_vec
// and the binary group.  Columns are device-resident; their metadata mirrors
// column<F> (include/core/storage/column.h:45-287).  Like the reference,
// operators return newly created columns owned by the caller, and errors are
// reported as std::runtime_error.
//
// Only the reference's AVX-512 default layouts exist on the device
// (default_formats.h:35-82); other template parameters fail to compile.
#pragma once

#include <ms_gpu.h>

#include <cstdint>
#include <cstdlib>
#include <initializer_list>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

namespace vectorlib {

template <class T> struct v512 {};

// The processing style that selects the GPU path.
template <class VV> struct gpu_b200 {
    using base_t = uint64_t;
    struct vector_helper_t {
        struct element_count { static const unsigned value = 8; };
        struct size_bit { static const unsigned value = 512; };
        struct size_byte { static const unsigned value = 64; };
    };
};

// Comparisons (include/vector/primitives/compare.h:22-76).
template <class VE, int G = 64> struct equal { static const int code = MS_CMP_EQ; };
template <class VE, int G = 64> struct less { static const int code = MS_CMP_LT; };
template <class VE, int G = 64> struct lessequal { static const int code = MS_CMP_LE; };
template <class VE, int G = 64> struct greater { static const int code = MS_CMP_GT; };
template <class VE, int G = 64> struct greaterequal { static const int code = MS_CMP_GE; };

}  // namespace vectorlib

namespace morphstore {

// --------------------------------------------------------------------------
// formats (format.h:90-96, vbp_format_rndaccess.h:61-87, static_vbp.h:61-68,
// dynamic_vbp.h:84-159, delta.h:79-157, for.h:85-164, rle.h:42-49)
// --------------------------------------------------------------------------
struct format {};

struct uncompr_f : format {
    static const int ms_code = MS_FMT_UNCOMPR;
    static const unsigned ms_bw = 0;
    static const size_t m_BlockSize = 1;
};

template <unsigned t_Bw, unsigned t_Step> struct vbp_l {
    static_assert(1 <= t_Bw && t_Bw <= 64, "vbp_l: bit width must be in 1..64");
    static_assert(t_Step == 8, "vbp_l: the device layout uses 8 interleaved lanes");
};

template <class t_layout> struct static_vbp_f;
template <unsigned t_Bw> struct static_vbp_f<vbp_l<t_Bw, 8>> : format {
    static const int ms_code = MS_FMT_STATIC_VBP;
    static const unsigned ms_bw = t_Bw;
    static const size_t m_BlockSize = 512;
};

template <size_t t_BlockSizeLog, size_t t_PageSizeBlocks, unsigned t_Step> struct dynamic_vbp_f : format {
    static_assert(t_BlockSizeLog == 512 && t_PageSizeBlocks == 64 && t_Step == 8,
                  "dynamic_vbp_f: the device layout is dynamic_vbp_f<512, 64, 8>");
    static const int ms_code = MS_FMT_DYNAMIC_VBP;
    static const unsigned ms_bw = 0;
    static const size_t m_BlockSize = 512;
};

template <size_t t_BlockSizeLog, unsigned t_Step, class t_inner_f> struct delta_f : format {
    static_assert(t_BlockSizeLog == 1024 && t_Step == 8 && std::is_same<t_inner_f, dynamic_vbp_f<512, 64, 8>>::value,
                  "delta_f: the device layout is delta_f<1024, 8, dynamic_vbp_f<512, 64, 8>>");
    static const int ms_code = MS_FMT_DELTA_DVBP;
    static const unsigned ms_bw = 0;
    static const size_t m_BlockSize = 1024;
};

template <size_t t_BlockSizeLog, size_t t_PageSizeBlocks, class t_inner_f> struct for_f : format {
    static_assert(t_BlockSizeLog == 1024 && t_PageSizeBlocks == 8 &&
                      std::is_same<t_inner_f, dynamic_vbp_f<512, 64, 8>>::value,
                  "for_f: the device layout is for_f<1024, 8, dynamic_vbp_f<512, 64, 8>>");
    static const int ms_code = MS_FMT_FOR_DVBP;
    static const unsigned ms_bw = 0;
    static const size_t m_BlockSize = 1024;
};

struct rle_f : format {
    static const int ms_code = MS_FMT_RLE;
    static const unsigned ms_bw = 0;
};

// Default formats of a processing style (default_formats.h:35-82).
#define DEFAULT_STATIC_VBP_F(ve, bw) morphstore::static_vbp_f<morphstore::vbp_l<bw, ve::vector_helper_t::element_count::value>>
#define DEFAULT_DYNAMIC_VBP_F(ve)                                                                 \
    morphstore::dynamic_vbp_f<ve::vector_helper_t::size_bit::value, ve::vector_helper_t::size_byte::value, \
                              ve::vector_helper_t::element_count::value>
#define DEFAULT_DELTA_DYNAMIC_VBP_F(ve) \
    morphstore::delta_f<1024, ve::vector_helper_t::element_count::value, DEFAULT_DYNAMIC_VBP_F(ve)>
#define DEFAULT_FOR_DYNAMIC_VBP_F(ve) \
    morphstore::for_f<1024, ve::vector_helper_t::element_count::value, DEFAULT_DYNAMIC_VBP_F(ve)>

// --------------------------------------------------------------------------
// device context: the arena that replaces the query memory manager
// (include/core/memory/management/query_mm.h:83-238) and the stream
// --------------------------------------------------------------------------
namespace gpu {

inline void check(int status, const char *where) {
    if (status != MS_OK) throw std::runtime_error(std::string(where) + ": " + ms_gpu_status_string(status));
}

struct context {
    ms_arena *arena = nullptr;
    void *stream = nullptr;
    static context &get() {
        static context c;
        if (!c.arena) {
            const char *env = std::getenv("MSV_GPU_ARENA_BYTES");
            const uint64_t cap = env ? std::strtoull(env, nullptr, 10) : (uint64_t(8) << 30);
            check(ms_gpu_arena_create(cap, &c.arena), "arena_create");
        }
        return c;
    }
};

inline ms_arena *arena() { return context::get().arena; }
inline void *stream() { return context::get().stream; }
inline void reset_query_memory() { check(ms_gpu_arena_reset(arena()), "arena_reset"); }

}  // namespace gpu

// --------------------------------------------------------------------------
// column<F> (column.h:45-287), device-resident
// --------------------------------------------------------------------------
template <class F> class column {
    ms_col m_Desc;

public:
    explicit column(const ms_col &d) : m_Desc(d) {}
    column(const column &) = delete;

    const ms_col *desc() const { return &m_Desc; }
    ms_col *desc() { return &m_Desc; }
    const void *get_data() const { return m_Desc.data; }  // a device pointer
    size_t get_count_values() const { return m_Desc.count_values; }
    size_t get_size_used_byte() const { return m_Desc.size_used_byte; }
    size_t get_size_compr_byte() const { return m_Desc.size_compr_byte; }

    // The raw bytes (compressed part, gap, uncompressed rest) on the host.
    std::vector<uint8_t> raw_bytes() const {
        std::vector<uint8_t> h(m_Desc.size_used_byte);
        gpu::check(ms_gpu_memcpy(h.data(), m_Desc.data, h.size(), 1, 1, gpu::stream()), "raw_bytes");
        return h;
    }

    // Decompressed values on the host.
    std::vector<uint64_t> to_host() const;

    // Upload bytes in the reference layout (e.g. written by binary_io<F>).
    static const column<F> *from_host_bytes(const uint8_t *bytes, uint64_t count, uint64_t used, uint64_t compr) {
        ms_col d{};
        d.format = F::ms_code;
        d.bw = F::ms_bw;
        d.count_values = count;
        d.size_used_byte = used;
        d.size_compr_byte = compr;
        d.size_alloc_byte = used + 64;
        gpu::check(ms_gpu_arena_alloc(gpu::arena(), used + 64, &d.data), "from_host_bytes");
        gpu::check(ms_gpu_memcpy(d.data, bytes, used, 0, 1, gpu::stream()), "from_host_bytes");
        auto *c = new column<F>(d);
        if (F::ms_code == MS_FMT_DYNAMIC_VBP || F::ms_code == MS_FMT_DELTA_DVBP || F::ms_code == MS_FMT_FOR_DVBP)
            gpu::check(ms_gpu_build_index(c->desc(), gpu::arena(), gpu::stream()), "build_index");
        return c;
    }
};

inline const column<uncompr_f> *make_column(const uint64_t *values, size_t n) {
    ms_col d{};
    d.format = MS_FMT_UNCOMPR;
    d.count_values = n;
    d.size_used_byte = 8 * n;
    d.size_alloc_byte = 8 * n + 8;
    gpu::check(ms_gpu_arena_alloc(gpu::arena(), 8 * n + 8, &d.data), "make_column");
    gpu::check(ms_gpu_memcpy(d.data, values, 8 * n, 0, 1, gpu::stream()), "make_column");
    return new column<uncompr_f>(d);
}

// make_column (column_gen.h:56-81)
inline const column<uncompr_f> *make_column(const std::vector<uint64_t> &v) { return make_column(v.data(), v.size()); }
inline const column<uncompr_f> *make_column(std::initializer_list<uint64_t> v) {
    return make_column(std::vector<uint64_t>(v));
}

// --------------------------------------------------------------------------
// morph (morph.h:81-241)
// --------------------------------------------------------------------------
template <class VE, class Dst, class Src> struct morph_t {
    static const column<Dst> *apply(const column<Src> *in) {
        ms_col out{};
        gpu::check(ms_gpu_morph(in->desc(), Dst::ms_code, Dst::ms_bw, &out, gpu::arena(), gpu::stream()), "morph");
        return new column<Dst>(out);
    }
};

template <class VE, class Dst, class Src> const column<Dst> *morph(const column<Src> *in) {
    return morph_t<VE, Dst, Src>::apply(in);
}

template <class F> std::vector<uint64_t> column<F>::to_host() const {
    const column<uncompr_f> *u = nullptr;
    ms_col d = m_Desc;
    if (F::ms_code != MS_FMT_UNCOMPR) {
        ms_col out{};
        gpu::check(ms_gpu_morph(&m_Desc, MS_FMT_UNCOMPR, 0, &out, gpu::arena(), gpu::stream()), "to_host");
        d = out;
    }
    std::vector<uint64_t> h(d.count_values);
    gpu::check(ms_gpu_memcpy(h.data(), d.data, 8 * h.size(), 1, 1, gpu::stream()), "to_host");
    (void)u;
    return h;
}

// --------------------------------------------------------------------------
// operators (include/core/operators/interfaces/*.h)
// --------------------------------------------------------------------------
template <template <class, int> class t_compare, class VE, class t_out_pos_f, class t_in_data_f>
struct my_select_wit_t {
    static const column<t_out_pos_f> *apply(const column<t_in_data_f> *in, const uint64_t val,
                                            const size_t /*outPosCountEstimate*/ = 0) {
        ms_col out{};
        gpu::check(ms_gpu_select(t_compare<VE, 64>::code, val, in->desc(), t_out_pos_f::ms_code, t_out_pos_f::ms_bw,
                                 &out, gpu::arena(), gpu::stream()),
                   "select");
        return new column<t_out_pos_f>(out);
    }
};

template <template <class, int> class t_compare, class VE, class t_out_pos_f, class t_in_data_f>
const column<t_out_pos_f> *select(const column<t_in_data_f> *in, const uint64_t val, const size_t est = 0) {
    return my_select_wit_t<t_compare, VE, t_out_pos_f, t_in_data_f>::apply(in, val, est);
}

template <class VE, class t_out_data_f, class t_in_data_f, class t_in_pos_f> struct my_project_wit_t {
    static const column<t_out_data_f> *apply(const column<t_in_data_f> *data, const column<t_in_pos_f> *pos) {
        ms_col out{};
        gpu::check(ms_gpu_project(data->desc(), pos->desc(), t_out_data_f::ms_code, t_out_data_f::ms_bw, &out,
                                  gpu::arena(), gpu::stream()),
                   "project");
        return new column<t_out_data_f>(out);
    }
};

template <class VE, class t_out_data_f, class t_in_data_f, class t_in_pos_f>
const column<t_out_data_f> *project(const column<t_in_data_f> *data, const column<t_in_pos_f> *pos) {
    return my_project_wit_t<VE, t_out_data_f, t_in_data_f, t_in_pos_f>::apply(data, pos);
}

// whole-column sum (agg_sum.h:56-65): a one-value uncompressed column
template <class VE, class F> const column<uncompr_f> *agg_sum(const column<F> *in) {
    void *d = nullptr;
    gpu::check(ms_gpu_arena_alloc(gpu::arena(), 8, &d), "agg_sum");
    gpu::check(ms_gpu_agg_sum(in->desc(), static_cast<uint64_t *>(d), gpu::arena(), gpu::stream()), "agg_sum");
    gpu::check(ms_gpu_arena_check(gpu::arena(), gpu::stream()), "agg_sum");
    ms_col out{};
    out.format = MS_FMT_UNCOMPR;
    out.count_values = 1;
    out.size_used_byte = 8;
    out.size_alloc_byte = 8;
    out.data = d;
    return new column<uncompr_f>(out);
}

// grouped sum (agg_sum.h:95-106)
template <class VE, class t_out_data_f, class t_in_gr_f, class t_in_data_f>
const column<t_out_data_f> *agg_sum(const column<t_in_gr_f> *gr, const column<t_in_data_f> *data, size_t ext_count) {
    static_assert(std::is_same<t_out_data_f, uncompr_f>::value, "grouped agg_sum writes uncompr_f");
    ms_col out{};
    gpu::check(ms_gpu_agg_sum_grouped(gr->desc(), data->desc(), ext_count, &out, gpu::arena(), gpu::stream()),
               "agg_sum(grouped)");
    return new column<t_out_data_f>(out);
}

// semi_join (join.h:193-218)
template <class VE, class OutF, class LF, class RF>
const column<OutF> *semi_join(const column<LF> *l, const column<RF> *r, size_t /*estimate*/ = 0) {
    ms_col out{};
    gpu::check(ms_gpu_semi_join(l->desc(), r->desc(), OutF::ms_code, OutF::ms_bw, &out, gpu::arena(), gpu::stream()),
               "semi_join");
    return new column<OutF>(out);
}

// intersect_sorted (intersect.h:52-63) / my_intersect_wit_t (intersect_compr.h:190-347)
template <class VE, class OutF, class LF, class RF>
const column<OutF> *intersect_sorted(const column<LF> *l, const column<RF> *r, size_t /*estimate*/ = 0) {
    ms_col out{};
    gpu::check(ms_gpu_intersect_sorted(l->desc(), r->desc(), OutF::ms_code, OutF::ms_bw, &out, gpu::arena(),
                                       gpu::stream()),
               "intersect_sorted");
    return new column<OutF>(out);
}

// natural equi-join (join.h:158-187): (build positions, probe positions)
template <class VE, class OutLF, class OutRF, class LF, class RF>
const std::tuple<const column<OutLF> *, const column<OutRF> *> join(const column<LF> *l, const column<RF> *r,
                                                                    size_t = 0) {
    ms_col ol{}, orr{};
    gpu::check(ms_gpu_natural_join(l->desc(), r->desc(), OutLF::ms_code, OutLF::ms_bw, OutRF::ms_code, OutRF::ms_bw,
                                   &ol, &orr, gpu::arena(), gpu::stream()),
               "join");
    return std::make_tuple(new column<OutLF>(ol), new column<OutRF>(orr));
}

template <class VE, class OutF, class LF, class RF> struct my_intersect_wit_t {
    static const column<OutF> *apply(const column<LF> *l, const column<RF> *r, size_t est = 0) {
        return intersect_sorted<VE, OutF, LF, RF>(l, r, est);
    }
};

// group_vec / unary group (group_compr.h:281-300, group.h:58-73)
template <class VE, class GrF, class ExtF, class InF>
const std::tuple<const column<GrF> *, const column<ExtF> *> group_vec(const column<InF> *in, size_t = 0) {
    ms_col gr{}, ext{};
    gpu::check(ms_gpu_group(nullptr, in->desc(), GrF::ms_code, &gr, ExtF::ms_code, &ext, gpu::arena(), gpu::stream()),
               "group");
    return std::make_tuple(new column<GrF>(gr), new column<ExtF>(ext));
}

template <class VE, class GrF, class ExtF, class InF>
const std::tuple<const column<GrF> *, const column<ExtF> *> group(const column<InF> *in, size_t est = 0) {
    return group_vec<VE, GrF, ExtF, InF>(in, est);
}

// binary group (group.h:97-112)
template <class VE, class GrF, class ExtF, class InGrF, class InF>
const std::tuple<const column<GrF> *, const column<ExtF> *> group(const column<InGrF> *gr_in, const column<InF> *in,
                                                                  size_t = 0) {
    ms_col gr{}, ext{};
    gpu::check(ms_gpu_group(gr_in->desc(), in->desc(), GrF::ms_code, &gr, ExtF::ms_code, &ext, gpu::arena(),
                            gpu::stream()),
               "group");
    return std::make_tuple(new column<GrF>(gr), new column<ExtF>(ext));
}

// --------------------------------------------------------------------------
// binary_io<F> (include/core/persistence/binary_io.h:40-87): the same file
// layout, columns loaded into device memory
// --------------------------------------------------------------------------
template <class F> class binary_io {
public:
    static const column<F> *load(const std::string &p_Filename) {
        ms_col d{};
        gpu::check(ms_col_load(p_Filename.c_str(), F::ms_code, F::ms_bw, &d, gpu::arena(), gpu::stream()), "load");
        return new column<F>(d);
    }
    static void store(const column<F> *p_Column, const std::string &p_FileName) {
        gpu::check(ms_col_store(p_Column->desc(), p_FileName.c_str(), gpu::stream()), "store");
    }
};

// --------------------------------------------------------------------------
// Additions with no single-call counterpart in the reference
// --------------------------------------------------------------------------
namespace gpu {

// Many columns in one persistent launch: for every column i, decompress ->
// select(value t_compare consts[i]) -> sum of the selected values; results are
// (count, sum) per column.  run() replays a CUDA graph captured on first use.
template <template <class, int> class t_compare> class select_sum_batch {
    ms_batch *m_B = nullptr;
    size_t m_N;
    void *m_Cnt = nullptr, *m_Sum = nullptr;

public:
    select_sum_batch(const std::vector<const ms_col *> &cols, const std::vector<uint64_t> &consts) : m_N(cols.size()) {
        if (consts.size() != cols.size()) throw std::runtime_error("select_sum_batch: one constant per column");
        std::vector<ms_col> d;
        for (const ms_col *c : cols) d.push_back(*c);
        check(ms_gpu_batch_create(d.data(), consts.data(), d.size(), t_compare<void, 64>::code, arena(), &m_B, stream()),
              "batch_create");
        check(ms_gpu_arena_alloc(arena(), 8 * (m_N + 1), &m_Cnt), "batch");
        check(ms_gpu_arena_alloc(arena(), 8 * (m_N + 1), &m_Sum), "batch");
    }
    select_sum_batch(const select_sum_batch &) = delete;
    ~select_sum_batch() { ms_gpu_batch_destroy(m_B); }

    void run(bool graph = true) {
        check((graph ? ms_gpu_batch_run_graph : ms_gpu_batch_run)(m_B, static_cast<uint64_t *>(m_Cnt),
                                                                   static_cast<uint64_t *>(m_Sum), stream()),
              "batch_run");
    }
    // (count, sum) per column, after the last run
    std::vector<std::pair<uint64_t, uint64_t>> results() const {
        check(ms_gpu_arena_check(arena(), stream()), "batch");
        std::vector<uint64_t> c(m_N), s(m_N);
        check(ms_gpu_memcpy(c.data(), m_Cnt, 8 * m_N, 1, 1, stream()), "batch");
        check(ms_gpu_memcpy(s.data(), m_Sum, 8 * m_N, 1, 1, stream()), "batch");
        std::vector<std::pair<uint64_t, uint64_t>> r(m_N);
        for (size_t i = 0; i < m_N; i++) r[i] = {c[i], s[i]};
        return r;
    }
};

// The fused star query: select(filter t_compare c) -> semi_join(dim, fk) ->
// intersect -> project(gkey, measure) -> group -> grouped agg_sum in one
// pass; the result equals the operator chain's (keys, extents, sums in
// group-id order).
struct star_query_result {
    std::vector<uint64_t> keys, extents, sums;
    uint64_t rows;  // |P|, the rows that pass both filters
};

template <template <class, int> class t_compare, class FF, class KF, class LF, class GF, class MF>
star_query_result star_query(const column<FF> *filter, uint64_t c, const column<KF> *fk, const column<LF> *dim,
                             const column<GF> *gkey, const column<MF> *measure, size_t max_groups = 1 << 20) {
    star_query_result r;
    r.keys.resize(max_groups);
    r.extents.resize(max_groups);
    r.sums.resize(max_groups);
    uint64_t ng = 0;
    check(ms_gpu_query3(filter->desc(), t_compare<void, 64>::code, c, fk->desc(), dim->desc(), gkey->desc(),
                        measure->desc(), max_groups, r.keys.data(), r.extents.data(), r.sums.data(), &ng, &r.rows,
                        arena(), stream()),
          "star_query");
    r.keys.resize(ng);
    r.extents.resize(ng);
    r.sums.resize(ng);
    return r;
}

}  // namespace gpu

}  // namespace morphstore
