// ref_style_diff.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The reference's own operator templates, called twice on the same columns:
// once with the reference's AVX-512 processing style (its CPU code) and once
// with the gpu_b200 style of engine_b200/include/morphstore_b200/ve_gpu_b200.h
// (the GPU path behind the same templates).  Every output column must be
// identical: metadata, compressed bytes (the never-written gap and for_f's
// never-written header words excepted) and values.  Where the reference's
// vectorised operator is unusable (my_intersect_wit_t crashes in this build;
// grouped agg_sum, binary group and intersect_sorted exist for the scalar
// style only) the scalar style is the CPU side.
//
// Built by oracle/Makefile (target `style`) from the reference's headers where
// they lie; linked against libms_gpu.so.  Prints one line per case and exits
// non-zero if any case differs.
#include <core/operators/scalar/agg_sum_uncompr.h>
#include <core/operators/scalar/group_uncompr.h>
#include <core/operators/scalar/intersect_uncompr.h>
#include <core/operators/scalar/select_uncompr.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace morphstore;
using namespace vectorlib;

using cpu = avx512<v512<uint64_t>>;
using gpu = gpu_b200<v512<uint64_t>>;
using sc = scalar<v64<uint64_t>>;
using uf = uncompr_f;
using dv = DEFAULT_DYNAMIC_VBP_F(cpu);
using dd = DEFAULT_DELTA_DYNAMIC_VBP_F(cpu);
using fd = DEFAULT_FOR_DYNAMIC_VBP_F(cpu);
using s10 = DEFAULT_STATIC_VBP_F(cpu, 10);
using s20 = DEFAULT_STATIC_VBP_F(cpu, 20);

static_assert(std::is_same<dv, DEFAULT_DYNAMIC_VBP_F(gpu)>::value, "gpu_b200 names the AVX-512 layouts");

static int g_failures = 0, g_cases = 0;

static uint64_t mix64(uint64_t seed, uint64_t i) {
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static const column<uf> *ucol(const std::vector<uint64_t> &v) {
    auto *c = new column<uf>(std::max<size_t>(8 * v.size(), 8));
    if (!v.empty()) std::memcpy(c->get_data(), v.data(), 8 * v.size());
    c->set_meta_data(v.size(), 8 * v.size());
    return c;
}

template <class F> static std::vector<uint64_t> values_of(const column<F> *c) {
    const column<uf> *u = morph<cpu, uf>(c);
    const uint64_t *p = u->get_data();
    std::vector<uint64_t> v(p, p + u->get_count_values());
    if (static_cast<const void *>(u) != static_cast<const void *>(c)) delete u;
    return v;
}

// for_f pages: 8 reference words, then per 1024-block an inner dynamic_vbp
// page (64-byte header whose first two bytes are the widths + 2 blocks); the
// words after a UINT64_MAX marker are never written (for.h:214-220)
static void mask_for_headers(std::vector<uint8_t> &d, size_t compr) {
    size_t i = 0;
    while (i < compr) {
        const size_t h0 = i;
        i += 64;
        for (unsigned j = 0; j < 8; j++) {
            uint64_t ref;
            std::memcpy(&ref, &d[h0 + 8 * j], 8);
            if (ref == ~uint64_t(0)) {
                std::memset(&d[h0 + 8 * (j + 1)], 0, 64 - 8 * (j + 1));
                break;
            }
            i += 64 + 64 * (size_t(d[i]) + size_t(d[i + 1]));
        }
    }
}

template <class F> static std::vector<uint8_t> meaningful_bytes(const column<F> *c) {
    const uint8_t *p = c->get_data();
    const size_t used = c->get_size_used_byte(), compr = c->get_size_compr_byte();
    std::vector<uint8_t> d(p, p + used);
    if (!std::is_same<F, uf>::value && !std::is_same<F, rle_f>::value && used > compr) {
        const size_t rest = static_cast<const uint8_t *>(c->get_data_uncompr_start()) - p;
        std::memset(d.data() + compr, 0, rest - compr);
    }
    if (std::is_same<F, fd>::value && compr) mask_for_headers(d, compr);
    return d;
}

template <class F> static void check(const std::string &name, const column<F> *want, const column<F> *got) {
    g_cases++;
    std::string why;
    if (want->get_count_values() != got->get_count_values()) why = "count";
    else if (want->get_size_used_byte() != got->get_size_used_byte()) why = "size_used_byte";
    else if (want->get_size_compr_byte() != got->get_size_compr_byte()) why = "size_compr_byte";
    else if (meaningful_bytes(want) != meaningful_bytes(got)) why = "bytes";
    else if (values_of(want) != values_of(got)) why = "values";
    std::printf("%s %s%s%s\n", why.empty() ? "ok  " : "FAIL", name.c_str(), why.empty() ? "" : ": ", why.c_str());
    if (!why.empty()) g_failures++;
}

template <class F> static void del(const column<F> *c) { delete c; }

template <class F> static const column<F> *as(const column<uf> *u) { return morph<cpu, F>(u); }

template <class F> static void per_format(const char *fname, const std::vector<uint64_t> &x, uint64_t c) {
    const column<uf> *xu = ucol(x);
    const column<F> *xc = std::is_same<F, uf>::value ? reinterpret_cast<const column<F> *>(xu) : as<F>(xu);
    const std::string tag = std::string(fname) + " n=" + std::to_string(x.size());
    if (!std::is_same<F, uf>::value) {
        const column<F> *g = morph<gpu, F>(xu);
        check("morph " + tag, xc, g);
        del(g);
    }
    {
        const column<uf> *w = my_select_wit_t<less, cpu, uf, F>::apply(xc, c);
        const column<uf> *g = my_select_wit_t<less, gpu, uf, F>::apply(xc, c);
        check("select<less> -> uncompr " + tag, w, g);
        del(w), del(g);
    }
    {
        const column<dv> *w = my_select_wit_t<greaterequal, cpu, dv, F>::apply(xc, c);
        const column<dv> *g = my_select_wit_t<greaterequal, gpu, dv, F>::apply(xc, c);
        check("select<greaterequal> -> dynamic_vbp " + tag, w, g);
        del(w), del(g);
    }
    {
        const column<dd> *w = my_select_wit_t<equal, cpu, dd, F>::apply(xc, c / 2);
        const column<dd> *g = my_select_wit_t<equal, gpu, dd, F>::apply(xc, c / 2);
        check("select<equal> -> delta " + tag, w, g);
        del(w), del(g);
    }
    {
        const column<uf> *w = agg_sum<cpu, F>(xc);
        const column<uf> *g = agg_sum<gpu, F>(xc);
        check("agg_sum " + tag, w, g);
        del(w), del(g);
    }
    {
        auto w = group_vec<cpu, uf, uf, F>(xc);
        auto g = group_vec<gpu, uf, uf, F>(xc);
        check("group_vec ids " + tag, std::get<0>(w), std::get<0>(g));
        check("group_vec extents " + tag, std::get<1>(w), std::get<1>(g));
        del(std::get<0>(w)), del(std::get<1>(w)), del(std::get<0>(g)), del(std::get<1>(g));
    }
    if (static_cast<const void *>(xc) != static_cast<const void *>(xu)) del(xc);
    del(xu);
}

int main() {
    for (size_t n : {size_t(100003), size_t(1) << 20, size_t(777)}) {
        std::vector<uint64_t> x(n), y(n);
        for (size_t i = 0; i < n; i++) {
            x[i] = mix64(11, i) >> 54;  // 10 bits
            y[i] = mix64(12, i) >> 44;  // 20 bits
        }
        per_format<uf>("uncompr", x, 512);
        per_format<s10>("static_vbp<10>", x, 512);
        per_format<dv>("dynamic_vbp", x, 512);
        per_format<dd>("delta+dvbp", x, 512);
        per_format<fd>("for+dvbp", x, 512);

        // select -> project (data uncompr / static_vbp; positions uncompr / dvbp)
        const column<uf> *xu = ucol(x), *yu = ucol(y);
        const column<s20> *ys = as<s20>(yu);
        const column<uf> *pos = my_select_wit_t<less, cpu, uf, uf>::apply(xu, 300);
        const column<dv> *posd = my_select_wit_t<less, cpu, dv, uf>::apply(xu, 300);
        const std::string tag = " n=" + std::to_string(n);
        {
            const column<uf> *w = my_project_wit_t<cpu, uf, uf, uf>::apply(yu, pos);
            const column<uf> *g = my_project_wit_t<gpu, uf, uf, uf>::apply(yu, pos);
            check("project uncompr[uncompr] -> uncompr" + tag, w, g);
            del(w), del(g);
        }
        {
            const column<dv> *w = my_project_wit_t<cpu, dv, s20, dv>::apply(ys, posd);
            const column<dv> *g = my_project_wit_t<gpu, dv, s20, dv>::apply(ys, posd);
            check("project static_vbp<20>[dynamic_vbp] -> dynamic_vbp" + tag, w, g);
            del(w), del(g);
        }
        {
            const column<uf> *w = agg_sum<cpu, uf>(my_project_wit_t<cpu, uf, uf, uf>::apply(yu, pos));
            const column<uf> *g = agg_sum<gpu, uf>(my_project_wit_t<gpu, uf, uf, uf>::apply(yu, pos));
            check("select -> project -> agg_sum" + tag, w, g);
            del(w), del(g);
        }

        // semi-join and natural join: build side = sorted unique keys (delta+dvbp),
        // probe side = foreign keys (for+dvbp)
        std::vector<uint64_t> keys, fk(n);
        for (uint64_t k = 0; k < (uint64_t(1) << 16); k++)
            if ((mix64(13, k) & 7) == 0) keys.push_back(k);
        for (size_t i = 0; i < n; i++) fk[i] = mix64(14, i) >> 48;
        const column<uf> *ku = ucol(keys), *fku = ucol(fk);
        const column<dd> *kd = as<dd>(ku);
        const column<fd> *fkf = as<fd>(fku);
        {
            const column<uf> *w = semi_join<cpu, uf, dd, fd>(kd, fkf);
            const column<uf> *g = semi_join<gpu, uf, dd, fd>(kd, fkf);
            check("semi_join delta x for -> uncompr" + tag, w, g);
            del(w), del(g);
        }
        {
            const column<dv> *w = semi_join<cpu, dv, uf, uf>(ku, fku);
            const column<dv> *g = semi_join<gpu, dv, uf, uf>(ku, fku);
            check("semi_join uncompr x uncompr -> dynamic_vbp" + tag, w, g);
            del(w), del(g);
        }
        {
            auto w = join<cpu, uf, uf, dd, uf>(kd, fku);
            auto g = join<gpu, uf, uf, dd, uf>(kd, fku);
            check("join build positions" + tag, std::get<0>(w), std::get<0>(g));
            check("join probe positions" + tag, std::get<1>(w), std::get<1>(g));
            del(std::get<0>(w)), del(std::get<1>(w)), del(std::get<0>(g)), del(std::get<1>(g));
        }

        // scalar-style-only operators
        {
            auto gw = group<sc, uf, uf, uf>(xu, 0);
            auto gg = group<gpu, uf, uf, uf>(xu, 0);
            check("group (unary, interface)" + tag, std::get<0>(gw), std::get<0>(gg));
            const size_t ng = std::get<1>(gw)->get_count_values();
            const column<uf> *w = agg_sum<sc, uf, uf, uf>(std::get<0>(gw), yu, ng);
            const column<uf> *g = agg_sum<gpu, uf, uf, uf>(std::get<0>(gw), yu, ng);
            check("grouped agg_sum" + tag, w, g);
            auto bw = group<sc, uf, uf, uf, uf>(std::get<0>(gw), fku, 0);
            auto bg = group<gpu, uf, uf, uf, uf>(std::get<0>(gw), fku, 0);
            check("group (binary) ids" + tag, std::get<0>(bw), std::get<0>(bg));
            check("group (binary) extents" + tag, std::get<1>(bw), std::get<1>(bg));
            del(w), del(g), del(std::get<0>(gw)), del(std::get<1>(gw)), del(std::get<0>(gg)), del(std::get<1>(gg));
            del(std::get<0>(bw)), del(std::get<1>(bw)), del(std::get<0>(bg)), del(std::get<1>(bg));
        }
        {
            const column<uf> *p2 = my_select_wit_t<greater, cpu, uf, uf>::apply(yu, 1u << 19);
            const column<uf> *w = intersect_sorted<sc, uf, uf, uf>(pos, p2, 0);
            const column<uf> *g = intersect_sorted<gpu, uf, uf, uf>(pos, p2, 0);
            check("intersect_sorted" + tag, w, g);
            del(w), del(g), del(p2);
        }
        {
            // the interface select with a std functor: the scalar style's unsigned compare
            std::vector<uint64_t> w64(n);
            for (size_t i = 0; i < n; i++) w64[i] = mix64(15, i);
            const column<uf> *wu = ucol(w64);
            const column<uf> *w = select<std::less, sc, uf, uf>(wu, uint64_t(1) << 63, 0);
            const column<uf> *g = select<std::less, gpu, uf, uf>(wu, uint64_t(1) << 63, 0);
            check("select<std::less> (unsigned) on 64-bit values" + tag, w, g);
            del(w), del(g), del(wu);
        }
        del(pos), del(posd), del(xu), del(yu), del(ys), del(ku), del(fku), del(kd), del(fkf);
    }
    std::printf("%d of %d cases differ\n", g_failures, g_cases);
    return g_failures ? 1 : 0;
}
