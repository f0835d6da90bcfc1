// star_and_batch.cpp -- the two additions of the drop-in header, checked
// against the reference-style operator chain and a host computation:
//   * gpu::star_query: select(filter < 400) -> semi_join(dim, fk) ->
//     group(gkey) -> sum(measure) in one pass;
//   * gpu::select_sum_batch: decompress -> select(< c_i) -> sum over many
//     columns in one persistent launch (replayed from a CUDA graph).
#include <morphstore_b200/morphstore.h>

#include <cinttypes>
#include <cstdio>
#include <map>
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
    using ve = gpu_b200<v512<uint64_t>>;
    using dv = DEFAULT_DYNAMIC_VBP_F(ve);
    using dd = DEFAULT_DELTA_DYNAMIC_VBP_F(ve);
    const size_t n = argc > 1 ? std::strtoull(argv[1], nullptr, 10) : 1000003;
    int bad = 0;

    // ---- star query --------------------------------------------------------
    std::vector<uint64_t> fk(n), filt(n), gkey(n), meas(n), dim;
    for (size_t i = 0; i < n; i++) {
        fk[i] = mix64(1, i) >> 50;  // 14 bits
        filt[i] = mix64(2, i) >> 52;
        gkey[i] = (mix64(3, i) >> 54) % 300;
        meas[i] = mix64(4, i) >> 48;
    }
    for (uint64_t k = 0; k < (1u << 14); k++)
        if (mix64(5, k) % 10 == 0) dim.push_back(k);
    auto cf = morph<ve, dv>(make_column(filt));
    auto ck = morph<ve, dv>(make_column(fk));
    auto cg = morph<ve, dv>(make_column(gkey));
    auto cm = morph<ve, dv>(make_column(meas));
    auto cd = morph<ve, dd>(make_column(dim));
    const auto r = gpu::star_query<less>(cf, 400, ck, cd, cg, cm);

    // the operator chain, as a reference query would write it
    auto p1 = my_select_wit_t<less, ve, uncompr_f, dv>::apply(cf, 400);
    auto p2 = semi_join<ve, uncompr_f, dd, dv>(cd, ck);
    auto p = intersect_sorted<ve, uncompr_f, uncompr_f, uncompr_f>(p1, p2);
    auto g = my_project_wit_t<ve, uncompr_f, dv, uncompr_f>::apply(cg, p);
    auto m = my_project_wit_t<ve, uncompr_f, dv, uncompr_f>::apply(cm, p);
    auto grext = group_vec<ve, uncompr_f, uncompr_f, uncompr_f>(g);
    auto s = agg_sum<ve, uncompr_f, uncompr_f, uncompr_f>(std::get<0>(grext), m,
                                                          std::get<1>(grext)->get_count_values());
    const auto ext = std::get<1>(grext)->to_host(), sums = s->to_host(), gv = g->to_host();
    bool ok = r.rows == p->get_count_values() && r.keys.size() == ext.size();
    for (size_t i = 0; ok && i < ext.size(); i++)
        ok = r.extents[i] == ext[i] && r.keys[i] == gv[ext[i]] && r.sums[i] == sums[i];
    // host check of the sums
    std::map<uint64_t, uint64_t> hs;
    for (size_t i = 0; i < n; i++)
        if (filt[i] < 400 && mix64(5, fk[i]) % 10 == 0) hs[gkey[i]] += meas[i];
    ok = ok && hs.size() == r.keys.size();
    for (size_t i = 0; ok && i < r.keys.size(); i++) ok = hs[r.keys[i]] == r.sums[i];
    std::printf("star_query: %zu groups over %" PRIu64 " rows: %s\n", r.keys.size(), r.rows, ok ? "ok" : "MISMATCH");
    bad |= !ok;

    // ---- batch -------------------------------------------------------------
    std::vector<const ms_col *> cols;
    std::vector<uint64_t> consts;
    std::vector<std::vector<uint64_t>> vals;
    for (int c = 0; c < 40; c++) {
        const size_t len = 1000 + mix64(6, c) % 300000;
        std::vector<uint64_t> v(len);
        for (size_t i = 0; i < len; i++) v[i] = mix64(7 + c, i) >> (40 + c % 20);
        auto u = make_column(v);
        const ms_col *d = (c % 3 == 0)   ? morph<ve, dv>(u)->desc()
                          : (c % 3 == 1) ? morph<ve, DEFAULT_FOR_DYNAMIC_VBP_F(ve)>(u)->desc()
                                         : morph<ve, DEFAULT_STATIC_VBP_F(ve, 64)>(u)->desc();
        cols.push_back(d);
        consts.push_back(v[len / 2]);
        vals.push_back(v);
    }
    gpu::select_sum_batch<less> batch(cols, consts);
    batch.run();
    batch.run();
    const auto br = batch.results();
    bool bok = true;
    for (size_t c = 0; c < cols.size(); c++) {
        uint64_t cnt = 0, sum = 0;
        for (uint64_t x : vals[c])
            if ((int64_t)x < (int64_t)consts[c]) cnt++, sum += x;
        bok = bok && br[c].first == cnt && br[c].second == sum;
    }
    std::printf("select_sum_batch: %zu columns: %s\n", cols.size(), bok ? "ok" : "MISMATCH");
    bad |= !bok;
    return bad;
}
