"""Pins the C oracle to the reference: every golden fixture (compressed
bytes, metadata, operator outputs written by the reference's own code) is
reproduced by the oracle."""
import numpy as np
import pytest

import oracle as O
from golden_util import codec_cases, load

FX = load()
pytestmark = pytest.mark.skipif(FX is None, reason="golden fixtures missing")


def test_codecs(orc):
    n_cases = 0
    for name, fmt, bw in codec_cases(FX):
        v = FX[f"in/{name}"]
        b, m = orc.compress(fmt, bw, v)
        key = f"codec/{name}/{fmt}/{bw}"
        assert tuple(int(x) for x in FX[key + "/meta"]) == m, key
        assert np.array_equal(O.mask_gap(fmt, bw, b, m, orc), FX[key + "/bytes"]), key
        assert np.array_equal(orc.decompress(fmt, bw, FX[key + "/bytes"], m), v), key
        n_cases += 1
    assert n_cases >= 60


def test_static_vbp_every_width(orc):
    for bw in range(1, 65):
        b, m = orc.compress(O.STATIC_VBP, bw, FX[f"static/{bw}/in"])
        assert tuple(int(x) for x in FX[f"static/{bw}/meta"]) == m
        assert np.array_equal(O.mask_gap(O.STATIC_VBP, bw, b, m, orc), FX[f"static/{bw}/bytes"]), bw


def test_select_write_iterator_outputs(orc):
    x = FX["in/uni12_40077"]
    for in_fmt in (O.UNCOMPR, O.DYNAMIC_VBP, O.DELTA_DVBP, O.FOR_DVBP):
        meta = (len(x), 8 * len(x), 0) if in_fmt == O.UNCOMPR else orc.compress(in_fmt, 0, x)[1]
        sf = orc.scalar_from(in_fmt, 0, meta)
        pos = orc.select(O.CMP_LT, 1500, x, sf)
        nscal = int((pos >= sf).sum())
        for out_fmt in (O.UNCOMPR, O.DYNAMIC_VBP, O.DELTA_DVBP, O.FOR_DVBP):
            b, m = orc.wi_write(out_fmt, 0, pos, nscal)
            key = f"select/{in_fmt}/{out_fmt}"
            assert tuple(int(v) for v in FX[key + "/meta"]) == m, key
            assert np.array_equal(O.mask_gap(out_fmt, 0, b, m, orc), FX[key + "/bytes"]), key


def test_select_comparisons(orc):
    x = FX["in/uni12_40077"]
    for cmp in range(5):
        assert np.array_equal(orc.select(cmp, 2048, x), FX[f"select_cmp/{cmp}"]), cmp


def test_select_signed(orc):
    w = FX["in/uni64_9000"]
    assert np.array_equal(orc.select(O.CMP_LT, 1 << 62, w), FX["select_signed"])


def test_project(orc):
    y = FX["in/uni20_33009"]
    pos = np.arange(3, len(y), 7, dtype=np.uint64)
    vals = y[pos.astype(np.int64)]
    for out_fmt in (O.UNCOMPR, O.DYNAMIC_VBP):
        b, m = orc.wi_write(out_fmt, 0, vals, len(pos) % 8)
        assert tuple(int(v) for v in FX[f"project/{out_fmt}/meta"]) == m
        assert np.array_equal(O.mask_gap(out_fmt, 0, b, m, orc), FX[f"project/{out_fmt}/bytes"])


def test_agg_sum(orc):
    v = FX["in/sorted_33009"]
    for fmt in (O.UNCOMPR, O.DYNAMIC_VBP, O.DELTA_DVBP, O.FOR_DVBP):
        assert orc.agg_sum(v) == int(FX[f"agg_sum/{fmt}"][0])


def test_semi_join(orc):
    pos = orc.semi_join(FX["semi/l"], FX["semi/r"])
    rm = orc.compress(O.FOR_DVBP, 0, FX["semi/r"])[1]
    sf = orc.scalar_from(O.FOR_DVBP, 0, rm)
    for out_fmt in (O.UNCOMPR, O.DYNAMIC_VBP, O.DELTA_DVBP):
        b, m = orc.wi_write(out_fmt, 0, pos, int((pos >= sf).sum()))
        assert tuple(int(v) for v in FX[f"semi/{out_fmt}/meta"]) == m
        assert np.array_equal(O.mask_gap(out_fmt, 0, b, m, orc), FX[f"semi/{out_fmt}/bytes"])


def test_natural_join(orc):
    """The oracle's natural equi-join, written through the write-iterator
    model, reproduces the reference's two output columns byte for byte."""
    lpos, rpos = orc.natural_join(FX["njoin/l"], FX["njoin/r"])
    rm = orc.compress(O.FOR_DVBP, 0, FX["njoin/r"])[1]
    sf = orc.scalar_from(O.FOR_DVBP, 0, rm)
    nscal = int((rpos >= sf).sum())
    for out_fmt in (O.UNCOMPR, O.DYNAMIC_VBP):
        for side, vals in (("l", lpos), ("r", rpos)):
            b, m = orc.wi_write(out_fmt, 0, vals, nscal)
            assert tuple(int(v) for v in FX[f"njoin/{out_fmt}/{side}/meta"]) == m, (out_fmt, side)
            assert np.array_equal(O.mask_gap(out_fmt, 0, b, m, orc), FX[f"njoin/{out_fmt}/{side}/bytes"]), (out_fmt, side)


def test_intersect(orc):
    assert np.array_equal(orc.intersect_sorted(FX["isect/l"], FX["isect/r"]), FX["isect/out"])


def test_group_and_grouped_sum(orc):
    gr, ext = orc.group(FX["group/in"])
    assert np.array_equal(gr, FX["group/gr"])
    assert np.array_equal(ext, FX["group/ext"])
    gm = orc.compress(O.DYNAMIC_VBP, 0, FX["group/in"])[1]
    sf = orc.scalar_from(O.DYNAMIC_VBP, 0, gm)
    b, m = orc.wi_write(O.DYNAMIC_VBP, 0, gr, len(gr) - sf)
    assert tuple(int(v) for v in FX["group/gr_dvbp/meta"]) == m
    assert np.array_equal(O.mask_gap(O.DYNAMIC_VBP, 0, b, m, orc), FX["group/gr_dvbp/bytes"])
    b, m = orc.wi_write(O.DYNAMIC_VBP, 0, ext, int((ext >= sf).sum()))
    assert tuple(int(v) for v in FX["group/ext_dvbp/meta"]) == m
    assert np.array_equal(O.mask_gap(O.DYNAMIC_VBP, 0, b, m, orc), FX["group/ext_dvbp/bytes"])
    assert np.array_equal(orc.agg_sum_grouped(gr, FX["group/meas"], len(ext)), FX["group/sum"])


KATS = {
    "select": ([95, 102, 100, 87, 120], 100, [0, 3]),
    "project": ([11, 44, 22, 33, 11], [1, 3, 4], [44, 33, 11]),
    "agg_sum": ([100, 150, 50, 500, 200, 100], 1100),
    "agg_sum_grouped": ([0, 0, 1, 0, 2, 1], [100, 150, 50, 500, 200, 100], 3, [750, 150, 200]),
    "group_unary": ([333, 333, 111, 333, 222, 111], [0, 0, 1, 0, 2, 1], [0, 2, 4]),
    "group_binary": ([0, 0, 1, 0, 2, 1], [77, 88, 77, 77, 88, 88], [0, 1, 2, 0, 3, 4], [0, 1, 2, 4, 5]),
    "intersect": ([1, 4, 5, 8, 9, 12], [1, 6, 8, 12, 15], [1, 8, 12]),
}


def test_reference_known_answers(orc):
    """The reference's operator KATs (test/core/operators/*_test.cpp)."""
    u = lambda a: np.array(a, dtype=np.uint64)  # noqa: E731
    d, c, e = KATS["select"]
    assert list(orc.select(O.CMP_LT, c, u(d))) == e
    d, p, e = KATS["project"]
    assert list(u(d)[u(p).astype(np.int64)]) == e
    d, e = KATS["agg_sum"]
    assert orc.agg_sum(u(d)) == e
    g, d, n, e = KATS["agg_sum_grouped"]
    assert list(orc.agg_sum_grouped(u(g), u(d), n)) == e
    d, eg, ee = KATS["group_unary"]
    gr, ext = orc.group(u(d))
    assert list(gr) == eg and list(ext) == ee
    g, d, eg, ee = KATS["group_binary"]
    gr, ext = orc.group(u(d), gr_in=u(g))
    assert list(gr) == eg and list(ext) == ee
    l, r, e = KATS["intersect"]
    assert list(orc.intersect_sorted(u(l), u(r))) == e


def test_blockwise_container_restatement(orc):
    """The restated blockwise_individual_f container (candidate payloads from
    the C oracle, layout of blockwise_individual.h:169-311) equals the
    reference's own container for the same per-block picks."""
    from oracle import selector_ref as SR
    x, choice, codes = FX["bwi/in"], FX["bwi/choice"], FX["bwi/codes"]
    pays, got_codes = [], []
    for b, c in enumerate(choice):
        code, pay = SR.candidate_payload(orc, x[b * SR.BLOCK:(b + 1) * SR.BLOCK], int(c))
        got_codes.append(code)
        pays.append(pay)
    assert np.array_equal(np.array(got_codes, dtype=np.uint8), codes)
    sizes = np.array([len(p) for p in pays])
    code_off, pay_off, total = SR.container_positions(sizes)
    mine = np.zeros(total, dtype=np.uint8)
    for b, pay in enumerate(pays):
        mine[code_off[b]] = codes[b]
        mine[pay_off[b]:pay_off[b] + len(pay)] = pay
    assert np.array_equal(SR.mask_container(mine, choice), FX["bwi/bytes"])


def test_exhaustive_choice_restatement(orc):
    """Wherever the reference's exhaustive selector picks a format the GPU
    also offers, the smallest of the restated candidates (static_vbp,
    dynamic_vbp, delta+dvbp, for+dvbp; first one on ties, the reference's
    order) is that format."""
    from oracle import selector_ref as SR
    x = FX["bwi/in"]
    compared = 0
    for b, rc in enumerate(FX["bwi/exhaustive"]):
        want = SR.shared_code(int(rc))
        if want < 0:
            continue
        cands = [SR.candidate_payload(orc, x[b * SR.BLOCK:(b + 1) * SR.BLOCK], c) for c in range(4)]
        best = min(range(4), key=lambda c: (len(cands[c][1]), c))
        assert cands[best][0] == want, (b, cands[best][0], want)
        compared += 1
    assert compared >= 40
