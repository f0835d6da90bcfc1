"""The CUDA path against the golden fixtures written by the reference's own
code (tests/golden/make_golden.py): compressed bytes and metadata of every
codec case, select outputs in compressed formats, semi-join, group."""
import numpy as np
import pytest

import oracle as O
from golden_util import codec_cases, load

FX = load()
pytestmark = [pytest.mark.gpu, pytest.mark.skipif(FX is None, reason="golden fixtures missing")]


def F(ms, code, bw=0):
    return {O.UNCOMPR: ms.uncompr_f, O.DYNAMIC_VBP: ms.dynamic_vbp_f, O.DELTA_DVBP: ms.delta_f,
            O.FOR_DVBP: ms.for_f, O.RLE: ms.rle_f}.get(code) or ms.static_vbp_f(bw)


def test_codecs_match_reference_bytes(ms, arena, orc):
    for name, fmt, bw in codec_cases(FX):
        v = FX[f"in/{name}"]
        key = f"codec/{name}/{fmt}/{bw}"
        c = ms.morph(ms.Column.from_numpy(v, arena), F(ms, fmt, bw))
        m = tuple(int(x) for x in FX[key + "/meta"])
        assert c.meta() == m, key
        assert np.array_equal(O.mask_gap(fmt, bw, c.raw_bytes(), m, orc), FX[key + "/bytes"]), key
        # and the reference's bytes decode on the device
        d = ms.Column.from_bytes(F(ms, fmt, bw), FX[key + "/bytes"], m, arena)
        assert np.array_equal(d.to_numpy(), v), key


def test_static_vbp_all_widths(ms, arena, orc):
    for bw in range(1, 65):
        c = ms.morph(ms.Column.from_numpy(FX[f"static/{bw}/in"], arena), ms.static_vbp_f(bw))
        m = tuple(int(x) for x in FX[f"static/{bw}/meta"])
        assert c.meta() == m
        assert np.array_equal(O.mask_gap(O.STATIC_VBP, bw, c.raw_bytes(), m, orc), FX[f"static/{bw}/bytes"]), bw


def test_select_outputs(ms, arena, orc):
    x = FX["in/uni12_40077"]
    for in_fmt in (O.UNCOMPR, O.DYNAMIC_VBP, O.DELTA_DVBP, O.FOR_DVBP):
        xc = ms.Column.from_numpy(x, arena) if in_fmt == O.UNCOMPR else ms.morph(ms.Column.from_numpy(x, arena),
                                                                               F(ms, in_fmt))
        for out_fmt in (O.UNCOMPR, O.DYNAMIC_VBP, O.DELTA_DVBP, O.FOR_DVBP):
            out = ms.select(O.CMP_LT, xc, 1500, F(ms, out_fmt))
            key = f"select/{in_fmt}/{out_fmt}"
            m = tuple(int(v) for v in FX[key + "/meta"])
            assert out.meta() == m, key
            assert np.array_equal(O.mask_gap(out_fmt, 0, out.raw_bytes(), m, orc), FX[key + "/bytes"]), key
    for cmp in range(5):
        assert np.array_equal(ms.select(cmp, ms.Column.from_numpy(x, arena), 2048).to_numpy(), FX[f"select_cmp/{cmp}"])
    w = FX["in/uni64_9000"]
    assert np.array_equal(ms.select(O.CMP_LT, ms.Column.from_numpy(w, arena), 1 << 62).to_numpy(), FX["select_signed"])


def test_semi_join_intersect_group(ms, arena, orc):
    lc = ms.morph(ms.Column.from_numpy(FX["semi/l"], arena), ms.delta_f)
    rc = ms.morph(ms.Column.from_numpy(FX["semi/r"], arena), ms.for_f)
    for out_fmt in (O.UNCOMPR, O.DYNAMIC_VBP, O.DELTA_DVBP):
        out = ms.semi_join(lc, rc, F(ms, out_fmt))
        m = tuple(int(v) for v in FX[f"semi/{out_fmt}/meta"])
        assert out.meta() == m
        assert np.array_equal(O.mask_gap(out_fmt, 0, out.raw_bytes(), m, orc), FX[f"semi/{out_fmt}/bytes"])
    isect = ms.intersect_sorted(ms.Column.from_numpy(FX["isect/l"], arena), ms.Column.from_numpy(FX["isect/r"], arena))
    assert np.array_equal(isect.to_numpy(), FX["isect/out"])
    gc = ms.morph(ms.Column.from_numpy(FX["group/in"], arena), ms.dynamic_vbp_f)
    gr, ext = ms.group(gc)
    assert np.array_equal(gr.to_numpy(), FX["group/gr"])
    assert np.array_equal(ext.to_numpy(), FX["group/ext"])
    gr2, ext2 = ms.group(gc, gr_f=ms.dynamic_vbp_f, ext_f=ms.dynamic_vbp_f)
    for col, key in ((gr2, "group/gr_dvbp"), (ext2, "group/ext_dvbp")):
        m = tuple(int(v) for v in FX[key + "/meta"])
        assert col.meta() == m, key
        assert np.array_equal(O.mask_gap(O.DYNAMIC_VBP, 0, col.raw_bytes(), m, orc), FX[key + "/bytes"]), key
    s = ms.agg_sum_grouped(gr, ms.Column.from_numpy(FX["group/meas"], arena), ext.get_count_values())
    assert np.array_equal(s.to_numpy(), FX["group/sum"])


def test_natural_join_golden(ms, arena, orc):
    """Both output columns of the reference's natural join, byte for byte
    (delta+dvbp build side, for+dvbp probe side, uncompr and dvbp outputs)."""
    lc = ms.morph(ms.Column.from_numpy(FX["njoin/l"], arena), ms.delta_f)
    rc = ms.morph(ms.Column.from_numpy(FX["njoin/r"], arena), ms.for_f)
    for out_fmt in (O.UNCOMPR, O.DYNAMIC_VBP):
        ol, orr = ms.natural_join(lc, rc, F(ms, out_fmt), F(ms, out_fmt))
        for side, col in (("l", ol), ("r", orr)):
            m = tuple(int(v) for v in FX[f"njoin/{out_fmt}/{side}/meta"])
            assert col.meta() == m, (out_fmt, side)
            assert np.array_equal(O.mask_gap(out_fmt, 0, col.raw_bytes(), m, orc),
                                  FX[f"njoin/{out_fmt}/{side}/bytes"]), (out_fmt, side)

