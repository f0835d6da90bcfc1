"""GPU operator parity (select, project, agg_sum, fused select-project-sum)
against the oracle, on seeded inputs in every input format."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

IN_FORMATS = [(O.UNCOMPR, 0), (O.STATIC_VBP, 12), (O.DYNAMIC_VBP, 0), (O.DELTA_DVBP, 0), (O.FOR_DVBP, 0)]
OUT_FORMATS = [(O.UNCOMPR, 0), (O.STATIC_VBP, 32), (O.DYNAMIC_VBP, 0), (O.DELTA_DVBP, 0), (O.FOR_DVBP, 0)]


def F(ms, code, bw=0):
    return {O.UNCOMPR: ms.uncompr_f, O.DYNAMIC_VBP: ms.dynamic_vbp_f, O.DELTA_DVBP: ms.delta_f,
            O.FOR_DVBP: ms.for_f, O.RLE: ms.rle_f}.get(code) or ms.static_vbp_f(bw)


def _col(ms, arena, orc, v, code, bw):
    """Upload in the reference byte layout (written by the oracle)."""
    if code == O.UNCOMPR:
        return ms.Column.from_numpy(v, arena)
    b, m = orc.compress(code, bw, v)
    return ms.Column.from_bytes(F(ms, code, bw), b, m, arena)


def _data(orc, code, n, seed):
    if code == O.DELTA_DVBP:
        return orc.sorted_gaps(seed, orc.geom_table(0.25), n) % np.uint64(4096)
    return orc.uniform_bits(seed, 12, n)


@pytest.mark.parametrize("code,bw", IN_FORMATS)
@pytest.mark.parametrize("n", [0, 5, 511, 512, 1025, 4099, 70_003])
def test_agg_sum(ms, arena, orc, code, bw, n):
    v = _data(orc, code, n, seed=n + 1)
    c = _col(ms, arena, orc, v, code, bw)
    assert ms.agg_sum(c) == orc.agg_sum(v)


def test_agg_sum_rle(ms, arena, orc):
    v = orc.runs(3, 5, 20, 100_003)
    c = ms.morph(ms.Column.from_numpy(v, arena), ms.rle_f)
    assert ms.agg_sum(c) == orc.agg_sum(v)


@pytest.mark.parametrize("code,bw", IN_FORMATS)
@pytest.mark.parametrize("cmp", [O.CMP_EQ, O.CMP_LT, O.CMP_LE, O.CMP_GT, O.CMP_GE])
def test_select_uncompr_out(ms, arena, orc, code, bw, cmp):
    n = 40_000 + 77
    v = _data(orc, code, n, seed=cmp + 10 * code)
    c = _col(ms, arena, orc, v, code, bw)
    val = int(np.median(v)) if n else 0
    out = ms.select(cmp, c, val)
    sf = orc.scalar_from(code, bw, c.meta())
    assert np.array_equal(out.to_numpy(), orc.select(cmp, val, v, sf))


@pytest.mark.parametrize("in_code,in_bw", IN_FORMATS)
@pytest.mark.parametrize("out_code,out_bw", OUT_FORMATS)
def test_select_compressed_out_bytes(ms, arena, orc, in_code, in_bw, out_code, out_bw):
    """Compressed positions follow the write iterator's 2048-value chunking."""
    n = 3 * 8192 + 1029
    v = _data(orc, in_code, n, seed=77)
    c = _col(ms, arena, orc, v, in_code, in_bw)
    out = ms.select(O.CMP_LT, c, 2000, F(ms, out_code, out_bw))
    sf = orc.scalar_from(in_code, in_bw, c.meta())
    pos = orc.select(O.CMP_LT, 2000, v, sf)
    n_scal = int((pos >= sf).sum())
    b, m = orc.wi_write(out_code, out_bw, pos, n_scal)
    assert out.meta() == m
    assert np.array_equal(O.mask_gap(out_code, out_bw, out.raw_bytes(), m, orc), O.mask_gap(out_code, out_bw, b, m, orc))
    assert np.array_equal(out.to_numpy(), pos)


def test_select_signed_semantics(ms, arena, orc):
    """Values >= 2^63 compare signed before the scalar remainder, unsigned in it."""
    v = orc.uniform_bits(5, 64, 4096 + 5)
    c = ms.Column.from_numpy(v, arena)
    out = ms.select(O.CMP_LT, c, 1 << 40)
    assert np.array_equal(out.to_numpy(), orc.select(O.CMP_LT, 1 << 40, v, len(v) - len(v) % 8))


@pytest.mark.parametrize("data_code,data_bw", IN_FORMATS + [(O.RLE, 0)])
@pytest.mark.parametrize("pos_code,pos_bw", [(O.UNCOMPR, 0), (O.DYNAMIC_VBP, 0), (O.DELTA_DVBP, 0)])
def test_project(ms, arena, orc, data_code, data_bw, pos_code, pos_bw):
    n = 20_000 + 13
    v = _data(orc, data_code, n, seed=3) if data_code != O.RLE else orc.runs(3, 5, 12, n)
    if data_code == O.RLE:
        d = ms.morph(ms.Column.from_numpy(v, arena), ms.rle_f)
    else:
        d = _col(ms, arena, orc, v, data_code, data_bw)
    pos = np.sort(orc.uniform_bits(4, 14, 9000) % np.uint64(n)).astype(np.uint64)
    pcol = _col(ms, arena, orc, pos, pos_code, pos_bw)
    out = ms.project(d, pcol)
    assert np.array_equal(out.to_numpy(), v[pos.astype(np.int64)])


def test_project_compressed_output(ms, arena, orc):
    n = 30_000
    v = orc.uniform_bits(8, 20, n)
    d = _col(ms, arena, orc, v, O.DYNAMIC_VBP, 0)
    pos = np.arange(0, n, 3, dtype=np.uint64)
    pcol = ms.Column.from_numpy(pos, arena)
    out = ms.project(d, pcol, ms.dynamic_vbp_f)
    vals = v[pos.astype(np.int64)]
    b, m = orc.wi_write(O.DYNAMIC_VBP, 0, vals, len(pos) % 8)
    assert out.meta() == m
    assert np.array_equal(O.mask_gap(O.DYNAMIC_VBP, 0, out.raw_bytes(), m, orc), O.mask_gap(O.DYNAMIC_VBP, 0, b, m, orc))


@pytest.mark.parametrize("xcode,xbw", [(O.STATIC_VBP, 10), (O.DYNAMIC_VBP, 0), (O.UNCOMPR, 0), (O.FOR_DVBP, 0)])
@pytest.mark.parametrize("ycode,ybw", [(O.DYNAMIC_VBP, 0), (O.UNCOMPR, 0), (O.STATIC_VBP, 20), (O.DELTA_DVBP, 0)])
@pytest.mark.parametrize("n", [1, 1000, 1 << 16, (1 << 16) + 333])
def test_select_project_sum(ms, arena, orc, xcode, xbw, ycode, ybw, n):
    x = orc.uniform_bits(1000 + n, 10, n)
    y = orc.uniform_bits(2000 + n, 20, n) if ycode != O.DELTA_DVBP else orc.sorted_gaps(n, orc.geom_table(0.25), n)
    xc = _col(ms, arena, orc, x, xcode, xbw)
    yc = _col(ms, arena, orc, y, ycode, ybw)
    sf = orc.scalar_from(xcode, xbw, xc.meta())
    s, k, pos, vals = ms.select_project_sum(xc, O.CMP_LT, 512, yc, want_positions=True)
    es, ek = orc.select_project_sum(O.CMP_LT, 512, x, y, sf)
    epos = orc.select(O.CMP_LT, 512, x, sf)
    assert (s, k) == (es, ek)
    assert np.array_equal(pos, epos)
    assert np.array_equal(vals, y[epos.astype(np.int64)])


@pytest.mark.parametrize("cfg", [
    dict(staged=0),
    dict(staged=1, warps=8, stages=3, stage_bytes=16384, values_per_thread=16),
    dict(staged=1, warps=24, stages=4, stage_bytes=49152, values_per_thread=16),
    dict(staged=1, warps=12, stages=6, stage_bytes=24576, values_per_thread=32),
    dict(staged=1, warps=24, stages=4, stage_bytes=49152, values_per_thread=32),
    dict(staged=1, warps=20, stages=3, stage_bytes=65536, values_per_thread=32),
])
@pytest.mark.parametrize("xcode,ycode", [(O.DYNAMIC_VBP, O.DYNAMIC_VBP), (O.STATIC_VBP, O.UNCOMPR),
                                         (O.FOR_DVBP, O.DELTA_DVBP)])
def test_select_project_sum_every_launch_config(ms, arena, orc, cfg, xcode, ycode):
    """Every kernel variant the autotuner can pick gives the oracle's result,
    including odd tile/warp splits, odd bit widths and 33..64-bit blocks."""
    n = (1 << 18) + 4321
    x = orc.uniform_bits(77, 13, n)
    x[::7] >>= np.uint64(6)           # blocks of mixed widths
    y = orc.uniform_bits(78, 40, n) if ycode != O.DELTA_DVBP else orc.sorted_gaps(3, orc.geom_table(0.25), n)
    xc = _col(ms, arena, orc, x, xcode, 13)
    yc = _col(ms, arena, orc, y, ycode, 0)
    old = ms.get_tuning()
    try:
        ms.set_tuning(**{**old, **cfg})
        for cmp, c in ((O.CMP_LT, 900), (O.CMP_GE, 4000), (O.CMP_EQ, 17), (O.CMP_LE, 0)):
            s, k = ms.select_project_sum(xc, cmp, c, yc)
            sf = orc.scalar_from(xcode, 13, xc.meta())
            assert (s, k) == orc.select_project_sum(cmp, c, x, y, sf), (cmp, c)
    finally:
        ms.set_tuning(**old)


@pytest.mark.parametrize("bw", list(range(1, 33)))
def test_threshold_path_every_width(ms, arena, orc, bw):
    """The in-register threshold test of the 32-values-per-thread path at
    every width up to 32 bits, with constants at the edges of the value
    range (0, 1, half, 2^bw - 1, 2^bw) and every comparison."""
    n = 4 * 1024 + 8 * 512 + 5
    x = orc.uniform_bits(100 + bw, bw, n)
    y = orc.uniform_bits(200 + bw, 20, n)
    xc = ms.morph(ms.Column.from_numpy(x, arena), ms.static_vbp_f(bw))
    xd = ms.morph(ms.Column.from_numpy(x, arena), ms.dynamic_vbp_f)
    yc = ms.morph(ms.Column.from_numpy(y, arena), ms.dynamic_vbp_f)
    old = ms.get_tuning()
    try:
        ms.set_tuning(**{**old, **dict(staged=1, warps=16, stages=3, stage_bytes=65536, values_per_thread=32)})
        for c in sorted({0, 1, 1 << (bw - 1), (1 << bw) - 1, 1 << bw}):
            for cmp in (O.CMP_LT, O.CMP_LE, O.CMP_GT, O.CMP_GE):
                for col, code, cbw in ((xc, O.STATIC_VBP, bw), (xd, O.DYNAMIC_VBP, 0)):
                    sf = orc.scalar_from(code, cbw, col.meta())
                    assert ms.select_project_sum(col, cmp, c, yc) == orc.select_project_sum(cmp, c, x, y, sf), \
                        (bw, c, cmp, code)
    finally:
        ms.set_tuning(**old)

