"""GPU parity of semi_join, intersect_sorted, group and grouped agg_sum
against the oracle, including compressed inputs and outputs."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def F(ms, code, bw=0):
    return {O.UNCOMPR: ms.uncompr_f, O.DYNAMIC_VBP: ms.dynamic_vbp_f, O.DELTA_DVBP: ms.delta_f,
            O.FOR_DVBP: ms.for_f, O.RLE: ms.rle_f}.get(code) or ms.static_vbp_f(bw)


def _col(ms, arena, orc, v, code, bw=0):
    if code == O.UNCOMPR:
        return ms.Column.from_numpy(v, arena)
    b, m = orc.compress(code, bw, v)
    return ms.Column.from_bytes(F(ms, code, bw), b, m, arena)


@pytest.mark.parametrize("l_code", [O.UNCOMPR, O.DELTA_DVBP])
@pytest.mark.parametrize("r_code", [O.UNCOMPR, O.DYNAMIC_VBP, O.FOR_DVBP])
@pytest.mark.parametrize("out_code", [O.UNCOMPR, O.DYNAMIC_VBP, O.DELTA_DVBP])
def test_semi_join(ms, arena, orc, l_code, r_code, out_code):
    dim = orc.sorted_gaps(3, orc.geom_table(0.25), 4096)        # sorted unique keys
    keep = orc.uniform_bits(4, 4, len(dim)) < 2                   # ~12% of them
    lkeys = dim[keep]
    fk = orc.uniform_bits(5, 14, 50_000 + 11)
    lc = _col(ms, arena, orc, lkeys, l_code)
    rc = _col(ms, arena, orc, fk, r_code)
    out = ms.semi_join(lc, rc, F(ms, out_code))
    pos = orc.semi_join(lkeys, fk)
    sf = orc.scalar_from(r_code, 0, rc.meta())
    b, m = orc.wi_write(out_code, 0, pos, int((pos >= sf).sum()))
    assert out.meta() == m
    assert np.array_equal(O.mask_gap(out_code, 0, out.raw_bytes(), m, orc), O.mask_gap(out_code, 0, b, m, orc))


def test_semi_join_hash_path(ms, arena, orc):
    """Build keys spanning more than 2^27 values use the hash set."""
    lkeys = orc.uniform_bits(6, 64, 3000)
    probe = np.concatenate([lkeys[::3], orc.uniform_bits(7, 64, 20_000)])
    probe = probe[orc.uniform_bits(8, 64, len(probe)).argsort(kind="stable")]
    out = ms.semi_join(ms.Column.from_numpy(lkeys, arena), ms.Column.from_numpy(probe, arena))
    assert np.array_equal(out.to_numpy(), orc.semi_join(lkeys, probe))


def test_semi_join_empty_build(ms, arena, orc):
    out = ms.semi_join(ms.Column.from_numpy(np.zeros(0, np.uint64), arena),
                       ms.Column.from_numpy(orc.uniform_bits(1, 8, 1000), arena))
    assert out.get_count_values() == 0


@pytest.mark.parametrize("l_code", [O.UNCOMPR, O.DYNAMIC_VBP, O.DELTA_DVBP])
@pytest.mark.parametrize("out_code", [O.UNCOMPR, O.DYNAMIC_VBP])
def test_intersect_sorted(ms, arena, orc, l_code, out_code):
    n = 60_000
    a = np.flatnonzero(orc.uniform_bits(1, 3, n) < 3).astype(np.uint64)
    b = np.flatnonzero(orc.uniform_bits(2, 3, n) < 5).astype(np.uint64)
    lc = _col(ms, arena, orc, a, l_code)
    rc = ms.Column.from_numpy(b, arena)
    out = ms.intersect_sorted(lc, rc, F(ms, out_code))
    exp = orc.intersect_sorted(a, b)
    sf = orc.scalar_from(l_code, 0, lc.meta())
    ob, om = orc.wi_write(out_code, 0, exp, int((np.searchsorted(a, exp) >= sf).sum()))
    assert out.meta() == om
    assert np.array_equal(out.to_numpy(), exp)


@pytest.mark.parametrize("in_code", [O.UNCOMPR, O.DYNAMIC_VBP, O.FOR_DVBP])
@pytest.mark.parametrize("n", [0, 7, 1000, 100_003])
def test_group_unary(ms, arena, orc, in_code, n):
    keys = orc.from_table(9, orc.zipf_table(1.1, 1000), n)
    c = _col(ms, arena, orc, keys, in_code)
    gr, ext = ms.group(c)
    egr, eext = orc.group(keys)
    assert np.array_equal(gr.to_numpy(), egr)
    assert np.array_equal(ext.to_numpy(), eext)


def test_group_many_keys(ms, arena, orc):
    """More distinct keys than the first table holds: the table grows."""
    keys = orc.uniform_bits(10, 40, 300_000)
    gr, ext = ms.group(ms.Column.from_numpy(keys, arena))
    egr, eext = orc.group(keys)
    assert np.array_equal(gr.to_numpy(), egr)
    assert np.array_equal(ext.to_numpy(), eext)


def test_group_binary(ms, arena, orc):
    n = 50_000
    g1 = orc.uniform_bits(11, 3, n)
    d = orc.uniform_bits(12, 4, n)
    gr, ext = ms.group(ms.Column.from_numpy(d, arena), gr_in=ms.Column.from_numpy(g1, arena))
    egr, eext = orc.group(d, gr_in=g1)
    assert np.array_equal(gr.to_numpy(), egr)
    assert np.array_equal(ext.to_numpy(), eext)


@pytest.mark.parametrize("gr_code,data_code", [(O.UNCOMPR, O.UNCOMPR), (O.DYNAMIC_VBP, O.DYNAMIC_VBP),
                                               (O.UNCOMPR, O.FOR_DVBP)])
@pytest.mark.parametrize("ngroups", [1, 37, 1000, 10_000])
def test_agg_sum_grouped(ms, arena, orc, gr_code, data_code, ngroups):
    n = 80_000 + 5
    gr = orc.from_table(13, orc.zipf_table(1.1, ngroups), n)
    data = orc.uniform_bits(14, 16, n)
    s = ms.agg_sum_grouped(_col(ms, arena, orc, gr, gr_code), _col(ms, arena, orc, data, data_code), ngroups)
    assert np.array_equal(s.to_numpy(), orc.agg_sum_grouped(gr, data, ngroups))


def test_group_then_sum_pipeline(ms, arena, orc):
    """group_vec -> agg_sum(gr, data, |ext|), the query tail of config 3."""
    n = 120_000
    keys = orc.from_table(15, orc.zipf_table(1.1, 1000), n)
    meas = orc.uniform_bits(16, 16, n)
    kc = _col(ms, arena, orc, keys, O.DYNAMIC_VBP)
    gr, ext = ms.group(kc)
    s = ms.agg_sum_grouped(gr, _col(ms, arena, orc, meas, O.DYNAMIC_VBP), ext.get_count_values())
    egr, eext = orc.group(keys)
    assert np.array_equal(s.to_numpy(), orc.agg_sum_grouped(egr, meas, len(eext)))


@pytest.mark.parametrize("l_code", [O.UNCOMPR, O.DYNAMIC_VBP, O.DELTA_DVBP, O.RLE])
@pytest.mark.parametrize("r_code", [O.UNCOMPR, O.DYNAMIC_VBP, O.FOR_DVBP])
@pytest.mark.parametrize("outs", [(O.UNCOMPR, O.UNCOMPR), (O.DYNAMIC_VBP, O.DELTA_DVBP)])
def test_natural_join(ms, arena, orc, l_code, r_code, outs):
    """Build keys with duplicates (the first position is kept), probe rows
    that miss, odd lengths; outputs in their formats."""
    lk = orc.uniform_bits(21, 12, 9_000 + 3)
    if l_code == O.RLE:
        lk = orc.runs(21, 3, 12, 9_000 + 3)
    rk = orc.uniform_bits(22, 13, 50_000 + 11)
    lc = ms.morph(ms.Column.from_numpy(lk, arena), F(ms, l_code)) if l_code != O.UNCOMPR else \
        ms.Column.from_numpy(lk, arena)
    rc = _col(ms, arena, orc, rk, r_code)
    ol, orr = ms.natural_join(lc, rc, F(ms, outs[0]), F(ms, outs[1]))
    el, er = orc.natural_join(lk, rk)
    sf = orc.scalar_from(r_code, 0, rc.meta())
    nscal = int((er >= sf).sum())
    for col, vals, code in ((ol, el, outs[0]), (orr, er, outs[1])):
        b, m = orc.wi_write(code, 0, vals, nscal)
        assert col.meta() == m
        assert np.array_equal(col.to_numpy(), vals)


def test_natural_join_hash_path_and_edges(ms, arena, orc):
    """Keys spanning more than 2^24 values use the hash table, including the
    key 2^64-1; an empty build side or probe side gives empty outputs."""
    lk = np.concatenate([orc.uniform_bits(31, 64, 4000), np.array([2 ** 64 - 1, 7, 7], np.uint64)])
    rk = np.concatenate([lk[::5], orc.uniform_bits(32, 64, 20_000), np.array([2 ** 64 - 1, 7], np.uint64)])
    rk = rk[orc.uniform_bits(33, 64, len(rk)).argsort(kind="stable")]
    ol, orr = ms.natural_join(ms.Column.from_numpy(lk, arena), ms.Column.from_numpy(rk, arena))
    el, er = orc.natural_join(lk, rk)
    assert np.array_equal(ol.to_numpy(), el) and np.array_equal(orr.to_numpy(), er)
    empty = ms.Column.from_numpy(np.zeros(0, np.uint64), arena)
    for a, b in ((empty, ms.Column.from_numpy(rk, arena)), (ms.Column.from_numpy(lk, arena), empty)):
        ol, orr = ms.natural_join(a, b)
        assert ol.get_count_values() == 0 and orr.get_count_values() == 0

