"""GPU parity of the fused compressed query (select -> semi_join ->
intersect -> project -> group -> grouped agg_sum in one pass) against the
oracle's operator-at-a-time pipeline, and against the GPU operators run one
at a time with compressed intermediates."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def F(ms, code, bw=0):
    return {O.UNCOMPR: ms.uncompr_f, O.DYNAMIC_VBP: ms.dynamic_vbp_f, O.DELTA_DVBP: ms.delta_f,
            O.FOR_DVBP: ms.for_f}.get(code) or ms.static_vbp_f(bw)


def _col(ms, arena, orc, v, code, bw=0):
    if code == O.UNCOMPR:
        return ms.Column.from_numpy(v, arena)
    b, m = orc.compress(code, bw, v)
    return ms.Column.from_bytes(F(ms, code, bw), b, m, arena)


def _data(orc, n, seed, key_bits=14, keep=1):
    """The fact/dimension shape of the star query, scaled: fk uniform over
    2^key_bits, filter uniform over 2^12, group key Zipf(1.1) over 1000,
    measure uniform over 2^16; dimension keys 0..2^key_bits-1 kept with
    probability keep/8 (sorted, unique)."""
    filt = orc.uniform_bits(seed, 12, n)
    fk = orc.uniform_bits(seed + 1, key_bits, n)
    gkey = orc.from_table(seed + 2, orc.zipf_table(1.1, 1000), n)
    meas = orc.uniform_bits(seed + 3, 16, n)
    dim = np.arange(1 << key_bits, dtype=np.uint64)
    lk = dim[orc.uniform_bits(seed + 4, 3, len(dim)) < keep]
    return filt, fk, gkey, meas, lk


def _expect(orc, cmp, c, filt, fk, gkey, meas, lk, filt_sf):
    p1 = orc.select(cmp, c, filt, filt_sf)
    p2 = orc.semi_join(lk, fk)
    p = orc.intersect_sorted(p1, p2)
    g = gkey[p.astype(np.int64)]
    m = meas[p.astype(np.int64)]
    gr, ext = orc.group(g)
    sums = orc.agg_sum_grouped(gr, m, len(ext))
    return g[ext.astype(np.int64)], ext, sums, len(p)


FORMATS = [
    (O.DYNAMIC_VBP, O.DYNAMIC_VBP, O.DYNAMIC_VBP, O.DYNAMIC_VBP, O.DELTA_DVBP),
    (O.STATIC_VBP, O.UNCOMPR, O.FOR_DVBP, O.DYNAMIC_VBP, O.UNCOMPR),
    (O.FOR_DVBP, O.FOR_DVBP, O.UNCOMPR, O.DELTA_DVBP, O.DYNAMIC_VBP),
    (O.UNCOMPR, O.DELTA_DVBP, O.DYNAMIC_VBP, O.FOR_DVBP, O.FOR_DVBP),
    (O.DYNAMIC_VBP, O.FOR_DVBP, O.FOR_DVBP, O.FOR_DVBP, O.DELTA_DVBP),
    (O.UNCOMPR, O.UNCOMPR, O.UNCOMPR, O.UNCOMPR, O.UNCOMPR),
]


@pytest.mark.parametrize("fmts", FORMATS)
@pytest.mark.parametrize("n", [0, 5, 512, 1000, 4096 + 13, 200_003])
def test_query3_matches_oracle(ms, arena, orc, fmts, n):
    ff, kf, gf, mf, lf = fmts
    filt, fk, gkey, meas, lk = _data(orc, n, seed=31 + n)
    cols = [_col(ms, arena, orc, v, code, 12 if code == O.STATIC_VBP else 0)
            for v, code in ((filt, ff), (fk, kf), (gkey, gf), (meas, mf), (lk, lf))]
    keys, ext, sums, npos = ms.query3(cols[0], O.CMP_LT, 2048, cols[1], cols[4], cols[2], cols[3])
    sf = orc.scalar_from(ff, 12 if ff == O.STATIC_VBP else 0, cols[0].meta())
    ek, ee, es, enp = _expect(orc, O.CMP_LT, 2048, filt, fk, gkey, meas, lk, sf)
    assert npos == enp
    assert np.array_equal(keys, ek)
    assert np.array_equal(ext, ee)
    assert np.array_equal(sums, es)


@pytest.mark.parametrize("cmp,c", [(O.CMP_EQ, 7), (O.CMP_GE, 4000), (O.CMP_LE, 0), (O.CMP_GT, 1 << 12)])
def test_query3_predicates(ms, arena, orc, cmp, c):
    n = 70_001
    filt, fk, gkey, meas, lk = _data(orc, n, seed=5, keep=4)
    cols = [_col(ms, arena, orc, v, O.DYNAMIC_VBP) for v in (filt, fk, gkey, meas, lk)]
    keys, ext, sums, npos = ms.query3(cols[0], cmp, c, cols[1], cols[4], cols[2], cols[3])
    sf = orc.scalar_from(O.DYNAMIC_VBP, 0, cols[0].meta())
    ek, ee, es, enp = _expect(orc, cmp, c, filt, fk, gkey, meas, lk, sf)
    assert (npos, len(keys)) == (enp, len(ek))
    assert np.array_equal(keys, ek) and np.array_equal(ext, ee) and np.array_equal(sums, es)


def test_query3_many_groups_and_wide_values(ms, arena, orc):
    """Group keys with up to 60 000 distinct values (spills the per-CTA
    tables to the global one) and 40-bit measures (64-bit sums)."""
    n = 300_017
    filt = orc.uniform_bits(1, 12, n)
    fk = orc.uniform_bits(2, 10, n)
    gkey = orc.uniform_bits(3, 64, n) % np.uint64(60_000) + np.uint64(1 << 50)
    meas = orc.uniform_bits(4, 40, n)
    lk = np.arange(0, 1 << 10, 2, dtype=np.uint64) + np.uint64(0)
    cols = [_col(ms, arena, orc, v, O.DYNAMIC_VBP) for v in (filt, fk, gkey, meas)]
    lcol = _col(ms, arena, orc, lk, O.DELTA_DVBP)
    keys, ext, sums, npos = ms.query3(cols[0], O.CMP_LT, 3000, cols[1], lcol, cols[2], cols[3])
    sf = orc.scalar_from(O.DYNAMIC_VBP, 0, cols[0].meta())
    ek, ee, es, enp = _expect(orc, O.CMP_LT, 3000, filt, fk, gkey, meas, lk, sf)
    assert len(ek) > 40_000
    assert npos == enp
    assert np.array_equal(keys, ek) and np.array_equal(ext, ee) and np.array_equal(sums, es)


def test_query3_empty_build_side(ms, arena, orc):
    n = 10_000
    filt, fk, gkey, meas, _ = _data(orc, n, seed=8)
    cols = [_col(ms, arena, orc, v, O.DYNAMIC_VBP) for v in (filt, fk, gkey, meas)]
    empty = ms.Column.from_numpy(np.zeros(0, np.uint64), arena)
    keys, ext, sums, npos = ms.query3(cols[0], O.CMP_LT, 2048, cols[1], empty, cols[2], cols[3])
    assert (len(keys), npos) == (0, 0)


def test_query3_rejects_bad_input(ms, arena, orc):
    v = orc.uniform_bits(1, 12, 4096)
    a = ms.Column.from_numpy(v, arena)
    b = ms.Column.from_numpy(v[:4000], arena)
    with pytest.raises(ms.MorphStoreError):
        ms.query3(a, O.CMP_LT, 5, b, a, a, a)
    wide = ms.Column.from_numpy(np.array([0, 1 << 40], np.uint64), arena)
    with pytest.raises(ms.MorphStoreError):
        ms.query3(a, O.CMP_LT, 5, a, wide, a, a)
    r = ms.morph(a, ms.rle_f)
    with pytest.raises(ms.MorphStoreError):
        ms.query3(r, O.CMP_LT, 5, a, a, a, a)


@pytest.mark.parametrize("cfg", [dict(staged=0), dict(staged=2, warps=16, stages=3, stage_bytes=57344),
                                 dict(warps=8, stages=2, stage_bytes=16384),
                                 dict(warps=16, stages=4, stage_bytes=40960),
                                 dict(warps=24, stages=3, stage_bytes=57344),
                                 dict(staged=3, warps=16, stages=3, stage_bytes=57344),
                                 dict(staged=3, warps=8, stages=2, stage_bytes=32768),
                                 dict(staged=3, warps=24, stages=4, stage_bytes=40960)])
def test_query3_launch_configs(ms, arena, orc, cfg):
    """Every staged-kernel configuration (and the direct kernel alone) gives
    the oracle's groups; ragged length so the tail kernel runs too."""
    n = 400_000 + 77
    filt, fk, gkey, meas, lk = _data(orc, n, seed=12, keep=3)
    codes = (O.DYNAMIC_VBP, O.FOR_DVBP, O.DYNAMIC_VBP, O.FOR_DVBP)
    cols = [_col(ms, arena, orc, v, code) for v, code in zip((filt, fk, gkey, meas), codes)]
    lcol = _col(ms, arena, orc, lk, O.DELTA_DVBP)
    old = ms.get_query_tuning()
    try:
        ms.set_query_tuning(**cfg)
        keys, ext, sums, npos = ms.query3(cols[0], O.CMP_LT, 1000, cols[1], lcol, cols[2], cols[3])
    finally:
        ms.set_query_tuning(**old)
    sf = orc.scalar_from(O.DYNAMIC_VBP, 0, cols[0].meta())
    ek, ee, es, enp = _expect(orc, O.CMP_LT, 1000, filt, fk, gkey, meas, lk, sf)
    assert (npos, len(keys)) == (enp, len(ek))
    assert np.array_equal(keys, ek) and np.array_equal(ext, ee) and np.array_equal(sums, es)


@pytest.mark.parametrize("staged", [1, 2, 3])
def test_query3_wide_build_side(ms, arena, orc, staged):
    """A build side over 2^20 keys: its 128 KB bitmap does not fit one CTA
    beside the ring, so staged=1 and 2 read it from global memory and
    staged=3 splits it over a 2-CTA cluster (read through distributed shared
    memory).  All equal the oracle, and the pass time is recorded."""
    n = 1_000_003
    filt, fk, gkey, meas, lk = _data(orc, n, seed=31, key_bits=20, keep=1)
    codes = (O.DYNAMIC_VBP, O.DYNAMIC_VBP, O.FOR_DVBP, O.DYNAMIC_VBP)
    cols = [_col(ms, arena, orc, v, code) for v, code in zip((filt, fk, gkey, meas), codes)]
    lcol = _col(ms, arena, orc, lk, O.DELTA_DVBP)
    old = ms.get_query_tuning()
    try:
        ms.set_query_tuning(staged=staged, warps=16, stages=3, stage_bytes=57344)
        keys, ext, sums, npos = ms.query3(cols[0], O.CMP_LT, 400, cols[1], lcol, cols[2], cols[3])
    finally:
        ms.set_query_tuning(**old)
    assert ms.query3_last_pass_ms() > 0
    sf = orc.scalar_from(O.DYNAMIC_VBP, 0, cols[0].meta())
    ek, ee, es, enp = _expect(orc, O.CMP_LT, 400, filt, fk, gkey, meas, lk, sf)
    assert (npos, len(keys)) == (enp, len(ek))
    assert np.array_equal(keys, ek) and np.array_equal(ext, ee) and np.array_equal(sums, es)


def test_query_tuning_rejects_bad_config(ms):
    with pytest.raises(ms.MorphStoreError):
        ms.set_query_tuning(warps=12)
    with pytest.raises(ms.MorphStoreError):
        ms.set_query_tuning(stages=8, stage_bytes=65536)


def test_query3_equals_gpu_operator_pipeline(ms, arena, orc):
    """The GPU operators one at a time, every intermediate compressed
    (positions as delta+dvbp, projected columns as dynamic_vbp), give the
    fused result."""
    n = 250_000
    filt, fk, gkey, meas, lk = _data(orc, n, seed=77)
    cols = [_col(ms, arena, orc, v, O.DYNAMIC_VBP) for v in (filt, fk, gkey, meas)]
    lcol = _col(ms, arena, orc, lk, O.DELTA_DVBP)
    p1 = ms.select(O.CMP_LT, cols[0], 2048, ms.delta_f)
    p2 = ms.semi_join(lcol, cols[1], ms.delta_f)
    p = ms.intersect_sorted(p1, ms.morph(p2, ms.uncompr_f), ms.delta_f)
    g = ms.project(cols[2], p, ms.dynamic_vbp_f)
    m = ms.project(cols[3], p, ms.dynamic_vbp_f)
    gr, ext = ms.group(g)
    s = ms.agg_sum_grouped(gr, m, ext.get_count_values())
    gk = g.to_numpy()[ext.to_numpy().astype(np.int64)]
    keys, e2, sums, npos = ms.query3(cols[0], O.CMP_LT, 2048, cols[1], lcol, cols[2], cols[3])
    assert npos == p.get_count_values()
    assert np.array_equal(keys, gk)
    assert np.array_equal(e2, ext.to_numpy())
    assert np.array_equal(sums, s.to_numpy())
