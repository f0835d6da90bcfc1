"""GPU parity of batched persistent execution: many columns of mixed formats
and lengths, decompress -> select(value < c_i) -> sum per column in one
launch, against the oracle (uncompressed select + sum) and against one
operator call per column."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

KINDS = ["static", "dvbp", "delta", "for", "rle"]


def _column(orc, kind, n, seed):
    if kind == "static":
        bw = 4 + seed % 29
        return orc.uniform_bits(seed, bw, n), bw
    if kind == "dvbp":
        return orc.uniform_bits(seed, 4 + seed % 29, n), 0
    if kind == "delta":
        return orc.sorted_gaps(seed, orc.geom_table(0.25), n), 0
    if kind == "for":
        return orc.uniform_bits(seed, 16, n) + np.uint64(1 << 40), 0
    return orc.runs(seed, 5, 20, n), 0


def _fmt(ms, kind, bw):
    return {"static": ms.static_vbp_f(bw) if bw else None, "dvbp": ms.dynamic_vbp_f, "delta": ms.delta_f,
            "for": ms.for_f, "rle": ms.rle_f}[kind]


def _expect(orc, v, c, cmp=O.CMP_LT):
    pos = orc.select(cmp, c, v, len(v) - len(v) % 8)
    return len(pos), int(v[pos.astype(np.int64)].sum(dtype=np.uint64))


def _median(v):
    return int(np.sort(v)[len(v) // 2]) if len(v) else 0


def _make(ms, arena, orc, lengths, seed0=0, ref_bytes_every=0):
    cols, vals, consts = [], [], []
    for i, n in enumerate(lengths):
        kind = KINDS[(i + seed0) % len(KINDS)]
        v, bw = _column(orc, kind, n, seed0 * 1000 + i + 1)
        f = _fmt(ms, kind, bw)
        if ref_bytes_every and i % ref_bytes_every == 0 and kind != "rle":
            code = {"static": O.STATIC_VBP, "dvbp": O.DYNAMIC_VBP, "delta": O.DELTA_DVBP, "for": O.FOR_DVBP}[kind]
            b, m = orc.compress(code, bw, v)
            col = ms.Column.from_bytes(f, b, m, arena)
        else:
            col = ms.morph(ms.Column.from_numpy(v, arena), f)
        cols.append(col)
        vals.append(v)
        consts.append(_median(v))
    return cols, vals, consts


def _lengths(orc, k, lo, hi, seed):
    u = orc.uniform_bits(seed, 32, k).astype(np.float64) / 2.0 ** 32
    return [int(2 ** (lo + (hi - lo) * x)) + int(x * 1000) % 7 for x in u]


def test_batch_matches_oracle(ms, arena, orc):
    lengths = _lengths(orc, 60, 10, 16, 3) + [0, 1, 7, 8, 511, 512, 513, 1023, 1024, 1025, 2048 + 5]
    cols, vals, consts = _make(ms, arena, orc, lengths, seed0=1, ref_bytes_every=4)
    b = ms.Batch(cols, consts)
    cnt, s = b.run()
    for i, (v, c) in enumerate(zip(vals, consts)):
        assert (int(cnt[i]), int(s[i])) == _expect(orc, v, c), (i, len(v), cols[i].format)
    # again, and through the captured graph (twice)
    for graph in (False, True, True):
        c2, s2 = b.run(graph=graph)
        assert np.array_equal(c2, cnt) and np.array_equal(s2, s)
    b.close()


@pytest.mark.parametrize("cfg", [dict(warps=4, stages=2, stage_bytes=4096), dict(warps=8, stages=3, stage_bytes=8192),
                                 dict(warps=12, stages=2, stage_bytes=8192),
                                 dict(warps=16, stages=3, stage_bytes=4096),
                                 dict(warps=4, stages=4, stage_bytes=4096, ctas_per_sm=2)])
def test_batch_launch_configs(ms, arena, orc, cfg):
    lengths = _lengths(orc, 30, 10, 17, 9)
    cols, vals, consts = _make(ms, arena, orc, lengths, seed0=2)
    b = ms.Batch(cols, consts)
    b.set_config(**cfg)
    assert b.get_config() == dict(dict(ctas_per_sm=1), **cfg)
    for graph in (False, True):
        cnt, s = b.run(graph=graph)
        for i, (v, c) in enumerate(zip(vals, consts)):
            assert (int(cnt[i]), int(s[i])) == _expect(orc, v, c), (i, cfg)
    b.close()


@pytest.mark.parametrize("kinds", [{"rle": dict(warps=16, stages=2, stage_bytes=4096)},
                                   {"delta": dict(warps=16, stages=2, stage_bytes=4096),
                                    "rle": dict(warps=16, stages=2, stage_bytes=4096)},
                                   {"vbp": dict(warps=8, stages=3, stage_bytes=8192),
                                    "for": dict(warps=12, stages=2, stage_bytes=8192),
                                    "delta": dict(warps=4, stages=4, stage_bytes=4096, ctas_per_sm=2),
                                    "rest": dict(warps=16, stages=2, stage_bytes=4096),
                                    "rle": dict(warps=8, stages=2, stage_bytes=4096)}])
def test_batch_per_kind_configs(ms, arena, orc, kinds):
    """Kinds with their own launch configuration: one launch per run of
    equally configured kinds, on forked streams; direct and graph replay
    give the oracle's counts and sums, and a kind returned to the plan's
    configuration leaves a single launch."""
    lengths = _lengths(orc, 40, 10, 17, 11)
    cols, vals, consts = _make(ms, arena, orc, lengths, seed0=6)
    b = ms.Batch(cols, consts)
    b.set_config(warps=12, stages=2, stage_bytes=8192)
    for k, cfg in kinds.items():
        b.set_kind_config(k, **cfg)
    got = b.kind_configs()
    for k, cfg in kinds.items():
        if k in got:
            assert {x: got[k][x] for x in ("warps", "stages", "stage_bytes", "ctas_per_sm")} == \
                dict(dict(ctas_per_sm=1), **cfg)
    for graph in (False, True, True):
        cnt, s = b.run(graph=graph)
        for i, (v, c) in enumerate(zip(vals, consts)):
            assert (int(cnt[i]), int(s[i])) == _expect(orc, v, c), (i, kinds)
    for k in kinds:
        b.set_kind_config(k, None)
    cnt2, s2 = b.run(graph=True)
    assert np.array_equal(cnt2, cnt) and np.array_equal(s2, s)
    b.close()


@pytest.mark.parametrize("cmp", [O.CMP_EQ, O.CMP_LE, O.CMP_GT, O.CMP_GE])
def test_batch_other_comparisons(ms, arena, orc, cmp):
    lengths = _lengths(orc, 15, 10, 14, 30 + cmp)
    cols, vals, consts = _make(ms, arena, orc, lengths, seed0=4)
    cnt, s = ms.Batch(cols, consts, cmp).run()
    for i, (v, c) in enumerate(zip(vals, consts)):
        assert (int(cnt[i]), int(s[i])) == _expect(orc, v, c, cmp), (i, cmp)


def test_batch_wide_values(ms, arena, orc):
    """64-bit static/dvbp blocks (signed compare), values >= 2^63, and a
    constant above every value."""
    n = 5000
    v64 = orc.uniform_bits(5, 64, n)
    v40 = orc.uniform_bits(6, 40, n)
    cols = [ms.morph(ms.Column.from_numpy(v64, arena), ms.static_vbp_f(64)),
            ms.morph(ms.Column.from_numpy(v64, arena), ms.dynamic_vbp_f),
            ms.morph(ms.Column.from_numpy(v40, arena), ms.for_f),
            ms.morph(ms.Column.from_numpy(v40, arena), ms.dynamic_vbp_f)]
    vals = [v64, v64, v40, v40]
    consts = [1 << 62, 0, 1 << 41, 0]
    # values around 2^63: for_f and delta_f blocks whose range crosses the
    # signed boundary (64-bit comparison) next to blocks that do not
    vf = orc.uniform_bits(7, 16, n) + np.uint64((1 << 63) - 30000)
    vd = orc.sorted_gaps(8, orc.geom_table(0.25), n) + np.uint64((1 << 63) - 9000)
    cols += [ms.morph(ms.Column.from_numpy(vf, arena), ms.for_f), ms.morph(ms.Column.from_numpy(vd, arena), ms.delta_f)]
    vals += [vf, vd]
    consts += [_median(vf), _median(vd)]
    for cmp in (O.CMP_LT, O.CMP_LE, O.CMP_GT, O.CMP_GE, O.CMP_EQ):
        cs = [int(v[len(v) // 3]) if cmp == O.CMP_EQ else c for v, c in zip(vals, consts)]
        cnt, s = ms.Batch(cols, cs, cmp).run()
        for i, (v, c) in enumerate(zip(vals, cs)):
            assert (int(cnt[i]), int(s[i])) == _expect(orc, v, c, cmp), (i, cmp)


def test_batch_equals_one_call_per_column(ms, arena, orc):
    lengths = _lengths(orc, 25, 10, 15, 21)
    cols, vals, consts = _make(ms, arena, orc, lengths, seed0=3)
    cnt, s = ms.Batch(cols, consts).run()
    for i, col in enumerate(cols):
        x = ms.morph(col, ms.uncompr_f) if col.format.code == ms.RLE else col
        got = ms.select_project_sum(x, ms.less, consts[i], x)
        assert (int(cnt[i]), int(s[i])) == (got[1], got[0]), i


def test_batch_empty_and_bad_config(ms, arena, orc):
    b = ms.Batch([], [], arena=arena)
    cnt, s = b.run()
    assert len(cnt) == 0
    v = orc.uniform_bits(1, 8, 3000)
    b = ms.Batch([ms.morph(ms.Column.from_numpy(v, arena), ms.dynamic_vbp_f)], [100])
    with pytest.raises(ms.MorphStoreError):
        b.set_config(warps=16, stages=8, stage_bytes=65536)
    with pytest.raises(ms.MorphStoreError):
        b.set_config(warps=5)
    cnt, s = b.run()  # the old configuration still works
    assert (int(cnt[0]), int(s[0])) == _expect(orc, v, 100)
