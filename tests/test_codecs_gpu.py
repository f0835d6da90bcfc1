"""GPU codec parity: bytes written by the CUDA encoders and values returned
by the CUDA decoders, against the oracle on the same seeded inputs."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

LENGTHS = [0, 1, 17, 512, 1000, 1024, 2047, 4096 + 17, 33000, 70001]


def _values(orc, fmt, bw, n, seed):
    if fmt == O.STATIC_VBP:
        return orc.uniform_bits(seed, bw, n)
    if fmt == O.DELTA_DVBP:
        return orc.sorted_gaps(seed, orc.geom_table(0.25), n)
    if fmt == O.RLE:
        return orc.runs(seed, 5, 20, n)
    return orc.uniform_bits(seed, 20, n)


def _masked(fmt, bw, data, meta, orc):
    return O.mask_gap(fmt, bw, data, meta, orc)


def _fmt(ms, fmt, bw):
    return {O.UNCOMPR: ms.uncompr_f, O.STATIC_VBP: ms.static_vbp_f(bw) if bw else None,
            O.DYNAMIC_VBP: ms.dynamic_vbp_f, O.DELTA_DVBP: ms.delta_f, O.FOR_DVBP: ms.for_f,
            O.RLE: ms.rle_f}[fmt]


@pytest.mark.parametrize("fmt", [O.DYNAMIC_VBP, O.DELTA_DVBP, O.FOR_DVBP, O.RLE])
@pytest.mark.parametrize("n", LENGTHS)
def test_compress_bytes_match_oracle(ms, arena, orc, fmt, n):
    v = _values(orc, fmt, 0, n, seed=100 + n)
    col = ms.Column.from_numpy(v, arena)
    c = ms.morph(col, _fmt(ms, fmt, 0))
    b, m = orc.compress(fmt, 0, v)
    assert c.meta() == m
    got = c.raw_bytes()
    assert np.array_equal(_masked(fmt, 0, got, m, orc), _masked(fmt, 0, b, m, orc))
    assert np.array_equal(c.to_numpy(), v)


@pytest.mark.parametrize("bw", list(range(1, 65)))
def test_static_vbp_every_bit_width(ms, arena, orc, bw):
    n = 3 * 512 + 17
    v = orc.uniform_bits(7 * bw, bw, n)
    c = ms.morph(ms.Column.from_numpy(v, arena), ms.static_vbp_f(bw))
    b, m = orc.compress(O.STATIC_VBP, bw, v)
    assert c.meta() == m
    assert np.array_equal(_masked(O.STATIC_VBP, bw, c.raw_bytes(), m, orc), _masked(O.STATIC_VBP, bw, b, m, orc))
    assert np.array_equal(c.to_numpy(), v)


@pytest.mark.parametrize("bits", [1, 8, 31, 32, 33, 63, 64])
def test_dvbp_and_for_wide_values(ms, arena, orc, bits):
    """Every block bit width, including 64-bit values (signed FOR minimum)."""
    n = 8 * 1024 + 300
    v = orc.uniform_bits(bits, bits, n)
    for fmt in (O.DYNAMIC_VBP, O.FOR_DVBP, O.DELTA_DVBP):
        c = ms.morph(ms.Column.from_numpy(v, arena), _fmt(ms, fmt, 0))
        b, m = orc.compress(fmt, 0, v)
        assert c.meta() == m, fmt
        assert np.array_equal(_masked(fmt, 0, c.raw_bytes(), m, orc), _masked(fmt, 0, b, m, orc)), fmt
        assert np.array_equal(c.to_numpy(), v), fmt


@pytest.mark.parametrize("fmt", [O.DYNAMIC_VBP, O.DELTA_DVBP, O.FOR_DVBP])
def test_decode_reference_bytes_with_host_index(ms, arena, orc, fmt):
    """Columns uploaded in the reference layout decode through the host index."""
    v = _values(orc, fmt, 0, 100_000 + 123, seed=5)
    b, m = orc.compress(fmt, 0, v)
    c = ms.Column.from_bytes(_fmt(ms, fmt, 0), b, m, arena)
    assert np.array_equal(c.to_numpy(), v)
    # and through the device-side page walk
    c2 = ms.Column.from_bytes(_fmt(ms, fmt, 0), b, m, arena, build_index=False)
    c2.build_index()
    assert np.array_equal(c2.to_numpy(), v)


def test_mixed_block_widths(ms, arena, orc):
    """Blocks of different widths inside one dynamic_vbp page."""
    n = 64 * 512 * 2 + 999
    v = orc.uniform_bits(11, 64, n)
    shifts = (np.arange(n) // 512) % 64
    v = v >> shifts.astype(np.uint64)
    for fmt in (O.DYNAMIC_VBP, O.FOR_DVBP):
        c = ms.morph(ms.Column.from_numpy(v, arena), _fmt(ms, fmt, 0))
        b, m = orc.compress(fmt, 0, v)
        assert c.meta() == m
        assert np.array_equal(_masked(fmt, 0, c.raw_bytes(), m, orc), _masked(fmt, 0, b, m, orc))
        assert np.array_equal(c.to_numpy(), v)


def test_compressed_to_compressed(ms, arena, orc):
    v = _values(orc, O.DELTA_DVBP, 0, 50_000, seed=9)
    a = ms.morph(ms.Column.from_numpy(v, arena), ms.delta_f)
    bcol = ms.morph(a, ms.for_f)
    b, m = orc.compress(O.FOR_DVBP, 0, v)
    assert bcol.meta() == m
    assert np.array_equal(bcol.to_numpy(), v)


def test_device_generators_match_oracle(ms, arena, orc):
    """The device generators produce the oracle's columns bit for bit."""
    import ctypes as C
    lib = ms.lib()
    n = 300_007
    geo = orc.geom_table(0.25)
    zipf = orc.zipf_table(1.2, 1 << 20)
    d_geo, d_zipf = arena.alloc(geo.nbytes), arena.alloc(zipf.nbytes)
    ms._memcpy_h2d(d_geo, geo)
    ms._memcpy_h2d(d_zipf, zipf)
    out = arena.alloc(8 * n)
    checks = [
        (lambda: lib.ms_gpu_gen_uniform_bits(5, 17, n, out, None), orc.uniform_bits(5, 17, n)),
        (lambda: lib.ms_gpu_gen_from_table(6, d_zipf, len(zipf), n, out, None), orc.from_table(6, zipf, n)),
        (lambda: lib.ms_gpu_gen_sorted_gaps(7, d_geo, len(geo), n, out, arena.h, None), orc.sorted_gaps(7, geo, n)),
        (lambda: lib.ms_gpu_gen_runs(8, 5, 20, n, out, arena.h, None), orc.runs(8, 5, 20, n)),
    ]
    for gen, expect in checks:
        ms._check(gen(), "gen")
        assert np.array_equal(ms._memcpy_d2h(out, 8 * n).view(np.uint64), expect)


@pytest.mark.parametrize("fmt", [O.STATIC_VBP, O.DYNAMIC_VBP, O.DELTA_DVBP, O.FOR_DVBP, O.RLE])
def test_compact_keeps_column(ms, arena, orc, fmt):
    """A compacted column has the same bytes, metadata and values, in
    storage of its used size."""
    v = _values(orc, fmt, 9, 40_000 + 3, seed=4)
    c = ms.morph(ms.Column.from_numpy(v, arena), _fmt(ms, fmt, 9))
    k = c.compact()
    assert k.meta() == c.meta()
    assert k.desc.size_alloc_byte == c.get_size_used_byte() + 64
    assert np.array_equal(k.raw_bytes(), c.raw_bytes())
    assert np.array_equal(k.to_numpy(), v)
    if fmt != O.RLE:
        assert ms.select_project_sum(k, ms.less, 1000, k) == ms.select_project_sum(c, ms.less, 1000, c)


def _rle_cases(orc):
    t = 2048  # the decoder's largest tile of runs
    T = 16384  # the encoder's tile of rows
    yield "every row a run", orc.uniform_bits(5, 40, 5 * t + 3)
    yield "one run over many tiles", np.full(37 * t + 11, 123456789, dtype=np.uint64)
    yield "two runs, boundary mid-tile", np.concatenate([np.full(9 * t + 700, 7, np.uint64),
                                                           np.full(4 * t + 5, 9, np.uint64)])
    yield "long geometric runs", orc.runs(6, 12, 20, 60 * t + 1)
    yield "tile-sized lengths", orc.runs(7, 5, 20, 3 * t)
    yield "one row", np.array([42], dtype=np.uint64)
    yield "runs of 64-bit values", orc.runs(8, 3, 64, 10 * t + 9)
    for k in (t - 1, t, t + 1, 2 * t - 1, 2 * t + 1):
        yield f"runs, n={k}", orc.runs(9 + k, 2, 8, k)
    yield "every row a run, 40 encoder tiles", orc.uniform_bits(10, 30, 40 * T + 5)
    for k in (T - 1, T, T + 1, 3 * T - 1, 3 * T + 1):
        yield f"short runs, n={k}", orc.runs(11 + k, 1, 8, k)
    yield "runs ending on encoder tiles", np.repeat(orc.uniform_bits(12, 20, 24), T)
    yield "long runs, small decoder tiles", orc.runs(13, 7, 20, 300 * T + 77)


N_RLE_CASES = 20


def test_rle_case_count(orc):
    assert len(list(_rle_cases(orc))) == N_RLE_CASES


@pytest.mark.parametrize("case", range(N_RLE_CASES))
def test_rle_codec_edge_cases(ms, arena, orc, case):
    name, v = list(_rle_cases(orc))[case]
    c = ms.morph(ms.Column.from_numpy(v, arena), ms.rle_f)
    b, m = orc.compress(O.RLE, 0, v)
    assert c.meta() == m, name
    assert np.array_equal(c.raw_bytes(), b), name
    assert np.array_equal(c.to_numpy(), v), name


@pytest.mark.parametrize("mean_log2", [0, 5, 9])
def test_rle_decode_zero_length_runs(ms, arena, orc, mean_log2):
    """Pairs with length 0 write nothing (rle.h:238-249): bursts of them at
    the start, inside and at the end of the column, longer than a warp's
    window and across decoder tiles, decode as the oracle decodes them."""
    v = orc.runs(14 + mean_log2, mean_log2, 20, 200_003) if mean_log2 else orc.uniform_bits(14, 20, 200_003)
    b, m = orc.compress(O.RLE, 0, v)
    pairs = b.view(np.uint64).reshape(-1, 2)
    rng = np.random.default_rng(mean_log2)
    at = np.sort(rng.choice(len(pairs), size=min(300, len(pairs)), replace=False))
    burst = np.array([[7, 0]] * 70, dtype=np.uint64)
    parts, last = [burst], 0
    for i, k in enumerate(at):
        parts.append(pairs[last:k])
        parts.append(burst[: 1 + (i % 5) * 10])
        last = k
    parts += [pairs[last:], burst[:3]]
    z = np.ascontiguousarray(np.concatenate(parts).astype(np.uint64)).reshape(-1)
    zm = (m[0], z.nbytes, z.nbytes)
    want = orc.decompress(O.RLE, 0, z.view(np.uint8), zm)
    assert np.array_equal(want, v)
    col = ms.Column.from_bytes(ms.rle_f, z.view(np.uint8), zm, arena)
    assert np.array_equal(ms.morph(col, ms.uncompr_f).to_numpy(), want)


@pytest.mark.parametrize("mean_log2", [0, 5])
@pytest.mark.parametrize("delta", [-1, 1, 1 << 40])
def test_rle_decode_reports_inconsistent_lengths(ms, arena, orc, mean_log2, delta):
    """Run lengths that do not add up to the column's count (one run short,
    one row long, 2^40 rows long) are a corrupt column: the decoder writes no
    row past the column's end and the call reports MS_ERR_CORRUPT.  Runs of
    one row take the one-pass decoder, runs of mean 32 the two-pass one."""
    v = orc.runs(3, mean_log2, 20, 50_000) if mean_log2 else orc.uniform_bits(3, 20, 50_000)
    b, m = orc.compress(O.RLE, 0, v)
    pairs = b.view(np.uint64).copy()
    pairs[2 * 7 + 1] = np.uint64(int(pairs[2 * 7 + 1]) + delta)  # one run short or long
    col = ms.Column.from_bytes(ms.rle_f, pairs.view(np.uint8), m, arena)
    with pytest.raises(ms.MorphStoreError) as e:
        ms.morph(col, ms.uncompr_f)
    assert e.value.status == 5
