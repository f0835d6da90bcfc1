"""Parity at the sizes the benchmark configurations name.

* Select-project-sum at its exact CPU-runnable shape: 2^24 rows, x uniform
  over 10 bits stored as static_vbp<10>, y uniform over 20 bits stored as
  dynamic_vbp<512,64,8>; select(x < 512) -> project(y) -> agg_sum.  The
  compressed bytes, positions, projected values and the sum are compared with
  the oracle and, where the reference library was built, with the reference's
  own codecs and operators on the same rows.
* The codec sweep at 2^28 values per case: the compressed bytes the GPU
  writes for every format x distribution (and static_vbp at several widths)
  are compared, as digests of the bytes that carry meaning, with the
  reference's own codecs run on the host cores over the same seeded values;
  the GPU's decoded column is compared with its input on the device.
"""
import multiprocessing as mp
import os

import numpy as np
import pytest

import oracle as O
from oracle import workloads as W

pytestmark = pytest.mark.gpu

N1 = 1 << 24
N2 = 1 << 28


def test_select_project_sum_at_full_shape(ms, orc):
    arena = ms.Arena(4 << 30)
    try:
        x = orc.uniform_bits(W.SEED_X, 10, N1)
        y = orc.uniform_bits(W.SEED_Y, 20, N1)
        xc = ms.morph(ms.Column.from_numpy(x, arena), ms.static_vbp_f(10))
        yc = ms.morph(ms.Column.from_numpy(y, arena), ms.dynamic_vbp_f)
        assert xc.get_size_used_byte() == 20_971_520 and yc.get_size_used_byte() == 41_975_808
        # the operator chain: select -> project -> agg_sum
        pos = ms.select(ms.less, xc, 512)
        vals = ms.project(yc, pos)
        s = ms.agg_sum(vals)
        # the fused form
        fs, fk, fpos, fvals = ms.select_project_sum(xc, ms.less, 512, yc, want_positions=True)
        want_pos = orc.select(O.CMP_LT, 512, x, orc.scalar_from(O.STATIC_VBP, 10, xc.meta()))
        want_vals = y[want_pos.astype(np.int64)]
        want_sum = int(want_vals.sum(dtype=np.uint64))
        got_pos, got_vals = pos.to_numpy(), vals.to_numpy()
        assert np.array_equal(got_pos, want_pos) and np.array_equal(fpos, want_pos)
        assert np.array_equal(got_vals, want_vals) and np.array_equal(fvals, want_vals)
        assert s == fs == want_sum and fk == len(want_pos)
        path = O.reference_path()
        if path is None:
            pytest.skip("reference library not built here; checked against the oracle only")
        ref = O.Reference(path)
        if ref.isa != 512:
            pytest.skip("host without AVX-512: the reference's AVX2 layouts differ; checked against the oracle")
        bx, mx = ref.compress(O.STATIC_VBP, 10, x)
        by, my = ref.compress(O.DYNAMIC_VBP, 0, y)
        assert xc.meta() == mx and yc.meta() == my
        assert np.array_equal(O.mask_gap(O.STATIC_VBP, 10, xc.raw_bytes(), mx, orc), O.mask_gap(O.STATIC_VBP, 10, bx,
                                                                                                  mx, orc))
        assert np.array_equal(O.mask_gap(O.DYNAMIC_VBP, 0, yc.raw_bytes(), my, orc), O.mask_gap(O.DYNAMIC_VBP, 0, by,
                                                                                                  my, orc))
        rp, rpm = ref.select(O.CMP_LT, 512, O.STATIC_VBP, 10, bx, mx, O.UNCOMPR)
        assert np.array_equal(rp.view(np.uint64)[: rpm[0]], got_pos)
        yd = ref.decompress(O.DYNAMIC_VBP, 0, by, my)  # the reference cannot project from dynamic_vbp
        rv, rvm = ref.project(O.UNCOMPR, 0, yd.view(np.uint8), (N1, 8 * N1, 0), O.UNCOMPR, 0, rp, rpm, O.UNCOMPR)
        assert np.array_equal(rv.view(np.uint64)[: rvm[0]], got_vals)
        assert ref.agg_sum(O.UNCOMPR, 0, rv, rvm) == s
    finally:
        arena.close()


# ---------------------------------------------------------------------------
# codec sweep at 2^28
# ---------------------------------------------------------------------------
CASES = [(d, f, 0, 20) for d in W.DISTRIBUTIONS for f in (O.DYNAMIC_VBP, O.DELTA_DVBP, O.FOR_DVBP, O.RLE)]
CASES += [("uniform", O.DYNAMIC_VBP, 0, 64), ("uniform", O.FOR_DVBP, 0, 64)]
CASES += [("uniform", O.STATIC_VBP, b, b) for b in (1, 10, 20, 33, 64)]


def _seed(case):
    return 0xC0DEC000 + CASES.index(case)


def _case_id(case):
    d, f, bw, bits = case
    return f"{O.FORMAT_NAMES[f]}{'<%d>' % bw if bw else ''}-{d}{bits if d == 'uniform' else ''}"


@pytest.fixture(scope="module")
def reference_digests():
    """Every case's reference digest, computed by spawned host processes
    while the GPU side runs (memory-bounded: a case holds up to ~6 GB)."""
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except ImportError:
        avail = 64 << 30
    procs = max(1, min(len(CASES), os.cpu_count() or 1, int(avail // (8 << 30))))
    pool = mp.get_context("spawn").Pool(procs)
    jobs = {c: pool.apply_async(W.reference_codec_digest, ((c[0], c[1], c[2], N2, _seed(c), c[3]),)) for c in CASES}
    yield jobs
    pool.terminate()
    pool.join()


def _device_values(ms, lib, arena, dist, seed, bits, tables):
    d = arena.alloc(8 * N2)
    if dist == "uniform":
        ms._check(lib.ms_gpu_gen_uniform_bits(seed, bits, N2, d, None), "gen")
    elif dist == "zipf":
        ms._check(lib.ms_gpu_gen_from_table(seed, tables["zipf"][0], tables["zipf"][1], N2, d, None), "gen")
    elif dist == "sorted":
        ms._check(lib.ms_gpu_gen_sorted_gaps(seed, tables["geo"][0], tables["geo"][1], N2, d, arena.h, None), "gen")
    else:
        ms._check(lib.ms_gpu_gen_runs(seed, 5, 20, N2, d, arena.h, None), "gen")
    return ms.Column(ms.MsCol(format=ms.UNCOMPR, count_values=N2, size_used_byte=8 * N2, size_alloc_byte=8 * N2,
                              data=d), arena)


@pytest.mark.parametrize("case", CASES, ids=[_case_id(c) for c in CASES])
def test_codec_bytes_match_reference_at_2p28(ms, orc, reference_digests, case):
    import torch
    dist, fmt, bw, bits = case
    arena = ms.Arena(16 << 30)
    try:
        lib = ms.lib()
        tables = {}
        for name, t in (("zipf", orc.zipf_table(1.2, 1 << 20)), ("geo", orc.geom_table(0.25))):
            dt = arena.alloc(t.nbytes)
            ms._memcpy_h2d(dt, t)
            tables[name] = (dt, len(t))
        u = _device_values(ms, lib, arena, dist, _seed(case), bits, tables)
        f = ms.static_vbp_f(bw) if fmt == O.STATIC_VBP else {O.DYNAMIC_VBP: ms.dynamic_vbp_f, O.DELTA_DVBP: ms.delta_f,
                                                             O.FOR_DVBP: ms.for_f, O.RLE: ms.rle_f}[fmt]
        c = ms.morph(u, f)
        back = ms.morph(c, ms.uncompr_f)
        assert torch.equal(ms._device_view(u.data_ptr, 8 * N2), ms._device_view(back.data_ptr, 8 * N2))
        arena.check()
        got = W.masked_digest(fmt, bw, c.raw_bytes(), c.meta(), orc)
        want, want_meta, isa = reference_digests[case].get(timeout=1800)
        assert c.meta() == want_meta, (isa, c.meta(), want_meta)
        assert got == want, f"compressed bytes differ from the {isa} codec"
    finally:
        arena.close()
