"""The allocation-free select entry point, ms_gpu_select_noalloc.

It exists for callers that may not allocate device memory themselves (the
device budget is reserved up front, memory belongs to another allocator, or
cudaMalloc/cudaFree would synchronise the device at a bad moment).  Its
scratch is a file-scope device array, so this test checks, through the C
ABI, that two calls in a row give exactly the positions and count of the
allocating entry point ms_gpu_select and of the CPU oracle -- i.e. that the
shared scratch left by one call does not leak into the next -- for every
comparison, for values on both sides of 2^63 (the signed compare before the
scalar remainder, the unsigned one inside it), for an empty column and for
one shorter than a 512-row block.  It also checks that a corrupt block index
is reported through the caller's error word and that a missing error word or
an input beyond the stated limit is rejected before anything runs.  The file
name makes pytest collect it last; it also passes on its own in a fresh
process.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

CMPS = [O.CMP_EQ, O.CMP_LT, O.CMP_LE, O.CMP_GT, O.CMP_GE]


def _bind(ms):
    lib = ms.lib()
    f = lib.ms_gpu_select_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_uint64, C.POINTER(ms.MsCol), C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                  C.c_void_p]
    lib.ms_gpu_select_noalloc_max_rows.restype = C.c_uint64
    return lib


def _noalloc(ms, lib, arena, desc, n, cmp, val):
    """One call with caller-owned outputs; returns (positions, count, error word)."""
    d_pos = arena.alloc(8 * max(n, 1))
    d_cnt = arena.alloc(8)
    d_err = arena.alloc(8)
    ms._memcpy_h2d(d_cnt, np.array([0xDEADBEEF], dtype=np.uint64))  # must be overwritten, also when empty
    ms._memcpy_h2d(d_err, np.array([0xFFFF], dtype=np.uint64))      # must be cleared by the call
    rc = lib.ms_gpu_select_noalloc(cmp, val, C.byref(desc), d_pos, n, d_cnt, d_err, None)
    ms._check(rc, "select_noalloc")
    cnt = int(ms._memcpy_d2h(d_cnt, 8).view(np.uint64)[0])
    err = int(ms._memcpy_d2h(d_err, 4).view(np.uint32)[0])
    pos = ms._memcpy_d2h(d_pos, 8 * cnt).view(np.uint64) if cnt and cnt <= n else np.zeros(0, np.uint64)
    return pos, cnt, err


def _fmt(ms, code):
    return {O.UNCOMPR: ms.uncompr_f, O.STATIC_VBP: ms.static_vbp_f(12), O.DYNAMIC_VBP: ms.dynamic_vbp_f,
            O.FOR_DVBP: ms.for_f}[code]


@pytest.mark.parametrize("cmp", CMPS)
@pytest.mark.parametrize("code", [O.UNCOMPR, O.STATIC_VBP, O.DYNAMIC_VBP, O.FOR_DVBP])
def test_noalloc_select_matches_select_and_oracle_twice(ms, orc, code, cmp):
    arena = ms.Arena(1 << 30)
    try:
        lib = _bind(ms)
        for call, (n, val) in enumerate([(300_007, 1500), (70_001, 3000)]):
            v = orc.uniform_bits(100 + call, 12, n)
            col = ms.Column.from_numpy(v, arena)
            if code != O.UNCOMPR:
                col = ms.morph(col, _fmt(ms, code))
            want = orc.select(cmp, val, v, orc.scalar_from(code, 12 if code == O.STATIC_VBP else 0, col.meta()))
            ref_pos = ms.select(cmp, col, val).to_numpy()
            got_pos, cnt, err = _noalloc(ms, lib, arena, col.desc, n, cmp, val)
            assert err == 0
            assert cnt == len(want) == len(ref_pos)
            assert np.array_equal(got_pos, ref_pos)
            assert np.array_equal(got_pos, want)
    finally:
        arena.close()


@pytest.mark.parametrize("cmp", CMPS)
def test_noalloc_signed_split_at_scalar_remainder(ms, orc, cmp):
    """64-bit values on both sides of 2^63 in an uncompressed column whose
    length leaves a scalar remainder: rows before it compare signed, rows in
    it unsigned, exactly as the allocating select and the oracle do."""
    arena = ms.Arena(256 << 20)
    try:
        lib = _bind(ms)
        for call, n in enumerate([4099, 517]):
            v = orc.uniform_bits(7 + call, 64, n)
            val = 1 << 63 | 12345
            col = ms.Column.from_numpy(v, arena)
            want = orc.select(cmp, val, v, orc.scalar_from(O.UNCOMPR, 0, col.meta()))
            got, cnt, err = _noalloc(ms, lib, arena, col.desc, n, cmp, val)
            assert err == 0 and cnt == len(want)
            assert np.array_equal(got, want)
            assert np.array_equal(got, ms.select(cmp, col, val).to_numpy())
    finally:
        arena.close()


def test_noalloc_empty_and_short_columns(ms, orc):
    arena = ms.Arena(64 << 20)
    try:
        lib = _bind(ms)
        empty = ms.MsCol(format=ms.UNCOMPR, count_values=0, size_used_byte=0, size_alloc_byte=64,
                         data=arena.alloc(64))
        got, cnt, err = _noalloc(ms, lib, arena, empty, 0, ms.less, 5)
        assert (cnt, err) == (0, 0)
        for n in (1, 7, 300, 511):  # shorter than one 512-row block: all rest rows
            v = orc.uniform_bits(40 + n, 9, n)
            col = ms.morph(ms.Column.from_numpy(v, arena), ms.dynamic_vbp_f)
            for cmp in CMPS:
                want = orc.select(cmp, 200, v, orc.scalar_from(O.DYNAMIC_VBP, 0, col.meta()))
                got, cnt, err = _noalloc(ms, lib, arena, col.desc, n, cmp, 200)
                assert err == 0 and cnt == len(want)
                assert np.array_equal(got, want)
    finally:
        arena.close()


def test_noalloc_reports_corrupt_block_index(ms, orc):
    """A block-index entry whose bit width is 0 (the offset stays valid, so
    nothing is read out of bounds) is a corrupt column: the call returns OK
    -- it does not synchronise -- and the kernel sets bit 1 of d_err."""
    arena = ms.Arena(256 << 20)
    try:
        lib = _bind(ms)
        n = 40_000
        v = orc.uniform_bits(3, 14, n)
        col = ms.morph(ms.Column.from_numpy(v, arena), ms.dynamic_vbp_f)
        d = col.desc
        nidx = int(d.n_index)
        idx = ms._memcpy_d2h(d.index, 8 * nidx).view(np.uint64).copy()
        idx[5] &= np.uint64((1 << 56) - 1)  # bit width 0
        bad_idx = arena.alloc(8 * nidx)
        ms._memcpy_h2d(bad_idx, idx)
        bad = ms.MsCol(format=d.format, bw=d.bw, count_values=d.count_values, size_used_byte=d.size_used_byte,
                       size_compr_byte=d.size_compr_byte, size_alloc_byte=d.size_alloc_byte, data=d.data,
                       index=bad_idx, index_aux=d.index_aux, n_index=nidx)
        _, _, err = _noalloc(ms, lib, arena, bad, n, ms.less, 100)
        assert err & 1
        # the next call on a sound column starts from a cleared error word
        got, cnt, err = _noalloc(ms, lib, arena, col.desc, n, ms.less, 100)
        assert err == 0 and np.array_equal(got, orc.select(O.CMP_LT, 100, v, orc.scalar_from(O.DYNAMIC_VBP, 0,
                                                                                                col.meta())))
    finally:
        arena.close()


def test_noalloc_rejects_bad_arguments(ms):
    arena = ms.Arena(64 << 20)
    try:
        lib = _bind(ms)
        limit = int(lib.ms_gpu_select_noalloc_max_rows())
        assert limit == 1 << 26
        d = ms.MsCol(format=ms.UNCOMPR, count_values=limit + 1, size_used_byte=8 * (limit + 1),
                     size_alloc_byte=8 * (limit + 1), data=arena.alloc(64))
        rc = lib.ms_gpu_select_noalloc(ms.less, 1, C.byref(d), arena.alloc(64), limit + 1, arena.alloc(8),
                                       arena.alloc(8), None)
        assert rc == 1  # MS_ERR_INVALID, before any kernel runs
        assert b"2^26" in lib.ms_gpu_status_string(rc)
        small = ms.MsCol(format=ms.UNCOMPR, count_values=8, size_used_byte=64, size_alloc_byte=64,
                         data=arena.alloc(64))
        rc = lib.ms_gpu_select_noalloc(ms.less, 1, C.byref(small), arena.alloc(64), 8, arena.alloc(8), None, None)
        assert rc == 1  # the error word is required
    finally:
        arena.close()
