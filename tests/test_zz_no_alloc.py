"""The allocation-free select entry point, ms_gpu_select_noalloc.

It exists for callers that may not allocate device memory themselves (the
device budget is reserved up front, memory belongs to another allocator, or
cudaMalloc/cudaFree would synchronise the device at a bad moment).  Its
scratch is a file-scope device array, so this test checks, through the C
ABI, that two calls in a row give exactly the positions and count of the
allocating entry point ms_gpu_select -- i.e. that the shared scratch left by
one call does not leak into the next.  The file name makes pytest collect it
last; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _bind(ms):
    lib = ms.lib()
    f = lib.ms_gpu_select_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_uint64, C.POINTER(ms.MsCol), C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                  C.c_void_p]
    lib.ms_gpu_select_noalloc_max_rows.restype = C.c_uint64
    return lib


def _noalloc(ms, lib, arena, col, cmp, val):
    n = col.get_count_values()
    d_pos = arena.alloc(8 * max(n, 1))     # the caller owns inputs and outputs
    d_cnt = arena.alloc(8)
    d_err = arena.alloc(8)
    rc = lib.ms_gpu_select_noalloc(cmp, val, C.byref(col.desc), d_pos, n, d_cnt, d_err, None)
    ms._check(rc, "select_noalloc")
    cnt = int(ms._memcpy_d2h(d_cnt, 8).view(np.uint64)[0])
    err = int(ms._memcpy_d2h(d_err, 4).view(np.uint32)[0])
    assert err == 0
    return ms._memcpy_d2h(d_pos, 8 * cnt).view(np.uint64), cnt


@pytest.mark.parametrize("code", [O.UNCOMPR, O.STATIC_VBP, O.DYNAMIC_VBP, O.FOR_DVBP])
def test_noalloc_select_matches_select_twice(ms, orc, code):
    arena = ms.Arena(1 << 30)
    try:
        lib = _bind(ms)
        fmt = {O.UNCOMPR: ms.uncompr_f, O.STATIC_VBP: ms.static_vbp_f(12), O.DYNAMIC_VBP: ms.dynamic_vbp_f,
               O.FOR_DVBP: ms.for_f}[code]
        for call, (n, val) in enumerate([(300_007, 1500), (70_001, 3000)]):
            v = orc.uniform_bits(100 + call, 12, n)
            col = ms.Column.from_numpy(v, arena)
            if code != O.UNCOMPR:
                col = ms.morph(col, fmt)
            ref_pos = ms.select(ms.less, col, val).to_numpy()
            got_pos, cnt = _noalloc(ms, lib, arena, col, ms.less, val)
            assert cnt == len(ref_pos)
            assert np.array_equal(got_pos, ref_pos)
    finally:
        arena.close()


def test_noalloc_rejects_oversized_input(ms):
    arena = ms.Arena(64 << 20)
    try:
        lib = _bind(ms)
        limit = int(lib.ms_gpu_select_noalloc_max_rows())
        assert limit == 1 << 26
        d = ms.MsCol(format=ms.UNCOMPR, count_values=limit + 1, size_used_byte=8 * (limit + 1),
                     size_alloc_byte=8 * (limit + 1), data=arena.alloc(64))
        rc = lib.ms_gpu_select_noalloc(ms.less, 1, C.byref(d), arena.alloc(64), limit + 1, arena.alloc(8), None,
                                       None)
        assert rc == 1  # MS_ERR_INVALID, before any kernel runs
        assert b"2^26" in lib.ms_gpu_status_string(rc)
    finally:
        arena.close()
