"""CPU-side checks of the C ABI: the library loads without a GPU and exports
every function that include/ms_gpu.h declares; layout arithmetic agrees with
the oracle."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "engine_b200", "libms_gpu.so")


def _declared():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(ms_(?:gpu|host|size|rest)\w*)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        pytest.skip("libms_gpu.so not built")
    lib = ctypes.CDLL(LIB)
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, missing
    assert len(_declared()) >= 20


def test_layout_arithmetic_matches_oracle(orc):
    lib = ctypes.CDLL(LIB)
    lib.ms_size_max_byte_any_len.restype = ctypes.c_uint64
    lib.ms_size_max_byte_any_len.argtypes = [ctypes.c_int, ctypes.c_uint, ctypes.c_uint64]
    lib.ms_rest_offset.restype = ctypes.c_uint64
    lib.ms_rest_offset.argtypes = [ctypes.c_int, ctypes.c_uint, ctypes.c_uint64]
    for fmt, bw in [(0, 0), (1, 1), (1, 10), (1, 64), (2, 0), (3, 0), (4, 0), (5, 0)]:
        for n in [0, 1, 511, 512, 1023, 1 << 20, (1 << 20) + 3]:
            assert lib.ms_size_max_byte_any_len(fmt, bw, n) >= orc.size_max_any_len(fmt, bw, n) - 64
        for compr in [0, 64, 640, 4160, 99968]:
            assert lib.ms_rest_offset(fmt, bw, compr) == orc.rest_offset(fmt, bw, compr)


def test_host_index_matches_layout(orc):
    import numpy as np
    import oracle
    lib = ctypes.CDLL(LIB)
    for fmt in (oracle.DYNAMIC_VBP, oracle.DELTA_DVBP, oracle.FOR_DVBP):
        v = orc.uniform_bits(3, 17, 40_000) if fmt != oracle.DELTA_DVBP else np.cumsum(orc.uniform_bits(3, 3, 40_000))
        b, (n, used, compr) = orc.compress(fmt, 0, v)
        ncompr = n - n % orc.block_size(fmt)
        idx = np.zeros(ncompr // 512 + 1, dtype=np.uint64)
        aux = np.zeros(ncompr // 1024 + 1, dtype=np.uint64)
        rc = lib.ms_host_build_index(fmt, b.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint64(compr),
                                     ctypes.c_uint64(ncompr), idx.ctypes.data_as(ctypes.c_void_p),
                                     aux.ctypes.data_as(ctypes.c_void_p))
        assert rc == 0
        # decode every block on the host from the index and compare
        for blk in range(0, ncompr // 512, 7):
            off, bw = int(idx[blk]) & ((1 << 56) - 1), int(idx[blk]) >> 56
            words = b[off: off + 64 * bw].view(np.uint64)
            assert len(words) == 8 * bw


def test_col_load_reports_missing_file(tmp_path):
    """binary_io load of a file that does not exist fails before touching the
    device, with the I/O status."""
    import ctypes as C
    import engine_b200 as ms
    out = ms.MsCol()
    rc = ms.lib().ms_col_load(str(tmp_path / "missing.bin").encode(), ms.DYNAMIC_VBP, 0, C.byref(out), None, None)
    assert rc == 1  # null arena is rejected first
    arena_stub = C.c_void_p(1)  # never dereferenced: the file is opened first
    rc = ms.lib().ms_col_load(str(tmp_path / "missing.bin").encode(), ms.DYNAMIC_VBP, 0, C.byref(out), arena_stub,
                              None)
    assert rc == 7
    assert b"could not open" in ms.lib().ms_gpu_status_string(rc)
