"""Column persistence in the reference's binary_io layout
([count u64][size_used_byte u64][buffer]): store -> load round trips for every
format, files written from the reference's own bytes load and decode, and
loaded columns feed the operators."""
import struct

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _fmt(ms, code, bw):
    return {O.UNCOMPR: ms.uncompr_f, O.DYNAMIC_VBP: ms.dynamic_vbp_f, O.DELTA_DVBP: ms.delta_f,
            O.FOR_DVBP: ms.for_f, O.RLE: ms.rle_f}.get(code) or ms.static_vbp_f(bw)


def _values(orc, code, bw, n, seed):
    if code == O.DELTA_DVBP:
        return orc.sorted_gaps(seed, orc.geom_table(0.25), n)
    if code == O.RLE:
        return orc.runs(seed, 5, 20, n)
    return orc.uniform_bits(seed, bw or 20, n)


CASES = [(O.UNCOMPR, 0), (O.STATIC_VBP, 7), (O.STATIC_VBP, 64), (O.DYNAMIC_VBP, 0), (O.DELTA_DVBP, 0),
         (O.FOR_DVBP, 0), (O.RLE, 0)]


@pytest.mark.parametrize("code,bw", CASES)
@pytest.mark.parametrize("n", [0, 5, 1000, 3 * 1024 + 7, 70_001])
def test_store_load_round_trip(ms, arena, orc, tmp_path, code, bw, n):
    v = _values(orc, code, bw, n, seed=n + 3)
    c = ms.morph(ms.Column.from_numpy(v, arena), _fmt(ms, code, bw))
    path = str(tmp_path / "col.bin")
    c.store(path)
    raw = open(path, "rb").read()
    assert struct.unpack("<QQ", raw[:16]) == (n, c.get_size_used_byte())
    assert np.array_equal(np.frombuffer(raw[16:], np.uint8), c.raw_bytes())
    k = ms.Column.load(path, _fmt(ms, code, bw), arena)
    assert k.meta() == c.meta()
    assert np.array_equal(k.to_numpy(), v)
    if code != O.RLE and n:
        assert ms.select_project_sum(k, ms.less, 1 << 10, k) == ms.select_project_sum(c, ms.less, 1 << 10, c)


@pytest.mark.parametrize("code", [O.DYNAMIC_VBP, O.DELTA_DVBP, O.FOR_DVBP])
def test_load_file_of_reference_bytes(ms, arena, orc, tmp_path, code):
    """A file holding the bytes the reference's codecs produce (the oracle's,
    pinned against them) loads, rebuilds its block index and decodes."""
    v = _values(orc, code, 0, 100_003, seed=11)
    b, m = orc.compress(code, 0, v)
    path = tmp_path / "ref.bin"
    path.write_bytes(struct.pack("<QQ", m[0], m[1]) + b.tobytes())
    k = ms.Column.load(str(path), _fmt(ms, code, 0), arena)
    assert k.meta() == m
    assert np.array_equal(k.to_numpy(), v)


def test_load_rejects_inconsistent_file(ms, arena, orc, tmp_path):
    v = orc.uniform_bits(1, 12, 5000)
    c = ms.morph(ms.Column.from_numpy(v, arena), ms.dynamic_vbp_f)
    path = str(tmp_path / "c.bin")
    c.store(path)
    with pytest.raises(ms.MorphStoreError):  # wrong format for the bytes
        ms.Column.load(path, ms.static_vbp_f(3), arena)
    raw = bytearray(open(path, "rb").read())
    raw[8:16] = struct.pack("<Q", c.get_size_used_byte() + 8)  # size disagrees with the payload
    open(path, "wb").write(bytes(raw) + bytes(8))
    with pytest.raises(ms.MorphStoreError):
        ms.Column.load(path, ms.dynamic_vbp_f, arena)
