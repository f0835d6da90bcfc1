"""B200-native compression-aware query path (host-side Python layer).

A thin mirror of MorphStore's column / operator API over the C ABI in
``include/ms_gpu.h`` (``libms_gpu.so``, built from ``engine_b200/csrc``).
Names follow the reference: ``morph``, ``select``, ``project``, ``agg_sum``,
``semi_join``, ``intersect_sorted``, ``group``, ``agg_sum_grouped``; formats
``uncompr_f``, ``static_vbp_f(bw)``, ``dynamic_vbp_f``, ``delta_f``,
``for_f``, ``rle_f``; comparisons ``equal``, ``less``, ``lessequal``,
``greater``, ``greaterequal``.

There is no CPU fallback: importing this package loads the CUDA library and
raises if it is missing, and every operator runs on the GPU.  A non-OK status
from the library becomes ``MorphStoreError`` (the reference's host code
throws ``std::runtime_error``).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libms_gpu.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"engine_b200: {LIB_PATH} is missing; run `python engine_b200/build.py` "
                      "(or __graft_entry__.build()) first -- there is no CPU fallback")

_lib = C.CDLL(LIB_PATH)

UNCOMPR, STATIC_VBP, DYNAMIC_VBP, DELTA_DVBP, FOR_DVBP, RLE = range(6)
equal, less, lessequal, greater, greaterequal = range(5)


class MorphStoreError(RuntimeError):
    """A non-OK ms_status returned by the C ABI."""

    def __init__(self, status: int, where: str):
        msg = _lib.ms_gpu_status_string(status).decode()
        super().__init__(f"{where}: {msg} (status {status})")
        self.status = status


class MsTuning(C.Structure):
    _fields_ = [("staged", C.c_int), ("warps", C.c_uint), ("stages", C.c_uint), ("stage_bytes", C.c_uint),
                ("ctas_per_sm", C.c_uint), ("values_per_thread", C.c_uint)]


class MsCol(C.Structure):
    _fields_ = [("format", C.c_uint32), ("bw", C.c_uint32), ("count_values", C.c_uint64),
                ("size_used_byte", C.c_uint64), ("size_compr_byte", C.c_uint64),
                ("size_alloc_byte", C.c_uint64), ("data", C.c_void_p), ("index", C.c_void_p),
                ("index_aux", C.c_void_p), ("n_index", C.c_uint64)]


_P = C.POINTER
_V = C.c_void_p
_U64 = C.c_uint64
_sig = {
    "ms_gpu_abi_version": (C.c_int, []),
    "ms_gpu_status_string": (C.c_char_p, [C.c_int]),
    "ms_gpu_device_info": (C.c_int, [_P(C.c_int), _P(C.c_int), _P(C.c_int)]),
    "ms_gpu_arena_create": (C.c_int, [_U64, _P(_V)]),
    "ms_gpu_arena_alloc": (C.c_int, [_V, _U64, _P(_V)]),
    "ms_gpu_arena_reset": (C.c_int, [_V]),
    "ms_gpu_arena_used": (C.c_int, [_V, _P(_U64)]),
    "ms_gpu_arena_destroy": (C.c_int, [_V]),
    "ms_gpu_arena_check": (C.c_int, [_V, _V]),
    "ms_size_max_byte_any_len": (_U64, [C.c_int, C.c_uint, _U64]),
    "ms_rest_offset": (_U64, [C.c_int, C.c_uint, _U64]),
    "ms_host_build_index": (C.c_int, [C.c_int, _V, _U64, _U64, _V, _V]),
    "ms_gpu_morph": (C.c_int, [_P(MsCol), C.c_int, C.c_uint, _P(MsCol), _V, _V]),
    "ms_gpu_build_index": (C.c_int, [_P(MsCol), _V, _V]),
    "ms_gpu_agg_sum": (C.c_int, [_P(MsCol), _V, _V, _V]),
    "ms_gpu_select": (C.c_int, [C.c_int, _U64, _P(MsCol), C.c_int, C.c_uint, _P(MsCol), _V, _V]),
    "ms_gpu_project": (C.c_int, [_P(MsCol), _P(MsCol), C.c_int, C.c_uint, _P(MsCol), _V, _V]),
    "ms_gpu_select_project_sum": (C.c_int, [_P(MsCol), C.c_int, _U64, _P(MsCol), _V, _V, _V, _V, _V, _V]),
    "ms_gpu_select_project_sum_async": (C.c_int, [_P(MsCol), C.c_int, _U64, _P(MsCol), _V, _V, _V, _V]),
    "ms_gpu_semi_join": (C.c_int, [_P(MsCol), _P(MsCol), C.c_int, C.c_uint, _P(MsCol), _V, _V]),
    "ms_gpu_intersect_sorted": (C.c_int, [_P(MsCol), _P(MsCol), C.c_int, C.c_uint, _P(MsCol), _V, _V]),
    "ms_gpu_group": (C.c_int, [_P(MsCol), _P(MsCol), C.c_int, _P(MsCol), C.c_int, _P(MsCol), _V, _V]),
    "ms_gpu_agg_sum_grouped": (C.c_int, [_P(MsCol), _P(MsCol), _U64, _P(MsCol), _V, _V]),
    "ms_gpu_query3": (C.c_int, [_P(MsCol), C.c_int, _U64, _P(MsCol), _P(MsCol), _P(MsCol), _P(MsCol), _U64, _V,
                                _V, _V, _P(_U64), _P(_U64), _V, _V]),
    "ms_gpu_set_tuning": (C.c_int, [_P(MsTuning)]),
    "ms_gpu_set_query_tuning": (C.c_int, [_P(MsTuning)]),
    "ms_gpu_col_compact": (C.c_int, [_P(MsCol), _P(MsCol), _V, _V]),
    "ms_gpu_natural_join": (C.c_int, [_P(MsCol), _P(MsCol), C.c_int, C.c_uint, C.c_int, C.c_uint, _P(MsCol),
                                      _P(MsCol), _V, _V]),
    "ms_col_store": (C.c_int, [_P(MsCol), C.c_char_p, _V]),
    "ms_col_load": (C.c_int, [C.c_char_p, C.c_int, C.c_uint, _P(MsCol), _V, _V]),
    "ms_gpu_batch_create": (C.c_int, [_P(MsCol), _V, _U64, C.c_int, _V, _P(_V), _V]),
    "ms_gpu_batch_set_config": (C.c_int, [_V, _P(MsTuning)]),
    "ms_gpu_batch_get_config": (C.c_int, [_V, _P(MsTuning)]),
    "ms_gpu_batch_set_kind_config": (C.c_int, [_V, C.c_int, _P(MsTuning)]),
    "ms_gpu_batch_get_kind_config": (C.c_int, [_V, C.c_int, _P(MsTuning), _P(_U64)]),
    "ms_gpu_batch_run": (C.c_int, [_V, _V, _V, _V]),
    "ms_gpu_batch_run_graph": (C.c_int, [_V, _V, _V, _V]),
    "ms_gpu_batch_info": (C.c_int, [_V, _P(_U64), _P(_U64)]),
    "ms_gpu_batch_destroy": (None, [_V]),
    "ms_gpu_get_query_tuning": (C.c_int, [_P(MsTuning)]),
    "ms_gpu_query3_last_pass_ms": (C.c_int, [_P(C.c_double)]),
    "ms_gpu_get_tuning": (C.c_int, [_P(MsTuning)]),
    "ms_gpu_gen_uniform_bits": (C.c_int, [_U64, C.c_uint, _U64, _V, _V]),
    "ms_gpu_gen_uniform_bits_at": (C.c_int, [_U64, C.c_uint, _U64, _U64, _V, _V]),
    "ms_gpu_col_slice": (C.c_int, [_P(MsCol), _U64, _U64, _V, _P(MsCol)]),
    "ms_gpu_delta_lane_sums": (C.c_int, [_P(MsCol), _V, _V, _V]),
    "ms_gpu_gen_from_table": (C.c_int, [_U64, _V, _U64, _U64, _V, _V]),
    "ms_gpu_gen_sorted_gaps": (C.c_int, [_U64, _V, _U64, _U64, _V, _V, _V]),
    "ms_gpu_gen_runs": (C.c_int, [_U64, C.c_uint, C.c_uint, _U64, _V, _V, _V]),
}
for _name, (_res, _args) in _sig.items():
    _f = getattr(_lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def _check(status: int, where: str) -> None:
    if status != 0:
        raise MorphStoreError(status, where)


def lib():
    """The loaded ctypes library (for callers that bind more entry points)."""
    return _lib


# ---------------------------------------------------------------------------
# formats
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class Format:
    code: int
    bw: int = 0

    def __call__(self, bw: int) -> "Format":  # static_vbp_f(bw)
        if self.code != STATIC_VBP:
            raise TypeError("only static_vbp_f takes a bit width")
        if not 1 <= bw <= 64:
            raise ValueError("static_vbp_f: bit width must be in 1..64")
        return Format(STATIC_VBP, bw)

    @property
    def name(self) -> str:
        n = {UNCOMPR: "uncompr_f", STATIC_VBP: "static_vbp_f", DYNAMIC_VBP: "dynamic_vbp_f",
             DELTA_DVBP: "delta_f", FOR_DVBP: "for_f", RLE: "rle_f"}[self.code]
        return f"{n}<{self.bw}>" if self.code == STATIC_VBP else n


uncompr_f = Format(UNCOMPR)
static_vbp_f = Format(STATIC_VBP)
dynamic_vbp_f = Format(DYNAMIC_VBP)
delta_f = Format(DELTA_DVBP)
for_f = Format(FOR_DVBP)
rle_f = Format(RLE)


def _fmt(f) -> Format:
    if isinstance(f, Format):
        if f.code == STATIC_VBP and not f.bw:
            raise ValueError("static_vbp_f needs a bit width: static_vbp_f(bw)")
        return f
    raise TypeError(f"not a format: {f!r}")


# ---------------------------------------------------------------------------
# device memory
# ---------------------------------------------------------------------------
def _torch():
    import torch  # plumbing only: host<->device copies and streams
    if not torch.cuda.is_available():
        raise MorphStoreError(3, "engine_b200 needs a CUDA device")
    return torch


class Arena:
    """Device arena (ms_arena): one cudaMalloc, bump allocation, reset."""

    def __init__(self, capacity_byte: int):
        _torch()
        h = _V()
        _check(_lib.ms_gpu_arena_create(capacity_byte, C.byref(h)), "arena_create")
        self.h = h
        self.capacity = capacity_byte

    def alloc(self, nbytes: int) -> int:
        p = _V()
        _check(_lib.ms_gpu_arena_alloc(self.h, nbytes, C.byref(p)), "arena_alloc")
        return p.value

    def reset(self) -> None:
        _check(_lib.ms_gpu_arena_reset(self.h), "arena_reset")

    def used(self) -> int:
        u = _U64()
        _check(_lib.ms_gpu_arena_used(self.h, C.byref(u)), "arena_used")
        return u.value

    def check(self, stream=None) -> None:
        _check(_lib.ms_gpu_arena_check(self.h, _stream_ptr(stream)), "arena_check")

    def close(self) -> None:
        if getattr(self, "h", None):
            _lib.ms_gpu_arena_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_arena: Arena | None = None


def default_arena() -> Arena:
    global _default_arena
    if _default_arena is None:
        size = int(os.environ.get("MS_ARENA_BYTES", str(8 << 30)))
        _default_arena = Arena(size)
    return _default_arena


def _stream_ptr(stream) -> int | None:
    if stream is None:
        torch = _torch()
        return torch.cuda.current_stream().cuda_stream or None
    return getattr(stream, "cuda_stream", stream) or None


def _memcpy_h2d(dst: int, src: np.ndarray, stream=None) -> None:
    torch = _torch()
    if src.nbytes == 0:
        return
    t = torch.from_numpy(np.ascontiguousarray(src).view(np.uint8))
    d = _device_view(dst, src.nbytes)
    d.copy_(t, non_blocking=False)


def _device_view(ptr: int, nbytes: int):
    """A torch uint8 tensor aliasing device memory at ptr (no ownership)."""
    torch = _torch()

    class _Holder:
        __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}

    return torch.as_tensor(_Holder(), device="cuda")


def _memcpy_d2h(src: int, nbytes: int) -> np.ndarray:
    if nbytes == 0:
        return np.zeros(0, dtype=np.uint8)
    _torch().cuda.synchronize()
    return _device_view(src, nbytes).cpu().numpy().copy()


# ---------------------------------------------------------------------------
# columns
# ---------------------------------------------------------------------------
class Column:
    """A device-resident column<F> (ms_col) plus the arena that owns it."""

    def __init__(self, desc: MsCol, arena: Arena, keep=None):
        self.desc = desc
        self.arena = arena
        self._keep = keep

    # metadata, as column<F> (column.h:118-144)
    @property
    def format(self) -> Format:
        return Format(self.desc.format, self.desc.bw)

    def get_count_values(self) -> int:
        return int(self.desc.count_values)

    def get_size_used_byte(self) -> int:
        return int(self.desc.size_used_byte)

    def get_size_compr_byte(self) -> int:
        return int(self.desc.size_compr_byte)

    def meta(self):
        return (self.get_count_values(), self.get_size_used_byte(), self.get_size_compr_byte())

    @staticmethod
    def from_numpy(values, arena: Arena | None = None) -> "Column":
        """Uncompressed device column from host values (make_column)."""
        arena = arena or default_arena()
        v = np.ascontiguousarray(values, dtype=np.uint64)
        p = arena.alloc(max(v.nbytes, 8))
        _memcpy_h2d(p, v)
        d = MsCol(format=UNCOMPR, bw=0, count_values=len(v), size_used_byte=v.nbytes, size_compr_byte=0,
                  size_alloc_byte=max(v.nbytes, 8), data=p)
        return Column(d, arena)

    @staticmethod
    def from_bytes(fmt: Format, data: np.ndarray, meta, arena: Arena | None = None,
                   build_index: bool = True) -> "Column":
        """Upload a column in the reference's byte layout (count, used, compr
        metadata as column<F>); the block index is built on the host."""
        arena = arena or default_arena()
        fmt = _fmt(fmt)
        n, used, compr = (int(x) for x in meta)
        buf = np.zeros(max(used, 8) + 64, dtype=np.uint8)
        buf[:used] = np.asarray(data, dtype=np.uint8)[:used]
        p = arena.alloc(len(buf))
        _memcpy_h2d(p, buf)
        d = MsCol(format=fmt.code, bw=fmt.bw, count_values=n, size_used_byte=used, size_compr_byte=compr,
                  size_alloc_byte=len(buf), data=p)
        col = Column(d, arena)
        if build_index and fmt.code in (DYNAMIC_VBP, DELTA_DVBP, FOR_DVBP):
            col._host_index(buf)
        return col

    def _host_index(self, host_bytes: np.ndarray) -> None:
        fmt = self.desc.format
        n, used, compr = self.meta()
        nrest = 0 if compr == used else (used - int(_lib.ms_rest_offset(fmt, self.desc.bw, compr))) // 8
        ncompr = n - nrest
        nb = ncompr // 512
        if nb == 0:
            return
        idx = np.zeros(nb + 1, dtype=np.uint64)
        aux = np.zeros(nb // 2 + 1, dtype=np.uint64)
        _check(_lib.ms_host_build_index(fmt, host_bytes.ctypes.data, compr, ncompr, idx.ctypes.data,
                                        aux.ctypes.data), "host_build_index")
        pi = self.arena.alloc(idx.nbytes)
        _memcpy_h2d(pi, idx)
        self.desc.index = pi
        self.desc.n_index = nb
        if fmt == FOR_DVBP:
            pa = self.arena.alloc(aux.nbytes)
            _memcpy_h2d(pa, aux)
            self.desc.index_aux = pa

    def store(self, path: str, stream=None) -> None:
        """binary_io<F>::store (binary_io.h:72-84): [count][used bytes][bytes]."""
        _check(_lib.ms_col_store(C.byref(self.desc), os.fsencode(path), _stream_ptr(stream)), "col_store")

    @staticmethod
    def load(path: str, fmt: "Format", arena: "Arena | None" = None, stream=None) -> "Column":
        """binary_io<F>::load (binary_io.h:43-70) into device memory."""
        arena = arena or default_arena()
        fmt = _fmt(fmt)
        out = MsCol()
        _check(_lib.ms_col_load(os.fsencode(path), fmt.code, fmt.bw, C.byref(out), arena.h, _stream_ptr(stream)),
               "col_load")
        return Column(out, arena)

    def compact(self, arena: "Arena | None" = None, stream=None) -> "Column":
        """A copy of this column in storage of exactly its used size."""
        arena = arena or self.arena
        out = MsCol()
        _check(_lib.ms_gpu_col_compact(C.byref(self.desc), C.byref(out), arena.h, _stream_ptr(stream)),
               "col_compact")
        return Column(out, arena)

    def slice(self, row_begin: int, row_end: int, carry_in: np.ndarray | None = None) -> "Column":
        """A view of rows [row_begin, row_end) sharing this column's storage
        (one rank's shard); carry_in: the 8 lane values before row_begin of a
        delta_f column (uploaded into the arena), None = zeros."""
        d_carry = None
        if carry_in is not None:
            d_carry = self.arena.alloc(64)
            _memcpy_h2d(d_carry, np.asarray(carry_in, dtype=np.uint64).reshape(8))
        out = MsCol()
        _check(_lib.ms_gpu_col_slice(C.byref(self.desc), row_begin, row_end, d_carry, C.byref(out)), "col_slice")
        return Column(out, self.arena, keep=self)

    def delta_lane_sums(self, stream=None) -> np.ndarray:
        """The 8 lane-wise wrapping sums of a delta_f column's deltas."""
        d = self.arena.alloc(64)
        _check(_lib.ms_gpu_delta_lane_sums(C.byref(self.desc), d, self.arena.h, _stream_ptr(stream)),
               "delta_lane_sums")
        return _memcpy_d2h(d, 64).view(np.uint64).copy()

    def build_index(self, stream=None) -> None:
        _check(_lib.ms_gpu_build_index(C.byref(self.desc), self.arena.h, _stream_ptr(stream)), "build_index")

    def raw_bytes(self) -> np.ndarray:
        """The column's bytes (compressed part, gap, rest) copied to the host."""
        return _memcpy_d2h(self.desc.data, int(self.desc.size_used_byte))

    def to_numpy(self) -> np.ndarray:
        """Decompressed values on the host (morph to uncompr_f + copy)."""
        u = morph(self, uncompr_f) if self.desc.format != UNCOMPR else self
        n = u.get_count_values()
        return _memcpy_d2h(u.desc.data, 8 * n).view(np.uint64)

    @property
    def data_ptr(self) -> int:
        return int(self.desc.data)


def _out(arena: Arena) -> MsCol:
    return MsCol()


def morph(col: Column, dst: Format, stream=None) -> Column:
    """morph<ve, dst>(col) (morph.h:114-116)."""
    dst = _fmt(dst)
    out = MsCol()
    _check(_lib.ms_gpu_morph(C.byref(col.desc), dst.code, dst.bw, C.byref(out), col.arena.h, _stream_ptr(stream)),
           f"morph<{dst.name}>")
    return Column(out, col.arena, keep=col)


def agg_sum(col: Column, stream=None) -> int:
    """agg_sum<ve, F>(col) (agg_sum.h:56-65); returns the uint64 sum."""
    p = col.arena.alloc(8)
    _check(_lib.ms_gpu_agg_sum(C.byref(col.desc), p, col.arena.h, _stream_ptr(stream)), "agg_sum")
    col.arena.check(stream)
    return int(_memcpy_d2h(p, 8).view(np.uint64)[0])


def select(cmp: int, col: Column, val: int, out_f: Format = uncompr_f, stream=None) -> Column:
    """my_select_wit_t<cmp, ve, out_f, F>::apply(col, val) (select_compr.h:100-260)."""
    out_f = _fmt(out_f)
    out = MsCol()
    _check(_lib.ms_gpu_select(cmp, val, C.byref(col.desc), out_f.code, out_f.bw, C.byref(out), col.arena.h,
                              _stream_ptr(stream)), "select")
    return Column(out, col.arena, keep=col)


def project(data: Column, pos: Column, out_f: Format = uncompr_f, stream=None) -> Column:
    """my_project_wit_t<ve, out_f, data_f, pos_f>::apply(data, pos) (project_compr.h:75-262)."""
    out_f = _fmt(out_f)
    out = MsCol()
    _check(_lib.ms_gpu_project(C.byref(data.desc), C.byref(pos.desc), out_f.code, out_f.bw, C.byref(out),
                               data.arena.h, _stream_ptr(stream)), "project")
    return Column(out, data.arena, keep=(data, pos))


def select_project_sum(x: Column, cmp: int, c: int, y: Column, want_positions: bool = False, stream=None):
    """Fused select(x cmp c) -> project(y) -> agg_sum.  Returns (sum, count)
    or, with want_positions, (sum, count, positions, values) as numpy."""
    a = x.arena
    ds = a.alloc(8)
    dc = a.alloc(8)
    dp = dv = None
    n = x.get_count_values()
    if want_positions:
        dp = a.alloc(max(8 * n, 8))
        dv = a.alloc(max(8 * n, 8))
    _check(_lib.ms_gpu_select_project_sum(C.byref(x.desc), cmp, c, C.byref(y.desc), ds, dc, dp, dv, a.h,
                                          _stream_ptr(stream)), "select_project_sum")
    a.check(stream)
    s = int(_memcpy_d2h(ds, 8).view(np.uint64)[0])
    k = int(_memcpy_d2h(dc, 8).view(np.uint64)[0])
    if not want_positions:
        return s, k
    return s, k, _memcpy_d2h(dp, 8 * k).view(np.uint64), _memcpy_d2h(dv, 8 * k).view(np.uint64)


def semi_join(l: Column, r: Column, out_f: Format = uncompr_f, stream=None) -> Column:
    """semi_join<ve, out_f, L_f, R_f>(L, R) (join.h:193-218): ascending
    positions of R whose value occurs in L."""
    out_f = _fmt(out_f)
    out = MsCol()
    _check(_lib.ms_gpu_semi_join(C.byref(l.desc), C.byref(r.desc), out_f.code, out_f.bw, C.byref(out), r.arena.h,
                                 _stream_ptr(stream)), "semi_join")
    return Column(out, r.arena, keep=(l, r))


def natural_join(l: Column, r: Column, out_l_f: Format = uncompr_f, out_r_f: Format = uncompr_f, stream=None):
    """join<ve, outL_f, outR_f, L_f, R_f>(L, R) (join.h:158-187): (positions
    in L of the first occurrence of each matching value, rows of R)."""
    fl, fr = _fmt(out_l_f), _fmt(out_r_f)
    ol, orr = MsCol(), MsCol()
    _check(_lib.ms_gpu_natural_join(C.byref(l.desc), C.byref(r.desc), fl.code, fl.bw, fr.code, fr.bw, C.byref(ol),
                                    C.byref(orr), r.arena.h, _stream_ptr(stream)), "natural_join")
    return Column(ol, r.arena, keep=(l, r)), Column(orr, r.arena, keep=(l, r))


def intersect_sorted(l: Column, r: Column, out_f: Format = uncompr_f, stream=None) -> Column:
    """intersect_sorted<ve, out_f, L_f, R_f>(L, R) (intersect.h:52-63)."""
    out_f = _fmt(out_f)
    out = MsCol()
    _check(_lib.ms_gpu_intersect_sorted(C.byref(l.desc), C.byref(r.desc), out_f.code, out_f.bw, C.byref(out),
                                        l.arena.h, _stream_ptr(stream)), "intersect_sorted")
    return Column(out, l.arena, keep=(l, r))


def group(col: Column, gr_in: Column | None = None, gr_f: Format = uncompr_f, ext_f: Format = uncompr_f,
          stream=None):
    """group_vec<ve, gr_f, ext_f, F>(col) (group_compr.h:281-300), or the
    binary group with gr_in (group.h:97-112).  Returns (group ids, extents)."""
    gr_f, ext_f = _fmt(gr_f), _fmt(ext_f)
    og, oe = MsCol(), MsCol()
    _check(_lib.ms_gpu_group(C.byref(gr_in.desc) if gr_in is not None else None, C.byref(col.desc), gr_f.code,
                             C.byref(og), ext_f.code, C.byref(oe), col.arena.h, _stream_ptr(stream)), "group")
    return Column(og, col.arena, keep=col), Column(oe, col.arena, keep=col)


def agg_sum_grouped(gr: Column, data: Column, n_groups: int, stream=None) -> Column:
    """agg_sum<ve>(gr, data, n_groups) (agg_sum.h:95-106): per-group sums."""
    out = MsCol()
    _check(_lib.ms_gpu_agg_sum_grouped(C.byref(gr.desc), C.byref(data.desc), n_groups, C.byref(out), gr.arena.h,
                                       _stream_ptr(stream)), "agg_sum_grouped")
    return Column(out, gr.arena, keep=(gr, data))


def set_tuning(staged: int = 1, warps: int = 24, stages: int = 4, stage_bytes: int = 49152,
               ctas_per_sm: int = 1, values_per_thread: int = 16) -> None:
    """Launch parameters of the fused kernels (ms_gpu_set_tuning)."""
    t = MsTuning(staged, warps, stages, stage_bytes, ctas_per_sm, values_per_thread)
    _check(_lib.ms_gpu_set_tuning(C.byref(t)), "set_tuning")


def get_tuning() -> dict:
    t = MsTuning()
    _check(_lib.ms_gpu_get_tuning(C.byref(t)), "get_tuning")
    return {k: getattr(t, k) for k, _ in MsTuning._fields_}


def query3(filter_col: Column, cmp: int, c: int, fk: Column, l: Column, gkey: Column, measure: Column,
           cap: int = 1 << 16, stream=None):
    """The fused select -> semi_join -> intersect -> project -> group -> sum
    query.  Returns (keys, extents, sums, |P|) in group-id order."""
    keys = np.zeros(cap, np.uint64)
    ext = np.zeros(cap, np.uint64)
    sums = np.zeros(cap, np.uint64)
    ng, npos = _U64(), _U64()
    _check(_lib.ms_gpu_query3(C.byref(filter_col.desc), cmp, c, C.byref(fk.desc), C.byref(l.desc),
                              C.byref(gkey.desc), C.byref(measure.desc), cap, keys.ctypes.data, ext.ctypes.data,
                              sums.ctypes.data, C.byref(ng), C.byref(npos), filter_col.arena.h, _stream_ptr(stream)),
           "query3")
    k = int(ng.value)
    return keys[:k], ext[:k], sums[:k], int(npos.value)


def set_query_tuning(staged: int = 1, warps: int = 16, stages: int = 3, stage_bytes: int = 57344) -> None:
    """Launch configuration of query3's staged kernel."""
    t = MsTuning(staged=staged, warps=warps, stages=stages, stage_bytes=stage_bytes, ctas_per_sm=1,
                 values_per_thread=16)
    _check(_lib.ms_gpu_set_query_tuning(C.byref(t)), "set_query_tuning")


def query3_last_pass_ms() -> float:
    """Device time of the last query3 call's fact-table pass, in ms (-1 before
    the first call)."""
    v = C.c_double()
    _check(_lib.ms_gpu_query3_last_pass_ms(C.byref(v)), "query3_last_pass_ms")
    return float(v.value)


def get_query_tuning() -> dict:
    t = MsTuning()
    _check(_lib.ms_gpu_get_query_tuning(C.byref(t)), "get_query_tuning")
    return {"staged": t.staged, "warps": t.warps, "stages": t.stages, "stage_bytes": t.stage_bytes}


class Batch:
    """Many columns, one persistent launch: for every column i,
    decompress -> select(value cmp consts[i]) -> sum of the selected values.
    run() returns (counts, sums) as uint64 arrays; graph=True replays a CUDA
    graph captured on first use."""

    def __init__(self, cols, consts, cmp: int = less, arena: "Arena | None" = None, stream=None):
        self.cols = list(cols)
        self.arena = arena or (self.cols[0].arena if self.cols else default_arena())
        n = len(self.cols)
        descs = (MsCol * max(n, 1))(*[c.desc for c in self.cols])
        cv = np.ascontiguousarray(consts, dtype=np.uint64)
        if len(cv) != n:
            raise ValueError("one constant per column")
        self.n = n
        self.h = _V()
        _check(_lib.ms_gpu_batch_create(descs, cv.ctypes.data if n else None, n, cmp, self.arena.h,
                                        C.byref(self.h), _stream_ptr(stream)), "batch_create")
        self.d_cnt = self.arena.alloc(8 * max(n, 1))
        self.d_sum = self.arena.alloc(8 * max(n, 1))

    def set_config(self, warps: int = 12, stages: int = 2, stage_bytes: int = 8192, ctas_per_sm: int = 1) -> None:
        t = MsTuning(staged=1, warps=warps, stages=stages, stage_bytes=stage_bytes, ctas_per_sm=ctas_per_sm,
                     values_per_thread=16)
        _check(_lib.ms_gpu_batch_set_config(self.h, C.byref(t)), "batch_set_config")

    def get_config(self) -> dict:
        t = MsTuning()
        _check(_lib.ms_gpu_batch_get_config(self.h, C.byref(t)), "batch_get_config")
        return {"warps": t.warps, "stages": t.stages, "stage_bytes": t.stage_bytes, "ctas_per_sm": t.ctas_per_sm}

    KINDS = {"vbp": 0, "for": 1, "delta": 2, "rest": 3, "rle": 4}

    def set_kind_config(self, kind: str, warps: int | None = None, stages: int = 2, stage_bytes: int = 8192,
                        ctas_per_sm: int = 1) -> None:
        """Give one decoder kind ("vbp", "for", "delta", "rest", "rle") its own
        launch configuration; warps=None returns it to the plan's."""
        t = None
        if warps is not None:
            t = MsTuning(staged=1, warps=warps, stages=stages, stage_bytes=stage_bytes, ctas_per_sm=ctas_per_sm,
                         values_per_thread=16)
        _check(_lib.ms_gpu_batch_set_kind_config(self.h, self.KINDS[kind], C.byref(t) if t else None),
               "batch_set_kind_config")

    def kind_configs(self) -> dict:
        out = {}
        for name, k in self.KINDS.items():
            t, n = MsTuning(), _U64()
            _check(_lib.ms_gpu_batch_get_kind_config(self.h, k, C.byref(t), C.byref(n)), "batch_get_kind_config")
            if n.value:
                out[name] = {"warps": t.warps, "stages": t.stages, "stage_bytes": t.stage_bytes,
                             "ctas_per_sm": t.ctas_per_sm, "items": int(n.value)}
        return out

    def launch(self, graph: bool = False, stream=None) -> None:
        f = _lib.ms_gpu_batch_run_graph if graph else _lib.ms_gpu_batch_run
        _check(f(self.h, self.d_cnt, self.d_sum, _stream_ptr(stream)), "batch_run")

    def results(self):
        self.arena.check()
        if not self.n:
            return np.zeros(0, np.uint64), np.zeros(0, np.uint64)
        cnt = _memcpy_d2h(self.d_cnt, 8 * self.n).view(np.uint64)
        s = _memcpy_d2h(self.d_sum, 8 * self.n).view(np.uint64)
        return cnt, s

    def run(self, graph: bool = False, stream=None):
        self.launch(graph, stream)
        return self.results()

    def info(self) -> dict:
        a, b = _U64(), _U64()
        _check(_lib.ms_gpu_batch_info(self.h, C.byref(a), C.byref(b)), "batch_info")
        return {"items": int(a.value), "plan_bytes": int(b.value)}

    def close(self) -> None:
        if self.h:
            _lib.ms_gpu_batch_destroy(self.h)
            self.h = _V()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_info():
    sm, ma, mi = C.c_int(), C.c_int(), C.c_int()
    _check(_lib.ms_gpu_device_info(C.byref(sm), C.byref(ma), C.byref(mi)), "device_info")
    return sm.value, ma.value, mi.value


def size_max_byte_any_len(fmt: Format, n: int) -> int:
    fmt = _fmt(fmt)
    return int(_lib.ms_size_max_byte_any_len(fmt.code, fmt.bw, n))


def rest_offset(fmt: Format, compr: int) -> int:
    fmt = _fmt(fmt)
    return int(_lib.ms_rest_offset(fmt.code, fmt.bw, compr))
