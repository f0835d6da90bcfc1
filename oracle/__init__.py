"""CPU oracle for the compression-aware query path -- TEST INFRASTRUCTURE ONLY.

Two checkers live here:

* ``Oracle``: ctypes wrapper over ``_build/libmsoracle.so``, the plain-C
  restatement of the reference's AVX-512-default layouts and operators
  (``ms_oracle.c``; each function cites the reference file:line it follows).
* ``Reference``: ctypes wrapper over ``_ref/libmsref_<isa>.so``, the
  reference's own codecs and operators compiled from its headers by
  ``Makefile`` (only where the reference source tree is present, i.e. not on
  the GPU box unless the prebuilt library travelled with the repo).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker / CPU baseline.  The
product (``engine_b200``) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "_build", "libmsoracle.so")
REF_DIR = os.path.join(HERE, "_ref")

UNCOMPR, STATIC_VBP, DYNAMIC_VBP, DELTA_DVBP, FOR_DVBP, RLE = range(6)
FORMAT_NAMES = {UNCOMPR: "uncompr", STATIC_VBP: "static_vbp", DYNAMIC_VBP: "dynamic_vbp",
                DELTA_DVBP: "delta_dvbp", FOR_DVBP: "for_dvbp", RLE: "rle"}
CMP_EQ, CMP_LT, CMP_LE, CMP_GT, CMP_GE = range(5)


class Meta(C.Structure):
    _fields_ = [("count_values", C.c_uint64), ("size_used_byte", C.c_uint64),
                ("size_compr_byte", C.c_uint64)]

    def tuple(self):
        return (int(self.count_values), int(self.size_used_byte), int(self.size_compr_byte))


U64P = C.POINTER(C.c_uint64)
U8P = C.POINTER(C.c_uint8)


def _u64(a: np.ndarray):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a, a.ctypes.data_as(U64P)


def _u8(a: np.ndarray):
    a = np.ascontiguousarray(a, dtype=np.uint8)
    return a, a.ctypes.data_as(U8P)


def build(quiet: bool = True) -> None:
    """Compile the C oracle (and nothing else)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


class Oracle:
    """The C restatement of the reference (ms_oracle.c)."""

    def __init__(self, path: str = LIB_ORACLE):
        if not os.path.exists(path):
            build()
        L = self.lib = C.CDLL(path)
        L.orc_size_max_byte_any_len.restype = C.c_uint64
        L.orc_size_max_byte_any_len.argtypes = [C.c_int, C.c_uint, C.c_uint64]
        L.orc_rest_offset.restype = C.c_uint64
        L.orc_rest_offset.argtypes = [C.c_int, C.c_uint, C.c_uint64]
        L.orc_block_size.restype = C.c_uint64
        L.orc_block_size.argtypes = [C.c_int]
        L.orc_compress.argtypes = [C.c_int, C.c_uint, U64P, C.c_uint64, U8P, C.c_uint64, C.POINTER(Meta)]
        L.orc_decompress.argtypes = [C.c_int, C.c_uint, U8P, C.POINTER(Meta), U64P]
        L.orc_wi_write.argtypes = [C.c_int, C.c_uint, U64P, C.c_uint64, C.c_uint64, U8P, C.c_uint64,
                                   C.POINTER(Meta)]
        L.orc_select.restype = C.c_uint64
        L.orc_select.argtypes = [C.c_int, C.c_uint64, U64P, C.c_uint64, C.c_uint64, U64P]
        L.orc_agg_sum.restype = C.c_uint64
        L.orc_agg_sum.argtypes = [U64P, C.c_uint64]
        L.orc_select_project_sum.restype = C.c_uint64
        L.orc_select_project_sum.argtypes = [C.c_int, C.c_uint64, U64P, U64P, C.c_uint64, C.c_uint64, U64P]
        L.orc_semi_join.restype = C.c_uint64
        L.orc_semi_join.argtypes = [U64P, C.c_uint64, U64P, C.c_uint64, U64P]
        L.orc_natural_join.restype = C.c_uint64
        L.orc_natural_join.argtypes = [U64P, C.c_uint64, U64P, C.c_uint64, U64P, U64P]
        L.orc_intersect_sorted.restype = C.c_uint64
        L.orc_intersect_sorted.argtypes = [U64P, C.c_uint64, U64P, C.c_uint64, U64P]
        L.orc_group.restype = C.c_uint64
        L.orc_group.argtypes = [U64P, U64P, C.c_uint64, U64P, U64P]
        L.orc_agg_sum_grouped.argtypes = [U64P, U64P, C.c_uint64, C.c_uint64, U64P]
        L.orc_mix64.restype = C.c_uint64
        L.orc_mix64.argtypes = [C.c_uint64, C.c_uint64]
        L.orc_gen_uniform_bits.argtypes = [C.c_uint64, C.c_uint, C.c_uint64, U64P]
        L.orc_gen_uniform_bits_at.argtypes = [C.c_uint64, C.c_uint, C.c_uint64, C.c_uint64, U64P]
        L.orc_cdf_table_zipf.argtypes = [C.c_double, C.c_uint64, U64P]
        L.orc_cdf_table_geom.restype = C.c_uint64
        L.orc_cdf_table_geom.argtypes = [C.c_double, C.c_uint64, U64P]
        L.orc_gen_from_table.argtypes = [C.c_uint64, U64P, C.c_uint64, C.c_uint64, U64P]
        L.orc_gen_sorted_gaps.argtypes = [C.c_uint64, U64P, C.c_uint64, C.c_uint64, U64P]
        L.orc_gen_runs.argtypes = [C.c_uint64, C.c_uint, C.c_uint, C.c_uint64, U64P]

    # --- layout helpers ---------------------------------------------------
    def size_max_any_len(self, fmt, bw, n):
        return int(self.lib.orc_size_max_byte_any_len(fmt, bw, n))

    def rest_offset(self, fmt, bw, compr):
        return int(self.lib.orc_rest_offset(fmt, bw, compr))

    def block_size(self, fmt):
        return int(self.lib.orc_block_size(fmt))

    def scalar_from(self, fmt, bw, meta):
        """Index where the operator's scalar remainder loop starts
        (select_compr.h:206-250): rest values beyond the last full vector."""
        n, used, compr = meta
        if fmt == RLE:
            raise ValueError("rle_f has no decompress_and_process_batch")
        if n == 0:
            return 0
        if fmt == UNCOMPR:
            nrest = n
        elif compr == used:
            nrest = 0
        else:
            nrest = (used - self.rest_offset(fmt, bw, compr)) // 8
        return n - nrest % 8

    # --- codecs -------------------------------------------------------------
    def compress(self, fmt, bw, values):
        v, vp = _u64(values)
        cap = self.size_max_any_len(fmt, bw, len(v)) + 64
        out = np.zeros(cap, dtype=np.uint8)
        m = Meta()
        rc = self.lib.orc_compress(fmt, bw, vp, len(v), out.ctypes.data_as(U8P), cap, C.byref(m))
        if rc:
            raise ValueError(f"orc_compress rc={rc}")
        return out[: m.size_used_byte].copy(), m.tuple()

    def decompress(self, fmt, bw, data, meta):
        d, dp = _u8(data)
        # the reference's static_vbp readers may touch the gap; pad generously
        pad = np.zeros(len(d) + 64, dtype=np.uint8)
        pad[: len(d)] = d
        m = Meta(*meta)
        out = np.zeros(max(meta[0], 1), dtype=np.uint64)
        rc = self.lib.orc_decompress(fmt, bw, pad.ctypes.data_as(U8P), C.byref(m), out.ctypes.data_as(U64P))
        if rc:
            raise ValueError(f"orc_decompress rc={rc}")
        return out[: meta[0]]

    def wi_write(self, fmt, bw, values, n_scalar=0):
        v, vp = _u64(values)
        n_vec = len(v) - n_scalar
        cap = self.size_max_any_len(fmt, bw, len(v)) + 64
        out = np.zeros(cap, dtype=np.uint8)
        m = Meta()
        rc = self.lib.orc_wi_write(fmt, bw, vp, n_vec, n_scalar, out.ctypes.data_as(U8P), cap, C.byref(m))
        if rc:
            raise ValueError(f"orc_wi_write rc={rc}")
        return out[: m.size_used_byte].copy(), m.tuple()

    # --- operators ----------------------------------------------------------
    def select(self, cmp, val, data, scalar_from=None):
        d, dp = _u64(data)
        sf = len(d) - len(d) % 8 if scalar_from is None else scalar_from
        out = np.zeros(max(len(d), 1), dtype=np.uint64)
        k = self.lib.orc_select(cmp, val, dp, len(d), sf, out.ctypes.data_as(U64P))
        return out[:k].copy()

    def agg_sum(self, data):
        d, dp = _u64(data)
        return int(self.lib.orc_agg_sum(dp, len(d)))

    def select_project_sum(self, cmp, c, x, y, scalar_from=None):
        x, xp = _u64(x)
        y, yp = _u64(y)
        sf = len(x) - len(x) % 8 if scalar_from is None else scalar_from
        cnt = C.c_uint64(0)
        s = self.lib.orc_select_project_sum(cmp, c, xp, yp, len(x), sf, C.byref(cnt))
        return int(s), int(cnt.value)

    def semi_join(self, l, r):
        l, lp = _u64(l)
        r, rp = _u64(r)
        out = np.zeros(max(len(r), 1), dtype=np.uint64)
        k = self.lib.orc_semi_join(lp, len(l), rp, len(r), out.ctypes.data_as(U64P))
        return out[:k].copy()

    def natural_join(self, l, r):
        """(build positions, probe positions) of the natural equi-join."""
        l, lp = _u64(l)
        r, rp = _u64(r)
        ol = np.zeros(max(len(r), 1), dtype=np.uint64)
        orr = np.zeros(max(len(r), 1), dtype=np.uint64)
        k = self.lib.orc_natural_join(lp, len(l), rp, len(r), ol.ctypes.data_as(U64P), orr.ctypes.data_as(U64P))
        return ol[:k].copy(), orr[:k].copy()

    def intersect_sorted(self, l, r):
        l, lp = _u64(l)
        r, rp = _u64(r)
        out = np.zeros(max(min(len(l), len(r)), 1), dtype=np.uint64)
        k = self.lib.orc_intersect_sorted(lp, len(l), rp, len(r), out.ctypes.data_as(U64P))
        return out[:k].copy()

    def group(self, data, gr_in=None):
        d, dp = _u64(data)
        gp = None
        if gr_in is not None:
            g, gp = _u64(gr_in)
        gr = np.zeros(max(len(d), 1), dtype=np.uint64)
        ext = np.zeros(max(len(d), 1), dtype=np.uint64)
        k = self.lib.orc_group(gp, dp, len(d), gr.ctypes.data_as(U64P), ext.ctypes.data_as(U64P))
        return gr[: len(d)].copy(), ext[:k].copy()

    def agg_sum_grouped(self, gr, data, n_groups):
        g, gp = _u64(gr)
        d, dp = _u64(data)
        out = np.zeros(max(n_groups, 1), dtype=np.uint64)
        self.lib.orc_agg_sum_grouped(gp, dp, len(d), n_groups, out.ctypes.data_as(U64P))
        return out[:n_groups]

    # --- generators -----------------------------------------------------------
    def uniform_bits(self, seed, bits, n, row0=0):
        """Rows [row0, row0 + n) of the seeded uniform column."""
        out = np.empty(n, dtype=np.uint64)
        self.lib.orc_gen_uniform_bits_at(seed, bits, row0, n, out.ctypes.data_as(U64P))
        return out

    def zipf_table(self, s, n_vals):
        t = np.empty(n_vals, dtype=np.uint64)
        self.lib.orc_cdf_table_zipf(s, n_vals, t.ctypes.data_as(U64P))
        return t

    def geom_table(self, p, max_len=4096):
        t = np.empty(max_len, dtype=np.uint64)
        k = self.lib.orc_cdf_table_geom(p, max_len, t.ctypes.data_as(U64P))
        return t[:k].copy()

    def from_table(self, seed, table, n):
        t, tp = _u64(table)
        out = np.empty(n, dtype=np.uint64)
        self.lib.orc_gen_from_table(seed, tp, len(t), n, out.ctypes.data_as(U64P))
        return out

    def sorted_gaps(self, seed, gap_table, n):
        t, tp = _u64(gap_table)
        out = np.empty(n, dtype=np.uint64)
        self.lib.orc_gen_sorted_gaps(seed, tp, len(t), n, out.ctypes.data_as(U64P))
        return out

    def runs(self, seed, log2_mean, value_bits, n):
        out = np.empty(n, dtype=np.uint64)
        self.lib.orc_gen_runs(seed, log2_mean, value_bits, n, out.ctypes.data_as(U64P))
        return out


def host_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
        return all(x in flags for x in ("avx512f", "avx512dq", "avx512bw", "avx512vl", "avx512cd"))
    except OSError:
        return False


def reference_path(isa: str | None = None) -> str | None:
    """Path of the compiled reference shim for this host, if it exists."""
    if isa is None:
        isa = "avx512" if host_has_avx512() else "avx2"
    p = os.path.join(REF_DIR, f"libmsref_{isa}.so")
    return p if os.path.exists(p) else None


class Reference:
    """The reference's own codecs/operators (ref_shim.cpp), AVX-512 or AVX2."""

    def __init__(self, path: str):
        L = self.lib = C.CDLL(path)
        M = C.POINTER(Meta)
        L.ref_isa.restype = C.c_int
        L.ref_compress.argtypes = [C.c_int, C.c_uint, U64P, C.c_uint64, U8P, C.c_uint64, M]
        L.ref_decompress.argtypes = [C.c_int, C.c_uint, U8P, M, U64P]
        L.ref_select.argtypes = [C.c_int, C.c_uint64, C.c_int, C.c_uint, U8P, M, C.c_int, C.c_uint, U8P,
                                 C.c_uint64, M]
        L.ref_project.argtypes = [C.c_int, C.c_uint, U8P, M, C.c_int, C.c_uint, U8P, M, C.c_int, C.c_uint,
                                  U8P, C.c_uint64, M]
        L.ref_agg_sum.argtypes = [C.c_int, C.c_uint, U8P, M, U64P]
        L.ref_semi_join.argtypes = [C.c_int, U8P, M, C.c_int, U8P, M, C.c_int, U8P, C.c_uint64, M]
        L.ref_intersect.argtypes = [C.c_int, U8P, M, U64P, C.c_uint64, C.c_int, U8P, C.c_uint64, M]
        L.ref_natural_join.argtypes = [C.c_int, U8P, M, C.c_int, U8P, M, C.c_int, U8P, C.c_uint64, M, U8P,
                                       C.c_uint64, M]
        L.ref_intersect_scalar.restype = C.c_uint64
        L.ref_intersect_scalar.argtypes = [U64P, C.c_uint64, U64P, C.c_uint64, U64P]
        L.ref_group.argtypes = [C.c_int, U8P, M, C.c_int, U8P, C.c_uint64, M, C.c_int, U8P, C.c_uint64, M]
        L.ref_agg_sum_grouped.argtypes = [U64P, U64P, C.c_uint64, C.c_uint64, U64P]
        L.ref_bwi_compress.argtypes = [U64P, C.c_uint64, U8P, U8P, C.c_uint64, U64P]
        L.ref_exhaustive_choose.argtypes = [U64P, C.c_uint64, U8P]
        L.ref_sps_prepare.restype = C.c_void_p
        L.ref_sps_prepare.argtypes = [U64P, U64P, C.c_uint64, U64P]
        L.ref_sps_run.restype = C.c_uint64
        L.ref_sps_run.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(C.c_double), U64P]
        L.ref_sps_free.argtypes = [C.c_void_p]
        L.ref_bench_select_project_sum.restype = C.c_uint64
        L.ref_bench_select_project_sum.argtypes = [U64P, U64P, C.c_uint64, C.c_uint64, C.POINTER(C.c_double),
                                                   U64P, U64P]
        self.isa = int(L.ref_isa())
        self._orc = None

    @staticmethod
    def _padded(data, extra=1 << 16):
        d = np.zeros(len(data) + extra, dtype=np.uint8)
        d[: len(data)] = data
        return d

    def _cap(self, n):
        return 16 * n + (1 << 20)

    def compress(self, fmt, bw, values):
        v, vp = _u64(values)
        cap = self._cap(len(v))
        out = np.zeros(cap, dtype=np.uint8)
        m = Meta()
        rc = self.lib.ref_compress(fmt, bw, vp, len(v), out.ctypes.data_as(U8P), cap, C.byref(m))
        if rc:
            raise ValueError(f"ref_compress rc={rc}")
        return out[: m.size_used_byte].copy(), m.tuple()

    def decompress(self, fmt, bw, data, meta):
        d = self._padded(data)
        m = Meta(*meta)
        out = np.zeros(max(meta[0], 1) + 8, dtype=np.uint64)
        rc = self.lib.ref_decompress(fmt, bw, d.ctypes.data_as(U8P), C.byref(m), out.ctypes.data_as(U64P))
        if rc:
            raise ValueError(f"ref_decompress rc={rc}")
        return out[: meta[0]]

    def select(self, cmp, val, in_fmt, in_bw, data, meta, out_fmt, out_bw=0):
        d = self._padded(data)
        cap = self._cap(meta[0])
        out = np.zeros(cap, dtype=np.uint8)
        m_in, m_out = Meta(*meta), Meta()
        rc = self.lib.ref_select(cmp, val, in_fmt, in_bw, d.ctypes.data_as(U8P), C.byref(m_in), out_fmt, out_bw,
                                 out.ctypes.data_as(U8P), cap, C.byref(m_out))
        if rc:
            raise ValueError(f"ref_select rc={rc}")
        return out[: m_out.size_used_byte].copy(), m_out.tuple()

    def project(self, data_fmt, data_bw, data, dmeta, pos_fmt, pos_bw, pos, pmeta, out_fmt, out_bw=0):
        d = self._padded(data, 1 << 20)
        p = self._padded(pos)
        cap = self._cap(pmeta[0])
        out = np.zeros(cap, dtype=np.uint8)
        md, mp, mo = Meta(*dmeta), Meta(*pmeta), Meta()
        rc = self.lib.ref_project(data_fmt, data_bw, d.ctypes.data_as(U8P), C.byref(md), pos_fmt, pos_bw,
                                  p.ctypes.data_as(U8P), C.byref(mp), out_fmt, out_bw, out.ctypes.data_as(U8P), cap,
                                  C.byref(mo))
        if rc:
            raise ValueError(f"ref_project rc={rc}")
        return out[: mo.size_used_byte].copy(), mo.tuple()

    def agg_sum(self, fmt, bw, data, meta):
        d = self._padded(data)
        s = C.c_uint64(0)
        rc = self.lib.ref_agg_sum(fmt, bw, d.ctypes.data_as(U8P), C.byref(Meta(*meta)), C.byref(s))
        if rc:
            raise ValueError(f"ref_agg_sum rc={rc}")
        return int(s.value)

    def semi_join(self, l_fmt, l, lmeta, r_fmt, r, rmeta, out_fmt):
        lp, rp = self._padded(l), self._padded(r)
        cap = self._cap(rmeta[0])
        out = np.zeros(cap, dtype=np.uint8)
        mo = Meta()
        rc = self.lib.ref_semi_join(l_fmt, lp.ctypes.data_as(U8P), C.byref(Meta(*lmeta)), r_fmt,
                                    rp.ctypes.data_as(U8P), C.byref(Meta(*rmeta)), out_fmt,
                                    out.ctypes.data_as(U8P), cap, C.byref(mo))
        if rc:
            raise ValueError(f"ref_semi_join rc={rc}")
        return out[: mo.size_used_byte].copy(), mo.tuple()

    def natural_join(self, l_fmt, l, lmeta, r_fmt, r, rmeta, out_fmt):
        """join<ve, out, out, L_f, R_f>(L, R): ((bytes, meta) of the build
        positions, (bytes, meta) of the probe positions)."""
        lp, rp = self._padded(l), self._padded(r)
        cap = self._cap(rmeta[0])
        ol = np.zeros(cap, dtype=np.uint8)
        orr = np.zeros(cap, dtype=np.uint8)
        ml, mr = Meta(), Meta()
        rc = self.lib.ref_natural_join(l_fmt, lp.ctypes.data_as(U8P), C.byref(Meta(*lmeta)), r_fmt,
                                       rp.ctypes.data_as(U8P), C.byref(Meta(*rmeta)), out_fmt,
                                       ol.ctypes.data_as(U8P), cap, C.byref(ml), orr.ctypes.data_as(U8P), cap,
                                       C.byref(mr))
        if rc:
            raise ValueError(f"ref_natural_join rc={rc}")
        return (ol[: ml.size_used_byte].copy(), ml.tuple()), (orr[: mr.size_used_byte].copy(), mr.tuple())

    def intersect(self, l_fmt, l, lmeta, r_values, out_fmt):
        lp = self._padded(l)
        r, rptr = _u64(r_values)
        cap = self._cap(lmeta[0])
        out = np.zeros(cap, dtype=np.uint8)
        mo = Meta()
        rc = self.lib.ref_intersect(l_fmt, lp.ctypes.data_as(U8P), C.byref(Meta(*lmeta)), rptr, len(r), out_fmt,
                                    out.ctypes.data_as(U8P), cap, C.byref(mo))
        if rc:
            raise ValueError(f"ref_intersect rc={rc}")
        return out[: mo.size_used_byte].copy(), mo.tuple()

    def intersect_scalar(self, l, r):
        """scalar intersect_sorted (scalar/intersect_uncompr.h:41-86)."""
        l, lp = _u64(l)
        r, rp = _u64(r)
        out = np.zeros(max(min(len(l), len(r)), 1), dtype=np.uint64)
        k = self.lib.ref_intersect_scalar(lp, len(l), rp, len(r), out.ctypes.data_as(U64P))
        return out[:k].copy()

    def group(self, in_fmt, data, meta, gr_fmt, ext_fmt):
        d = self._padded(data)
        cap = self._cap(meta[0])
        gr = np.zeros(cap, dtype=np.uint8)
        ext = np.zeros(cap, dtype=np.uint8)
        mg, me = Meta(), Meta()
        rc = self.lib.ref_group(in_fmt, d.ctypes.data_as(U8P), C.byref(Meta(*meta)), gr_fmt, gr.ctypes.data_as(U8P),
                                cap, C.byref(mg), ext_fmt, ext.ctypes.data_as(U8P), cap, C.byref(me))
        if rc:
            raise ValueError(f"ref_group rc={rc}")
        return (gr[: mg.size_used_byte].copy(), mg.tuple()), (ext[: me.size_used_byte].copy(), me.tuple())

    def agg_sum_grouped(self, gr, data, n_groups):
        g, gp = _u64(gr)
        d, dp = _u64(data)
        out = np.zeros(max(n_groups, 1), dtype=np.uint64)
        self.lib.ref_agg_sum_grouped(gp, dp, len(d), n_groups, out.ctypes.data_as(U64P))
        return out[:n_groups]

    def bwi_compress(self, values, codes):
        """The reference's blockwise_individual_f<2048, …> container of
        len(values)/2048 blocks, block b in the format with code codes[b]
        (bytes as written; padding and for_f's unwritten header words are
        zero here because the shim compresses into a zeroed buffer)."""
        v, vp = _u64(values)
        nblk = len(v) // 2048
        c, cp = _u8(codes)
        cap = 16 * len(v) + 128 * nblk + 4096
        out = np.zeros(cap, dtype=np.uint8)
        nb = C.c_uint64(0)
        rc = self.lib.ref_bwi_compress(vp, nblk, cp, out.ctypes.data_as(U8P), cap, C.byref(nb))
        if rc:
            raise ValueError(f"ref_bwi_compress rc={rc}")
        return out[: nb.value].copy()

    def exhaustive_choose(self, values):
        """The reference's exhaustive_size_format_selector's format code per
        2048-value block (candidates: uncompr, static_vbp at the block's width,
        dynamic_vbp, group_simple and the delta / for cascades over both)."""
        v, vp = _u64(values)
        nblk = len(v) // 2048
        out = np.zeros(max(nblk, 1), dtype=np.uint8)
        if self.lib.ref_exhaustive_choose(vp, nblk, out.ctypes.data_as(U8P)):
            raise MemoryError("ref_exhaustive_choose")
        return out[:nblk]

    def sps_prepare(self, x, y):
        """Compress x and y (dynamic_vbp) with the reference and keep them:
        (handle, compressed bytes)."""
        x, xp = _u64(x)
        y, yp = _u64(y)
        cb = C.c_uint64(0)
        h = self.lib.ref_sps_prepare(xp, yp, len(x), C.byref(cb))
        return h, int(cb.value)

    def sps_run(self, handle, c):
        """select(x < c) -> project(y) -> agg_sum on a prepared pair:
        (sum, count, operator seconds)."""
        secs = C.c_double(0)
        cnt = C.c_uint64(0)
        s = self.lib.ref_sps_run(handle, c, C.byref(secs), C.byref(cnt))
        return int(s), int(cnt.value), float(secs.value)

    def sps_free(self, handle):
        self.lib.ref_sps_free(handle)

    def bench_select_project_sum(self, x, y, c):
        x, xp = _u64(x)
        y, yp = _u64(y)
        secs = C.c_double(0)
        cnt = C.c_uint64(0)
        cb = C.c_uint64(0)
        s = self.lib.ref_bench_select_project_sum(xp, yp, len(x), c, C.byref(secs), C.byref(cnt), C.byref(cb))
        return int(s), int(cnt.value), float(secs.value), int(cb.value)


def mask_gap(fmt: int, bw: int, data: np.ndarray, meta, oracle: Oracle) -> np.ndarray:
    """Bytes that carry meaning: the gap between the compressed part and the
    uncompressed rest (never written by the reference, column.h:186-195) and
    the FOR header words after an end marker (for.h:214-220) are zeroed."""
    d = np.array(data, dtype=np.uint8, copy=True)
    n, used, compr = meta
    if fmt not in (UNCOMPR, RLE) and used > compr:
        d[compr: oracle.rest_offset(fmt, bw, compr)] = 0
    if fmt == FOR_DVBP and compr:
        _mask_for_headers(d, compr)
    return d


def _mask_for_headers(d: np.ndarray, compr: int) -> None:
    """Walk the for_f pages and zero header words after a UINT64_MAX marker."""
    i = 0
    while i < compr:
        h0 = i
        hdr = d[i: i + 64].view(np.uint64).copy()
        i += 64
        for j in range(8):
            if int(hdr[j]) == 0xFFFFFFFFFFFFFFFF:
                d[h0 + 8 * (j + 1): h0 + 64] = 0
                break
            # inner dvbp page of one 1024-block: 64-B header + two packed blocks
            bws = d[i: i + 2]
            i += 64 + 64 * (int(bws[0]) + int(bws[1]))
