"""Autotuner for the fused decode kernels, per format and bit width.

For a workload (the fused select -> project -> sum over two device columns)
it times every candidate launch configuration -- direct-load kernel, or the
TMA-staged pipeline with W consumer warps, S stages of B bytes and C CTAs per
SM, 16 or 32 values per thread -- with CUDA events on the launching stream,
and keeps the fastest.  Results are stored in ``tuning.json`` beside this
file, keyed by "<x format>:<x width class>/<y format>:<y width class>/<sm
count>"; the width class of a column is the bucket (1-8, 9-16, 17-24, 25-32,
33-64 bits) of its mean bits per value in the compressed part (a static_vbp
column's width; a dynamic_vbp-family column's compressed bits per row).
``apply()`` sets the entry of a workload's formats and classes, else the
nearest class of the same formats, with ``engine_b200.set_tuning``.

    python -m engine_b200.autotune               # the 2^28-row dynamic_vbp workload
    python -m engine_b200.autotune --grid [log2] # every format x width class (x and y alike)
"""
from __future__ import annotations

import ctypes as C
import itertools
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CACHE = os.path.join(HERE, "tuning.json")

CANDIDATES = [dict(staged=0, warps=8, stages=8, stage_bytes=24576, ctas_per_sm=1, values_per_thread=16)] + [
    dict(staged=1, warps=w, stages=s, stage_bytes=b, ctas_per_sm=1, values_per_thread=v)
    for v, w, s, b in itertools.product((16, 32), (12, 16, 20, 24), (3, 4, 6), (24576, 32768, 49152, 65536))
    if s * b <= 200 * 1024
]


CLASSES = ((1, 8), (9, 16), (17, 24), (25, 32), (33, 64))


def _fmt_name(code: int) -> str:
    return {0: "uncompr", 1: "static_vbp", 2: "dynamic_vbp", 3: "delta", 4: "for", 5: "rle"}[code]


def width_class(c) -> int:
    """Index into CLASSES of a column's mean bits per value in its compressed
    part (uncompressed columns: 64 bits)."""
    if c.format == 0:
        bits = 64.0
    elif c.format == 1:
        bits = float(c.bw)
    else:
        n = int(c.count_values)
        nrest = 0
        if int(c.size_used_byte) > int(c.size_compr_byte) and c.format != 5:
            nrest = n % (1024 if c.format in (3, 4) else 512)
        bits = 8.0 * int(c.size_compr_byte) / max(1, n - nrest)
    for i, (lo, hi) in enumerate(CLASSES):
        if bits <= hi + 0.999:
            return i
    return len(CLASSES) - 1


def _side(c) -> str:
    lo, hi = CLASSES[width_class(c)]
    return f"{_fmt_name(c.format)}:{lo}-{hi}"


def key(x, y, sm: int) -> str:
    return f"{_side(x)}/{_side(y)}/{sm}"


def time_config(ms, xc, yc, cfg, reps=10, pred=512):
    """Average device time (ms) of one fused launch under cfg."""
    import torch
    lib = ms.lib()
    ms.set_tuning(**cfg)
    stream = torch.cuda.current_stream()
    a = ms.default_arena()
    d_sum, d_cnt, d_err = a.alloc(8), a.alloc(8), a.alloc(8)

    if 3 in (xc.format, yc.format):  # delta_f: the allocating entry prepares the carries every call
        mark = a.used()

        def launch():
            ms._check(lib.ms_gpu_arena_reset(a.h), "reset")
            a.alloc(mark)
            ms._check(lib.ms_gpu_select_project_sum(C.byref(xc), ms.less, pred, C.byref(yc), d_sum, d_cnt, None,
                                                    None, a.h, stream.cuda_stream), "sps")
    else:
        def launch():
            ms._check(lib.ms_gpu_select_project_sum_async(C.byref(xc), ms.less, pred, C.byref(yc), d_sum, d_cnt,
                                                          d_err, stream.cuda_stream), "sps")

    for _ in range(3):
        launch()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        launch()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps, int(ms._memcpy_d2h(d_sum, 8).view("uint64")[0])


def tune(ms, xc, yc, candidates=CANDIDATES, reps=10, verbose=True, pred=512):
    sm = ms.device_info()[0]
    results = []
    ref_sum = None
    for cfg in candidates:
        t, s = time_config(ms, xc, yc, cfg, reps, pred)
        if ref_sum is None:
            ref_sum = s
        ok = s == ref_sum
        results.append((t, cfg, ok))
        if verbose:
            print(f"{t * 1e3:9.1f} us  {'ok ' if ok else 'BAD'} {cfg}", flush=True)
    best = min((r for r in results if r[2]), key=lambda r: r[0])
    k = key(xc, yc, sm)
    cache = load_cache()
    cache[k] = dict(best[1], us=round(best[0] * 1e3, 1))
    with open(CACHE, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    ms.set_tuning(**best[1])
    return best, results


def load_cache() -> dict:
    try:
        with open(CACHE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def lookup(xc, yc, sm: int, cache: dict | None = None):
    """(key used, entry) for a workload: its own key, else the nearest width
    classes (by summed class distance) of the same formats, else None."""
    cache = load_cache() if cache is None else cache
    k = key(xc, yc, sm)
    if k in cache:
        return k, cache[k]
    fx, fy = _fmt_name(xc.format), _fmt_name(yc.format)
    cx, cy = width_class(xc), width_class(yc)
    best = None
    for kk, entry in cache.items():
        parts = kk.split("/")
        if len(parts) != 3 or parts[2] != str(sm) or ":" not in parts[0] or ":" not in parts[1]:
            continue
        (gx, wx), (gy, wy) = parts[0].split(":"), parts[1].split(":")
        if gx != fx or gy != fy:
            continue
        ix = [f"{lo}-{hi}" for lo, hi in CLASSES].index(wx)
        iy = [f"{lo}-{hi}" for lo, hi in CLASSES].index(wy)
        d = abs(ix - cx) + abs(iy - cy)
        if best is None or d < best[0]:
            best = (d, kk, entry)
    return (best[1], best[2]) if best else (None, None)


def apply(ms, xc, yc) -> bool:
    """Set the tuned configuration for this workload (its formats and width
    classes, or the nearest classes tuned), if any."""
    _, entry = lookup(xc, yc, ms.device_info()[0])
    if not entry:
        return False
    ms.set_tuning(**{k: entry[k] for k in ("staged", "warps", "stages", "stage_bytes", "ctas_per_sm",
                                            "values_per_thread") if k in entry})
    return True


GRID_FORMATS = ((1, "static_vbp"), (2, "dynamic_vbp"), (4, "for"), (3, "delta"))
GRID_WIDTHS = (4, 12, 20, 28, 40)  # uniform inputs, one per width class
GRID_GAPS = (0.25, 1 / 64)         # delta columns: sorted, gaps 1 + Geom(p) (means 4 and 64)


def _grid_column(ms, lib, arena, code, param, seed, n):
    from engine_b200.datagen import geom_table
    u = arena.alloc(8 * n)
    if code == 3:
        t = geom_table(param)
        dt = arena.alloc(t.nbytes)
        ms._memcpy_h2d(dt, t)
        ms._check(lib.ms_gpu_gen_sorted_gaps(seed, dt, len(t), n, u, arena.h, None), "gen")
    else:
        ms._check(lib.ms_gpu_gen_uniform_bits(seed, param, n, u, None), "gen")
    uc = ms.MsCol(format=0, count_values=n, size_used_byte=8 * n, size_alloc_byte=8 * n, data=u)
    c = ms.MsCol()
    ms._check(lib.ms_gpu_morph(C.byref(uc), code, param if code == 1 else 0, C.byref(c), arena.h, None), "morph")
    return c


def grid(log2_rows: int = 26, reps: int = 8):
    """Tune every format x width class with x and y alike: uniform inputs over
    b bits with select x < 2^(b-1), delta columns sorted with geometric gaps
    and select x < 2^62 (every row)."""
    sys.path.insert(0, os.path.dirname(HERE))
    import engine_b200 as ms
    n = 1 << log2_rows
    arena = ms.Arena(8 << 30)
    ms._default_arena = arena
    lib = ms.lib()
    out = {}
    for code, name in GRID_FORMATS:
        for param in (GRID_GAPS if code == 3 else GRID_WIDTHS):
            ms._check(lib.ms_gpu_arena_reset(arena.h), "reset")
            x = _grid_column(ms, lib, arena, code, param, 0x7E57, n)
            y = _grid_column(ms, lib, arena, code, param, 0x7E58, n)
            pred = (1 << 62) if code == 3 else (1 << (param - 1))
            best, _ = tune(ms, x, y, reps=reps, verbose=False, pred=pred)
            k = key(x, y, ms.device_info()[0])
            nbytes = int(x.size_used_byte) + int(y.size_used_byte)
            out[k] = dict(best[1], us=round(best[0] * 1e3, 1), gbs=round(nbytes / best[0] / 1e6, 1))
            print(json.dumps({k: out[k]}), flush=True)
    arena.close()
    return out


def main():
    sys.path.insert(0, os.path.dirname(HERE))
    import engine_b200 as ms
    if "--grid" in sys.argv:
        rest = [a for a in sys.argv[1:] if a != "--grid"]
        grid(int(rest[0]) if rest else 26)
        return
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 1 << 28
    arena = ms.Arena(16 << 30)
    ms._default_arena = arena
    lib = ms.lib()
    xu, yu = arena.alloc(8 * n), arena.alloc(8 * n)
    ms._check(lib.ms_gpu_gen_uniform_bits(0x5EED0001, 10, n, xu, None), "gen")
    ms._check(lib.ms_gpu_gen_uniform_bits(0x5EED0002, 20, n, yu, None), "gen")
    cols = []
    for p in (xu, yu):
        u = ms.MsCol(format=0, count_values=n, size_used_byte=8 * n, size_alloc_byte=8 * n, data=p)
        c = ms.MsCol()
        ms._check(lib.ms_gpu_morph(C.byref(u), ms.DYNAMIC_VBP, 0, C.byref(c), arena.h, None), "morph")
        cols.append(c)
    nbytes = cols[0].size_used_byte + cols[1].size_used_byte
    best, _ = tune(ms, cols[0], cols[1])
    print(f"best {best[1]}: {best[0] * 1e3:.1f} us = {nbytes / best[0] / 1e6:.1f} GB/s")


if __name__ == "__main__":
    main()
