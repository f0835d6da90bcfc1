"""Autotuner for the fused decode kernels.

For a workload (the fused select -> project -> sum over two device columns)
it times every candidate launch configuration -- direct-load kernel, or the
TMA-staged pipeline with W consumer warps, S stages of B bytes and C CTAs per
SM -- with CUDA events on the launching stream, and keeps the fastest.  The
result is stored per format class in ``tuning.json`` beside this file, keyed
by "<x format>/<y format>/<sm count>", and applied with
``engine_b200.set_tuning`` by ``apply()``.

    python -m engine_b200.autotune            # tunes the 2^28-row dynamic_vbp workload
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


def _fmt_name(code: int, bw: int) -> str:
    return {0: "uncompr", 1: f"static_vbp{bw}", 2: "dynamic_vbp", 3: "delta", 4: "for", 5: "rle"}[code]


def key(x, y, sm: int) -> str:
    return f"{_fmt_name(x.format, x.bw)}/{_fmt_name(y.format, y.bw)}/{sm}"


def time_config(ms, xc, yc, cfg, reps=10, pred=512):
    """Average device time (ms) of one fused launch under cfg."""
    import torch
    lib = ms.lib()
    ms.set_tuning(**cfg)
    stream = torch.cuda.current_stream()
    a = ms.default_arena()
    d_sum, d_cnt, d_err = a.alloc(8), a.alloc(8), a.alloc(8)

    def launch():
        ms._check(lib.ms_gpu_select_project_sum_async(C.byref(xc), ms.less, pred, C.byref(yc), d_sum, d_cnt, d_err,
                                                      stream.cuda_stream), "sps")

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


def tune(ms, xc, yc, candidates=CANDIDATES, reps=10, verbose=True):
    sm = ms.device_info()[0]
    results = []
    ref_sum = None
    for cfg in candidates:
        t, s = time_config(ms, xc, yc, cfg, reps)
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


def apply(ms, xc, yc) -> bool:
    """Set the tuned configuration for this workload's format class, if any."""
    entry = load_cache().get(key(xc, yc, ms.device_info()[0]))
    if not entry:
        return False
    ms.set_tuning(**{k: entry[k] for k in ("staged", "warps", "stages", "stage_bytes", "ctas_per_sm",
                                            "values_per_thread") if k in entry})
    return True


def main():
    sys.path.insert(0, os.path.dirname(HERE))
    import engine_b200 as ms
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
