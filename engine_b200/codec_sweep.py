"""Codec round-trip sweep on the GPU (uncompr <-> every format).

Every case compresses n uint64 values generated on the device, decompresses
them again and checks the round trip on the device; times are CUDA events
around the public morph call (which includes its size read-back).
Distributions: uniform over b bits, Zipf(1.2) over [0, 2^20), sorted with
geometric gaps of mean 4, runs with geometric lengths of mean 32 (run values
uniform over 20 bits).

    python -m engine_b200.codec_sweep [log2_n] [out.json]
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    sys.path.insert(0, os.path.dirname(HERE))
    import torch

    import engine_b200 as ms
    from engine_b200.datagen import geom_table, zipf_table
    log2n = int(sys.argv[1]) if len(sys.argv) > 1 else 28
    out_path = sys.argv[2] if len(sys.argv) > 2 else None
    n = 1 << log2n
    lib = ms.lib()
    arena = ms.Arena(24 << 30)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    zipf = zipf_table(1.2, 1 << 20)
    geo = geom_table(0.25)
    d_zipf = arena.alloc(zipf.nbytes)
    ms._memcpy_h2d(d_zipf, zipf)
    d_geo = arena.alloc(geo.nbytes)
    ms._memcpy_h2d(d_geo, geo)
    base = arena.used()

    def make(dist, seed):
        d = arena.alloc(8 * n)
        if dist.startswith("uniform"):
            ms._check(lib.ms_gpu_gen_uniform_bits(seed, int(dist[7:]), n, d, sp), "gen")
        elif dist == "zipf":
            ms._check(lib.ms_gpu_gen_from_table(seed, d_zipf, len(zipf), n, d, sp), "gen")
        elif dist == "sorted":
            ms._check(lib.ms_gpu_gen_sorted_gaps(seed, d_geo, len(geo), n, d, arena.h, sp), "gen")
        else:
            ms._check(lib.ms_gpu_gen_runs(seed, 5, 20, n, d, arena.h, sp), "gen")
        return ms.MsCol(format=0, count_values=n, size_used_byte=8 * n, size_alloc_byte=8 * n, data=d)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    cases = [("uniform%d" % b, ms.STATIC_VBP, b) for b in range(1, 65)]
    for dist in ("uniform8", "uniform16", "uniform20", "uniform32", "uniform64", "zipf", "sorted", "runs"):
        for fmt in (ms.DYNAMIC_VBP, ms.DELTA_DVBP, ms.FOR_DVBP, ms.RLE):
            cases.append((dist, fmt, 0))
    results = []
    for dist, fmt, bw in cases:
        ms._check(lib.ms_gpu_arena_reset(arena.h), "reset")
        arena.alloc(base)
        u = make(dist, 0x5EED + bw)
        torch.cuda.synchronize()
        c = ms.MsCol()
        e0, e1, e2 = ev(), ev(), ev()
        e0.record(stream)
        ms._check(lib.ms_gpu_morph(C.byref(u), fmt, bw, C.byref(c), arena.h, sp), "compress")
        e1.record(stream)
        d = ms.MsCol()
        ms._check(lib.ms_gpu_morph(C.byref(c), ms.UNCOMPR, 0, C.byref(d), arena.h, sp), "decompress")
        e2.record(stream)
        torch.cuda.synchronize()
        tc, td = e0.elapsed_time(e1), e1.elapsed_time(e2)
        a = ms._device_view(u.data, 8 * n)
        b = ms._device_view(d.data, 8 * n)
        ok = bool(torch.equal(a, b))
        cb = int(c.size_used_byte)
        r = {"dist": dist, "format": {1: "static_vbp", 2: "dynamic_vbp", 3: "delta+dvbp", 4: "for+dvbp",
                                      5: "rle"}[fmt] + (f"<{bw}>" if bw else ""),
             "bytes": cb, "bits_per_value": round(8 * cb / n, 3), "compress_ms": round(tc, 3),
             "decompress_ms": round(td, 3), "compress_gbs": round((8 * n + cb) / tc / 1e6, 1),
             "decompress_gbs": round((8 * n + cb) / td / 1e6, 1), "roundtrip_ok": ok}
        results.append(r)
        print(json.dumps(r), flush=True)
    summary = {"n": n, "cases": len(results), "all_roundtrips_ok": all(r["roundtrip_ok"] for r in results),
               "results": results}
    if out_path:
        with open(out_path, "w") as f:
            json.dump(summary, f, indent=1)
    arena.close()
    return 0 if summary["all_roundtrips_ok"] else 1


if __name__ == "__main__":
    sys.exit(main())
