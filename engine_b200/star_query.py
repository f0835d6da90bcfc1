"""Star query over a compressed fact table on one GPU.

Fact table of n rows with four uint64 columns -- a foreign key uniform in
[0, 2^20), a filter uniform in [0, 2^12), a group key Zipf(1.1) over 1000
values and a measure uniform in [0, 2^16) -- each stored in the smallest of
dynamic_vbp, for+dynamic_vbp and delta+dynamic_vbp; a dimension of 2^20
sorted unique keys filtered to ~10% (delta+dynamic_vbp).  The query is

    select(filter < 400) -> semi_join(dim keys, fk) -> intersect ->
    project(group key, measure) -> group -> grouped sum

run two ways: the fused one-pass kernel (``query3``) and the operators one
at a time with every intermediate recompressed (positions delta+dvbp,
projected columns dynamic_vbp).  Both results are checked against a torch
computation on the uncompressed columns.  GB/s counts the compressed bytes
of the five input columns.

    python -m engine_b200.star_query [log2_rows] [reps] [--sweep]
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SEED = 0x5A17
FILTER_LT = 400
DIM_KEYS = 1 << 20


# staged=1 keeps the build side's bitmap in shared memory when it fits beside
# the ring, staged=2 always reads it from global memory, staged=3 splits it
# over a 2-CTA cluster.  The small rings leave part of the SM's unified
# L1/shared memory to L1, which can then hold the bitmap's hot lines.
QUERY_CONFIGS = ([dict(staged=0)] +
                 [dict(staged=st, warps=w, stages=s, stage_bytes=b)
                  for st in (1, 2) for w in (8, 16, 24)
                  for s, b in ((2, 81920), (3, 57344), (4, 40960), (6, 27648))] +
                 [dict(staged=2, warps=w, stages=s, stage_bytes=b)
                  for w in (16, 24) for s, b in ((2, 40960), (3, 24576), (2, 28672), (4, 16384))] +
                 [dict(staged=3, warps=16, stages=3, stage_bytes=57344)])


def run(log2_rows: int = 28, reps: int = 5, sweep: bool = False) -> dict:
    """sweep: time the fused query under every launch configuration in
    QUERY_CONFIGS and keep the fastest (reported under "sweep")."""
    import torch

    import engine_b200 as ms
    from engine_b200.datagen import zipf_table
    lib = ms.lib()
    n = 1 << log2_rows
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    arena = ms.Arena(40 << 30)
    try:
        zipf = zipf_table(1.1, 1000)
        d_zipf = arena.alloc(zipf.nbytes)
        ms._memcpy_h2d(d_zipf, zipf)

        def uncompr(ptr, count):
            return ms.MsCol(format=ms.UNCOMPR, count_values=count, size_used_byte=8 * count,
                            size_alloc_byte=8 * count, data=ptr)

        raw = {}
        for name, gen in (("fk", lambda d: lib.ms_gpu_gen_uniform_bits(SEED, 20, n, d, sp)),
                          ("filter", lambda d: lib.ms_gpu_gen_uniform_bits(SEED + 1, 12, n, d, sp)),
                          ("gkey", lambda d: lib.ms_gpu_gen_from_table(SEED + 2, d_zipf, len(zipf), n, d, sp)),
                          ("measure", lambda d: lib.ms_gpu_gen_uniform_bits(SEED + 3, 16, n, d, sp))):
            d = arena.alloc(8 * n)
            ms._check(gen(d), "gen " + name)
            raw[name] = d
        keep = np.random.default_rng(SEED).random(DIM_KEYS) < 0.1
        dim = np.flatnonzero(keep).astype(np.uint64)
        d_dim = arena.alloc(8 * len(dim))
        ms._memcpy_h2d(d_dim, dim)

        def best(col):
            """The smallest of dynamic_vbp, for+dvbp and delta+dvbp."""
            out = []
            for f in (ms.DYNAMIC_VBP, ms.FOR_DVBP, ms.DELTA_DVBP):
                c = ms.MsCol()
                ms._check(lib.ms_gpu_morph(C.byref(col), f, 0, C.byref(c), arena.h, sp), "morph")
                out.append(c)
            return min(out, key=lambda c: int(c.size_used_byte))

        comp = {k: best(uncompr(v, n)) for k, v in raw.items()}
        comp["dim"] = best(uncompr(d_dim, len(dim)))
        names = {ms.DYNAMIC_VBP: "dynamic_vbp", ms.FOR_DVBP: "for+dvbp", ms.DELTA_DVBP: "delta+dvbp"}
        in_bytes = sum(int(c.size_used_byte) for c in comp.values())

        # expected result from the uncompressed columns (torch, on the device)
        t = {k: ms._device_view(v, 8 * n).view(torch.int64) for k, v in raw.items()}
        in_dim = torch.zeros(DIM_KEYS, dtype=torch.bool, device=t["fk"].device)
        in_dim[torch.from_numpy(dim.astype(np.int64)).to(in_dim.device)] = True
        rows = torch.nonzero((t["filter"] < FILTER_LT) & in_dim[t["fk"]]).flatten()
        g, m = t["gkey"][rows], t["measure"][rows]
        uniq, inv = torch.unique(g, return_inverse=True)
        first = torch.full((len(uniq),), len(rows), dtype=torch.int64, device=g.device)
        first.scatter_reduce_(0, inv, torch.arange(len(rows), device=g.device), reduce="amin")
        sums = torch.zeros(len(uniq), dtype=torch.int64, device=g.device).index_add_(0, inv, m)
        order = torch.argsort(first)
        exp = (uniq[order].cpu().numpy().astype(np.uint64), first[order].cpu().numpy().astype(np.uint64),
               sums[order].cpu().numpy().astype(np.uint64), int(len(rows)))
        del t, in_dim, rows, g, m, uniq, inv, first, sums, order
        torch.cuda.empty_cache()

        cols = {k: ms.Column(v, arena) for k, v in comp.items()}
        mark = arena.used()

        def fused():
            ms._check(lib.ms_gpu_arena_reset(arena.h), "reset")
            arena.alloc(mark)
            return ms.query3(cols["filter"], ms.less, FILTER_LT, cols["fk"], cols["dim"], cols["gkey"],
                             cols["measure"], stream=stream)

        def pipeline():
            ms._check(lib.ms_gpu_arena_reset(arena.h), "reset")
            arena.alloc(mark)
            p1 = ms.select(ms.less, cols["filter"], FILTER_LT, ms.delta_f, stream=stream)
            p2 = ms.semi_join(cols["dim"], cols["fk"], ms.uncompr_f, stream=stream)
            p = ms.intersect_sorted(p1, p2, ms.delta_f, stream=stream)
            gk = ms.project(cols["gkey"], p, ms.dynamic_vbp_f, stream=stream)
            me = ms.project(cols["measure"], p, ms.dynamic_vbp_f, stream=stream)
            gr, ext = ms.group(gk, stream=stream)
            s = ms.agg_sum_grouped(gr, me, ext.get_count_values(), stream=stream)
            e = ext.to_numpy()
            return (gk.to_numpy()[e.astype(np.int64)], e, s.to_numpy(), p.get_count_values())

        pass_ms = []  # fact-table pass of each timed fused call

        def timed(fn):
            res = fn()
            torch.cuda.synchronize()
            best_ms, tot = 1e30, 0.0
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                t0 = time.perf_counter()
                e0.record(stream)
                fn()
                e1.record(stream)
                torch.cuda.synchronize()
                wall = (time.perf_counter() - t0) * 1e3
                dt = max(e0.elapsed_time(e1), wall)
                best_ms, tot = min(best_ms, dt), tot + dt
                if fn is fused:
                    pass_ms.append(ms.query3_last_pass_ms())
            return res, tot / reps, best_ms

        def same(a, b):
            return (all(np.array_equal(x, y) for x, y in zip(a[:3], b[:3])) and a[3] == b[3])

        swept = None
        if sweep:
            swept = []
            for cfg in QUERY_CONFIGS:
                ms.set_query_tuning(**cfg)
                pass_ms.clear()
                r, t_mean, t_best = timed(fused)
                swept.append(dict(cfg, best_ms=round(t_best, 3), pass_best_ms=round(min(pass_ms), 4),
                                  ok=bool(same(r, exp))))
            fastest = min((c for c in swept if c["ok"]), key=lambda c: c["best_ms"])
            ms.set_query_tuning(**{k: v for k, v in fastest.items() if k in ("staged", "warps", "stages",
                                                                               "stage_bytes")})
        pass_ms.clear()
        rf, f_ms, f_best = timed(fused)
        k_best, k_mean = min(pass_ms), sum(pass_ms) / len(pass_ms)
        rp, p_ms, p_best = timed(pipeline)
        return {
            "launch": ms.get_query_tuning(), "sweep": swept,
            "workload": "star query, 2^%d fact rows (fk U[0,2^20), filter U[0,2^12), group key Zipf(1.1) over "
                        "1000, measure U[0,2^16)); dimension 2^20 sorted keys filtered to 10%%; "
                        "select(filter < 400) -> semi_join -> group -> sum" % log2_rows,
            "formats": {k: names[int(c.format)] for k, c in comp.items()},
            "compressed_input_bytes": in_bytes,
            "groups": len(rf[0]), "rows_selected": rf[3],
            "fused": {"ms": round(f_ms, 3), "best_ms": round(f_best, 3),
                      "gbs": round(in_bytes / (f_best * 1e-3) / 1e9, 1),
                      "pass": {"ms": round(k_mean, 4), "best_ms": round(k_best, 4),
                               "gbs": round(in_bytes / (k_best * 1e-3) / 1e9, 1),
                               "what": "the fact-table pass alone (staged kernel + direct kernel for the rest), "
                                       "CUDA events inside the call"}},
            "operator_at_a_time": {"ms": round(p_ms, 3), "best_ms": round(p_best, 3),
                                   "gbs": round(in_bytes / (p_best * 1e-3) / 1e9, 1),
                                   "intermediates": "positions delta+dvbp, projections dynamic_vbp"},
            "speedup_fused": round(p_best / f_best, 2),
            "bit_exact": bool(same(rf, exp) and same(rp, exp)),
            "timing": "CUDA events and host wall clock around the public call (max of the two); "
                      "includes the result read-back",
        }
    finally:
        arena.close()


def main():
    sys.path.insert(0, os.path.dirname(HERE))
    log2 = int(sys.argv[1]) if len(sys.argv) > 1 else 28
    reps = int(sys.argv[2]) if len(sys.argv) > 2 else 5
    r = run(log2, reps, sweep="--sweep" in sys.argv)
    print(json.dumps(r), flush=True)
    return 0 if r["bit_exact"] else 1


if __name__ == "__main__":
    sys.exit(main())
