"""Batched persistent execution over many columns on one GPU.

4096 uint64 columns with log-uniform lengths in [2^10, 2^24] (seeded), each
in a seeded random format -- static_vbp with bit width 4..32 (uniform
values of that width), dynamic_vbp (uniform values of 4..32 bits),
delta+dynamic_vbp (sorted, geometric gaps of mean 4), for+dynamic_vbp
(2^40 + uniform 16-bit) or rle (runs of geometric length, mean 32, 20-bit
values).  Every column runs decompress -> select(value < median) -> sum of
the selected values:

* batched: one persistent launch off the device work queue, replayed from a
  CUDA graph, launch configuration from the autotuner (``tune``);
* per column: one operator call per column through the public API
  (``ms_gpu_select_project_sum``; rle columns are decompressed first).

Both are checked against torch on the uncompressed columns (count and sum
per column).  GB/s counts the compressed bytes of all columns.

    python -m engine_b200.batch_bench [n_columns] [steps] [--tune] [--kinds] [--no-per-column]

--kinds also runs one batch per format (the same columns, grouped by kind),
times each under the global configuration and under every candidate, and
stores each kind's best as "batch:<kind>/<sm count>" in tuning.json.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SEED = 0xBA7C
KINDS = ("static", "dvbp", "delta", "for", "rle")
TUNE_CONFIGS = [dict(warps=w, stages=s, stage_bytes=b, ctas_per_sm=c)
                for w in (4, 8, 12, 16) for s in (2, 3, 4) for b in (4096, 8192, 16384) for c in (1, 2)]
_CFG_KEYS = ("warps", "stages", "stage_bytes", "ctas_per_sm")


def _shm(cfg):
    meta = (8 * cfg["stages"] + 176 * cfg["stages"] + 127) // 128 * 128
    return cfg["warps"] * (meta + cfg["stages"] * cfg["stage_bytes"])


def plan_columns(n_cols: int, lo: int = 10, hi: int = 24, seed: int = SEED):
    """(length, kind, bits) per column, seeded."""
    rng = np.random.default_rng(seed)
    lens = np.floor(2.0 ** rng.uniform(lo, hi, n_cols)).astype(np.int64)
    kinds = rng.integers(0, len(KINDS), n_cols)
    bits = rng.integers(4, 33, n_cols)
    return [(int(n), KINDS[int(k)], int(b)) for n, k, b in zip(lens, kinds, bits)]


def build(ms, arena, scratch, plan, stream):
    """Generate, compress (into scratch, then compacted into `arena`) and
    describe every column; returns (columns, medians, expected counts,
    expected sums)."""
    import torch
    from engine_b200.datagen import geom_table
    lib = ms.lib()
    sp = stream.cuda_stream
    geo = geom_table(0.25)
    d_geo = arena.alloc(geo.nbytes)
    ms._memcpy_h2d(d_geo, geo)
    base = scratch.used()
    cols, meds, e_cnt, e_sum = [], [], [], []
    for i, (n, kind, bits) in enumerate(plan):
        ms._check(lib.ms_gpu_arena_reset(scratch.h), "reset")
        scratch.alloc(base)
        d = scratch.alloc(8 * n)
        seed = SEED * 7919 + i
        if kind in ("static", "dvbp"):
            ms._check(lib.ms_gpu_gen_uniform_bits(seed, bits, n, d, sp), "gen")
        elif kind == "delta":
            ms._check(lib.ms_gpu_gen_sorted_gaps(seed, d_geo, len(geo), n, d, scratch.h, sp), "gen")
        elif kind == "for":
            ms._check(lib.ms_gpu_gen_uniform_bits(seed, 16, n, d, sp), "gen")
        else:
            ms._check(lib.ms_gpu_gen_runs(seed, 5, 20, n, d, scratch.h, sp), "gen")
        t = ms._device_view(d, 8 * n).view(torch.int64)
        if kind == "for":
            t += 1 << 40
        med = int(torch.kthvalue(t, n // 2 + 1).values.item())
        hit = t < med
        e_cnt.append(int(hit.sum().item()))
        e_sum.append(int(torch.where(hit, t, torch.zeros_like(t)).sum().item()) & ((1 << 64) - 1))
        del t, hit
        u = ms.MsCol(format=ms.UNCOMPR, count_values=n, size_used_byte=8 * n, size_alloc_byte=8 * n, data=d)
        fmt = {"static": ms.STATIC_VBP, "dvbp": ms.DYNAMIC_VBP, "delta": ms.DELTA_DVBP, "for": ms.FOR_DVBP,
               "rle": ms.RLE}[kind]
        c, k = ms.MsCol(), ms.MsCol()
        ms._check(lib.ms_gpu_morph(C.byref(u), fmt, bits if kind == "static" else 0, C.byref(c), scratch.h, sp),
                  "morph")
        ms._check(lib.ms_gpu_col_compact(C.byref(c), C.byref(k), arena.h, sp), "compact")
        cols.append(ms.Column(k, arena))
        meds.append(med)
    torch.cuda.synchronize()
    return cols, meds, np.array(e_cnt, np.uint64), np.array(e_sum, np.uint64)


def tune(batch, stream, reps=3):
    """Time every launch configuration (graph replay) and keep the fastest."""
    import torch
    res = []
    for cfg in TUNE_CONFIGS:
        if _shm(cfg) > 227 * 1024 or (_shm(cfg) + 1024) * cfg["ctas_per_sm"] > 228 * 1024:
            continue
        batch.set_config(**cfg)
        batch.launch(graph=True, stream=stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            batch.launch(graph=True, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        res.append(dict(cfg, ms=round(e0.elapsed_time(e1) / reps, 4)))
    best = min(res, key=lambda r: r["ms"])
    batch.set_config(**{k: best[k] for k in _CFG_KEYS})
    return best, res


def _tuning_key(ms):
    return "batch/%d" % ms.device_info()[0]


def load_tuning(ms):
    try:
        with open(os.path.join(HERE, "tuning.json")) as f:
            return json.load(f).get(_tuning_key(ms))
    except (OSError, ValueError):
        return None


# benchmark kinds -> the plan's decoder kinds (static_vbp and dynamic_vbp share the vbp decoder)
DECODER_OF = {"static": "vbp", "dvbp": "vbp", "for": "for", "delta": "delta", "rle": "rle"}


def apply_kind_tuning(ms, batch) -> dict:
    """Per-kind configurations stored by --kinds ("batch:<kind>/<sm>"), where
    one differs from the plan's; returns the decoder kinds set."""
    try:
        with open(os.path.join(HERE, "tuning.json")) as f:
            d = json.load(f)
    except (OSError, ValueError):
        return {}
    sm = ms.device_info()[0]
    glob = batch.get_config()
    applied = {}
    for kind, dec in DECODER_OF.items():
        cfg = d.get("batch:%s/%d" % (kind, sm))
        if not cfg or dec in applied:
            continue
        cfg = {k: cfg[k] for k in _CFG_KEYS}
        if cfg != {k: glob[k] for k in _CFG_KEYS}:
            batch.set_kind_config(dec, **cfg)
            applied[dec] = cfg
    return applied


def save_tuning(ms, cfg, key=None):
    path = os.path.join(HERE, "tuning.json")
    try:
        with open(path) as f:
            d = json.load(f)
    except (OSError, ValueError):
        d = {}
    d[key or _tuning_key(ms)] = {k: cfg[k] for k in _CFG_KEYS}
    with open(path, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)


def time_graph(batch, stream, reps=5) -> float:
    import torch
    batch.launch(graph=True, stream=stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        batch.launch(graph=True, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def per_kind(ms, arena, cols, meds, plan, global_cfg, stream) -> dict:
    """One batch per kind: bytes, GB/s under the global configuration, the
    best configuration of the sweep and its GB/s."""
    out = {}
    for kind in KINDS:
        idx = [i for i, p in enumerate(plan) if p[1] == kind]
        if not idx:
            continue
        sub = ms.Batch([cols[i] for i in idx], [meds[i] for i in idx], ms.less, arena=arena, stream=stream)
        try:
            nbytes = sum(cols[i].get_size_used_byte() for i in idx)
            sub.set_config(**{k: global_cfg[k] for k in _CFG_KEYS})
            t_glob = time_graph(sub, stream)
            best, _ = tune(sub, stream)
            out[kind] = {"columns": len(idx), "compressed_bytes": nbytes,
                         "global_cfg_gbs": round(nbytes / (t_glob * 1e-3) / 1e9, 1),
                         "best": {k: best[k] for k in _CFG_KEYS},
                         "best_gbs": round(nbytes / (best["ms"] * 1e-3) / 1e9, 1)}
        finally:
            sub.close()
    return out


def run(n_cols: int = 4096, steps: int = 10, do_tune: bool = False, per_column_steps: int = 2,
        per_column: bool = True, kinds: bool = False) -> dict:
    import torch

    import engine_b200 as ms
    stream = torch.cuda.current_stream()
    arena = ms.Arena(40 << 30)
    scratch = ms.Arena(3 << 30)
    try:
        plan = plan_columns(n_cols)
        t0 = time.perf_counter()
        cols, meds, e_cnt, e_sum = build(ms, arena, scratch, plan, stream)
        t_build = time.perf_counter() - t0
        scratch.close()
        rows = sum(p[0] for p in plan)
        comp = sum(c.get_size_used_byte() for c in cols)
        t0 = time.perf_counter()
        batch = ms.Batch(cols, meds, ms.less, arena=arena, stream=stream)
        t_plan = time.perf_counter() - t0
        swept = None
        if do_tune:
            tuned, swept = tune(batch, stream)
        else:
            cfg = load_tuning(ms)
            if cfg:
                batch.set_config(**{k: cfg[k] for k in _CFG_KEYS})
            tuned = dict(batch.get_config(), source="tuning.json" if cfg else "default")
        if not kinds:
            apply_kind_tuning(ms, batch)
        tuned["per_kind"] = batch.kind_configs()
        # batched: graph replay, K steps (events around each replay)
        batch.launch(graph=True, stream=stream)
        batch.launch(graph=True, stream=stream)
        torch.cuda.synchronize()
        cnt, sm = batch.results()
        ok_b = bool(np.array_equal(cnt, e_cnt) and np.array_equal(sm, e_sum))
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a, b in ev:
            a.record(stream)
            batch.launch(graph=True, stream=stream)
            b.record(stream)
        torch.cuda.synchronize()
        per = [a.elapsed_time(b) for a, b in ev]
        t_batch = float(np.mean(per))
        cnt, sm = batch.results()
        ok_b = ok_b and bool(np.array_equal(cnt, e_cnt) and np.array_equal(sm, e_sum))
        info = batch.info()
        kind_res = per_kind(ms, arena, cols, meds, plan, batch.get_config(), stream) if kinds else None
        batch.close()
        out = {
            "workload": "%d columns, log-uniform lengths 2^10..2^24 (%d rows), formats %s; decompress -> "
                        "select(value < median) -> sum per column"
                        % (n_cols, rows, {k: sum(1 for p in plan if p[1] == k) for k in KINDS}),
            "compressed_bytes": comp, "rows": rows, "items": info["items"], "launch": tuned,
            "batched_graph": {"ms": round(t_batch, 4), "min_ms": round(min(per), 4),
                              "gbs": round(comp / (t_batch * 1e-3) / 1e9, 1),
                              "grows_per_s": round(rows / (t_batch * 1e-3) / 1e9, 2)},
            "bit_exact": ok_b,
            "setup_s": {"generate_and_compress": round(t_build, 2), "plan": round(t_plan, 3)},
            "sweep": swept,
        }
        if kind_res is not None:
            out["per_kind"] = kind_res
        if not per_column:
            return out
        # one operator call per column, through the public API
        lib = ms.lib()
        ds, dc = arena.alloc(8 * n_cols), arena.alloc(8 * n_cols)
        mark = arena.used()

        def per_column_pass():
            for i, c in enumerate(cols):
                x = c.desc
                if x.format == ms.RLE:
                    u = ms.MsCol()
                    ms._check(lib.ms_gpu_morph(C.byref(x), ms.UNCOMPR, 0, C.byref(u), arena.h, stream.cuda_stream),
                              "decompress")
                    x = u
                ms._check(lib.ms_gpu_select_project_sum(C.byref(x), ms.less, meds[i], C.byref(x), ds + 8 * i,
                                                        dc + 8 * i, None, None, arena.h, stream.cuda_stream), "sps")
            ms._check(lib.ms_gpu_arena_reset(arena.h), "reset")
            arena.alloc(mark)

        per_column_pass()
        torch.cuda.synchronize()
        pc_sum = ms._memcpy_d2h(ds, 8 * n_cols).view(np.uint64)
        pc_cnt = ms._memcpy_d2h(dc, 8 * n_cols).view(np.uint64)
        ok_p = bool(np.array_equal(pc_cnt, e_cnt) and np.array_equal(pc_sum, e_sum))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        e0.record(stream)
        for _ in range(per_column_steps):
            per_column_pass()
        e1.record(stream)
        torch.cuda.synchronize()
        t_pc = max(e0.elapsed_time(e1), (time.perf_counter() - w0) * 1e3) / per_column_steps
        out["per_column_calls"] = {"ms": round(t_pc, 3), "gbs": round(comp / (t_pc * 1e-3) / 1e9, 1),
                                   "launches": "one fused select-sum per column (+ decompress for rle), "
                                               "public API, host synchronisation per call"}
        out["speedup_batched"] = round(t_pc / t_batch, 2)
        out["bit_exact"] = ok_b and ok_p
        return out
    finally:
        arena.close()


def main():
    sys.path.insert(0, os.path.dirname(HERE))
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    n_cols = int(args[0]) if args else 4096
    steps = int(args[1]) if len(args) > 1 else 10
    r = run(n_cols, steps, do_tune="--tune" in sys.argv, per_column="--no-per-column" not in sys.argv,
            kinds="--kinds" in sys.argv)
    if "--tune" in sys.argv and r["bit_exact"]:
        import engine_b200 as ms
        save_tuning(ms, r["launch"])
    if r.get("per_kind") and r["bit_exact"]:
        import engine_b200 as ms
        for kind, v in r["per_kind"].items():
            save_tuning(ms, v["best"], key="batch:%s/%d" % (kind, ms.device_info()[0]))
    print(json.dumps(r), flush=True)
    return 0 if r["bit_exact"] else 1


if __name__ == "__main__":
    sys.exit(main())
