#!/usr/bin/env python
"""Benchmark of the fused compression-aware select -> project -> sum path.

Workload (one "step"): the select_sum_query pipeline over 2^28 rows --
select(x < 512) on x (uniform over 10 bits), project the hits onto y
(uniform over 20 bits), agg_sum -- with both columns stored as
dynamic_vbp_f<512,64,8>, decompression fused into the operator.  Inputs are
seeded synthetic columns generated and compressed on the device; they are
larger than L2 (1.0 GB compressed), so no flush is needed between steps.

value: algorithmic GB/s = (compressed bytes of x + y + 8-B result) / kernel
time, inputs resident in HBM.  e2e: the same through the public C ABI with
host buffers: each step copies both compressed columns (and their block
indexes) from pinned host memory, runs the operator and reads the sum back.

`--impl reference` times the reference's own CPU implementation (the
MorphStore operators compiled from source under oracle/_ref, or the C
restatement of them when that library is absent) on the host cores.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_ROWS = 1 << 28
X_BITS, Y_BITS, PRED = 10, 20, 512
SEED_X, SEED_Y = 0x5EED0001, 0x5EED0002
METRIC = "fused decompress+select+project+sum GB/s (2^28-row dynamic_vbp columns)"
WORKLOAD = "select(x<512)->project(y)->agg_sum, 2^28 rows, x uniform 10-bit, y uniform 20-bit, both dynamic_vbp<512,64,8>"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic_per_launch():
    """DRAM bytes per launch of the fused kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "k_sps_dvbp_2p28.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return int(line.split(":")[1].strip())
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=2)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------------------
# reference / CPU baseline
# ---------------------------------------------------------------------------
def _cpu_sample_rows():
    return 1 << 24


_WORKER = {}


def _cpu_init(kind):
    """Pool initializer: the oracle / reference libraries, loaded once."""
    import oracle
    _WORKER["orc"] = oracle.Oracle()
    _WORKER["ref"] = oracle.Reference(oracle.reference_path()) if kind == "reference" else None


def _cpu_worker(args):
    """One process: its shard (generated once per process and kept), then the
    reference operators timed on it.  Returns (seconds, compressed bytes,
    sum)."""
    shard, rows, kind = args
    import oracle
    if "orc" not in _WORKER:
        _cpu_init(kind)
    orc = _WORKER["orc"]
    key = ("data", shard, rows)
    if key not in _WORKER:
        _WORKER[key] = (orc.uniform_bits(SEED_X + shard, X_BITS, rows), orc.uniform_bits(SEED_Y + shard, Y_BITS, rows))
    x, y = _WORKER[key]
    if kind == "reference":
        s, cnt, secs, cb = _WORKER["ref"].bench_select_project_sum(x, y, PRED)
        return secs, cb, s
    # port: the C restatement (decompress both columns, then select/project/sum)
    bx, mx = orc.compress(oracle.DYNAMIC_VBP, 0, x)
    by, my = orc.compress(oracle.DYNAMIC_VBP, 0, y)
    t0 = time.perf_counter()
    dx = orc.decompress(oracle.DYNAMIC_VBP, 0, bx, mx)
    dy = orc.decompress(oracle.DYNAMIC_VBP, 0, by, my)
    s, _ = orc.select_project_sum(oracle.CMP_LT, PRED, dx, dy)
    secs = time.perf_counter() - t0
    return secs, mx[1] + my[1], s


def _cpu_kind():
    import oracle
    return "reference" if oracle.reference_path() else "port"


def _cpu_sample(procs, kind, rows):
    isa = ""
    if kind == "reference":
        import oracle
        isa = "avx512" if oracle.host_has_avx512() else "avx2"
    return (f"{procs} process(es) x {rows} rows (2^24) each, same shapes and seeds scheme as the workload; "
            f"operator time only (inputs compressed beforehand); {kind}{'/' + isa if isa else ''}")


def _cpu_step(pool, procs, kind, rows):
    res = pool.map(_cpu_worker, [(i, rows, kind) for i in range(procs)])
    secs = max(r[0] for r in res)
    return sum(r[1] for r in res) / secs / 1e9


def cpu_baseline(procs: int, reps: int = 1):
    import multiprocessing as mp
    kind = _cpu_kind()
    rows = _cpu_sample_rows()
    with mp.get_context("spawn").Pool(procs, initializer=_cpu_init, initargs=(kind,)) as pool:
        best = max(_cpu_step(pool, procs, kind, rows) for _ in range(reps))
    return {"value": round(best, 3), "unit": "GB/s", "cores": procs, "kind": kind,
            "sample": _cpu_sample(procs, kind, rows)}


def run_reference(args):
    """The reference's own CPU operators on every host core: each step is one
    pass over a 2^24-row sample per process (the processes and their samples
    persist across steps)."""
    import multiprocessing as mp
    rank, world, _ = _dist()
    if rank != 0:
        return 0
    procs = max(1, os.cpu_count() or 1)
    kind = _cpu_kind()
    rows = _cpu_sample_rows()
    with mp.get_context("spawn").Pool(procs, initializer=_cpu_init, initargs=(kind,)) as pool:
        for _ in range(max(1, args.warmup)):
            _cpu_step(pool, procs, kind, rows)
        vals = []
        t0 = time.perf_counter()
        for _ in range(args.steps):
            vals.append(_cpu_step(pool, procs, kind, rows))
        wall = time.perf_counter() - t0
    value = round(float(np.median(vals)), 3)
    cb = cpu_baseline(1)
    cb_all = {"value": value, "unit": "GB/s", "cores": procs, "kind": kind,
              "sample": f"each step: {procs} processes x 2^24 rows, reference operators on the host cores"}
    line = {"metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1000 * wall / max(1, args.steps), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "impl": "reference", "config": {"workload": WORKLOAD + " (CPU sample: 2^24 rows per process)",
                                            "parallelism": f"{procs} host processes"},
            "cpu_baseline": cb_all, "single_thread_gbs": cb["value"],
            "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_gpu(args):
    import torch
    rank, world, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import engine_b200 as ms
    lib = ms.lib()
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    arena = ms.Arena(16 << 30)

    # --- data: generated and compressed on the device (outside timing) -------
    n = 1 << args.log2_rows
    xu = arena.alloc(8 * n)
    yu = arena.alloc(8 * n)
    ms._check(lib.ms_gpu_gen_uniform_bits(SEED_X + rank, X_BITS, n, xu, sp), "gen x")
    ms._check(lib.ms_gpu_gen_uniform_bits(SEED_Y + rank, Y_BITS, n, yu, sp), "gen y")
    ux = ms.MsCol(format=ms.UNCOMPR, count_values=n, size_used_byte=8 * n, size_alloc_byte=8 * n, data=xu)
    uy = ms.MsCol(format=ms.UNCOMPR, count_values=n, size_used_byte=8 * n, size_alloc_byte=8 * n, data=yu)
    xc, yc = ms.MsCol(), ms.MsCol()
    ms._check(lib.ms_gpu_morph(C.byref(ux), ms.DYNAMIC_VBP, 0, C.byref(xc), arena.h, sp), "morph x")
    ms._check(lib.ms_gpu_morph(C.byref(uy), ms.DYNAMIC_VBP, 0, C.byref(yc), arena.h, sp), "morph y")
    algo_bytes = int(xc.size_used_byte) + int(yc.size_used_byte) + 8
    from engine_b200 import autotune
    tuned = autotune.apply(ms, xc, yc)

    # expected result (device-side check with torch on the uncompressed inputs)
    tx = ms._device_view(xu, 8 * n).view(torch.int64)
    ty = ms._device_view(yu, 8 * n).view(torch.int64)
    mask = tx < PRED
    exp_sum = int(torch.where(mask, ty, torch.zeros_like(ty)).sum().item()) & ((1 << 64) - 1)
    exp_cnt = int(mask.sum().item())
    del tx, ty, mask

    d_sum = arena.alloc(8)
    d_cnt = arena.alloc(8)
    d_err = arena.alloc(8)
    torch.cuda.synchronize()

    def step():
        ms._check(lib.ms_gpu_select_project_sum_async(C.byref(xc), ms.less, PRED, C.byref(yc), d_sum, d_cnt, d_err,
                                                      sp), "sps")

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    got_sum = int(ms._memcpy_d2h(d_sum, 8).view(np.uint64)[0])
    got_cnt = int(ms._memcpy_d2h(d_cnt, 8).view(np.uint64)[0])
    ok = (got_sum == exp_sum and got_cnt == exp_cnt)

    # --- timed region: K steps, events around each launch ---------------------
    if world > 1:
        torch.distributed.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t_all0 = torch.cuda.Event(enable_timing=True)
        t_all1 = torch.cuda.Event(enable_timing=True)
        t_all0.record(stream)
        for i in range(args.steps):
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
        t_all1.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    per = [a.elapsed_time(b) for a, b in ev]
    total_ms = t_all0.elapsed_time(t_all1)
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
        # the shards' results combined once (outside the timed region): the
        # query over the whole table is the sum of the per-shard sums
        def s64(v):
            return v - (1 << 64) if v >= 1 << 63 else v
        comb = torch.tensor([s64(got_sum), got_cnt, s64(exp_sum), exp_cnt, int(not ok)], dtype=torch.int64,
                            device=dev)
        torch.distributed.all_reduce(comb)
        ok = bool(comb[4].item() == 0 and comb[0].item() == comb[2].item() and comb[1].item() == comb[3].item())
        got_cnt = int(comb[1].item())
    ms_per_step = total_ms / args.steps
    kern_ms = statistics.mean(per)
    value = world * algo_bytes / (ms_per_step * 1e-3) / 1e9

    # --- e2e: host buffers through the public API ----------------------------
    e2e = None if args.no_e2e else e2e_run(ms, lib, arena, xc, yc, sp, args, exp_sum)

    peak, peak_kind = _peaks()
    achieved = algo_bytes / (kern_ms * 1e-3) / 1e9
    line = {"metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "rows_per_gpu": n, "compressed_bytes_per_gpu": algo_bytes,
                       "parallelism": f"shards{world} (one per rank, results combined by all_reduce)"
                       if world > 1 else "single",
                       "l2": "inputs (1.0 GB) larger than L2; no flush",
                       "launch": dict(ms.get_tuning(), source="tuning.json" if tuned else "default")},
            "parity": {"sum_ok": ok, "count": got_cnt},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "traffic": _traffic_per_launch(), "kernel": "k_sps_tma (sps_tma.cu)" if ms.get_tuning()["staged"] else "k_sps (ops.cu)",
                         "algorithmic_bytes_per_launch": algo_bytes},
            "clocks": clk.summary(), "e2e": e2e, "gpu_launches": args.steps}
    if args.log2_rows != 28:
        line["config"]["note"] = "reduced size: profiling run, not the benchmark workload"
    arena.close()
    if not args.no_selector and world == 1:
        line["learned_selector"] = selector_run(ms, args)
    if not args.no_star and world == 1:
        from engine_b200 import star_query
        line["star_query"] = star_query.run(args.log2_rows, 5)
        ok = ok and line["star_query"]["bit_exact"]
    if not args.no_batch and world == 1:
        from engine_b200 import batch_bench
        line["batched"] = batch_bench.run(4096, 10, per_column_steps=1)
        ok = ok and line["batched"]["bit_exact"]
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            line["cpu_baseline"] = cpu_baseline(1)
        except Exception as exc:  # baseline is reported, not required
            line["cpu_baseline"] = {"error": str(exc)[:200]}
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0 if ok else 1


def selector_run(ms, args):
    """Learned vs exhaustive format pick on a 2^30-value column of 64K-value
    segments cycling through uniform-b-bit, sorted-with-gaps, long-run and
    Zipf data; MLP trained on 2^20 labelled 2048-value blocks (2000 Adam
    steps, batch 4096).  Times are device times (CUDA events) on this GPU."""
    import torch
    import engine_b200.selector as S
    from engine_b200.datagen import zipf_table
    zipf = zipf_table(1.2, 1 << 20)
    stream = torch.cuda.current_stream()
    arena = ms.Arena(20 << 30)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    try:
        # --- training set: 2^20 blocks, labelled by the codecs themselves -------
        n_train = 1 << (args.sel_log2_train)
        chunk = 1 << 17
        feats = arena.alloc(4 * 32 * n_train)
        sizes = arena.alloc(4 * 5 * n_train)
        mark = arena.used()
        t_label = 0.0
        for c0 in range(0, n_train, chunk):
            nb = min(chunk, n_train - c0)
            d = S.gen(arena, 1000 + c0, nb, 32, zipf)
            st = arena.alloc(S.STATS_BYTES * nb)
            e0, e1 = ev(), ev()
            e0.record(stream)
            ms._check(S._L.ms_gpu_sel_analyze(d, nb, st, sizes + 4 * 5 * c0, stream.cuda_stream), "analyze")
            ms._check(S._L.ms_gpu_sel_features(d, nb, feats + 4 * 32 * c0, stream.cuda_stream), "features")
            e1.record(stream)
            torch.cuda.synchronize()
            t_label += e0.elapsed_time(e1)
            ms._check(ms.lib().ms_gpu_arena_reset(arena.h), "reset")
            arena.alloc(mark)  # keep feats/sizes
        m = S.Mlp(seed=1, max_batch=4096)
        e0, e1 = ev(), ev()
        e0.record(stream)
        curve = m.train(arena, feats, sizes, n_train, steps=args.sel_steps, batch=4096, lr=2e-3)
        e1.record(stream)
        torch.cuda.synchronize()
        t_train = e0.elapsed_time(e1)
        # --- evaluation column: 2^30 values ------------------------------------
        n_eval = 1 << (args.sel_log2_eval - 11)
        col = S.gen(arena, 77, n_eval, 32, zipf)
        scratch = arena.alloc(int(S._L.ms_gpu_sel_compress_all_scratch_bytes()))
        st_all = arena.alloc(S.STATS_BYTES * n_eval)
        sz_all = arena.alloc(4 * 5 * n_eval)
        err = arena.alloc(8)
        ch_ex = arena.alloc(n_eval)
        tot = arena.alloc(8)
        feats_e = arena.alloc(4 * 32 * n_eval)
        ch_ml = arena.alloc(n_eval)
        nfb = arena.alloc(8)
        margin = float(np.log2(1.02))
        sp = stream.cuda_stream

        def exhaustive_materialising():
            ms._check(S._L.ms_gpu_sel_compress_all(col, n_eval, st_all, sz_all, scratch, err, sp), "compress_all")
            ms._check(S._L.ms_gpu_sel_argmin(sz_all, n_eval, ch_ex, tot, sp), "argmin")

        def exhaustive_size_only():
            ms._check(S._L.ms_gpu_sel_analyze(col, n_eval, st_all, sz_all, sp), "analyze")
            ms._check(S._L.ms_gpu_sel_argmin(sz_all, n_eval, ch_ex, tot, sp), "argmin")

        def learned():
            ms._check(S._L.ms_gpu_sel_features(col, n_eval, feats_e, sp), "features")
            ms._check(S._L.ms_gpu_mlp_choose(m.h, feats_e, n_eval, margin, None, ch_ml, nfb, sp), "choose")
            ms._check(S._L.ms_gpu_sel_resolve(col, n_eval, ch_ml, sp), "resolve")

        t_all = timed(exhaustive_materialising)
        t_size = timed(exhaustive_size_only)
        t_ml = timed(learned)
        exhaustive_size_only()
        n_fb = int(S.to_host(nfb, 1, np.uint64)[0])
        fp_ex = S.footprint(arena, sz_all, ch_ex, n_eval)
        fp_ml = S.footprint(arena, sz_all, ch_ml, n_eval)
        picks = np.bincount(S.to_host(ch_ml, n_eval, np.uint8), minlength=5).tolist()
        # --- end to end: selection + compression + select-sum ------------------
        cmp_val = 1 << 20
        tv = ms._device_view(col, 8 * n_eval * S.BLOCK).view(torch.int64)
        hit = tv < cmp_val  # values stay below 2^63: signed compare as the operator's
        exp_s = int(torch.where(hit, tv, torch.zeros_like(tv)).sum().item()) & ((1 << 64) - 1)
        exp_c = int(hit.sum().item())
        del tv, hit
        results = {}
        for name, pick in (("exhaustive", ch_ex), ("learned", ch_ml)):
            mark2 = arena.used()

            def e2e(pick=pick, name=name):
                ms._check(ms.lib().ms_gpu_arena_reset(arena.h), "reset")
                arena.alloc(mark2)
                if name == "exhaustive":
                    exhaustive_materialising()
                    stp = st_all
                else:
                    learned()
                    ms._check(S._L.ms_gpu_sel_analyze(col, n_eval, st_all, None, sp), "analyze")
                    stp = st_all
                cont = S.Container(arena, col, n_eval, stp, pick, stream=stream)
                results[name] = cont.select_sum(ms.less, cmp_val, stream=stream) + (cont.nbytes,)

            results[name + "_ms"] = timed(e2e, reps=2)
        ok = (results["exhaustive"][:2] == (exp_s, exp_c) and results["learned"][:2] == (exp_s, exp_c)
              and results["exhaustive"][2] == 0 and results["learned"][2] == 0)
        m.close()
        return {
            "workload": "2^%d-value column, 64K-value segments cycling uniform(1..40 bit)/sorted/runs/Zipf(1.2); "
                        "2048-value blocks; candidates static_vbp, dynamic_vbp, delta+dvbp, for+dvbp, rle"
                        % args.sel_log2_eval,
            "train": {"blocks": n_train, "steps": args.sel_steps, "batch": 4096, "ms": round(t_train, 1),
                      "label_and_feature_ms": round(t_label, 1), "loss_first": float(curve[:10].mean()),
                      "loss_last": float(curve[-10:].mean())},
            "footprint_bytes": {"exhaustive": fp_ex, "learned": fp_ml},
            "regret": round(fp_ml / fp_ex - 1, 5),
            "fallback_fraction": round(n_fb / n_eval, 4),
            "picks": dict(zip(S.CAND_NAMES, picks)),
            "selection_ms": {"compress_all": round(t_all, 3), "exhaustive_size_only": round(t_size, 3),
                             "learned": round(t_ml, 3)},
            "selection_speedup_vs_compress_all": round(t_all / t_ml, 2),
            "e2e_ms": {"exhaustive": round(results["exhaustive_ms"], 3), "learned": round(results["learned_ms"], 3)},
            "container_bytes": {"exhaustive": results["exhaustive"][3], "learned": results["learned"][3]},
            "select_sum_bit_exact": ok,
        }
    finally:
        arena.close()


def e2e_run(ms, lib, arena, xc, yc, sp, args, exp_sum):
    """Per step: H2D of both compressed columns + block indexes from pinned
    host memory, the fused operator, D2H of the 8-byte sum."""
    import torch
    host = {}
    for name, c in (("x", xc), ("y", yc)):
        used = int(c.size_used_byte)
        hb = torch.empty(used, dtype=torch.uint8, pin_memory=True)
        hb.copy_(ms._device_view(c.data, used).cpu())
        nb = int(c.n_index)
        hi = torch.empty(8 * nb, dtype=torch.uint8, pin_memory=True)
        idx = np.zeros(nb + 1, dtype=np.uint64)
        hnp = hb.numpy()
        ms._check(lib.ms_host_build_index(int(c.format), hnp.ctypes.data, int(c.size_compr_byte),
                                          nb * 512, idx.ctypes.data, None), "host index")
        hi.copy_(torch.from_numpy(idx[:nb].view(np.uint8)))
        dbuf = arena.alloc(used + 64)
        didx = arena.alloc(8 * nb + 8)
        desc = ms.MsCol(format=c.format, bw=c.bw, count_values=c.count_values, size_used_byte=used,
                        size_compr_byte=c.size_compr_byte, size_alloc_byte=used + 64, data=dbuf, index=didx,
                        n_index=nb)
        host[name] = (hb, hi, dbuf, didx, desc)
    d_sum = arena.alloc(8)
    d_err = arena.alloc(8)
    h_sum = torch.empty(8, dtype=torch.uint8, pin_memory=True)
    stream = torch.cuda.current_stream()
    h2d = sum(h[0].numel() + h[1].numel() for h in host.values())
    algo = int(xc.size_used_byte) + int(yc.size_used_byte) + 8

    def step():
        for hb, hi, dbuf, didx, desc in host.values():
            ms._device_view(dbuf, hb.numel()).copy_(hb, non_blocking=True)
            ms._device_view(didx, hi.numel()).copy_(hi, non_blocking=True)
        ms._check(lib.ms_gpu_select_project_sum_async(C.byref(host["x"][4]), ms.less, PRED, C.byref(host["y"][4]),
                                                      d_sum, None, d_err, sp), "sps e2e")
        h_sum.copy_(ms._device_view(d_sum, 8), non_blocking=True)

    for _ in range(2):
        step()
    torch.cuda.synchronize()
    ok = int(h_sum.numpy().view(np.uint64)[0]) == exp_sum
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k = max(1, min(args.steps, 20))
    e0.record(stream)
    for _ in range(k):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_step = e0.elapsed_time(e1) / k
    return {"value": round(algo / (ms_step * 1e-3) / 1e9, 2), "unit": "GB/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": 8, "ms_per_step": round(ms_step, 3), "sum_ok": ok,
            "path": "ms_gpu_select_project_sum_async via ctypes, pinned host buffers"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end (host buffer) leg")
    ap.add_argument("--log2-rows", type=int, default=28, help="rows per GPU = 2^N (profiling runs use less)")
    ap.add_argument("--no-selector", action="store_true", help="skip the learned-vs-exhaustive selector leg")
    ap.add_argument("--sel-log2-train", type=int, default=20, help="training blocks = 2^N")
    ap.add_argument("--sel-log2-eval", type=int, default=30, help="evaluation column values = 2^N")
    ap.add_argument("--sel-steps", type=int, default=2000, help="Adam steps")
    ap.add_argument("--no-star", action="store_true", help="skip the fused star-query leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched many-column leg")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
