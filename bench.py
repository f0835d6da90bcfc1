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
host buffers in the reference's byte layout: each step builds the block
indexes on the host, copies both compressed columns and their indexes from
pinned host memory, runs the operator and reads the sum back.  Rank r of N
holds rows [r 2^28, (r+1) 2^28) of one table.

Parity: the sum and count are checked on the device against torch over the
uncompressed rows and, at N = 1, against the reference's own operators run
over exactly the same rows on the host cores.  Further legs (each reported
beside the headline, not as it): the learned format selector, the fused
star query, the batched many-column execution, the codec round-trip sweep
and a one-core CPU baseline.

`--impl reference` times the reference's own CPU implementation (the
MorphStore operators compiled from source under oracle/_ref, or the C
restatement of them when that library is absent) on all host cores over the
GPU arm's whole table.  `--gpus N` without a launcher starts N ranks under
torch.distributed.run.
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
def _config(n, world, compressed_per_gpu):
    """The workload as both arms name it."""
    return {"workload": WORKLOAD, "rows_per_gpu": n, "total_rows": world * n,
            "compressed_bytes_per_gpu": int(compressed_per_gpu),
            "parallelism": "single" if world == 1 else f"rows split across {world} ranks"}


def _cpu_kind():
    import oracle
    return "reference" if oracle.reference_path() else "port"


def _isa(kind):
    import oracle
    if kind != "reference":
        return "C restatement"
    return "reference/" + ("avx512" if oracle.host_has_avx512() else "avx2")


def cpu_baseline(log2_rows: int = 24, reps: int = 3):
    """The reference's operators on one host core, on rows [0, 2^log2_rows)
    of the benchmark's columns (operator time only, best of `reps`)."""
    from oracle import workloads
    kind = _cpu_kind()
    rows = 1 << log2_rows
    with workloads.ShardWorkers(rows, 1, kind) as w:
        cb = w.prepare()
        w.run()
        secs = min(w.run()[0] for _ in range(reps))
    return {"value": round(cb / secs / 1e9, 3), "unit": "GB/s", "cores": 1, "kind": kind,
            "sample": f"rows [0, 2^{log2_rows}) of the workload's x and y, 1 process, {_isa(kind)}, operator time "
                      f"only (inputs compressed beforehand), best of {reps}",
            "host": workloads.host_record()}


def reference_check(n):
    """The reference's result over exactly the GPU's rows, on every host core:
    (sum, count, compressed bytes)."""
    from oracle import workloads
    kind = _cpu_kind()
    with workloads.ShardWorkers(n, max(1, os.cpu_count() or 1), kind) as w:
        cb = w.prepare()
        _, s, cnt = w.run()
    return s, cnt, cb, kind


def run_reference(args):
    """The reference's own CPU operators on every host core over the GPU arm's
    whole table (rows split into page-aligned shards, one process per core;
    each shard generated and compressed once before timing).  A step is one
    pass of select -> project -> sum over all rows; its time is the slowest
    process's operator time."""
    from oracle import workloads
    rank, world, _ = _dist()
    if rank != 0:
        return 0
    n = 1 << args.log2_rows
    total = world * n
    procs = max(1, os.cpu_count() or 1)
    kind = _cpu_kind()
    with workloads.ShardWorkers(total, procs, kind) as w:
        cb = w.prepare()
        for _ in range(max(1, args.warmup)):
            w.run()
        secs = []
        for _ in range(args.steps):
            t, s, cnt = w.run()
            secs.append(t)
        nshards, used = len(w.shards), w.procs
    value = round(cb * len(secs) / sum(secs) / 1e9, 3)
    line = {"metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1000 * statistics.mean(secs), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "impl": "reference", "config": _config(n, world, cb // world),
            "result": {"sum": s, "count": cnt},
            "cpu_baseline": {"value": value, "unit": "GB/s", "cores": used, "kind": kind,
                             "sample": f"each step: all {total} rows of the workload in {nshards} page-aligned "
                                       f"shards over {used} processes, {_isa(kind)}, operator time only",
                             "host": workloads.host_record()},
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
    # rank r holds rows [r n, (r+1) n) of one table (the same generator as the
    # reference arm's shards)
    ms._check(lib.ms_gpu_gen_uniform_bits_at(SEED_X, X_BITS, rank * n, n, xu, sp), "gen x")
    ms._check(lib.ms_gpu_gen_uniform_bits_at(SEED_Y, Y_BITS, rank * n, n, yu, sp), "gen y")
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
    got_sum_all = got_sum
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
        got_sum_all = int(comb[0].item()) & ((1 << 64) - 1)
    ms_per_step = total_ms / args.steps
    kern_ms = statistics.mean(per)
    value = world * algo_bytes / (ms_per_step * 1e-3) / 1e9

    # --- e2e: host buffers through the public API ----------------------------
    e2e = None if args.no_e2e else e2e_run(ms, lib, arena, xc, yc, sp, args, exp_sum)

    peak, peak_kind = _peaks()
    achieved = algo_bytes / (kern_ms * 1e-3) / 1e9
    parity = {"sum_ok": ok, "sum": got_sum_all, "count": got_cnt, "checked_against": "torch on the uncompressed rows"}
    if world == 1 and not args.no_ref_check:
        # the reference's own operators over exactly these rows, on the host cores
        try:
            rs, rc, rcb, rkind = reference_check(n)
            parity.update({"vs_reference": rs == got_sum and rc == got_cnt, "reference_sum": rs, "reference_count": rc,
                           "reference_kind": rkind, "reference_compressed_bytes": rcb,
                           "compressed_bytes_equal": rcb == algo_bytes - 8})
            ok = ok and parity["vs_reference"]
        except Exception as exc:  # reported, and the run fails: parity is not optional
            parity.update({"vs_reference": False, "reference_error": str(exc)[:300]})
            ok = False
    line = {"metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": _config(n, world, algo_bytes - 8),
            "l2": "inputs (1.0 GB per GPU) larger than L2; no flush",
            "launch": dict(ms.get_tuning(), source="tuning.json" if tuned else "default"),
            "parity": parity,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "traffic": _traffic_per_launch(), "kernel": "k_sps_tma (sps_tma.cu)" if ms.get_tuning()["staged"] else "k_sps (ops.cu)",
                         "algorithmic_bytes_per_launch": algo_bytes},
            "clocks": clk.summary(), "e2e": e2e, "gpu_launches": args.steps}
    if args.log2_rows != 28:
        line["note"] = "reduced size: profiling run, not the benchmark workload"
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
    if not args.no_sweep and world == 1:
        line["codec_sweep"] = codec_sweep_run(args.log2_rows, peak)
        ok = ok and line["codec_sweep"]["all_roundtrips_ok"]
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            line["cpu_baseline"] = cpu_baseline()
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


def codec_sweep_run(log2_rows, peak):
    """The codec round-trip sweep: uncompr -> format -> uncompr over 2^log2_rows
    values per case, for static_vbp at every bit width (uniform over that
    width) and dynamic_vbp, delta+dvbp, for+dvbp and rle over uniform (8, 16,
    20, 32, 64 bits), Zipf(1.2) over [0, 2^20), sorted (gaps 1 + Geom, mean 4)
    and runs (geometric lengths, mean 32).  Inputs are generated on the device;
    each direction is timed with CUDA events around the public morph call
    (which includes its size read-back) and the decoded column is compared
    with the input on the device.  Bytes per direction: 8 n + compressed
    size.  Compressed bytes are compared with the reference's codecs by the
    full-size tests."""
    import torch

    import engine_b200 as ms
    from engine_b200.datagen import geom_table, zipf_table
    n = 1 << log2_rows
    lib = ms.lib()
    arena = ms.Arena(24 << 30)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    zipf, geo = zipf_table(1.2, 1 << 20), geom_table(0.25)
    d_zipf, d_geo = arena.alloc(zipf.nbytes), arena.alloc(geo.nbytes)
    ms._memcpy_h2d(d_zipf, zipf)
    ms._memcpy_h2d(d_geo, geo)
    base = arena.used()
    names = {1: "static_vbp", 2: "dynamic_vbp", 3: "delta+dvbp", 4: "for+dvbp", 5: "rle"}

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

    cases = [("uniform%d" % b, ms.STATIC_VBP, b) for b in range(1, 65)]
    for dist in ("uniform8", "uniform16", "uniform20", "uniform32", "uniform64", "zipf", "sorted", "runs"):
        for fmt in (ms.DYNAMIC_VBP, ms.DELTA_DVBP, ms.FOR_DVBP, ms.RLE):
            cases.append((dist, fmt, 0))
    rows = []
    try:
        for dist, fmt, bw in cases:
            ms._check(lib.ms_gpu_arena_reset(arena.h), "reset")
            arena.alloc(base)
            u = make(dist, 0x5EED + bw)
            best_c = best_d = None
            for _ in range(2):  # the second pass is timed warm (first-touch of the arena pages excluded)
                ms._check(lib.ms_gpu_arena_reset(arena.h), "reset")
                arena.alloc(base + 8 * n)
                c, d = ms.MsCol(), ms.MsCol()
                torch.cuda.synchronize()
                e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
                e0.record(stream)
                ms._check(lib.ms_gpu_morph(C.byref(u), fmt, bw, C.byref(c), arena.h, sp), "compress")
                e1.record(stream)
                ms._check(lib.ms_gpu_morph(C.byref(c), ms.UNCOMPR, 0, C.byref(d), arena.h, sp), "decompress")
                e2.record(stream)
                torch.cuda.synchronize()
                best_c, best_d = e0.elapsed_time(e1), e1.elapsed_time(e2)
            ms._check(lib.ms_gpu_arena_check(arena.h, sp), "sweep kernels")
            ok = bool(torch.equal(ms._device_view(u.data, 8 * n), ms._device_view(d.data, 8 * n)))
            cb = int(c.size_used_byte)
            byt = 8 * n + cb
            rows.append([dist, names[fmt] + (f"<{bw}>" if bw else ""), cb, round(byt / best_c / 1e6, 1),
                         round(byt / best_d / 1e6, 1), ok])
    finally:
        arena.close()

    def frac(col, pred):
        v = [r[col] for r in rows if pred(r)]
        return {"min": round(min(v) / peak, 3), "median": round(statistics.median(v) / peak, 3),
                "max": round(max(v) / peak, 3)} if v else None

    by_fmt = {}
    for f in names.values():
        sel = (lambda r, f=f: r[1].split("<")[0] == f)
        by_fmt[f] = {"compress_frac": frac(3, sel), "decompress_frac": frac(4, sel)}
    return {"rows": n, "cases": len(rows), "all_roundtrips_ok": all(r[5] for r in rows),
            "columns": ["dist", "format", "compressed_bytes", "compress_gbs", "decompress_gbs", "roundtrip_ok"],
            "results": rows, "frac_of_peak_by_format": by_fmt, "peak_gbs": peak,
            "bytes": "8 n + compressed bytes per direction"}


def e2e_run(ms, lib, arena, xc, yc, sp, args, exp_sum):
    """The query through the public C ABI from host buffers that hold the
    columns in the reference's byte layout.  Per step: the block index of each
    column is built on the host from its page headers (ms_host_build_index --
    what a caller holding reference-layout bytes has to do), both columns and
    their indexes are copied from pinned host memory, the fused operator runs
    and the 8-byte sum is read back.  Timed by the wall clock around all
    steps (host index builds overlap the previous step's copies; two index
    buffers alternate), with one synchronisation at the end."""
    import torch
    host = {}
    for name, c in (("x", xc), ("y", yc)):
        used = int(c.size_used_byte)
        hb = torch.empty(used, dtype=torch.uint8, pin_memory=True)
        hb.copy_(ms._device_view(c.data, used).cpu())
        nb = int(c.n_index)
        hidx = [torch.empty(8 * nb + 8, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
        dbuf = arena.alloc(used + 64)
        didx = arena.alloc(8 * nb + 8)
        desc = ms.MsCol(format=c.format, bw=c.bw, count_values=c.count_values, size_used_byte=used,
                        size_compr_byte=c.size_compr_byte, size_alloc_byte=used + 64, data=dbuf, index=didx,
                        n_index=nb)
        host[name] = (hb, hidx, dbuf, didx, desc, nb)
    d_sum = arena.alloc(8)
    d_err = arena.alloc(8)
    h_sum = torch.empty(8, dtype=torch.uint8, pin_memory=True)
    stream = torch.cuda.current_stream()
    algo = int(xc.size_used_byte) + int(yc.size_used_byte) + 8
    done = [torch.cuda.Event(), torch.cuda.Event()]

    def step(i):
        j = i & 1
        done[j].synchronize()  # the copies that last read index buffer j have finished
        for hb, hidx, dbuf, didx, desc, nb in host.values():
            ms._check(lib.ms_host_build_index(int(desc.format), hb.data_ptr(), int(desc.size_compr_byte), nb * 512,
                                              hidx[j].data_ptr(), None), "host index")
            ms._device_view(dbuf, hb.numel()).copy_(hb, non_blocking=True)
            ms._device_view(didx, 8 * nb).copy_(hidx[j][: 8 * nb], non_blocking=True)
        done[j].record(stream)
        ms._check(lib.ms_gpu_select_project_sum_async(C.byref(host["x"][4]), ms.less, PRED, C.byref(host["y"][4]),
                                                      d_sum, None, d_err, sp), "sps e2e")
        h_sum.copy_(ms._device_view(d_sum, 8), non_blocking=True)

    for i in range(2):
        step(i)
    torch.cuda.synchronize()
    ok = int(h_sum.numpy().view(np.uint64)[0]) == exp_sum
    k = max(1, min(args.steps, 20))
    h2d = sum(h[0].numel() + 8 * h[5] for h in host.values())
    t0 = time.perf_counter()
    for i in range(k):
        step(i)
    torch.cuda.synchronize()
    ms_step = 1000 * (time.perf_counter() - t0) / k
    ok = ok and int(h_sum.numpy().view(np.uint64)[0]) == exp_sum
    return {"value": round(algo / (ms_step * 1e-3) / 1e9, 2), "unit": "GB/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": 8, "ms_per_step": round(ms_step, 3), "sum_ok": ok,
            "path": "host page walk (ms_host_build_index) + H2D of reference-layout bytes and index from pinned "
                    "memory + ms_gpu_select_project_sum_async + D2H of the sum, via ctypes; wall clock"}


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
    ap.add_argument("--no-sweep", action="store_true", help="skip the codec round-trip sweep leg")
    ap.add_argument("--no-ref-check", action="store_true",
                    help="skip the comparison with the reference's result over the same rows")
    args = ap.parse_args()
    world = os.environ.get("WORLD_SIZE")
    if args.gpus > 1 and world is None:
        return _launch_ranks(args.gpus)
    if world is not None and int(world) != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}", file=sys.stderr)
        return 2
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


def _launch_ranks(n):
    """`--gpus N` without a launcher: start N ranks (one per GPU) under
    torch.distributed.run on 127.0.0.1 and return their status."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.run(cmd).returncode


if __name__ == "__main__":
    sys.exit(main())
