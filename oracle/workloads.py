"""Reference-side runs of the benchmark workloads -- TEST / BENCH INFRASTRUCTURE ONLY.

The headline query (select(x < 512) -> project(y) -> agg_sum over seeded
uniform columns, both stored as dynamic_vbp_f<512,64,8>) is run here on the
host cores by the reference's own operators (``_ref/libmsref_<isa>.so``) or,
where that library was not built, by the C restatement.  The rows are
exactly the GPU's: both sides draw row i of x and y from the same
counter-based generator, so a shard of rows [row0, row0 + rows) holds the
GPU column's rows and the shards' sums and counts add up to the GPU's.

``ShardWorkers`` keeps one spawned process per host core, each owning a fixed
set of shards that it generates and compresses once (outside any timing) and
then runs on command, so a timed step is operator time only.

Also here: the per-case inputs and masked-byte digests of the codec sweep at
full size, and a record of the host's CPU (model, sockets, cores, AVX-512).
"""
from __future__ import annotations

import hashlib
import multiprocessing as mp
import os
import re
import subprocess
import time

import numpy as np

SEED_X, SEED_Y = 0x5EED0001, 0x5EED0002
X_BITS, Y_BITS, PRED = 10, 20, 512


# ---------------------------------------------------------------------------
# host record
# ---------------------------------------------------------------------------
def host_record() -> dict:
    """CPU model, sockets, physical and logical cores, AVX-512 (from lscpu,
    /proc/cpuinfo as a fallback)."""
    rec = {"model": None, "sockets": None, "physical_cores": None, "logical_cores": os.cpu_count(),
           "avx512": False}
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        kv = {}
        for line in out.splitlines():
            if ":" in line:
                k, v = line.split(":", 1)
                kv[k.strip()] = v.strip()
        rec["model"] = kv.get("Model name")
        if kv.get("Socket(s)", "").isdigit():
            rec["sockets"] = int(kv["Socket(s)"])
        if kv.get("Core(s) per socket", "").isdigit() and rec["sockets"]:
            rec["physical_cores"] = int(kv["Core(s) per socket"]) * rec["sockets"]
        if kv.get("CPU(s)", "").isdigit():
            rec["logical_cores"] = int(kv["CPU(s)"])
    except (OSError, subprocess.SubprocessError):
        pass
    try:
        with open("/proc/cpuinfo") as f:
            info = f.read()
        flags = set(re.findall(r"^flags\s*:\s*(.*)$", info, re.M)[0].split()) if "flags" in info else set()
        rec["avx512"] = all(x in flags for x in ("avx512f", "avx512dq", "avx512bw", "avx512vl", "avx512cd"))
        if rec["model"] is None:
            m = re.search(r"^model name\s*:\s*(.*)$", info, re.M)
            rec["model"] = m.group(1) if m else None
        if rec["physical_cores"] is None:
            pairs = set(re.findall(r"^physical id\s*:\s*(\d+)\s*$.*?^core id\s*:\s*(\d+)\s*$", info, re.M | re.S))
            rec["physical_cores"] = len(pairs) or None
    except (OSError, IndexError):
        pass
    return rec


# ---------------------------------------------------------------------------
# headline query on shards of the GPU's rows
# ---------------------------------------------------------------------------
def plan_shards(total_rows: int, procs: int) -> list[tuple[int, int]]:
    """Row ranges (row0, rows): a power-of-two count >= max(16, procs), each a
    whole number of dynamic_vbp pages (32768 rows), so the shards' compressed
    sizes add up to the whole column's."""
    n = 16
    while n < procs:
        n *= 2
    while n > 1 and (total_rows // n) % 32768:
        n //= 2
    rows = total_rows // n
    return [(i * rows, rows) for i in range(n)]


def _worker_loop(conn, kind: str, shards):
    import oracle
    orc = oracle.Oracle()
    ref = oracle.Reference(oracle.reference_path()) if kind == "reference" else None
    held = []
    try:
        while True:
            cmd, arg = conn.recv()
            if cmd == "prepare":
                cb = 0
                for row0, rows in shards:
                    x = orc.uniform_bits(SEED_X, X_BITS, rows, row0)
                    y = orc.uniform_bits(SEED_Y, Y_BITS, rows, row0)
                    if ref is not None:
                        h, b = ref.sps_prepare(x, y)
                        held.append(h)
                    else:
                        bx, mx = orc.compress(oracle.DYNAMIC_VBP, 0, x)
                        by, my = orc.compress(oracle.DYNAMIC_VBP, 0, y)
                        held.append((bx, mx, by, my))
                        b = mx[1] + my[1]
                    cb += b
                    del x, y
                conn.send(cb)
            elif cmd == "run":
                secs, s, cnt = 0.0, 0, 0
                for h in held:
                    if ref is not None:
                        hs, hc, t = ref.sps_run(h, arg)
                    else:
                        bx, mx, by, my = h
                        t0 = time.perf_counter()
                        dx = orc.decompress(oracle.DYNAMIC_VBP, 0, bx, mx)
                        dy = orc.decompress(oracle.DYNAMIC_VBP, 0, by, my)
                        hs, hc = orc.select_project_sum(oracle.CMP_LT, arg, dx, dy,
                                                        orc.scalar_from(oracle.DYNAMIC_VBP, 0, mx))
                        t = time.perf_counter() - t0
                    secs += t
                    s = (s + hs) & ((1 << 64) - 1)
                    cnt += hc
                conn.send((secs, s, cnt))
            else:
                break
    finally:
        if ref is not None:
            for h in held:
                ref.sps_free(h)
        conn.close()


class ShardWorkers:
    """One spawned process per slot, each owning shards i with i % procs ==
    slot.  prepare() generates and compresses every shard once; run(c) runs
    the query on all shards and returns (max process seconds, sum, count)."""

    def __init__(self, total_rows: int, procs: int, kind: str):
        self.shards = plan_shards(total_rows, procs)
        self.procs = min(procs, len(self.shards))
        self.kind = kind
        ctx = mp.get_context("spawn")
        self.conns, self.ps = [], []
        for slot in range(self.procs):
            a, b = ctx.Pipe()
            p = ctx.Process(target=_worker_loop, args=(b, kind, self.shards[slot::self.procs]), daemon=True)
            p.start()
            b.close()
            self.conns.append(a)
            self.ps.append(p)

    def prepare(self) -> int:
        for c in self.conns:
            c.send(("prepare", None))
        return sum(c.recv() for c in self.conns)

    def run(self, pred: int = PRED):
        for c in self.conns:
            c.send(("run", pred))
        res = [c.recv() for c in self.conns]
        s = 0
        for r in res:
            s = (s + r[1]) & ((1 << 64) - 1)
        return max(r[0] for r in res), s, sum(r[2] for r in res)

    def close(self):
        for c in self.conns:
            try:
                c.send(("quit", None))
                c.close()
            except OSError:
                pass
        for p in self.ps:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


# ---------------------------------------------------------------------------
# codec sweep at full size: inputs and digests of the meaningful bytes
# ---------------------------------------------------------------------------
DISTRIBUTIONS = ("uniform", "zipf", "sorted", "runs")


def sweep_values(orc, dist: str, n: int, seed: int, bits: int = 20):
    """The sweep's seeded inputs (the device generators draw the same rows):
    uniform over `bits` bits; Zipf(1.2) over [0, 2^20); sorted ascending with
    gaps 1 + Geom (mean 4); runs with geometric lengths (mean 32) of values
    uniform over 20 bits."""
    if dist == "uniform":
        return orc.uniform_bits(seed, bits, n)
    if dist == "zipf":
        return orc.from_table(seed, orc.zipf_table(1.2, 1 << 20), n)
    if dist == "sorted":
        return orc.sorted_gaps(seed, orc.geom_table(0.25), n)
    if dist == "runs":
        return orc.runs(seed, 5, 20, n)
    raise ValueError(dist)


def masked_digest(fmt: int, bw: int, data: np.ndarray, meta, orc) -> str:
    """blake2b of the bytes that carry meaning (the compressed part with
    for_f's never-written header words zeroed, then the uncompressed rest; the
    gap between them is skipped).  `data` may be modified in place."""
    import oracle
    n, used, compr = meta
    h = hashlib.blake2b(digest_size=16)
    h.update(np.array([n, used, compr], dtype=np.uint64).tobytes())
    if fmt in (oracle.UNCOMPR, oracle.RLE) or used == compr:
        h.update(memoryview(data[:used]))
        return h.hexdigest()
    if fmt == oracle.FOR_DVBP and compr:
        oracle._mask_for_headers(data, compr)
    h.update(memoryview(data[:compr]))
    h.update(memoryview(data[orc.rest_offset(fmt, bw, compr):used]))
    return h.hexdigest()


def reference_codec_digest(args):
    """Pool task: (dist, fmt, bw, n, seed, bits) -> (digest, meta, isa) from
    the reference codec (the C restatement where the reference library is
    absent: isa 'port')."""
    dist, fmt, bw, n, seed, bits = args
    import oracle
    orc = oracle.Oracle()
    v = sweep_values(orc, dist, n, seed, bits)
    path = oracle.reference_path()
    if path:
        ref = oracle.Reference(path)
        cap = orc.size_max_any_len(fmt, bw, n) + (1 << 20)
        out = np.zeros(cap, dtype=np.uint8)
        m = oracle.Meta()
        import ctypes as C
        rc = ref.lib.ref_compress(fmt, bw, v.ctypes.data_as(oracle.U64P), n, out.ctypes.data_as(oracle.U8P), cap,
                                  C.byref(m))
        if rc:
            raise ValueError(f"ref_compress rc={rc}")
        meta, isa = m.tuple(), ("avx512" if ref.isa == 512 else "avx2")
    else:
        out, meta = orc.compress(fmt, bw, v)
        isa = "port"
    del v
    return masked_digest(fmt, bw, out, meta, orc), meta, isa
