"""The multi-GPU combine steps (engine_b200/dist.py) on two gloo ranks on the
CPU: every rank evaluates its row shard with the oracle, the ranks combine
through torch.distributed, and the result must equal the oracle on the whole
column -- sum, select positions, group ids / extents / grouped sums and the
delta_f carry-in."""
import os
import socket
import tempfile

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, outdir):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import datetime

    import torch.distributed as dist

    import oracle
    from engine_b200 import dist as D
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        orc = oracle.Oracle()
        n = 100_003
        x = orc.uniform_bits(1, 12, n)
        y = orc.uniform_bits(2, 20, n)
        g = orc.from_table(3, orc.zipf_table(1.1, 1000), n)
        b, e = D.shard_rows(n, world, rank)
        xs, ys, gs = x[b:e], y[b:e], g[b:e]
        # sum of y where x < 1500
        s_local, c_local = orc.select_project_sum(oracle.CMP_LT, 1500, xs, ys, len(xs))
        s = D.all_reduce_sum_u64(s_local)
        c = D.all_reduce_sum_u64(c_local)
        # positions
        pos = D.gather_positions(orc.select(oracle.CMP_LT, 1500, xs, len(xs)), b)
        off, total = D.rank_offsets(len(orc.select(oracle.CMP_LT, 1500, xs, len(xs))))
        # group by g with sum of y
        gr, ext = orc.group(gs)
        sums = orc.agg_sum_grouped(gr, ys, len(ext))
        keys = gs[ext.astype(np.int64)]
        mk, mf, msum = D.merge_groups(keys, ext + np.uint64(b), sums)
        # delta carry of a sorted column split across ranks
        z = np.cumsum(orc.uniform_bits(4, 4, n)).astype(np.uint64)
        d = (z - np.concatenate([np.zeros(8, np.uint64), z[:-8]])).astype(np.uint64)
        lane = np.zeros(8, np.uint64)
        for k in range(b, e):
            lane[k % 8] += d[k]
        carry = D.delta_carry(lane)
        np.savez(os.path.join(outdir, f"r{rank}.npz"), s=s, c=c, pos=pos, off=off, total=total, mk=mk, mf=mf,
                 msum=msum, carry=carry, b=b)
    finally:
        dist.destroy_process_group()


def test_two_rank_combine_matches_single_column(orc):
    import torch.multiprocessing as mp
    import oracle
    world = 2
    port = _free_port()
    with tempfile.TemporaryDirectory() as td:
        mp.start_processes(_worker, args=(world, port, td), nprocs=world, join=True, start_method="spawn")
        r = [np.load(os.path.join(td, f"r{i}.npz")) for i in range(world)]
    n = 100_003
    x = orc.uniform_bits(1, 12, n)
    y = orc.uniform_bits(2, 20, n)
    g = orc.from_table(3, orc.zipf_table(1.1, 1000), n)
    es, ec = orc.select_project_sum(oracle.CMP_LT, 1500, x, y, n)
    epos = orc.select(oracle.CMP_LT, 1500, x, n)
    gr, ext = orc.group(g)
    esums = orc.agg_sum_grouped(gr, y, len(ext))
    for rr in r:
        assert int(rr["s"]) == es and int(rr["c"]) == ec
        assert np.array_equal(rr["pos"], epos)
        assert int(rr["total"]) == len(epos)
        assert np.array_equal(rr["mk"], g[ext.astype(np.int64)])
        assert np.array_equal(rr["mf"], ext)
        assert np.array_equal(rr["msum"], esums)
    assert int(r[0]["off"]) == 0 and int(r[1]["off"]) == int((epos < int(r[1]["b"])).sum())
    # carry-in of rank 1 = lane sums of rank 0's deltas = z at rank 1's first row - its delta
    z = np.cumsum(orc.uniform_bits(4, 4, n)).astype(np.uint64)
    b1 = int(r[1]["b"])
    assert np.array_equal(r[1]["carry"], z[b1 - 8: b1][np.argsort(np.arange(b1 - 8, b1) % 8)])
    assert np.all(r[0]["carry"] == 0)


def test_shard_rows_cover_the_column():
    from engine_b200 import dist as D
    for n in (0, 1, 1023, 1024, 100_003, 1 << 20):
        for world in (1, 2, 3, 8):
            ranges = [D.shard_rows(n, world, r) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            for (a, b), (c, d) in zip(ranges, ranges[1:]):
                assert b == c and a <= b and (b % 1024 == 0 or b == n)
