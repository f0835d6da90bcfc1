"""One column sharded across ranks on the GPU: two processes (gloo for the
combine steps), each running the operators on its block-range views
(ms_gpu_col_slice) of the same compressed columns, combined through
engine_b200/dist.py -- sums and counts all-reduced, positions offset and
gathered, delta_f carry-ins from the earlier shards' lane sums
(ms_gpu_delta_lane_sums) -- must equal the unsharded GPU result and the
oracle on the whole column.  Both ranks use cuda:0; their kernels do not wait
on one another."""
import multiprocessing as mp
import os
import socket
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 300_007
CASES = [("dynamic_vbp_f", "delta_f"), ("for_f", ("static_vbp", 21)), (("static_vbp", 12), "dynamic_vbp_f"),
         ("uncompr_f", "for_f"), ("delta_f", "delta_f")]


def _fmt(ms, f):
    if isinstance(f, tuple):
        return ms.static_vbp_f(f[1])
    return getattr(ms, f)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _columns(orc):
    x = orc.uniform_bits(21, 12, N)
    y = orc.sorted_gaps(22, orc.geom_table(0.25), N)
    return x, y


def _worker(rank, world, port, outdir):
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist

    import engine_b200 as ms
    import oracle
    from engine_b200 import dist as D
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    arena = ms.Arena(2 << 30)
    try:
        orc = oracle.Oracle()
        x, y = _columns(orc)
        b, e = D.shard_rows(N, world, rank)
        res = {}
        for ci, (fx, fy) in enumerate(CASES):
            xc = ms.morph(ms.Column.from_numpy(x, arena), _fmt(ms, fx))
            yc = ms.morph(ms.Column.from_numpy(y, arena), _fmt(ms, fy))
            xs = xc.slice(b, e)
            if fy == "delta_f":
                carry = D.delta_carry(yc.slice(b, e).delta_lane_sums())
                ys = yc.slice(b, e, carry)
            else:
                ys = yc.slice(b, e)
            if fx == "delta_f":
                xs = xc.slice(b, e, D.delta_carry(xc.slice(b, e).delta_lane_sums()))
            res[f"{ci}/xlocal_ok"] = np.array_equal(xs.to_numpy(), x[b:e])
            s, k, pos, vals = ms.select_project_sum(xs, ms.less, 1500, ys, want_positions=True)
            lp = orc.select(oracle.CMP_LT, 1500, x[b:e])
            res[f"{ci}/local_ok"] = (len(pos) == len(lp) and np.array_equal(pos, lp) and
                                     s == int(y[b:e][lp.astype(np.int64)].sum(dtype=np.uint64)))
            res[f"{ci}/sum"] = D.all_reduce_sum_u64(s)
            res[f"{ci}/count"] = D.all_reduce_sum_u64(k)
            res[f"{ci}/pos"] = D.gather_positions(pos, b)
            res[f"{ci}/vals"] = D.gather_positions(vals, 0)
            res[f"{ci}/ysum"] = D.all_reduce_sum_u64(ms.agg_sum(ys))
            res[f"{ci}/ylocal_ok"] = np.array_equal(ys.to_numpy(), y[b:e])
            if rank == 0:
                fs, fk = ms.select_project_sum(xc, ms.less, 1500, yc)[:2]
                res[f"{ci}/full"] = np.array([fs, fk], dtype=np.uint64)
            arena.reset()
        np.savez(os.path.join(outdir, f"r{rank}.npz"), **{k: np.asarray(v) for k, v in res.items()})
    finally:
        arena.close()
        dist.destroy_process_group()


def test_sharded_column_on_gpu_equals_unsharded(ms, orc):
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with tempfile.TemporaryDirectory() as d:
        ps = [ctx.Process(target=_worker, args=(r, world, port, d)) for r in range(world)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(timeout=600)
        assert all(p.exitcode == 0 for p in ps), [p.exitcode for p in ps]
        r0 = dict(np.load(os.path.join(d, "r0.npz")))
        r1 = dict(np.load(os.path.join(d, "r1.npz")))
    x, y = _columns(orc)
    import oracle as O
    want_pos = orc.select(O.CMP_LT, 1500, x)
    want_vals = y[want_pos.astype(np.int64)]
    want_sum = int(want_vals.sum(dtype=np.uint64))
    ysum = int(y.sum(dtype=np.uint64))
    for ci in range(len(CASES)):
        for rk, r in enumerate((r0, r1)):
            assert bool(r[f"{ci}/ylocal_ok"]), ("y view decode", rk, CASES[ci])
            assert bool(r[f"{ci}/xlocal_ok"]), ("x view decode", rk, CASES[ci])
            assert bool(r[f"{ci}/local_ok"]), ("shard select-project-sum", rk, CASES[ci])
            assert int(r[f"{ci}/sum"]) == want_sum and int(r[f"{ci}/count"]) == len(want_pos), CASES[ci]
            assert np.array_equal(r[f"{ci}/pos"], want_pos), CASES[ci]
            assert np.array_equal(r[f"{ci}/vals"], want_vals), CASES[ci]
            assert int(r[f"{ci}/ysum"]) == ysum, CASES[ci]
        assert list(r0[f"{ci}/full"]) == [want_sum, len(want_pos)], CASES[ci]


def test_slice_rejects_misaligned_and_carry_misuse(ms, arena, orc):
    v = orc.uniform_bits(5, 16, 10_000)
    dv = ms.morph(ms.Column.from_numpy(v, arena), ms.dynamic_vbp_f)
    de = ms.morph(ms.Column.from_numpy(np.cumsum(v).astype(np.uint64), arena), ms.delta_f)
    with pytest.raises(ms.MorphStoreError):
        dv.slice(100, 1024)                      # not on a block boundary
    with pytest.raises(ms.MorphStoreError):
        de.slice(512, 2048)                      # delta_f blocks are 1024 rows
    with pytest.raises(ms.MorphStoreError):
        dv.slice(0, 1024, np.zeros(8, np.uint64))  # a carry-in is for delta_f
    sl = de.slice(1024, 10_000, de.slice(0, 1024).delta_lane_sums())
    with pytest.raises(ms.MorphStoreError):
        sl.slice(1024, 2048)                     # no views of a delta_f view with a carry-in
    assert np.array_equal(sl.to_numpy(), np.cumsum(v).astype(np.uint64)[1024:])
