"""Multi-GPU sharding of the compression-aware query path (host logic).

One process per GPU; each rank owns a contiguous range of 512-row blocks of
every column (block-aligned, so each shard is decoded with its own block
index and no data moves between GPUs).  Only results are exchanged, over
torch.distributed (NCCL on GPUs, gloo in the CPU tests):

* sum / count            all_reduce of uint64 (wrapping, as the reference's sum)
* select / semi_join     all_gather of per-rank hit counts -> exclusive offsets;
                         local positions + shard row offset are global positions
* group (+ grouped sum)  all_gather of each rank's (key, first row, sum) for at
                         most a few thousand groups; merged by smallest first row,
                         ids in order of first occurrence as the reference assigns
* delta_f carries        all_gather of each shard's 8 lane sums -> exclusive scan

No collective runs inside the per-block kernels.
"""
from __future__ import annotations

import numpy as np

BLOCK = 512


def shard_rows(n_rows: int, world: int, rank: int, align: int = 1024) -> tuple[int, int]:
    """Row range [begin, end) of `rank`: contiguous, aligned to `align` rows
    (1024 covers every format's block) except the last shard's end."""
    units = (n_rows + align - 1) // align
    u0 = units * rank // world
    u1 = units * (rank + 1) // world
    return min(n_rows, u0 * align), min(n_rows, u1 * align)


def _torch():
    import torch
    import torch.distributed as dist
    return torch, dist


def _as_i64(values):
    torch, _ = _torch()
    a = np.asarray(values, dtype=np.uint64).view(np.int64)
    return torch.from_numpy(a.copy())


def all_reduce_sum_u64(value: int, device="cpu") -> int:
    """Wrapping uint64 sum over ranks."""
    torch, dist = _torch()
    t = _as_i64([value]).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(np.array([t.cpu().item()], dtype=np.int64).view(np.uint64)[0])


def rank_offsets(local_count: int, device="cpu") -> tuple[int, int]:
    """(exclusive offset of this rank, global total) of per-rank counts."""
    torch, dist = _torch()
    t = torch.tensor([local_count], dtype=torch.int64, device=device)
    out = [torch.zeros_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(out, t)
    counts = [int(x.item()) for x in out]
    r = dist.get_rank()
    return sum(counts[:r]), sum(counts)


def gather_positions(local_pos: np.ndarray, row_begin: int, device="cpu") -> np.ndarray:
    """Global ascending positions from every rank's local positions."""
    torch, dist = _torch()
    g = np.asarray(local_pos, dtype=np.uint64) + np.uint64(row_begin)
    n = torch.tensor([len(g)], dtype=torch.int64, device=device)
    sizes = [torch.zeros_like(n) for _ in range(dist.get_world_size())]
    dist.all_gather(sizes, n)
    mx = max(int(s.item()) for s in sizes)
    buf = torch.zeros(mx, dtype=torch.int64, device=device)
    buf[: len(g)] = _as_i64(g).to(device)
    bufs = [torch.zeros_like(buf) for _ in sizes]
    dist.all_gather(bufs, buf)
    parts = [b[: int(s.item())].cpu().numpy().view(np.uint64) for b, s in zip(bufs, sizes)]
    return np.concatenate(parts) if parts else np.zeros(0, np.uint64)


def merge_groups(keys: np.ndarray, first_rows: np.ndarray, sums: np.ndarray, device="cpu"):
    """Merge per-rank groups: (keys, first rows, sums) of every rank -> global
    keys ordered by first occurrence, their first rows and summed values."""
    torch, dist = _torch()
    k = np.asarray(keys, np.uint64)
    f = np.asarray(first_rows, np.uint64)
    s = np.asarray(sums, np.uint64)
    n = torch.tensor([len(k)], dtype=torch.int64, device=device)
    sizes = [torch.zeros_like(n) for _ in range(dist.get_world_size())]
    dist.all_gather(sizes, n)
    mx = max(int(x.item()) for x in sizes)
    pack = torch.zeros((3, mx), dtype=torch.int64, device=device)
    for i, a in enumerate((k, f, s)):
        pack[i, : len(a)] = _as_i64(a).to(device)
    packs = [torch.zeros_like(pack) for _ in sizes]
    dist.all_gather(packs, pack)
    merged: dict[int, list[int]] = {}
    for p, sz in zip(packs, sizes):
        a = p[:, : int(sz.item())].cpu().numpy().view(np.uint64)
        for key, fr, sm in zip(a[0], a[1], a[2]):
            e = merged.get(int(key))
            if e is None:
                merged[int(key)] = [int(fr), int(sm)]
            else:
                e[0] = min(e[0], int(fr))
                e[1] = (e[1] + int(sm)) & ((1 << 64) - 1)
    order = sorted(merged.items(), key=lambda kv: kv[1][0])
    out_k = np.array([kk for kk, _ in order], dtype=np.uint64)
    out_f = np.array([v[0] for _, v in order], dtype=np.uint64)
    out_s = np.array([v[1] for _, v in order], dtype=np.uint64)
    return out_k, out_f, out_s


def delta_carry(lane_sums: np.ndarray, device="cpu") -> np.ndarray:
    """Exclusive lane-wise prefix of every rank's 8 lane sums (uint64, wrapping):
    the carry-in a delta_f shard needs to decode its first block."""
    torch, dist = _torch()
    t = _as_i64(np.asarray(lane_sums, np.uint64).reshape(8)).to(device)
    out = [torch.zeros_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(out, t)
    carry = np.zeros(8, dtype=np.uint64)
    for r in range(dist.get_rank()):
        carry = carry + out[r].cpu().numpy().view(np.uint64)
    return carry
