"""Sharded execution across GPUs (one process per GPU).

Tablets are independent, so a table is split into contiguous runs of whole
segments, one run per rank, and every rank runs the query over its own run
with no data exchanged.  A query's result is the concatenation of the ranks'
results in rank order (the single-core CPU VM's row order,
src/vm/virginia.c:476-578, since segment runs are contiguous), so the one
exchange the path has is each rank's result row count: an all-gather of one
integer per rank, whose exclusive prefix is the rank's first row in the
global result.  The collective runs on whatever process group the caller
set up (NCCL between GPUs, gloo on CPU).
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def segment_runs(seg_rows: Sequence[int], world: int) -> List[Tuple[int, int]]:
    """Contiguous runs of segments, one per rank, balanced by rows:
    rank r gets segments [runs[r][0], runs[r][1])."""
    total = sum(seg_rows)
    runs, start, acc = [], 0, 0
    for r in range(world):
        target = total * (r + 1) / world
        end = start
        while end < len(seg_rows) and (acc + seg_rows[end] <= target or end == start) and \
                len(seg_rows) - end > world - r - 1:
            acc += seg_rows[end]
            end += 1
        if r == world - 1:
            while end < len(seg_rows):
                acc += seg_rows[end]
                end += 1
        runs.append((start, end))
        start = end
    return runs


def exchange_counts(n: int, group=None, device: str = "cpu") -> Tuple[int, int]:
    """All-gather every rank's result row count; returns (this rank's first
    row in the global result, the global row count)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    if world == 1:
        return 0, n
    t = torch.tensor([n], dtype=torch.int64, device=device)
    out = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(out, t, group=group)
    counts = [int(x.item()) for x in out]
    r = dist.get_rank(group)
    return sum(counts[:r]), sum(counts)


def assign_tables(table_rows: Sequence[int], world: int) -> List[int]:
    """Whole tables per rank (the batched and serving workloads): each table
    has one owner, largest tables first onto the least-loaded rank (ties to
    the lower rank), so every rank computes the same assignment."""
    load = [0] * world
    owner = [0] * len(table_rows)
    for t in sorted(range(len(table_rows)), key=lambda i: (-int(table_rows[i]), i)):
        r = min(range(world), key=lambda k: (load[k], k))
        owner[t] = r
        load[r] += int(table_rows[t])
    return owner


def my_queries(query_tables: Sequence[int], owner: Sequence[int], rank: int) -> List[int]:
    """The queries a rank runs: those over the tables it owns, in order."""
    return [q for q, t in enumerate(query_tables) if owner[t] == rank]


def result_directory(nq: int, mine: Sequence[int], rows: Sequence[int], group=None,
                     device: str = "cpu") -> List[int]:
    """Every query's result row count on every rank: a query's result stays
    on the rank that ran it (its table's owner), and one all-reduce of the
    per-query counts tells every rank how long each result is."""
    import torch
    import torch.distributed as dist
    t = torch.zeros(nq, dtype=torch.int64, device=device)
    for q, n in zip(mine, rows):
        t[q] = int(n)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, group=group)
    return [int(x) for x in t.cpu().tolist()]
