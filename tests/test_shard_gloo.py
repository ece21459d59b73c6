"""Host logic of sharded execution on two CPU ranks (gloo): each rank filters
its own contiguous run of segments, the ranks exchange only their result
counts, and every rank's rows placed at its offset give the single-table
result in order.  The per-rank result here is a numpy restatement of the
query's filter on the rank's rows (the oracle VM is exercised elsewhere);
what is tested is the partitioning, the exchange and the placement."""
import os
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from virginian_b200 import datagen, shard

N = 300_001
SEG = 40_000


def _rank(rank, world, port, outdir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cols = datagen.table(N, datagen.SCHEMA_A, seed=7)
        seg_rows = [min(SEG, N - a) for a in range(0, N, SEG)]
        lo, hi = shard.segment_runs(seg_rows, world)[rank]
        a, b = sum(seg_rows[:lo]), sum(seg_rows[:hi])
        keep = (cols["uniformi"][a:b] > 60) & (cols["normali5"][a:b] < 0)
        mine = cols["id"][a:b][keep]
        first, total = shard.exchange_counts(len(mine))
        out = np.lib.format.open_memmap(os.path.join(outdir, "out.npy"), mode="r+")
        out[first:first + len(mine)] = mine
        out.flush()
        with open(os.path.join(outdir, f"total{rank}"), "w") as f:
            f.write(str(total))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_shards_place_rows_in_global_order(world):
    cols = datagen.table(N, datagen.SCHEMA_A, seed=7)
    want = cols["id"][(cols["uniformi"] > 60) & (cols["normali5"] < 0)]
    with tempfile.TemporaryDirectory() as d:
        np.lib.format.open_memmap(os.path.join(d, "out.npy"), mode="w+", dtype=np.int32,
                                  shape=(len(want),))[:] = -1
        port = 29400 + world + (os.getpid() % 500)
        mp.start_processes(_rank, args=(world, port, d), nprocs=world, start_method="spawn")
        got = np.load(os.path.join(d, "out.npy"))
        assert np.array_equal(got, want)
        for r in range(world):
            with open(os.path.join(d, f"total{r}")) as f:
                assert int(f.read()) == len(want)


def test_segment_runs_cover_every_segment_once():
    for seg_rows in ([5], [3, 3, 3], [10, 1, 1, 1, 10], [232992] * 17 + [1000]):
        for world in (1, 2, 3, 4):
            if world > len(seg_rows):
                continue
            runs = shard.segment_runs(seg_rows, world)
            assert runs[0][0] == 0 and runs[-1][1] == len(seg_rows)
            assert all(runs[i][1] == runs[i + 1][0] for i in range(world - 1))
            assert all(hi > lo for lo, hi in runs)


def _rank_tables(rank, world, port, outdir):
    """Config-4 style: whole tables per rank; each rank runs the queries over
    its tables (here a numpy restatement of a per-table filter) and the
    ranks all-reduce the per-query row counts into one directory."""
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes = [int(x) for x in np.random.default_rng(404).integers(1, 40_000, size=13)]
        qt = [int(x) for x in np.random.default_rng(5).integers(0, len(sizes), size=40)]
        owner = shard.assign_tables(sizes, world)
        mine = shard.my_queries(qt, owner, rank)
        rows = []
        for q in mine:
            cols = datagen.table(sizes[qt[q]], datagen.SCHEMA_A, seed=qt[q])
            rows.append(int(((cols["uniformi"] > q % 100) & (cols["normali5"] < 0)).sum()))
        directory = shard.result_directory(len(qt), mine, rows)
        np.save(os.path.join(outdir, f"dir{rank}.npy"), np.array(directory))
        np.save(os.path.join(outdir, f"mine{rank}.npy"), np.array(mine, dtype=np.int64))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_tables_per_rank_directory(world):
    sizes = [int(x) for x in np.random.default_rng(404).integers(1, 40_000, size=13)]
    qt = [int(x) for x in np.random.default_rng(5).integers(0, len(sizes), size=40)]
    want = []
    for q, t in enumerate(qt):
        cols = datagen.table(sizes[t], datagen.SCHEMA_A, seed=t)
        want.append(int(((cols["uniformi"] > q % 100) & (cols["normali5"] < 0)).sum()))
    with tempfile.TemporaryDirectory() as d:
        port = 29600 + world + (os.getpid() % 300)
        mp.start_processes(_rank_tables, args=(world, port, d), nprocs=world, start_method="spawn")
        ran = np.concatenate([np.load(os.path.join(d, f"mine{r}.npy")) for r in range(world)])
        assert sorted(ran.tolist()) == list(range(len(qt)))  # every query once
        for r in range(world):
            assert np.load(os.path.join(d, f"dir{r}.npy")).tolist() == want


def test_assign_tables_balances_and_is_deterministic():
    sizes = [int(x) for x in np.exp(np.random.default_rng(404).uniform(np.log(1e4), np.log(2e7), size=64))]
    for world in (1, 2, 4, 8):
        owner = shard.assign_tables(sizes, world)
        assert owner == shard.assign_tables(list(sizes), world)
        load = [sum(s for s, o in zip(sizes, owner) if o == r) for r in range(world)]
        assert set(owner) == set(range(world))
        assert max(load) <= sum(sizes) / world + max(sizes)
