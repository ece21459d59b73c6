#!/usr/bin/env python
"""Filter-scan benchmark of the B200 query VM.

Workload (one step = one query over one resident table): the 7-column
benchmark table at 50,000,000 rows held in HBM (seeded synthetic data, ~1.4 GB,
larger than the 126 MB L2, so no flush is needed between steps) and the scan +
arithmetic query

    SELECT id, uniformf + normalf5 * 2.5 AS fsum, normali20 / 3 AS idiv,
           uniformi - normali5 AS isub
    FROM test WHERE uniformf < c OR normalf20 > d

with c and d taken from the data so the filter keeps 10% of the rows
(headline); the sweep reports 0.1%, 1%, 10%, 50% and 99%.  The metric is
filter-scan GB/s of algorithmic bytes: rows x (strides of the columns the
program reads) + result rows x (result strides).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

With --gpus N > 1 (launched by torchrun, one rank per GPU) every rank scans
its own 50M-row shard (weak scaling) and the ranks all-gather their result
counts each step, the one exchange the path needs to place every shard's rows
in global order.  --impl reference times the reference's own CPU VM
(virginia_multi with every host thread, built from the reference sources) on
a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

ROWS = 50_000_000
HEADLINE_SEL = 0.10
METRIC = "filter scan GB/s (% HBM peak)"
WORKLOAD = ("device-resident filter scan + arithmetic (7-column table, 50M rows per GPU, "
            "10% selectivity)")
# DRAM bytes of the headline kernel per scanned row and per result row,
# from ncu (dram__bytes_read.sum, dram__bytes_write.sum) on an 8M-row launch
# of the same query: 229.66 MB read, 10.04 MB written for 800,581 result rows
TRAFFIC_READ_PER_ROW = 229.662976e6 / 8_000_000
TRAFFIC_WRITE_PER_RESULT_ROW = 10.035456e6 / 800_581
SWEEP = [0.001, 0.01, 0.10, 0.50, 0.99]
# the plain CPU-runnable filter (1M rows)
CONFIG1 = "SELECT id, uniformi, normali5 FROM test WHERE uniformi > 60 AND normali5 < 0"
QUERY = ("SELECT id, uniformf + normalf5 * 2.5 AS fsum, normali20 / 3 AS idiv, "
         "uniformi - normali5 AS isub FROM test WHERE uniformf < {c:.6f} OR normalf20 > {d:.6f}")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            with open(p) as f:
                return float(json.load(f)["hbm_gbs"]), "measured"
        except (OSError, ValueError, KeyError, TypeError):
            pass
    return 6650.0, "fallback"


def constants(cols, sel):
    """c and d such that the OR of the two independent conditions, each
    keeping q of the rows, keeps 1 - (1 - q)^2 = sel of them."""
    q = 1 - (1 - sel) ** 0.5
    c = float(np.quantile(cols["uniformf"][:4_000_000], q))
    d = float(np.quantile(cols["normalf20"][:4_000_000], 1 - q))
    return c, d


class Clocks:
    """nvidia-smi samples during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-i", str(self.device), "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p:
            time.sleep(0.15)
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        sm, smax, reasons, power = [], 0.0, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def allreduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def exchange_counts(n, world):
    """Each rank's first row in the global result (virginian_b200.shard)."""
    if world == 1:
        return 0, n
    from virginian_b200 import shard
    return shard.exchange_counts(n, device="cuda")


def pinned_table(n, seed):
    """The table's columns in pinned host memory (torch) as numpy views."""
    import torch
    from virginian_b200 import datagen
    cols = {}
    for name in ["id"] + [c for c, _ in datagen.SCHEMA_A]:
        arr = datagen.column(name, n, seed=seed) if name != "id" else np.arange(n, dtype=np.int32)
        t = torch.empty(n, dtype={np.dtype(np.int32): torch.int32,
                                  np.dtype(np.float32): torch.float32}[arr.dtype], pin_memory=True)
        t.numpy()[:] = arr
        cols[name] = (t, t.numpy())
    return cols


def cpu_baseline(sql_for, rows, threads, repeat=3):
    """The reference CPU VM on a bounded sample (same query, same columns)."""
    from oracle import oracle
    from virginian_b200 import datagen
    cols = datagen.table(rows, datagen.SCHEMA_A, seed=0)
    c, d = constants(cols, HEADLINE_SEL)
    sql = sql_for(c, d)
    db = oracle.OracleDB()
    try:
        db.create_table("test", datagen.SCHEMA_A)
        db.insert("test", cols["id"], [cols[x] for x, _ in datagen.SCHEMA_A])
        r = db.query(sql, mode=1 if threads > 1 else 0, threads=threads, repeat=repeat)
        out_rows = r.rows
        secs = r.seconds
    finally:
        db.close()
    alg = rows * 28 + out_rows * 16
    return alg / secs / 1e9, secs, out_rows


# ---- batched, serving and streamed workloads --------------------------------

_T0 = time.perf_counter()


def log(msg):
    print(f"[bench {time.perf_counter() - _T0:8.1f}s] {msg}", file=sys.stderr, flush=True)

def _accept_for(cat, types, layout=None):
    """compiles, decodes cleanly and, for the serving loop, fits its layout"""
    import virginian_b200 as vb

    def ok(q):
        try:
            c = cat.compile(q)
            p = vb.Program(c.op_list(), c.pc, types)
        except vb.VirgError:
            return False
        if p.maybe_undefined:
            return False
        if layout:
            i = p.info
            return (i.load_bytes_per_row <= layout[0] and i.row_vector_bytes <= layout[1]
                    and i.sel_vector_bytes <= layout[2])
        return True
    return ok


def _device_tables(eng, sizes, seed0, table_nos=None):
    """Resident tables of the benchmark schema generated on the GPU (table i
    seeded as table number table_nos[i], default i)."""
    import torch
    import virginian_b200 as vb
    from virginian_b200 import datagen
    types = [t for _, t in datagen.SCHEMA_A]
    tables = []
    for i, n in enumerate(sizes):
        segs, keep = datagen.device_table(int(n), datagen.SCHEMA_A,
                                          seed=seed0 + (i if table_nos is None else table_nos[i]))
        t = vb.Table(eng, types)
        t.append(segs)
        del segs, keep
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        tables.append(t)
    return tables


def _host_tables(eng, sizes, seed0, table_nos=None):
    """Resident tables of the benchmark schema from the seeded host generator
    (the reference CPU VM rebuilds the same bytes to check the results);
    table i is generated as table number table_nos[i] (default i)."""
    import virginian_b200 as vb
    from oracle.digest import host_table
    from virginian_b200 import datagen
    types = [t for _, t in datagen.SCHEMA_A]
    tables = []
    for i, n in enumerate(sizes):
        cols = host_table(int(n), seed0, i if table_nos is None else table_nos[i],
                          threads=min(16, os.cpu_count() or 1))
        t = vb.Table(eng, types)
        if n:
            t.append(datagen.segments(cols, datagen.SCHEMA_A))
        del cols
        tables.append(t)
    return tables


def _oracle_pool():
    """Worker processes (spawned, never forked from the CUDA process) that
    run the reference CPU VM for the parity checks."""
    import multiprocessing as mp
    return mp.get_context("spawn").Pool(max(1, min(16, os.cpu_count() or 1)))


def _same(got, want):
    """digests of one result stream: the same rows and, when there are rows,
    the same bytes column by column"""
    return got[0] == want[0] and (got[0] == 0 or tuple(got[1]) == tuple(want[1]))


def _queries(n, seed, ntables, layout=None):
    import virginian_b200 as vb
    from virginian_b200 import datagen, querygen, sql as vsql
    types = [t for _, t in datagen.SCHEMA_A]
    check = vsql.Catalog()
    check.add_table("test", datagen.SCHEMA_A)
    qs = querygen.generate(n, seed=seed, accept=_accept_for(check, types, layout))
    rng = np.random.default_rng(seed + 1)
    out = []
    for q, k in zip(qs, rng.integers(0, ntables, size=n)):
        c = check.compile(q)
        out.append((q, int(k), vb.Program(c.op_list(), c.pc, types)))
    return out


def bench_batched(eng, reps=5, world=1, rank=0):
    """256 generated queries over 64 resident tables of log-uniform size in
    [10k, 20M] rows: one persistent graph-replayed launch (autotuned shape)
    against one launch per query; every batched result compared with the
    reference CPU VM (virginia_single) on the same table.  With N ranks each
    rank holds the tables it owns (virginian_b200.shard.assign_tables) and
    runs the queries over them; times are the slowest rank's, and the result
    directory (every query's row count) is one all-reduce."""
    import torch
    import virginian_b200 as vb
    from oracle.digest import digest, table_digests_star
    from virginian_b200 import shard
    hbm, _ = peaks()
    rng = np.random.default_rng(404)
    sizes = np.exp(rng.uniform(np.log(1e4), np.log(2e7), size=64)).astype(np.int64)
    owner = shard.assign_tables([int(x) for x in sizes], world)
    mine_t = [k for k in range(len(sizes)) if owner[k] == rank]
    tables = dict(zip(mine_t, _host_tables(eng, [sizes[k] for k in mine_t], 1000, mine_t)))
    log("batched: tables ready")
    all_work = _queries(256, 77, len(sizes))
    mine = shard.my_queries([k for _, k, _ in all_work], owner, rank)
    work = [all_work[i] for i in mine]
    log("batched: per-query path")
    # one launch per query (the result count read back after each)
    for q, k, p in work[:8]:
        r = tables[k].query(p)
        _ = r.rows
        r.close()
    # the median of three passes (one pass varies by a third between runs)
    per_times = []
    for _ in range(3):
        barrier(world)
        t0 = time.perf_counter()
        per_rows = []
        for q, k, p in work:
            r = tables[k].query(p)
            per_rows.append(r.rows)
            r.close()
        per_times.append(allreduce_max(time.perf_counter() - t0, world))
    per_s = statistics.median(per_times)
    log("batched: batch path")
    b = vb.Batch(eng, autotune=True)
    for q, k, p in work:
        b.add(p, tables[k])
    b.run(graph=True)  # autotunes the shape, captures the graph
    b.wait()
    l0 = eng.launches
    b.run(graph=True)  # one replay, untimed: the kernel launches it holds
    b.wait()
    per_rep = eng.launches - l0
    stream = torch.cuda.ExternalStream(eng.stream)
    times, dev_ms = [], []
    for _ in range(reps):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(world)
        t0 = time.perf_counter()
        ev0.record(stream)
        b.run(graph=True)
        ev1.record(stream)
        b.wait()
        times.append(allreduce_max(time.perf_counter() - t0, world))
        ev1.synchronize()
        dev_ms.append(allreduce_max(ev0.elapsed_time(ev1), world))
    batch_s = statistics.median(times)
    batch_dev_ms = statistics.median(dev_ms)
    rows_equal = all(b.rows(i) == per_rows[i] for i in range(len(work)))
    log("batched: result digests")
    got = [digest(b.download(i)) for i in range(len(work))]
    shape = b.shape()
    b.close()
    directory = shard.result_directory(len(all_work), mine, [g[0] for g in got],
                                       device="cuda" if world > 1 else "cpu")
    alg_local = sum(int(sizes[k]) * p.info.load_bytes_per_row + got[i][0] * p.info.out_bytes_per_row
                    for i, (q, k, p) in enumerate(work))
    alg = alg_local
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([float(alg_local)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t)
        alg = int(t.item())
    for t in tables.values():
        t.close()
    out = {"workload": "256 generated queries (predicate trees of depth 1-4, 1-5 result columns) over 64 "
                       "resident tables, rows log-uniform in [1e4, 2e7]" +
                       ("" if world == 1 else f"; whole tables per rank over {world} ranks"),
           "tables": 64, "queries": len(all_work), "table_rows": int(sizes.sum()),
           "batched_qps": round(len(all_work) / batch_s, 1), "per_query_qps": round(len(all_work) / per_s, 1),
           "speedup": round(per_s / batch_s, 2), "batched_ms": round(batch_s * 1e3, 3),
           "batched_device_ms": round(batch_dev_ms, 3),
           "per_query_ms": round(per_s * 1e3, 3), "result_rows": int(sum(directory)),
           "algorithmic_bytes": int(alg),
           "batched_gbs": round(alg / (batch_dev_ms / 1e3) / 1e9, 1),
           "frac_of_hbm": round(alg / (batch_dev_ms / 1e3) / 1e9 / (hbm * world), 3),
           "rows_equal_per_query_path": bool(rows_equal), "shape": shape,
           "launches": {"batched_per_rep": per_rep, "per_query": len(work)}}
    if world > 1:
        out["queries_this_rank"] = len(work)
        out["oracle_checked"] = 0
        out["oracle_note"] = "checked at one GPU; the per-rank split changes which GPU runs a query, not its bytes"
        return out
    # the reference CPU VM on every (table, query): one task per table,
    # largest first, in spawned workers while the GPU idles
    log("batched: reference CPU VM on every query")
    by_table = {}
    for i, (q, k, p) in enumerate(work):
        by_table.setdefault(k, []).append(i)
    order = sorted(by_table, key=lambda k: -int(sizes[k]))
    t0 = time.perf_counter()
    with _oracle_pool() as pool:
        res = pool.map(table_digests_star, [(int(sizes[k]), 1000, k, [work[i][0] for i in by_table[k]])
                                            for k in order], chunksize=1)
    mismatch = []
    for k, digs in zip(order, res):
        for i, d in zip(by_table[k], digs):
            if not _same(got[i], d):
                mismatch.append(i)
    out.update({"oracle_checked": len(work), "oracle_mismatches": mismatch,
                "oracle_seconds": round(time.perf_counter() - t0, 1)})
    return out


def bench_serving(eng, rates=(1000, 10000, 50000), per_rate=300, world=1, rank=0):
    """The serving loop over 32 resident tables (~40 GB, 10M-200M rows each):
    Poisson arrivals of generated queries at each rate, latency from arrival
    to completion seen by the host, against serial one-launch-per-query
    execution of the same arrival sequence.  With N ranks each rank holds the
    tables it owns (virginian_b200.shard.assign_tables) and serves the
    arrivals over them; latencies are pooled over ranks."""
    import virginian_b200 as vb
    from virginian_b200 import shard
    rng = np.random.default_rng(505)
    raw = np.exp(rng.uniform(np.log(1e7), np.log(2e8), size=32))
    sizes = np.clip(raw * (1.43e9 / raw.sum()), 1e7, 2e8).astype(np.int64)
    owner = shard.assign_tables([int(x) for x in sizes], world)
    mine_t = [k for k in range(len(sizes)) if owner[k] == rank]
    tables = dict(zip(mine_t, _device_tables(eng, [sizes[k] for k in mine_t], 2000, mine_t)))
    log("serving: tables ready")
    layout = (32, 12, 20)
    all_work = _queries(per_rate, 88, len(sizes), layout)
    mine = shard.my_queries([k for _, k, _ in all_work], owner, rank)
    work = [all_work[i] for i in mine]
    srv = vb.Serve(eng, result_budget_bytes=20 << 30, max_load_bytes_per_row=layout[0],
                   max_row_vector_bytes=layout[1], max_sel_vector_bytes=layout[2])
    # warm: one query through each path
    t = srv.submit(work[0][2], tables[work[0][1]])
    srv.wait(t, timeout_s=120)
    srv.release(t)
    r = tables[work[0][1]].query(work[0][2])
    _ = r.rows
    r.close()
    out = {}
    import threading

    def pooled(xs):
        if world == 1:
            return list(xs)
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, list(xs))
        return [x for part in parts for x in part]

    for ri, rate in enumerate(rates):
        # the same queries at every rate; only the arrival process differs
        chunk = work
        log(f"serving: rate {rate}")
        gaps = np.random.default_rng(600 + ri).exponential(1.0 / rate, size=len(all_work))
        arrivals = (np.cumsum(gaps) - gaps[0])[mine]
        barrier(world)
        # a client thread consumes results as they complete and releases
        # their memory, while arrivals keep coming
        tickets, lag = [None] * len(chunk), [0.0] * len(chunk)
        lat, done_at, errors = [0.0] * len(chunk), [0.0] * len(chunk), []
        srows = [0] * len(chunk)
        ready = threading.Semaphore(0)

        def consume():
            try:
                for n in range(len(chunk)):
                    ready.acquire()
                    st = srv.wait(tickets[n], timeout_s=120)
                    lat[n] = lag[n] * 1e3 + st["latency_us"] / 1e3
                    done_at[n] = arrivals[n] + lat[n] / 1e3
                    srows[n] = st["rows"]
                    srv.release(tickets[n])
            except Exception as ex:  # surfaced after the join
                errors.append(ex)

        th = threading.Thread(target=consume)
        th.start()
        t0 = time.perf_counter()
        for n, ((q, k, p), at) in enumerate(zip(chunk, arrivals)):
            # wait for the arrival without holding the interpreter lock, so
            # the client thread keeps consuming results meanwhile
            while time.perf_counter() - t0 < at:
                time.sleep(0)
            lag[n] = time.perf_counter() - t0 - at
            tickets[n] = srv.submit(p, tables[k])
            ready.release()
        th.join()
        if errors:
            raise errors[0]
        serve_span = allreduce_max(max(done_at), world)
        barrier(world)
        # serial: one launch per query, in arrival order
        log(f"serving: serial at rate {rate}")
        slat, serial_rows = [], []
        t0 = time.perf_counter()
        for (q, k, p), at in zip(chunk, arrivals):
            while time.perf_counter() - t0 < at:
                pass
            r = tables[k].query(p)
            serial_rows.append(r.rows)
            r.close()
            slat.append((time.perf_counter() - t0 - at) * 1e3)
        serial_span = allreduce_max(time.perf_counter() - t0, world)
        bad_rows = pooled(mine[n] for n in range(len(chunk)) if srows[n] != serial_rows[n])
        lat, slat, lag = pooled(lat), pooled(slat), pooled(lag)
        out[str(rate)] = {
            "queries": len(all_work), "offered_qps": rate,
            "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
            "sustained_qps": round(len(all_work) / serve_span, 1),
            "serial_p50_ms": round(float(np.percentile(slat, 50)), 3),
            "serial_p99_ms": round(float(np.percentile(slat, 99)), 3),
            "serial_qps": round(len(all_work) / serial_span, 1),
            "submit_lag_p99_ms": round(float(np.percentile(lag, 99)) * 1e3, 3),
            "rows_checked": len(all_work), "rows_mismatch": bad_rows}
    if world > 1:
        st = srv.stats()
        srv.close()
        for t in tables.values():
            t.close()
        return {"workload": "32 resident tables, generated queries, Poisson arrivals; whole tables per rank "
                            f"over {world} ranks", "rates": out, "queries_this_rank": len(work),
                "sessions": st["sessions"], "readmitted": st["readmitted"], "sampled": st["sampled"]}
    # the look-back ring: queries back to back until the session's work
    # numbering has passed the ring's size, then the bytes of the last
    # results against the one-launch-per-query path
    log("serving: look-back ring wrap")
    ring = srv.stats()["status_ring"]
    inflight, wrap_rows_bad, submitted, last = [], [], 0, []
    per_rows = {}
    # programs of the narrow session layout (at most 8 filter-vector and 20
    # projection-vector bytes per row): a query needing the other layout
    # would end the session, and the ring only wraps within one session
    wrap_idx = [i for i, (_, _, p) in enumerate(work)
                if p.info.row_vector_bytes <= 8 and p.info.sel_vector_bytes <= 20]
    while submitted < 20000:
        n = wrap_idx[submitted % len(wrap_idx)]
        q, k, p = work[n]
        inflight.append((n, srv.submit(p, tables[k])))
        submitted += 1
        st = srv.stats()
        wrapped = st["work_items"] > ring + 200_000
        while len(inflight) > (0 if wrapped else 48):
            m, tk = inflight.pop(0)
            got = srv.download(tk) if wrapped else None
            rows = srv.wait(tk)["rows"]
            srv.release(tk)
            if m not in per_rows:
                r = tables[work[m][1]].query(work[m][2])
                per_rows[m] = r.rows
                r.close()
            if rows != per_rows[m]:
                wrap_rows_bad.append(m)
            if got is not None:
                last.append((m, got))
        if wrapped:
            break
    ring_work = st["work_items"]
    exact = True
    for m, got in last[-8:]:
        r = tables[work[m][1]].query(work[m][2])
        a = r.download()
        r.close()
        exact = exact and len(a) == len(got) and all(
            np.array_equal(x.view(np.uint8), y.view(np.uint8)) for x, y in zip(a, got))
    st = srv.stats()
    srv.close()
    total_rows = int(sizes.sum())
    for t in tables.values():
        t.close()
    return {"workload": "32 resident tables (rows log-uniform in [1e7, 2e8], %.1f GB), generated queries, "
                        "Poisson arrivals; latency from arrival to completion seen by the host" %
                        (total_rows * 28 / 1e9),
            "table_rows": total_rows, "result_budget_gb": 20, "rates": out,
            "ring_wrap": {"status_ring_words": ring, "session_work_items": ring_work,
                          "queries": submitted, "rows_mismatch": wrap_rows_bad,
                          "bytes_checked": min(8, len(last)), "bytes_equal": bool(exact and last)},
            "sessions": st["sessions"], "restarts": st["restarts"],
            "readmitted": st["readmitted"], "sampled": st["sampled"], "shape": st["shape"]}


STREAM_QUERY = ("SELECT id, uniformi, uniforml, normald FROM test "
                "WHERE normali20 > 15 AND uniformf < 50.0")


def bench_streamed(eng, rows=400_000_000, chunk=25_000_000):
    """400M rows of the 9-column schema in pinned host memory, streamed
    through the staging ring, against the same query on the table resident
    in HBM."""
    import torch
    import virginian_b200 as vb
    from virginian_b200 import datagen, sql as vsql
    schema = datagen.SCHEMA_B
    types = [t for _, t in schema]
    names = ["id"] + [c for c, _ in schema]
    dt = {"id": torch.int32, "uniformi": torch.int32, "normali5": torch.int32, "normali20": torch.int32,
          "uniformf": torch.float32, "normalf5": torch.float32, "normalf20": torch.float32,
          "uniforml": torch.int64, "normald": torch.float64}
    host = {nm: torch.empty(rows, dtype=dt[nm], pin_memory=True) for nm in names}
    for a in range(0, rows, chunk):
        b = min(rows, a + chunk)
        segs, keep = datagen.device_table(b - a, schema, seed=3000 + a // chunk, seg_rows=b - a)
        for nm, tsr in zip(names, keep):
            host[nm][a:b].copy_(tsr)
        if a:
            host["id"][a:b] += a
        del segs, keep
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    log("streamed: host data ready")
    seg_rows = 161_000 * 8
    segs = [{"rows": min(rows, a + seg_rows) - a,
             "key": host["id"][a:].data_ptr(),
             "cols": [host[c][a:].data_ptr() for c, _ in schema]} for a in range(0, rows, seg_rows)]
    cat = vsql.Catalog()
    cat.add_table("test", schema)
    c = cat.compile(STREAM_QUERY)
    p = vb.Program(c.op_list(), c.pc, types)
    r, st0 = vb.query_streamed(eng, p, segs, 4)
    r.close()
    runs = []
    for _ in range(3):
        r, st = vb.query_streamed(eng, p, segs, 4)
        n = r.rows
        r.close()
        runs.append(st)
    best = min(runs, key=lambda x: x["seconds"])
    # the same query on the table resident in HBM
    log("streamed: resident comparison")
    t = vb.Table(eng, types)
    t.append(segs)
    eng.timing(5)
    for _ in range(2):
        rr = t.query(p)
        _ = rr.rows
        rr.close()
    for _ in range(5):
        rr = t.query(p)
        nres = rr.rows
        rr.close()
    kms = statistics.median(eng.kernel_times(5))
    t.close()
    alg = rows * p.info.load_bytes_per_row + n * p.info.out_bytes_per_row
    del host
    return {"workload": "%dM rows of the 9-column schema (%.1f GB) in pinned host memory; %s" %
                        (rows // 1_000_000, rows * 48 / 1e9, STREAM_QUERY),
            "rows": rows, "result_rows": int(n), "h2d_bytes": int(best["h2d_bytes"]),
            "seconds": round(best["seconds"], 4),
            "host_link_gbs": round(best["h2d_bytes"] / best["seconds"] / 1e9, 2),
            "scan_gbs_streamed": round(alg / best["seconds"] / 1e9, 2),
            "resident_kernel_ms": round(kms, 3), "scan_gbs_resident": round(alg / (kms / 1e3) / 1e9, 1),
            "rows_equal": bool(nres == n)}


# ---- the reference's own entry points, in child processes -----------------

_DROPIN_CHILD = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, ROOT)
from virginian_b200 import _lib, datagen
_lib.lib()                                   # the GPU VM first, RTLD_GLOBAL
from oracle import oracle as O
from oracle.digest import host_table
n, sql, reps = int(sys.argv[1]), sys.argv[2], int(sys.argv[3])
cols = host_table(n, 41, 0, threads=8)
db = O.OracleDB(path=O.HOST_LIB, mode=ctypes.RTLD_GLOBAL)
db.create_table("test", datagen.SCHEMA_A)
db.insert("test", cols["id"], [cols[c] for c, _ in datagen.SCHEMA_A])
del cols
cpu = db.query(sql, mode=0)
gpu = db.query(sql, mode=2)
same = (gpu.tablet_rows == cpu.tablet_rows and len(gpu.columns) == len(cpu.columns) and
        all(a.tobytes() == b.tobytes() for a, b in zip(gpu.columns, cpu.columns)))
t_cpu = min(db.query(sql, mode=0).seconds for _ in range(reps))
runs = [db.query(sql, mode=2) for _ in range(reps)]
best = min(runs, key=lambda r: r.seconds)
db.close()
print("JSON " + json.dumps({"rows": n, "result_rows": int(cpu.rows), "result_tablets": len(cpu.tablet_rows),
                           "same_tablets_and_bytes": bool(same), "virginia_single_s": t_cpu,
                           "virg_vm_gpu_s": best.seconds, "h2d_s": best.gpu_timing[0],
                           "kernel_s": best.gpu_timing[1], "d2h_s": best.gpu_timing[2]}))
"""

_REFGPU_CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, ROOT)
from virginian_b200 import datagen
from oracle import oracle as O
from oracle.digest import host_table
n, sql = int(sys.argv[1]), sys.argv[2]
cols = host_table(n, 31, 0, threads=8)
db = O.OracleDB(path=O.REFGPU_LIB)
db.create_table("test", datagen.SCHEMA_A)
db.insert("test", cols["id"], [cols[c] for c, _ in datagen.SCHEMA_A])
del cols
runs = [db.query(sql, mode=2) for _ in range(3)]
best = min(runs, key=lambda r: r.gpu_timing[1])
db.close()
print("JSON " + json.dumps({"rows": n, "result_rows": int(best.rows), "kernel_s": best.gpu_timing[1],
                           "h2d_s": best.gpu_timing[0], "d2h_s": best.gpu_timing[2]}))
"""


def _child(script, *argv, timeout=900):
    p = subprocess.run([sys.executable, "-c", "ROOT = %r\n" % ROOT + script] + [str(a) for a in argv],
                       capture_output=True, text=True, timeout=timeout, cwd=ROOT)
    lines = [x for x in p.stdout.splitlines() if x.startswith("JSON ")]
    if p.returncode != 0 or not lines:
        raise RuntimeError((p.stdout + p.stderr)[-600:])
    return json.loads(lines[-1][5:])


def _headline_sql(n, seed):
    from oracle.digest import host_table
    cols = host_table(min(n, 4_000_000), seed, 0, threads=8)
    c, d = constants(cols, HEADLINE_SEL)
    return QUERY.format(c=c, d=d)


def bench_dropin(eng):
    """virg_query with the drop-in virg_vm_gpu against virg_query on
    virginia_single, inside the unmodified reference host library (stock
    virginian.h: 64 memory tablets of 8 MB, so the larger tables page
    tablets through the library's own database file), same database and
    query, result-tablet chains compared tablet by tablet."""
    out = {}
    for name, n, sql in (("config1_1M", 1_000_000, None), ("config2_8M", 8_000_000, "h"),
                         ("config2_50M", 50_000_000, "h")):
        q = CONFIG1 if sql is None else _headline_sql(n, 41)
        try:
            r = _child(_DROPIN_CHILD, n, q, 3)
            r["speedup"] = round(r["virginia_single_s"] / r["virg_vm_gpu_s"], 2)
            out[name] = r
        except Exception as ex:  # report, keep the others
            out[name] = {"error": f"{type(ex).__name__}: {ex}"}
    return out


def bench_ref_gpu_vm(eng):
    """The reference's own GPU VM (src/vm/vm_gpu.cu compiled for sm_100a,
    unordered results) on 8M rows of config 1 and of the headline query:
    its kernel seconds (vm->timing2, serial transfer mode) next to this
    VM's kernel time on the same rows resident in HBM."""
    import virginian_b200 as vb
    from oracle.digest import host_table
    from virginian_b200 import datagen, sql as vsql
    n = 8_000_000
    types = [t for _, t in datagen.SCHEMA_A]
    cols = host_table(n, 31, 0, threads=8)
    t = vb.Table(eng, types)
    t.append(datagen.segments(cols, datagen.SCHEMA_A))
    cat = vsql.Catalog()
    cat.add_table("test", datagen.SCHEMA_A)
    c, d = constants(cols, HEADLINE_SEL)
    del cols
    out = {}
    for name, q in (("config1", CONFIG1), ("config2_10pct", QUERY.format(c=c, d=d))):
        comp = cat.compile(q)
        p = vb.Program(comp.op_list(), comp.pc, types)
        for _ in range(3):
            r = t.query(p)
            rows = r.rows
            r.close()
        eng.timing(10)
        for _ in range(10):
            r = t.query(p)
            r.close()
        ours_ms = statistics.median(eng.kernel_times(10))
        try:
            ref = _child(_REFGPU_CHILD, n, q)
            out[name] = {"rows": n, "result_rows": rows, "ref_kernel_ms": round(ref["kernel_s"] * 1e3, 3),
                         "ref_result_rows": ref["result_rows"], "kernel_ms": round(ours_ms, 4),
                         "speedup": round(ref["kernel_s"] * 1e3 / ours_ms, 1)}
        except Exception as ex:
            out[name] = {"error": f"{type(ex).__name__}: {ex}", "kernel_ms": round(ours_ms, 4)}
    t.close()
    return out


def run_reference(args):
    """The reference's own CPU VM (virginia_multi with every host thread,
    built from the reference sources) on the headline workload: the same
    seeded 50M-row table and query, one query per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    rows = args.rows
    from oracle import oracle
    from oracle.digest import host_table
    from virginian_b200 import datagen
    cols = host_table(rows, 0, 0, threads=min(16, threads))
    c, d = constants(cols, HEADLINE_SEL)
    sql = QUERY.format(c=c, d=d)
    db = oracle.OracleDB()
    times = []
    try:
        db.create_table("test", datagen.SCHEMA_A)
        db.insert("test", cols["id"], [cols[x] for x, _ in datagen.SCHEMA_A])
        del cols
        out_rows = 0
        for i in range(args.warmup + args.steps):
            r = db.query(sql, mode=1, threads=threads, repeat=1)
            out_rows = r.rows
            if i >= args.warmup:
                times.append(r.seconds)
    finally:
        db.close()
    alg = rows * 28 + out_rows * 16
    total = sum(times)
    value = alg * len(times) / total / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total / len(times) * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32/float32", "data": "synthetic",
        "rows_per_s": round(rows * len(times) / total, 1),
        "config": {"workload": WORKLOAD, "rows_per_step": rows, "query": sql, "same_config": rows == ROWS,
                   "result_rows": out_rows},
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"the whole {rows}-row table and the headline query per step, "
                                   "virginia_multi (src/vm/virginia.c) built from the reference sources"},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_b200(args):
    world, rank, local = dist_setup(args.gpus)
    import torch
    import virginian_b200 as vb
    from virginian_b200 import datagen, sql as vsql

    torch.cuda.set_device(local)
    rows = args.rows
    log(f"headline: generating {rows} rows")
    pcols = pinned_table(rows, seed=rank)
    cols = {k: v[1] for k, v in pcols.items()}
    types = [t for _, t in datagen.SCHEMA_A]
    cat = vsql.Catalog()
    cat.add_table("test", datagen.SCHEMA_A)

    def program(sel):
        c, d = constants(cols, sel)
        comp = cat.compile(QUERY.format(c=c, d=d))
        return vb.Program(comp.op_list(), comp.pc, types)

    eng = vb.Engine(local)
    segs = datagen.segments(cols, datagen.SCHEMA_A)
    table = vb.Table(eng, types)
    table.append(segs)
    stream = torch.cuda.ExternalStream(eng.stream)
    load_b = None

    def alg_bytes(p, out_rows):
        return rows * p.info.load_bytes_per_row + out_rows * p.info.out_bytes_per_row

    def timed(p, steps, warmup):
        # pick the launch shape for this program and table (untimed; cached)
        if args.shape:
            eng.set_shape(*args.shape)
        else:
            vb.tune(eng, p, table)
        for _ in range(warmup):
            r = table.query(p)
            n = r.rows
            r.close()
        eng.timing(max(steps, 1))
        barrier(world)
        torch.cuda.synchronize()
        l0 = eng.launches
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            r = table.query(p)
            if world > 1:
                exchange_counts(r.rows, world)
            r.close()
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        ms = ev0.elapsed_time(ev1)
        kt = eng.kernel_times(steps)
        launches = eng.launches - l0
        err = eng.device_error()
        if err:
            raise RuntimeError(f"device error {err}")
        return n, ms, kt, launches

    # headline
    log("headline: table resident, timing")
    p = program(HEADLINE_SEL)
    with Clocks(local) as clk:
        out_rows, ms, kt, launches = timed(p, args.steps, args.warmup)
    ms_max = allreduce_max(ms, world)
    alg = alg_bytes(p, out_rows)
    # every rank processes the same number of bytes up to its result rows;
    # sum the algorithmic bytes over ranks
    alg_total = alg
    if world > 1:
        t = torch.tensor([alg], dtype=torch.float64, device="cuda")
        import torch.distributed as dist
        dist.all_reduce(t)
        alg_total = float(t.item())
    value = alg_total * args.steps / (ms_max / 1e3) / 1e9
    rows_per_s = rows * world * args.steps / (ms_max / 1e3)
    kernel_ms = statistics.mean(kt) if kt else None
    hbm, peak_kind = peaks()
    achieved = alg / (kernel_ms / 1e3) / 1e9 if kernel_ms else None
    from oracle.digest import digest
    r = table.query(p)
    head_digest = digest(r.download())
    r.close()
    # the read ceiling of the same columns: kernels that only read them
    ceiling = {}
    load_cols = [-1] + list(range(len(types)))
    for name, mode in (("loads_16B", 0), ("bulk_copies", 1)):
        cms, cbytes = table.read_ceiling(load_cols, mode, 5)
        ceiling[name] = {"ms": round(cms, 4), "gbs": round(cbytes / (cms / 1e3) / 1e9, 1)}

    # selectivity sweep (device-resident)
    log("sweep")
    sweep = {}
    for sel in SWEEP:
        ps = program(sel)
        n, sms, skt, _ = timed(ps, max(20, args.steps // 5), 2)
        km = statistics.mean(skt)
        sweep[f"{sel:g}"] = {"result_rows": n, "ms_per_step": round(sms / max(20, args.steps // 5), 4),
                             "kernel_ms": round(km, 4),
                             "gbs": round(alg_bytes(ps, n) / (km / 1e3) / 1e9, 1),
                             "frac_of_hbm": round(alg_bytes(ps, n) / (km / 1e3) / 1e9 / hbm, 3)}

    # end to end through the C ABI from pinned host buffers
    log("e2e")
    info = p.info
    outs = [torch.empty(max(out_rows, 1) + 1024, dtype={0: torch.int32, 2: torch.float32}[info.out_type[j]],
                        pin_memory=True) for j in range(info.nout)]
    import ctypes
    from virginian_b200._lib import lib as vlib
    seg_arr, keep = vb._segments(segs, types)
    ptrs = (ctypes.c_void_p * info.nout)(*[o.data_ptr() for o in outs])
    nrows = ctypes.c_uint64()
    e2e_steps = max(3, min(args.steps // 50, 10))
    vb.check(vlib().virg_gpu_query_host(eng.h, p.h, seg_arr, len(segs), ptrs, out_rows + 1024,
                                        ctypes.byref(nrows)), "query_host")
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        vb.check(vlib().virg_gpu_query_host(eng.h, p.h, seg_arr, len(segs), ptrs, out_rows + 1024,
                                            ctypes.byref(nrows)), "query_host")
        if world > 1:
            exchange_counts(nrows.value, world)
    e2e_s = time.perf_counter() - t0
    e2e_s = allreduce_max(e2e_s, world)
    assert nrows.value == out_rows
    e2e_same = _same(digest([o.numpy()[:out_rows] for o in outs]), head_digest)
    e2e_value = alg_total * e2e_steps / e2e_s / 1e9
    h2d = rows * info.load_bytes_per_row
    d2h = out_rows * info.out_bytes_per_row

    line = None
    if rank == 0:
        cpu = None
        if args.cpu_baseline and world == 1:
            log("cpu baseline")
            v1, s1, _ = cpu_baseline(lambda c, d: QUERY.format(c=c, d=d), args.cpu_rows, 1)
            cpu = {"value": round(v1, 3), "unit": "GB/s", "cores": 1, "kind": "reference",
                   "sample": f"{args.cpu_rows} rows of the same table and query, virginia_single "
                             "(src/vm/virginia.c) built from the reference sources, best of 3"}
            vm_, sm_, _ = cpu_baseline(lambda c, d: QUERY.format(c=c, d=d), args.cpu_rows,
                                       os.cpu_count() or 1)
            cpu_multi = {"value": round(vm_, 3), "unit": "GB/s", "cores": os.cpu_count(),
                         "kind": "reference", "vm": "virginia_multi"}
        shape = eng.last_launch()
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32/float32", "data": "synthetic",
            "config": {"workload": WORKLOAD,
                       "rows_per_gpu": rows, "query": QUERY.format(c=constants(cols, 0.1)[0],
                                                                   d=constants(cols, 0.1)[1]),
                       "result_rows": out_rows, "l2": "inputs larger than L2 (1.4 GB per step)",
                       "launch": shape},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1) if achieved else None,
                         "peak": hbm, "unit": "GB/s",
                         "frac": round(achieved / hbm, 4) if achieved else None,
                         "traffic": int(rows * TRAFFIC_READ_PER_ROW + out_rows * TRAFFIC_WRITE_PER_RESULT_ROW),
                         "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture "
                                           "of this kernel on 8M rows of the same query, scaled by rows",
                         "peak_kind": peak_kind,
                         "kernel_ms": round(kernel_ms, 4) if kernel_ms else None,
                         "algorithmic_bytes": alg},
            "rows_per_s": round(rows_per_s, 1),
            "read_ceiling": dict(ceiling, frac_of_bulk=round(achieved / ceiling["bulk_copies"]["gbs"], 3)
                                 if achieved else None),
            "sweep": sweep,
            "e2e": {"value": round(e2e_value, 3), "unit": "GB/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                    "ms_per_step": round(e2e_s / e2e_steps * 1e3, 3),
                    "same_bytes_as_device_path": bool(e2e_same)},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        if cpu:
            line["cpu_baseline"] = cpu
            line["cpu_multicore"] = cpu_multi
    del keep
    table.close()
    # the other workloads: batched and serving on every rank (whole tables
    # per rank); the others on one GPU, rank 0 (the sharded path covers the
    # scan)
    sections = [x for x in args.sections.split(",") if x]
    eng.set_shared_scan(args.shared_scan)
    for name, fn, multi in (("batched", bench_batched, True), ("serving", bench_serving, True),
                            ("streamed", bench_streamed, False), ("dropin", bench_dropin, False),
                            ("ref_gpu_vm", bench_ref_gpu_vm, False)):
        if name not in sections or (world > 1 and not multi):
            continue
        log(name)
        try:
            if multi:
                res = fn(eng, world=world, rank=rank)
            elif name == "streamed":
                res = fn(eng, rows=args.stream_rows, chunk=min(25_000_000, args.stream_rows))
            else:
                res = fn(eng)
        except Exception as ex:  # report, keep the headline line
            res = {"error": f"{type(ex).__name__}: {ex}"}
        if name == "batched":
            res["shared_scan"] = args.shared_scan
        if rank == 0:
            line[name] = res
    if rank == 0 and args.parity:
        # the headline's own result against the reference CPU VM
        # (virginia_single) on the same table, in a spawned worker
        log("parity: reference CPU VM on the headline table")
        from oracle.digest import table_digests_star
        sql = QUERY.format(c=constants(cols, HEADLINE_SEL)[0], d=constants(cols, HEADLINE_SEL)[1])
        t0 = time.perf_counter()
        with _oracle_pool() as pool:
            want = pool.map(table_digests_star, [(rows, rank, 0, [sql], 8)])[0][0]
        line["parity"] = {"config2_50M" if rows == ROWS else f"config2_{rows}": _same(head_digest, want),
                          "rows": want[0], "checked_against": "virginia_single (src/vm/virginia.c) built from "
                                                              "the reference sources, same table and query",
                          "seconds": round(time.perf_counter() - t0, 1)}
    if rank == 0:
        print(json.dumps(line))
    eng.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--rows", type=int, default=ROWS)
    ap.add_argument("--cpu-rows", type=int, default=4_000_000)
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--shape", default="", help="threads,stage_kb,stages,ctas_per_sm,chunk_rows: force the launch "
                    "shape of the scan instead of tuning it (for profiling one launch)")
    ap.add_argument("--stream-rows", type=int, default=400_000_000,
                    help="rows of the streamed section's host table (400M: the streamed workload)")
    ap.add_argument("--no-parity", dest="parity", action="store_false",
                    help="skip the headline's byte comparison with the reference CPU VM")
    ap.add_argument("--shared-scan", action="store_true",
                    help="batched queries over one table claim its chunks interleaved (shared scans)")
    ap.add_argument("--sections", default="batched,serving,streamed,dropin,ref_gpu_vm",
                    help="workloads besides the headline scan (comma list; empty for none)")
    args = ap.parse_args()
    args.shape = tuple(int(x) for x in args.shape.split(",")) if args.shape else ()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
