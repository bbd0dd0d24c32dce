"""The N > 1 path of bench.py on the CPU: two gloo ranks (the GPU run uses NCCL the same way). The replicas share
nothing but the timing reductions: the job's time is the maximum over ranks, every rank passes the same barriers, the
serving cases are partitioned over the ranks and their summaries merged, and in the reference arm rank 0 alone works
and prints while the other ranks exit 0 without work."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch
    import bench
    w, r, local, pg = bench.dist_setup(backend="gloo", timeout_s=60)
    dev = torch.device("cpu")
    out = {"world": w, "rank": r}
    bench.barrier(pg, dev)
    out["max"] = bench.max_over_ranks(pg, 1.5 + rank, dev)            # per-rank times 1.5, 2.5 -> 2.5
    bench.barrier(pg, dev)
    # serving: the cases partitioned over the ranks, every rank's part gathered and merged as bench does
    mine = bench.partition_requests(list(range(10)), world, rank)
    part = ([0.5 * (x + 1) for x in mine], 0.0 + rank, 10.0 + rank, 100 * len(mine), len(mine), [])
    parts = [None] * world
    pg.all_gather_object(parts, part)
    out["mine"], out["merged"] = mine, bench.merge_serving(parts)
    # the reference arm: ranks other than 0 return at once without work or output
    if rank != 0:
        buf = io.StringIO()
        args = type("A", (), {"n": 8, "steps": 1, "warmup": 1})()
        with redirect_stdout(buf):
            out["ref_rc"] = bench.run_reference(args)
        out["ref_out"] = buf.getvalue()
    pg.destroy_process_group()
    q.put(out)


def test_two_gloo_ranks_time_as_the_max_over_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda d: d["rank"])
    assert [d["world"] for d in res] == [2, 2]
    assert [d["max"] for d in res] == [2.5, 2.5]
    assert res[1]["ref_rc"] == 0 and res[1]["ref_out"] == ""
    assert sorted(res[0]["mine"] + res[1]["mine"]) == list(range(10)) and not set(res[0]["mine"]) & set(res[1]["mine"])
    m = res[0]["merged"]
    assert m == res[1]["merged"]
    assert m["cases_completed"] == 10 and m["makespan_s"] == 11.0 and m["p50_s"] == 2.75
    assert m["cell_updates_per_s"] == 1000 / 11.0 and m["failed"] == []


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    w, r, local, pg = bench.dist_setup()
    assert (w, r, local, pg) == (1, 0, 0, None)
    assert bench.max_over_ranks(None, 3.25, None) == 3.25
