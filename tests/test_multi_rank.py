"""The N > 1 path of bench.py on the CPU: two gloo ranks (the GPU run uses NCCL the same way). The replicas share
nothing but the timing reductions: the job's time is the maximum over ranks, every rank passes the same barriers, the
serving cases are partitioned over the ranks and their summaries merged, and in the reference arm rank 0 alone works
and prints while the other ranks exit 0 without work."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import numpy as np
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


# ---------------------------------------------------------------------------------------------------------------------
# Blocks partitioned over ranks (mosegpu/partition.py): the 2 x 2 x 2-block Taylor-Green field split over two gloo
# ranks, each rank stepping its own blocks with the oracle and exchanging its halo rows through the partition's
# schedule; the result must equal the one-rank oracle bit for bit.

class OracleRank:
    """One rank's blocks on the CPU restatement, with the rank-driver interface of partition.EngineRank."""

    def __init__(self, rank_case):
        import oracle
        self.rc = rank_case
        self.o = oracle.Oracle(rank_case.case)
        self.P = rank_case.case.P0.copy()
        self.PO = np.zeros_like(self.P)
        self.dt = None

    def set_stage(self, irk):
        pass                                   # the oracle updates P in place: every stage reads P

    def pack(self, rows, rnd, tag):
        import torch
        return torch.from_numpy(np.ascontiguousarray(self.P[:, rows]).ravel())

    def unpack(self, rows, buf):
        self.P[:, rows] = np.asarray(buf).reshape(5, len(rows))

    def local_dtmin(self):
        return self.o.dt(self.P)

    def start(self, dt):
        self.dt = dt
        self.PO[...] = self.P

    def stage(self, irk, part):
        if part == 0:
            self.o.fill_ghosts(self.P)
        else:
            # the oracle copies bc_pg at its ghost fill (Ghost_Connection_pairs_B), the engine's records read those
            # rows in place: after the round-2 rows have landed the fill runs again (the ghost values are the same,
            # the copied donor rows now current)
            self.o.fill_ghosts(self.P)
            R = self.o.residual(self.P)
            assert self.o.update(self.P, self.PO, R, irk, self.dt) == 0

    def state(self):
        return self.P


def _tgv_case():
    from mosegpu import case as cs
    return cs.taylor_green(n=12, blocks=2)


def _partition_rank_main(rank, world, port, q, steps):
    try:
        _partition_rank(rank, world, port, q, steps)
    except Exception:
        import traceback
        q.put({"rank": rank, "error": traceback.format_exc()})
        raise


def _partition_rank(rank, world, port, q, steps):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "mose-gpu_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import datetime

    import torch
    import torch.distributed as dist
    from mosegpu import partition as pt
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    case = _tgv_case()
    owner = pt.partition_blocks(case, world)
    ranks = [pt.split_case(case, owner, r) for r in range(world)]
    plan = pt.halo_plan(case, owner, ranks, visc=True)
    drv = OracleRank(ranks[rank])
    ex = pt.DistExchange(drv, plan, rank, world, torch.device("cpu"))
    pt.step_rank(drv, ex, True, case.scheme["n_rk"], nsteps=steps)
    out = {"rank": rank, "own": ranks[rank].own, "ext": ranks[rank].ext,
           "interior": {g: ranks[rank].case.interior(drv.state(), q).copy() for q, g in enumerate(ranks[rank].own)},
           "pairs": sorted(plan)}
    dist.destroy_process_group()
    q.put(out)


def test_partitioned_blocks_match_one_rank_bit_for_bit():
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "mose-gpu_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    steps = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_partition_rank_main, args=(r, 2, port, q, steps)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda d: d["rank"])
    assert not any("error" in d for d in res), [d.get("error") for d in res]
    case = _tgv_case()
    assert sorted(res[0]["own"] + res[1]["own"]) == list(range(8)) and len(res[0]["own"]) == 4
    assert res[0]["ext"] and res[1]["ext"] and res[0]["pairs"] == [(0, 1), (1, 0)]
    P = case.P0.copy()
    assert oracle.Oracle(case).step(P, steps) == 0
    for d in res:
        for g, v in d["interior"].items():
            assert np.array_equal(v, case.interior(P, g)), g


def test_partition_and_halo_plan_on_one_process():
    """The partition balances the cells, every remote donor block of a rank is one of its external copies, and the
    halo rows of each pair are rows of the owner's own blocks (round 1) or of its padded blocks (round 2)."""
    sys.path.insert(0, os.path.join(ROOT, "mose-gpu_b200"))
    from mosegpu import case as cs
    from mosegpu import partition as pt
    case = cs.taylor_green(n=24, blocks=3)                   # 27 blocks of 8^3
    for world in (2, 3, 4):
        owner = pt.partition_blocks(case, world)
        loads = [sum(int(np.prod(case.blocks[b]["n"])) for b in range(27) if owner[b] == r) for r in range(world)]
        assert max(loads) - min(loads) <= 512
        ranks = [pt.split_case(case, owner, r) for r in range(world)]
        plan = pt.halo_plan(case, owner, ranks, visc=True)
        for (src, dst), (s1, d1, s2, d2) in plan.items():
            assert src != dst and len(s1) == len(d1) and len(s2) == len(d2) and len(s1) > 0
            own_rows = np.zeros(ranks[src].case.ncell, dtype=bool)
            for q in range(len(ranks[src].own)):
                own_rows[ranks[src].case.blocks[q]["boff"] + np.arange(pt._padded(ranks[src].case.blocks[q]["n"]))] = True
            assert own_rows[s1].all() and own_rows[s2].all()
            ext_rows = np.zeros(ranks[dst].case.ncell, dtype=bool)
            n_own = len(ranks[dst].own)
            for q in range(n_own, n_own + len(ranks[dst].ext)):
                b = ranks[dst].case.blocks[q]
                ext_rows[b["boff"] + np.arange(pt._padded(b["n"]))] = True
            assert ext_rows[d1].all() and ext_rows[d2].all()
        for rc in ranks:
            for b in rc.case.blocks[len(rc.own):]:
                assert b["group"] == -1
            assert all(int(rc.case.rec[q]["blk"]) < len(rc.own) for q in range(len(rc.case.rec)))
