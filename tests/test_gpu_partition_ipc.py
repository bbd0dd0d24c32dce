"""Blocks partitioned over two or three processes, the halo rows stored straight into the other processes' arenas:
each process holds one rank's engine context, exports its stage buffers by CUDA IPC and maps its receivers'
(mosegpu.partition.DistPeerExchange over a gloo process group for the barriers and the MIN all-reduce of dt). The
processes share one GPU here; no kernel of one waits on another (every round ends with the streams drained and a
host barrier). The interiors after three steps equal one context holding every block, bit for bit."""
import os
import socket
import sys

import numpy as np
import pytest

from mosegpu import abi

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, precision, steps, q):
    try:
        _rank(rank, world, port, precision, steps, q)
    except Exception:
        import traceback
        q.put({"rank": rank, "error": traceback.format_exc()})
        raise


def _rank(rank, world, port, precision, steps, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, os.path.join(ROOT, "mose-gpu_b200"))
    import datetime

    import torch.distributed as dist
    from mosegpu import case as cs
    from mosegpu import partition as pt
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    case = cs.taylor_green(n=24, blocks=2)
    owner = pt.partition_blocks(case, world)
    ranks = [pt.split_case(case, owner, r) for r in range(world)]
    plan = pt.halo_plan(case, owner, ranks, visc=True)
    drv = pt.EngineRank(ranks[rank], precision=precision, device=0)
    ex = pt.DistPeerExchange(drv, plan, rank, world, dist)
    pt.step_rank(drv, ex, True, case.scheme["n_rk"], nsteps=steps)
    S = drv.state()
    st = drv.eng.status()
    ex.close()
    out = {"rank": rank, "code": st.code, "steps": st.steps, "time": st.time,
           "interior": {g: ranks[rank].case.interior(S, i).copy() for i, g in enumerate(ranks[rank].own)}}
    dist.destroy_process_group()
    q.put(out)


@pytest.mark.parametrize("nranks", [2, 3])
@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_processes_push_halo_rows_by_ipc(torch_cuda, precision, nranks):
    import torch.multiprocessing as mp
    from mosegpu import case as cs
    from mosegpu.engine import Engine
    steps = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, nranks, port, precision, steps, q)) for r in range(nranks)]
    for p in procs:
        p.start()
    try:
        res = [q.get(timeout=300) for _ in procs]
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert not any("error" in d for d in res), [d.get("error") for d in res]
    assert all(p.exitcode == 0 for p in procs)
    case = cs.taylor_green(n=24, blocks=2)
    one = Engine(case, precision=precision)
    one.step(steps, graph=False)
    P1 = one.state()
    st1 = one.status()
    got = {}
    for d in res:
        assert d["code"] == 0 and d["steps"] == steps and d["time"] == st1.time
        got.update(d["interior"])
    assert sorted(got) == list(range(len(case.blocks)))
    for g, v in got.items():
        assert np.array_equal(v, case.interior(P1, g)), g
