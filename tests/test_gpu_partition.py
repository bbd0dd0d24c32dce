"""Blocks partitioned over ranks on the GPU path (mosegpu/partition.py through the C ABI): two ranks emulated as two
engine contexts on one GPU (mb_step_prepare / mb_copy_dtmin / mb_step_start, the split stages, the halo rows moved
by mb_pack_rows / mb_unpack_rows, or stored straight into the receiver's arena by mb_push_rows), stepped in the order a
two-process run follows, against one context holding every block. No kernel of one rank waits on the other: the
exchange is stream-ordered between the steps' calls."""
import numpy as np
import pytest

from mosegpu import abi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("exchange", ["copies", "peer stores", "peer stores, own streams"])
@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
@pytest.mark.parametrize("nranks", [2, 3])
def test_partitioned_engine_matches_one_context(torch_cuda, precision, nranks, exchange):
    from mosegpu import case as cs
    from mosegpu import partition as pt
    from mosegpu.engine import Engine
    case = cs.taylor_green(n=24, blocks=2)                 # 8 blocks of 12^3, periodic connections everywhere
    steps = 3
    owner = pt.partition_blocks(case, nranks)
    ranks = [pt.split_case(case, owner, r) for r in range(nranks)]
    plan = pt.halo_plan(case, owner, ranks, visc=True)
    streams = [torch_cuda.cuda.Stream() if "own streams" in exchange else None for _ in ranks]
    drivers = [pt.EngineRank(rc, precision=precision, stream=st) for rc, st in zip(ranks, streams)]
    ex = pt.LocalExchange(drivers, plan) if exchange == "copies" else pt.PeerExchange(drivers, plan)
    pt.step_ranks(drivers, ex, True, case.scheme["n_rk"], nsteps=steps)
    one = Engine(case, precision=precision)
    one.step(steps, graph=False)
    P1 = one.state()
    Pr = pt.gather_interiors(case, ranks, [d.state() for d in drivers])
    for b in range(len(case.blocks)):
        assert np.array_equal(case.interior(Pr, b), case.interior(P1, b)), b
    st = [d.eng.status() for d in drivers]
    assert all(s.code == 0 and s.steps == steps for s in st)
    assert len({s.time for s in st}) == 1 and st[0].time == one.status().time


def test_peer_access_entry_point(torch_cuda):
    """mb_enable_peer: the same device is success; a device against every other GPU of the node either succeeds (twice:
    already enabled is success) or reports that there is no peer path."""
    from mosegpu.engine import load_library
    L = load_library()
    assert L.mb_enable_peer(0, 0) == abi.MB_OK
    assert L.mb_enable_peer(-1, 0) == abi.MB_E_ARG
    for peer in range(1, torch_cuda.cuda.device_count()):
        rc = L.mb_enable_peer(0, peer)
        assert rc in (abi.MB_OK, abi.MB_E_UNSUPPORTED)
        if rc == abi.MB_OK:
            assert L.mb_enable_peer(0, peer) == abi.MB_OK
