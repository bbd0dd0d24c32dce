"""The engine at the benchmarked sizes, where the CPU oracle is too slow to run alongside: properties that hold
whatever the size. The 256^3 Taylor-Green field (the headline case) conserves mass and total energy to round-off on
its periodic mesh and keeps a zero total momentum, in both forms; a 128^3 field split into 2 x 2 x 2 blocks joined by
connections matches the single periodic block to round-off (the connection records keep their own arithmetic); the
mixed form stays within the north-star gate of the FP64 form on the 2-D batch case."""
import numpy as np
import pytest

import helpers as H
from mosegpu import abi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _sums(case, P):
    q = H.conserved(case, P)                            # the interior cells' conserved variables
    return q.sum(axis=1), np.abs(q).sum(axis=1)


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_tgv256_conserves_mass_energy_and_zero_momentum(torch_cuda, precision):
    from mosegpu import case as cs
    from mosegpu.engine import Engine
    case = cs.taylor_green(n=256, share_geometry=True)
    eng = Engine(case, precision=precision)
    s0, a0 = _sums(case, case.P0)
    eng.step(5, graph=True)
    st = eng.status()
    assert st.code == 0 and st.steps == 5 and all(np.isfinite(st.res[:])) and st.res[0] > 0
    P = eng.state()
    s1, a1 = _sums(case, P)
    # uniform volumes, periodic: mass and total energy to round-off (the mixed form sums each cell's six FP32 net
    # face fluxes in FP32 before its FP64 update: its round-off is that of FP32 on the increments)
    tol = 1e-12 if precision == abi.PREC_FP64 else 1e-10
    assert abs(s1[0] - s0[0]) <= tol * a0[0]
    assert abs(s1[4] - s0[4]) <= tol * a0[4]
    # the field's momentum sums to zero and stays there, to the round-off of the form (the mixed form's FP32 fluxes
    # break the symmetry of the field at their own precision), measured on the momentum vector
    mtol = 1e-10 if precision == abi.PREC_FP64 else 1e-8
    for v in (1, 2, 3):
        assert abs(s1[v]) <= mtol * a1[1:4].sum()


def test_tgv128_blocks_match_one_block(torch_cuda):
    from mosegpu import case as cs
    from mosegpu.engine import Engine
    a = cs.taylor_green(n=128, blocks=1)
    b = cs.taylor_green(n=128, blocks=2, share_geometry=True)
    ea, eb = Engine(a), Engine(b)
    ea.step(5, graph=True)
    eb.step(5, graph=True)
    Pa, Pb = ea.state(), eb.state()
    full = np.zeros_like(a.interior(Pa, 0))
    for q, blk in enumerate(b.blocks):
        lo, n = blk["lo"], blk["n"]
        full[:, lo[0]:lo[0] + n[0], lo[1]:lo[1] + n[1], lo[2]:lo[2] + n[2]] = b.interior(Pb, q)
    e = H.rel_err(full, a.interior(Pa, 0))
    assert np.all(e < 1e-11), e


def test_batch2d_mixed_within_gate_of_fp64(torch_cuda):
    from mosegpu import case as cs
    from mosegpu.engine import Engine
    case = cs.multiblock_2d()                           # the 8 x 6 block batch of the benchmark (3.0 M cells)
    a = Engine(case, precision=abi.PREC_FP64)
    b = Engine(case, precision=abi.PREC_MIXED)
    a.step(50, graph=True)
    b.step(50, graph=True)
    l1, l2, li = H.norms(H.conserved(case, b.state()), H.conserved(case, a.state()))
    assert l2[0] < 1e-5, l2
    assert a.status().steps == 50 and b.status().steps == 50
