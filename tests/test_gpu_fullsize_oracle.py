"""The benchmarked configurations at their real sizes, against the CPU oracle (the size-dependent paths: 256-wide
tiles with their k-chunks, the persistent queue over 48 uneven blocks and 64 equal ones, 32-bit intra-block offsets,
the connection records between blocks of different extents).

  C2  Taylor-Green, one periodic block of 256^3, Navier-Stokes, Roe + van Albada, SSP-RK3
  C3  the 8 x 6 block 2-D batch of the seeded layout (3.0 M cells), walls + 405 inlet, AUSM+ / van Leer, RK4
  C5  Taylor-Green at Mach 0.3 with seeded noise, 4 x 4 x 4 blocks of 128^3 (134 M cells), HLLC + van Albada

Gates (per conserved variable, max-norm relative to the field): 1e-12 after one step, 1e-9 after several. The oracle
runs with OpenMP on the host's cores: about 7 s per step of C2, 2 s of C3, 60 s of C5.
"""
import numpy as np
import pytest

import helpers as H
from mosegpu import abi

pytestmark = pytest.mark.gpu

TOL_ONE = 1e-12
TOL_MANY = 1e-9


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _run_both(case, steps, precision=abi.PREC_FP64, time_tol=1e-14):
    """`steps` whole steps of the case from its initial state on the engine (step graph) and on the oracle, one
    chunk after the other; returns the conserved fields of both after each chunk."""
    import oracle
    from mosegpu.engine import Engine
    eng = Engine(case, precision=precision)
    orc = oracle.Oracle(case)
    P = case.P0.copy()
    out = []
    done = 0
    for n in steps:
        assert orc.step(P, n - done) == 0
        eng.step(n - done, graph=True)
        done = n
        so, sg = orc.status(), eng.status()
        assert sg.code == 0 and sg.steps == so.steps == n
        assert abs(sg.time - so.time) <= time_tol * so.time
        out.append((n, H.conserved(case, eng.state()), H.conserved(case, P)))
    eng.close()
    del orc
    return out


def _check(out, cid):
    for n, g, o in out:
        e = H.rel_err(g, o)
        tol = TOL_ONE if n == 1 else TOL_MANY
        assert np.all(e <= tol), (cid, n, e)


def test_c2_tgv256_against_the_oracle(torch_cuda):
    from mosegpu import case as cs
    case = cs.taylor_green(n=256, share_geometry=True)
    _check(_run_both(case, [1, 3]), "tgv256")


def test_c2_tgv256_fp64_production_form_against_the_oracle(torch_cuda):
    """The FP64 production form (FMA, simplified flux path) at 256^3: within the gates, not bit for bit."""
    from mosegpu import case as cs
    case = cs.taylor_green(n=256, share_geometry=True)
    _check(_run_both(case, [1, 3], precision=abi.PREC_FP64_FAST, time_tol=1e-12), "tgv256 fp64 fast")


def test_c3_batch2d_against_the_oracle(torch_cuda):
    from mosegpu import case as cs
    case = cs.multiblock_2d()                            # the seeded 8 x 6 layout of the benchmark
    assert len(case.blocks) == 48 and case.n_interior > 2_900_000
    _check(_run_both(case, [1, 10]), "mb2d_8x6")


def test_c5_tgv_64_blocks_against_the_oracle(torch_cuda):
    from mosegpu import case as cs
    case = cs.taylor_green_blocks()                      # 4 x 4 x 4 blocks of 128^3
    assert len(case.blocks) == 64
    _check(_run_both(case, [1]), "tgv_4x4x4_128")
