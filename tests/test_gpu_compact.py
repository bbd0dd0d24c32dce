"""One-plane blocks without k-face records on the GPU path: the engine takes them as extrapolated k faces, so the
compact case (implicit k faces) and the same case with the k-face records written out (oracle.explicit_k_records)
step bit for bit alike in both forms, and the FP64 parity form equals the oracle."""
import numpy as np
import pytest

import helpers as H
from mosegpu import abi
from mosegpu import case as cs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _implicit(case):
    """The case without its k-face records (the connections renumbered)."""
    keep = case.rec["face"] < 5
    old = np.nonzero(keep)[0]
    remap = -np.ones(len(case.rec), dtype=np.int64)
    remap[old] = np.arange(old.size)
    out = cs.Case(case.name + "_implicit_k")
    out.__dict__.update(case.__dict__)
    out.rec = case.rec[keep].copy()
    out.conn = case.conn.copy()
    if len(out.conn):
        out.conn["rec"] = remap[case.conn["rec"]]
    return out


CASES = {"riemann2d_40": lambda: cs.riemann_2d(n=40, compact=True),
         "riemann1d_96": lambda: cs.riemann_1d(n=96, compact=True),
         "mb2d_ns_3x2": lambda: _implicit(cs.multiblock_2d(cols=3, rows=2, lo=9, hi=30, seed=7))}


@pytest.mark.parametrize("cid", sorted(CASES))
@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_implicit_k_faces_equal_explicit_records(torch_cuda, cid, precision):
    import oracle
    from mosegpu.engine import Engine
    comp = CASES[cid]()
    assert not np.any(comp.rec["face"] >= 5)
    full = cs.Case(comp.name + "_explicit")
    full.__dict__.update(comp.__dict__)
    full.rec, full.conn = oracle.explicit_k_records(comp)
    steps = 6
    a, b = Engine(comp, precision=precision), Engine(full, precision=precision)
    a.step(steps, graph=True)
    b.step(steps, graph=True)
    m = comp.interior_mask()
    assert np.array_equal(a.state()[:, m], b.state()[:, m])
    sa, sb = a.status(), b.status()
    assert sa.code == 0 and sb.code == 0 and sa.time == sb.time
    if precision == abi.PREC_FP64:
        P = comp.P0.copy()
        o = oracle.Oracle(comp)
        assert o.step(P, steps) == 0
        e = H.rel_err(H.conserved(comp, a.state()), H.conserved(comp, P))
        assert np.all(e == 0.0), e
