"""The reference's own 1-D regression cases (tests/golden/reference_1d_cases.npz) through the engine's C ABI: the FP64
parity form writes, after one iteration, exactly the field.tec of the oracle (same md5); the FP64 production form
(the same scheme with FMA contraction and the simplified formulas) stays within the one-step gate of it but prints a
different file. That difference is what a 15-digit md5 pin measures: the arithmetic's last bits, compiler choices
included (tests/test_reference_fixtures.py)."""
import hashlib

import numpy as np
import pytest

import helpers as H
import refcases
from mosegpu import abi
from test_reference_fixtures import CASES, ORACLE_MD5, REFERENCE_STEPS, field_md5

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _one_iteration(case, precision):
    from mosegpu.engine import Engine
    e = Engine(case, precision=precision)
    e.step(1, graph=False)
    st = e.status()
    assert st.code == 0 and st.steps == 1
    P = e.state()
    e.close()
    return P, st.time


@pytest.mark.parametrize("name", CASES)
def test_parity_form_writes_the_oracle_field(torch_cuda, name, tmp_path):
    case = refcases.load(name)
    P, t = _one_iteration(case, abi.PREC_FP64)
    assert field_md5(case, P, t, tmp_path / "field.tec") == ORACLE_MD5[name]


def test_contraction_changes_the_printed_field(torch_cuda, tmp_path):
    changed = {}
    for name in CASES:
        case = refcases.load(name)
        Pa, ta = _one_iteration(case, abi.PREC_FP64)
        Pb, tb = _one_iteration(case, abi.PREC_FP64_FAST)
        e = H.rel_err(H.conserved(case, Pb), H.conserved(case, Pa))
        assert np.all(e <= 1e-12), (name, e)
        fa, fb = tmp_path / ("a_%s.tec" % name), tmp_path / ("b_%s.tec" % name)
        field_md5(case, Pa, ta, fa)
        field_md5(case, Pb, tb, fb)
        la, lb = open(fa).read().split("\n"), open(fb).read().split("\n")
        changed[name] = sum(x != y for x, y in zip(la, lb))
    print("printed lines that differ between the two FP64 builds after one iteration:", changed)
    assert sum(changed.values()) > 0, changed


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_FP64_FAST, abi.PREC_MIXED])
def test_engine_runs_take_the_reference_steps(torch_cuda, precision):
    """Each reference case run to its time-threshold on the GPU: the FP64 forms take the reference's own number of
    steps (docs/vv/mose-comparison.md), the mixed form (dt in FP32) the same within one step."""
    from mosegpu.engine import Engine
    for name in CASES:
        case = refcases.load(name)
        e = Engine(case, precision=precision)
        n = e.run_to(case.scheme["time_threshold"])
        st = e.status()
        e.close()
        assert st.code == 0
        if precision == abi.PREC_MIXED:
            assert abs(n - REFERENCE_STEPS[name]) <= 1, (name, n)
        else:
            assert n == REFERENCE_STEPS[name], (name, n)
