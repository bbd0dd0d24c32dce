"""mb_dt_block_noalloc: Compute_dt of one block for callers that cannot allocate device memory (a host whose
device arrays belong to another runtime, a serving loop at its HBM budget, code that must not synchronise
the device or is capturing a CUDA graph). Its only scratch is a static device array; this file checks it
through the C ABI against the context-based mb_dt, call after call, so that contents left in that shared
array by one call cannot leak into the next. Collected last (the name sorts after the other test files)."""
import ctypes as C

import numpy as np
import pytest

from mosegpu import abi
from mosegpu import case as cs
from mosegpu import engine

pytestmark = pytest.mark.gpu

TOL = 1e-14


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _bind():
    L = engine.load_library()
    f = L.mb_dt_block_noalloc
    vp = C.c_void_p
    f.argtypes = [vp, C.c_int64, C.c_int64, C.POINTER(C.c_int32), vp, vp, vp, vp, vp, C.c_int32, C.c_int32,
                  C.c_double, C.POINTER(abi.MBScheme), vp, vp]
    f.restype = C.c_int
    return f


class Caller:
    """The device inputs of one block of a case as a caller without an engine context would hold them."""

    def __init__(self, torch, case, blk=0):
        dev = torch.device("cuda", 0)
        b = case.blocks[blk]
        self.n = (C.c_int32 * 3)(*b["n"])
        self.boff = b["boff"]
        self.ncell = case.ncell
        self.dl = torch.from_numpy(b["dl"]).to(dev)
        self.m = torch.from_numpy(b["m"]).to(dev)
        th = case.thermo
        self.cp = torch.from_numpy(th["cp"]).to(dev)
        self.mu = torch.from_numpy(th["mu"]).to(dev)
        self.k = torch.from_numpy(th["k"]).to(dev)
        self.th = th
        self.sc = case.scheme_struct()
        self.out = torch.zeros(1, dtype=torch.float64, device=dev)
        self.torch = torch

    def dt(self, f, P):
        s = self.torch.cuda.current_stream()
        rc = f(P.data_ptr(), self.ncell, self.boff, self.n, self.dl.data_ptr(), self.m.data_ptr(),
               self.cp.data_ptr(), self.mu.data_ptr(), self.k.data_ptr(), self.th["tmin"], self.th["tmax"],
               self.th["wm"], C.byref(self.sc), self.out.data_ptr(), C.c_void_p(s.cuda_stream))
        assert rc == abi.MB_OK, rc
        return float(self.out.item())


def test_dt_without_allocation_matches_mb_dt(torch_cuda):
    f = _bind()
    tgv = cs.taylor_green(n=40)                       # Navier-Stokes, additive rule, 2 x 5 x 3 tiles
    sod = cs.riemann_1d(n=300)                        # Euler, min rule, another tile count
    e_tgv, e_sod = engine.Engine(tgv), engine.Engine(sod)
    c_tgv, c_sod = Caller(torch_cuda, tgv), Caller(torch_cuda, sod)
    calls = []
    # two calls in a row on different blocks, then a third on the TGV after two steps changed its field
    calls.append((c_tgv.dt(f, e_tgv.P), e_tgv.dt()))
    calls.append((c_sod.dt(f, e_sod.P), e_sod.dt()))
    e_tgv.step(2, graph=False)
    calls.append((c_tgv.dt(f, e_tgv.P), e_tgv.dt()))
    for got, want in calls:
        assert abs(got - want) <= TOL * want, (got, want)
    assert calls[0][0] != calls[2][0]


def test_block_with_a_row_offset_in_a_multi_block_arena(torch_cuda):
    """A block that does not start at row 0 (boff > 0) of an 8-block arena: the flow of the last block is made the
    fastest, so the minimum step of the whole case lies there and mb_dt must equal that block's own minimum."""
    f = _bind()
    case = cs.taylor_green(n=16, blocks=2)            # 8 blocks of 8^3 cells in one arena
    last = len(case.blocks) - 1
    assert case.blocks[last]["boff"] > 0
    P = np.array(case.P0, copy=True)
    case.block_view(P, last)[1:4] *= 3.0              # Mach 0.3 in the last block, 0.1 elsewhere
    e = engine.Engine(case)
    e.set_state(P)
    want = e.dt()
    got = [Caller(torch_cuda, case, b).dt(f, e.P) for b in range(len(case.blocks))]
    assert abs(got[last] - want) <= TOL * want, (got[last], want)
    assert min(got) == got[last]
    assert all(g > want * (1 + 1e-3) for g in got[:last])


def test_cfl_rise_ramp_is_left_to_the_caller(torch_cuda):
    """During the cfl-rise ramp mb_dt scales the minimum by iter / cfl_rise; this entry point returns the minimum
    without the ramp (stated in the header), so the caller's product reproduces mb_dt."""
    f = _bind()
    sod = cs.riemann_1d(n=200)
    sod.scheme["cfl_rise"] = 10
    e = engine.Engine(sod)
    c = Caller(torch_cuda, sod)
    got, want = c.dt(f, e.P), e.dt()                  # first step: iter 1, factor 1 / 10
    assert abs(got * (1.0 / 10.0) - want) <= TOL * want, (got, want)


def test_oversized_block_is_rejected_before_any_launch(torch_cuda):
    f = _bind()
    sc = cs.taylor_green(n=8).scheme_struct()
    n = (C.c_int32 * 3)(32 * 4096, 8 * 32, 1)          # 4096 x 32 = 131072 (i, j) tiles > 65536
    dummy = C.c_void_p(1)                               # never dereferenced: the size check comes first
    rc = f(dummy, 1 << 40, 0, n, dummy, dummy, dummy, dummy, dummy, 0, 10000, 28.97, C.byref(sc), dummy, None)
    assert rc == abi.MB_E_ARG
