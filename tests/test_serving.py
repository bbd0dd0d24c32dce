"""Continuous batching (mosegpu.serving): the request stream and the arena allocator on the CPU; on the GPU,
each case served in a batch -- admitted while others run, queued when the HBM budget is full -- ends
bit-identical to the same case run alone through the single-case engine (tolerance 0: the cases share
launches but no arithmetic)."""
import math

import numpy as np
import pytest

from mosegpu import abi
from mosegpu import serving as sv


def test_request_stream_is_seeded_and_in_range():
    a = sv.request_stream(n_cases=400, rate=2.0, seed=5)
    b = sv.request_stream(n_cases=400, rate=2.0, seed=5)
    assert a == b
    t = np.array([x[0] for x in a])
    assert (np.diff(t) > 0).all()
    assert abs(len(a) / t[-1] - 2.0) < 0.5                       # Poisson rate
    d1 = [x for x in a if x[1] == 1]
    d2 = [x for x in a if x[1] == 2]
    assert 150 < len(d1) < 250
    assert all(256 <= x[2] <= 8192 and x[4] == 0.15 for x in d1)
    assert all(128 <= x[2] <= 1024 and x[4] == 0.25 for x in d2)
    for x in d1:
        for r, u, p in x[3]:
            assert 0.1 <= r <= 2 and -1 <= u <= 1 and 0.1 <= p <= 10
    # log-uniform: the median of log N sits mid-range
    med = np.median([math.log(x[2]) for x in d1])
    assert abs(med - 0.5 * (math.log(256) + math.log(8192))) < 0.4


def test_arena_ranges_first_fit_and_coalesce():
    r = sv._Ranges(100)
    a = r.alloc(30); b = r.alloc(30); c = r.alloc(30)
    assert (a, b, c) == (0, 30, 60) and r.alloc(20) is None
    r.release(b, 30)
    assert r.alloc(40) is None and r.alloc(25) == 30
    r.release(30, 25); r.release(a, 30); r.release(c, 30)
    assert r.free == [(0, 100)]


def test_riemann_request_initial_states():
    q = sv.riemann_request(0, 2, 16, [(1, 0, 0, 1), (2, 0.5, 0, 2), (3, 0, -0.5, 3), (4, 0, 0, 4)], 0.25)
    I = q.case.interior(q.case.P0, 0)[:, :, :, 0]
    assert I[0, -1, -1] == 1 and I[0, 0, -1] == 2 and I[0, 0, 0] == 3 and I[0, -1, 0] == 4
    assert I[1, 0, -1] == 0.5 and I[2, 0, 0] == -0.5 and I[4, 0, 0] == 3


def _alone(req, precision):
    from mosegpu.engine import Engine
    e = Engine(req.case, precision=precision)
    e.run_to(req.t_end, chunk=8)
    st = e.status()
    out = e.state()
    e.close()
    return out, st


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_batched_cases_equal_each_case_alone(precision):
    reqs = [sv.riemann_request(0, 1, 60, [(1.0, 0.0, 1.0), (0.125, 0.0, 0.1)], 0.15, arrival=0.0),
            sv.riemann_request(1, 2, 20, [(1.5, 0, 0, 1.5), (0.53, 1.2, 0, 0.3), (0.14, 1.2, 1.2, 0.03),
                                          (0.53, 0, 1.2, 0.3)], 0.25, arrival=0.0),
            sv.riemann_request(2, 1, 90, [(0.4, 0.5, 3.0), (1.7, -0.8, 0.7)], 0.15, arrival=0.01),
            sv.riemann_request(3, 2, 24, [(1.0, 0.2, -0.1, 2.0), (0.3, -0.5, 0.4, 0.6), (1.9, 0.9, 0.0, 9.0),
                                          (0.8, 0.0, 0.7, 4.0)], 0.25, arrival=0.02)]
    srv = sv.Server(reqs[0].case.scheme, reqs[0].case.thermo, budget_bytes=1 << 30, max_cases=8,
                    precision=precision, poll_steps=7)
    done = srv.serve(reqs, max_wall=120.0)
    srv.close()
    assert len(done) == len(reqs)
    for r in done:
        want, st = _alone(r, precision)
        assert r.status.code == abi.MB_OK and r.status.done == 1
        assert r.status.steps == st.steps and r.status.time == st.time
        m = r.case.interior_mask()
        assert np.array_equal(r.result[:, m], want[:, m]), r.rid


@pytest.mark.gpu
def test_admission_waits_for_budget_and_overlaps_running_cases():
    mk = lambda rid, n, t: sv.riemann_request(rid, 1, n, [(1.0, 0.0, 1.0), (0.125, 0.0, 0.1)], 0.15, arrival=t)  # noqa
    reqs = [mk(0, 400, 0.0), mk(1, 300, 0.0), mk(2, 500, 0.0), mk(3, 200, 0.001), mk(4, 2000, 0.002)]
    assert reqs[0].npad == 25 * 404            # (n + 4) x 5 x 5 padded cells of a 1-D case
    rows = reqs[0].npad + reqs[1].npad + 10     # room for the first two cases only; case 4 never fits
    srv = sv.Server(reqs[0].case.scheme, reqs[0].case.thermo, budget_bytes=1 << 30, max_cases=4,
                    precision=abi.PREC_FP64, poll_steps=5, arena_rows=rows)
    done = {r.rid: r for r in srv.serve(reqs, max_wall=120.0)}
    srv.close()
    assert sorted(done) == [0, 1, 2, 3, 4]
    assert done[4].error == abi.MB_E_BUDGET and done[4].result is None
    del done[4]
    # 0 and 1 ran together; 2 and 3 could only start after a case had left the arena
    assert done[0].admit_round == done[1].admit_round
    assert done[1].start < done[0].finish and done[0].start < done[1].finish
    first_out = min(done[0].finish, done[1].finish)
    assert done[2].start >= first_out and done[3].start >= first_out
    for r in done.values():
        want, _ = _alone(r, abi.PREC_FP64)
        m = r.case.interior_mask()
        assert np.array_equal(r.result[:, m], want[:, m]), r.rid


@pytest.mark.gpu
def test_two_lanes_run_independently_and_match_alone():
    """1-D cases in one lane, 2-D cases in another (each its own context and stream): every case ends
    bit-identical to itself alone."""
    reqs = [sv.riemann_request(0, 1, 300, [(1.0, 0.0, 1.0), (0.125, 0.0, 0.1)], 0.15, arrival=0.0),
            sv.riemann_request(1, 2, 40, [(1.5, 0, 0, 1.5), (0.53, 1.2, 0, 0.3), (0.14, 1.2, 1.2, 0.03),
                                          (0.53, 0, 1.2, 0.3)], 0.25, arrival=0.0),
            sv.riemann_request(2, 1, 120, [(0.4, 0.5, 3.0), (1.7, -0.8, 0.7)], 0.15, arrival=0.005)]
    mk = lambda: sv.Server(reqs[0].case.scheme, reqs[0].case.thermo, budget_bytes=1 << 29, max_cases=4,  # noqa
                           precision=abi.PREC_FP64, poll_steps=9)
    lanes = [mk(), mk()]
    done = sv.serve_lanes(lanes, lambda r: 0 if r.case.blocks[0]["n"][1] == 1 else 1, reqs, max_wall=120.0)
    for lane in lanes:
        lane.close()
    assert sorted(r.rid for r in done) == [0, 1, 2]
    for r in done:
        want, st = _alone(r, abi.PREC_FP64)
        assert r.status.done == 1 and r.status.steps == st.steps
        m = r.case.interior_mask()
        assert np.array_equal(r.result[:, m], want[:, m]), r.rid
