"""Parity of the B200 engine (through its C ABI) with the CPU oracle on the same seeded inputs.

Tolerances (the north-star gates, per conserved variable, max-norm relative to the field): 1e-12 after
one step, 1e-9 after the case's step count. The FP64 form is built without FMA contraction and keeps the
oracle's operation order, so most comparisons are expected to be exact; the tolerance is the bar.
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


def _pair(builder):
    import oracle
    from mosegpu.engine import Engine
    case = builder()
    return case, Engine(case), oracle.Oracle(case)


@pytest.mark.parametrize("cid,builder", H.small_cases(), ids=[c[0] for c in H.small_cases()])
def test_ghosts_and_residual(torch_cuda, cid, builder):
    case, eng, orc = _pair(builder)
    P = case.P0.copy()
    orc.fill_ghosts(P)
    eng.fill_ghosts()
    Pg = eng.state()
    assert np.array_equal(Pg, P), "ghost fill differs"
    Ro = orc.residual(P)
    Rg = eng.residual().cpu().numpy()
    e = H.rel_err(H.interior_rows(case, Rg), H.interior_rows(case, Ro), floor=1e-30)
    assert np.all(e <= TOL_ONE), (cid, e)


@pytest.mark.parametrize("cid,builder", H.small_cases(), ids=[c[0] for c in H.small_cases()])
def test_dt(torch_cuda, cid, builder):
    case, eng, orc = _pair(builder)
    d_o = orc.dt(case.P0)
    d_g = eng.dt()
    assert abs(d_g - d_o) <= 1e-14 * d_o, (d_g, d_o)


@pytest.mark.parametrize("cid,builder", H.small_cases(), ids=[c[0] for c in H.small_cases()])
def test_update_hook(torch_cuda, cid, builder):
    """mb_update alone (RK_Newstate) on the oracle's residual, every stage coefficient."""
    torch = torch_cuda
    case, eng, orc = _pair(builder)
    P = case.P0.copy()
    orc.fill_ghosts(P)
    R = orc.residual(P)
    dt = orc.dt(P)
    for irk in range(1, case.scheme["n_rk"] + 1):
        Po = P.copy()
        orc.update(Po, P, R, irk, dt)
        Pg = torch.from_numpy(P.copy()).cuda()
        eng.update(Pg, torch.from_numpy(P.copy()).cuda(), torch.from_numpy(R).cuda(), irk, dt)
        e = H.rel_err(H.conserved(case, Pg.cpu().numpy()), H.conserved(case, Po))
        assert np.all(e <= TOL_ONE), (irk, e)


@pytest.mark.parametrize("cid,builder", H.small_cases(), ids=[c[0] for c in H.small_cases()])
@pytest.mark.parametrize("graph", [False, True])
def test_one_step_and_many(torch_cuda, cid, builder, graph):
    case, eng, orc = _pair(builder)
    P = case.P0.copy()
    assert orc.step(P, 1) == 0
    eng.step(1, graph=graph)
    e1 = H.rel_err(H.conserved(case, eng.state()), H.conserved(case, P))
    assert np.all(e1 <= TOL_ONE), ("one step", e1)
    nmany = 15
    assert orc.step(P, nmany) == 0
    eng.step(nmany, graph=graph)
    en = H.rel_err(H.conserved(case, eng.state()), H.conserved(case, P))
    assert np.all(en <= TOL_MANY), ("%d steps" % (nmany + 1), en)
    so, sg = orc.status(), eng.status()
    assert sg.code == 0 and sg.steps == so.steps
    assert abs(sg.time - so.time) <= 1e-12 * so.time


@pytest.mark.parametrize("cid,builder", H.small_cases(), ids=[c[0] for c in H.small_cases()])
def test_fp64_production_form_within_the_gates(torch_cuda, cid, builder):
    """The FP64 production form (FP64 values, the simplified flux path with FMA contraction) against the oracle at
    the north-star gates: 1e-12 after one step, 1e-9 after 16 (not bit for bit: FMA and the reordered formulas)."""
    import oracle
    from mosegpu.engine import Engine
    case = builder()
    eng, orc = Engine(case, precision=abi.PREC_FP64_FAST), oracle.Oracle(case)
    P = case.P0.copy()
    assert orc.step(P, 1) == 0
    eng.step(1, graph=True)
    e1 = H.rel_err(H.conserved(case, eng.state()), H.conserved(case, P))
    assert np.all(e1 <= TOL_ONE), ("one step", e1)
    assert orc.step(P, 15) == 0
    eng.step(15, graph=True)
    en = H.rel_err(H.conserved(case, eng.state()), H.conserved(case, P))
    assert np.all(en <= TOL_MANY), ("16 steps", en)
    so, sg = orc.status(), eng.status()
    assert sg.code == 0 and sg.steps == so.steps
    assert abs(sg.time - so.time) <= 1e-11 * so.time


TMA_CASES = {"tgv24_2x2x2": lambda cs: cs.taylor_green(n=24, blocks=2),
             "mb2d_3x2": lambda cs: cs.multiblock_2d(cols=3, rows=2, lo=9, hi=40, seed=11),
             "sod300": lambda cs: cs.riemann_1d(n=300)}


@pytest.mark.parametrize("cid", sorted(TMA_CASES))
def test_tma_staging_matches_plain_staging(torch_cuda, cid, monkeypatch):
    """The mixed sweep stages its tiles by TMA (boxes of the state arena landing on an mbarrier) or, without a tensor
    map, by plain loads: the tile values, and so every result, are the same bit for bit."""
    from mosegpu import case as cs
    from mosegpu.engine import Engine
    case = TMA_CASES[cid](cs)
    if case.ncell % 2:                                   # the variable stride must be a multiple of 16 bytes
        pad = 1
        case.ncell += pad
        case.P0 = np.concatenate([case.P0, np.zeros((5, pad))], axis=1)
    a = Engine(case, precision=abi.PREC_MIXED)
    monkeypatch.setenv("MB_NO_TMA", "1")
    b = Engine(case, precision=abi.PREC_MIXED)
    monkeypatch.delenv("MB_NO_TMA")
    a.step(6, graph=True)
    b.step(6, graph=True)
    ta, pa = a.staging()
    tb, pb = b.staging()
    assert ta > 0 and pa == 0, (ta, pa)
    assert tb == 0 and pb > 0, (tb, pb)
    m = case.interior_mask()
    assert np.array_equal(a.state()[:, m], b.state()[:, m])
    sa, sb = a.status(), b.status()
    assert sa.code == 0 and sb.code == 0 and sa.time == sb.time


def test_staging_modes_agree_within_the_mixed_form(torch_cuda):
    """The mixed sweep's two tile stagings (TMA boxes into a 5-value tile, plain loads into a 6-value tile) differ in
    the FP32 rounding of p only: both stay within 1e-6 of each other (max-norm, per conserved variable, the momentum
    against its vector) after 10 steps of the 24^3 Taylor-Green field."""
    from mosegpu import case as cs
    from mosegpu.engine import Engine
    case = cs.taylor_green(n=24, blocks=2)
    a, b = Engine(case, precision=abi.PREC_MIXED), Engine(case, precision=abi.PREC_MIXED)
    b.set_staging(0)
    a.step(10, graph=True)
    b.step(10, graph=True)
    assert a.staging()[0] > 0 and b.staging() == (0, b.staging()[1]) and b.staging()[1] > 0
    e = H.rel_err(H.conserved(case, a.state()), H.conserved(case, b.state()))   # momentum against its vector
    assert np.all(e < 1e-6), e


def test_staging_mode_of_each_tile_list(torch_cuda):
    """mb_set_staging sets the staging of both tile lists and mb_get_staging_mode reports it; mb_autotune chooses
    each list's staging by time, and on a mesh of one-plane blocks only (the 2-D batch) reports the one-plane list's.
    The two stagings of the one-plane tiles agree within the mixed form's rounding of p."""
    from mosegpu import case as cs
    from mosegpu.engine import Engine
    case = cs.multiblock_2d(cols=3, rows=2, lo=9, hi=40, seed=11)
    a, b = Engine(case, precision=abi.PREC_MIXED), Engine(case, precision=abi.PREC_MIXED)
    a.set_staging(1)
    b.set_staging(0)
    assert a.staging_mode() == 1 and b.staging_mode() == 0
    assert b.staging_label() == "6-value tile, plain loads"
    a.step(8, graph=True)
    b.step(8, graph=True)
    e = H.rel_err(H.conserved(case, a.state()), H.conserved(case, b.state()))
    assert np.all(e < 1e-6), e
    a.autotune()
    assert a.staging_mode() in (0, 1)
    a.step(2, graph=True)
    assert a.status().code == 0 and a.status().steps == 10


def test_bounded_wait_runs_out_and_the_device_stays_usable(torch_cuda):
    """The TMA staging waits on its mbarrier with an iteration limit: a wait on a phase nothing completes gives up and
    the kernel returns (the device then runs the next work as usual)."""
    import ctypes as C
    from mosegpu import case as cs
    from mosegpu.engine import Engine, load_library
    gave = C.c_int(-1)
    assert load_library().mb_selftest_bounded_wait(0, 2000, C.byref(gave)) == abi.MB_OK
    assert gave.value == 1
    e = Engine(cs.taylor_green(n=12), precision=abi.PREC_MIXED)
    e.step(2, graph=False)
    assert e.status().code == 0 and e.status().steps == 2


def test_stage_by_stage_matches_fused(torch_cuda):
    """begin_step + stage(1..n) (the reference's call sequence) equals the fused mb_step."""
    from mosegpu import case as cs
    from mosegpu.engine import Engine
    case = cs.taylor_green(n=12, blocks=2)
    a, b = Engine(case), Engine(case)
    for _ in range(3):
        a.begin_step()
        for irk in range(1, 4):
            a.stage(irk)
    b.step(3, graph=False)
    assert np.array_equal(a.state()[:, case.interior_mask()], b.state()[:, case.interior_mask()])


def test_sod_to_t_end(torch_cuda):
    """The 1-D Sod config (1000 cells, HLLC + minmod, SSP-RK3, CFL 0.5) to t = 0.2: GPU = oracle, and
    both close to the exact solution."""
    import oracle
    from mosegpu import case as cs
    from mosegpu.engine import Engine
    case = cs.riemann_1d(n=1000)
    eng, orc = Engine(case), oracle.Oracle(case)
    P = case.P0.copy()
    no = orc.run_to(P, 0.2)
    ng = eng.run_to(0.2)
    assert no == ng
    e = H.rel_err(H.conserved(case, eng.state()), H.conserved(case, P))
    assert np.all(e <= TOL_MANY), e
    x = case.blocks[0]["centres"][:, 0, 0, 0]
    r, u, p = cs.exact_riemann((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), x, eng.status().time)
    rho = case.interior(eng.state(), 0)[0, :, 0, 0]
    assert np.abs(rho - r).mean() < 2e-3


@pytest.mark.parametrize("riemann", [abi.RS_LMROE, abi.RS_HLLC, abi.RS_HLLE, abi.RS_SLAU, abi.RS_AUSMP, abi.RS_LLF,
                                     abi.RS_SLAU2, abi.RS_EXACT, abi.RS_MICZEKROE, abi.RS_AUSMPM, abi.RS_HLLEPP,
                                     abi.RS_HLLC_TRAMEL, abi.RS_HLLC_CHEN])
def test_mixed_precision_error(torch_cuda, riemann):
    """The mixed form (FP32 flux arithmetic, FP64 state) against the FP64 form on a small TGV, every solver."""
    from mosegpu import case as cs
    from mosegpu.engine import Engine
    case = cs.taylor_green(n=24, riemann=riemann)
    a = Engine(case, precision=abi.PREC_FP64)
    b = Engine(case, precision=abi.PREC_MIXED)
    a.step(20, graph=True)
    b.step(20, graph=True)
    qa, qb = H.conserved(case, a.state()), H.conserved(case, b.state())
    l1, l2, li = H.norms(qb, qa)
    assert l2[0] < 1e-5, l2
    assert l2[4] < 1e-4, l2
    # the momentum as one vector field (w of this flow starts at zero: its own norm is no scale)
    dm = (qb[1:4] - qa[1:4]).reshape(3, -1)
    assert np.sqrt((dm * dm).sum()) < 1e-4 * np.sqrt((qa[1:4].reshape(3, -1) ** 2).sum()), l2


def test_state_check_reports_injected_nan(torch_cuda):
    """Failure detection with a host-injected bad input: a NaN cell is reported, nothing faults."""
    from mosegpu import case as cs
    from mosegpu.engine import Engine
    case = cs.riemann_1d(n=64)
    eng = Engine(case)
    P = case.P0.copy()
    case.interior(P, 0)[4, 10, 0, 0] = np.nan
    eng.set_state(P)
    eng.step(1, graph=False)
    st = eng.status()
    assert st.code == abi.MB_E_STATE and st.n_bad_state > 0
    assert st.bad_blk == 0 and st.bad_j == 1 and st.bad_k == 1


def test_thermo_guard_reports_off_table_temperature(torch_cuda):
    from mosegpu import case as cs
    from mosegpu.engine import Engine
    case = cs.taylor_green(n=12)
    eng = Engine(case)
    P = case.P0.copy()
    case.interior(P, 0)[4, 3, 3, 3] *= 60.0   # T ~ 18000 K, off the 10000 K table
    eng.set_state(P)
    eng.step(1, graph=False)
    st = eng.status()
    assert st.code == abi.MB_E_THERMO and st.n_bad_thermo > 0


@pytest.mark.parametrize("kchunk,persistent", [(8, 0), (32, 1), (5, 1)])
def test_tile_configuration_does_not_change_results(torch_cuda, kchunk, persistent):
    """The k-chunk of the tiles and the persistent work queue change only which CTA computes a face: the state
    after several steps is bit-identical to the default configuration, on a 3-D multi-block case and on the
    2-D wall / inlet batch; the autotuner's choice likewise."""
    from mosegpu import case as cs
    from mosegpu.engine import Engine
    for case in (cs.taylor_green(n=24, blocks=2, riemann=abi.RS_HLLC), cs.multiblock_2d(cols=2, rows=2, lo=9, hi=20,
                                                                                      seed=2)):
        a, b = Engine(case), Engine(case)
        b.set_tuning(kchunk, persistent)
        assert b.tuning()[:2] == (kchunk, persistent)
        a.step(4, graph=True)
        b.step(4, graph=True)
        m = case.interior_mask()
        assert np.array_equal(a.state()[:, m], b.state()[:, m])
        c = Engine(case)
        k, q, ms = c.autotune()
        assert k in (8, 16, 32, 64) and q in (0, 1) and ms > 0
        c.step(4, graph=True)
        assert np.array_equal(a.state()[:, m], c.state()[:, m])
        assert a.status().time == b.status().time == c.status().time


def test_multiblock_2d_many_steps_fp64_and_mixed(torch_cuda):
    """The 2-D wall / inlet batch (RK4, AUSM+, van Leer) for 30 steps: FP64 = oracle within the many-step gate,
    the mixed form within L2(rho) 1e-5 of FP64."""
    import oracle
    from mosegpu import case as cs
    from mosegpu.engine import Engine
    case = cs.multiblock_2d(cols=3, rows=2, lo=16, hi=40, seed=9)
    orc = oracle.Oracle(case)
    P = case.P0.copy()
    assert orc.step(P, 30) == 0
    a = Engine(case, precision=abi.PREC_FP64)
    b = Engine(case, precision=abi.PREC_MIXED)
    a.step(30, graph=True)
    b.step(30, graph=True)
    e = H.rel_err(H.conserved(case, a.state()), H.conserved(case, P))
    assert np.all(e <= TOL_MANY), e
    l1, l2, li = H.norms(H.conserved(case, b.state()), H.conserved(case, a.state()))
    assert l2[0] < 1e-5, l2


@pytest.mark.parametrize("cid", ["sod_hllc_minmod", "tgv_hllc_minmod_8blk", "mb2d_ausm_vanleer_rk4",
                                 "duct3d_hllc_vanleer", "tgv_irs2_roe_8blk"])
def test_residual_diagnostic_matches_the_oracle(torch_cuda, cid):
    """The residual diagnostic accumulated in the fused last stage (sum of (new - old)^2, reduced per tile) equals
    the oracle's after one and after several steps in the FP64 form; the mixed form's agrees to its accuracy."""
    import oracle
    from mosegpu.engine import Engine
    case = dict(H.small_cases())[cid]()
    orc = oracle.Oracle(case)
    eng = Engine(case)
    mix = Engine(case, precision=abi.PREC_MIXED)
    P = case.P0.copy()
    for n in (1, 6):
        assert orc.step(P, n) == 0
        eng.step(n, graph=(n > 1))
        mix.step(n, graph=(n > 1))
        want = np.array(orc.status().res[:])
        got = np.array(eng.status().res[:])
        scale = want.max()
        assert scale > 0
        assert np.all(np.abs(got - want) <= 1e-10 * scale), (got, want)
        gm = np.array(mix.status().res[:])
        assert np.all(np.abs(gm - want) <= 1e-3 * scale), (gm, want)


def test_residual_stop_matches_the_oracle(torch_cuda):
    """A case with a residual stop (res_stop between two steps' residuals) stops at the oracle's step, in the same
    state, and further steps leave it alone (the device clock marks it done)."""
    import oracle
    from mosegpu.engine import Engine
    case = dict(H.small_cases())["mb2d_ausm_vanleer_rk4"]()
    orc = oracle.Oracle(case)
    P = case.P0.copy()
    res = []
    for _ in range(10):
        assert orc.step(P, 1) == 0
        res.append(orc.status().res[0])
    thr = res[5] * (1.0 + 1e-8)
    assert all(abs(r - thr) > 1e-6 * thr for i, r in enumerate(res) if i != 5)   # no other residual near it
    k = next(i for i, r in enumerate(res) if r <= thr) + 1
    case.scheme["res_stop"] = thr
    eng = Engine(case)
    eng.step(12, graph=True)
    st = eng.status()
    assert st.done == 1 and st.steps == k, (st.steps, k, res)
    ref = oracle.Oracle(case)
    Pk = case.P0.copy()
    assert ref.step(Pk, 12) == 0 and ref.status().steps == k
    e = H.rel_err(H.conserved(case, eng.state()), H.conserved(case, Pk))
    assert np.all(e <= TOL_ONE), e


def test_record_params_changed_between_steps_match_the_oracle(torch_cuda):
    """A host-driven time-dependent inlet (the reference's 402: p0(t) handed to the records each step): the inlet
    records' stagnation pressure raised between steps through mb_set_record_params, the same on the oracle's
    records; the states stay equal."""
    import oracle
    from mosegpu.engine import Engine
    case = dict(H.small_cases())["duct3d_401_stagnation_inlet"]()
    eng, orc = Engine(case), oracle.Oracle(case)
    P = case.P0.copy()
    inlet = [q for q in range(len(case.rec)) if case.rec["type"][q] == abi.BC_INFLOW]
    assert inlet
    for n, p0 in ((3, 1.25e5), (3, 1.32e5), (3, 1.28e5)):
        for q in inlet:
            qv = np.array(case.rec["q"][q])
            qv[2] = p0
            eng.set_record_params(q, qv)
            orc.set_record_params(q, qv)
        assert orc.step(P, n) == 0
        eng.step(n, graph=True)
    e = H.rel_err(H.conserved(case, eng.state()), H.conserved(case, P))
    assert np.all(e <= TOL_MANY), e
    with pytest.raises(abi.MoseError):
        bad = np.array(case.rec["q"][inlet[0]])
        bad[1] = -1.0                                     # T0 <= 0 is rejected as at mb_init
        eng.set_record_params(inlet[0], bad)


@pytest.mark.parametrize("cid", ["tgv_irs2_roe_8blk", "mb2d_irs3_ausm_rk2_beta07", "duct3d_irs1_hllc_beta03",
                                 "mb2d_local_dt_ausm_rk3_rise10", "tgv_local_dt_roe_8blk", "sod_local_dt_irs2_hllc",
                                 "mb2d_prec_hllcpc_ns", "duct3d_prec_mach03_smooth2"])
def test_irs_mixed_within_gate_and_stages_match_fused(torch_cuda, cid):
    """With residual smoothing, local time stepping or preconditioning: the mixed form (FP32 fluxes; the smoothing,
    Ur, the preconditioned steps and the update in FP64; the local steps of the fused sweep in FP32) stays within
    L2(rho) 1e-5 of the FP64 form after 20 steps, and the reference's call sequence (begin_step + stage 1..n) equals
    mb_step bit for bit."""
    from mosegpu.engine import Engine
    case = dict(H.small_cases())[cid]()
    a = Engine(case, precision=abi.PREC_FP64)
    b = Engine(case, precision=abi.PREC_MIXED)
    a.step(20, graph=True)
    b.step(20, graph=True)
    assert a.status().code == 0 and b.status().code == 0
    l1, l2, li = H.norms(H.conserved(case, b.state()), H.conserved(case, a.state()))
    assert l2[0] < 1e-5, l2
    c, d = Engine(case), Engine(case)
    for _ in range(3):
        c.begin_step()
        for irk in range(1, case.scheme["n_rk"] + 1):
            c.stage(irk)
    d.step(3, graph=False)
    m = case.interior_mask()
    assert np.array_equal(c.state()[:, m], d.state()[:, m])
