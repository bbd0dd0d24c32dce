"""The oracle's wall, inlet and RK4 paths against known answers (no GPU): a gas at rest in a closed
curvilinear box stays at rest (walls balance the pressure exactly), a uniform supersonic stream entering
through a 405 inlet whose state is the stream's own leaves a zero residual, outward flow closes a 405
face (no mass through it), the no-slip wall drags a tangential stream, an isothermal wall conducts the
heat k (T_wall - T) / (dy / 2) into a gas at rest, symmetry faces act as the extrapolated faces of a
transversely uniform tube, a 406 outlet at the stream's pressure passes a subsonic stream unchanged and
one below it draws more mass out, inward flow closes a 406 face, the 401 / 403 / 404 / 407 inlets fed with the
stagnation or mass-flux state of a uniform subsonic stream pass it unchanged, and classical RK4 converges at
fourth order in time (SSP-RK3 at third) on a smooth periodic problem."""
import math

import numpy as np
import pytest

import helpers as H
import oracle
from mosegpu import abi
from mosegpu import case as cs

WALLS = {1: abi.BC_WALL, 2: abi.BC_WALL, 3: abi.BC_WALL, 4: abi.BC_WALL, 5: abi.BC_EXTRAPOLATION,
         6: abi.BC_EXTRAPOLATION}


def _residual(case):
    o = oracle.Oracle(case)
    P = case.P0.copy()
    o.fill_ghosts(P)
    return o, P, o.residual(P)


@pytest.mark.parametrize("riemann", [abi.RS_HLLC, abi.RS_AUSMP, abi.RS_LMROE])
def test_gas_at_rest_in_a_walled_curvilinear_box_stays_at_rest(riemann):
    c = cs.multiblock_2d(cols=2, rows=2, lo=6, hi=9, seed=3, velocity=0.0, bc=WALLS, riemann=riemann)
    o, P, R = _residual(c)
    Ri = H.interior_rows(c, R)
    p = c.P0[4, c.interior_mask()].max()
    area = c.blocks[0]["fm1"][3::4].max()
    assert np.abs(Ri[0]).max() == 0.0 and np.abs(Ri[4]).max() <= 1e-12 * p * area
    assert np.abs(Ri[1:4]).max() <= 1e-10 * p * area          # sum of p n A over a closed cell
    P1 = c.P0.copy()
    assert o.step(P1, 5) == 0
    m = c.interior_mask()
    assert np.abs(P1[1:4, m]).max() <= 1e-9 * c.meta["V"]


def test_uniform_supersonic_inflow_has_zero_residual():
    bc = {1: abi.BC_INFLOW, 2: abi.BC_EXTRAPOLATION, 3: abi.BC_EXTRAPOLATION, 4: abi.BC_EXTRAPOLATION,
          5: abi.BC_EXTRAPOLATION, 6: abi.BC_EXTRAPOLATION}
    for riemann in (abi.RS_HLLC, abi.RS_AUSMP, abi.RS_LMROE):
        c = cs.multiblock_2d(cols=2, rows=1, lo=6, hi=9, seed=4, amp=0.0, bc=bc, riemann=riemann, visc=0)
        _, P, R = _residual(c)
        Ri = H.interior_rows(c, R)
        rho, V = c.meta["rho"], c.meta["V"]
        A = c.blocks[0]["fm1"][3::4].max()
        scale = np.array([rho * V, rho * V * V, rho * V * V, rho * V * V, rho * V ** 3]) * A
        assert (np.abs(Ri).max(axis=1) <= 1e-9 * scale).all(), np.abs(Ri).max(axis=1) / scale


def test_outward_flow_closes_a_405_face():
    bc = {1: abi.BC_INFLOW, 2: abi.BC_EXTRAPOLATION, 3: abi.BC_EXTRAPOLATION, 4: abi.BC_EXTRAPOLATION,
          5: abi.BC_EXTRAPOLATION, 6: abi.BC_EXTRAPOLATION}
    c = cs.multiblock_2d(cols=1, rows=1, lo=8, hi=8, seed=4, amp=0.0, bc=bc, visc=0, velocity=-300.0)
    _, P, R = _residual(c)
    I = c.interior(R, 0)                          # (5, n1, n2, 1)
    rho = c.meta["rho"]
    A = c.blocks[0]["fm1"][3::4].max()
    # cells at i = 1: only the interior face i + 1/2 carries mass (rho u A, u < 0); cells inside: zero
    assert np.allclose(I[0, 0], rho * -300.0 * A, rtol=1e-12)
    assert np.abs(I[0, 1:-1]).max() <= 1e-12 * rho * 300.0 * A


def test_no_slip_wall_drags_a_tangential_stream():
    bc = {1: abi.BC_EXTRAPOLATION, 2: abi.BC_EXTRAPOLATION, 3: abi.BC_WALL, 4: abi.BC_WALL,
          5: abi.BC_EXTRAPOLATION, 6: abi.BC_EXTRAPOLATION}
    c = cs.multiblock_2d(cols=1, rows=1, lo=8, hi=8, seed=4, amp=0.0, bc=bc, visc=1, velocity=100.0)
    _, P, R = _residual(c)
    I = c.interior(R, 0)
    # the wall stress opposes the stream at the wall cells (R = sum of outgoing fluxes: positive x-momentum)
    mu = c.meta["mu"]
    assert (I[1, :, 0] > 0).all() and (I[1, :, -1] > 0).all()
    assert np.abs(I[1, :, 1:-1]).max() <= 1e-9 * np.abs(I[1, :, 0]).max()
    n2 = c.blocks[0]["n"][1]
    dy = 1.0 / n2
    A = c.blocks[0]["fm2"][3::4].max()
    # tau = mu du/dy with du/dy = u / (dy/2) between the wall and the first cell centre
    assert np.allclose(I[1, :, 0], mu * 100.0 / (0.5 * dy) * A, rtol=1e-10)


SYM = abi.BC_SYMMETRY


def test_isothermal_wall_conducts_heat_into_a_gas_at_rest():
    Tw, T = 330.0, 300.0
    bc = {1: SYM, 2: SYM, 3: (abi.BC_WALL_T, (Tw,)), 4: (abi.BC_WALL_T, (Tw,)), 5: SYM, 6: SYM}
    c = cs.multiblock_2d(cols=1, rows=1, lo=8, hi=8, seed=4, amp=0.0, bc=bc, visc=1, velocity=0.0, T=T)
    _, P, R = _residual(c)
    I = c.interior(R, 0)
    mu, cp, prandtl = c.meta["mu"], c.thermo["cp"][0], 0.71
    kl = mu * cp / prandtl                        # constant viscosity and cp: k at the wall = k of the gas
    dy = 1.0 / c.blocks[0]["n"][1]
    A = c.blocks[0]["fm2"][3::4].max()
    q = kl * (Tw - T) / (0.5 * dy) * A            # heat conducted in through each wall face
    assert np.allclose(I[4, :, 0], -q, rtol=1e-9) and np.allclose(I[4, :, -1], -q, rtol=1e-9)
    assert np.abs(I[4, :, 1:-1]).max() <= 1e-9 * q
    assert np.abs(I[0]).max() == 0.0              # no mass through walls or symmetry faces, gas at rest


def test_symmetry_faces_act_as_extrapolated_faces_of_a_uniform_tube():
    a = cs.riemann_1d(n=100)
    b = cs.riemann_1d(n=100)
    b.rec["type"][b.rec["face"] >= 3] = SYM
    Pa, Pb = a.P0.copy(), b.P0.copy()
    oa, ob = oracle.Oracle(a), oracle.Oracle(b)
    assert oa.step(Pa, 40) == 0 and ob.step(Pb, 40) == 0
    e = H.rel_err(H.conserved(b, Pb), H.conserved(a, Pa))
    assert np.all(e[[0, 1, 4]] <= 1e-12), e
    assert np.abs(b.interior(Pb, 0)[2:4]).max() == 0.0   # no transverse motion


def _outlet_stream(p_exit_ratio, velocity=None):
    bc = {1: abi.BC_INFLOW, 2: (abi.BC_OUTLET, (p_exit_ratio * 1.0e5, 1.0)), 3: SYM, 4: SYM, 5: SYM, 6: SYM}
    c = cs.multiblock_2d(cols=2, rows=1, lo=6, hi=9, seed=4, amp=0.0, bc=bc, visc=0, mach=0.5, velocity=velocity)
    return c


def test_outlet_at_the_stream_pressure_passes_a_subsonic_stream():
    c = _outlet_stream(1.0)
    _, P, R = _residual(c)
    Ri = H.interior_rows(c, R)
    rho, V = c.meta["rho"], c.meta["V"]
    A = c.blocks[0]["fm1"][3::4].max()
    scale = np.array([rho * V, rho * V * V, rho * V * V, rho * V * V, rho * V ** 3]) * A
    assert (np.abs(Ri).max(axis=1) <= 1e-9 * scale).all(), np.abs(Ri).max(axis=1) / scale


def test_outlet_below_the_stream_pressure_draws_more_mass_out():
    c = _outlet_stream(0.8)
    _, P, R = _residual(c)
    last = c.interior(R, 1)                       # the block at the outlet
    rho, V = c.meta["rho"], c.meta["V"]
    A = c.blocks[1]["fm1"][3::4].max()
    assert (last[0, -1] > 1e-3 * rho * V * A).all()          # net mass out of the outlet cells
    assert np.abs(last[0, :-1]).max() <= 1e-9 * rho * V * A  # the stream elsewhere untouched


def test_inward_flow_closes_a_406_face():
    bc = {1: abi.BC_EXTRAPOLATION, 2: (abi.BC_OUTLET, (1.0e5, 0.5)), 3: SYM, 4: SYM, 5: SYM, 6: SYM}
    c = cs.multiblock_2d(cols=1, rows=1, lo=8, hi=8, seed=4, amp=0.0, bc=bc, visc=0, velocity=-300.0)
    _, P, R = _residual(c)
    I = c.interior(R, 0)
    rho = c.meta["rho"]
    A = c.blocks[0]["fm1"][3::4].max()
    # cells at i = max: only the interior face i - 1/2 carries mass (u < 0); cells inside: zero
    assert np.allclose(I[0, -1], rho * 300.0 * A, rtol=1e-12)
    assert np.abs(I[0, 1:-1]).max() <= 1e-12 * rho * 300.0 * A


def _inlet_stream(inlet, mach=0.5, outlet=None):
    """A uniform subsonic stream along +x on a Cartesian 2-block channel: the given type-4 inlet at i = 1, the 406
    outlet at the stream's pressure at i = max (or `outlet`), symmetry elsewhere."""
    bc = {1: inlet, 2: outlet or (abi.BC_OUTLET, (1.0e5, 1.0)), 3: SYM, 4: SYM, 5: SYM, 6: SYM}
    return cs.multiblock_2d(cols=2, rows=1, lo=6, hi=9, seed=4, amp=0.0, bc=bc, visc=0, mach=mach)


def _stream_state(mach=0.5, T=300.0, p=1.0e5):
    th = cs.ideal_gas_tables()
    R, gam = th["R"], th["gamma"]
    d = 0.5 * (gam - 1.0)
    rho = p / (R * T)
    U = mach * math.sqrt(gam * R * T)
    T0 = T * (1.0 + d * mach * mach)
    p0 = p * (1.0 + d * mach * mach) ** (gam / (gam - 1.0))
    return rho, U, T0, p0


@pytest.mark.parametrize("code", [401, 403, 404, 407])
def test_subsonic_inlets_pass_a_matching_stream(code):
    rho, U, T0, p0 = _stream_state()
    if code in (401, 407):
        q = (0.0, T0, p0, 0.0, 0.0, 1.0, code, 1.0e5)      # stagnation T0, p0 (407: ambient pressure p outwards)
    elif code == 403:
        q = (0.0, T0, rho * U, 0.0, 0.0, 1.0, code)        # mass flux, total temperature
    else:
        q = (0.0, 300.0, rho * U, 0.0, 0.0, 1.0, code)     # mass flux, static temperature
    c = _inlet_stream((abi.BC_INFLOW, q))
    _, P, R = _residual(c)
    Ri = H.interior_rows(c, R)
    A = c.blocks[0]["fm1"][3::4].max()
    scale = np.array([rho * U, rho * U * U, rho * U * U, rho * U * U, rho * U ** 3]) * A
    assert (np.abs(Ri).max(axis=1) <= 1e-8 * scale).all(), np.abs(Ri).max(axis=1) / scale


def test_ambient_boundary_lets_a_stream_out_at_its_pressure():
    rho, U, T0, p0 = _stream_state()
    amb = (abi.BC_INFLOW, (0.0, T0, p0, 0.0, 0.0, 1.0, 407, 1.0e5))
    c = _inlet_stream((abi.BC_INFLOW, (0.5, 300.0, 1.0e5, 0.0, 0.0, 1.0)), outlet=amb)   # 405 in, 407 out
    _, P, R = _residual(c)
    Ri = H.interior_rows(c, R)
    A = c.blocks[0]["fm1"][3::4].max()
    assert np.abs(Ri[0]).max() <= 1e-8 * rho * U * A


def _entropy_wave(n, cfl, n_rk, t_end=0.05):
    th = cs.ideal_gas_tables()
    h = 1.0 / n

    def nodes(iu, iv, iw):
        return np.stack([iu * h, iv * h, iw * h], axis=-1)

    def prim(c):
        x = c[..., 0]
        z = np.zeros_like(x)
        return np.stack([1.0 + 0.2 * np.sin(2 * math.pi * x), z + 1.0, z, z, z + 1.0])

    scheme = dict(limiter=abi.LIM_FIRST, riemann=abi.RS_HLLC, visc=0, n_rk=n_rk, ndir=1, cfl=cfl,
                  time_clip=1, time_threshold=t_end)
    bc = {f: abi.BC_EXTRAPOLATION for f in range(3, 7)}
    return cs.layout_case("wave", [[0, n], [0, 1], [0, 1]], nodes, (True, False, False), bc, th, scheme, prim)


@pytest.mark.parametrize("n_rk,order", [(4, 4), (3, 3)])
def test_temporal_order_on_a_smooth_periodic_problem(n_rk, order):
    sols = []
    for cfl in (0.8, 0.4, 0.2, 0.05):
        c = _entropy_wave(32, cfl, n_rk)
        o = oracle.Oracle(c)
        P = c.P0.copy()
        o.run_to(P, 0.05)
        sols.append(c.interior(P, 0)[0].ravel())
    e = [np.abs(s - sols[-1]).max() for s in sols[:-1]]
    rate = math.log2(e[1] / e[2])
    assert order - 0.5 < rate < order + 0.7, (e, rate)
