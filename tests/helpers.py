"""Shared helpers of the tests: small cases, conserved variables, error norms."""
import numpy as np

from mosegpu import abi
from mosegpu import case as cs


def conserved(case, P):
    """Interior conserved variables (rho, rho u, rho v, rho w, rho E) of every block, concatenated
    (E = h(T) - p / rho + |u|^2 / 2 with h from the case's table, as prim2cons of the state update)."""
    th = case.thermo
    out = []
    for b in range(len(case.blocks)):
        I = case.interior(P, b).reshape(5, -1)
        rho, u, v, w, p = I
        T = p / (rho * th["R"])
        ti = np.clip(np.floor(T).astype(np.int64), th["tmin"], th["tmax"] - 1)
        h = th["h"][ti - th["tmin"]] + (T - ti) * (th["h"][ti + 1 - th["tmin"]] - th["h"][ti - th["tmin"]])
        E = h - p / rho + 0.5 * (u * u + v * v + w * w)
        out.append(np.stack([rho, rho * u, rho * v, rho * w, rho * E]))
    return np.concatenate(out, axis=1)


def rel_err(a, b, floor=1e-300):
    """Per conserved variable: max |a - b| / max |b| (relative to the field's magnitude). For the five conserved
    variables the three momentum components are one vector field: each is measured against the largest of the
    three (a component that is pure round-off, as w of a 2-D case, is not a scale)."""
    a = np.asarray(a).reshape(a.shape[0], -1)
    b = np.asarray(b).reshape(b.shape[0], -1)
    scale = np.abs(b).max(axis=1)
    if b.shape[0] == 5:
        scale[1:4] = scale[1:4].max()
    return np.abs(a - b).max(axis=1) / np.maximum(scale, floor)


def norms(a, b):
    """L1, L2, Linf of a - b relative to the same norms of b, per variable."""
    a = np.asarray(a).reshape(a.shape[0], -1)
    b = np.asarray(b).reshape(b.shape[0], -1)
    d = a - b
    l1 = np.abs(d).sum(axis=1) / np.maximum(np.abs(b).sum(axis=1), 1e-300)
    l2 = np.sqrt((d * d).sum(axis=1)) / np.maximum(np.sqrt((b * b).sum(axis=1)), 1e-300)
    li = np.abs(d).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-300)
    return l1, l2, li


def interior_rows(case, R):
    """R (5, ncell) restricted to the interior rows."""
    return R[:, case.interior_mask()]


def reversed_records(case):
    """The same case with its boundary records in reverse order (a case without connections: the connection
    table refers to records by index). The ghost fill of the reference runs its record loop in this order."""
    assert len(case.conn) == 0
    case.rec = case.rec[::-1].copy()
    return case


def with_scheme(case, **kw):
    """The case with scheme entries replaced (e.g. mco)."""
    case.scheme.update(kw)
    return case


def prec_case(case, **kw):
    """The case with integration-variables = prec (HLLC-PC, local steps) and the given preconditioning keys."""
    case.scheme["riemann"] = abi.RS_HLLC_PC
    return with_scheme(case, intvar=abi.INTVAR_PREC, local_dt=1, **kw)


def small_cases():
    """(id, builder) of the parity cases: every boundary type, Riemann solver and limiter served."""
    return [
        ("sod_hllc_minmod", lambda: cs.riemann_1d(n=64)),
        ("sod_ausm_vanleer", lambda: cs.riemann_1d(n=64, riemann=abi.RS_AUSMP, limiter=abi.LIM_VANLEER)),
        ("sod_roe_vanalbada", lambda: cs.riemann_1d(n=64, riemann=abi.RS_LMROE, limiter=abi.LIM_VANALBADA)),
        ("quad2d_hllc_minmod", lambda: cs.riemann_2d(n=20)),
        ("quad2d_ausm_mc", lambda: cs.riemann_2d(n=20, riemann=abi.RS_AUSMP, limiter=abi.LIM_MC)),
        ("tgv_roe_vanalbada_1blk", lambda: cs.taylor_green(n=12)),
        ("tgv_hllc_minmod_8blk", lambda: cs.taylor_green(n=12, blocks=2, riemann=abi.RS_HLLC,
                                                         limiter=abi.LIM_MINMOD)),
        ("tgv_ausm_superbee_noise", lambda: cs.taylor_green(n=12, riemann=abi.RS_AUSMP, limiter=abi.LIM_SUPERBEE,
                                                            noise=1e-3)),
        ("tgv_blocks_hllc_vanalbada_m03", lambda: cs.taylor_green_blocks(nb=2, nblk=6)),
        ("mb2d_ausm_vanleer_rk4", lambda: cs.multiblock_2d(cols=2, rows=2, lo=6, hi=14, seed=7)),
        ("mb2d_hllc_minmod_rk3", lambda: cs.multiblock_2d(cols=3, rows=2, lo=5, hi=12, seed=11, riemann=abi.RS_HLLC,
                                                          limiter=abi.LIM_MINMOD, n_rk=3)),
        ("mb2d_roe_mc_euler_rk4", lambda: cs.multiblock_2d(cols=2, rows=3, lo=5, hi=11, seed=5, riemann=abi.RS_LMROE,
                                                           limiter=abi.LIM_MC, visc=0)),
        # the solvers of no benchmarked case (the run-time solver unit): interior faces, connections, walls, inlet
        ("sod_hlle_minmod", lambda: cs.riemann_1d(n=64, riemann=abi.RS_HLLE)),
        ("sod79_slau_mc_cfl09", lambda: cs.riemann_1d(n=64, riemann=abi.RS_SLAU, limiter=abi.LIM_MC, cfl=0.9)),
        ("sod_llf_vanleer", lambda: cs.riemann_1d(n=64, riemann=abi.RS_LLF, limiter=abi.LIM_VANLEER)),
        ("sod_slau2_superbee", lambda: cs.riemann_1d(n=64, riemann=abi.RS_SLAU2, limiter=abi.LIM_SUPERBEE)),
        ("quad2d_hlle_vanalbada", lambda: cs.riemann_2d(n=20, riemann=abi.RS_HLLE, limiter=abi.LIM_VANALBADA)),
        ("tgv_slau2_vanalbada_8blk", lambda: cs.taylor_green(n=12, blocks=2, riemann=abi.RS_SLAU2)),
        ("tgv_llf_mc", lambda: cs.taylor_green(n=12, riemann=abi.RS_LLF, limiter=abi.LIM_MC)),
        ("mb2d_slau_vanleer_rk3", lambda: cs.multiblock_2d(cols=2, rows=2, lo=5, hi=10, seed=3, riemann=abi.RS_SLAU,
                                                           n_rk=3)),
        ("mb2d_llf_minmod_rk4", lambda: cs.multiblock_2d(cols=2, rows=2, lo=5, hi=10, seed=9, riemann=abi.RS_LLF,
                                                         limiter=abi.LIM_MINMOD)),
        ("mb2d_hlle_mc_euler", lambda: cs.multiblock_2d(cols=2, rows=2, lo=5, hi=10, seed=4, riemann=abi.RS_HLLE,
                                                        limiter=abi.LIM_MC, visc=0)),
        # the exact Godunov solver (Newton on the star state) and MiczekRoe (preconditioned below Mco)
        ("sod_exact_minmod", lambda: cs.riemann_1d(n=64, riemann=abi.RS_EXACT)),
        ("quad2d_exact_vanleer", lambda: cs.riemann_2d(n=20, riemann=abi.RS_EXACT, limiter=abi.LIM_VANLEER)),
        ("mb2d_exact_minmod_rk3", lambda: cs.multiblock_2d(cols=2, rows=2, lo=5, hi=9, seed=21, riemann=abi.RS_EXACT,
                                                           limiter=abi.LIM_MINMOD, n_rk=3)),
        ("tgv_miczek_mco02", lambda: with_scheme(cs.taylor_green(n=12, riemann=abi.RS_MICZEKROE), mco=0.2)),
        ("duct3d_miczek_mco03", lambda: with_scheme(cs.duct_3d(riemann=abi.RS_MICZEKROE), mco=0.3)),
        # the solvers that read the shock sensor (beta of the face's left cell; connection records: their own cell's)
        # and a base solver with a sensor (the slopes scaled by beta)
        ("sod_ausmpm_chen_mco02", lambda: with_scheme(cs.riemann_1d(n=64, riemann=abi.RS_AUSMPM), mco=0.2)),
        ("sod_hllepp_tramel", lambda: cs.riemann_1d(n=64, riemann=abi.RS_HLLEPP, limiter=abi.LIM_VANLEER)),
        ("quad2d_hllc_tramel_mc", lambda: cs.riemann_2d(n=20, riemann=abi.RS_HLLC_TRAMEL, limiter=abi.LIM_MC)),
        ("tgv_hllc_chen_8blk", lambda: with_scheme(cs.taylor_green(n=12, blocks=2, riemann=abi.RS_HLLC_CHEN,
                                                                   noise=1e-3), mco=0.2)),
        ("mb2d_hllc_sensor_tramel", lambda: with_scheme(cs.multiblock_2d(cols=2, rows=2, lo=5, hi=9, seed=23,
                                                                         riemann=abi.RS_HLLC), sensor=abi.SENSOR_TRAMEL)),
        ("mb2d_ausmpm_chen_euler", lambda: with_scheme(cs.multiblock_2d(cols=2, rows=1, lo=6, hi=9, seed=29, visc=0,
                                                                        riemann=abi.RS_AUSMPM), mco=0.3)),
        ("duct3d_hllepp_tramel", lambda: cs.duct_3d(riemann=abi.RS_HLLEPP)),
        # the primitive-variable update (integration-variables = prim)
        ("sod_prim_hllc", lambda: with_scheme(cs.riemann_1d(n=64), intvar=abi.INTVAR_PRIM)),
        ("tgv_prim_roe_8blk", lambda: with_scheme(cs.taylor_green(n=12, blocks=2), intvar=abi.INTVAR_PRIM)),
        ("mb2d_prim_ausm_rk3", lambda: with_scheme(cs.multiblock_2d(cols=2, rows=2, lo=5, hi=9, seed=31, n_rk=3),
                                                   intvar=abi.INTVAR_PRIM)),
        # implicit residual smoothing (IRS = t): the Jacobi sweeps along every direction, the ghost residual from the
        # face cell or a connection's donor, on the conservative (scaled) and the primitive (raw) residual
        ("sod_irs2_hllc", lambda: with_scheme(cs.riemann_1d(n=64), irs=2, cfl=0.8)),
        ("tgv_irs2_roe_8blk", lambda: with_scheme(cs.taylor_green(n=12, blocks=2, noise=1e-3), irs=2)),
        ("mb2d_irs3_ausm_rk2_beta07", lambda: with_scheme(cs.multiblock_2d(cols=2, rows=2, lo=5, hi=9, seed=37,
                                                                           n_rk=2), irs=3, irs_beta=0.7)),
        ("duct3d_irs1_hllc_beta03", lambda: with_scheme(cs.duct_3d(), irs=1, irs_beta=0.3)),
        ("sod_prim_irs4_hllc", lambda: with_scheme(cs.riemann_1d(n=64), intvar=abi.INTVAR_PRIM, irs=4)),
        # local time stepping (time-accurate = false) and the cfl-rise ramp, alone and with the smoothing and the
        # primitive update
        ("mb2d_local_dt_ausm_rk3_rise10", lambda: with_scheme(cs.multiblock_2d(cols=2, rows=2, lo=5, hi=9, seed=43,
                                                                               n_rk=3), local_dt=1, cfl_rise=10)),
        ("tgv_local_dt_roe_8blk", lambda: with_scheme(cs.taylor_green(n=12, blocks=2, noise=1e-3), local_dt=1)),
        ("sod_local_dt_irs2_hllc", lambda: with_scheme(cs.riemann_1d(n=64), local_dt=1, irs=2)),
        ("duct3d_local_dt_prim_rise4", lambda: with_scheme(cs.duct_3d(), local_dt=1, intvar=abi.INTVAR_PRIM,
                                                           cfl_rise=4)),
        ("sod_rise5_hllc", lambda: with_scheme(cs.riemann_1d(n=64), cfl_rise=5)),
        # integration-variables = prec: Ur (the three modes, smoothing), the preconditioned local steps, Theta of the
        # primitive update and HLLC-PC at interior faces, connections (the ghost's Ur 0), symmetry faces and walls
        ("mb2d_prec_hllcpc_ns", lambda: prec_case(cs.multiblock_2d(cols=2, rows=2, lo=5, hi=9, seed=47, n_rk=3,
                                                                    mach=0.2, cfl=0.3))),
        ("duct3d_prec_mach03_smooth2", lambda: prec_case(cs.duct_3d(cfl=0.3), prec_mach=0.3, prec_smooth=2)),
        ("tgv_prec_uref_8blk", lambda: prec_case(with_scheme(cs.taylor_green(n=12, blocks=2, noise=1e-3), cfl=0.3),
                                                 prec_uref=200.0)),
        ("sod_prec_irs2_rk2", lambda: prec_case(cs.riemann_1d(n=64, n_rk=2, cfl=0.3), irs=2, prec_eps_min=0.9)),
        # symmetry (300), isothermal walls (302) and the back-pressure outlet (406)
        ("duct3d_hllc_vanleer", lambda: cs.duct_3d()),
        ("duct3d_roe_vanalbada_rk4", lambda: cs.duct_3d(widths=(5, 6), heights=(4, 3), depths=(4,),
                                                        riemann=abi.RS_LMROE, limiter=abi.LIM_VANALBADA, n_rk=4)),
        ("duct3d_ausm_euler_supersonic", lambda: cs.duct_3d(mach=1.6, visc=0, riemann=abi.RS_AUSMP)),
        ("duct3d_slau_reversed_outlet", lambda: cs.duct_3d(velocity=-60.0, riemann=abi.RS_SLAU,
                                                           limiter=abi.LIM_MINMOD)),
        ("mb2d_isowall_outlet_symk", lambda: cs.multiblock_2d(
            cols=2, rows=2, lo=5, hi=9, seed=13, mach=0.5,
            bc={1: abi.BC_INFLOW, 2: (abi.BC_OUTLET, (0.9e5, 1.0)), 3: (abi.BC_WALL_T, (350.0,)),
                4: (abi.BC_WALL_T, (280.0,)), 5: abi.BC_SYMMETRY, 6: abi.BC_SYMMETRY})),
        # the subsonic inlets (401 stagnation, 403 / 404 mass flux) and the 407 ambient boundary
        ("duct3d_401_stagnation_inlet", lambda: cs.duct_3d(bc={1: (abi.BC_INFLOW, (0.0, 320.0, 1.25e5, 0.0, 0.0, 0.5, 401))})),
        ("duct3d_404_massflux_407_euler", lambda: cs.duct_3d(visc=0, riemann=abi.RS_AUSMP, bc={
            1: (abi.BC_INFLOW, (0.0, 300.0, 210.0, 0.0, 0.0, 1.0, 404)),
            2: (abi.BC_INFLOW, (0.0, 315.0, 1.19e5, 0.0, 0.0, 1.0, 407, 0.97e5))})),
        ("mb2d_403_massflux_inlet", lambda: cs.multiblock_2d(cols=2, rows=2, lo=5, hi=9, seed=17, mach=0.4, bc={
            1: (abi.BC_INFLOW, (0.0, 310.0, 180.0, 0.1, 0.0, 1.0, 403)), 2: (abi.BC_OUTLET, (1.0e5, 0.5)),
            3: abi.BC_WALL, 4: abi.BC_WALL, 5: abi.BC_EXTRAPOLATION, 6: abi.BC_EXTRAPOLATION})),
        # blocks two cells and one cell high between walls: a wall's cubic ghosts read the opposite face's ghosts,
        # so the fill must follow the record order
        # (Euler slip walls: no-slip walls two cells apart diverge in the oracle itself)
        ("mb2d_thin_walls_hllc", lambda: cs.multiblock_2d(cols=2, rows=1, widths=[6, 7], heights=[2], visc=0,
                                                          riemann=abi.RS_HLLC, limiter=abi.LIM_MINMOD)),
        ("mb2d_thin_walls_reversed", lambda: reversed_records(cs.multiblock_2d(cols=1, rows=1, widths=[8],
                                                                               heights=[2], visc=0, mach=0.5))),
        ("mb2d_one_row_walls_reversed", lambda: reversed_records(cs.multiblock_2d(cols=1, rows=1, widths=[7],
                                                                                  heights=[1], visc=0))),
    ]
