"""The reference's own 1-D regression cases as engine cases, from the committed fixture
tests/golden/reference_1d_cases.npz (made by tests/golden/make_reference_fixtures.py from test/1D/<name>/).

Each case is built as the reference's set-up builds it:
  - nodes: the 401 x 2 x 2 (Shu-Osher: 201 x 2 x 2) nodes of INPUT/ic.tec; the ghost nodes of every boundary face are
    continued as BC_Extrapolate_Metrics does (src/lib/numerics/space/Lib_Metrics.f90:766-1041): cubically,
    3 N(g+1) - 3 N(g+2) + N(g+3), along an axis of more than two cells, linearly, 2 N(g+1) - N(g+2), along a thinner
    one; the metrics of every cell then follow from Compute_Metric_Tensor / Compute_Norm_Area (mosegpu/case.py);
  - state: rho, u, v, w, p of ic.tec, cell-centred;
  - records: INPUT/bc.txt in its order; code 400 -> extrapolation (type 11, IO_BC_Open.f90:196-198), code 0 -> no
    boundary condition (type 0: zero-gradient ghosts and no face flux, Mod_BC.f90:55-59);
  - thermo: the 1 K table of INPUT/thermo.dat with row 0 = (cp(1), h = 0) (Load_ThermoTransport.f90:82-97), R =
    Runiv / wm of INPUT/phase.txt (gamma = cp / (cp - R) = 1.3999968 for these tables, not 1.4);
  - scheme: input.ini ([MOSE-Numerics] riemann-solver, flux-limiter, space-reconstruction, cfl, time-scheme).
"""
import configparser
import json
import os

import numpy as np

from mosegpu import abi
from mosegpu import case as cs

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "reference_1d_cases.npz")
GC = abi.GC

RIEMANN = {"hllc": abi.RS_HLLC, "hlle": abi.RS_HLLE, "slau": abi.RS_SLAU, "ausm+": abi.RS_AUSMP,
           "hlle++": abi.RS_HLLEPP, "llf": abi.RS_LLF, "lmroe": abi.RS_LMROE}
LIMITER = {"minmod": abi.LIM_MINMOD, "vanleer": abi.LIM_VANLEER, "vanalbada": abi.LIM_VANALBADA, "mc": abi.LIM_MC,
           "superbee": abi.LIM_SUPERBEE}
N_RK = {"euler": 1, "rk1": 1, "rk2": 2, "rk3": 3}


def _data():
    d = np.load(FIXTURE)
    return d, json.loads(str(d["meta"]))


def names():
    return list(_data()[1].keys())


def _extend(X, periodic=(False, False, False)):
    """Node array (ni, nj, nk, 3) -> (ni + 4, nj + 4, nk + 4, 3) with two ghost-node layers per side: along a periodic
    axis the donor nodes translated by one period (BC_Connect_Metrics for 201, Lib_Metrics.f90:1175), otherwise the
    continuation of BC_Extrapolate_Metrics."""
    ni, nj, nk = X.shape[:3]
    E = np.zeros((ni + 2 * GC, nj + 2 * GC, nk + 2 * GC, 3))
    E[GC:GC + ni, GC:GC + nj, GC:GC + nk] = X
    for ax, n in enumerate((ni, nj, nk)):
        cubic = (n - 1) > 2                    # cells along the axis
        sl = [slice(None)] * 4

        def at(q):
            s = list(sl)
            s[ax] = q
            return tuple(s)
        if periodic[ax]:
            span = E[at(GC + n - 1)] - E[at(GC)]
            for g in (1, 2):
                E[at(GC - g)] = E[at(GC + n - 1 - g)] - span
                E[at(GC + n - 1 + g)] = E[at(GC + g)] + span
            continue
        for g in (1, 2):
            lo, hi = GC - g, GC + n - 1 + g
            if cubic:
                E[at(lo)] = 3.0 * E[at(lo + 1)] - 3.0 * E[at(lo + 2)] + E[at(lo + 3)]
                E[at(hi)] = 3.0 * E[at(hi - 1)] - 3.0 * E[at(hi - 2)] + E[at(hi - 3)]
            else:
                E[at(lo)] = 2.0 * E[at(lo + 1)] - E[at(lo + 2)]
                E[at(hi)] = 2.0 * E[at(hi - 1)] - E[at(hi - 2)]
    return E


def load(name):
    """The engine case of the reference's test 1D/<name>, with `case.meta['md5_1it']` its one-iteration pin."""
    d, meta = _data()
    m = meta[name]
    X = d[name + "/nodes"]
    cells = d[name + "/cells"]
    bc = d[name + "/bc"]
    cn = d[name + "/conn"]
    tab = d[name + "/thermo"]
    codes = {int(code) for code in bc[:, 5]}
    assert codes <= {0, 201, 400}, codes
    # periodic axes: the 201 records of both faces of the axis
    periodic = tuple(bool(np.any((bc[:, 5] == 201) & ((bc[:, 4] + 1) // 2 == ax + 1))) for ax in range(3))
    E = _extend(X, periodic)

    def node_fn(iu, iv, iw):
        return E[iu.astype(np.int64) + GC, iv.astype(np.int64) + GC, iw.astype(np.int64) + GC]

    ini = configparser.ConfigParser()
    ini.read_string(m["ini"])
    num = ini["MOSE-Numerics"]
    recon = num.get("space-reconstruction", "MUSCL").strip().lower()
    lim = abi.LIM_FIRST if recon == "first-order" else LIMITER[num.get("flux-limiter").strip().lower()]
    scheme = dict(limiter=lim, riemann=RIEMANN[num.get("riemann-solver").strip().lower()], visc=0,
                  n_rk=N_RK[num.get("time-scheme", "RK3").strip().lower()], ndir=1,
                  cfl=float(num.get("cfl")), time_clip=1,
                  time_threshold=float(ini["MOSE-Parameters"].get("time-threshold", "0")))
    wm = m["wm"]
    T = np.arange(cs.TMIN, cs.TMAX + 1, dtype=np.float64)
    assert tab.shape[0] == cs.TMAX and tab[0, 0] == 1.0
    cp = np.empty(T.shape); h = np.empty(T.shape)
    cp[1:] = tab[:, 1]; h[1:] = tab[:, 2]
    cp[0] = cp[1]; h[0] = cp[1] * 0.0
    R = cs.RUNIV / wm
    th = dict(tmin=cs.TMIN, tmax=cs.TMAX, wm=wm, cp=cp, h=h, mu=np.zeros(T.shape), k=np.zeros(T.shape), R=R,
              cp_value=cp[1], gamma=cp[1] / (cp[1] - R))
    n = [s_ - 1 for s_ in X.shape[:3]]
    scheme["ndir"] = 1 if n[1] == 1 and n[2] == 1 else (2 if n[2] == 1 else 3)
    case = cs.layout_case("ref_" + name, [[0, n[0]], [0, n[1]], [0, n[2]]], node_fn, periodic,
                          {f: abi.BC_EXTRAPOLATION for f in range(1, 7)}, th, scheme, lambda c: cells)
    # the records of bc.txt in its order: 400 -> extrapolation (11), 0 -> no condition (0), 201 -> periodic connection
    # (1) whose donor must be the one bc.txt names
    want = [(int(b) - 1, int(i), int(j), int(k), int(f)) for b, i, j, k, f, code in bc]
    got = [(int(r["blk"]), int(r["i"]), int(r["j"]), int(r["k"]), int(r["face"])) for r in case.rec]
    assert got == want, "record order differs from bc.txt"
    case.rec["type"] = np.where(bc[:, 5] == 0, abi.BC_NONE,
                                np.where(bc[:, 5] == 201, abi.BC_CONNECTION, abi.BC_EXTRAPOLATION))
    for q in np.nonzero(bc[:, 5] == 201)[0]:
        c = case.conn[int(case.rec[q]["conn"])]
        got = (int(c["bs"]) + 1, int(c["is"]), int(c["js"]), int(c["ks"]), int(c["fs"]), int(c["d11"]),
               int(c["d12"]), int(c["d21"]), int(c["d22"]))
        assert got == tuple(int(x) for x in cn[q]), (q, got, cn[q])
    case.meta = dict(md5_1it=m["md5_1it"], ini=m["ini"], reference_case="test/1D/" + name)
    return case
