"""Generates the oracle's golden vectors under tests/golden/ (run: python tests/golden/make_golden.py).

Each case stores the interior residual of the initial state after the ghost fill, the interior state after
nsteps explicit steps and the first dt. They pin the CPU restatement against regressions; its agreement
with the reference is pinned by the physics known-answers of tests/test_oracle.py."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "mose-gpu_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import oracle  # noqa: E402
from mosegpu import abi  # noqa: E402
from mosegpu import case as cs  # noqa: E402

CASES = [
    ("sod64_hllc_minmod", lambda: cs.riemann_1d(n=64), 5),
    ("quad16_ausm_vanleer", lambda: cs.riemann_2d(n=16, riemann=abi.RS_AUSMP, limiter=abi.LIM_VANLEER), 3),
    ("tgv8_roe_vanalbada_ns", lambda: cs.taylor_green(n=8), 3),
]


def run(case, nsteps):
    o = oracle.Oracle(case)
    P = case.P0.copy()
    dt = o.dt(P)
    o.fill_ghosts(P)
    R = o.residual(P)[:, case.interior_mask()]
    P = case.P0.copy()
    rc = o.step(P, nsteps)
    assert rc == 0
    return R, P[:, case.interior_mask()], dt


if __name__ == "__main__":
    for name, builder, nsteps in CASES:
        R, P, dt = run(builder(), nsteps)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), R=R, P=P, dt=np.float64(dt))
        print(name, R.shape, P.shape, dt)
