"""Compact serving cases (mosegpu/case.py: uniform-grid geometry, implicit k faces): the geometry of
uniform_geometry against cell_metrics / face_metrics on the same grid, and the records a one-plane block without
k-face records stands for (oracle.explicit_k_records) against the records the full builder writes."""
import numpy as np
import pytest

import helpers as H
from mosegpu import case as cs


@pytest.mark.parametrize("build", [lambda c: cs.riemann_2d(n=40, compact=c), lambda c: cs.riemann_1d(n=64, compact=c)])
def test_compact_case_is_the_full_case(build):
    import oracle
    full, comp = build(False), build(True)
    for f in ("fm1", "fm2", "fm3", "dl", "m", "vol"):
        x, y = full.blocks[0][f], comp.blocks[0][f]
        assert x.shape == y.shape
        assert np.max(np.abs(x - y) / np.maximum(np.abs(x), 1e-300)) < 1e-13, f
    assert len(comp.rec) < len(full.rec)
    assert not np.any(comp.rec["face"] >= 5)
    rec, conn = oracle.explicit_k_records(comp)
    assert np.array_equal(rec, full.rec)
    assert np.array_equal(comp.P0, full.P0)


def test_explicit_k_records_renumber_connections():
    """A 2-D batch of blocks with connections between them: the synthesized k-face records are appended block by
    block and every connection still names its own record."""
    import oracle
    case = cs.multiblock_2d(cols=3, rows=2, lo=9, hi=20, seed=5)
    keep = case.rec["face"] < 5
    old_idx = np.nonzero(keep)[0]
    comp_rec = case.rec[keep]
    remap = -np.ones(len(case.rec), dtype=np.int64)
    remap[old_idx] = np.arange(old_idx.size)
    comp = cs.Case("mb2d_implicit_k")
    comp.__dict__.update(case.__dict__)
    comp.rec = comp_rec
    comp.conn = case.conn.copy()
    comp.conn["rec"] = remap[case.conn["rec"]]
    assert np.all(comp.conn["rec"] >= 0)
    rec, conn = oracle.explicit_k_records(comp)
    assert np.array_equal(rec, case.rec) and np.array_equal(conn, case.conn)


def test_oracle_runs_compact_case_as_full_case():
    """The oracle on the compact 2-D case (uniform geometry, implicit k faces) and on the full one: the same
    evolution up to the geometry's last-bit rounding."""
    import oracle
    full, comp = cs.riemann_2d(n=24), cs.riemann_2d(n=24, compact=True)
    Pa, Pb = full.P0.copy(), comp.P0.copy()
    assert oracle.Oracle(full).step(Pa, 5) == 0
    assert oracle.Oracle(comp).step(Pb, 5) == 0
    e = H.rel_err(H.conserved(full, Pa), H.conserved(comp, Pb))
    assert np.all(e < 1e-11), e
