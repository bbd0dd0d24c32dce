"""The Tecplot ASCII solution file (write_vtk_tec + ORION tec_write_structured_multiblock, ascii branch): the E23.15E3
formatter against lines that ORION itself wrote (tests/golden/orion_tecplot_lines.txt, from the reference's test
inputs), and the file layout of a written case read back."""
import os
import re

import numpy as np
import pytest

from mosegpu import case as cs
from mosegpu.tecplot import fortran_e23_15e3, gamma_rtot, temperature, write_tecplot_ascii

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "orion_tecplot_lines.txt")


def _golden():
    with open(GOLDEN) as f:
        return [ln.rstrip("\n") for ln in f if ln.strip()]


def test_formatter_reproduces_orion_value_lines():
    vals = [ln[1:] for ln in _golden() if ln.startswith("V")]
    assert len(vals) > 1500
    bad = [v for v in vals if fortran_e23_15e3(float(v)) != v]
    assert not bad, bad[:5]


def test_formatter_reproduces_orion_solutiontime():
    zones = [ln[1:] for ln in _golden() if ln.startswith("H") and "SOLUTIONTIME=" in ln]
    assert zones
    for z in zones:
        t = z.split("SOLUTIONTIME=")[1].split(",")[0]
        assert fortran_e23_15e3(float(t))[1:] == t          # str(no_sign=.true.) of a subnormal time


def test_formatter_edge_values():
    assert fortran_e23_15e3(0.0) == " 0.000000000000000E+000"
    assert fortran_e23_15e3(-0.0) == "-0.000000000000000E+000"
    assert fortran_e23_15e3(1.0) == " 0.100000000000000E+001"
    assert fortran_e23_15e3(-2.5e-3) == "-0.250000000000000E-002"
    assert fortran_e23_15e3(9.9999999999999995) == " 0.100000000000000E+002"   # rounding carries into the exponent
    assert fortran_e23_15e3(1.0e-300) == " 0.100000000000000E-299"
    assert fortran_e23_15e3(float("nan")).strip() == "NaN"
    assert fortran_e23_15e3(float("-inf")).strip() == "-Infinity"
    assert all(len(fortran_e23_15e3(x)) == 23 for x in (1e308, -1e-308, 5e-324, 123.456))


def _read(path):
    with open(path) as f:
        return f.read().split("\n")[:-1]


def test_written_case_layout_and_values(tmp_path):
    c = cs.multiblock_2d(cols=2, rows=1, lo=5, hi=9, seed=3)
    rng = np.random.default_rng(2)
    P = c.P0 * (1.0 + 1e-3 * rng.standard_normal(c.P0.shape))
    path = tmp_path / "field.tec"
    write_tecplot_ascii(path, c, P, 0.0123)
    L = _read(path)
    assert L[0] == ' VARIABLES ="x" "y" "z" "rho(1)" "u" "v" "w" "p" "T" "g" "R"'
    q = 1
    for b in range(len(c.blocks)):
        n1, n2, n3 = c.blocks[b]["n"]
        assert L[q] == (f" ZONE  T = Block{b + 1}, I={n1 + 1}, J={n2 + 1}, K={n3 + 1}, DATAPACKING=BLOCK, "
                        f"VARLOCATION=([1-3]=NODAL,[4-11]=CELLCENTERED), SOLUTIONTIME=0.123000000000000E-001")
        q += 1
        nn, nc = (n1 + 1) * (n2 + 1) * (n3 + 1), n1 * n2 * n3
        X = c.nodes(b)
        for d in range(3):
            got = np.array([float(v) for v in L[q:q + nn]])
            assert np.allclose(got, X[..., d].ravel(order="F"), rtol=1e-14, atol=1e-300)
            q += nn
        v = c.interior(P, b)
        g, r = gamma_rtot(c, v[0], v[4])
        want = [v[s] for s in range(5)] + [temperature(c, v[0], v[4]), g, r]
        assert np.allclose(g, c.thermo["gamma"], rtol=1e-12) and np.allclose(r, c.thermo["R"], rtol=1e-15)
        for w in want:
            got = np.array([float(x) for x in L[q:q + nc]])
            assert np.allclose(got, w.ravel(order="F"), rtol=1e-14, atol=0)
            q += nc
        assert all(len(x) == 23 for x in L[q - nc:q])
    assert q == len(L)


def test_steady_run_zone_and_temperature(tmp_path):
    c = cs.riemann_1d(n=16)
    path = tmp_path / "field.tec"
    write_tecplot_ascii(path, c, c.P0, -1.0)
    z = _read(path)[1]
    assert re.search(r"SOLUTIONTIME=0\.100000000000000E\+001, STRANDID = 0$", z)
    v = c.interior(c.P0, 0)
    R = 8314.46261815324 / c.thermo["wm"]
    assert np.allclose(temperature(c, v[0], v[4]), v[4] / (v[0] * R), rtol=1e-15)


def test_reader_round_trip_of_the_writer(tmp_path):
    from mosegpu.tecplot import read_tecplot_ascii
    c = cs.multiblock_2d(cols=2, rows=2, lo=5, hi=8, seed=5)
    rng = np.random.default_rng(4)
    P = c.P0 * (1.0 + 1e-3 * rng.standard_normal(c.P0.shape))
    path = tmp_path / "field.tec"
    write_tecplot_ascii(path, c, P, 0.5)
    Q, t, steady = read_tecplot_ascii(path, c)
    assert t == 0.5 and not steady
    m = c.interior_mask()
    assert np.allclose(Q[:, m], P[:, m], rtol=1e-14, atol=0)      # 15 significant digits
    assert np.array_equal(Q[:, ~m], c.P0[:, ~m])
    write_tecplot_ascii(path, c, P, -1.0)
    _, t, steady = read_tecplot_ascii(path, c)
    assert t == 1.0 and steady


def test_reader_takes_orion_zone_headers_and_skips_extra_variables(tmp_path):
    """A one-cell-deep block written in the two header styles of the reference's test inputs (one ZONE line with
    DATAPACKING / VARLOCATION / SOLUTIONTIME, as ORION writes; and a multi-line header), values several per line
    and with D exponents, a sixth variable that the reader skips."""
    from mosegpu.tecplot import read_tecplot_ascii
    c = cs.riemann_1d(n=3)
    n1, n2, n3 = c.blocks[0]["n"]
    nn, nc = (n1 + 1) * (n2 + 1) * (n3 + 1), n1 * n2 * n3
    xyz = list(np.arange(3 * nn, dtype=float))
    fields = [[10.0 * s + i + 0.5 for i in range(nc)] for s in range(6)]
    zone_line = [ln[1:] for ln in _golden() if ln.startswith("H ZONE") and "CELLCENTERED" in ln][0]
    zone_line = re.sub(r"I=\d+, J=\d+, K=\d+", f"I={n1 + 1}, J={n2 + 1}, K={n3 + 1}", zone_line)
    zone_line = zone_line.replace("[4-8]", "[4-9]")
    body = " ".join("%.17g" % v for v in xyz) + "\n" + "\n".join(
        " ".join(("%.17e" % v).replace("e", "D") for v in f) for f in fields) + "\n"
    times = []
    for header in (zone_line + "\n",
                   f' ZONE T="BLOCCO 1"\n I= {n1 + 1}, J= {n2 + 1}, K= {n3 + 1}, DATAPACKING=BLOCK, '
                   f'VARLOCATION=([1-3]=NODAL,[4-9]=CELLCENTERED)\n'):
        path = tmp_path / "ic.tec"
        path.write_text(' VARIABLES ="x" "y" "z" "rho1" "u" "v" "w" "p" "T"\n' + header + body)
        Q, t, _ = read_tecplot_ascii(path, c)
        v = c.interior(Q, 0)
        for s in range(5):
            assert np.array_equal(v[s].ravel(order="F"), np.array(fields[s]))
        times.append(t)
    assert times == [float("0.695304987880493E-309"), 0.0]     # the subnormal SOLUTIONTIME; no SOLUTIONTIME key


def test_reader_rejects_a_file_that_does_not_fit(tmp_path):
    from mosegpu.tecplot import read_tecplot_ascii
    c = cs.riemann_1d(n=8)
    path = tmp_path / "field.tec"
    write_tecplot_ascii(path, c, c.P0, 0.0)
    with pytest.raises(ValueError, match="nodes"):
        read_tecplot_ascii(path, cs.riemann_1d(n=9))
    text = path.read_text().splitlines()
    (tmp_path / "cut.tec").write_text("\n".join(text[:-3]) + "\n")
    with pytest.raises(ValueError, match="ends"):
        read_tecplot_ascii(tmp_path / "cut.tec", c)
