"""The reference's solution file in Tecplot ASCII (`sol-format = tecplot ascii`, the default writer of MOSE).

`write_vtk_tec` (`src/lib/io/IO_Solution.f90:499-587`) fills the ORION field of every block with the primitive
variables of its interior cells and the temperature `T = EOS(p, rho, Rtot) = p / (rho * Rtot)`, with
`Rtot = f_Rtot(rhoi) = 0 + Ri * rho_s / rho` (`lib/FLINT/src/lib/Lib_ThermoTransport.f90:139-146,238-252`), and
`tec_write_structured_multiblock` (`lib/ORION/src/fortran/lib/Lib_Tecplot.f90:71-354`, the `ascii` branch) writes:

  ' VARIABLES ="x" "y" "z" "rho(1)" "u" "v" "w" "p" "T"'          (IO_Solution.f90:347-378)
  per block b:
  ' ZONE  T = Block<b>, I=<n1+1>, J=<n2+1>, K=<n3+1>, DATAPACKING=BLOCK, VARLOCATION=([1-3]=NODAL,[4-9]=CELLCENTERED),
   SOLUTIONTIME=<|time|>'  (one line; ', STRANDID = 0' appended for a steady run, time < 0)
  x, y, z of the nodes (i fastest, then j, k), then each variable over the interior cells (i fastest),
  one value per line in the edit descriptor E23.15E3 (IR_Precision FR8P: the format's single descriptor is reused,
  so every value starts a new record)

Cell-centred variables and no ghost layer are MOSE's settings (`IOfield%tec%node = .false.`, `%bc = .false.`,
IO_Solution.f90:409-418). The optional "thermo" and "transport" variables are not written.

`fortran_e23_15e3(x)` restates Fortran's Ew.dEe editing for w = 23, d = 15, e = 3: the mantissa 0.d1...d15 with the
value rounded to 15 significant digits (nearest), a 3-digit signed exponent, right-justified in 23 characters
(a leading blank for a positive value). Negative zero prints with a minus sign, NaN and infinities as `NaN`,
`Infinity`, `-Infinity` right-justified, as gfortran writes them.
"""
import math

import numpy as np

RUNIV = 8314.46261815324  # Lib_ThermoTransport.f90:13


def fortran_e23_15e3(x):
    x = float(x)
    if math.isnan(x):
        return "NaN".rjust(23)
    if math.isinf(x):
        return ("Infinity" if x > 0 else "-Infinity").rjust(23)
    neg = math.copysign(1.0, x) < 0
    if x == 0.0:
        digits, exp = "0" * 15, 0
    else:
        m, e = ("%.14e" % abs(x)).split("e")     # d.dddddddddddddd, 15 significant digits, rounded to nearest
        digits = m.replace(".", "")
        exp = int(e) + 1                          # 0.d1 d2 ... x 10^(e+1)
    s = "0." + digits + "E" + ("-" if exp < 0 else "+") + "%03d" % abs(exp)
    return ("-" + s if neg else s).rjust(23)


def _int(n):
    """str(no_sign=.true., n) of an integer (IR_Precision str_I4P): the digits without blanks."""
    return str(abs(int(n)))


def _lines(values):
    return "\n".join(fortran_e23_15e3(v) for v in values) + "\n"


def temperature(case, rho, p):
    """T of write_vtk_tec: p / (rho * Rtot), Rtot = 0 + Ri * rho / rho (single species), in that order."""
    ri = RUNIV / case.thermo["wm"]
    rtot = 0.0 + (ri * rho) / rho
    return p / (rho * rtot)


def write_tecplot_ascii(path, case, P, time):
    """Writes the Tecplot ASCII solution file of `case` from the state `P (5, ncell)` (host, float64) at `time`
    (negative for a steady run: the zone then carries |time| and STRANDID = 0, Lib_Tecplot.f90:127-131,318-319)."""
    P = np.asarray(P, dtype=np.float64)
    if P.shape != (5, case.ncell):
        raise ValueError(f"state of shape {P.shape}, expected {(5, case.ncell)}")
    if case.node_fn is None:
        raise ValueError("the case carries no node mapping")
    time_accurate = time >= 0
    t = abs(float(time))
    tstr = fortran_e23_15e3(t)[1:]            # str(no_sign=.true.): drop the sign position
    with open(path, "w") as f:
        f.write(' VARIABLES ="x" "y" "z" "rho(1)" "u" "v" "w" "p" "T"\n')
        for b in range(len(case.blocks)):
            n1, n2, n3 = case.blocks[b]["n"]
            zone = (f" ZONE  T = Block{b + 1}, I={_int(n1 + 1)}, J={_int(n2 + 1)}, K={_int(n3 + 1)}, DATAPACKING=BLOCK"
                    f", VARLOCATION=([1-3]=NODAL,[4-9]=CELLCENTERED), SOLUTIONTIME={tstr}")
            if not time_accurate:
                zone += ", STRANDID = 0"
            f.write(zone + "\n")
            X = case.nodes(b)
            for d in range(3):
                f.write(_lines(X[..., d].ravel(order="F")))
            v = case.interior(P, b)
            for s in range(5):
                f.write(_lines(v[s].ravel(order="F")))
            f.write(_lines(temperature(case, v[0], v[4]).ravel(order="F")))
