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
IO_Solution.f90:409-418). The "thermo" variables are MOSE's default (`sol-variables = thermo`, IO_Solution.f90:128):
after T come "g" = f_gamma = cp / (cp - Rtot), cp from the 1 K table at T (f_cp, Lib_ThermoTransport.f90:273-293,
329-339; the row idint(T), no clamp), and "R" = Rtot (IO_Solution.f90:384-389,536-539); `variables=""` writes T only
(`sol-variables` without "thermo"). The optional "transport" variables are not written.

`fortran_e23_15e3(x)` restates Fortran's Ew.dEe editing for w = 23, d = 15, e = 3: the mantissa 0.d1...d15 with the
value rounded to 15 significant digits (nearest), a 3-digit signed exponent, right-justified in 23 characters
(a leading blank for a positive value). Negative zero prints with a minus sign, NaN and infinities as `NaN`,
`Infinity`, `-Infinity` right-justified, as gfortran writes them.
"""
import math
import re

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


def gamma_rtot(case, rho, p):
    """g and R of write_vtk_tec's "thermo" variables: Rtot = 0 + Ri rho / rho, T = p / (Rtot rho), cp = 0 + rho / rho
    (cp(int T) + (cp(int T + 1) - cp(int T)) (T - int T)), g = cp / (cp - Rtot), in that order (one species)."""
    th = case.thermo
    ri = RUNIV / th["wm"]
    rtot = 0.0 + (ri * rho) / rho
    T = p / (rtot * rho)
    ti = np.trunc(T).astype(np.int64)
    td = T - ti
    cpt = th["cp"]
    c1, c2 = cpt[ti - th["tmin"]], cpt[ti + 1 - th["tmin"]]
    cp = 0.0 + (rho / rho) * (c1 + (c2 - c1) * td)
    return cp / (cp - rtot), rtot


def write_tecplot_ascii(path, case, P, time, variables="thermo"):
    """Writes the Tecplot ASCII solution file of `case` from the state `P (5, ncell)` (host, float64) at `time`
    (negative for a steady run: the zone then carries |time| and STRANDID = 0, Lib_Tecplot.f90:127-131,318-319).
    variables: "thermo" (MOSE's default: T, g, R after the primitives) or "" (T only)."""
    P = np.asarray(P, dtype=np.float64)
    if P.shape != (5, case.ncell):
        raise ValueError(f"state of shape {P.shape}, expected {(5, case.ncell)}")
    if case.node_fn is None:
        raise ValueError("the case carries no node mapping")
    time_accurate = time >= 0
    t = abs(float(time))
    tstr = fortran_e23_15e3(t)[1:]            # str(no_sign=.true.): drop the sign position
    thermo = "thermo" in variables
    nvt = 3 + 6 + (2 if thermo else 0)
    with open(path, "w") as f:
        f.write(' VARIABLES ="x" "y" "z" "rho(1)" "u" "v" "w" "p" "T"' + (' "g" "R"' if thermo else "") + "\n")
        for b in range(len(case.blocks)):
            n1, n2, n3 = case.blocks[b]["n"]
            zone = (f" ZONE  T = Block{b + 1}, I={_int(n1 + 1)}, J={_int(n2 + 1)}, K={_int(n3 + 1)}, DATAPACKING=BLOCK"
                    f", VARLOCATION=([1-3]=NODAL,[4-{nvt}]=CELLCENTERED), SOLUTIONTIME={tstr}")
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
            if thermo:
                g, r = gamma_rtot(case, v[0], v[4])
                f.write(_lines(g.ravel(order="F")))
                f.write(_lines(r.ravel(order="F")))


def _zone_fields(text):
    """KEY=value pairs of zone header text (T, I, J, K, DATAPACKING, VARLOCATION, SOLUTIONTIME, STRANDID ...)."""
    out = {}
    for m in re.finditer(r"([A-Za-z]+)\s*=\s*(\([^)]*\)\)?|\"[^\"]*\"|[^,\s]+)", text):
        out[m.group(1).upper()] = m.group(2)
    return out


def _is_number_line(line):
    try:
        [float(x.replace("D", "E").replace("d", "e")) for x in line.split()]
        return bool(line.split())
    except ValueError:
        return False


def read_tecplot_ascii(path, case, P=None):
    """Reads a Tecplot ASCII field in ORION's structured block layout (tec_read_structured_multiblock, ascii branch,
    Lib_Tecplot.f90:452-600: one zone per block, nodal x, y, z, then cell-centred variables; the reader of an
    `ini-format` / `rst-format = tecplot ascii` start, read_vtk_tec, IO_Solution.f90:294-328). Returns
    `(P, time, steady)`: the first five variables of every zone (rho, u, v, w, p; further ones such as T are skipped,
    as the reference keeps only its nprim) written into the interior of a copy of `P` (or of `case.P0`), the zone's
    SOLUTIONTIME and whether the zone carries a STRANDID (a steady run's file). The zone count and I, J, K must match
    the case's blocks (nodes = cells + 1); nodal variables are not served (ORION writes MOSE's fields cell-centred)."""
    base = case.P0 if P is None else P
    out = np.array(base, dtype=np.float64, copy=True)
    with open(path) as f:
        lines = f.read().splitlines()
    names = None
    q = 0
    while q < len(lines) and "ZONE" not in lines[q].upper():
        if "VARIABLES" in lines[q].upper():
            names = re.findall(r"\"([^\"]*)\"", lines[q])
        q += 1
    if not names or len(names) < 8:
        raise ValueError("no VARIABLES line with x, y, z and five field variables")
    nvar = len(names) - 3
    time, steady = 0.0, False
    for b in range(len(case.blocks)):
        if q >= len(lines):
            raise ValueError(f"the file holds {b} zones, the case has {len(case.blocks)} blocks")
        head = []
        while q < len(lines) and not _is_number_line(lines[q]):
            head.append(lines[q])
            q += 1
        z = _zone_fields(" ".join(head))
        n1, n2, n3 = case.blocks[b]["n"]
        dims = tuple(int(z.get(k, "0")) for k in ("I", "J", "K"))
        if dims != (n1 + 1, n2 + 1, n3 + 1):
            raise ValueError(f"zone {b + 1}: I, J, K = {dims}, the block has {(n1 + 1, n2 + 1, n3 + 1)} nodes")
        if "CELLCENTERED" not in z.get("VARLOCATION", "").upper():
            raise ValueError(f"zone {b + 1}: the variables are not cell-centred")
        if "SOLUTIONTIME" in z:
            time = float(z["SOLUTIONTIME"].replace("D", "E"))
        steady = "STRANDID" in z
        nn, nc = (n1 + 1) * (n2 + 1) * (n3 + 1), n1 * n2 * n3
        need = 3 * nn + nvar * nc
        vals = []
        while len(vals) < need:
            if q >= len(lines):
                raise ValueError(f"zone {b + 1}: the file ends after {len(vals)} of {need} values")
            vals += [float(x.replace("D", "E").replace("d", "e")) for x in lines[q].split()]
            q += 1
        if len(vals) != need:
            raise ValueError(f"zone {b + 1}: {len(vals)} values, expected {need}")
        v = np.asarray(vals[3 * nn:], dtype=np.float64)
        for s in range(5):
            case.interior(out, b)[s] = v[s * nc:(s + 1) * nc].reshape(n3, n2, n1).transpose(2, 1, 0)
    return out, time, steady
