"""Packs the inputs of the reference's own 1-D regression cases and of its isentropic vortex into
tests/golden/reference_1d_cases.npz, with the md5 pins of their one-iteration field (test/reference_1it.md5).

Run where the reference's test tree is present:
    python tests/golden/make_reference_fixtures.py --reference <path of the MOSE-GPU checkout>
(or with the path in the environment variable MOSE_REFERENCE). The tests read only the npz.

For each case test/<path>: input.ini (kept as text), INPUT/ic.tec (the node coordinates x, y, z and the cell-centred
rho, u, v, w, p of the one block), INPUT/bc.txt (one record per line: block, i, j, k, face, code; a 101 / 201
connection record followed by its donor line: block, i, j, k, face, d11, d12, d21, d22),
INPUT/thermo.dat (T, cp, h of the 1 K table) and INPUT/phase.txt (species and molar mass). The values are parsed as
Fortran's list-directed read does (decimal text to the nearest double), so the arrays hold exactly the reference's
doubles.
"""
import argparse
import hashlib
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["1D/Sod79", "1D/Ein91", "1D/Noh87", "1D/Shu-Osher", "1D/Tor99", "2D/euler/isentropic-vortex"]


def read_ic(path):
    with open(path) as f:
        lines = f.read().split("\n")
    head = lines[1]
    dims = {}
    for key in ("I", "J", "K"):
        tok = head.split(key + "=")[1].split(",")[0]
        dims[key] = int(tok)
    vals = np.array([float(x.replace("D", "E")) for ln in lines[2:] for x in ln.split()], dtype=np.float64)
    ni, nj, nk = dims["I"], dims["J"], dims["K"]
    nn, nc = ni * nj * nk, (ni - 1) * (nj - 1) * (nk - 1)
    assert vals.size == 3 * nn + 5 * nc, (path, vals.size)
    nodes = vals[:3 * nn].reshape(3, nk, nj, ni).transpose(3, 2, 1, 0)          # (ni, nj, nk, 3), i fastest in the file
    cells = vals[3 * nn:].reshape(5, nk - 1, nj - 1, ni - 1).transpose(0, 3, 2, 1)
    return lines[0], head, nodes, cells


def read_bc(path):
    """(records (b, i, j, k, face, code), connections (bs, is, js, ks, fs, d11, d12, d21, d22) aligned with the
    records, -1 where a record has none): a 101 / 201 record line is followed by its connection line."""
    lines = [[int(x) for x in ln.split()] for ln in open(path) if ln.strip()]
    recs, conns = [], []
    q = 0
    while q < len(lines):
        r = lines[q][:6]
        recs.append(r)
        if r[5] in (101, 201):
            conns.append(lines[q + 1][:9])
            q += 2
        else:
            conns.append([-1] * 9)
            q += 1
    return np.array(recs, dtype=np.int32), np.array(conns, dtype=np.int32)


def read_thermo(path):
    rows = []
    for ln in open(path):
        t = ln.split()
        try:
            rows.append([float(x) for x in t[:3]])
        except ValueError:
            continue
    return np.array(rows, dtype=np.float64)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("MOSE_REFERENCE"))
    args = ap.parse_args()
    if not args.reference:
        raise SystemExit("give the reference checkout with --reference or MOSE_REFERENCE")
    ref = args.reference
    pins = {}
    for ln in open(os.path.join(ref, "test", "reference_1it.md5")):
        if ln.strip() and not ln.startswith("#"):
            name, h = ln.split()
            pins[name] = h
    out = {}
    meta = {}
    for path in CASES:
        c = path.split("/")[-1]
        d = os.path.join(ref, "test", path)
        l0, l1, nodes, cells = read_ic(os.path.join(d, "INPUT", "ic.tec"))
        phase = [ln.split() for ln in open(os.path.join(d, "INPUT", "phase.txt")) if ln.strip()][1:]
        out[c + "/nodes"] = nodes
        out[c + "/cells"] = cells
        out[c + "/bc"], out[c + "/conn"] = read_bc(os.path.join(d, "INPUT", "bc.txt"))
        out[c + "/thermo"] = read_thermo(os.path.join(d, "INPUT", "thermo.dat"))
        # md5 of the value lines of ic.tec as ORION wrote them (one E23.15E3 value per line): the formatter of the
        # solution writer is checked against the whole file through it
        ic_lines = open(os.path.join(d, "INPUT", "ic.tec")).read().split("\n")[2:]
        ic_md5 = hashlib.md5("\n".join(ln for ln in ic_lines if ln.strip()).encode()).hexdigest()
        meta[c] = {"ini": open(os.path.join(d, "input.ini")).read().replace("\r", ""), "ic_values_md5": ic_md5,
                   "ic_header": [l0, l1], "species": phase[0][0], "wm": float(phase[0][1]),
                   "md5_1it": pins.get(path.replace("/", "_"))}
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, "reference_1d_cases.npz"), **out)


if __name__ == "__main__":
    main()
