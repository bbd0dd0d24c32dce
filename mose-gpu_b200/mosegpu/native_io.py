"""The reference's native field file (backup / restart, `bck-format = native`, `rst-format = native`).

`write_native` (`src/lib/io/IO_Solution.f90:450-496`) writes, and `read_native` (`IO_Solution.f90:223-292`) reads,
one Fortran sequential unformatted file opened with `convert='big_endian'`. Every `write` statement is one record:
a 4-byte big-endian length, the data, the same length again. The records, in order:

  1. nb (default integer, int32)
  2. nb records: dim(1) of block b;  nb records: dim(2);  nb records: dim(3)
  3. nb records: the species densities of block b over its interior cells, s fastest, then i, j, k
     (nsc = 1 here: rho over i, j, k)
  4. for s = u, v, w, p: nb records, the variable of block b over its interior cells, i fastest
  5. the simulated time (real(8)); a steady run (`time-accurate = false`) writes -1 (`Wrap_Setup.f90:152-166`)

Ghost cells are not stored: the ghost fill at the start of the next stage rebuilds them.

The engine's state is `P (5, ncell)`, the reference's `P_flat(ncell, 5)` (`MOSE_Field_m.f90:128-146`); a block's
interior is `case.interior(P, b)`. Records of 2**31 bytes or more (a block of more than 268 M cells) have no single
4-byte length and are rejected: compilers split them in ways of their own.
"""
import struct

import numpy as np

NSC = 1
NPRIM = 5
_MAX_REC = 2 ** 31 - 1


def _record(f, payload):
    n = len(payload)
    if n > _MAX_REC:
        raise ValueError(f"native field record of {n} bytes: the 4-byte record length holds at most {_MAX_REC}")
    m = struct.pack(">i", n)
    f.write(m)
    f.write(payload)
    f.write(m)


def _read_record(f, where):
    head = f.read(4)
    if len(head) != 4:
        raise ValueError(f"native field file ends before {where}")
    n = struct.unpack(">i", head)[0]
    if n < 0:
        raise ValueError(f"native field file: record {where} is split (length marker {n}), not supported")
    data = f.read(n)
    tail = f.read(4)
    if len(data) != n or len(tail) != 4 or struct.unpack(">i", tail)[0] != n:
        raise ValueError(f"native field file: record {where} is truncated or its end marker does not match")
    return data


def write_native(path, case, P, time):
    """Writes the interior cells of every block of `case` from the state `P (5, ncell)` (float64, host) and the
    simulated `time` in the layout of `write_native` (IO_Solution.f90:450-496)."""
    P = np.asarray(P, dtype=np.float64)
    if P.shape != (NPRIM, case.ncell):
        raise ValueError(f"state of shape {P.shape}, expected {(NPRIM, case.ncell)}")
    nb = len(case.blocks)
    with open(path, "wb") as f:
        _record(f, struct.pack(">i", nb))
        for d in range(3):
            for b in range(nb):
                _record(f, struct.pack(">i", int(case.blocks[b]["n"][d])))
        # species densities (s fastest, then i, j, k), then u, v, w, p block by block (i fastest)
        for s in range(NPRIM):
            for b in range(nb):
                v = case.interior(P, b)[s]                          # (n1, n2, n3)
                _record(f, np.ascontiguousarray(v.transpose(2, 1, 0)).astype(">f8").tobytes())
        _record(f, struct.pack(">d", float(time)))


def read_native(path, case, P=None):
    """Reads a native field file of `case` (read_native, IO_Solution.f90:223-292). Returns `(P, time)`: the interior
    cells of every block written into a copy of `P` (or of `case.P0` when `P` is None; ghost rows keep those
    values) and the stored time (-1 for a steady run). The block count and dimensions in the file must equal the
    case's (the reference takes them from its mesh file and skips these records; a mismatch here is an error)."""
    base = case.P0 if P is None else P
    out = np.array(base, dtype=np.float64, copy=True)
    if out.shape != (NPRIM, case.ncell):
        raise ValueError(f"state of shape {out.shape}, expected {(NPRIM, case.ncell)}")
    nb = len(case.blocks)
    with open(path, "rb") as f:
        nbf = struct.unpack(">i", _read_record(f, "nb"))[0]
        if nbf != nb:
            raise ValueError(f"native field file holds {nbf} blocks, the case has {nb}")
        for d in range(3):
            for b in range(nb):
                n = struct.unpack(">i", _read_record(f, f"dim({d + 1}) of block {b + 1}"))[0]
                if n != case.blocks[b]["n"][d]:
                    raise ValueError(f"block {b + 1}: dim({d + 1}) = {n} in the file, {case.blocks[b]['n'][d]} in the case")
        for s in range(NPRIM):
            for b in range(nb):
                n1, n2, n3 = case.blocks[b]["n"]
                data = _read_record(f, f"variable {s + 1} of block {b + 1}")
                if len(data) != 8 * n1 * n2 * n3:
                    raise ValueError(f"block {b + 1}: variable {s + 1} has {len(data) // 8} values, expected {n1 * n2 * n3}")
                v = np.frombuffer(data, dtype=">f8").astype(np.float64).reshape(n3, n2, n1).transpose(2, 1, 0)
                case.interior(out, b)[s] = v
        time = struct.unpack(">d", _read_record(f, "time"))[0]
    return out, time
