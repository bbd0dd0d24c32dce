"""The reference's native field file (write_native / read_native, src/lib/io/IO_Solution.f90:223-292,450-496):
the record layout read back byte by byte, round trips, the errors on a file that does not fit the case, and a
restart from the file that continues exactly as the run that was never interrupted (the oracle on the CPU, the
engine through the C ABI on the GPU)."""
import struct

import numpy as np
import pytest

from mosegpu import abi
from mosegpu import case as cs
from mosegpu.native_io import read_native, write_native


def _records(path):
    """Every record of a big-endian Fortran sequential unformatted file, as bytes."""
    out = []
    with open(path, "rb") as f:
        data = f.read()
    p = 0
    while p < len(data):
        n = struct.unpack(">i", data[p:p + 4])[0]
        out.append(data[p + 4:p + 4 + n])
        assert struct.unpack(">i", data[p + 4 + n:p + 8 + n])[0] == n
        p += 8 + n
    return out


def _two_block_case():
    return cs.multiblock_2d(cols=2, rows=1, lo=5, hi=9, seed=3)


def test_record_layout_matches_write_native(tmp_path):
    c = _two_block_case()
    P = np.arange(5 * c.ncell, dtype=np.float64).reshape(5, c.ncell) * 0.5 + 1.0
    path = tmp_path / "field.bin"
    write_native(path, c, P, 0.125)
    recs = _records(path)
    nb = len(c.blocks)
    assert len(recs) == 1 + 3 * nb + 5 * nb + 1
    assert struct.unpack(">i", recs[0])[0] == nb
    for d in range(3):
        for b in range(nb):
            assert struct.unpack(">i", recs[1 + d * nb + b])[0] == c.blocks[b]["n"][d]
    for s in range(5):
        for b in range(nb):
            n1, n2, n3 = c.blocks[b]["n"]
            v = np.frombuffer(recs[1 + 3 * nb + s * nb + b], dtype=">f8")
            # i fastest, then j, k: element (i, j, k) at i + n1*(j + n2*k)
            want = c.interior(P, b)[s]
            assert v.size == n1 * n2 * n3
            for (i, j, k) in [(0, 0, 0), (n1 - 1, 0, 0), (1, n2 - 1, 0), (n1 - 1, n2 - 1, n3 - 1)]:
                assert v[i + n1 * (j + n2 * k)] == want[i, j, k]
    assert struct.unpack(">d", recs[-1])[0] == 0.125


def test_round_trip_interior_and_ghosts(tmp_path):
    c = cs.taylor_green(n=6, blocks=2)
    rng = np.random.default_rng(11)
    P = rng.standard_normal((5, c.ncell))
    path = tmp_path / "field.bin"
    write_native(path, c, P, -1.0)
    base = rng.standard_normal((5, c.ncell))
    Q, t = read_native(path, c, base)
    assert t == -1.0
    m = c.interior_mask()
    assert np.array_equal(Q[:, m], P[:, m])            # interior from the file, bit for bit
    assert np.array_equal(Q[:, ~m], base[:, ~m])       # ghost rows from the given state


def test_mismatched_or_truncated_file_is_rejected(tmp_path):
    c = _two_block_case()
    path = tmp_path / "field.bin"
    write_native(path, c, c.P0, 0.0)
    with pytest.raises(ValueError, match="blocks"):
        read_native(path, cs.multiblock_2d(cols=3, rows=1, lo=5, hi=9, seed=3))
    other = cs.multiblock_2d(cols=2, rows=1, lo=5, hi=9, seed=4)
    if [b["n"] for b in other.blocks] != [b["n"] for b in c.blocks]:
        with pytest.raises(ValueError, match="dim"):
            read_native(path, other)
    data = path.read_bytes()
    (tmp_path / "cut.bin").write_bytes(data[:-6])
    with pytest.raises(ValueError):
        read_native(tmp_path / "cut.bin", c)
    with pytest.raises(ValueError, match="shape"):
        write_native(path, c, c.P0[:, :-1], 0.0)


def test_restart_continues_as_the_uninterrupted_run_oracle(tmp_path):
    import oracle
    c = cs.taylor_green(n=8, blocks=2, riemann=abi.RS_HLLC, noise=1e-3)
    P = c.P0.copy()
    o = oracle.Oracle(c)
    assert o.step(P, 2) == 0
    path = tmp_path / "field.bin"
    write_native(path, c, P, o.status().time)
    assert o.step(P, 2) == 0                                 # uninterrupted: 4 steps
    Q, t = read_native(path, c)                              # restart on the initial ghost rows
    assert t > 0.0
    o2 = oracle.Oracle(c)
    assert o2.step(Q, 2) == 0
    m = c.interior_mask()
    assert np.array_equal(Q[:, m], P[:, m])


@pytest.mark.gpu
def test_restart_continues_as_the_uninterrupted_run_engine(tmp_path):
    from mosegpu.engine import Engine
    c = cs.taylor_green(n=12, blocks=2, riemann=abi.RS_HLLC, noise=1e-3)
    e = Engine(c)
    e.step(2, graph=False)
    path = tmp_path / "field.bin"
    e.save_native(path)
    t_saved = e.status().time
    e.step(2, graph=False)
    e2 = Engine(c)
    t = e2.load_native(path)
    assert t == t_saved
    e2.step(2, graph=False)
    m = c.interior_mask()
    assert np.array_equal(e2.state()[:, m], e.state()[:, m])
    # an engine that has stepped already: the loaded state, not its own, sets the next step
    e3 = Engine(c)
    e3.step(1, graph=False)
    e3.load_native(path)
    e3.step(2, graph=False)
    assert np.array_equal(e3.state()[:, m], e.state()[:, m])
    for x in (e, e2, e3):
        x.close()
