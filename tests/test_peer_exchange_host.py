"""The host-side checks of the peer-store exchange between processes (mosegpu.partition.DistPeerExchange), on the CPU
with a stand-in for the library and the process group: a rank maps a receiver's buffers only if every halo row it
will write lies inside the receiver's arena and the arena inside the mapped allocation; buffers of one allocation
are mapped once. These checks are what keeps a wrong plan or a short allocation from becoming a store out of
bounds on the GPU."""
import ctypes as C

import numpy as np
import pytest

from mosegpu import abi
from mosegpu import partition as pt


class _Lib:
    """mb_ipc_export / mb_ipc_open / mb_ipc_close over fake allocations: handle = allocation id."""

    def __init__(self, allocs):
        self.allocs = allocs              # device pointer -> (allocation id, offset, allocation size)
        self.opened = []

    def mb_ipc_export(self, ptr, h, off, size):
        aid, o, sz = self.allocs[ptr]
        C.memmove(h, aid.to_bytes(8, "little") + bytes(56), 64)
        off._obj.value, size._obj.value = o, sz
        return abi.MB_OK

    def mb_ipc_open(self, h, dev, base):
        aid = int.from_bytes(h.value[:1] or b"\0", "little")
        self.opened.append(aid)
        base._obj.value = 1 << 40 | aid << 32
        return abi.MB_OK

    def mb_ipc_close(self, b):
        return abi.MB_OK


class _PG:
    def __init__(self, theirs):
        self.theirs = theirs

    def all_gather_object(self, out, mine):
        for r in range(len(out)):
            out[r] = mine if self.theirs[r] is None else self.theirs[r]

    def barrier(self):
        pass


class _Driver:
    def __init__(self, lib, bufs, ncell):
        self.eng = type("E", (), {"lib": lib})()
        self.dev = type("D", (), {"index": 0})()
        self.rc = type("R", (), {"case": type("Cs", (), {"ncell": ncell})()})()
        self._bufs = bufs

    def stage_buffers(self):
        return list(self._bufs)


def _exchange(receiver_ncell, receiver_alloc_size, dst_rows, share=False):
    lib = _Lib({1000: (1, 0, 10 ** 7), 2000: (2, 0, 10 ** 7), 3000: (3, 0, 10 ** 7)})
    drv = _Driver(lib, [1000, 2000, 3000], ncell=100)
    ids = (7, 7, 7) if share else (7, 8, 9)
    theirs = [(bytes([ids[k]]) + bytes(63), 8 * receiver_ncell * NP5 * k if share else 0, receiver_alloc_size)
              for k in range(3)]
    plan = {(0, 1): (np.array([1, 2]), np.asarray(dst_rows), np.zeros(0, np.int64), np.zeros(0, np.int64))}
    pg = _PG([None, (theirs, receiver_ncell)])
    return pt.DistPeerExchange(drv, plan, 0, 2, pg), lib


NP5 = abi.NPRIM


def test_maps_the_receivers_buffers_when_everything_fits():
    ex, lib = _exchange(50, 50 * NP5 * 8, [3, 49])
    ptrs, nc = ex.peer[1]
    assert nc == 50 and len(ptrs) == 3 and sorted(lib.opened) == [7, 8, 9]


def test_buffers_of_one_allocation_are_mapped_once():
    ex, lib = _exchange(50, 3 * 50 * NP5 * 8, [3, 49], share=True)
    assert lib.opened == [7]
    ptrs, _ = ex.peer[1]
    assert ptrs[1] - ptrs[0] == 50 * NP5 * 8 and ptrs[2] - ptrs[1] == 50 * NP5 * 8


@pytest.mark.parametrize("rows", [[3, 50], [-1, 3]])
def test_refuses_a_row_outside_the_receivers_arena(rows):
    with pytest.raises(RuntimeError, match="outside the arena"):
        _exchange(50, 50 * NP5 * 8, rows)


def test_refuses_an_arena_longer_than_its_allocation():
    with pytest.raises(RuntimeError, match="does not fit"):
        _exchange(50, 50 * NP5 * 8 - 8, [3, 49])
