"""ctypes binding of the CPU oracle (oracle/mose_oracle.cpp). TEST INFRASTRUCTURE ONLY: the tests,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use it as the checker; the product never
imports it.

Builds libmose_oracle.so with the Makefile beside this file if it is missing.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "mose-gpu_b200"))
from mosegpu import abi  # noqa: E402

LIB = os.path.join(HERE, "libmose_oracle.so")


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp = C.c_void_p
        L.orc_init.argtypes = [C.POINTER(abi.MBMesh), C.POINTER(abi.MBScheme), C.POINTER(abi.MBThermo),
                               C.POINTER(vp)]
        L.orc_destroy.argtypes = [vp]
        L.orc_fill_ghosts.argtypes = [vp, vp]
        L.orc_residual.argtypes = [vp, vp, vp]
        L.orc_update.argtypes = [vp, vp, vp, vp, C.c_int, C.c_double]
        L.orc_dt.argtypes = [vp, vp, C.POINTER(C.c_double)]
        L.orc_step.argtypes = [vp, vp, vp, vp, C.c_int]
        L.orc_get_status.argtypes = [vp, C.POINTER(abi.MBStatus)]
        L.orc_set_record_params.argtypes = [vp, C.c_int, C.POINTER(C.c_double)]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def explicit_k_records(case):
    """(records, connections) of the case with the implicit k faces made explicit: a block one cell deep in k with no
    record on faces 5 and 6 gets type-11 (extrapolation) records on every cell of both, appended to its own records
    (faces ordered within the block); the connections' record indices follow the renumbering. The reference's 2-D
    meshes carry those records; the engine takes their absence as the same faces."""
    rec, conn = case.rec, case.conn
    need = [q for q, b in enumerate(case.blocks) if b["n"][2] == 1 and
            not np.any((rec["blk"] == q) & (rec["face"] >= 5))]
    if not need:
        return rec, conn
    parts, newidx, pos = [], np.empty(len(rec), dtype=np.int64), 0
    for q in range(len(case.blocks)):
        sel = np.nonzero(rec["blk"] == q)[0]
        newidx[sel] = pos + np.arange(sel.size)
        parts.append(rec[sel])
        pos += sel.size
        if q in need:
            n1, n2 = case.blocks[q]["n"][:2]
            I, J = [a.ravel(order="F") for a in np.meshgrid(np.arange(1, n1 + 1), np.arange(1, n2 + 1), indexing="ij")]
            for face in (5, 6):
                r = np.zeros(I.size, dtype=abi.BC_DTYPE)
                r["blk"] = q; r["i"] = I; r["j"] = J; r["k"] = 1; r["face"] = face
                r["type"] = abi.BC_EXTRAPOLATION; r["conn"] = -1
                parts.append(r)
                pos += I.size
    rec2 = np.concatenate(parts)
    conn2 = conn.copy()
    if len(conn2):
        conn2["rec"] = newidx[conn2["rec"]]
    return rec2, conn2


class Oracle:
    """The CPU restatement bound to one case (host arrays). A one-plane block without k-face records is run with
    explicit extrapolation records there (explicit_k_records)."""

    def __init__(self, case):
        self.case = case
        L = lib()
        nb = len(case.blocks)
        self._blk = (abi.MBBlock * nb)()
        self._keep = []
        for q, b in enumerate(case.blocks):
            B = self._blk[q]
            B.n[0], B.n[1], B.n[2] = b["n"]
            B.boff = b["boff"]
            B.group = b.get("group", 0)          # -1: an external block (a halo copy, partition.py)
            for f in ("fm1", "fm2", "fm3", "dl", "m", "vol"):
                a = np.ascontiguousarray(b[f], dtype=np.float64)
                self._keep.append(a)
                setattr(B, f, _ptr(a).value)
        rec, conn = explicit_k_records(case)
        self._rec = np.ascontiguousarray(rec)
        self._conn = np.ascontiguousarray(conn)
        mesh = abi.MBMesh()
        mesh.nblk = nb; mesh.nrec = len(self._rec); mesh.nconn = len(self._conn)
        mesh.ncell_total = case.ncell
        mesh.blk = self._blk
        mesh.rec = _ptr(self._rec).value if len(self._rec) else None
        mesh.conn = _ptr(self._conn).value if len(self._conn) else None
        th = case.thermo
        self._tabs = [np.ascontiguousarray(th[k], dtype=np.float64) for k in ("cp", "h", "mu", "k")]
        T = abi.MBThermo()
        T.tmin = th["tmin"]; T.tmax = th["tmax"]; T.wm = th["wm"]
        T.cp, T.h, T.mu, T.k = [_ptr(a).value for a in self._tabs]
        self._mesh, self._th, self._sc = mesh, T, case.scheme_struct()
        h = C.c_void_p()
        rc = L.orc_init(C.byref(mesh), C.byref(self._sc), C.byref(T), C.byref(h))
        if rc != 0:
            raise abi.MoseError(rc, "orc_init")
        self.h = h

    def __del__(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.orc_destroy(self.h)
            self.h = None

    def fill_ghosts(self, P):
        lib().orc_fill_ghosts(self.h, _ptr(P))

    def residual(self, P):
        R = np.zeros_like(P)
        lib().orc_residual(self.h, _ptr(P), _ptr(R))
        return R

    def update(self, P, PO, R, irk, dt):
        return lib().orc_update(self.h, _ptr(P), _ptr(PO), _ptr(R), irk, dt)

    def dt(self, P):
        d = C.c_double()
        lib().orc_dt(self.h, _ptr(P), C.byref(d))
        return d.value

    def step(self, P, nsteps):
        PO = np.zeros_like(P)
        R = np.zeros_like(P)
        rc = lib().orc_step(self.h, _ptr(P), _ptr(PO), _ptr(R), nsteps)
        return rc

    def status(self):
        st = abi.MBStatus()
        lib().orc_get_status(self.h, C.byref(st))
        return st

    def set_record_params(self, rec, q):
        qa = (C.c_double * abi.BC_NQ)(*[float(x) for x in q])
        rc = lib().orc_set_record_params(self.h, int(rec), qa)
        if rc != 0:
            raise abi.MoseError(rc, "orc_set_record_params")

    def run_to(self, P, t_end, max_steps=1000000):
        """Steps until the simulated time reaches t_end (the reference's `time >= timemax` stop)."""
        n = 0
        while self.status().time < t_end and not self.status().done and n < max_steps:
            rc = self.step(P, 1)
            if rc != 0:
                raise abi.MoseError(rc, "orc_step")
            n += 1
        return n
