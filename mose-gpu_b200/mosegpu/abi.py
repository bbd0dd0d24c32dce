"""ctypes mirror of include/mose_b200.h (the C ABI of the engine).

The structures follow the header field for field; the numpy record dtypes below are the
same layouts, so a record table built in numpy is handed to C by pointer.
"""
import ctypes as C

import numpy as np

GC = 2
NSC = 1
NPRIM = 5
BC_NQ = 12

MB_OK = 0
MB_E_ARG = -1
MB_E_UNSUPPORTED = -2
MB_E_CUDA = -3
MB_E_STATE = -4
MB_E_THERMO = -5
MB_E_BUDGET = -6
MB_E_TIMEOUT = -7
MB_E_NOMEM = -8
MB_E_NODEV = -9

STATUS_NAMES = {
    MB_OK: "ok", MB_E_ARG: "bad argument", MB_E_UNSUPPORTED: "unsupported scheme or boundary type",
    MB_E_CUDA: "CUDA error", MB_E_STATE: "non-physical state (p < 0 or NaN)",
    MB_E_THERMO: "temperature off the thermo table", MB_E_BUDGET: "HBM budget exceeded",
    MB_E_TIMEOUT: "device wait timed out", MB_E_NOMEM: "device allocation failed",
    MB_E_NODEV: "no CUDA device",
}

BC_NONE = 0          # no condition (bc.txt 0): zero-gradient ghosts, no face flux
BC_CONNECTION = 1
BC_INFLOW = 4
BC_WALL = 5
BC_EXTRAPOLATION = 11
BC_SYMMETRY = 3
BC_WALL_T = 6       # q = (T_wall,)
BC_OUTLET = 24      # q = (exit pressure, relaxation factor)

LIM_MINMOD, LIM_VANLEER, LIM_VANALBADA, LIM_MC, LIM_SUPERBEE, LIM_FIRST = 1, 2, 3, 4, 5, 6
RS_HLLC, RS_HLLE, RS_SLAU, RS_AUSMP, RS_LLF, RS_SLAU2, RS_LMROE = 1, 2, 3, 4, 8, 9, 12
RS_EXACT, RS_MICZEKROE, RS_HLLC_PC = 11, 13, 14
RS_AUSMPM, RS_HLLEPP, RS_HLLC_TRAMEL, RS_HLLC_CHEN = 5, 6, 7, 10
SENSOR_DEFAULT, SENSOR_TRAMEL, SENSOR_CHEN, SENSOR_NONE = 0, 1, 2, 3
INTVAR_CONS, INTVAR_PRIM, INTVAR_PREC = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
PREC_FP64_FAST = 2   # FP64 values, the simplified flux path with FMA (the gates, not bit parity)


class MBBlock(C.Structure):
    _fields_ = [("n", C.c_int32 * 3), ("group", C.c_int32), ("boff", C.c_int64),
                ("fm1", C.c_void_p), ("fm2", C.c_void_p), ("fm3", C.c_void_p),
                ("dl", C.c_void_p), ("m", C.c_void_p), ("vol", C.c_void_p)]


class MBBc(C.Structure):
    _fields_ = [("blk", C.c_int32), ("i", C.c_int32), ("j", C.c_int32), ("k", C.c_int32),
                ("face", C.c_int32), ("type", C.c_int32), ("conn", C.c_int32), ("pad0", C.c_int32),
                ("q", C.c_double * BC_NQ)]


class MBConn(C.Structure):
    _fields_ = [("rec", C.c_int32), ("bs", C.c_int32), ("is_", C.c_int32), ("js", C.c_int32),
                ("ks", C.c_int32), ("fs", C.c_int32), ("d11", C.c_int32), ("d12", C.c_int32),
                ("d21", C.c_int32), ("d22", C.c_int32)]


class MBMesh(C.Structure):
    _fields_ = [("nblk", C.c_int32), ("nrec", C.c_int32), ("nconn", C.c_int32), ("ngroups", C.c_int32),
                ("ncell_total", C.c_int64), ("blk", C.POINTER(MBBlock)), ("rec", C.c_void_p),
                ("conn", C.c_void_p)]


class MBThermo(C.Structure):
    _fields_ = [("tmin", C.c_int32), ("tmax", C.c_int32), ("wm", C.c_double),
                ("cp", C.c_void_p), ("h", C.c_void_p), ("mu", C.c_void_p), ("k", C.c_void_p)]


class MBScheme(C.Structure):
    _fields_ = [("limiter", C.c_int32), ("riemann", C.c_int32), ("visc", C.c_int32), ("n_rk", C.c_int32),
                ("precision", C.c_int32), ("ndir", C.c_int32), ("time_clip", C.c_int32),
                ("state_check", C.c_int32), ("dt_additive", C.c_int32), ("sensor", C.c_int32),
                ("intvar", C.c_int32), ("irs", C.c_int32),
                ("cfl", C.c_double), ("vnn", C.c_double),
                ("prandtl", C.c_double), ("schmidt", C.c_double), ("mco", C.c_double),
                ("time_threshold", C.c_double), ("res_stop", C.c_double), ("irs_beta", C.c_double),
                ("local_dt", C.c_int32), ("cfl_rise", C.c_int32), ("prec_smooth", C.c_int32), ("pad2", C.c_int32),
                ("prec_eps_min", C.c_double), ("prec_uref", C.c_double), ("prec_mach", C.c_double),
                ("prec_ur_factor", C.c_double), ("prec_ur_min", C.c_double)]


class MBStatus(C.Structure):
    _fields_ = [("code", C.c_int32), ("n_bad_state", C.c_int32), ("n_bad_thermo", C.c_int32),
                ("bad_blk", C.c_int32), ("bad_i", C.c_int32), ("bad_j", C.c_int32), ("bad_k", C.c_int32),
                ("steps", C.c_int32), ("time", C.c_double), ("dt", C.c_double), ("done", C.c_int32),
                ("pad0", C.c_int32), ("res", C.c_double * 5)]


class MBGroup(C.Structure):
    _fields_ = [("time_clip", C.c_int32), ("pad0", C.c_int32), ("t_end", C.c_double), ("res_stop", C.c_double)]


BC_DTYPE = np.dtype([("blk", "<i4"), ("i", "<i4"), ("j", "<i4"), ("k", "<i4"), ("face", "<i4"),
                     ("type", "<i4"), ("conn", "<i4"), ("pad0", "<i4"), ("q", "<f8", (BC_NQ,))])
CONN_DTYPE = np.dtype([("rec", "<i4"), ("bs", "<i4"), ("is", "<i4"), ("js", "<i4"), ("ks", "<i4"),
                       ("fs", "<i4"), ("d11", "<i4"), ("d12", "<i4"), ("d21", "<i4"), ("d22", "<i4")])
assert BC_DTYPE.itemsize == C.sizeof(MBBc)
assert CONN_DTYPE.itemsize == C.sizeof(MBConn)


def status_message(code):
    return STATUS_NAMES.get(int(code), "status %d" % int(code))


class MoseError(RuntimeError):
    """A non-zero status returned through the C ABI (the reference would `error stop` here)."""

    def __init__(self, code, where):
        self.code = int(code)
        super().__init__("%s: %s (%d)" % (where, status_message(code), int(code)))
