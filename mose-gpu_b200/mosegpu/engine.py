"""Host binding of the B200 engine through its C ABI (include/mose_b200.h).

torch provides device memory and streams only; every computation runs in the CUDA kernels of
libmose_b200.so. There is no CPU fallback: without the built library or a CUDA device the
constructor raises.

Engine mirrors the reference's per-stage calls (Mod_Explicit.f90:52-279): fill_ghosts
(Fill_Ghost_Cell), residual (Fluxes + BC_Fluxes), update (RK_Newstate), dt (Compute_dt), and the
fused forms stage / step.
"""
import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmose_b200.so")

_lib = None


def load_library():
    """Loads libmose_b200.so (built by mose-gpu_b200/build.py); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libmose_b200.so is not built (run python mose-gpu_b200/build.py): the engine has no "
                           "CPU fallback")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.mb_init.argtypes = [C.POINTER(abi.MBMesh), C.POINTER(abi.MBScheme), C.POINTER(abi.MBThermo), C.c_int,
                          C.POINTER(vp)]
    L.mb_init.restype = C.c_int
    L.mb_destroy.argtypes = [vp]
    L.mb_destroy.restype = None
    L.mb_fill_ghosts.argtypes = [vp, vp, vp]
    L.mb_residual.argtypes = [vp, vp, vp, vp]
    L.mb_update.argtypes = [vp, vp, vp, vp, C.c_int, C.c_double, vp]
    L.mb_dt.argtypes = [vp, vp, C.POINTER(C.c_double), vp]
    L.mb_stage.argtypes = [vp, vp, vp, C.c_int, vp]
    L.mb_step.argtypes = [vp, vp, vp, C.c_int, C.c_int, vp]
    L.mb_begin_step.argtypes = [vp, vp, vp]
    L.mb_get_status.argtypes = [vp, C.POINTER(abi.MBStatus)]
    L.mb_profile_stage.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), vp]
    L.mb_reconfigure.argtypes = [vp, C.POINTER(abi.MBMesh)]
    L.mb_reconfigure_async.argtypes = [vp, C.POINTER(abi.MBMesh), vp]
    L.mb_reconfigure_async.restype = C.c_int
    L.mb_group_reset.argtypes = [vp, C.c_int, C.POINTER(abi.MBGroup), vp, vp]
    L.mb_set_record_params.argtypes = [vp, C.c_int, C.POINTER(C.c_double), vp]
    L.mb_get_group_status.argtypes = [vp, C.c_int, C.c_int, C.POINTER(abi.MBStatus)]
    L.mb_read_group_status.argtypes = [vp, C.c_int, C.c_int, C.POINTER(abi.MBStatus), vp]
    L.mb_autotune.argtypes = [vp, vp, vp]
    L.mb_set_tuning.argtypes = [vp, C.c_int, C.c_int]
    L.mb_get_tuning.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float)]
    L.mb_step_prepare.argtypes = [vp, vp, vp]
    L.mb_copy_dtmin.argtypes = [vp, C.c_int, vp, C.c_int, vp]
    L.mb_step_start.argtypes = [vp, vp]
    L.mb_stage_begin.argtypes = [vp, vp, vp, C.c_int, vp]
    L.mb_stage_input.argtypes = [vp, vp, vp, C.c_int, C.POINTER(vp)]
    L.mb_stage_input.restype = C.c_int
    L.mb_stage_end.argtypes = [vp, vp, vp, C.c_int, vp]
    L.mb_pack_rows.argtypes = [vp, C.c_int64, vp, C.c_int32, vp, vp]
    L.mb_unpack_rows.argtypes = [vp, C.c_int64, vp, C.c_int32, vp, vp]
    L.mb_push_rows.argtypes = [vp, C.c_int64, vp, vp, C.c_int64, vp, C.c_int32, vp]
    L.mb_enable_peer.argtypes = [C.c_int, C.c_int]
    L.mb_enable_peer.restype = C.c_int
    L.mb_ipc_export.argtypes = [vp, vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.mb_ipc_open.argtypes = [vp, C.c_int, C.POINTER(vp)]
    L.mb_ipc_close.argtypes = [vp]
    for f in ("mb_ipc_export", "mb_ipc_open", "mb_ipc_close"):
        getattr(L, f).restype = C.c_int
    for f in ("mb_step_prepare", "mb_copy_dtmin", "mb_step_start", "mb_stage_begin", "mb_stage_end", "mb_pack_rows",
              "mb_unpack_rows", "mb_push_rows"):
        getattr(L, f).restype = C.c_int
    L.mb_selftest_bounded_wait.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int)]
    L.mb_selftest_bounded_wait.restype = C.c_int
    L.mb_set_staging.argtypes = [vp, C.c_int]
    L.mb_set_staging.restype = C.c_int
    L.mb_get_staging.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.mb_get_staging.restype = C.c_int
    L.mb_get_staging_mode.argtypes = [vp, C.POINTER(C.c_int)]
    L.mb_get_staging_mode.restype = C.c_int
    L.mb_launch_count.argtypes = [vp]
    L.mb_launch_count.restype = C.c_int64
    L.mb_version.restype = C.c_char_p
    for f in ("mb_fill_ghosts", "mb_residual", "mb_update", "mb_dt", "mb_stage", "mb_step", "mb_begin_step",
              "mb_get_status", "mb_profile_stage", "mb_reconfigure", "mb_group_reset", "mb_get_group_status",
              "mb_read_group_status", "mb_autotune", "mb_set_tuning", "mb_get_tuning"):
        getattr(L, f).restype = C.c_int
    _lib = L
    return L


def _check(rc, where):
    if rc != abi.MB_OK:
        raise abi.MoseError(rc, where)


class Engine:
    """One case resident on one GPU, driven through the C ABI."""

    def __init__(self, case, precision=abi.PREC_FP64, device=0, stream=None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device: the engine has no CPU fallback")
        self.torch = torch
        self.case = case
        self.dev = torch.device("cuda", device)
        L = load_library()
        self.lib = L
        nb = len(case.blocks)
        self._geo = {}                     # one device copy per geometry array (blocks may share arrays)
        self._blk = (abi.MBBlock * nb)()
        for q, b in enumerate(case.blocks):
            B = self._blk[q]
            B.n[0], B.n[1], B.n[2] = b["n"]
            B.boff = b["boff"]
            B.group = b.get("group", 0)          # -1: an external block (a halo copy, partition.py)
            for f in ("fm1", "fm2", "fm3", "dl", "m", "vol"):
                key = id(b[f])
                if key not in self._geo:
                    self._geo[key] = (b[f], torch.from_numpy(np.ascontiguousarray(b[f], dtype=np.float64)).to(self.dev))
                setattr(B, f, self._geo[key][1].data_ptr())
        self._rec = np.ascontiguousarray(case.rec)
        self._conn = np.ascontiguousarray(case.conn)
        mesh = abi.MBMesh()
        mesh.nblk = nb
        mesh.nrec = len(self._rec)
        mesh.nconn = len(self._conn)
        mesh.ncell_total = case.ncell
        mesh.blk = self._blk
        mesh.rec = self._rec.ctypes.data if len(self._rec) else None
        mesh.conn = self._conn.ctypes.data if len(self._conn) else None
        th = case.thermo
        self._tabs = [np.ascontiguousarray(th[k], dtype=np.float64) for k in ("cp", "h", "mu", "k")]
        T = abi.MBThermo()
        T.tmin, T.tmax, T.wm = th["tmin"], th["tmax"], th["wm"]
        T.cp, T.h, T.mu, T.k = [a.ctypes.data for a in self._tabs]
        sc = case.scheme_struct()
        sc.precision = precision
        self.precision = precision
        self.n_rk = sc.n_rk
        h = C.c_void_p()
        with torch.cuda.device(self.dev):
            _check(L.mb_init(C.byref(mesh), C.byref(sc), C.byref(T), device, C.byref(h)), "mb_init")
        self.ctx = h
        self.stream = stream
        self.P = torch.from_numpy(case.P0.copy()).to(self.dev)          # (5, ncell): P_flat(ncell, 5)
        self.PO = torch.zeros_like(self.P)

    # ------------------------------------------------------------------ plumbing
    def _s(self):
        s = self.stream if self.stream is not None else self.torch.cuda.current_stream(self.dev)
        return C.c_void_p(s.cuda_stream)

    def close(self):
        if getattr(self, "ctx", None) is not None and self.ctx.value:
            self.lib.mb_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, P_host):
        self.P.copy_(self.torch.from_numpy(np.ascontiguousarray(P_host)))

    def state(self):
        return self.P.cpu().numpy()

    def set_staging(self, tma):
        """The mixed sweep's tile staging: 1 TMA (5-value tile), 0 plain loads (6-value tile) (mb_set_staging)."""
        _check(self.lib.mb_set_staging(self.ctx, int(tma)), "mb_set_staging")

    def staging(self):
        """(sweep launches staged by TMA, by plain loads) of the mixed form so far (mb_get_staging)."""
        a, b = C.c_int64(), C.c_int64()
        _check(self.lib.mb_get_staging(self.ctx, C.byref(a), C.byref(b)), "mb_get_staging")
        return a.value, b.value

    def staging_mode(self):
        """The configured staging of the mixed sweep: 1 = the 5-value tile (TMA where a tensor map exists), 0 = the
        6-value tile by plain loads (mb_get_staging_mode)."""
        m = C.c_int()
        _check(self.lib.mb_get_staging_mode(self.ctx, C.byref(m)), "mb_get_staging_mode")
        return m.value

    def staging_label(self):
        """A description of the staging the mixed sweep uses now."""
        if not self.staging_mode():
            return "6-value tile, plain loads"
        return "5-value tile, TMA" if self.staging()[0] > 0 else "5-value tile, plain loads (no tensor map)"

    @property
    def launches(self):
        return int(self.lib.mb_launch_count(self.ctx))

    # ------------------------------------------------------------------ the reference's calls
    def fill_ghosts(self, P=None):
        P = self.P if P is None else P
        _check(self.lib.mb_fill_ghosts(self.ctx, P.data_ptr(), self._s()), "mb_fill_ghosts")

    def residual(self, P=None, R=None):
        P = self.P if P is None else P
        R = self.torch.zeros_like(P) if R is None else R
        _check(self.lib.mb_residual(self.ctx, P.data_ptr(), R.data_ptr(), self._s()), "mb_residual")
        return R

    def update(self, P, PO, R, irk, dt):
        _check(self.lib.mb_update(self.ctx, P.data_ptr(), PO.data_ptr(), R.data_ptr(), irk, dt, self._s()),
               "mb_update")

    def dt(self, P=None):
        P = self.P if P is None else P
        d = C.c_double()
        _check(self.lib.mb_dt(self.ctx, P.data_ptr(), C.byref(d), self._s()), "mb_dt")
        return d.value

    def begin_step(self):
        _check(self.lib.mb_begin_step(self.ctx, self.P.data_ptr(), self._s()), "mb_begin_step")

    def stage(self, irk):
        _check(self.lib.mb_stage(self.ctx, self.P.data_ptr(), self.PO.data_ptr(), irk, self._s()), "mb_stage")

    def step(self, nsteps=1, graph=True):
        _check(self.lib.mb_step(self.ctx, self.P.data_ptr(), self.PO.data_ptr(), nsteps, 1 if graph else 0,
                                self._s()), "mb_step")

    def profile_stage(self, irk, nrep):
        """(ghost-fill ms, sweep ms) averaged over nrep runs of stage irk, CUDA events on the stream."""
        g, w = C.c_float(), C.c_float()
        _check(self.lib.mb_profile_stage(self.ctx, self.P.data_ptr(), self.PO.data_ptr(), irk, nrep, C.byref(g),
                                         C.byref(w), self._s()), "mb_profile_stage")
        return g.value, w.value

    def autotune(self):
        """Runs the sweep autotuner on the current state; returns (k-chunk, persistent, sweep ms)."""
        _check(self.lib.mb_autotune(self.ctx, self.P.data_ptr(), self._s()), "mb_autotune")
        return self.tuning()

    def set_tuning(self, kchunk, persistent):
        _check(self.lib.mb_set_tuning(self.ctx, kchunk, 1 if persistent else 0), "mb_set_tuning")

    def tuning(self):
        k, q, ms = C.c_int(), C.c_int(), C.c_float()
        _check(self.lib.mb_get_tuning(self.ctx, C.byref(k), C.byref(q), C.byref(ms)), "mb_get_tuning")
        return k.value, q.value, ms.value

    def status(self):
        st = abi.MBStatus()
        _check(self.lib.mb_get_status(self.ctx, C.byref(st)), "mb_get_status")
        return st

    def set_record_params(self, rec, q):
        """New parameters (mb_bc.q) of record `rec` from the next stage on (a host-driven time-dependent boundary)."""
        qa = (C.c_double * abi.BC_NQ)(*[float(x) for x in q])
        _check(self.lib.mb_set_record_params(self.ctx, int(rec), qa, self._s()), "mb_set_record_params")

    def save_native(self, path):
        """Backup of the case in the reference's native field file (write_native, IO_Solution.f90:450-496): the
        interior of every block and the simulated time, -1 for a steady run (local_dt) as Wrap_Setup.f90:152-166."""
        from .native_io import write_native
        t = -1.0 if self.case.scheme.get("local_dt", 0) else self.status().time
        write_native(path, self.case, self.state(), t)

    def save_tecplot(self, path):
        """The solution file in Tecplot ASCII (write_vtk_tec, IO_Solution.f90:499-587, through ORION's ASCII
        writer): nodes, the interior primitive variables and T of every block."""
        from .tecplot import write_tecplot_ascii
        t = -1.0 if self.case.scheme.get("local_dt", 0) else self.status().time
        write_tecplot_ascii(path, self.case, self.state(), t)

    def load_tecplot(self, path):
        """Start or restart from a Tecplot ASCII field in ORION's layout (read_vtk_tec, IO_Solution.f90:294-328):
        replaces the interior of every block of the device state; returns (time, steady) of the file."""
        from .tecplot import read_tecplot_ascii
        P, t, steady = read_tecplot_ascii(path, self.case, self.state())
        self.set_state(P)
        self.dt()        # the device minimum of the local steps now belongs to the loaded state (mb_step reuses it)
        return t, steady

    def load_native(self, path):
        """Restart from a native field file (read_native, IO_Solution.f90:223-292): replaces the interior of every
        block of the device state (the ghost rows are refilled by the next stage) and returns the stored time. The
        case clock is not moved: a time-accurate restart that must stop at t_end gives mb_group_reset the time
        still to run."""
        from .native_io import read_native
        P, t = read_native(path, self.case, self.state())
        self.set_state(P)
        self.dt()        # the device minimum of the local steps now belongs to the loaded state (mb_step reuses it)
        return t

    def run_to(self, t_end, max_steps=10 ** 7, chunk=1):
        """Steps until the simulated time reaches t_end (the reference's `time >= timemax` stop) or the case's
        residual stop (scheme res_stop) ends it."""
        n = 0
        while self.status().time < t_end and not self.status().done and n < max_steps:
            self.step(chunk, graph=False)
            n += chunk
        return n
