"""Continuous batching of independent cases on one GPU (no counterpart in the reference, which runs one case
per process).

A `Server` owns one engine context whose arena holds every admitted case: each case is one group of blocks
with its own clock (dt = the minimum over its own cells, its own stop time), so a case advances exactly as it
would alone. Every step of the batch is one replay of the captured step graph: per stage one ghost fill and
ONE sweep over the tiles of all running cases. Between bursts of `poll_steps` steps the host reads the case
clocks (one device read), downloads finished cases, frees their rows and clock, and admits arrived requests
while the HBM budget, a contiguous range of arena rows and a clock are free; admitting rebuilds the context's
tables (mb_reconfigure_async, ordered on the lane's stream: the other lanes keep running) without touching the state
of the running cases.

Cases of one server share the scheme (limiter, Riemann solver, RK, precision, CFL) and the thermo table; each
brings its own mesh, initial state and stop time. Cases with equal meshes share one device copy of the
geometry (the request's `geo_key`).
"""
import ctypes as C
import math
import time

import numpy as np

from . import abi
from . import case as cs
from .engine import _check, load_library

ROW_BYTES_STATE = 3 * 5 * 8          # P, PO and the engine's stage buffer, per arena row
GEO_BYTES_PER_CELL = (3 * 4 + 3 + 9 + 1) * 8


class Request:
    """One case to solve: a Case (cs.layout_case) with its stop time (and, for a steady case, the residual of rho
    at which it stops: res_stop, 0 = none), arriving at `arrival` seconds."""

    def __init__(self, rid, case, t_end, arrival=0.0, geo_key=None, res_stop=0.0):
        self.rid = rid
        self.case = case
        self.t_end = float(t_end)
        self.res_stop = float(res_stop)
        self.arrival = float(arrival)
        self.geo_key = geo_key
        self.npad = int(case.ncell)
        self.start = None        # admission time
        self.finish = None       # result on the host
        self.result = None       # (5, npad) primitive state of the case's own rows
        self.status = None
        self.error = None        # MB_E_BUDGET: the case cannot fit the server even when it is empty
        self.steps = 0


class _Ranges:
    """First-fit allocator of arena rows with coalescing."""

    def __init__(self, n):
        self.free = [(0, n)]

    def alloc(self, n):
        for q, (a, b) in enumerate(self.free):
            if b - a >= n:
                if b - a == n:
                    self.free.pop(q)
                else:
                    self.free[q] = (a + n, b)
                return a
        return None

    def release(self, a, n):
        self.free.append((a, a + n))
        self.free.sort()
        out = []
        for x, y in self.free:
            if out and out[-1][1] == x:
                out[-1] = (out[-1][0], y)
            else:
                out.append((x, y))
        self.free = out


class Server:
    """Continuous-batching server of independent cases (see the module docstring).

    scheme       : dict of the shared scheme (as Case.scheme; time_clip / time_threshold are per request)
    thermo       : the shared thermo table (cs.ideal_gas_tables)
    budget_bytes : HBM the server may use for state rows and geometry
    max_cases    : case clocks (groups) of the context
    """

    def __init__(self, scheme, thermo, budget_bytes, max_cases=256, precision=abi.PREC_MIXED, device=0,
                 poll_steps=16, arena_rows=None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device: the engine has no CPU fallback")
        if max_cases < 2:
            raise ValueError("a server batches at least two cases")
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.L = load_library()
        self.scheme = dict(scheme)
        self.thermo = thermo
        self.budget = int(budget_bytes)
        self.max_cases = int(max_cases)
        self.precision = precision
        self.poll_steps = int(poll_steps)
        per_row = ROW_BYTES_STATE + (40 if scheme.get("n_rk", 3) == 4 else 0)
        self.rows = int(arena_rows) if arena_rows else max(1, self.budget // (2 * per_row))
        self.used_bytes = self.rows * per_row
        self.P = torch.zeros((5, self.rows), dtype=torch.float64, device=self.dev)
        self.PO = torch.zeros_like(self.P)
        self.stream = torch.cuda.Stream(self.dev)
        self.ranges = _Ranges(self.rows)
        self.free_groups = list(range(self.max_cases))[::-1]
        self.geo = {}            # geo_key -> [device tensors, refcount, bytes]
        self.active = {}         # group -> (request, boff)
        self.done = []
        self.ctx = None
        self._tabs = [np.ascontiguousarray(thermo[k], dtype=np.float64) for k in ("cp", "h", "mu", "k")]
        self.steps = 0
        self.launches = 0
        self.rounds = 0          # admission rounds (table rebuilds)

    # ------------------------------------------------------------------ device tables
    def _s(self):
        return C.c_void_p(self.stream.cuda_stream)

    def _geometry(self, req):
        key = req.geo_key if req.geo_key is not None else ("req", req.rid)
        g = self.geo.get(key)
        if g is None:
            ts = []
            nbytes = 0
            for b in req.case.blocks:
                d = {}
                for f in ("fm1", "fm2", "fm3", "dl", "m", "vol"):
                    t = self.torch.from_numpy(np.ascontiguousarray(b[f], dtype=np.float64)).to(self.dev)
                    d[f] = t
                    nbytes += t.numel() * 8 * (1.5 if self.precision == abi.PREC_MIXED and f != "vol" else 1)
                ts.append(d)
            g = [ts, 0, int(nbytes)]
            self.geo[key] = g
            self.used_bytes += g[2]
        g[1] += 1
        return key, g[0]

    def _drop_geometry(self, req):
        key = req.geo_key if req.geo_key is not None else ("req", req.rid)
        g = self.geo[key]
        g[1] -= 1
        if g[1] == 0:
            self.used_bytes -= g[2]
            del self.geo[key]

    def _mesh(self):
        """The mb_mesh of every admitted case (running or finished but not yet retired)."""
        blks, recs, conns = [], [], []
        nb = 0
        nr = 0
        for grp in sorted(self.active):
            req, boff, geo = self.active[grp]
            c = req.case
            for q, b in enumerate(c.blocks):
                blks.append((b["n"], grp, boff + b["boff"], geo[q]))
            r = c.rec.copy()
            r["blk"] += nb
            r["conn"] = np.where(r["conn"] >= 0, r["conn"] + sum(len(x) for x in conns), -1)
            cn = c.conn.copy()
            cn["rec"] += nr
            cn["bs"] += nb
            recs.append(r)
            conns.append(cn)
            nb += len(c.blocks)
            nr += len(r)
        self._blk = (abi.MBBlock * len(blks))()
        for q, (n, grp, boff, g) in enumerate(blks):
            B = self._blk[q]
            B.n[0], B.n[1], B.n[2] = n
            B.group = grp
            B.boff = boff
            for f in ("fm1", "fm2", "fm3", "dl", "m", "vol"):
                setattr(B, f, g[f].data_ptr())
        self._rec = np.ascontiguousarray(np.concatenate(recs)) if recs else np.zeros(0, dtype=abi.BC_DTYPE)
        self._conn = np.ascontiguousarray(np.concatenate(conns)) if conns else np.zeros(0, dtype=abi.CONN_DTYPE)
        mesh = abi.MBMesh()
        mesh.nblk = len(blks)
        mesh.nrec = len(self._rec)
        mesh.nconn = len(self._conn)
        mesh.ngroups = self.max_cases
        mesh.ncell_total = self.rows
        mesh.blk = self._blk
        mesh.rec = self._rec.ctypes.data if len(self._rec) else None
        mesh.conn = self._conn.ctypes.data if len(self._conn) else None
        return mesh

    def _rebuild(self):
        mesh = self._mesh()
        if mesh.nblk == 0:
            return
        if self.ctx is None:
            T = abi.MBThermo()
            th = self.thermo
            T.tmin, T.tmax, T.wm = th["tmin"], th["tmax"], th["wm"]
            T.cp, T.h, T.mu, T.k = [a.ctypes.data for a in self._tabs]
            tmp = cs.Case("server")
            tmp.scheme = dict(self.scheme)
            sc = tmp.scheme_struct()
            sc.precision = self.precision
            h = C.c_void_p()
            with self.torch.cuda.device(self.dev):
                _check(self.L.mb_init(C.byref(mesh), C.byref(sc), C.byref(T), self.dev.index, C.byref(h)), "mb_init")
            self.ctx = h
        else:
            # stream-ordered: the other lanes' work is not drained
            _check(self.L.mb_reconfigure_async(self.ctx, C.byref(mesh), self._s()), "mb_reconfigure_async")

    # ------------------------------------------------------------------ admission / retirement
    def fits(self, req):
        geo_new = 0 if (req.geo_key is not None and req.geo_key in self.geo) else \
            sum(b["m"].size // 9 for b in req.case.blocks) * GEO_BYTES_PER_CELL * (1.5 if self.precision else 1)
        return self.used_bytes + geo_new <= self.budget

    def try_admit(self, req, now):
        """Admits req if its rows, a clock and the HBM budget are free; returns True when admitted."""
        if not self.free_groups or not self.fits(req):
            return False
        boff = self.ranges.alloc(req.npad)
        if boff is None:
            return False
        grp = self.free_groups.pop()
        _, geo = self._geometry(req)
        host = self.torch.from_numpy(np.ascontiguousarray(req.case.P0)).pin_memory()
        with self.torch.cuda.stream(self.stream):
            self.P[:, boff:boff + req.npad].copy_(host, non_blocking=True)
        self.active[grp] = (req, boff, geo)
        req.start = now
        req.group = grp
        req.admit_round = self.rounds
        return True

    def commit_admissions(self, new_groups):
        """Rebuilds the tables for the admitted set and starts the clocks of the new cases."""
        self.rounds += 1
        self._rebuild()
        for grp in new_groups:
            req = self.active[grp][0]
            spec = abi.MBGroup()
            spec.time_clip = 1
            spec.t_end = req.t_end
            spec.res_stop = req.res_stop
            _check(self.L.mb_group_reset(self.ctx, grp, C.byref(spec), self.P.data_ptr(), self._s()), "mb_group_reset")

    def poll(self, now_fn):
        """Reads every clock; downloads and retires the finished cases. Returns the retired requests."""
        if self.ctx is None or not self.active:
            return []
        st = (abi.MBStatus * self.max_cases)()
        _check(self.L.mb_read_group_status(self.ctx, 0, self.max_cases, st, self._s()), "mb_read_group_status")
        out = []
        for grp in list(self.active):
            s = st[grp]
            if s.done or s.code != abi.MB_OK:
                req, boff, _ = self.active.pop(grp)
                with self.torch.cuda.stream(self.stream):
                    req.result = self.P[:, boff:boff + req.npad].cpu().numpy()
                req.finish = now_fn()
                req.status = s
                req.steps = s.steps
                self.ranges.release(boff, req.npad)
                self.free_groups.append(grp)
                self._drop_geometry(req)
                out.append(req)
        return out

    def advance(self, nsteps):
        _check(self.L.mb_step(self.ctx, self.P.data_ptr(), self.PO.data_ptr(), nsteps, 1, self._s()), "mb_step")
        self.steps += nsteps

    def close(self):
        if self.ctx is not None:
            self.L.mb_destroy(self.ctx)
            self.ctx = None

    # ------------------------------------------------------------------ the request loop
    def serve(self, requests, max_wall=None):
        """Serves `requests` (arrival times in seconds from the start) on this server alone; returns them with
        their start / finish times (see serve_lanes)."""
        return serve_lanes([self], lambda r: 0, requests, max_wall=max_wall)


def serve_lanes(lanes, route, requests, max_wall=None):
    """The request loop over one or more servers ("lanes", each an engine context with its own arena, clocks and
    stream). route(request) picks a request's lane: cases whose steps cost about the same share a lane, so that a
    cheap case with many steps is not held to the step time of an expensive one. The lanes run independently on
    their streams: whenever a lane's last burst of poll_steps steps has finished on the GPU, the loop reads its
    clocks (waiting for that stream only), retires its finished cases, admits what fits of its queue (a request
    that cannot fit its empty lane is rejected with MB_E_BUDGET) and launches its next burst. With nothing running
    it waits for the next arrival. Returns the finished requests."""
    import torch
    pending = sorted(requests, key=lambda r: r.arrival)
    t0 = time.perf_counter()
    now = lambda: time.perf_counter() - t0  # noqa: E731
    qi = 0
    waiting = [[] for _ in lanes]
    events = [None for _ in lanes]       # the event after a lane's burst in flight
    finished = []
    while qi < len(pending) or any(waiting) or any(l.active for l in lanes):
        if max_wall is not None and now() > max_wall:
            break
        while qi < len(pending) and pending[qi].arrival <= now():
            waiting[route(pending[qi])].append(pending[qi])
            qi += 1
        progressed = False
        for li, (lane, wq) in enumerate(zip(lanes, waiting)):
            if events[li] is not None:
                if not events[li].query():
                    continue
                events[li] = None
                finished += lane.poll(now)
            new = []
            while wq:
                if lane.try_admit(wq[0], now()):
                    new.append(wq.pop(0).group)
                elif not lane.active and not new:
                    # nothing runs in the lane and it still does not fit: it never will (rows or HBM budget)
                    r = wq.pop(0)
                    r.error = abi.MB_E_BUDGET
                    r.finish = now()
                    finished.append(r)
                else:
                    break
            if new:
                lane.commit_admissions(new)
            if lane.active:
                lane.advance(lane.poll_steps)
                events[li] = torch.cuda.Event()
                events[li].record(lane.stream)
                progressed = True
        if not progressed:
            if all(e is None for e in events) and qi < len(pending):
                time.sleep(max(0.0, min(pending[qi].arrival - now(), 0.01)))
            else:
                time.sleep(5e-5)
    for lane in lanes:
        lane.stream.synchronize()
    return finished


# ---------------------------------------------------------------------- the serving request stream
_TEMPLATES = {}


def riemann_request(rid, dim, n, states, t_end, arrival=0.0):
    """A 1-D or 2-D Riemann case on [0,1]^dim with n cells per direction (HLLC + MUSCL minmod, SSP-RK3,
    CFL 0.5, extrapolation on every face, gamma 1.4). 1-D: states = (left, right) of (rho, u, p); 2-D:
    states = four quadrant states (rho, u, v, p) for (x>.5,y>.5), (x<.5,y>.5), (x<.5,y<.5), (x>.5,y<.5).
    Cases of one (dim, n) share the mesh (geometry, records) and differ only in their initial state."""
    key = (dim, n)
    base = _TEMPLATES.get(key)
    if base is None:
        base = cs.riemann_1d(n=n, t_end=t_end, compact=True) if dim == 1 else cs.riemann_2d(n=n, t_end=t_end, compact=True)
        _TEMPLATES[key] = base
    c = cs.Case(base.name)
    c.blocks, c.rec, c.conn, c.ncell, c.thermo = base.blocks, base.rec, base.conn, base.ncell, base.thermo
    c.scheme = dict(base.scheme, time_threshold=t_end)
    P = np.zeros((5, c.ncell), dtype=np.float64)
    cen = base.blocks[0]["centres"]
    x, y = cen[..., 0], cen[..., 1]
    I = c.interior(P, 0)
    if dim == 1:
        (rl, ul, pl), (rr, ur, pr) = states
        left = x < 0.5
        I[0] = np.where(left, rl, rr); I[1] = np.where(left, ul, ur); I[4] = np.where(left, pl, pr)
    else:
        sel = [(x > 0.5) & (y > 0.5), (x <= 0.5) & (y > 0.5), (x <= 0.5) & (y <= 0.5), (x > 0.5) & (y <= 0.5)]
        for m, (r, u, v, p) in zip(sel, states):
            I[0][m] = r; I[1][m] = u; I[2][m] = v; I[4][m] = p
    c.P0 = P
    return Request(rid, c, t_end, arrival, geo_key=key)


def request_stream(n_cases=4096, rate=1.0, seed=20261203, n1=(256, 8192), n2=(128, 1024), t1=0.15, t2=0.25):
    """The seeded serving stream: Poisson arrivals at `rate` per second; each case is 1-D or 2-D with probability
    1/2. 1-D: N log-uniform in n1, left / right rho in U[0.1, 2], u in U[-1, 1], p in U[0.1, 10], to t1. 2-D
    four-quadrant: N^2 cells, N log-uniform in n2, four states drawn the same way (v like u), to t2. Returns
    (arrival, dim, n, states, t_end) tuples; build each with riemann_request when it is needed."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for q in range(n_cases):
        t += rng.exponential(1.0 / rate)
        dim = 1 if rng.random() < 0.5 else 2
        lo, hi = n1 if dim == 1 else n2
        n = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        if dim == 1:
            st = tuple((rng.uniform(0.1, 2.0), rng.uniform(-1.0, 1.0), rng.uniform(0.1, 10.0)) for _ in range(2))
        else:
            st = tuple((rng.uniform(0.1, 2.0), rng.uniform(-1.0, 1.0), rng.uniform(-1.0, 1.0), rng.uniform(0.1, 10.0))
                       for _ in range(4))
        out.append((t, dim, n, st, t1 if dim == 1 else t2))
    return out
