"""Blocks partitioned over several GPUs: the block -> rank partition, each rank's local mesh with external copies of
its remote donor blocks, the halo schedule, and a rank driver that steps one rank's share through the C ABI.

The reference decomposes a multi-block mesh over MPI ranks by blocks (src/lib/parallel/Mod_MPI.f90:147-258) and
exchanges, per stage, the ghost layers of the connections that cross ranks (build_ghost_schedule and the persistent
exchange of src/lib/parallel/Mod_GhostExchange.f90:217-383,685-957), with one MIN all-reduce of the time step per
step (mpi_allreduce_min_r8, Mod_MPI.f90:571-581). Here:

  partition_blocks  largest-first assignment of blocks to the least-loaded rank (interior cells), ties to the lower
                    rank; every rank computes the same partition.
  split_case        the rank's mesh: its own blocks (case group 0) and, as external blocks (group -1), copies of
                    the remote blocks its connection records take donor cells from, in one arena; records and
                    connections of its own blocks only, the donors renumbered.
  halo_plan         per ordered rank pair (owner q -> receiver r), the rows the receiver reads from q's blocks:
                    round 1, the donor cells of its connection ghosts (gc layers, the ghost copies of
                    Lib_Extrapolation.f90:1023-1134), sent before the receiver's ghost fill; round 2, the six donor
                    cells of every viscous connection record (bc_pg, Lib_Extrapolation.f90:1136-1191), sent after
                    the owner's own ghost fill (some of them are the owner's ghost cells). Row = the row in the
                    owner's arena; the receiver writes it at the same offset inside its external copy.
  EngineRank        one rank's blocks on its GPU: mb_step_prepare, MIN all-reduce of the clock minimum
                    (mb_copy_dtmin), mb_step_start, then per stage round 1 -> mb_stage_begin -> round 2 ->
                    mb_stage_end; the halo rows of the stage's input buffer (mb_stage_input: the engine rotates
                    three buffers through the stages) move through mb_pack_rows / mb_unpack_rows and an exchange
                    object.
  DistExchange      the exchange between processes over torch.distributed (NCCL on GPUs: grouped send / recv
                    of each pair's packed rows; gloo on the CPU).
  LocalExchange     the exchange between rank drivers of one process (device copies; ranks emulated on one GPU).
  PeerExchange      the same without buffers: one kernel per pair stores the owner's rows straight into the
                    receiver's arena (mb_push_rows: same GPU, or a peer GPU over NVLink).
  DistPeerExchange  the peer stores between processes: stage buffers mapped by CUDA IPC, a barrier per round.

Scope: 3-D blocks (n3 > 1) with 1:1 / periodic connections; donor blocks one cell deep (2-D meshes, whose k
ghosts are mirrored) are refused. The oracle counterpart (tests/test_multi_rank.py) runs the same schedule on the
CPU restatement and is compared bit for bit with one rank.
"""
import numpy as np

from . import abi

GC = abi.GC
NP = abi.NPRIM


def partition_blocks(case, nranks):
    """owner[b] for every block b of the case: the blocks in decreasing interior-cell order, each to the rank with
    the fewest cells so far (the lower rank on a tie)."""
    n = [int(np.prod(b["n"])) for b in case.blocks]
    order = sorted(range(len(n)), key=lambda b: (-n[b], b))
    load = [0] * nranks
    owner = [0] * len(n)
    for b in order:
        r = min(range(nranks), key=lambda q: (load[q], q))
        owner[b] = r
        load[r] += n[b]
    return owner


def _padded(n):
    return (n[0] + 2 * GC) * (n[1] + 2 * GC) * (n[2] + 2 * GC)


def _row(blk, i, j, k):
    n = blk["n"]
    pi, pj = n[0] + 2 * GC, n[1] + 2 * GC
    return blk["boff"] + (i + GC - 1) + (j + GC - 1) * pi + (k + GC - 1) * pi * pj


def _guide(F, ax):
    d = (F + 1) // 2 - 1
    return (1 if F % 2 else -1) if ax == d else 0


def _donor_rows(case, cn, visc_rows):
    """The rows of the donor block (global arena) that connection cn is read at: its gc donor layers (ghost copies)
    and, with visc_rows, the six bc_pg cells (face cell, the next cell inwards, the four transverse neighbours; the
    same construction as the engine's table, mb_api.cu build_tables)."""
    b = case.blocks[int(cn["bs"])]
    I, J, K, fs = int(cn["is"]), int(cn["js"]), int(cn["ks"]), int(cn["fs"])
    if not visc_rows:
        return [_row(b, I + _guide(fs, 0) * (g - 1), J + _guide(fs, 1) * (g - 1), K + _guide(fs, 2) * (g - 1))
                for g in range(1, GC + 1)]
    d11, d12, d21, d22 = (int(cn[x]) for x in ("d11", "d12", "d21", "d22"))
    if fs <= 2:
        t = [(I, J - d11, K - d12), (I, J + d11, K + d12), (I, J - d21, K - d22), (I, J + d21, K + d22)]
    elif fs <= 4:
        t = [(I - d11, J, K - d12), (I + d11, J, K + d12), (I - d21, J, K - d22), (I + d21, J, K + d22)]
    else:
        t = [(I - d11, J - d12, K), (I + d11, J + d12, K), (I - d21, J - d22, K), (I + d21, J + d22, K)]
    rows = [_row(b, I, J, K), _row(b, I + _guide(fs, 0), J + _guide(fs, 1), K + _guide(fs, 2))]
    rows += [_row(b, *c) for c in t]
    return rows


class RankCase:
    """One rank's share of a partitioned case: `case` (a Case of its own blocks then its external copies), `own` and
    `ext` (global block ids in local order), `boff_of` (global block id -> its row offset in this rank's arena)."""

    def __init__(self, case, own, ext, local):
        self.case = local
        self.own = own
        self.ext = ext
        self.boff_of = {g: local.blocks[q]["boff"] for q, g in enumerate(own + ext)}
        self.global_case = case

    def to_local_row(self, g, grow):
        """Row of this rank's arena of the cell at global row grow of global block g."""
        return grow - self.global_case.blocks[g]["boff"] + self.boff_of[g]


def split_case(case, owner, rank):
    """The RankCase of `rank` (see the module docstring)."""
    import copy
    nb = len(case.blocks)
    own = [b for b in range(nb) if owner[b] == rank]
    owned = set(own)
    recs = [q for q in range(len(case.rec)) if int(case.rec[q]["blk"]) in owned]
    ext = set()
    for q in recs:
        c = int(case.rec[q]["conn"])
        if c >= 0:
            bs = int(case.conn[c]["bs"])
            if bs not in owned:
                ext.add(bs)
    ext = sorted(ext)
    for g in ext:
        if case.blocks[g]["n"][2] == 1:
            raise NotImplementedError("a remote donor block one cell deep (2-D): its mirrored k ghosts are not served")
    lid = {g: q for q, g in enumerate(own + ext)}
    local = copy.copy(case)
    blocks = []
    boff = 0
    for g in own + ext:
        b = dict(case.blocks[g])
        b["boff"] = boff
        b["group"] = 0 if g in owned else -1
        b["global_id"] = g
        blocks.append(b)
        boff += _padded(b["n"])
    local.blocks = blocks
    local.ncell = boff
    rec = case.rec[recs].copy()
    conn_rows = []
    for q in range(len(rec)):
        rec[q]["blk"] = lid[int(rec[q]["blk"])]
        c = int(rec[q]["conn"])
        if c >= 0:
            cn = case.conn[c].copy()
            cn["rec"] = q
            cn["bs"] = lid[int(cn["bs"])]
            rec[q]["conn"] = len(conn_rows)
            conn_rows.append(cn)
    local.rec = rec
    local.conn = np.array(conn_rows, dtype=case.conn.dtype) if conn_rows else np.zeros(0, dtype=case.conn.dtype)
    P = np.zeros((NP, boff), dtype=np.float64)
    for q, g in enumerate(own + ext):
        n = _padded(case.blocks[g]["n"])
        P[:, blocks[q]["boff"]:blocks[q]["boff"] + n] = case.P0[:, case.blocks[g]["boff"]:case.blocks[g]["boff"] + n]
    local.P0 = P
    local.name = "%s_rank%d" % (case.name, rank)
    return RankCase(case, own, ext, local)


def halo_plan(case, owner, ranks, visc):
    """{(q, r): (round-1 rows in q's arena, round-1 rows in r's arena, round-2 rows in q's arena, round-2 rows in r's
    arena)} for every ordered pair of ranks with data to move; `ranks` are the RankCase objects of all ranks."""
    plan = {}
    for r, rc in enumerate(ranks):
        need = {}
        for q in range(len(case.rec)):
            if owner[int(case.rec[q]["blk"])] != r:
                continue
            c = int(case.rec[q]["conn"])
            if c < 0:
                continue
            cn = case.conn[c]
            g = int(cn["bs"])
            src = owner[g]
            if src == r:
                continue
            d = need.setdefault(src, (set(), set()))
            d[0].update((g, x) for x in _donor_rows(case, cn, False))
            if visc:
                d[1].update((g, x) for x in _donor_rows(case, cn, True))
        for src, (r1, r2) in need.items():
            out = []
            for s in (sorted(r1), sorted(r2)):
                out.append(np.array([ranks[src].to_local_row(g, x) for g, x in s], dtype=np.int64))
                out.append(np.array([rc.to_local_row(g, x) for g, x in s], dtype=np.int64))
            plan[(src, r)] = tuple(out)
    return plan


class LocalExchange:
    """Moves halo rows between rank drivers of one process (device or host arrays through their pack / unpack)."""

    def __init__(self, drivers, plan):
        self.drivers = drivers
        self.plan = plan

    def __call__(self, rnd):
        for (q, r), rows in self.plan.items():
            src, dst = rows[2 * rnd], rows[2 * rnd + 1]
            if len(src):
                buf = self.drivers[q].pack(src, rnd, ("to", r))
                self.drivers[r].unpack(dst, buf)

    def min_all(self, values):
        return min(values)


class PeerExchange:
    """Moves halo rows between rank drivers of one process by peer stores: per round and ordered pair, one
    mb_push_rows on the owner's stream from its stage input straight into the receiver's (on the same GPU, or on a
    peer GPU with peer access: the stores cross NVLink), no staging buffer and no send / receive; the receiver's
    stream then waits for the owner's (a CUDA event). The reference's persistent exchange
    (Mod_GhostExchange.f90:685-957) with the buffers and the messages taken out."""

    def __init__(self, drivers, plan):
        self.drivers = drivers
        self.plan = plan
        for (q, r) in plan:
            dq, dr = drivers[q].dev, drivers[r].dev
            if dq != dr:                       # the owner's kernels store into the receiver's GPU
                rc = drivers[q].eng.lib.mb_enable_peer(dq.index, dr.index)
                if rc != abi.MB_OK:
                    raise abi.MoseError(rc, "mb_enable_peer %d -> %d" % (dq.index, dr.index))

    def __call__(self, rnd):
        import torch
        waits = {}
        for (q, r), rows in self.plan.items():
            src, dst = rows[2 * rnd], rows[2 * rnd + 1]
            if not len(src):
                continue
            a, b = self.drivers[q], self.drivers[r]
            rc = a.eng.lib.mb_push_rows(a.cur_in, a.rc.case.ncell, a._dev_rows(src).data_ptr(), b.cur_in,
                                        b.rc.case.ncell, a._dev_rows(dst).data_ptr(), len(src), a._s())
            if rc != abi.MB_OK:
                raise abi.MoseError(rc, "mb_push_rows")
            waits.setdefault(r, set()).add(q)
        for r, owners in waits.items():
            b = self.drivers[r]
            for q in owners:
                a = self.drivers[q]
                if a.ts.cuda_stream == b.ts.cuda_stream:
                    continue
                ev = torch.cuda.Event()
                ev.record(a.ts)
                b.ts.wait_event(ev)

    def min_all(self, values):
        return min(values)


class DistPeerExchange:
    """The peer-store exchange between processes (one per rank; on one node, one GPU each or several on one GPU): at
    set-up every rank exports its stage buffers by CUDA IPC (mb_ipc_export) and maps those of the ranks it sends to
    (mb_ipc_open), after checking on the host that every row it will write lies inside the receiver's arena and the
    arena inside the mapped allocation. Per round each rank pushes its rows straight into the receivers' current
    stage input (mb_push_rows), then all ranks meet: its stream drained, a barrier of the process group. No send /
    receive, no staging buffer; no kernel waits on another rank."""

    def __init__(self, driver, plan, rank, world, pg):
        import ctypes as C
        self.driver, self.plan, self.rank, self.world, self.pg = driver, plan, rank, world, pg
        L = driver.eng.lib
        self.bufs = driver.stage_buffers()
        mine = []
        for ptr in self.bufs:
            h = (C.c_char * 64)()
            off, size = C.c_int64(), C.c_int64()
            rc = L.mb_ipc_export(ptr, h, C.byref(off), C.byref(size))
            if rc != abi.MB_OK:
                raise abi.MoseError(rc, "mb_ipc_export")
            mine.append((bytes(h), off.value, size.value))
        everyone = [None] * world
        pg.all_gather_object(everyone, (mine, int(driver.rc.case.ncell)))
        self.peer, self._bases, opened = {}, [], {}
        for (q, r), rows in plan.items():
            if q != rank or r in self.peer:
                continue
            theirs, nc = everyone[r]
            if len(theirs) != len(self.bufs):
                raise RuntimeError("rank %d has %d stage buffers, rank %d %d" % (r, len(theirs), rank, len(self.bufs)))
            need = NP * nc * 8
            for rr in (rows[1], rows[3]):
                if len(rr) and (rr.min() < 0 or rr.max() >= nc):
                    raise RuntimeError("halo row outside the arena of rank %d" % r)
            ptrs = []
            for h, off, size in theirs:
                if off < 0 or off + need > size:
                    raise RuntimeError("the arena of rank %d does not fit its allocation" % r)
                if h not in opened:            # buffers in one allocation share its handle: map it once
                    base = C.c_void_p()
                    rc = L.mb_ipc_open(C.c_char_p(h), driver.dev.index, C.byref(base))
                    if rc != abi.MB_OK:
                        raise abi.MoseError(rc, "mb_ipc_open")
                    opened[h] = base.value
                    self._bases.append(base.value)
                ptrs.append(opened[h] + off)
            self.peer[r] = (ptrs, nc)

    def __call__(self, rnd):
        d = self.driver
        k = self.bufs.index(d.cur_in)
        for (q, r), rows in sorted(self.plan.items()):
            src, dst = rows[2 * rnd], rows[2 * rnd + 1]
            if q != self.rank or not len(src):
                continue
            ptrs, nc = self.peer[r]
            rc = d.eng.lib.mb_push_rows(d.cur_in, d.rc.case.ncell, d._dev_rows(src).data_ptr(), ptrs[k], nc,
                                        d._dev_rows(dst).data_ptr(), len(src), d._s())
            if rc != abi.MB_OK:
                raise abi.MoseError(rc, "mb_push_rows")
        d.ts.synchronize()
        self.pg.barrier()

    def min_all(self, value):
        import torch
        t = torch.tensor([value], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MIN)
        return float(t.item())

    def close(self):
        self.pg.barrier()                      # every rank's last push has landed before the mappings go
        for b in self._bases:
            self.driver.eng.lib.mb_ipc_close(b)
        self._bases = []


class DistExchange:
    """Moves halo rows between processes over torch.distributed: per round, every rank packs what each peer needs and
    the pairs exchange with one grouped send / receive (batch_isend_irecv), then every rank unpacks."""

    def __init__(self, driver, plan, rank, world, device):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.driver, self.plan, self.rank, self.world, self.device = driver, plan, rank, world, device

    def __call__(self, rnd):
        torch, dist = self.torch, self.dist
        ops, recvs = [], []
        for (q, r), rows in sorted(self.plan.items()):
            src, dst = rows[2 * rnd], rows[2 * rnd + 1]
            if not len(src):
                continue
            if q == self.rank:
                ops.append(dist.P2POp(dist.isend, self.driver.pack(src, rnd, ("to", r)), r))
            elif r == self.rank:
                buf = torch.empty(NP * len(dst), dtype=torch.float64, device=self.device)
                ops.append(dist.P2POp(dist.irecv, buf, q))
                recvs.append((dst, buf))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        for dst, buf in recvs:
            self.driver.unpack(dst, buf)

    def min_all(self, value):
        t = self.torch.tensor([value], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN)
        return float(t.item())


class EngineRank:
    """One rank's blocks on its GPU, stepped through the split stage calls of the C ABI (mosegpu.engine.Engine for
    the context and the state buffers)."""

    def __init__(self, rank_case, precision=abi.PREC_FP64, device=0, stream=None):
        import torch
        from .engine import Engine
        self.torch = torch
        self.rc = rank_case
        self.eng = Engine(rank_case.case, precision=precision, device=device, stream=stream)
        self.dev = self.eng.dev
        self.ts = stream if stream is not None else torch.cuda.current_stream(self.dev)   # the rank's stream
        self._rows = {}
        self._bufs = {}
        with torch.cuda.stream(self.ts):
            self.dtbuf = torch.zeros(1, dtype=torch.int64, device=self.dev)
        self.cur_in = self.eng.P.data_ptr()     # the device buffer the current stage reads (set_stage)

    def set_stage(self, irk):
        """The stage about to run: its input buffer (P, PO or the engine's own) is where the halo rows go."""
        import ctypes as C
        ptr = C.c_void_p()
        e = self.eng
        rc = e.lib.mb_stage_input(e.ctx, e.P.data_ptr(), e.PO.data_ptr(), irk, C.byref(ptr))
        if rc != abi.MB_OK:
            raise abi.MoseError(rc, "mb_stage_input")
        self.cur_in = ptr.value

    def _s(self):
        return self.eng._s()

    def stage_buffers(self):
        """The device buffers the stages read, in a fixed order: P, PO, then the engine's own (mb_stage_input over
        the stages); a rank's stage irk reads the buffer of the same place in every rank's list."""
        import ctypes as C
        e = self.eng
        out = [e.P.data_ptr(), e.PO.data_ptr()]
        for irk in range(1, e.case.scheme["n_rk"] + 1):
            ptr = C.c_void_p()
            rc = e.lib.mb_stage_input(e.ctx, e.P.data_ptr(), e.PO.data_ptr(), irk, C.byref(ptr))
            if rc != abi.MB_OK:
                raise abi.MoseError(rc, "mb_stage_input")
            if ptr.value not in out:
                out.append(ptr.value)
        return out

    def _dev_rows(self, rows):
        key = (rows.ctypes.data, len(rows))
        if key not in self._rows:
            with self.torch.cuda.stream(self.ts):
                self._rows[key] = (rows, self.torch.from_numpy(rows).to(self.dev))
        return self._rows[key][1]

    def pack(self, rows, rnd, tag):
        d = self._dev_rows(rows)
        key = (tag, rnd)
        if key not in self._bufs or self._bufs[key].numel() != NP * len(rows):
            with self.torch.cuda.stream(self.ts):
                self._bufs[key] = self.torch.empty(NP * len(rows), dtype=self.torch.float64, device=self.dev)
        buf = self._bufs[key]
        rc = self.eng.lib.mb_pack_rows(self.cur_in, self.rc.case.ncell, d.data_ptr(), len(rows), buf.data_ptr(),
                                       self._s())
        if rc != abi.MB_OK:
            raise abi.MoseError(rc, "mb_pack_rows")
        return buf

    def unpack(self, rows, buf):
        d = self._dev_rows(rows)
        if buf.device != self.dev:
            buf = buf.to(self.dev)
        rc = self.eng.lib.mb_unpack_rows(self.cur_in, self.rc.case.ncell, d.data_ptr(), len(rows), buf.data_ptr(),
                                         self._s())
        if rc != abi.MB_OK:
            raise abi.MoseError(rc, "mb_unpack_rows")

    def local_dtmin(self):
        """The clock minimum of this rank's blocks (mb_step_prepare, mb_copy_dtmin out) as a float."""
        e = self.eng
        for f, a in (("mb_step_prepare", (e.ctx, e.P.data_ptr(), self._s())),
                     ("mb_copy_dtmin", (e.ctx, 0, self.dtbuf.data_ptr(), 0, self._s()))):
            rc = getattr(e.lib, f)(*a)
            if rc != abi.MB_OK:
                raise abi.MoseError(rc, f)
        self.ts.synchronize()
        return float(self.dtbuf.view(self.torch.float64).item())

    def start(self, dtmin):
        e = self.eng
        with self.torch.cuda.stream(self.ts):
            self.dtbuf.view(self.torch.float64).fill_(dtmin)
        for f, a in (("mb_copy_dtmin", (e.ctx, 0, self.dtbuf.data_ptr(), 1, self._s())),
                     ("mb_step_start", (e.ctx, self._s()))):
            rc = getattr(e.lib, f)(*a)
            if rc != abi.MB_OK:
                raise abi.MoseError(rc, f)

    def stage(self, irk, part):
        e = self.eng
        f = "mb_stage_begin" if part == 0 else "mb_stage_end"
        rc = getattr(e.lib, f)(e.ctx, e.P.data_ptr(), e.PO.data_ptr(), irk, self._s())
        if rc != abi.MB_OK:
            raise abi.MoseError(rc, f)

    def state(self):
        self.ts.synchronize()
        return self.eng.state()


def step_ranks(drivers, exchange, visc, n_rk, nsteps=1):
    """nsteps time steps of every rank driver of one process (LocalExchange), in the order each process of a
    distributed run follows (step_rank)."""
    for _ in range(nsteps):
        dt = exchange.min_all([d.local_dtmin() for d in drivers])
        for d in drivers:
            d.start(dt)
        for irk in range(1, n_rk + 1):
            for d in drivers:
                d.set_stage(irk)
            exchange(0)
            for d in drivers:
                d.stage(irk, 0)
            if visc:
                exchange(1)
            for d in drivers:
                d.stage(irk, 1)


def step_rank(driver, exchange, visc, n_rk, nsteps=1):
    """nsteps time steps of this process's rank (DistExchange): the same calls as step_ranks, one rank."""
    for _ in range(nsteps):
        driver.start(exchange.min_all(driver.local_dtmin()))
        for irk in range(1, n_rk + 1):
            driver.set_stage(irk)
            exchange(0)
            driver.stage(irk, 0)
            if visc:
                exchange(1)
            driver.stage(irk, 1)


def gather_interiors(case, ranks, states):
    """The interior cells of every block of the global case from the ranks' states (5, ncell_rank), as a global P
    whose interior rows are filled."""
    P = np.zeros_like(case.P0)
    for rc, S in zip(ranks, states):
        for q, g in enumerate(rc.own):
            lb = rc.case.blocks[q]
            n = case.blocks[g]["n"]
            gv = case.interior(P, g)
            lv = rc.case.interior(S, q)
            assert lv.shape == gv.shape and lb["global_id"] == g and tuple(n) == tuple(lb["n"])
            gv[...] = lv
    return P
