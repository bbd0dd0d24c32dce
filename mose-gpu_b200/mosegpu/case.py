"""Case construction on the host: meshes, grid metrics, boundary records, thermo tables and
initial states of the configurations the engine serves, in the reference's data layouts.

The reference keeps all of this on the host (case reading, Setup_Metrics, Setup_BC); the engine
receives the finished arrays. Grid metrics restate src/lib/numerics/space/Lib_Metrics.f90
(Compute_Metric_Tensor :382-511, Compute_Norm_Area :199-379) on a node array that carries two
ghost-node layers, so ghost cells get the metrics of the continued mesh (the donor's cells across
a connection, a linear continuation at a physical boundary).

Layouts (Fortran column-major, flattened with order='F'), per block of n = (n1, n2, n3) cells:
  fm1 (4, n1+1, n2, n3), fm2 (4, n1, n2+1, n3), fm3 (4, n1, n2, n3+1): nx, ny, nz, area
  dl (3, n1+4, n2+4, n3+4), m (3, 3, n1+4, n2+4, n3+4), vol (n1+4, n2+4, n3+4)
The state arena P has shape (5, ncell) in C order, i.e. P_flat(ncell, 5) column-major.
"""
import math

import numpy as np

from . import abi

GC = abi.GC
NPRIM = abi.NPRIM
RUNIV = 8314.46261815324       # lib/FLINT/src/lib/Lib_ThermoTransport.f90:13
W_AIR = 28.970418               # test/1D/Sod79/INPUT/phase.txt
TMIN, TMAX = 0, 10000           # 1 K table, row 0 added by Load_ThermoTransport.f90:82-97


# ----------------------------------------------------------------------------- thermo tables
def ideal_gas_tables(gamma=1.4, wm=W_AIR, mu=1.8e-5, prandtl=0.71):
    """Calorically perfect single-species tables on the 1 K grid: cp = gamma/(gamma-1) R,
    h(T) = cp T (row 0: cp(0) = cp(1), h(0) = 0, as Load_ThermoTransport.f90:92-97),
    constant viscosity, conductivity mu cp / Pr (transport.dat of the reference's test cases)."""
    R = RUNIV / wm
    cp = gamma / (gamma - 1.0) * R
    T = np.arange(TMIN, TMAX + 1, dtype=np.float64)
    cpt = np.full(T.shape, cp)
    h = cp * T
    h[0] = cp * 0.0
    mut = np.full(T.shape, float(mu))
    kt = mut * cpt / prandtl
    return dict(tmin=TMIN, tmax=TMAX, wm=float(wm), cp=cpt, h=h, mu=mut, k=kt, R=R, cp_value=cp,
                gamma=gamma)


# ----------------------------------------------------------------------------- metrics
def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def _tvol(vx, vy, vz, i1, i2, i3, i4):
    return np.abs(((vx[i2] - vx[i1]) * ((vy[i3] - vy[i1]) * (vz[i4] - vz[i1]) - (vy[i4] - vy[i1]) * (vz[i3] - vz[i1]))
                   + (vy[i2] - vy[i1]) * ((vx[i4] - vx[i1]) * (vz[i3] - vz[i1]) - (vx[i3] - vx[i1]) * (vz[i4] - vz[i1]))
                   + (vz[i2] - vz[i1]) * ((vx[i3] - vx[i1]) * (vy[i4] - vy[i1]) - (vx[i4] - vx[i1]) * (vy[i3] - vy[i1])))
                  / 6.0)


def cell_metrics(X):
    """Compute_Metric_Tensor over every cell of a node array X (nx, ny, nz, 3) -> m (cells, 3, 3),
    dl (cells, 3), vol (cells), for the (nx-1)(ny-1)(nz-1) cells."""
    N1 = X[:-1, :-1, :-1]; N2 = X[:-1, :-1, 1:]; N3 = X[:-1, 1:, :-1]; N4 = X[:-1, 1:, 1:]
    N5 = X[1:, :-1, :-1]; N6 = X[1:, :-1, 1:]; N7 = X[1:, 1:, :-1]; N8 = X[1:, 1:, 1:]
    A1 = N5 - N1 + N6 - N2 + N7 - N3 + N8 - N4
    A2 = N3 - N1 + N4 - N2 + N7 - N5 + N8 - N6
    A3 = N2 - N1 + N4 - N3 + N6 - N5 + N8 - N7
    A = 0.25 * np.stack([A1, A2, A3], axis=-2)  # A[..., h, c]
    a = lambda r, c: A[..., r - 1, c - 1]
    det = (a(1, 1) * a(2, 2) * a(3, 3) - a(1, 1) * a(2, 3) * a(3, 2) - a(1, 2) * a(2, 1) * a(3, 3)
           + a(1, 2) * a(2, 3) * a(3, 1) + a(1, 3) * a(2, 1) * a(3, 2) - a(1, 3) * a(2, 2) * a(3, 1))
    if np.any(det == 0.0):
        raise ValueError("degenerate cell in the mesh (metric determinant 0)")
    cof = np.empty(A.shape)
    cof[..., 0, 0] = (a(2, 2) * a(3, 3) - a(2, 3) * a(3, 2))
    cof[..., 0, 1] = -(a(2, 1) * a(3, 3) - a(2, 3) * a(3, 1))
    cof[..., 0, 2] = (a(2, 1) * a(3, 2) - a(2, 2) * a(3, 1))
    cof[..., 1, 0] = -(a(1, 2) * a(3, 3) - a(1, 3) * a(3, 2))
    cof[..., 1, 1] = (a(1, 1) * a(3, 3) - a(1, 3) * a(3, 1))
    cof[..., 1, 2] = -(a(1, 1) * a(3, 2) - a(1, 2) * a(3, 1))
    cof[..., 2, 0] = (a(1, 2) * a(2, 3) - a(1, 3) * a(2, 2))
    cof[..., 2, 1] = -(a(1, 1) * a(2, 3) - a(1, 3) * a(2, 1))
    cof[..., 2, 2] = (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1))
    M = cof / det[..., None, None]
    dl = np.sqrt(A[..., 0] ** 2 + A[..., 1] ** 2 + A[..., 2] ** 2)
    nodes = [N1, N5, N3, N7, N2, N6, N4, N8]
    vx = [n[..., 0] for n in nodes]; vy = [n[..., 1] for n in nodes]; vz = [n[..., 2] for n in nodes]
    vol = (_tvol(vx, vy, vz, 0, 1, 2, 4) + _tvol(vx, vy, vz, 1, 3, 2, 7) + _tvol(vx, vy, vz, 4, 7, 5, 1)
           + _tvol(vx, vy, vz, 4, 6, 7, 2) + _tvol(vx, vy, vz, 4, 7, 1, 2))
    if np.any(vol <= 0.0):
        raise ValueError("negative cell volume")
    return M, dl, vol


def face_metrics(X):
    """Compute_Norm_Area on the interior node array X (n1+1, n2+1, n3+1, 3): returns
    fm1 (n1+1, n2, n3, 4), fm2 (n1, n2+1, n3, 4), fm3 (n1, n2, n3+1, 4)."""
    def sgn(d1, d2, c1, c2):
        d3 = _cross(d1, d2)
        return 1.0 if float(np.dot(c1 - c2, d3)) >= 0.0 else -1.0
    n = lambda i, j, k: X[i, j, k]
    si = sgn(n(1, 1, 1) - n(1, 0, 0), n(1, 0, 1) - n(1, 1, 0),
             0.25 * (n(1, 1, 1) + n(1, 0, 1) + n(1, 0, 0) + n(1, 1, 0)),
             0.25 * (n(0, 1, 1) + n(0, 0, 1) + n(0, 0, 0) + n(0, 1, 0)))
    sj = sgn(n(0, 1, 1) - n(1, 1, 0), n(1, 1, 1) - n(0, 1, 0),
             0.25 * (n(1, 1, 1) + n(0, 1, 1) + n(0, 1, 0) + n(1, 1, 0)),
             0.25 * (n(1, 0, 1) + n(0, 0, 1) + n(0, 0, 0) + n(1, 0, 0)))
    sk = sgn(n(0, 1, 1) - n(1, 0, 1), n(0, 0, 1) - n(1, 1, 1),
             0.25 * (n(1, 1, 1) + n(0, 1, 1) + n(0, 0, 1) + n(1, 0, 1)),
             0.25 * (n(1, 1, 0) + n(0, 1, 0) + n(0, 0, 0) + n(1, 0, 0)))

    def pack(d1, d2, s):
        d3 = _cross(d1, d2) * 0.5
        A = np.sqrt(d3[..., 0] ** 2 + d3[..., 1] ** 2 + d3[..., 2] ** 2)
        with np.errstate(invalid="ignore", divide="ignore"):
            nn = np.where(A[..., None] == 0.0, 0.0, d3 / A[..., None] * s)
        return np.concatenate([nn, A[..., None]], axis=-1)
    # i-faces: node(i,j,k) - node(i,j-1,k-1), node(i,j-1,k) - node(i,j,k-1)
    fm1 = pack(X[:, 1:, 1:] - X[:, :-1, :-1], X[:, :-1, 1:] - X[:, 1:, :-1], si)
    # j-faces: node(i-1,j,k) - node(i,j,k-1), node(i,j,k) - node(i-1,j,k-1)
    fm2 = pack(X[:-1, :, 1:] - X[1:, :, :-1], X[1:, :, 1:] - X[:-1, :, :-1], sj)
    # k-faces: node(i-1,j,k) - node(i,j-1,k), node(i-1,j-1,k) - node(i,j,k)
    fm3 = pack(X[:-1, 1:, :] - X[1:, :-1, :], X[:-1, :-1, :] - X[1:, 1:, :], sk)
    return fm1, fm2, fm3


# ----------------------------------------------------------------------------- the case
class Case:
    """A mesh of structured blocks, its boundary records and connections, thermo tables, scheme and
    initial state, in the layouts of include/mose_b200.h."""

    def __init__(self, name):
        self.name = name
        self.blocks = []     # dicts: n, boff, fm1, fm2, fm3, dl, m, vol (flat F-order float64)
        self.rec = np.zeros(0, dtype=abi.BC_DTYPE)
        self.conn = np.zeros(0, dtype=abi.CONN_DTYPE)
        self.ncell = 0
        self.thermo = None
        self.scheme = {}
        self.P0 = None
        self.steps = 1
        self.meta = {}
        self.node_fn = None  # (iu, iv, iw) global node indices -> (..., 3) coordinates

    def nodes(self, b):
        """Node coordinates (n1+1, n2+1, n3+1, 3) of the interior of block b, from the mapping the case was built
        with (the mesh file's nodes of the reference)."""
        blk = self.blocks[b]
        n, lo = blk["n"], blk["lo"]
        ax = [np.arange(lo[d], lo[d] + n[d] + 1, dtype=np.float64) for d in range(3)]
        IU, IV, IW = np.meshgrid(ax[0], ax[1], ax[2], indexing="ij")
        return self.node_fn(IU, IV, IW)

    # --- indexing helpers (MOSE_Field_m.f90:78-109)
    def padded(self, b):
        n1, n2, n3 = self.blocks[b]["n"]
        return n1 + 2 * GC, n2 + 2 * GC, n3 + 2 * GC

    def block_view(self, P, b):
        """P (5, ncell) -> view (5, pi, pj, pk) of block b, padded index ii = i + gc - 1."""
        pi, pj, pk = self.padded(b)
        o = self.blocks[b]["boff"]
        return P[:, o:o + pi * pj * pk].reshape(NPRIM, pk, pj, pi).transpose(0, 3, 2, 1)

    def interior(self, P, b):
        n1, n2, n3 = self.blocks[b]["n"]
        return self.block_view(P, b)[:, GC:GC + n1, GC:GC + n2, GC:GC + n3]

    def interior_mask(self):
        m = np.zeros(self.ncell, dtype=bool)
        for b in range(len(self.blocks)):
            pi, pj, pk = self.padded(b)
            v = m[self.blocks[b]["boff"]:self.blocks[b]["boff"] + pi * pj * pk].reshape(pk, pj, pi).transpose(2, 1, 0)
            n1, n2, n3 = self.blocks[b]["n"]
            v[GC:GC + n1, GC:GC + n2, GC:GC + n3] = True
        return m

    @property
    def n_interior(self):
        return int(sum(int(np.prod(b["n"])) for b in self.blocks))

    def scheme_struct(self):
        s = abi.MBScheme()
        d = self.scheme
        s.limiter = d["limiter"]; s.riemann = d["riemann"]; s.visc = d["visc"]; s.n_rk = d["n_rk"]
        s.precision = d.get("precision", abi.PREC_FP64); s.ndir = d["ndir"]
        s.time_clip = d.get("time_clip", 0); s.state_check = d.get("state_check", 1)
        s.dt_additive = d.get("dt_additive", 0)
        s.sensor = d.get("sensor", 0)
        s.intvar = d.get("intvar", 0)
        s.cfl = d["cfl"]; s.vnn = d.get("vnn", 0.3); s.prandtl = d.get("prandtl", 0.0)
        s.schmidt = d.get("schmidt", 0.7); s.mco = d.get("mco", 1.0)
        s.time_threshold = d.get("time_threshold", 0.0)
        s.res_stop = d.get("res_stop", 0.0)
        s.irs = d.get("irs", 0)                         # Jacobi sweeps of the residual smoothing (0: off)
        s.irs_beta = d.get("irs_beta", 0.5)
        s.local_dt = d.get("local_dt", 0)               # time-accurate = false: each cell its own step
        s.cfl_rise = d.get("cfl_rise", 0)               # cfl-rise-threshold
        s.prec_smooth = d.get("prec_smooth", 0)         # integration-variables = prec: the preconditioning keys
        s.prec_eps_min = d.get("prec_eps_min", 0.05)
        s.prec_uref = d.get("prec_uref", 0.0)
        s.prec_mach = d.get("prec_mach", 0.0)
        s.prec_ur_factor = d.get("prec_ur_factor", 1.0)
        s.prec_ur_min = d.get("prec_ur_min", 0.0)
        return s


def _axis_nodes(N, L, x0=0.0):
    """Uniform node coordinates of N cells on [x0, x0+L], with gc ghost nodes on each side."""
    nu = np.arange(-GC, N + GC + 1, dtype=np.float64)
    return x0 + nu * (L / N)


def uniform_geometry(n, h):
    """The metric arrays of a block of n cells on a uniform Cartesian grid of spacings h = (hx, hy, hz), in the
    layouts of cell_metrics / face_metrics (padded cells, interior faces): M = diag(1 / h), dl = h, vol = hx hy hz,
    unit face normals along the axes with the face areas. The values of cell_metrics / face_metrics on such a grid up
    to the rounding of the node coordinates, without evaluating them cell by cell."""
    hx, hy, hz = (float(x) for x in h)
    npad = (n[0] + 2 * GC) * (n[1] + 2 * GC) * (n[2] + 2 * GC)
    m = np.zeros((npad, 9))
    m[:, 0], m[:, 4], m[:, 8] = 1.0 / hx, 1.0 / hy, 1.0 / hz
    dl = np.empty((npad, 3))
    dl[:] = (hx, hy, hz)
    out = dict(m=m.ravel(), dl=dl.ravel(), vol=np.full(npad, hx * hy * hz))
    for q, (nf, nrm, area) in enumerate((((n[0] + 1) * n[1] * n[2], (1.0, 0.0, 0.0), hy * hz),
                                         (n[0] * (n[1] + 1) * n[2], (0.0, 1.0, 0.0), hx * hz),
                                         (n[0] * n[1] * (n[2] + 1), (0.0, 0.0, 1.0), hx * hy))):
        f = np.empty((nf, 4))
        f[:] = nrm + (area,)
        out["fm%d" % (q + 1)] = f.ravel()
    return out


def layout_case(name, cuts, node_fn, periodic, bc_faces, thermo, scheme, prim_fn, share_geometry=False,
                uniform=None, implicit_k=False):
    """A structured layout of blocks.

    cuts      : per axis, the cell-index cut points of the blocks, e.g. [[0, 128, 256], [0, 256], [0, 256]]
    node_fn   : (iu, iv, iw) extended global node indices (3 float arrays, ghosts included)
                -> node coordinates (..., 3)
    periodic  : per axis, True if the global domain is periodic along it
    bc_faces  : {global face 1..6: boundary type, or (type, q) with the record parameters q (mb_bc.q)} for the
                non-periodic global faces
    prim_fn   : cell-centre coordinates (..., 3) -> primitive state (5, ...) (rho, u, v, w, p)
    share_geometry : blocks of equal extents reuse the metric arrays of the first such block (exact for a
                node_fn that is a translation from block to block, e.g. a uniform Cartesian grid; the
                engine then holds one copy of the geometry on the device)
    uniform   : (hx, hy, hz) when node_fn is a uniform Cartesian grid of those spacings: the metric arrays from
                uniform_geometry instead of cell by cell (large serving cases)
    implicit_k: blocks one cell deep in k get no records on their extrapolated k faces (5, 6): the engine and the
                oracle take a one-plane block without k-face records as extrapolated there (2 n1 n2 records fewer)
    Blocks are numbered i fastest over the layout; faces between blocks are 1:1 connections with
    identity orientation; periodic axes wrap onto the first / last block.
    """
    case = Case(name)
    case.thermo = thermo
    case.scheme = dict(scheme)
    case.node_fn = node_fn
    nb = [len(c) - 1 for c in cuts]
    Ntot = [c[-1] for c in cuts]
    blocks = []
    boff = 0
    bid = {}
    for bz in range(nb[2]):
        for by in range(nb[1]):
            for bx in range(nb[0]):
                lo = (cuts[0][bx], cuts[1][by], cuts[2][bz])
                n = (cuts[0][bx + 1] - lo[0], cuts[1][by + 1] - lo[1], cuts[2][bz + 1] - lo[2])
                bid[(bx, by, bz)] = len(blocks)
                blocks.append(dict(n=n, lo=lo, pos=(bx, by, bz), boff=boff))
                boff += (n[0] + 2 * GC) * (n[1] + 2 * GC) * (n[2] + 2 * GC)
    case.ncell = boff
    # geometry
    shared = {}
    for b in blocks:
        n, lo = b["n"], b["lo"]
        if uniform is not None:
            b.update(uniform_geometry(n, uniform))
            ax = [np.arange(lo[d], lo[d] + n[d] + 1, dtype=np.float64) for d in range(3)]
            IU, IV, IW = np.meshgrid(ax[0], ax[1], ax[2], indexing="ij")
            Xi = node_fn(IU, IV, IW)
        elif share_geometry and tuple(n) in shared:
            b.update(shared[tuple(n)])
            ax = [np.arange(lo[d], lo[d] + n[d] + 1, dtype=np.float64) for d in range(3)]
            IU, IV, IW = np.meshgrid(ax[0], ax[1], ax[2], indexing="ij")
            Xi = node_fn(IU, IV, IW)
        else:
            ax = [np.arange(lo[d] - GC, lo[d] + n[d] + GC + 1, dtype=np.float64) for d in range(3)]
            IU, IV, IW = np.meshgrid(ax[0], ax[1], ax[2], indexing="ij")
            X = node_fn(IU, IV, IW)                           # (n1+5, n2+5, n3+5, 3)
            M, dl, vol = cell_metrics(X)                      # padded cells
            Xi = X[GC:GC + n[0] + 1, GC:GC + n[1] + 1, GC:GC + n[2] + 1]
            fm1, fm2, fm3 = face_metrics(Xi)
            b["fm1"] = np.ascontiguousarray(np.moveaxis(fm1, -1, 0)).ravel(order="F")
            b["fm2"] = np.ascontiguousarray(np.moveaxis(fm2, -1, 0)).ravel(order="F")
            b["fm3"] = np.ascontiguousarray(np.moveaxis(fm3, -1, 0)).ravel(order="F")
            b["dl"] = np.moveaxis(dl, -1, 0).ravel(order="F").copy()
            b["m"] = np.moveaxis(np.moveaxis(M, -1, 0), -1, 0).ravel(order="F").copy()  # (h, c, ...) -> m(h,c)
            b["vol"] = vol.ravel(order="F").copy()
            del X, M, dl, vol
            if share_geometry:
                shared[tuple(n)] = {f: b[f] for f in ("fm1", "fm2", "fm3", "dl", "m", "vol")}
        # cell centres of the interior cells (mean of the 8 nodes)
        C8 = 0.125 * (Xi[:-1, :-1, :-1] + Xi[1:, :-1, :-1] + Xi[:-1, 1:, :-1] + Xi[1:, 1:, :-1] +
                      Xi[:-1, :-1, 1:] + Xi[1:, :-1, 1:] + Xi[:-1, 1:, 1:] + Xi[1:, 1:, 1:])
        b["centres"] = C8
    case.blocks = blocks
    # boundary records, grouped per block, face-ordered within a block; cells i fastest
    recs = []
    conns = []
    nrec = 0
    for bi, b in enumerate(blocks):
        n = b["n"]
        pos = b["pos"]
        for face in range(1, 7):
            ax = (face - 1) // 2
            low = face % 2 == 1
            npos = list(pos)
            npos[ax] += -1 if low else 1
            neighbour = None
            if 0 <= npos[ax] < nb[ax]:
                neighbour = bid[tuple(npos)]
            elif periodic[ax]:
                npos[ax] %= nb[ax]
                neighbour = bid[tuple(npos)]
            rng = [np.arange(1, n[0] + 1), np.arange(1, n[1] + 1), np.arange(1, n[2] + 1)]
            rng[ax] = np.array([1 if low else n[ax]])
            I, J, K = [a.ravel(order="F") for a in np.meshgrid(*rng, indexing="ij")]
            m = I.size
            r = np.zeros(m, dtype=abi.BC_DTYPE)
            r["blk"] = bi; r["i"] = I; r["j"] = J; r["k"] = K; r["face"] = face; r["conn"] = -1
            if neighbour is not None:
                r["type"] = abi.BC_CONNECTION
                nd = blocks[neighbour]["n"]
                cn = np.zeros(m, dtype=abi.CONN_DTYPE)
                cn["rec"] = nrec + np.arange(m); cn["bs"] = neighbour
                src = [I.copy(), J.copy(), K.copy()]
                src[ax][:] = nd[ax] if low else 1
                cn["is"], cn["js"], cn["ks"] = src
                cn["fs"] = face + 1 if low else face - 1
                cn["d11"], cn["d12"], cn["d21"], cn["d22"] = 1, 0, 0, 1
                r["conn"] = sum(len(x) for x in conns) + np.arange(m)
                conns.append(cn)
            else:
                spec = bc_faces[face]
                if implicit_k and face >= 5 and n[2] == 1 and spec == abi.BC_EXTRAPOLATION:
                    continue
                if isinstance(spec, tuple):
                    r["type"] = spec[0]
                    qv = np.asarray(spec[1], dtype=np.float64)
                    r["q"][:, :qv.size] = qv
                else:
                    r["type"] = spec
                if r["type"][0] == abi.BC_INFLOW:
                    # the unit tangent of each face: the diagonal of its nodes (Mod_BC.f90:226-240)
                    lo = b["lo"]
                    Fi = [I.astype(np.float64), J.astype(np.float64), K.astype(np.float64)]
                    Fi[ax] = Fi[ax] - (face % 2)
                    A = [Fi[d] + lo[d] for d in range(3)]
                    Bn = [A[d] - (0 if d == ax else 1) for d in range(3)]
                    tv = node_fn(*A) - node_fn(*Bn)
                    r["q"][:, 8:11] = tv / np.linalg.norm(tv, axis=-1, keepdims=True)
            recs.append(r)
            nrec += m
    case.rec = np.concatenate(recs) if recs else np.zeros(0, dtype=abi.BC_DTYPE)
    case.conn = np.concatenate(conns) if conns else np.zeros(0, dtype=abi.CONN_DTYPE)
    # initial state (interior cells; ghosts are filled by the ghost fill)
    P = np.zeros((NPRIM, case.ncell), dtype=np.float64)
    for bi, b in enumerate(blocks):
        case.interior(P, bi)[...] = prim_fn(b["centres"])
    case.P0 = P
    return case


# ----------------------------------------------------------------------------- configurations
def taylor_green(n=256, mach=0.1, re=1600.0, prandtl=0.71, blocks=1, noise=0.0, seed=20261203,
                 riemann=abi.RS_LMROE, limiter=abi.LIM_VANALBADA, cfl=0.8, steps=100, T0=300.0, rho0=1.0,
                 share_geometry=None):
    """3-D compressible Navier-Stokes Taylor-Green vortex on the periodic box [0, 2 pi]^3, n^3 cells
    (split into blocks^3 equal blocks). Dimensional so that T stays on the table and inside the
    viscous thermo guard: T0 = 300 K, p0 = rho0 R T0, V0 = Mach sqrt(gamma R T0), L = 1,
    mu = rho0 V0 L / Re (constant), kl = mu cp / Pr. Roe = LMRoe with Mco = 1."""
    th = ideal_gas_tables(prandtl=prandtl)
    R, gam = th["R"], th["gamma"]
    p0 = rho0 * R * T0
    V0 = mach * math.sqrt(gam * R * T0)
    mu = rho0 * V0 * 1.0 / re
    th = ideal_gas_tables(mu=mu, prandtl=prandtl)
    L = 2.0 * math.pi
    rng = np.random.default_rng(seed)

    def nodes(iu, iv, iw):
        h = L / n
        return np.stack([iu * h, iv * h, iw * h], axis=-1)

    def prim(c):
        x, y, z = c[..., 0], c[..., 1], c[..., 2]
        u = V0 * np.sin(x) * np.cos(y) * np.cos(z)
        v = -V0 * np.cos(x) * np.sin(y) * np.cos(z)
        w = np.zeros_like(x)
        if noise > 0.0:
            u = u + noise * V0 * rng.uniform(-1.0, 1.0, x.shape)
            v = v + noise * V0 * rng.uniform(-1.0, 1.0, x.shape)
            w = w + noise * V0 * rng.uniform(-1.0, 1.0, x.shape)
        p = p0 + rho0 * V0 ** 2 / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
        rho = np.full(x.shape, rho0)
        return np.stack([rho, u, v, w, p])

    cuts = [list(np.linspace(0, n, blocks + 1).astype(int))] * 3
    # dt-rule = additive: with the min rule (the reference default) CFL 0.8 per direction is a
    # multi-dimensional CFL near 2.4 in 3-D and the SSP-RK3 step diverges within ten steps
    scheme = dict(limiter=limiter, riemann=riemann, visc=1, n_rk=3, ndir=3, cfl=cfl, vnn=0.3,
                  prandtl=prandtl, schmidt=0.7, mco=1.0, dt_additive=1)
    if share_geometry is None:
        share_geometry = blocks > 1 and n % blocks == 0
    case = layout_case("tgv%d" % n, cuts, nodes, (True, True, True), {}, th, scheme, prim,
                       share_geometry=share_geometry)
    case.steps = steps
    case.meta = dict(V0=V0, p0=p0, T0=T0, rho0=rho0, mu=mu, L=L)
    return case


def taylor_green_blocks(nb=4, nblk=128, steps=50, seed=20261203, **kw):
    """The large multi-block Taylor-Green case: nb^3 blocks of nblk^3 cells on the periodic [0, 2 pi]^3, Mach 0.3,
    Re 1600, seeded uniform velocity noise of amplitude 1e-3 V0, HLLC + MUSCL van Albada, central viscous fluxes,
    SSP-RK3. The blocks share one copy of the (uniform) geometry."""
    args = dict(n=nb * nblk, blocks=nb, mach=0.3, noise=1e-3, seed=seed, riemann=abi.RS_HLLC,
                limiter=abi.LIM_VANALBADA, steps=steps, share_geometry=True)
    args.update(kw)
    case = taylor_green(**args)
    case.name = "tgv_%dx%dx%d_%d" % (nb, nb, nb, nblk)
    return case


def multiblock_2d(cols=8, rows=6, lo=64, hi=512, seed=20261203, mach=2.0, T=300.0, p=1.0e5, re=1.0e5,
                  amp=0.05, steps=200, cfl=0.5, n_rk=4, riemann=abi.RS_AUSMP, limiter=abi.LIM_VANLEER,
                  prandtl=0.71, widths=None, heights=None, visc=1, bc=None, velocity=None):
    """2-D laminar Navier-Stokes batch: a cols x rows layout of blocks whose column widths and row heights are
    drawn from the seed uniformly in [lo, hi] cells (1:1 interfaces), one k layer, on the global (xi, eta) in
    [0, 1]^2 mapped by x = xi + amp sin(2 pi eta), y = eta + amp sin(2 pi xi). Uniform supersonic inflow
    (405: Mach, static T and p, flow along +x) at i = 1, extrapolation outflow (400) at i = max, adiabatic
    no-slip walls (301) at j = 1 and j = max, extrapolation on the k faces. Re on the domain length 1 with a
    constant viscosity, kl = mu cp / Pr. AUSM+, MUSCL van Leer, classical RK4 (no reference), min dt rule."""
    rng = np.random.default_rng(seed)
    if widths is None:
        widths = rng.integers(lo, hi + 1, size=cols)
    if heights is None:
        heights = rng.integers(lo, hi + 1, size=rows)
    cx = [0] + list(np.cumsum(widths).astype(int))
    cy = [0] + list(np.cumsum(heights).astype(int))
    NI, NJ = cx[-1], cy[-1]
    th = ideal_gas_tables(prandtl=prandtl)
    R, gam = th["R"], th["gamma"]
    rho = p / (R * T)
    a = math.sqrt(gam * R * T)
    V = mach * a
    mu = rho * V * 1.0 / re
    th = ideal_gas_tables(mu=mu, prandtl=prandtl)
    dz = 1.0 / max(NI, NJ)

    def nodes(iu, iv, iw):
        xi, eta = iu / NI, iv / NJ
        x = xi + amp * np.sin(2.0 * np.pi * eta)
        y = eta + amp * np.sin(2.0 * np.pi * xi)
        return np.stack([x, y, iw * dz], axis=-1)

    u0 = V if velocity is None else velocity

    def prim(c):
        shp = c.shape[:-1]
        return np.stack([np.full(shp, rho), np.full(shp, u0), np.zeros(shp), np.zeros(shp), np.full(shp, p)])

    inflow = (abi.BC_INFLOW, (mach, T, p, 0.0, 0.0, 1.0))   # mach, T0, p0, alpha, beta, rel_fac
    if bc is None:
        bc = {1: inflow, 2: abi.BC_EXTRAPOLATION, 3: abi.BC_WALL, 4: abi.BC_WALL, 5: abi.BC_EXTRAPOLATION,
              6: abi.BC_EXTRAPOLATION}
    else:
        bc = {f: (inflow if t == abi.BC_INFLOW else t) for f, t in bc.items()}
    scheme = dict(limiter=limiter, riemann=riemann, visc=visc, n_rk=n_rk, ndir=2, cfl=cfl, vnn=0.3,
                  prandtl=prandtl, schmidt=0.7, mco=1.0, dt_additive=0)
    case = layout_case("mb2d_%dx%d" % (cols, rows), [cx, cy, [0, 1]], nodes, (False, False, False), bc, th,
                       scheme, prim)
    case.steps = steps
    case.meta = dict(widths=[int(w) for w in widths], heights=[int(h) for h in heights], rho=rho, V=V, mu=mu)
    return case


def duct_3d(widths=(6, 5), heights=(5,), depths=(3, 4), mach=0.5, T=300.0, p=1.0e5, re=2.0e3, amp=0.05,
            cfl=0.5, n_rk=3, riemann=abi.RS_HLLC, limiter=abi.LIM_VANLEER, prandtl=0.71, visc=1, bc=None,
            velocity=None, steps=20):
    """3-D laminar duct: blocks of the given column widths (i), row heights (j) and slab depths (k) in cells, 1:1
    interfaces, on (xi, eta, zeta) in [0, 1] x [0, 1] x [0, 0.5] mapped by x = xi + amp sin(2 pi eta),
    y = eta + amp sin(2 pi xi), z = zeta + amp sin(2 pi xi) sin(2 pi eta) (curvilinear in all three directions).
    Uniform flow along +x at the given Mach number; by default the 405 static inlet at i = 1, the 406 outlet at
    i = max (exit pressure 0.95 p, relaxation 0.5), isothermal no-slip walls (302) at 320 K and 290 K on the j faces,
    symmetry (300) on the k faces. bc overrides {global face: type or (type, q)}."""
    cx = [0] + list(np.cumsum(widths).astype(int))
    cy = [0] + list(np.cumsum(heights).astype(int))
    cz = [0] + list(np.cumsum(depths).astype(int))
    NI, NJ, NK = cx[-1], cy[-1], cz[-1]
    th = ideal_gas_tables(prandtl=prandtl)
    R, gam = th["R"], th["gamma"]
    rho = p / (R * T)
    V = mach * math.sqrt(gam * R * T)
    mu = rho * V * 1.0 / re
    th = ideal_gas_tables(mu=mu, prandtl=prandtl)

    def nodes(iu, iv, iw):
        xi, eta, zeta = iu / NI, iv / NJ, 0.5 * iw / NK
        x = xi + amp * np.sin(2.0 * np.pi * eta)
        y = eta + amp * np.sin(2.0 * np.pi * xi)
        z = zeta + amp * np.sin(2.0 * np.pi * xi) * np.sin(2.0 * np.pi * eta)
        return np.stack([x, y, z], axis=-1)

    u0 = V if velocity is None else velocity

    def prim(c):
        shp = c.shape[:-1]
        return np.stack([np.full(shp, rho), np.full(shp, u0), np.zeros(shp), np.zeros(shp), np.full(shp, p)])

    inflow = (abi.BC_INFLOW, (mach, T, p, 0.0, 0.0, 1.0))
    faces = {1: inflow, 2: (abi.BC_OUTLET, (0.95 * p, 0.5)), 3: (abi.BC_WALL_T, (320.0,)),
             4: (abi.BC_WALL_T, (290.0,)), 5: abi.BC_SYMMETRY, 6: abi.BC_SYMMETRY}
    if bc is not None:
        faces.update({f: (inflow if t == abi.BC_INFLOW else t) for f, t in bc.items()})
    scheme = dict(limiter=limiter, riemann=riemann, visc=visc, n_rk=n_rk, ndir=3, cfl=cfl, vnn=0.3,
                  prandtl=prandtl, schmidt=0.7, mco=1.0, dt_additive=0)
    case = layout_case("duct3d_%dx%dx%d" % (len(widths), len(heights), len(depths)), [cx, cy, cz], nodes,
                       (False, False, False), faces, th, scheme, prim)
    case.steps = steps
    case.meta = dict(rho=rho, V=V, mu=mu)
    return case


def riemann_1d(n=1000, left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1), x0=0.5, t_end=0.2, cfl=0.5,
               riemann=abi.RS_HLLC, limiter=abi.LIM_MINMOD, n_rk=3, compact=False):
    """1-D Euler Riemann problem on [0, 1] (non-dimensional: T < 1 K sits in table row 0, allowed
    for Euler), transmissive ends (400 -> extrapolation, type 11) and type-11 lateral faces as in
    test/1D/Sod79/INPUT/bc.txt. left/right = (rho, u, p). compact: uniform-grid geometry and implicit k faces
    (layout_case)."""
    th = ideal_gas_tables()
    h = 1.0 / n

    def nodes(iu, iv, iw):
        return np.stack([iu * h, iv * h, iw * h], axis=-1)

    def prim(c):
        x = c[..., 0]
        L = np.array(left, dtype=np.float64); Rr = np.array(right, dtype=np.float64)
        rho = np.where(x < x0, L[0], Rr[0]); u = np.where(x < x0, L[1], Rr[1]); p = np.where(x < x0, L[2], Rr[2])
        z = np.zeros_like(x)
        return np.stack([rho, u, z, z, p])

    scheme = dict(limiter=limiter, riemann=riemann, visc=0, n_rk=n_rk, ndir=1, cfl=cfl, time_clip=1,
                  time_threshold=t_end)
    bc = {f: abi.BC_EXTRAPOLATION for f in range(1, 7)}
    case = layout_case("riemann1d_%d" % n, [[0, n], [0, 1], [0, 1]], nodes, (False, False, False), bc, th,
                       scheme, prim, uniform=(h, h, h) if compact else None, implicit_k=compact)
    case.meta = dict(left=left, right=right, x0=x0, t_end=t_end)
    case.steps = None
    return case


def riemann_2d(n=128, states=None, t_end=0.25, cfl=0.5, riemann=abi.RS_HLLC, limiter=abi.LIM_MINMOD, compact=False):
    """2-D four-quadrant Riemann problem on [0,1]^2 (n x n cells, one k layer), extrapolation on every
    face. states = [(rho,u,v,p)] for the quadrants (x>.5,y>.5), (x<.5,y>.5), (x<.5,y<.5), (x>.5,y<.5).
    compact: uniform-grid geometry and implicit k faces (layout_case)."""
    th = ideal_gas_tables()
    h = 1.0 / n
    if states is None:
        states = [(1.5, 0.0, 0.0, 1.5), (0.5323, 1.206, 0.0, 0.3), (0.138, 1.206, 1.206, 0.029),
                  (0.5323, 0.0, 1.206, 0.3)]

    def nodes(iu, iv, iw):
        return np.stack([iu * h, iv * h, iw * h], axis=-1)

    def prim(c):
        x, y = c[..., 0], c[..., 1]
        q = [np.array(s, dtype=np.float64) for s in states]
        sel = [(x > 0.5) & (y > 0.5), (x <= 0.5) & (y > 0.5), (x <= 0.5) & (y <= 0.5), (x > 0.5) & (y <= 0.5)]
        out = np.zeros((5,) + x.shape)
        for m, s in zip(sel, q):
            out[0][m] = s[0]; out[1][m] = s[1]; out[2][m] = s[2]; out[4][m] = s[3]
        return out

    scheme = dict(limiter=limiter, riemann=riemann, visc=0, n_rk=3, ndir=2, cfl=cfl, time_clip=1,
                  time_threshold=t_end)
    bc = {f: abi.BC_EXTRAPOLATION for f in range(1, 7)}
    case = layout_case("riemann2d_%d" % n, [[0, n], [0, n], [0, 1]], nodes, (False, False, False), bc, th,
                       scheme, prim, uniform=(h, h, h) if compact else None, implicit_k=compact)
    case.meta = dict(t_end=t_end)
    return case


def exact_riemann(left, right, x, t, gamma=1.4, x0=0.5):
    """Exact solution of the 1-D Euler Riemann problem (Toro, Riemann Solvers and Numerical Methods for
    Fluid Dynamics, ch. 4: Newton iteration on the star pressure, then wave sampling).
    left/right = (rho, u, p); returns rho, u, p at the points x and time t."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl = math.sqrt(gamma * pl / rl)
    cr = math.sqrt(gamma * pr / rr)
    g1 = (gamma - 1) / (2 * gamma); g2 = (gamma + 1) / (2 * gamma); g3 = 2 * gamma / (gamma - 1)
    g4 = 2 / (gamma - 1); g5 = 2 / (gamma + 1); g6 = (gamma - 1) / (gamma + 1); g7 = (gamma - 1) / 2

    def f(p, rk, pk, ck):
        if p <= pk:
            pr_ = p / pk
            fv = g4 * ck * (pr_ ** g1 - 1.0)
            fd = (1.0 / (rk * ck)) * pr_ ** (-g2)
        else:
            ak = g5 / rk; bk = g6 * pk
            q = math.sqrt(ak / (bk + p))
            fv = (p - pk) * q
            fd = (1.0 - 0.5 * (p - pk) / (bk + p)) * q
        return fv, fd

    p = max(1e-12, 0.5 * (pl + pr) - 0.125 * (ur - ul) * (rl + rr) * (cl + cr))
    for _ in range(100):
        fl, fdl = f(p, rl, pl, cl)
        fr, fdr = f(p, rr, pr, cr)
        pn = p - (fl + fr + ur - ul) / (fdl + fdr)
        pn = max(pn, 1e-12)
        if abs(pn - p) / (0.5 * (pn + p)) < 1e-14:
            p = pn
            break
        p = pn
    fl, _ = f(p, rl, pl, cl)
    fr, _ = f(p, rr, pr, cr)
    um = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    rho = np.empty_like(x); u = np.empty_like(x); pp = np.empty_like(x)
    for n_, xx in enumerate(x):
        s = (xx - x0) / t
        if s <= um:
            if p <= pl:
                shl = ul - cl
                if s <= shl:
                    rho[n_], u[n_], pp[n_] = rl, ul, pl
                else:
                    cml = cl * (p / pl) ** g1
                    stl = um - cml
                    if s > stl:
                        rho[n_], u[n_], pp[n_] = rl * (p / pl) ** (1 / gamma), um, p
                    else:
                        u_ = g5 * (cl + g7 * ul + s)
                        c_ = g5 * (cl + g7 * (ul - s))
                        rho[n_] = rl * (c_ / cl) ** g4; u[n_] = u_; pp[n_] = pl * (c_ / cl) ** g3
            else:
                sl = ul - cl * math.sqrt(g2 * p / pl + g1)
                if s <= sl:
                    rho[n_], u[n_], pp[n_] = rl, ul, pl
                else:
                    rho[n_] = rl * ((p / pl + g6) / ((p / pl) * g6 + 1)); u[n_] = um; pp[n_] = p
        else:
            if p > pr:
                sr = ur + cr * math.sqrt(g2 * p / pr + g1)
                if s >= sr:
                    rho[n_], u[n_], pp[n_] = rr, ur, pr
                else:
                    rho[n_] = rr * ((p / pr + g6) / ((p / pr) * g6 + 1)); u[n_] = um; pp[n_] = p
            else:
                shr = ur + cr
                if s >= shr:
                    rho[n_], u[n_], pp[n_] = rr, ur, pr
                else:
                    cmr = cr * (p / pr) ** g1
                    str_ = um + cmr
                    if s <= str_:
                        rho[n_], u[n_], pp[n_] = rr * (p / pr) ** (1 / gamma), um, p
                    else:
                        u_ = g5 * (-cr + g7 * ur + s)
                        c_ = g5 * (cr - g7 * (ur - s))
                        rho[n_] = rr * (c_ / cr) ** g4; u[n_] = u_; pp[n_] = pr * (c_ / cr) ** g3
    return rho, u, pp
