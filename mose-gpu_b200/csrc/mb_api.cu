// mb_api.cu -- the C ABI of include/mose_b200.h: context set-up (device tables built once from the
// host descriptions, as Setup_BC_Device / Setup_Device_Residency do), the per-call entry points
// and the time loop with a device-side clock, optionally replayed as a CUDA graph.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <unordered_map>
#include <algorithm>
#include "../../include/mose_b200.h"
#include <cudaTypedefs.h>  // CUtensorMap and the driver's tensor-map encoder type (taken at run time, no -lcuda)
#include "mb_launch.h"

using namespace mb;

struct mb_ctx {
  int device = 0;
  mb_scheme sc;
  Params p;
  GhostLists g;
  // device allocations
  DBlk* d_blk = nullptr;
  int* d_recmap = nullptr;
  DRec* d_rec = nullptr;
  std::vector<mb_bc> hrec;      // the host records of the current mesh (mb_set_record_params)
  std::vector<DRec> hdrec;      // their device form (the source of single-record updates)
  GRec* d_grec = nullptr;
  int* d_phys = nullptr;
  int* d_cubic = nullptr;
  int* d_physf = nullptr;       // the fused stage's ghost lists: only the layers some computation reads
  int* d_cubicf = nullptr;
  GhostLists gf;
  long long* d_cdst = nullptr;
  long long* d_csrc = nullptr;
  long long* d_pgsrc = nullptr;
  double* d_recflux = nullptr;  // boundary-record contributions [nrec][10] (flux type)
  int* d_brec = nullptr;        // records in type order (the record kernel's work list)
  int* d_bcell = nullptr;       // their blk, i, j, k, face
  int nrec = 0;
  double* d_tab = nullptr;
  float* d_tabf = nullptr;
  DevState* d_st = nullptr;
  DTile* d_tiles_sweep = nullptr;
  int ntiles_sweep = 0;
  DTile* d_tiles_km = nullptr;  // tiles of the mirrored one-plane blocks (their own sweep instantiation)
  int ntiles_km = 0;
  std::vector<int> hkm;         // mirrored-block flag per block
  std::vector<int> hdims;       // 3 per block of the current mesh (interior extents)
  int kc3 = 16;                 // k-chunk of the sweep tiles of blocks deeper than one cell (mb_set_tuning; the value
                                // reported by mb_get_tuning: the chunk of the class with the most cells)
  int kcls[4] = {16, 16, 16, 16};  // the k-chunk per depth class of 3-D blocks (kclass_of), autotuned per class
  int persistent = 0;           // persistent work-queue sweep of the main tile list (autotuned)
  int persistent_km = 0;        // the same for the tiles of mirrored one-plane blocks (autotuned)
  float tuned_ms = 0.f;         // sweep time of the chosen configuration
  int* d_queue = nullptr;       // tile counter of the persistent sweep
  int ty_sweep = 4;
  DTile* d_tiles_aux = nullptr;
  int ntiles_aux = 0;
  double* d_scratch = nullptr;  // the engine's own stage buffer (ncell x 5)
  // TMA tensor maps of the state buffers the mixed sweep stages from: (buffer, its row count) -> a CUtensorMap in
  // device memory; made outside any capture, never rewritten (a captured step keeps pointing at its maps)
  struct Tmap { const double* ptr; long long nc; void* dev; };
  std::vector<Tmap> tmaps;
  bool no_tma = false;          // MB_NO_TMA set at mb_init: no tensor maps (the TMA staging is never used)
  bool stage_tma = true;        // the mixed sweep stages by TMA where a map exists (mb_set_staging, mb_autotune)
  bool stage_tma_km = true;     // the same for the tile list of mirrored one-plane blocks (tuned separately)
  cudaStream_t tstream = 0;     // the stream the mesh tables are (re)built in the order of (build_tables)
  long long sweeps_tma = 0, sweeps_plain = 0;  // sweep launches of the mixed form by staging path
  double* d_acc4 = nullptr;     // RK4: conserved accumulator (ncell x 5)
  double* d_irs = nullptr;      // residual smoothing: two residual buffers (2 x ncell x 5)
  long long* d_idst = nullptr;  // its first-ghost-layer copies, direction by direction: row idst[e] <- row isrc[e]
  long long* d_isrc = nullptr;
  int irs_off[4] = {0, 0, 0, 0};
  double* d_ur = nullptr;       // prec: Ur of every row (ghost rows 0), its smoothing buffer, the step's local steps
  double* d_urb = nullptr;
  double* d_dtl = nullptr;
  struct Geo32 { const double* src; float* buf; long long n; };
  std::vector<Geo32> geo32;     // FP32 geometry copies of the mixed form (source array, copy, elements)
  int ngroups = 1;              // case clocks
  long long ncell = 0;
  bool dt_valid = false;
  long long launches = 0;
  // graph of one step
  cudaGraphExec_t gexec = nullptr;
  cudaGraph_t graph = nullptr;
  const double* gP = nullptr;
  const double* gPO = nullptr;
  cudaStream_t gstream = nullptr;
  int graph_kernels = 0;
};

#define CK(x)                                    \
  do {                                           \
    cudaError_t e_ = (x);                        \
    if (e_ != cudaSuccess) {                     \
      fprintf(stderr, "[mose_b200] CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
      return MB_E_CUDA;                          \
    }                                            \
  } while (0)

// a device copy of a host array, allocated and copied in the order of stream s (the stream-ordered allocator: a
// table rebuilt while the previous tables are still read by queued work on s is released after that work)
// (s = 0, the legacy stream: the copy is complete on return, ready for work on any stream)
template <typename T>
static int upload(T** dst, const T* src, size_t n, cudaStream_t s = 0) {
  if (n == 0) { *dst = nullptr; return MB_OK; }
  if (cudaMallocAsync((void**)dst, n * sizeof(T), s) != cudaSuccess) return MB_E_NOMEM;
  CK(cudaMemcpyAsync(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice, s));
  if (s == 0) CK(cudaStreamSynchronize(0));
  return MB_OK;
}

static void free_ctx(mb_ctx* c) {
  if (!c) return;
  for (auto& m : c->tmaps) cudaFree(m.dev);
  c->tmaps.clear();
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->graph) cudaGraphDestroy(c->graph);
  void* ptrs[] = {c->d_blk, c->d_recmap, c->d_rec, c->d_grec, c->d_phys, c->d_cubic, c->d_cdst, c->d_csrc,
                  c->d_pgsrc, c->d_tab, c->d_tabf, c->d_st, c->d_tiles_sweep, c->d_tiles_aux, c->d_scratch, c->d_acc4, c->d_queue, c->d_recflux, c->d_brec, c->d_bcell,
                  c->d_physf, c->d_cubicf, c->d_tiles_km, c->d_irs, c->d_idst, c->d_isrc, c->d_ur, c->d_urb, c->d_dtl};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  for (auto& q : c->geo32)
    if (q.buf) cudaFree(q.buf);
  delete c;
}

// the tiles (32 x ty cells, kc planes) of the blocks whose class (3: deeper than one cell in k, 2: one k plane,
// 1: one cell deep in j and k) is in mask (bit cls), block-major
// km: the mirrored-block flag per block; km_sel 0 / 1 keeps only the blocks with that flag (-1: all)
// the depth class of a 3-D block for the k-chunk autotuning: n3 <= 16, <= 64, <= 256, more
static int kclass_of(int n3) { return n3 <= 16 ? 0 : (n3 <= 64 ? 1 : (n3 <= 256 ? 2 : 3)); }

// kcls: the k-chunk per depth class (null: kc for every block); dsel >= 0 keeps only the 3-D blocks of that class
static std::vector<DTile> make_tiles(const std::vector<int>& dims, int ty, int kc, int mask = 0xe,
                                     const std::vector<int>* km = nullptr, int km_sel = -1, const int* kcls = nullptr,
                                     int dsel = -1) {
  std::vector<DTile> t;
  const int nb = (int)dims.size() / 3;
  for (int b = 0; b < nb; ++b) {
    const int* n = &dims[3 * b];
    const int cls = n[2] > 1 ? 3 : (n[1] > 1 ? 2 : 1);
    if (!(mask & (1 << cls))) continue;
    if (dsel >= 0 && (cls != 3 || kclass_of(n[2]) != dsel)) continue;
    const int kcb = (kcls && n[2] > 1) ? kcls[kclass_of(n[2])] : kc;
    if (km && (*km)[b] < 0) continue;  // an external block: nothing is computed on it
    if (km && km_sel >= 0 && (*km)[b] != km_sel) continue;
    for (int k0 = 1; k0 <= n[2]; k0 += kcb)
      for (int j0 = 1; j0 <= n[1]; j0 += ty)
        for (int i0 = 1; i0 <= n[0]; i0 += 32) t.push_back(DTile{b, i0, j0, k0, std::min(k0 + kcb, n[2] + 1)});
  }
  return t;
}

// the tile order of a persistent sweep: the largest tiles first, so that the queue ends on small ones
static void sort_by_work(std::vector<DTile>& t, const std::vector<int>& dims, int ty) {
  auto w = [&](const DTile& d) {
    const int* n = &dims[3 * d.blk];
    return (long long)(d.k1 - d.k0) * std::min(32, n[0] - d.i0 + 1) * std::min(ty, n[1] - d.j0 + 1);
  };
  std::stable_sort(t.begin(), t.end(), [&](const DTile& a, const DTile& b) { return w(a) > w(b); });
}

static const double RKC[3][3] = {{1.0, 0.0, 0.0}, {1.0, 0.50, 0.0}, {1.0, 0.25, 2.0 / 3.0}};  // Lib_RK.f90:6-9

// rk_coeff of stage irk (the SSP forms); RK4 carries its own weights in the update (cons_update)
static double rkc_of(int n, int irk) { return n == 4 ? 0.0 : RKC[n - 1][irk - 1]; }

// stage irk of the step: input / output buffers so that the state lands back in P after the last stage (the
// old state u^n in P is only read at the updated cell itself, so the last stage updates P in place):
//   RK4: P -> S, S -> PO, PO -> S, S -> P     RK3: P -> S, S -> PO, PO -> P
//   RK2: P -> S, S -> P                       Euler: P -> S, then S copied to P
static void stage_buffers(int n, int irk, double* P, double* PO, double* S, const double** in, double** out) {
  if (irk == 1) { *in = P; *out = S; }
  else if (n == 2) { *in = S; *out = P; }
  else if (n == 3) { *in = (irk == 2) ? S : PO; *out = (irk == 2) ? PO : P; }
  else {
    const double* ins[4] = {P, S, PO, S};
    double* outs[4] = {S, PO, S, P};
    *in = ins[irk - 1];
    *out = outs[irk - 1];
  }
}

extern "C" {

const char* mb_version(void) { return "mose_b200 0.1 (sm_100a)"; }

int mb_selftest_bounded_wait(int device, int tries, int* gave_up) {
  if (!gave_up || tries < 1) return MB_E_ARG;
  CK(cudaSetDevice(device));
  int* d = nullptr;
  CK(cudaMalloc((void**)&d, sizeof(int)));
  cudaError_t e = wait_selftest((unsigned)tries, d, 0);
  if (e == cudaSuccess) e = cudaMemcpy(gave_up, d, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  CK(e);
  return MB_OK;
}

int mb_set_staging(mb_ctx* ctx, int tma) {
  if (!ctx || tma < 0 || tma > 1) return MB_E_ARG;
  if (ctx->stage_tma != (tma == 1) || ctx->stage_tma_km != (tma == 1)) {
    ctx->stage_tma = tma == 1;
    ctx->stage_tma_km = tma == 1;
    if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }  // a replay in flight completes
    if (ctx->graph) { cudaGraphDestroy(ctx->graph); ctx->graph = nullptr; }
    ctx->gP = nullptr;
    ctx->gPO = nullptr;
  }
  return MB_OK;
}

int mb_get_staging(const mb_ctx* ctx, int64_t* tma_sweeps, int64_t* plain_sweeps) {
  if (!ctx || !tma_sweeps || !plain_sweeps) return MB_E_ARG;
  *tma_sweeps = ctx->sweeps_tma;
  *plain_sweeps = ctx->sweeps_plain;
  return MB_OK;
}

int mb_get_staging_mode(const mb_ctx* ctx, int* tma) {
  if (!ctx || !tma) return MB_E_ARG;
  *tma = (ctx->ntiles_sweep > 0 ? ctx->stage_tma : ctx->stage_tma_km) ? 1 : 0;
  return MB_OK;
}

int64_t mb_launch_count(const mb_ctx* ctx) { return ctx ? ctx->launches : 0; }

// the checks of a mesh description that mb_init and mb_reconfigure share
// the parameters of one record (mb_bc.q) for its type
static int check_record_params(const mb_bc& r) {
  if (r.type == MB_BC_INFLOW) {
    if (!(r.q[1] > 0.0 && r.q[2] > 0.0)) return MB_E_ARG;  // T0, p0 (or the mass flux)
    const int code = (int)r.q[6];
    if (code != 0 && code != 401 && code != 403 && code != 404 && code != 405 && code != 407) return MB_E_UNSUPPORTED;
    if (code == 404 && r.q[5] != 1.0) return MB_E_UNSUPPORTED;  // IO_BC_Open.f90:276-281
    if (code == 401 || code == 403 || code == 404 || code == 407) {  // the face tangent is read
      const double tn = r.q[8] * r.q[8] + r.q[9] * r.q[9] + r.q[10] * r.q[10];
      if (!(fabs(tn - 1.0) < 1e-6)) return MB_E_ARG;
    }
  }
  if (r.type == MB_BC_WALL_T && !(r.q[0] > 0.0)) return MB_E_ARG;                   // T_wall
  if (r.type == MB_BC_OUTLET && !(r.q[0] >= 0.0 && r.q[1] >= 0.0 && r.q[1] <= 1.0)) return MB_E_ARG;
  return MB_OK;
}

// the device record of one mb_bc: the type, the connection row and the parameters in the form the kernels read
static void fill_drec(const mb_bc& r, DRec* d) {
  d->type = r.type;
  d->pg = r.conn;
  for (int s = 0; s < 16; ++s) d->q[s] = 0.0;
  if (r.type == MB_BC_INFLOW) {  // mach, T0, p0, rel_fac, cos / sin of alpha and beta, code, pamb, alpha, beta, t
    const double v[8] = {r.q[0], r.q[1], r.q[2], r.q[5], cos(r.q[3]), sin(r.q[3]), cos(r.q[4]), sin(r.q[4])};
    for (int s = 0; s < 8; ++s) d->q[s] = v[s];
    d->q[8] = r.q[6]; d->q[9] = r.q[7]; d->q[10] = r.q[3]; d->q[11] = r.q[4];
    d->q[12] = r.q[8]; d->q[13] = r.q[9]; d->q[14] = r.q[10];
  }
  if (r.type == MB_BC_WALL_T) d->q[0] = r.q[0];                                 // T_wall
  if (r.type == MB_BC_OUTLET) { d->q[0] = r.q[0]; d->q[1] = r.q[1]; }         // exit pressure, relaxation
}

static int check_mesh(const mb_mesh* mesh, int ngroups) {
  int rc;
  if (!mesh || mesh->nblk <= 0 || mesh->ncell_total <= 0 || !mesh->blk) return MB_E_ARG;
  if (mesh->nrec > 0 && !mesh->rec) return MB_E_ARG;
  if (mesh->nrec >= (1 << 28)) return MB_E_ARG;  // record ids share a 32-bit word with a layer count
  if (mesh->nconn > 0 && !mesh->conn) return MB_E_ARG;
  for (int b = 0; b < mesh->nblk; ++b) {
    const mb_block& q = mesh->blk[b];
    if (q.n[0] < 1 || q.n[1] < 1 || q.n[2] < 1 || !q.fm1 || !q.fm2 || !q.fm3 || !q.dl || !q.m || !q.vol) return MB_E_ARG;
    if (q.group < -1 || q.group >= ngroups) return MB_E_ARG;  // -1: an external block (a halo copy)
    // intra-block offsets of the sweep are 32-bit: 9 metric values per padded cell, 4 per face
    const long long npad = (long long)(q.n[0] + 2 * MB_GC) * (q.n[1] + 2 * MB_GC) * (q.n[2] + 2 * MB_GC);
    if (9 * npad >= (1LL << 31)) return MB_E_ARG;
    const long long np = (long long)(q.n[0] + 2 * MB_GC) * (q.n[1] + 2 * MB_GC) * (q.n[2] + 2 * MB_GC);
    if (q.boff < 0 || q.boff + np > mesh->ncell_total) return MB_E_ARG;
  }
  for (int q = 0; q < mesh->nrec; ++q) {
    const mb_bc& r = mesh->rec[q];
    if (r.type != MB_BC_CONNECTION && r.type != MB_BC_EXTRAPOLATION && r.type != MB_BC_WALL &&
        r.type != MB_BC_INFLOW && r.type != MB_BC_SYMMETRY && r.type != MB_BC_WALL_T && r.type != MB_BC_OUTLET &&
        r.type != MB_BC_NONE)
      return MB_E_UNSUPPORTED;
    if (r.blk < 0 || r.blk >= mesh->nblk || r.face < 1 || r.face > 6) return MB_E_ARG;
    if (mesh->blk[r.blk].group < 0) return MB_E_ARG;  // an external block carries no records
    if ((rc = check_record_params(r)) != MB_OK) return rc;
  }
  return MB_OK;
}

// frees the mesh-dependent device tables (blocks, record maps, records, ghost lists, tiles, FP32 geometry)
static void free_tables(mb_ctx* c) {
  void* ptrs[] = {c->d_blk, c->d_recmap, c->d_rec, c->d_grec, c->d_phys, c->d_cubic, c->d_cdst, c->d_csrc,
                  c->d_pgsrc, c->d_tiles_sweep, c->d_tiles_aux, c->d_recflux, c->d_brec, c->d_bcell,
                  c->d_physf, c->d_cubicf, c->d_tiles_km, c->d_idst, c->d_isrc};
  for (void* q : ptrs)
    if (q) cudaFreeAsync(q, c->tstream);  // after the work queued on the table stream that may still read them
  c->d_idst = nullptr; c->d_isrc = nullptr;
  for (int d = 0; d < 4; ++d) c->irs_off[d] = 0;
  c->d_physf = nullptr; c->d_cubicf = nullptr; c->d_tiles_km = nullptr; c->ntiles_km = 0;
  c->d_recflux = nullptr; c->d_brec = nullptr; c->d_bcell = nullptr; c->nrec = 0;
  c->d_blk = nullptr; c->d_recmap = nullptr; c->d_rec = nullptr; c->d_grec = nullptr; c->d_phys = nullptr;
  c->d_cubic = nullptr; c->d_cdst = nullptr; c->d_csrc = nullptr; c->d_pgsrc = nullptr;
  c->d_tiles_sweep = nullptr; c->d_tiles_aux = nullptr;
}

// the sweep unit of a scheme: the benchmarked solvers' own (the solver a compile-time constant) unless a shock sensor,
// the primitive update or local time stepping is on, which only the run-time solver unit carries
static int sweep_unit(const mb_scheme* sc) {
  return (mb_effective_sensor(sc->riemann, sc->sensor) || sc->intvar || sc->local_dt || sc->riemann > 13) ? 0
                                                                                                          : sc->riemann;
}

// record types with physical ghosts (Fill_Ghost_Cell_blk, Lib_Extrapolation.f90:643-730)
static bool phys_type(int t) {
  return t == MB_BC_EXTRAPOLATION || t == MB_BC_INFLOW || t == MB_BC_WALL || t == MB_BC_SYMMETRY ||
         t == MB_BC_WALL_T || t == MB_BC_OUTLET || t == MB_BC_NONE;
}

// builds the mesh-dependent device tables from the host description (Setup_BC_Device, Mod_BC.f90:99-338) and
// points the kernel parameters and ghost lists at them
static int build_tables(mb_ctx* c, const mb_mesh* mesh) {
  const mb_scheme* sc = &c->sc;
  int rc;
  // ---- blocks and the per-face record maps
  std::vector<DBlk> hb(mesh->nblk);
  std::vector<int> recmap;
  // ndir: the scheme's for one case; per case, from the dimensions of its first block as the reference sets it
  // for its one case (Lib_Metrics.f90:150-172: nk > 1 -> 3, nj = nk = 1 -> 1, else 2)
  std::vector<int> gndir(c->ngroups, 0);
  for (int b = 0; b < mesh->nblk; ++b) {
    const mb_block& q = mesh->blk[b];
    if (q.group < 0) continue;
    if (gndir[q.group] == 0) gndir[q.group] = (q.n[2] > 1) ? 3 : ((q.n[1] == 1 && q.n[2] == 1) ? 1 : 2);
  }
  for (int b = 0; b < mesh->nblk; ++b) {
    const mb_block& q = mesh->blk[b];
    DBlk& d = hb[b];
    memset(&d, 0, sizeof(d));
    d.n1 = q.n[0]; d.n2 = q.n[1]; d.n3 = q.n[2];
    d.pi = q.n[0] + 2 * MB_GC; d.pj = q.n[1] + 2 * MB_GC;
    d.grp = q.group;
    d.ndir = (c->ngroups > 1 && q.group >= 0) ? gndir[q.group] : sc->ndir;
    d.boff = q.boff;
    d.fm1 = q.fm1; d.fm2 = q.fm2; d.fm3 = q.fm3; d.dl = q.dl; d.m = q.m; d.vol = q.vol;
    for (int f = 0; f < 6; ++f) d.rmap[f] = -1;
  }
  for (int q = 0; q < mesh->nrec; ++q) {
    const mb_bc& r = mesh->rec[q];
    if (r.type == MB_BC_NONE) continue;  // no face flux: the sweep finds no record on that face
    DBlk& d = hb[r.blk];
    const int ax = (r.face - 1) / 2;
    const int nt = (ax == 0) ? d.n2 * d.n3 : (ax == 1 ? d.n1 * d.n3 : d.n1 * d.n2);
    if (d.rmap[r.face - 1] < 0) {
      d.rmap[r.face - 1] = (int)recmap.size();
      recmap.resize(recmap.size() + nt, -1);
    }
    const int n[3] = {d.n1, d.n2, d.n3};
    const int cc[3] = {r.i, r.j, r.k};
    if (r.i < 1 || r.i > d.n1 || r.j < 1 || r.j > d.n2 || r.k < 1 || r.k > d.n3 ||
        cc[ax] != ((r.face & 1) ? 1 : n[ax]))
      return MB_E_ARG;
    int t = (ax == 0) ? (r.j - 1) + (r.k - 1) * d.n2 : (ax == 1 ? (r.i - 1) + (r.k - 1) * d.n1 : (r.i - 1) + (r.j - 1) * d.n1);
    recmap[d.rmap[r.face - 1] + t] = q;
  }
  // ---- records
  std::vector<DRec> hr(mesh->nrec);
  std::vector<GRec> hg(mesh->nrec);
  std::vector<int> phys, cubic;
  for (int q = 0; q < mesh->nrec; ++q) {
    const mb_bc& r = mesh->rec[q];
    fill_drec(r, &hr[q]);
    hg[q] = GRec{r.blk, r.i, r.j, r.k, r.face, r.type};
    if (phys_type(r.type)) phys.push_back(q);
    if (r.type == MB_BC_EXTRAPOLATION) cubic.push_back(q);
  }
  // The fused stage fills only the ghost layers that some computation of the stage reads (entries carry their
  // layer count in bits 28-29; mb_fill_ghosts keeps the reference's full fill):
  //  - along an axis of two or more cells, the second layer of a type 11 / 4 / 5 / 6 / 24 face is read by nothing
  //    (interior faces read one layer, these records read the boundary cell and its neighbours): one layer (a
  //    symmetry face fills its first layer only, in both fills);
  //  - along an axis one cell deep whose two faces are both type 11, an Euler stage reads no ghost there (no
  //    faces along it, no viscous stencil, extrapolation records read the cell): no layer;
  //  - otherwise both layers (the cubic ghost of a one-cell-deep axis reads the opposite face's layers).
  std::vector<int> physf, cubicf;
  {
    std::vector<int> all11(3 * (size_t)mesh->nblk, 1);
    std::vector<long long> nface(6 * (size_t)mesh->nblk, 0);
    for (int q = 0; q < mesh->nrec; ++q) {
      const mb_bc& r = mesh->rec[q];
      if (r.type != MB_BC_EXTRAPOLATION) all11[3 * r.blk + (r.face - 1) / 2] = 0;
      nface[6 * r.blk + r.face - 1] += 1;
    }
    for (int b = 0; b < mesh->nblk; ++b) {
      DBlk& d = hb[b];
      const long long nk = (long long)d.n1 * d.n2;
      // extrapolation records on every cell of both k faces, or no k-face record at all (a one-plane block
      // without k-face records is taken as extrapolated there: the reference's 2-D meshes, 2 n1 n2 records fewer)
      const bool kfull = nface[6 * b + 4] == nk && nface[6 * b + 5] == nk;
      const bool knone = nface[6 * b + 4] == 0 && nface[6 * b + 5] == 0;
      d.kmirror = (d.n3 == 1 && all11[3 * b + 2] && (kfull || knone)) ? 1 : 0;
    }
    for (int q = 0; q < mesh->nrec; ++q) {
      const mb_bc& r = mesh->rec[q];
      if (!phys_type(r.type)) continue;
      if (hb[r.blk].kmirror && r.face >= 5) continue;  // the k ghosts of a mirrored block are never read
      const int ax = (r.face - 1) / 2;
      const int nax = mesh->blk[r.blk].n[ax];
      int layers = 2;
      if (nax >= 2) layers = 1;
      else if (!sc->visc && !mb_effective_sensor(sc->riemann, sc->sensor) && all11[3 * r.blk + ax]) layers = 0;
      if (layers == 0) continue;
      physf.push_back(q | (layers << 28));
      if (r.type == MB_BC_EXTRAPOLATION) cubicf.push_back(q | (layers << 28));
    }
  }
  // the record kernel's work list: records grouped by type (one code path per warp where possible), without the
  // k-face records of mirrored blocks (their sweep computes those)
  std::vector<int> brec;
  for (int q = 0; q < mesh->nrec; ++q)
    if (!(hb[mesh->rec[q].blk].kmirror && mesh->rec[q].face >= 5) && mesh->rec[q].type != MB_BC_NONE) brec.push_back(q);
  std::stable_sort(brec.begin(), brec.end(), [&](int a, int b) { return mesh->rec[a].type < mesh->rec[b].type; });
  std::vector<int> bcell(5 * brec.size());
  for (size_t q = 0; q < brec.size(); ++q) {
    const mb_bc& r = mesh->rec[brec[q]];
    const int v[5] = {r.blk, r.i, r.j, r.k, r.face};
    for (int a = 0; a < 5; ++a) bcell[5 * q + a] = v[a];
  }
  // ---- connections: ghost copies (2 layers) and the bc_pg source rows
  auto rowof = [&](int b, int i, int j, int k) -> long long {
    const DBlk& d = hb[b];
    return d.boff + (long long)(i + MB_GC - 1) + (long long)(j + MB_GC - 1) * d.pi + (long long)(k + MB_GC - 1) * d.pi * d.pj;
  };
  auto guide = [](int F, int ax) { int d = (F + 1) / 2 - 1; return ax == d ? ((F % 2) ? 1 : -1) : 0; };
  std::vector<long long> cdst, csrc, pgsrc;
  for (int q = 0; q < mesh->nconn; ++q) {
    const mb_conn& cn = mesh->conn[q];
    if (cn.rec < 0 || cn.rec >= mesh->nrec || cn.bs < 0 || cn.bs >= mesh->nblk || mesh->rec[cn.rec].conn != q)
      return MB_E_ARG;
    const mb_bc& r = mesh->rec[cn.rec];
    for (int g = 1; g <= MB_GC; ++g) {
      cdst.push_back(rowof(r.blk, r.i - guide(r.face, 0) * g, r.j - guide(r.face, 1) * g, r.k - guide(r.face, 2) * g));
      csrc.push_back(rowof(cn.bs, cn.is + guide(cn.fs, 0) * (g - 1), cn.js + guide(cn.fs, 1) * (g - 1),
                           cn.ks + guide(cn.fs, 2) * (g - 1)));
    }
    const int I = cn.is, J = cn.js, K = cn.ks;
    int t[4][3];
    if (cn.fs <= 2) {
      int a[4][3] = {{I, J - cn.d11, K - cn.d12}, {I, J + cn.d11, K + cn.d12}, {I, J - cn.d21, K - cn.d22}, {I, J + cn.d21, K + cn.d22}};
      memcpy(t, a, sizeof(t));
    } else if (cn.fs <= 4) {
      int a[4][3] = {{I - cn.d11, J, K - cn.d12}, {I + cn.d11, J, K + cn.d12}, {I - cn.d21, J, K - cn.d22}, {I + cn.d21, J, K + cn.d22}};
      memcpy(t, a, sizeof(t));
    } else {
      int a[4][3] = {{I - cn.d11, J - cn.d12, K}, {I + cn.d11, J + cn.d12, K}, {I - cn.d21, J - cn.d22, K}, {I + cn.d21, J + cn.d22, K}};
      memcpy(t, a, sizeof(t));
    }
    pgsrc.push_back(rowof(cn.bs, I, J, K));
    pgsrc.push_back(rowof(cn.bs, I + guide(cn.fs, 0), J + guide(cn.fs, 1), K + guide(cn.fs, 2)));
    for (int m = 0; m < 4; ++m)  // a mirrored donor's k ghosts are its k = 1 cells
      pgsrc.push_back(rowof(cn.bs, t[m][0], t[m][1], hb[cn.bs].kmirror ? 1 : t[m][2]));
  }
  // every row must lie inside the arena
  for (const auto* v : {&cdst, &csrc, &pgsrc})
    for (long long x : *v)
      if (x < 0 || x >= c->ncell) return MB_E_ARG;
  // ---- tiles
  c->hdims.assign(3 * (size_t)mesh->nblk, 0);
  for (int b = 0; b < mesh->nblk; ++b)
    for (int a = 0; a < 3; ++a) c->hdims[3 * b + a] = mesh->blk[b].n[a];
  c->hkm.assign(mesh->nblk, 0);
  for (int b = 0; b < mesh->nblk; ++b) c->hkm[b] = mesh->blk[b].group < 0 ? -1 : hb[b].kmirror;
  std::vector<DTile> ts = make_tiles(c->hdims, c->ty_sweep, c->kc3, 0xe, &c->hkm, 0, c->kcls);
  std::vector<DTile> tk = make_tiles(c->hdims, c->ty_sweep, c->kc3, 0xe, &c->hkm, 1);
  if (c->persistent) sort_by_work(ts, c->hdims, c->ty_sweep);
  if (c->persistent_km) sort_by_work(tk, c->hdims, c->ty_sweep);
  std::vector<DTile> ta = make_tiles(c->hdims, TY_AUX, 16, 0xe, &c->hkm, -1);
  // ---- the mixed form reads its geometry in FP32: one conversion per distinct array of this mesh (blocks may
  // share arrays). Every copy is converted afresh (a caller may have replaced an array at the same address);
  // the buffers of the previous mesh are reused where the size matches.
  if (sc->precision == MB_PREC_MIXED) {
    std::vector<mb_ctx::Geo32> keep, pool = c->geo32;
    for (auto& d : hb) {
      const long long pk = d.n3 + 2 * MB_GC;
      const long long npad = (long long)d.pi * d.pj * pk;
      const long long n[5] = {4LL * (d.n1 + 1) * d.n2 * d.n3, 4LL * d.n1 * (d.n2 + 1) * d.n3, 4LL * d.n1 * d.n2 * (d.n3 + 1),
                              3 * npad, 9 * npad};
      const double* src[5] = {d.fm1, d.fm2, d.fm3, d.dl, d.m};
      float* dst[5];
      for (int q = 0; q < 5; ++q) {
        dst[q] = nullptr;
        for (auto& m : keep)
          if (m.src == src[q]) dst[q] = m.buf;
        if (dst[q]) continue;
        for (auto& m : pool)
          if (m.buf && m.n == n[q]) { dst[q] = m.buf; m.buf = nullptr; break; }
        if (!dst[q] && cudaMallocAsync((void**)&dst[q], n[q] * sizeof(float), c->tstream) != cudaSuccess) {
          for (auto& m : keep) cudaFreeAsync(m.buf, c->tstream);
          for (auto& m : pool) if (m.buf) cudaFreeAsync(m.buf, c->tstream);
          c->geo32.clear();
          return MB_E_NOMEM;
        }
        keep.push_back({src[q], dst[q], n[q]});
        if (to_float(src[q], dst[q], n[q], c->tstream) != cudaSuccess) {
          c->geo32 = keep;  // every buffer stays owned by the context
          for (auto& m : pool)
            if (m.buf) c->geo32.push_back(m);
          return MB_E_CUDA;
        }
      }
      d.fm1f = dst[0]; d.fm2f = dst[1]; d.fm3f = dst[2]; d.dlf = dst[3]; d.mf = dst[4];
    }
    for (auto& m : pool)
      if (m.buf) cudaFreeAsync(m.buf, c->tstream);
    c->geo32 = keep;
  }
  free_tables(c);
  if ((rc = upload(&c->d_blk, hb.data(), hb.size(), c->tstream)) != MB_OK) return rc;
  if ((rc = upload(&c->d_recmap, recmap.data(), recmap.size(), c->tstream)) != MB_OK) return rc;
  if ((rc = upload(&c->d_rec, hr.data(), hr.size(), c->tstream)) != MB_OK) return rc;
  c->hrec.assign(mesh->rec, mesh->rec + mesh->nrec);
  c->hdrec = hr;
  if ((rc = upload(&c->d_grec, hg.data(), hg.size(), c->tstream)) != MB_OK) return rc;
  // Ghost passes in two halves where the record order changes values. The extrapolating ghosts of a face (walls in
  // the first pass, type 11 in the second) read the opposite face's ghost layers when the axis has at most two
  // cells, so of two records on opposite faces of one column the later one in record order must see the earlier
  // one's ghosts (the reference fills them in one sequential record loop). Every record goes into the first half
  // unless its opposite partner on the same column comes earlier in record order; only pairs interact, so two
  // launches per pass reproduce the sequential order exactly. An axis of one cell with type 11 on both faces is
  // order-free (every ghost equals the cell), as are axes of three or more cells.
  int ordered = 0;
  std::vector<char> late_phys(mesh->nrec, 0), late_cubic(mesh->nrec, 0);
  {
    std::vector<int> ax11(3 * (size_t)mesh->nblk, 1);
    for (int q = 0; q < mesh->nrec; ++q)
      if (mesh->rec[q].type != MB_BC_EXTRAPOLATION) ax11[3 * mesh->rec[q].blk + (mesh->rec[q].face - 1) / 2] = 0;
    for (int q = 0; q < mesh->nrec; ++q) {
      const mb_bc& r = mesh->rec[q];
      const int ax = (r.face - 1) / 2, nax = mesh->blk[r.blk].n[ax];
      if (r.type != MB_BC_EXTRAPOLATION && r.type != MB_BC_WALL && r.type != MB_BC_WALL_T) continue;
      if (nax == 2 || (nax == 1 && !ax11[3 * r.blk + ax])) ordered = 1;
    }
    if (ordered) {
      std::unordered_map<unsigned long long, int> seen_phys, seen_cubic;  // column -> face of its first record
      for (int q = 0; q < mesh->nrec; ++q) {
        const mb_bc& r = mesh->rec[q];
        if (!phys_type(r.type)) continue;
        const int ax = (r.face - 1) / 2;
        const int t1 = ax == 0 ? r.j : r.i, t2 = ax == 2 ? r.j : r.k;
        const unsigned long long key = ((unsigned long long)(3 * (unsigned long long)r.blk + ax) << 40) |
                                       ((unsigned long long)(unsigned)t1 << 20) | (unsigned long long)(unsigned)t2;
        auto mark = [&](std::unordered_map<unsigned long long, int>& seen, std::vector<char>& late) {
          auto it = seen.find(key);
          if (it == seen.end()) seen.emplace(key, r.face);
          else if (it->second != r.face) late[q] = 1;
        };
        mark(seen_phys, late_phys);
        if (r.type == MB_BC_EXTRAPOLATION) mark(seen_cubic, late_cubic);
      }
    }
  }
  auto split = [&](std::vector<int>& v, const std::vector<char>& late, int* off) {
    std::stable_partition(v.begin(), v.end(), [&](int e) { return !late[e & 0x0fffffff]; });
    off[0] = 0; off[2] = (int)v.size(); off[1] = 0;
    for (int e : v) off[1] += !late[e & 0x0fffffff];
  };
  int po[3], co[3], pof[3], cof[3];
  split(phys, late_phys, po);
  split(cubic, late_cubic, co);
  split(physf, late_phys, pof);
  split(cubicf, late_cubic, cof);
  if ((rc = upload(&c->d_phys, phys.data(), phys.size(), c->tstream)) != MB_OK) return rc;
  if ((rc = upload(&c->d_cubic, cubic.data(), cubic.size(), c->tstream)) != MB_OK) return rc;
  if ((rc = upload(&c->d_physf, physf.data(), physf.size(), c->tstream)) != MB_OK) return rc;
  if ((rc = upload(&c->d_cubicf, cubicf.data(), cubicf.size(), c->tstream)) != MB_OK) return rc;
  if ((rc = upload(&c->d_cdst, cdst.data(), cdst.size(), c->tstream)) != MB_OK) return rc;
  if ((rc = upload(&c->d_csrc, csrc.data(), csrc.size(), c->tstream)) != MB_OK) return rc;
  if ((rc = upload(&c->d_pgsrc, pgsrc.data(), pgsrc.size(), c->tstream)) != MB_OK) return rc;
  if ((rc = upload(&c->d_tiles_sweep, ts.data(), ts.size(), c->tstream)) != MB_OK) return rc;
  if ((rc = upload(&c->d_tiles_aux, ta.data(), ta.size(), c->tstream)) != MB_OK) return rc;
  if ((rc = upload(&c->d_tiles_km, tk.data(), tk.size(), c->tstream)) != MB_OK) return rc;
  c->ntiles_km = (int)tk.size();
  if ((rc = upload(&c->d_brec, brec.data(), brec.size(), c->tstream)) != MB_OK) return rc;
  if ((rc = upload(&c->d_bcell, bcell.data(), bcell.size(), c->tstream)) != MB_OK) return rc;
  c->nrec = (int)brec.size();
  if (mesh->nrec > 0 &&
      cudaMallocAsync((void**)&c->d_recflux, (size_t)mesh->nrec * 2 * MB_NPRIM * sizeof(double), c->tstream) !=
          cudaSuccess)
    return MB_E_NOMEM;
  c->ntiles_sweep = (int)ts.size();
  c->ntiles_aux = (int)ta.size();
  Params& p = c->p;
  p.blk = c->d_blk; p.rec_map = c->d_recmap; p.rec = c->d_rec; p.pgsrc = c->d_pgsrc;
  p.recflux = c->d_recflux;
  GhostLists& g = c->g;
  g.rec = c->d_grec; g.phys = c->d_phys; g.nphys = (int)phys.size(); g.cubic = c->d_cubic; g.ncubic = (int)cubic.size();
  g.cdst = c->d_cdst; g.csrc = c->d_csrc; g.ncopy = (int)cdst.size(); g.pgsrc = c->d_pgsrc; g.nconn = mesh->nconn;
  g.ordered = ordered;
  for (int f = 0; f < 3; ++f) { g.phys_off[f] = po[f]; g.cubic_off[f] = co[f]; }
  c->gf = g;
  c->gf.phys = c->d_physf; c->gf.nphys = (int)physf.size(); c->gf.cubic = c->d_cubicf; c->gf.ncubic = (int)cubicf.size();
  for (int f = 0; f < 3; ++f) { c->gf.phys_off[f] = pof[f]; c->gf.cubic_off[f] = cof[f]; }
  // ---- residual smoothing: the first ghost layer of the faces of each direction (Ghost_Residual_Extrapolation,
  // Lib_IRS.f90:119-177): every face cell's ghost from the cell itself, a connection record's from its donor face
  // cell instead; blocks of a case with fewer directions are left out
  if (sc->irs > 0) {
    std::vector<long long> idst, isrc;
    for (int d = 1; d <= 3; ++d) {
      c->irs_off[d - 1] = (int)idst.size();
      std::vector<size_t> fbase(2 * (size_t)mesh->nblk, 0);  // first entry of (block, side) in this direction
      for (int b = 0; b < mesh->nblk; ++b) {
        const DBlk& q = hb[b];
        if (q.ndir < d) continue;
        const int n[3] = {q.n1, q.n2, q.n3};
        const int a = (d == 1) ? 1 : 0, bb = (d == 3) ? 1 : 2;  // the two transverse axes
        for (int side = 0; side < 2; ++side) {
          fbase[2 * b + side] = idst.size();
          for (int v = 1; v <= n[bb]; ++v)
            for (int u = 1; u <= n[a]; ++u) {
              int cc[3];
              cc[d - 1] = side ? n[d - 1] : 1;
              cc[a] = u; cc[bb] = v;
              int gg[3] = {cc[0], cc[1], cc[2]};
              gg[d - 1] += side ? 1 : -1;
              idst.push_back(row(q, gg[0], gg[1], gg[2]));
              isrc.push_back(row(q, cc[0], cc[1], cc[2]));
            }
        }
      }
      for (int e = 0; e < mesh->nconn; ++e) {
        const mb_conn& cn = mesh->conn[e];
        const mb_bc& r = mesh->rec[cn.rec];
        if ((r.face + 1) / 2 != d || hb[r.blk].ndir < d) continue;
        const DBlk& q = hb[r.blk];
        const int n[3] = {q.n1, q.n2, q.n3};
        const int a = (d == 1) ? 1 : 0, bb = (d == 3) ? 1 : 2;
        const int cc[3] = {r.i, r.j, r.k};
        const size_t pos = fbase[2 * r.blk + ((r.face & 1) ? 0 : 1)] + (size_t)(cc[a] - 1) +
                           (size_t)(cc[bb] - 1) * n[a];
        isrc[pos] = row(hb[cn.bs], cn.is, cn.js, cn.ks);
      }
    }
    c->irs_off[3] = (int)idst.size();
    if ((rc = upload(&c->d_idst, idst.data(), idst.size(), c->tstream)) != MB_OK) return rc;
    if ((rc = upload(&c->d_isrc, isrc.data(), isrc.size(), c->tstream)) != MB_OK) return rc;
  }
  return MB_OK;
}

int mb_init(const mb_mesh* mesh, const mb_scheme* sc, const mb_thermo* th, int device, mb_ctx** out) {
  if (!mesh || !sc || !th || !out) return MB_E_ARG;
  *out = nullptr;
  if (sc->riemann < MB_RS_HLLC || sc->riemann > MB_RS_HLLC_PC) return MB_E_UNSUPPORTED;
  if (sc->sensor < 0 || sc->sensor > 3) return MB_E_UNSUPPORTED;
  if (sc->intvar < 0 || sc->intvar > 2 || (sc->intvar >= 1 && sc->n_rk == 4)) return MB_E_UNSUPPORTED;
  // HLLC-PC only with preconditioning (Assign_RS, Lib_Riemann.f90:88-89), preconditioning only for steady runs
  // (IO_Ini_Open.f90:125-127)
  if ((sc->riemann == MB_RS_HLLC_PC) != (sc->intvar == 2) || (sc->intvar == 2 && sc->local_dt != 1))
    return MB_E_UNSUPPORTED;
  if (sc->intvar == 2 && !(sc->prec_eps_min > 0.0 && sc->prec_eps_min < 1.0 && sc->prec_smooth >= 0)) return MB_E_ARG;
  if (sc->irs < 0 || sc->irs > 4 || (sc->irs > 0 && sc->n_rk == 4)) return MB_E_UNSUPPORTED;
  if (sc->irs > 0 && !(sc->irs_beta >= 0.0 && std::isfinite(sc->irs_beta))) return MB_E_ARG;
  if (sc->local_dt < 0 || sc->local_dt > 1 || sc->cfl_rise < 0) return MB_E_ARG;
  if (sc->limiter < 1 || sc->limiter > 6) return MB_E_UNSUPPORTED;
  if (sc->n_rk < 1 || sc->n_rk > 4) return MB_E_UNSUPPORTED;
  if (!(sc->res_stop >= 0.0)) return MB_E_ARG;
  if (sc->precision != MB_PREC_FP64 && sc->precision != MB_PREC_MIXED && sc->precision != MB_PREC_FP64_FAST)
    return MB_E_UNSUPPORTED;
  if (sc->ndir < 1 || sc->ndir > 3) return MB_E_ARG;
  if (th->tmax - th->tmin < 2 || !th->cp || !th->h || !th->mu || !th->k) return MB_E_ARG;
  const int ngroups = mesh->ngroups > 0 ? mesh->ngroups : 1;
  int rc = check_mesh(mesh, ngroups);
  if (rc != MB_OK) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return MB_E_NODEV;
  if (device < 0 || device >= ndev) return MB_E_ARG;
  CK(cudaSetDevice(device));
  mb_ctx* c = new mb_ctx();
  c->device = device;
  c->sc = *sc;
  c->ncell = mesh->ncell_total;
  c->ngroups = ngroups;
  c->ty_sweep = sc->precision == MB_PREC_MIXED ? TY_F32 : TY_F64;
  c->no_tma = getenv("MB_NO_TMA") != nullptr;
#define TRY(x)                 \
  do {                         \
    rc = (x);                  \
    if (rc != MB_OK) {         \
      free_ctx(c);             \
      return rc;               \
    }                          \
  } while (0)
  // ---- thermo tables (FP64 and FP32 copies)
  const int nt = th->tmax - th->tmin + 1;
  std::vector<double> tab(4 * (size_t)nt);
  std::vector<float> tabf(4 * (size_t)nt);
  for (int q = 0; q < nt; ++q) {
    tab[q] = th->cp[q]; tab[nt + q] = th->h[q]; tab[2 * nt + q] = th->mu[q]; tab[3 * nt + q] = th->k[q];
  }
  for (size_t q = 0; q < tab.size(); ++q) tabf[q] = (float)tab[q];
  TRY(upload(&c->d_tab, tab.data(), tab.size()));
  TRY(upload(&c->d_tabf, tabf.data(), tabf.size()));
  // ---- one clock per case; every case starts with the scheme's stop rule
  if (cudaMalloc((void**)&c->d_st, ngroups * sizeof(DevState)) != cudaSuccess) { free_ctx(c); return MB_E_NOMEM; }
  {
    std::vector<DevState> hs(ngroups);
    for (auto& h : hs) {
      memset(&h, 0, sizeof(h));
      double big = 1e300;
      memcpy(&h.dtmin_bits, &big, sizeof(double));
      h.time_clip = sc->time_clip;
      h.t_end = sc->time_clip ? sc->time_threshold : 0.0;
      h.res_stop = sc->res_stop;
      h.rampf = (1 < sc->cfl_rise) ? 1.0 / sc->cfl_rise : 1.0;  // the factor of step 1
    }
    if (cudaMemcpy(c->d_st, hs.data(), ngroups * sizeof(DevState), cudaMemcpyHostToDevice) != cudaSuccess) {
      free_ctx(c);
      return MB_E_CUDA;
    }
  }
  // ---- the engine's stage buffer (and the RK4 accumulator) over the whole arena
  if (cudaMalloc((void**)&c->d_scratch, (size_t)c->ncell * MB_NPRIM * sizeof(double)) != cudaSuccess) {
    free_ctx(c);
    return MB_E_NOMEM;
  }
  if (cudaMemset(c->d_scratch, 0, (size_t)c->ncell * MB_NPRIM * sizeof(double)) != cudaSuccess) { free_ctx(c); return MB_E_CUDA; }
  if (sc->intvar == 2) {
    const size_t nb = (size_t)c->ncell * sizeof(double);
    double** bufs[3] = {&c->d_ur, &c->d_urb, &c->d_dtl};
    for (double** q : bufs) {
      if (cudaMalloc((void**)q, nb) != cudaSuccess) { free_ctx(c); return MB_E_NOMEM; }
      if (cudaMemset(*q, 0, nb) != cudaSuccess) { free_ctx(c); return MB_E_CUDA; }
    }
  }
  if (sc->irs > 0) {
    const size_t nb = 2 * (size_t)c->ncell * MB_NPRIM * sizeof(double);
    if (cudaMalloc((void**)&c->d_irs, nb) != cudaSuccess) { free_ctx(c); return MB_E_NOMEM; }
    if (cudaMemset(c->d_irs, 0, nb) != cudaSuccess) { free_ctx(c); return MB_E_CUDA; }
  }
  if (sc->n_rk == 4) {
    if (cudaMalloc((void**)&c->d_acc4, (size_t)c->ncell * MB_NPRIM * sizeof(double)) != cudaSuccess) {
      free_ctx(c);
      return MB_E_NOMEM;
    }
    if (cudaMemset(c->d_acc4, 0, (size_t)c->ncell * MB_NPRIM * sizeof(double)) != cudaSuccess) { free_ctx(c); return MB_E_CUDA; }
  }
  {
    cudaError_t e = MB_BY_FORM(sc->precision, sweep_unit(sc), _setup, ());
    if (e != cudaSuccess) { free_ctx(c); return MB_E_CUDA; }
  }
  // ---- kernel parameters
  Params& p = c->p;
  memset(&p, 0, sizeof(p));
  p.cp = c->d_tab - th->tmin; p.h = c->d_tab + nt - th->tmin; p.mu = c->d_tab + 2 * nt - th->tmin; p.k = c->d_tab + 3 * nt - th->tmin;
  p.cpf = c->d_tabf - th->tmin; p.hf = c->d_tabf + nt - th->tmin; p.muf = c->d_tabf + 2 * nt - th->tmin; p.kf = c->d_tabf + 3 * nt - th->tmin;
  p.st = c->d_st;
  p.ngroups = ngroups;
  p.nc = c->ncell;
  p.tmin = th->tmin; p.tmax = th->tmax;
  p.wm = th->wm; p.ri = RUNIV / th->wm; p.iri = th->wm / RUNIV;
  p.sd = mb_effective_sensor(sc->riemann, sc->sensor);
  p.intvar = sc->intvar;
  p.local_dt = sc->local_dt;
  p.cfl_rise = sc->cfl_rise;
  p.prec = sc->intvar == 2 ? 1 : 0;
  p.ur = c->d_ur;
  p.dtl = c->d_dtl;
  p.prec_eps_min = sc->prec_eps_min; p.prec_uref = sc->prec_uref; p.prec_mach = sc->prec_mach;
  p.prec_ur_factor = sc->prec_ur_factor; p.prec_ur_min = sc->prec_ur_min;
  p.lim = sc->limiter; p.rs = sc->riemann; p.visc = sc->visc ? 1 : 0; p.ndir = sc->ndir; p.dt_additive = sc->dt_additive;
  p.guard = sc->visc ? 1 : 0; p.state_check = sc->state_check;
  p.cfl = sc->cfl; p.vnn = sc->vnn; p.prandtl = sc->prandtl; p.schmidt = sc->schmidt; p.mco = sc->mco;
  p.n_rk = sc->n_rk; p.irk = 0; p.acc4 = c->d_acc4;
  if (cudaMalloc((void**)&c->d_queue, sizeof(int)) != cudaSuccess) { free_ctx(c); return MB_E_NOMEM; }
  {
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    const int v = sc->visc ? 1 : 0;
    int occ = MB_BY_FORM(sc->precision, sweep_unit(sc), _occupancy, (v));
    p.pgrid = std::max(1, occ) * std::max(1, nsm);
    int occ_km = MB_BY_FORM(sc->precision, sweep_unit(sc), _occupancy_km, (v));
    p.pgrid_km = std::max(1, occ_km) * std::max(1, nsm);
  }
  p.queue = nullptr;
  // ---- the mesh tables
  TRY(build_tables(c, mesh));
  if (getenv("MB_REPORT")) {
    const int v = sc->visc ? 1 : 0;
    int occ = MB_BY_FORM(sc->precision, sweep_unit(sc), _occupancy, (v));
    int occ_km = MB_BY_FORM(sc->precision, sweep_unit(sc), _occupancy_km, (v));
    fprintf(stderr, "[mose_b200] sweep: %s, %d threads per CTA, %d CTAs per SM (%d for one-plane blocks), %d + %d tiles\n",
            sc->precision == MB_PREC_MIXED ? "mixed" : (sc->precision == MB_PREC_FP64_FAST ? "fp64 fast" : "fp64"),
            32 * c->ty_sweep, occ, occ_km, c->ntiles_sweep, c->ntiles_km);
  }
#undef TRY
  CK(cudaStreamSynchronize(0));  // the tables were built in the order of the legacy stream: ready for any stream
  *out = c;
  return MB_OK;
}

static int reconfigure(mb_ctx* ctx, const mb_mesh* mesh, cudaStream_t s, bool device_sync) {
  if (!ctx || !mesh) return MB_E_ARG;
  if (mesh->ncell_total > ctx->ncell) return MB_E_ARG;
  const int ng = mesh->ngroups > 0 ? mesh->ngroups : 1;
  if (ng > ctx->ngroups) return MB_E_ARG;
  int rc = check_mesh(mesh, ctx->ngroups);
  if (rc != MB_OK) return rc;
  CK(cudaSetDevice(ctx->device));
  if (device_sync) CK(cudaDeviceSynchronize());  // the old tables may still be read by queued work on any stream
  // a step graph in flight is freed when it completes; the next mb_step captures one over the new tables
  if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
  if (ctx->graph) { cudaGraphDestroy(ctx->graph); ctx->graph = nullptr; }
  ctx->gP = nullptr;
  ctx->gPO = nullptr;
  ctx->tstream = s;
  rc = build_tables(ctx, mesh);
  ctx->tstream = 0;
  if (device_sync) CK(cudaStreamSynchronize(s));
  return rc;
}

int mb_reconfigure(mb_ctx* ctx, const mb_mesh* mesh) { return reconfigure(ctx, mesh, 0, true); }

int mb_reconfigure_async(mb_ctx* ctx, const mb_mesh* mesh, void* stream) {
  return reconfigure(ctx, mesh, (cudaStream_t)stream, false);
}

int mb_set_record_params(mb_ctx* ctx, int rec, const double* q, void* stream) {
  if (!ctx || !q || rec < 0 || rec >= (int)ctx->hrec.size()) return MB_E_ARG;
  mb_bc r = ctx->hrec[rec];
  for (int s = 0; s < MB_BC_NQ; ++s) r.q[s] = q[s];
  int rc = check_record_params(r);
  if (rc != MB_OK) return rc;
  CK(cudaSetDevice(ctx->device));
  ctx->hrec[rec] = r;
  fill_drec(r, &ctx->hdrec[rec]);
  CK(cudaMemcpyAsync(ctx->d_rec + rec, &ctx->hdrec[rec], sizeof(DRec), cudaMemcpyHostToDevice,
                     (cudaStream_t)stream));
  return MB_OK;
}

int mb_group_reset(mb_ctx* ctx, int g, const mb_group* spec, const double* P, void* stream) {
  if (!ctx || !spec || !P || g < 0 || g >= ctx->ngroups || spec->t_end < 0.0 || spec->res_stop < 0.0) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  CK(group_reset(ctx->p, g, spec->time_clip, spec->t_end, spec->res_stop, s));
  CK(ctx->sc.precision == MB_PREC_MIXED       ? sweep_f32_rs1_dt(ctx->p, ctx->d_tiles_aux, ctx->ntiles_aux, P, g, s)
     : ctx->sc.precision == MB_PREC_FP64_FAST ? sweep_f64f_rs1_dt(ctx->p, ctx->d_tiles_aux, ctx->ntiles_aux, P, g, s)
                                              : dt_cells(ctx->p, ctx->d_tiles_aux, ctx->ntiles_aux, P, s, g));
  ctx->launches += 2;
  return MB_OK;
}

static void to_status(const DevState& h, int state_check, mb_status* st) {
  memset(st, 0, sizeof(*st));
  st->n_bad_state = h.n_bad_state;
  st->n_bad_thermo = h.n_bad_thermo;
  st->bad_blk = h.bad_blk; st->bad_i = h.bad_i; st->bad_j = h.bad_j; st->bad_k = h.bad_k;
  st->steps = h.steps;
  st->time = h.time;
  st->dt = h.dt;
  st->done = h.done;
  for (int v = 0; v < MB_NPRIM; ++v) st->res[v] = sqrt(h.res2[v]);
  st->code = MB_OK;
  if (h.code == MB_E_TIMEOUT) st->code = MB_E_TIMEOUT;  // a bounded wait of the sweep's TMA staging gave up
  else if (h.n_bad_thermo > 0) st->code = MB_E_THERMO;
  else if (h.n_bad_state > 0 && state_check) st->code = MB_E_STATE;
}

int mb_read_group_status(mb_ctx* ctx, int g0, int n, mb_status* out, void* stream) {
  if (!ctx || !out || g0 < 0 || n < 1 || g0 + n > ctx->ngroups) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<DevState> h(n);
  CK(cudaMemcpyAsync(h.data(), ctx->d_st + g0, n * sizeof(DevState), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (int q = 0; q < n; ++q) to_status(h[q], ctx->sc.state_check, out + q);
  return MB_OK;
}

int mb_get_group_status(mb_ctx* ctx, int g0, int n, mb_status* out) {
  if (!ctx || !out || g0 < 0 || n < 1 || g0 + n > ctx->ngroups) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaDeviceSynchronize());
  std::vector<DevState> h(n);
  CK(cudaMemcpy(h.data(), ctx->d_st + g0, n * sizeof(DevState), cudaMemcpyDeviceToHost));
  for (int q = 0; q < n; ++q) to_status(h[q], ctx->sc.state_check, out + q);
  return MB_OK;
}

void mb_destroy(mb_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  free_ctx(ctx);
}

// ---- TMA staging of the mixed sweep: the state buffer P viewed as a 2-D tensor of ncell rows x 5 FP64 variables
// (var-last, the variable stride ncell x 8 bytes), boxes of 38 rows x 5 variables (one staged j-row of a tile plane)
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)f;
  }
  return fn;
}

// the tensor map of P for the current row count, or null: the form does not stage by TMA, P is not 16-byte aligned,
// ncell is odd (the variable stride must be a multiple of 16 bytes), or (create) the stream is capturing and the map
// does not exist yet. Without a map the sweep stages with plain loads; both paths give the same tile values.
static const void* tmap_of(mb_ctx* c, const double* P, cudaStream_t s, bool create) {
  if (c->sc.precision != MB_PREC_MIXED || !P || c->no_tma) return nullptr;
  for (const auto& m : c->tmaps)
    if (m.ptr == P && m.nc == c->ncell) return m.dev;
  if (!create || ((uintptr_t)P & 15u) || (c->ncell & 1) || c->tmaps.size() >= 64) return nullptr;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return nullptr;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
  if (!enc) return nullptr;
  CUtensorMap m;
  cuuint64_t dims[2] = {(cuuint64_t)c->ncell, (cuuint64_t)MB_NPRIM};
  cuuint64_t strides[1] = {(cuuint64_t)c->ncell * sizeof(double)};
  cuuint32_t box[2] = {(cuuint32_t)TMA_BOX_ROWS, (cuuint32_t)MB_NPRIM};
  cuuint32_t es[2] = {1, 1};
  if (enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void*)P, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
      CUDA_SUCCESS)
    return nullptr;
  void* d = nullptr;
  if (cudaMalloc(&d, sizeof(CUtensorMap)) != cudaSuccess) return nullptr;
  if (cudaMemcpyAsync(d, &m, sizeof(CUtensorMap), cudaMemcpyHostToDevice, s) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  c->tmaps.push_back({P, c->ncell, d});
  return d;
}

// the maps of the buffers a stage or step may read (before any capture)
static void prepare_tmaps(mb_ctx* c, const double* P, const double* PO, cudaStream_t s) {
  tmap_of(c, P, s, true);
  tmap_of(c, PO, s, true);
  tmap_of(c, c->d_scratch, s, true);
}

static int sweep_on(mb_ctx* c, const DTile* t, int n, int persistent, int mode, const double* Pin,
                    const double* Pold, double* Pout, double* Rout, int irk, int last, cudaStream_t s, int km = 0) {
  if (n <= 0) return MB_OK;
  Params p = c->p;
  p.irk = irk;
  p.queue = persistent ? c->d_queue : nullptr;
  p.stg = (c->sc.precision == MB_PREC_MIXED && (km ? c->stage_tma_km : c->stage_tma)) ? STG_TMA : STG_PLAIN;
  p.tmap = p.stg == STG_TMA ? tmap_of(c, Pin, s, false) : nullptr;
  if (c->sc.precision == MB_PREC_MIXED) (p.tmap ? c->sweeps_tma : c->sweeps_plain) += 1;
  const double rkc = irk > 0 ? rkc_of(c->sc.n_rk, irk) : 0.0;
  cudaError_t e;
  e = MB_BY_FORM(c->sc.precision, sweep_unit(&c->sc), , (p, t, n, mode, Pin, Pold, Pout, Rout, rkc, last, km, s));
  c->launches += 1;
  CK(e);
  return MB_OK;
}

// the boundary records of the stage input (BC_Fluxes), before the sweep that adds them
static int records(mb_ctx* c, const double* Pin, cudaStream_t s) {
  if (c->nrec <= 0) return MB_OK;
  const Params& p = c->p;
  cudaError_t e;
  e = MB_BY_FORM(c->sc.precision, sweep_unit(&c->sc), _records, (p, c->d_brec, c->d_bcell, c->nrec, Pin, s));
  c->launches += 1;
  CK(e);
  return MB_OK;
}

static int sweep(mb_ctx* c, int mode, const double* Pin, const double* Pold, double* Pout, double* Rout, int irk,
                 int last, cudaStream_t s) {
  int rc = sweep_on(c, c->d_tiles_sweep, c->ntiles_sweep, c->persistent, mode, Pin, Pold, Pout, Rout, irk, last, s);
  if (rc == MB_OK)
    rc = sweep_on(c, c->d_tiles_km, c->ntiles_km, c->persistent_km, mode, Pin, Pold, Pout, Rout, irk, last, s, 1);
  return rc;
}

// average device time of nrep sweeps (MODE_UPDATE of stage 1 from P into the stage buffer, no dt) over a tile
// list, after one untimed sweep; the state P and the clocks are not changed
static int time_sweep(mb_ctx* c, const std::vector<DTile>& tl, int persistent, const double* P, int nrep,
                      cudaStream_t s, float* ms, int km = 0) {
  DTile* d = nullptr;
  int rc = upload(&d, tl.data(), tl.size());
  if (rc != MB_OK) return rc;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  rc = records(c, P, s);
  if (rc == MB_OK)
    rc = sweep_on(c, d, (int)tl.size(), persistent, MODE_UPDATE, P, P, c->d_scratch, nullptr, 1, 0, s, km);
  cudaEventRecord(e0, s);
  for (int q = 0; q < nrep && rc == MB_OK; ++q)
    rc = sweep_on(c, d, (int)tl.size(), persistent, MODE_UPDATE, P, P, c->d_scratch, nullptr, 1, 0, s, km);
  cudaEventRecord(e1, s);
  cudaEventSynchronize(e1);
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  *ms = t / nrep;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamSynchronize(s);
  cudaFree(d);
  return rc;
}

static int fill(mb_ctx* c, double* P, cudaStream_t s, bool fused = true) {
  int nl = 0;
  cudaError_t e = ghost_fill(c->p, fused ? c->gf : c->g, P, s, &nl);
  c->launches += nl;
  CK(e);
  return MB_OK;
}

// IRS_apply (Lib_IRS.f90:57-105) on R, the first of the engine's two residual buffers: on the conservative path the
// scaling -R / vol * dt (dt < 0: each case's clock dt), then per direction the first ghost layer and the Jacobi
// sweeps, alternating between the two buffers; *out receives the buffer that holds the result
static int smooth_residual(mb_ctx* c, double* R, double dt, const double* Pold, cudaStream_t s, const double** out) {
  double* cur = R;
  double* alt = (cur == c->d_irs) ? c->d_irs + (size_t)c->ncell * MB_NPRIM : c->d_irs;
  if (c->sc.intvar == 0) {
    CK(irs_scale(c->p, c->d_tiles_aux, c->ntiles_aux, cur, dt, Pold, s));
    c->launches += 1;
  }
  for (int d = 1; d <= 3; ++d) {
    const int n = c->irs_off[d] - c->irs_off[d - 1];
    if (n <= 0) continue;  // no block of the mesh has this direction
    CK(irs_ghosts(c->p, c->d_idst + c->irs_off[d - 1], c->d_isrc + c->irs_off[d - 1], n, cur, s));
    CK(irs_smooth(c->p, c->d_tiles_aux, c->ntiles_aux, cur, alt, d, c->sc.irs, c->sc.irs_beta, s));
    c->launches += 2;
    std::swap(cur, alt);
  }
  *out = cur;
  return MB_OK;
}

// prec: Ur of the state P (Update_Derived_Variables). Every entry point that reads Ur computes it from the state it is
// given, and the time loop from each stage's input: the reference refreshes it after every update, so it is always the
// Ur of the current state
static int ur_pass(mb_ctx* c, const double* P, cudaStream_t s) {
  if (!c->p.prec) return MB_OK;
  int nl = 0;
  CK(prec_ur(c->p, c->d_tiles_aux, c->ntiles_aux, P, c->d_ur, c->d_urb, c->sc.prec_smooth, s, &nl));
  c->launches += nl;
  return MB_OK;
}

int mb_fill_ghosts(mb_ctx* ctx, double* P, void* stream) {
  if (!ctx || !P) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  return fill(ctx, P, (cudaStream_t)stream, false);
}

int mb_residual(mb_ctx* ctx, const double* P, double* R, void* stream) {
  if (!ctx || !P || !R) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  tmap_of(ctx, P, (cudaStream_t)stream, true);
  int rc = ur_pass(ctx, P, (cudaStream_t)stream);
  if (rc != MB_OK) return rc;
  rc = records(ctx, P, (cudaStream_t)stream);
  if (rc != MB_OK) return rc;
  return sweep(ctx, MODE_RESIDUAL, P, nullptr, nullptr, R, 0, 0, (cudaStream_t)stream);
}

int mb_update(mb_ctx* ctx, double* P, const double* PO, const double* R, int irk, double dt, void* stream) {
  if (!ctx || !P || !PO || !R || irk < 1 || irk > ctx->sc.n_rk) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  Params p = ctx->p;
  p.irk = irk;
  cudaStream_t s = (cudaStream_t)stream;
  int prescaled = 0;
  if (p.prec) {  // Ur of the stage input, then each cell's local step from PO (not reduced into the clock)
    int rc = ur_pass(ctx, P, s);
    if (rc != MB_OK) return rc;
    CK(prec_dt(p, ctx->d_tiles_aux, ctx->ntiles_aux, PO, ctx->d_dtl, 0, s));
    ctx->launches += 1;
  }
  if (ctx->sc.irs > 0) {  // IRS_apply on the engine's copy of R, then the update takes the smoothed residual
    double* R0 = ctx->d_irs;
    CK(cudaMemcpyAsync(R0, R, (size_t)ctx->ncell * MB_NPRIM * sizeof(double), cudaMemcpyDeviceToDevice, s));
    int rc = smooth_residual(ctx, R0, dt, PO, s, &R);
    if (rc != MB_OK) return rc;
    prescaled = ctx->sc.intvar == 0;
  }
  cudaError_t e = update_cells(p, ctx->d_tiles_aux, ctx->ntiles_aux, P, PO, R, rkc_of(ctx->sc.n_rk, irk), dt, s,
                               prescaled);
  ctx->launches += 1;
  CK(e);
  return MB_OK;
}

static int dt_min(mb_ctx* c, const double* P, cudaStream_t s) {
  if (c->p.prec) {  // Ur of P, then the preconditioned local steps of the step into dtl and their minimum
    int rc = ur_pass(c, P, s);
    if (rc != MB_OK) return rc;
    CK(reset_dt(c->p, s));
    CK(prec_dt(c->p, c->d_tiles_aux, c->ntiles_aux, P, c->d_dtl, 1, s));
    c->launches += 2;
    return MB_OK;
  }
  CK(reset_dt(c->p, s));
  CK(c->sc.precision == MB_PREC_MIXED       ? sweep_f32_rs1_dt(c->p, c->d_tiles_aux, c->ntiles_aux, P, -1, s)
     : c->sc.precision == MB_PREC_FP64_FAST ? sweep_f64f_rs1_dt(c->p, c->d_tiles_aux, c->ntiles_aux, P, -1, s)
                                            : dt_cells(c->p, c->d_tiles_aux, c->ntiles_aux, P, s));
  c->launches += 2;
  return MB_OK;
}

int mb_dt(mb_ctx* ctx, const double* P, double* dt_host, void* stream) {
  if (!ctx || !P || !dt_host) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  int rc = dt_min(ctx, P, s);
  if (rc != MB_OK) return rc;
  unsigned long long bits;
  int steps = 0;
  CK(cudaMemcpyAsync(&bits, &ctx->d_st->dtmin_bits, sizeof(bits), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&steps, &ctx->d_st->steps, sizeof(steps), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  double dm;
  memcpy(&dm, &bits, sizeof(dm));
  const int iter = steps + 1;  // the ramp factor of the case's next step (cfl-rise-threshold)
  const double f = (iter < ctx->sc.cfl_rise) ? (double)iter / ctx->sc.cfl_rise : 1.0;
  *dt_host = std::min(dm * f, 1e5);
  ctx->dt_valid = true;  // the device minimum now belongs to P
  return MB_OK;
}

int mb_begin_step(mb_ctx* ctx, const double* P, void* stream) {
  if (!ctx || !P) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  int rc = dt_min(ctx, P, s);
  if (rc != MB_OK) return rc;
  CK(clock_step(ctx->p, s));
  ctx->launches += 1;
  return MB_OK;
}

// ---- the step start and the stage split into its exchange points, for a host that partitions the blocks over
// several GPUs (one context per GPU, external blocks holding the halo copies; mosegpu/partition.py): the minimum
// local step of each rank is all-reduced (MIN) between mb_step_prepare and mb_step_start, and the halo rows are
// exchanged before mb_stage_begin (the donor cells the ghost copies read) and between mb_stage_begin and
// mb_stage_end (the donor ghost cells the viscous connection records read after the donors' own ghost fill)
int mb_step_prepare(mb_ctx* ctx, const double* P, void* stream) {
  if (!ctx || !P) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  if (ctx->dt_valid) return MB_OK;  // the last stage of the previous step left the minimum of P in the clocks
  int rc = dt_min(ctx, P, (cudaStream_t)stream);
  if (rc == MB_OK) ctx->dt_valid = true;
  return rc;
}

int mb_copy_dtmin(mb_ctx* ctx, int g, void* buf, int to_clock, void* stream) {
  if (!ctx || !buf || g < 0 || g >= ctx->ngroups) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  void* clk = (void*)&ctx->d_st[g].dtmin_bits;
  CK(cudaMemcpyAsync(to_clock ? clk : buf, to_clock ? buf : clk, sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                     (cudaStream_t)stream));
  return MB_OK;
}

int mb_step_start(mb_ctx* ctx, void* stream) {
  if (!ctx) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(clock_step(ctx->p, (cudaStream_t)stream));
  ctx->launches += 1;
  return MB_OK;
}

// the stage's computation after its ghost fill and boundary records: the fused sweep, or with residual smoothing the
// sweep's residual, IRS_apply and the update on the smoothed residual (old state in P)
static int stage_compute(mb_ctx* c, const double* in, const double* P, double* outp, int irk, int last,
                         cudaStream_t s) {
  if (c->sc.irs <= 0) return sweep(c, MODE_UPDATE, in, P, outp, nullptr, irk, last, s);
  int rc = sweep(c, MODE_RESIDUAL, in, nullptr, nullptr, c->d_irs, irk, 0, s);
  if (rc != MB_OK) return rc;
  const double* R = nullptr;
  rc = smooth_residual(c, c->d_irs, -1.0, P, s, &R);
  if (rc != MB_OK) return rc;
  Params p = c->p;
  p.irk = irk;
  CK(irs_stage_update(p, c->d_tiles_aux, c->ntiles_aux, in, P, outp, R, rkc_of(c->sc.n_rk, irk), last, s));
  c->launches += 1;
  return MB_OK;
}

static int stage(mb_ctx* c, double* P, double* PO, int irk, cudaStream_t s) {
  const int n = c->sc.n_rk;
  double* S = c->d_scratch;
  const double* in;
  double* outp;
  stage_buffers(n, irk, P, PO, S, &in, &outp);
  int rc = ur_pass(c, in, s);  // prec: Ur of the stage input
  if (rc != MB_OK) return rc;
  rc = fill(c, const_cast<double*>(in), s);
  if (rc != MB_OK) return rc;
  rc = records(c, in, s);
  if (rc != MB_OK) return rc;
  const int last = (irk == n) ? 1 : 0;
  rc = stage_compute(c, in, P, outp, irk, last, s);
  if (rc != MB_OK) return rc;
  if (n == 1) {
    CK(cudaMemcpyAsync(P, S, (size_t)c->ncell * MB_NPRIM * sizeof(double), cudaMemcpyDeviceToDevice, s));
  }
  return MB_OK;
}

int mb_stage_input(mb_ctx* ctx, double* P, double* PO, int irk, double** in) {
  if (!ctx || !P || !PO || !in || irk < 1 || irk > ctx->sc.n_rk) return MB_E_ARG;
  const double* i;
  double* o;
  stage_buffers(ctx->sc.n_rk, irk, P, PO, ctx->d_scratch, &i, &o);
  *in = const_cast<double*>(i);
  return MB_OK;
}

int mb_stage_begin(mb_ctx* ctx, double* P, double* PO, int irk, void* stream) {
  if (!ctx || !P || !PO || irk < 1 || irk > ctx->sc.n_rk) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  prepare_tmaps(ctx, P, PO, s);
  const double* in;
  double* outp;
  stage_buffers(ctx->sc.n_rk, irk, P, PO, ctx->d_scratch, &in, &outp);
  int rc = ur_pass(ctx, in, s);
  if (rc != MB_OK) return rc;
  return fill(ctx, const_cast<double*>(in), s);
}

int mb_stage_end(mb_ctx* ctx, double* P, double* PO, int irk, void* stream) {
  if (!ctx || !P || !PO || irk < 1 || irk > ctx->sc.n_rk) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  const int n = ctx->sc.n_rk;
  const double* in;
  double* outp;
  stage_buffers(n, irk, P, PO, ctx->d_scratch, &in, &outp);
  int rc = records(ctx, in, s);
  if (rc != MB_OK) return rc;
  rc = stage_compute(ctx, in, P, outp, irk, irk == n ? 1 : 0, s);
  if (rc != MB_OK) return rc;
  if (n == 1) CK(cudaMemcpyAsync(P, ctx->d_scratch, (size_t)ctx->ncell * MB_NPRIM * sizeof(double),
                                 cudaMemcpyDeviceToDevice, s));
  return MB_OK;
}

int mb_pack_rows(const double* P, int64_t ncell, const int64_t* rows, int32_t n, double* buf, void* stream) {
  if (!P || ncell < 1 || n < 0 || (n > 0 && (!rows || !buf))) return MB_E_ARG;
  if (n == 0) return MB_OK;
  CK(pack_rows(P, ncell, (const long long*)rows, n, buf, (cudaStream_t)stream));
  return MB_OK;
}

int mb_unpack_rows(double* P, int64_t ncell, const int64_t* rows, int32_t n, const double* buf, void* stream) {
  if (!P || ncell < 1 || n < 0 || (n > 0 && (!rows || !buf))) return MB_E_ARG;
  if (n == 0) return MB_OK;
  CK(unpack_rows(P, ncell, (const long long*)rows, n, buf, (cudaStream_t)stream));
  return MB_OK;
}

// ---- CUDA IPC of stage buffers (a peer-store exchange between processes)
static PFN_cuMemGetAddressRange_v3020 addr_range_fn() {
  static PFN_cuMemGetAddressRange_v3020 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuMemGetAddressRange_v3020)f;
  }
  return fn;
}

int mb_ipc_export(const void* ptr, void* handle, int64_t* offset, int64_t* size) {
  if (!ptr || !handle || !offset || !size) return MB_E_ARG;
  PFN_cuMemGetAddressRange_v3020 range = addr_range_fn();
  if (!range) return MB_E_UNSUPPORTED;
  CUdeviceptr base = 0;
  size_t sz = 0;
  if (range(&base, &sz, (CUdeviceptr)ptr) != CUDA_SUCCESS) return MB_E_ARG;  // not device memory
  cudaIpcMemHandle_t h;
  CK(cudaIpcGetMemHandle(&h, (void*)base));
  static_assert(sizeof(h) == 64, "a CUDA IPC handle is 64 bytes");
  memcpy(handle, &h, sizeof(h));
  *offset = (int64_t)((const char*)ptr - (const char*)base);
  *size = (int64_t)sz;
  return MB_OK;
}

int mb_ipc_open(const void* handle, int device, void** base) {
  if (!handle || !base || device < 0) return MB_E_ARG;
  cudaIpcMemHandle_t h;
  memcpy(&h, handle, sizeof(h));
  int cur = 0;
  CK(cudaGetDevice(&cur));
  CK(cudaSetDevice(device));
  const cudaError_t e = cudaIpcOpenMemHandle(base, h, cudaIpcMemLazyEnablePeerAccess);
  cudaSetDevice(cur);  // the caller's current device is left as it was
  CK(e);
  return MB_OK;
}

int mb_ipc_close(void* base) {
  if (!base) return MB_E_ARG;
  CK(cudaIpcCloseMemHandle(base));
  return MB_OK;
}

int mb_enable_peer(int device, int peer) {
  if (device < 0 || peer < 0) return MB_E_ARG;
  if (device == peer) return MB_OK;
  int can = 0;
  CK(cudaDeviceCanAccessPeer(&can, device, peer));
  if (!can) return MB_E_UNSUPPORTED;
  int cur = 0;
  CK(cudaGetDevice(&cur));
  CK(cudaSetDevice(device));
  cudaError_t e = cudaDeviceEnablePeerAccess(peer, 0);
  if (e == cudaErrorPeerAccessAlreadyEnabled) {
    cudaGetLastError();  // the error of that call is not sticky: clear it
    e = cudaSuccess;
  }
  cudaSetDevice(cur);
  CK(e);
  return MB_OK;
}

int mb_push_rows(const double* src, int64_t nsrc, const int64_t* src_rows, double* dst, int64_t ndst,
                 const int64_t* dst_rows, int32_t n, void* stream) {
  if (!src || !dst || nsrc < 1 || ndst < 1 || n < 0 || (n > 0 && (!src_rows || !dst_rows))) return MB_E_ARG;
  if (n == 0) return MB_OK;
  CK(push_rows(src, nsrc, (const long long*)src_rows, dst, ndst, (const long long*)dst_rows, n, (cudaStream_t)stream));
  return MB_OK;
}

int mb_stage(mb_ctx* ctx, double* P, double* PO, int irk, void* stream) {
  if (!ctx || !P || !PO || irk < 1 || irk > ctx->sc.n_rk) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  prepare_tmaps(ctx, P, PO, (cudaStream_t)stream);
  return stage(ctx, P, PO, irk, (cudaStream_t)stream);
}

static int one_step(mb_ctx* c, double* P, double* PO, cudaStream_t s) {
  if (c->p.prec) {  // the preconditioned local steps need the Ur of the step's state: their own pass, not the fused one
    int rc = dt_min(c, P, s);
    if (rc != MB_OK) return rc;
  }
  CK(clock_step(c->p, s));
  c->launches += 1;
  for (int irk = 1; irk <= c->sc.n_rk; ++irk) {
    int rc = stage(c, P, PO, irk, s);
    if (rc != MB_OK) return rc;
  }
  return MB_OK;
}

int mb_step(mb_ctx* ctx, double* P, double* PO, int nsteps, int use_graph, void* stream) {
  if (!ctx || !P || !PO || nsteps < 0) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  prepare_tmaps(ctx, P, PO, s);
  if (!ctx->dt_valid) {
    int rc = dt_min(ctx, P, s);
    if (rc != MB_OK) return rc;
    ctx->dt_valid = true;
  }
  if (!use_graph) {
    for (int q = 0; q < nsteps; ++q) {
      int rc = one_step(ctx, P, PO, s);
      if (rc != MB_OK) return rc;
    }
    return MB_OK;
  }
  if (!ctx->gexec || ctx->gP != P || ctx->gPO != PO) {
    if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
    if (ctx->graph) { cudaGraphDestroy(ctx->graph); ctx->graph = nullptr; }
    // capture on a private stream so the caller's stream may be the legacy default stream
    cudaStream_t cs;
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    long long l0 = ctx->launches;
    CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    int rc = one_step(ctx, P, PO, cs);
    cudaGraph_t gr = nullptr;
    cudaError_t e = cudaStreamEndCapture(cs, &gr);
    cudaStreamDestroy(cs);
    ctx->graph_kernels = (int)(ctx->launches - l0);
    ctx->launches = l0;
    if (rc != MB_OK) { if (gr) cudaGraphDestroy(gr); return rc; }
    CK(e);
    ctx->graph = gr;
    CK(cudaGraphInstantiate(&ctx->gexec, gr, 0));
    ctx->gP = P;
    ctx->gPO = PO;
  }
  for (int q = 0; q < nsteps; ++q) {
    CK(cudaGraphLaunch(ctx->gexec, s));
    ctx->launches += ctx->graph_kernels;
  }
  return MB_OK;
}

int mb_profile_stage(mb_ctx* ctx, double* P, double* PO, int irk, int nrep, float* ms_ghost, float* ms_sweep,
                     void* stream) {
  if (!ctx || !P || !PO || irk < 1 || irk > ctx->sc.n_rk || nrep < 1 || !ms_ghost || !ms_sweep) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  prepare_tmaps(ctx, P, PO, s);
  const int n = ctx->sc.n_rk;
  double* S = ctx->d_scratch;
  const double* in;
  double* outp;
  stage_buffers(n, irk, P, PO, S, &in, &outp);
  cudaEvent_t e0, e1, e2;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventCreate(&e2));
  float tg = 0.f, ts = 0.f;
  int rc = MB_OK;
  for (int q = 0; q < nrep && rc == MB_OK; ++q) {
    cudaEventRecord(e0, s);
    rc = fill(ctx, const_cast<double*>(in), s);
    if (rc == MB_OK) rc = records(ctx, in, s);
    cudaEventRecord(e1, s);
    if (rc == MB_OK) rc = stage_compute(ctx, in, P, outp, irk, irk == n ? 1 : 0, s);
    cudaEventRecord(e2, s);
    cudaEventSynchronize(e2);
    float a = 0.f, b = 0.f;
    cudaEventElapsedTime(&a, e0, e1);
    cudaEventElapsedTime(&b, e1, e2);
    tg += a;
    ts += b;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  *ms_ghost = tg / nrep;
  *ms_sweep = ts / nrep;
  return rc;
}

int mb_get_status(mb_ctx* ctx, mb_status* st) { return mb_get_group_status(ctx, 0, 1, st); }

// The sweep's project-written autotuner, timed on the caller's state over the current mesh (call between steps: it
// uses the stage buffer):
//  - per depth class of the 3-D blocks (n3 <= 16, <= 64, <= 256, more; kclass_of), the k-chunk of their tiles
//    (8, 16, 32 or 64 planes), each class timed over its own tiles;
//  - for the main tile list and, separately, for the tiles of the mirrored one-plane blocks (2-D meshes): a plain
//    grid of one CTA per tile against the persistent work queue (about one wave of CTAs taking tiles, largest first,
//    from a counter);
//  - the mixed form: the tile staging (TMA boxes into a 5-value tile, or plain loads into a 6-value tile).
// The k-chunk and the queue never change a result; the staging changes the FP32 rounding of p in the mixed form.
int mb_autotune(mb_ctx* ctx, const double* P, void* stream) {
  if (!ctx || !P) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  prepare_tmaps(ctx, P, P, s);
  const int ty = ctx->ty_sweep;
  int rc;
  long long ccells[4] = {0, 0, 0, 0};
  int cmaxk[4] = {0, 0, 0, 0};
  for (size_t b = 0; b < ctx->hdims.size() / 3; ++b) {
    const int* n = &ctx->hdims[3 * b];
    if (n[2] <= 1 || ctx->hkm[b] < 0) continue;
    const int c = kclass_of(n[2]);
    ccells[c] += (long long)n[0] * n[1] * n[2];
    cmaxk[c] = std::max(cmaxk[c], n[2]);
  }
  int big = -1;
  for (int c = 0; c < 4; ++c) {
    if (!ccells[c]) continue;
    float best = 1e30f;
    int kbest = ctx->kcls[c];
    for (int kc : {8, 16, 32, 64}) {
      if (kc > 16 && kc / 2 >= cmaxk[c]) break;
      std::vector<DTile> tl = make_tiles(ctx->hdims, ty, kc, 1 << 3, &ctx->hkm, 0, nullptr, c);
      float ms = 0.f;
      if ((rc = time_sweep(ctx, tl, 0, P, 3, s, &ms)) != MB_OK) return rc;
      if (ms < best) { best = ms; kbest = kc; }
    }
    ctx->kcls[c] = kbest;
    if (big < 0 || ccells[c] > ccells[big]) big = c;
  }
  if (big >= 0) ctx->kc3 = ctx->kcls[big];
  std::vector<DTile> all = make_tiles(ctx->hdims, ty, ctx->kc3, 0xe, &ctx->hkm, 0, ctx->kcls);
  std::vector<DTile> sorted = all;
  sort_by_work(sorted, ctx->hdims, ty);
  float ms_plain = 0.f, ms_pers = 0.f;
  if (!all.empty()) {
    if ((rc = time_sweep(ctx, all, 0, P, 3, s, &ms_plain)) != MB_OK) return rc;
    if ((rc = time_sweep(ctx, sorted, 1, P, 3, s, &ms_pers)) != MB_OK) return rc;
  }
  ctx->persistent = ms_pers < ms_plain ? 1 : 0;
  ctx->tuned_ms = std::min(ms_plain, ms_pers);
  const std::vector<DTile>& use = ctx->persistent ? sorted : all;
  // the one-plane (mirrored) blocks' list: its own queue mode
  std::vector<DTile> km = make_tiles(ctx->hdims, ty, ctx->kc3, 0xe, &ctx->hkm, 1);
  std::vector<DTile> km_sorted = km;
  sort_by_work(km_sorted, ctx->hdims, ty);
  float km_plain = 0.f, km_pers = 0.f;
  if (!km.empty()) {
    if ((rc = time_sweep(ctx, km, 0, P, 3, s, &km_plain, 1)) != MB_OK) return rc;
    if ((rc = time_sweep(ctx, km_sorted, 1, P, 3, s, &km_pers, 1)) != MB_OK) return rc;
    ctx->persistent_km = km_pers < km_plain ? 1 : 0;
    ctx->tuned_ms += std::min(km_plain, km_pers);
  }
  const std::vector<DTile>& use_km = ctx->persistent_km ? km_sorted : km;
  // the mixed form: the tile staging that is faster on this state and mesh, per tile list: the 6-value tile by plain
  // loads against the 5-value tile, staged by TMA where the state buffer has a tensor map (by plain loads into the
  // same 5-value tile where it has none)
  float ms_stage[2] = {0.f, 0.f}, ms_stage_km[2] = {0.f, 0.f};
  if (ctx->sc.precision == MB_PREC_MIXED) {
    tmap_of(ctx, P, s, true);
    const bool keep = ctx->stage_tma, keep_km = ctx->stage_tma_km;
    for (int m = 0; m < 2; ++m) {
      ctx->stage_tma = ctx->stage_tma_km = m == 1;
      if ((!use.empty() && (rc = time_sweep(ctx, use, ctx->persistent, P, 3, s, &ms_stage[m])) != MB_OK) ||
          (!use_km.empty() && (rc = time_sweep(ctx, use_km, ctx->persistent_km, P, 3, s, &ms_stage_km[m], 1)) != MB_OK)) {
        ctx->stage_tma = keep;
        ctx->stage_tma_km = keep_km;
        return rc;
      }
    }
    ctx->stage_tma = ms_stage[1] < ms_stage[0];
    ctx->stage_tma_km = ms_stage_km[1] < ms_stage_km[0];
    ctx->tuned_ms = std::min(ms_stage[0], ms_stage[1]) + std::min(ms_stage_km[0], ms_stage_km[1]);
  }
  for (auto* d : {&ctx->d_tiles_sweep, &ctx->d_tiles_km}) {
    if (*d) cudaFree(*d);
    *d = nullptr;
  }
  if ((rc = upload(&ctx->d_tiles_sweep, use.data(), use.size())) != MB_OK) return rc;
  if ((rc = upload(&ctx->d_tiles_km, use_km.data(), use_km.size())) != MB_OK) return rc;
  ctx->ntiles_sweep = (int)use.size();
  ctx->ntiles_km = (int)use_km.size();
  CK(cudaStreamSynchronize(0));
  if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
  if (ctx->graph) { cudaGraphDestroy(ctx->graph); ctx->graph = nullptr; }
  ctx->gP = nullptr;
  ctx->gPO = nullptr;
  if (getenv("MB_REPORT")) {
    const bool mixed = ctx->sc.precision == MB_PREC_MIXED, mapped = mixed && tmap_of(ctx, P, s, false);
    auto label = [&](bool tma) {
      return !mixed ? "none (FP64 form)" : !tma ? "6-value tile, plain loads"
                                       : mapped ? "5-value tile, TMA" : "5-value tile, plain loads (no tensor map)";
    };
    fprintf(stderr, "[mose_b200] autotune: k-chunks %d %d %d %d (depth classes); main list: %s (plain %.3f ms, "
                    "persistent %.3f ms, %d tiles), staging %s (6-value %.3f ms, 5-value %.3f ms); one-plane list: %s "
                    "(plain %.3f ms, persistent %.3f ms, %d tiles), staging %s (6-value %.3f ms, 5-value %.3f ms)\n",
            ctx->kcls[0], ctx->kcls[1], ctx->kcls[2], ctx->kcls[3], ctx->persistent ? "persistent" : "plain", ms_plain,
            ms_pers, ctx->ntiles_sweep, label(ctx->stage_tma), ms_stage[0], ms_stage[1],
            ctx->persistent_km ? "persistent" : "plain", km_plain, km_pers, ctx->ntiles_km, label(ctx->stage_tma_km),
            ms_stage_km[0], ms_stage_km[1]);
  }
  return MB_OK;
}

int mb_set_tuning(mb_ctx* ctx, int kchunk, int persistent) {
  if (!ctx || kchunk < 1 || persistent < 0 || persistent > 1) return MB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaDeviceSynchronize());
  ctx->kc3 = kchunk;
  for (int c = 0; c < 4; ++c) ctx->kcls[c] = kchunk;
  ctx->persistent = persistent;
  std::vector<DTile> use = make_tiles(ctx->hdims, ctx->ty_sweep, kchunk, 0xe, &ctx->hkm, 0);
  if (persistent) sort_by_work(use, ctx->hdims, ctx->ty_sweep);
  if (ctx->d_tiles_sweep) cudaFree(ctx->d_tiles_sweep);
  ctx->d_tiles_sweep = nullptr;
  int rc = upload(&ctx->d_tiles_sweep, use.data(), use.size());
  if (rc != MB_OK) return rc;
  ctx->ntiles_sweep = (int)use.size();
  if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
  if (ctx->graph) { cudaGraphDestroy(ctx->graph); ctx->graph = nullptr; }
  ctx->gP = nullptr;
  ctx->gPO = nullptr;
  return MB_OK;
}

int mb_get_tuning(const mb_ctx* ctx, int* kchunk, int* persistent, float* ms) {
  if (!ctx || !kchunk || !persistent || !ms) return MB_E_ARG;
  *kchunk = ctx->kc3;
  *persistent = ctx->persistent;
  *ms = ctx->tuned_ms;
  return MB_OK;
}

}  // extern "C"
