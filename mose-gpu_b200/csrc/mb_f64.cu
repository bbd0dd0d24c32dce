// mb_f64.cu -- the per-cell and ghost kernels of the engine (FP64). Built with --fmad=false so that every
// statement rounds as written (the operation order of the reference statements is kept in
// mb_physics.cuh / mb_engine.cuh). The fused sweep is instantiated in the mb_sweep_*.cu units.
#include "mb_launch.h"

namespace mb {

// ---- ghost fill (numerics/fluxes/bc/Lib_Extrapolation.f90) ----
// Fill_Ghost_Cell_blk (:643-730): the mirrored first layer of symmetry faces (type 3, Ghost_Symmetry :558-587),
// zero-gradient ghosts of types 4 / 11 / 24 (Ghost_ZG_Extrapolate :590-614), the second-order extrapolation
// 3 x3 - 3 x2 + x1 of the walls 5 / 6 (Ghost_Extrapolate :616-641)
__global__ void k_ghost_phys(Params p, const GRec* __restrict__ rec, const int* __restrict__ list, int n, double* P) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int e = list[q];
  const int nl = (e >> 28) ? (e >> 28) : GC;  // ghost layers to fill (entries of the fused lists carry theirs)
  const GRec r = rec[e & 0x0fffffff];
  const DBlk b = p.blk[r.blk];
  const int dir = (r.face + 1) / 2, gstep = 2 * (r.face % 2) - 1;
  const long long st = (dir == 1) ? 1 : (dir == 2 ? (long long)b.pi : (long long)b.pi * b.pj);
  const long long src = row(b, r.i, r.j, r.k);
  const long long nc = p.nc;
  if (r.type == 3) {  // Ghost_Symmetry (Lib_Extrapolation.f90:558-587): the first layer, normal velocity reversed
    double g[4];
    bc_face_geom(b, r.i, r.j, r.k, r.face, g);
    const long long dst = src - (long long)gstep * st;
    double vel[3] = {P[src + MB_IU * nc], P[src + MB_IV * nc], P[src + MB_IW * nc]};
    const double udotn = vel[0] * g[0] + vel[1] * g[1] + vel[2] * g[2];
    for (int a = 0; a < 3; ++a) vel[a] = vel[a] - 2.0 * udotn * g[a];
    P[dst] = P[src];
    P[dst + MB_IU * nc] = vel[0]; P[dst + MB_IV * nc] = vel[1]; P[dst + MB_IW * nc] = vel[2];
    P[dst + MB_IPR * nc] = P[src + MB_IPR * nc];
  } else if (r.type == 5 || r.type == 6) {
    const int step = -gstep;
    for (int g = 1; g <= nl; ++g) {
      long long d0 = src + (long long)(g * step) * st, a1 = src + (long long)((g - 1) * step) * st,
                a2 = src + (long long)((g - 2) * step) * st, a3 = src + (long long)((g - 3) * step) * st;
      for (int s = 0; s < MB_NP; ++s) P[d0 + s * nc] = 3.0 * P[a1 + s * nc] - 3.0 * P[a2 + s * nc] + P[a3 + s * nc];
    }
  } else {
    for (int g = 1; g <= nl; ++g) {
      long long dst = src - (long long)(gstep * g) * st;
      for (int s = 0; s < MB_NP; ++s) P[dst + s * nc] = P[src + s * nc];
    }
  }
}

// extrapolation-ghost = cubic on the 400 faces (Fill_Ghost_Cubic_Extrapolation_blk, :859-879),
// a separate launch after every zero-gradient ghost is written
__global__ void k_ghost_cubic(Params p, const GRec* __restrict__ rec, const int* __restrict__ list, int n, double* P) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int e = list[q];
  const int nl = (e >> 28) ? (e >> 28) : GC;
  const GRec r = rec[e & 0x0fffffff];
  const DBlk b = p.blk[r.blk];
  const int dir = (r.face + 1) / 2, gstep = 2 * (r.face % 2) - 1, step = -gstep;
  const long long st = (dir == 1) ? 1 : (dir == 2 ? (long long)b.pi : (long long)b.pi * b.pj);
  const long long src = row(b, r.i, r.j, r.k);
  const long long nc = p.nc;
  for (int g = 1; g <= nl; ++g) {
    long long d0 = src + (long long)(g * step) * st, a1 = src + (long long)((g - 1) * step) * st,
              a2 = src + (long long)((g - 2) * step) * st, a3 = src + (long long)((g - 3) * step) * st;
    for (int s = 0; s < MB_NP; ++s) P[d0 + s * nc] = 3.0 * P[a1 + s * nc] - 3.0 * P[a2 + s * nc] + P[a3 + s * nc];
  }
}

// 1:1 and periodic connections (Ghost_Connection_pair, :1023-1134): receiver ghost layer g <- donor layer g.
// The donor layers are interior cells, so the copies of one launch never read what another writes.
__global__ void k_ghost_copy(const long long* __restrict__ dst, const long long* __restrict__ src, int n, long long nc,
                             double* P) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)n * MB_NP) return;
  const int e = (int)(q % n), s = (int)(q / n);
  P[dst[e] + s * nc] = P[src[e] + s * nc];
}


// ---- Compute_dt alone: k_dt_t<double> of mb_engine.cuh ----

// ---- RK_Newstate alone: the conservative update of every interior cell from a given residual ----
__global__ void __launch_bounds__(32 * TY_AUX) k_update(Params p, const DTile* __restrict__ tiles, double* P,
                                                        const double* PO, const double* R, double rkc, double dt,
                                                        int prescaled) {
  const DTile t = tiles[blockIdx.x];
  const DBlk b = p.blk[t.blk];
  DevState* st = p.st + b.grp;
  const int i = t.i0 + (threadIdx.x & 31), j = t.j0 + (threadIdx.x >> 5);
  if (i > b.n1 || j > b.n2) return;
  for (int k = t.k0; k < t.k1; ++k) {
    const long long r = row(b, i, j, k);
    double pc[MB_NP], po[MB_NP], res[MB_NP], pn[MB_NP];
    for (int s = 0; s < MB_NP; ++s) { pc[s] = P[r + s * p.nc]; po[s] = PO[r + s * p.nc]; res[s] = R[r + s * p.nc]; }
    double rho, T;
    cell_rho_T(p, pc[0], pc[MB_IPR], rho, T);
    if (p.guard && !(T > 1.0 && T < 9990.0)) {
      atomicAdd(&st->n_bad_thermo, 1);
      if (T != T) T = 300.0;
      T = mn(mx(T, 1.0), 9990.0);
    }
    const double dtc = step_dt(p, b, st, r - b.boff, po, dt);
    if (p.intvar) prim_update(p, pc, po, res, ld(b.vol + (r - b.boff)), dtc, rkc, pn, p.prec ? p.ur[r] : 0.0);
    else cons_update(p, pc, po, res, ld(b.vol + (r - b.boff)), dtc, rkc, T, pn, r, prescaled != 0);
    bool bad = !(pn[MB_IPR] >= 0.0);
    for (int s = 0; s < MB_NP; ++s) bad = bad || !isfinite(pn[s]);
    if (bad) report_bad_state(st, t.blk, i, j, k);
    for (int s = 0; s < MB_NP; ++s) P[r + s * p.nc] = pn[s];
  }
}

__global__ void k_to_float(const double* __restrict__ src, float* __restrict__ dst, long long n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    dst[q] = (float)src[q];
}

cudaError_t to_float(const double* src, float* dst, long long n, cudaStream_t s) {
  k_to_float<<<1184, 256, 0, s>>>(src, dst, n);
  return cudaGetLastError();
}

__global__ void k_reset_dt(Params p, int only_group) {
  for (int g = threadIdx.x; g < p.ngroups; g += blockDim.x)
    if (only_group < 0 || g == only_group) p.st[g].dtmin_bits = (unsigned long long)__double_as_longlong(1e300);
}

// the step's dt of every case (Compute_dt's dtglobal = 1e5 then the cell minimum, Mod_Explicit.f90:122;
// Set_Global_dt; Clip_dt_To_Timemax, Mod_dt.f90:283-296), its simulated time, and a fresh minimum for the
// next step. A case whose time has reached its stop time (the reference's time-loop exit) is marked done and
// no longer advances.
__global__ void k_clock(Params p) {
  for (int g = threadIdx.x; g < p.ngroups; g += blockDim.x) {
    DevState* st = p.st + g;
    if (st->done) continue;
    if (st->t_end > 0.0 && st->time >= st->t_end) {
      st->done = 1;
      continue;
    }
    // the residual end test of the step just taken (Mod_Explicit.f90:363-370: residuotot(1) <= restop)
    if (st->res_stop > 0.0 && st->steps > 0 && sqrt(st->res2[0]) <= st->res_stop) {
      st->done = 1;
      continue;
    }
    // cfl-rise-threshold: the factor of step iter (Mod_dt.f90:57-58); the minimum of the scaled local steps is the
    // scaled minimum (a product with a positive factor rounds monotonically)
    const int iter = st->steps + 1;
    st->rampf = (iter < p.cfl_rise) ? (double)iter / p.cfl_rise : 1.0;
    double dtg = 1e5;
    double dm = __longlong_as_double((long long)st->dtmin_bits);
    dtg = mn(dm * st->rampf, dtg);
    if (st->time_clip && !p.local_dt) {
      double rem = st->t_end - st->time;
      if (rem > 0.0 && dtg > rem) dtg = rem * (1.0 + 1e-12);
    }
    st->dt = dtg;
    if (!p.local_dt) st->time = st->time + dtg;  // time-accurate = false: no simulated time (Mod_Explicit.f90:124-128)
    st->steps = st->steps + 1;
    st->dtmin_bits = (unsigned long long)__double_as_longlong(1e300);
    for (int v = 0; v < MB_NP; ++v) st->res2[v] = 0.0;
  }
}

// mb_group_reset: case g starts afresh with its stop rule
__global__ void k_group_reset(Params p, int g, int time_clip, double t_end, double res_stop) {
  DevState* st = p.st + g;
  st->dtmin_bits = (unsigned long long)__double_as_longlong(1e300);
  st->dt = 0.0; st->time = 0.0; st->steps = 0; st->code = 0;
  st->n_bad_state = 0; st->n_bad_thermo = 0;
  st->bad_blk = 0; st->bad_i = 0; st->bad_j = 0; st->bad_k = 0; st->first_bad_claimed = 0;
  st->time_clip = time_clip; st->done = 0; st->t_end = t_end; st->res_stop = res_stop;
  st->rampf = (1 < p.cfl_rise) ? 1.0 / p.cfl_rise : 1.0;  // the factor of step 1 (the update hook before any step)
  for (int v = 0; v < MB_NP; ++v) st->res2[v] = 0.0;
}

// ---- launchers ----
static inline unsigned nblk_for(long long n, int t) { return (unsigned)((n + t - 1) / t); }

cudaError_t ghost_fill(const Params& p, const GhostLists& g, double* P, cudaStream_t s, int* nl) {
  *nl = 0;
  if (!g.ordered) {
    if (g.nphys > 0) { k_ghost_phys<<<nblk_for(g.nphys, 128), 128, 0, s>>>(p, g.rec, g.phys, g.nphys, P); ++*nl; }
    if (g.ncubic > 0) { k_ghost_cubic<<<nblk_for(g.ncubic, 128), 128, 0, s>>>(p, g.rec, g.cubic, g.ncubic, P); ++*nl; }
  } else {
    for (int f = 0; f < 2; ++f) {
      const int n = g.phys_off[f + 1] - g.phys_off[f];
      if (n > 0) { k_ghost_phys<<<nblk_for(n, 128), 128, 0, s>>>(p, g.rec, g.phys + g.phys_off[f], n, P); ++*nl; }
    }
    for (int f = 0; f < 2; ++f) {
      const int n = g.cubic_off[f + 1] - g.cubic_off[f];
      if (n > 0) { k_ghost_cubic<<<nblk_for(n, 128), 128, 0, s>>>(p, g.rec, g.cubic + g.cubic_off[f], n, P); ++*nl; }
    }
  }
  if (g.ncopy > 0) {
    k_ghost_copy<<<nblk_for((long long)g.ncopy * MB_NP, 256), 256, 0, s>>>(g.cdst, g.csrc, g.ncopy, p.nc, P);
    ++*nl;
  }
  return cudaGetLastError();
}

cudaError_t dt_cells(const Params& p, const DTile* tiles, int ntiles, const double* P, cudaStream_t s,
                     int only_group) {
  k_dt_t<double><<<ntiles, 32 * TY_AUX, 0, s>>>(p, tiles, P, only_group);
  return cudaGetLastError();
}

cudaError_t update_cells(const Params& p, const DTile* tiles, int ntiles, double* P, const double* PO, const double* R,
                         double rkc, double dt, cudaStream_t s, int prescaled) {
  k_update<<<ntiles, 32 * TY_AUX, 0, s>>>(p, tiles, P, PO, R, rkc, dt, prescaled);
  return cudaGetLastError();
}

cudaError_t reset_dt(const Params& p, cudaStream_t s, int only_group) {
  k_reset_dt<<<1, 256, 0, s>>>(p, only_group);
  return cudaGetLastError();
}

// the halo rows of a partitioned mesh, gathered into / scattered from a contiguous buffer [variable][row] (one
// thread per row and variable, coalesced on the buffer side)
__global__ void k_pack_rows(const double* __restrict__ P, long long nc, const long long* __restrict__ rows, int n,
                            double* __restrict__ buf) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)n * MB_NP) return;
  const int v = (int)(q / n), e = (int)(q - (long long)v * n);
  buf[q] = P[rows[e] + v * nc];
}

__global__ void k_unpack_rows(double* __restrict__ P, long long nc, const long long* __restrict__ rows, int n,
                              const double* __restrict__ buf) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)n * MB_NP) return;
  const int v = (int)(q / n), e = (int)(q - (long long)v * n);
  P[rows[e] + v * nc] = buf[q];
}

// the halo rows moved straight from the owner's stage input into the receiver's (another arena, on this GPU or a
// peer's: the stores cross NVLink, no staging buffer and no send / receive): one thread per row and variable, the
// loads local, the stores posted to the receiver
__global__ void k_push_rows(const double* __restrict__ src, long long nsrc, const long long* __restrict__ srows,
                            double* __restrict__ dst, long long ndst, const long long* __restrict__ drows, int n) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)n * MB_NP) return;
  const int v = (int)(q / n), e = (int)(q - (long long)v * n);
  dst[drows[e] + v * ndst] = src[srows[e] + v * nsrc];
}

cudaError_t push_rows(const double* src, long long nsrc, const long long* srows, double* dst, long long ndst,
                      const long long* drows, int n, cudaStream_t s) {
  const long long tot = (long long)n * MB_NP;
  k_push_rows<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(src, nsrc, srows, dst, ndst, drows, n);
  return cudaGetLastError();
}

cudaError_t pack_rows(const double* P, long long ncell, const long long* rows, int n, double* buf, cudaStream_t s) {
  const long long tot = (long long)n * MB_NP;
  k_pack_rows<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(P, ncell, rows, n, buf);
  return cudaGetLastError();
}

cudaError_t unpack_rows(double* P, long long ncell, const long long* rows, int n, const double* buf, cudaStream_t s) {
  const long long tot = (long long)n * MB_NP;
  k_unpack_rows<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(P, ncell, rows, n, buf);
  return cudaGetLastError();
}

// the bounded wait of the TMA staging run out on purpose: one CTA waits for phase 0 of an mbarrier that nothing
// arrives at, with a limit of `tries` rounds, and writes 1 once it gave up (a sweep then records MB_E_TIMEOUT and
// returns); the kernel ends either way
__global__ void k_wait_selftest(unsigned tries, int* gave_up) {
  __shared__ __align__(8) unsigned long long bar;
  if (threadIdx.x == 0) mbar_init(&bar);
  __syncthreads();
  bool ok = false;
  for (unsigned q = 0; q < tries && !ok; ++q) ok = mbar_test(&bar, 0);
  if (threadIdx.x == 0) *gave_up = ok ? 0 : 1;
}

cudaError_t wait_selftest(unsigned tries, int* gave_up, cudaStream_t s) {
  k_wait_selftest<<<1, 32, 0, s>>>(tries, gave_up);
  return cudaGetLastError();
}

cudaError_t clock_step(const Params& p, cudaStream_t s) {
  k_clock<<<1, 256, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t group_reset(const Params& p, int g, int time_clip, double t_end, double res_stop, cudaStream_t s) {
  k_group_reset<<<1, 1, 0, s>>>(p, g, time_clip, t_end, res_stop);
  return cudaGetLastError();
}

}  // namespace mb
