// mb_irs.cu -- implicit residual smoothing (IRS_apply, numerics/time/explicit/Lib_IRS.f90:57-236) and the state
// update that takes its result, for schemes with mb_scheme.irs > 0. Built with --fmad=false: the smoothing rounds
// as the reference's statements do, in both forms (the mixed form's FP32 arithmetic ends with the residual).
//
// A stage with smoothing runs as separate passes, because every cell's smoothed residual depends on the residuals
// of its whole line: the sweep writes R (MODE_RESIDUAL), k_irs_scale scales it, then per direction the first ghost
// layer is filled (a row-copy list: zero gradient, connection records from their donor face cell) and
// k_irs_smooth writes the direction's njacobi Jacobi sweeps into the other buffer, and k_irs_stage_update applies
// the update (and, on the last stage, the next step's dt and the residual diagnostic, as the fused sweep does).
#include "mb_launch.h"

namespace mb {

// Scale_Residual_Cons (irs_scale_blk, Lib_IRS.f90:108-116): R = -R / vol * dtlocal * strang on the interior cells;
// dt < 0: the case's clock dt (the stage path), else the given dt (mb_update); with local time stepping each cell's
// own step from Pold, the state at the start of the step
__global__ void __launch_bounds__(32 * TY_AUX) k_irs_scale(Params p, const DTile* __restrict__ tiles, double* R,
                                                           double dt_arg, const double* __restrict__ Pold) {
  const DTile t = tiles[blockIdx.x];
  const DBlk b = p.blk[t.blk];
  const int i = t.i0 + (threadIdx.x & 31), j = t.j0 + (threadIdx.x >> 5);
  if (i > b.n1 || j > b.n2) return;
  const double strang = 1.0;
  const DevState* st = p.st + b.grp;
  const double dt = dt_arg >= 0.0 ? dt_arg : st->dt;
  for (int k = t.k0; k < t.k1; ++k) {
    const long long r = row(b, i, j, k);
    const double vol = ld(b.vol + (r - b.boff));
    double dtc = dt;
    if (p.local_dt) {
      double po[MB_NP];
#pragma unroll
      for (int s = 0; s < MB_NP; ++s) po[s] = Pold[r + s * p.nc];
      dtc = step_dt(p, b, st, r - b.boff, po, dt);
    }
#pragma unroll
    for (int s = 0; s < MB_NP; ++s) R[r + s * p.nc] = -R[r + s * p.nc] / vol * dtc * strang;
  }
}

// Residual_Smoothing_Blk along direction d (irs_smooth_blk, :204-236): NJ Jacobi sweeps of
// R*(c) = (R(c) + beta (R*(c - off) + R*(c + off))) / (1 + 2 beta), R* starting from R, the first ghost layer held
// at its value. Sweep m changes a cell from its neighbours' values of sweep m-1, so the result at a cell depends
// only on the cells within NJ of it along d: each thread takes that window of 2 NJ + 1 values of its line (ghosts
// included, nothing beyond them) and runs the sweeps on it, the values at distance q valid through sweep NJ - q.
// Every value is the reference's, operation for operation; the sweeps' intermediate arrays never reach memory.
// Blocks of a case with fewer directions than d are copied through.
template <int NJ>
__global__ void __launch_bounds__(32 * TY_AUX) k_irs_smooth(Params p, const DTile* __restrict__ tiles,
                                                            const double* __restrict__ Rin, double* __restrict__ Rout,
                                                            int d, double beta) {
  constexpr int W = 2 * NJ + 1;
  const DTile t = tiles[blockIdx.x];
  const DBlk b = p.blk[t.blk];
  const int i = t.i0 + (threadIdx.x & 31), j = t.j0 + (threadIdx.x >> 5);
  if (i > b.n1 || j > b.n2) return;
  const long long off = (d == 1) ? 1 : (d == 2 ? (long long)b.pi : (long long)b.pi * b.pj);
  const int nd = (d == 1) ? b.n1 : (d == 2 ? b.n2 : b.n3);
  const double den = 1.0 + 2.0 * beta;
  for (int k = t.k0; k < t.k1; ++k) {
    const long long r = row(b, i, j, k);
    if (d > b.ndir) {
#pragma unroll
      for (int s = 0; s < MB_NP; ++s) Rout[r + s * p.nc] = Rin[r + s * p.nc];
      continue;
    }
    const int c = (d == 1) ? i : (d == 2 ? j : k);
#pragma unroll
    for (int s = 0; s < MB_NP; ++s) {
      const double* src = Rin + r + s * p.nc;
      double rw[W], x[W];
#pragma unroll
      for (int o = -NJ; o <= NJ; ++o) {
        const int q = c + o;  // 0 and nd + 1: the first ghost layer
        rw[o + NJ] = (q >= 0 && q <= nd + 1) ? src[o * off] : 0.0;
        x[o + NJ] = rw[o + NJ];
      }
#pragma unroll
      for (int m = 1; m <= NJ; ++m) {
        double y[W];
#pragma unroll
        for (int o = -(NJ - m); o <= NJ - m; ++o) {
          const int q = c + o;
          y[o + NJ] = (q >= 1 && q <= nd) ? (rw[o + NJ] + beta * (x[o + NJ - 1] + x[o + NJ + 1])) / den : x[o + NJ];
        }
#pragma unroll
        for (int o = -(NJ - m); o <= NJ - m; ++o) x[o + NJ] = y[o + NJ];
      }
      Rout[r + s * p.nc] = x[NJ];
    }
  }
}

// RK_Newstate on the smoothed residual of stage irk: Pout <- update(Pin, Pold, R) (newstate_cons_body.inc with the
// residual prescaled, or Newstate_Primitive on the smoothed raw residual), the state check and thermo guard as the
// fused sweep, and on the last stage the new state's local dt and the residual diagnostic of the step (FP64).
// Cases that reached their stop are skipped.
__global__ void __launch_bounds__(32 * TY_AUX) k_irs_stage_update(Params p, const DTile* __restrict__ tiles,
                                                                  const double* Pin, const double* Pold, double* Pout,
                                                                  const double* __restrict__ R, double rkc, int last) {
  __shared__ double sred[32];
  const DTile t = tiles[blockIdx.x];
  const DBlk b = p.blk[t.blk];
  DevState* st = p.st + b.grp;
  if (st->done) return;  // uniform over the CTA
  const int i = t.i0 + (threadIdx.x & 31), j = t.j0 + (threadIdx.x >> 5);
  const bool own = i <= b.n1 && j <= b.n2;
  const double dt = st->dt;
  double dtloc = 1e300;
  double rsq[MB_NP] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (own) {
    for (int k = t.k0; k < t.k1; ++k) {
      const long long r = row(b, i, j, k);
      double pc[MB_NP], po[MB_NP], res[MB_NP], pn[MB_NP];
#pragma unroll
      for (int s = 0; s < MB_NP; ++s) { pc[s] = Pin[r + s * p.nc]; po[s] = Pold[r + s * p.nc]; res[s] = R[r + s * p.nc]; }
      double rho, T;
      cell_rho_T(p, pc[0], pc[MB_IPR], rho, T);
      if (p.guard && !(T > 1.0 && T < 9990.0)) {
        atomicAdd(&st->n_bad_thermo, 1);
        if (T != T) T = 300.0;
        T = mn(mx(T, 1.0), 9990.0);
      }
      const double vol = ld(b.vol + (r - b.boff));
      const double dtc = step_dt(p, b, st, r - b.boff, po, dt);
      if (p.intvar) prim_update(p, pc, po, res, vol, dtc, rkc, pn, p.prec ? p.ur[r] : 0.0);
      else cons_update(p, pc, po, res, vol, dtc, rkc, T, pn, r, true);
      bool bad = !(pn[MB_IPR] >= 0.0);
#pragma unroll
      for (int s = 0; s < MB_NP; ++s) bad = bad || !isfinite(pn[s]);
      if (bad) report_bad_state(st, t.blk, i, j, k);
#pragma unroll
      for (int s = 0; s < MB_NP; ++s) Pout[r + s * p.nc] = pn[s];
      if (last) {
#pragma unroll
        for (int v = 0; v < MB_NP; ++v) {
          const double dv = pn[v] - po[v];
          rsq[v] += dv * dv;
        }
        dtloc = mn(dtloc, cell_dt(p, b, r - b.boff, pn));
      }
    }
  }
  if (last) {  // uniform over the CTA
#pragma unroll
    for (int v = 0; v < MB_NP; ++v) {
      double x = rsq[v];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if ((threadIdx.x & 31) == 0 && x != 0.0) atomicAdd(&st->res2[v], x);
    }
    cta_min_dt(st, dtloc, sred);
  }
}

// the first ghost layer of the smoothing direction: row dst[e] <- row src[e] (an interior cell: the adjacent one, or
// a connection record's donor face cell), so the copies of one launch never read what another writes
__global__ void k_irs_ghost(const long long* __restrict__ dst, const long long* __restrict__ src, int n, long long nc,
                            double* R) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)n * MB_NP) return;
  const int e = (int)(q % n), s = (int)(q / n);
  R[dst[e] + s * nc] = R[src[e] + s * nc];
}

// ---- launchers ----
cudaError_t irs_scale(const Params& p, const DTile* tiles, int ntiles, double* R, double dt, const double* Pold,
                      cudaStream_t s) {
  k_irs_scale<<<ntiles, 32 * TY_AUX, 0, s>>>(p, tiles, R, dt, Pold);
  return cudaGetLastError();
}

cudaError_t irs_ghosts(const Params& p, const long long* dst, const long long* src, int n, double* R, cudaStream_t s) {
  if (n > 0) k_irs_ghost<<<(unsigned)(((long long)n * MB_NP + 255) / 256), 256, 0, s>>>(dst, src, n, p.nc, R);
  return cudaGetLastError();
}

cudaError_t irs_smooth(const Params& p, const DTile* tiles, int ntiles, const double* Rin, double* Rout, int d,
                       int njacobi, double beta, cudaStream_t s) {
  switch (njacobi) {
    case 1: k_irs_smooth<1><<<ntiles, 32 * TY_AUX, 0, s>>>(p, tiles, Rin, Rout, d, beta); break;
    case 2: k_irs_smooth<2><<<ntiles, 32 * TY_AUX, 0, s>>>(p, tiles, Rin, Rout, d, beta); break;
    case 3: k_irs_smooth<3><<<ntiles, 32 * TY_AUX, 0, s>>>(p, tiles, Rin, Rout, d, beta); break;
    case 4: k_irs_smooth<4><<<ntiles, 32 * TY_AUX, 0, s>>>(p, tiles, Rin, Rout, d, beta); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t irs_stage_update(const Params& p, const DTile* tiles, int ntiles, const double* Pin, const double* Pold,
                             double* Pout, const double* R, double rkc, int last, cudaStream_t s) {
  k_irs_stage_update<<<ntiles, 32 * TY_AUX, 0, s>>>(p, tiles, Pin, Pold, Pout, R, rkc, last);
  return cudaGetLastError();
}

}  // namespace mb
