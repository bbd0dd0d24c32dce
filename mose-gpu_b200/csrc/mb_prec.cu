// mb_prec.cu -- integration-variables = prec: the reference velocity Ur of every cell (Update_Derived_Variables,
// numerics/time/explicit/Lib_Preconditioning.f90:84-295) and the local steps of the preconditioned system
// (Compute_dt_blk with prec, dt_blk.inc), FP64, built with --fmad=false.
//
// Ur is a field: Ur-smooth takes the max over the face neighbours, so it is computed by its own passes over the stage
// input (the state the reference's Update_Derived_Variables has seen after the previous update) before the sweep reads
// it, and the local steps of a step, which the reference fixes at its start with the Ur of that state, are stored per
// row for the stages to read.
#include "mb_launch.h"

namespace mb {

// comp_Ur (Lib_Preconditioning.f90:84-142): mode 1 a uniform Uref (the sound speed above it), mode 2 the target
// preconditioned Mach number (the root w < 1 of A w^2 + B w + A = 0, w = (Ur / a)^2), mode 3 Weiss-Smith (|u| Ur-factor
// between eps_min a and a); the viscous floor in modes 2 and 3, then Ur-min
__device__ double comp_ur(const Params& p, double vel, double sound, double ur_visc) {
  double Ur;
  const double eps = p.prec_eps_min;
  if (p.prec_uref > 0.0) {
    Ur = (vel > p.prec_uref) ? sound : p.prec_uref;
  } else if (p.prec_mach > 0.0) {
    const double Mt = p.prec_mach, m = vel / sound;
    const double A_q = 0.25 * m * m * (Mt * Mt - 1.0);
    const double B_q = Mt * Mt - 0.5 * m * m * (Mt * Mt + 1.0);
    if (fabs(A_q) > 1.0e-30) {
      const double S_q = -B_q / A_q, disc = S_q * S_q - 4.0;
      if (disc > 0.0 && S_q > 2.0) Ur = sound * sqrt(2.0 / (S_q + sqrt(disc)));
      else Ur = sound;
    } else {
      Ur = sound * eps;
    }
    Ur = mx(Ur, eps * sound);
    Ur = mn(Ur, sound);
    Ur = mx(Ur, ur_visc);
  } else {
    if (vel < eps * sound) Ur = sound * eps;
    else if (vel >= sound) Ur = sound;
    else Ur = vel * p.prec_ur_factor;
    Ur = mx(Ur, ur_visc);
  }
  if (p.prec_ur_min > 0.0) Ur = mx(Ur, p.prec_ur_min);
  return Ur;
}

// Ur_Blk (:187-264) on the interior cells of P: the viscous floor max(mu / (rho dx_min), k / (rho cp dx_min)) with mu
// and k of the Wilke rule (not the Prandtl-number k)
__global__ void __launch_bounds__(32 * TY_AUX) k_ur(Params p, const DTile* __restrict__ tiles,
                                                    const double* __restrict__ P, double* __restrict__ ur) {
  const DTile t = tiles[blockIdx.x];
  const DBlk b = p.blk[t.blk];
  const int i = t.i0 + (threadIdx.x & 31), j = t.j0 + (threadIdx.x >> 5);
  if (i > b.n1 || j > b.n2) return;
  for (int k = t.k0; k < t.k1; ++k) {
    const long long r = row(b, i, j, k), l = r - b.boff;
    double pl[MB_NP];
#pragma unroll
    for (int s = 0; s < MB_NP; ++s) pl[s] = P[r + s * p.nc];
    double rho, R;
    rotot_rtot(p, pl[0], rho, R);
    const double T = pl[MB_IPR] / (rho * R);
    const double vel_mag = sqrt(pl[MB_IU] * pl[MB_IU] + pl[MB_IV] * pl[MB_IV] + pl[MB_IW] * pl[MB_IW]);
    double ur_visc = 0.0;
    if (p.visc) {
      const double* dl = b.dl + 3 * l;
      double dx_min = ld(dl);
      for (int d = 1; d < b.ndir; ++d) dx_min = mn(dx_min, ld(dl + d));
      const int ti = tidx(p, T);
      const double td = T - (double)ti;
      const double cp = f_cp(p, pl[0], ti, td, rho);
      double mu, lambda;
      wilke(p, pl[0], rho, ti, td, mu, lambda);
      ur_visc = mx(mu / (rho * dx_min), lambda / (rho * cp * dx_min));
    }
    const double sound = f_ss(p, pl[0], pl[MB_IPR], rho, R);
    ur[r] = comp_ur(p, vel_mag, sound, ur_visc);
  }
}

// Smooth_Ur_Blk (:269-295), one pass: urb = the max over the cell and its six face neighbours (ghost rows of ur are 0)
__global__ void __launch_bounds__(32 * TY_AUX) k_ur_smooth(Params p, const DTile* __restrict__ tiles,
                                                           const double* __restrict__ ur, double* __restrict__ urb) {
  const DTile t = tiles[blockIdx.x];
  const DBlk b = p.blk[t.blk];
  const int i = t.i0 + (threadIdx.x & 31), j = t.j0 + (threadIdx.x >> 5);
  if (i > b.n1 || j > b.n2) return;
  const long long sj = b.pi, sk = (long long)b.pi * b.pj;
  for (int k = t.k0; k < t.k1; ++k) {
    const long long r = row(b, i, j, k);
    double m = ur[r];
    m = mx(m, ur[r - 1]); m = mx(m, ur[r + 1]);
    m = mx(m, ur[r - sj]); m = mx(m, ur[r + sj]);
    m = mx(m, ur[r - sk]); m = mx(m, ur[r + sk]);
    urb[r] = m;
  }
}

__global__ void __launch_bounds__(32 * TY_AUX) k_ur_copy(Params p, const DTile* __restrict__ tiles,
                                                         const double* __restrict__ urb, double* __restrict__ ur) {
  const DTile t = tiles[blockIdx.x];
  const DBlk b = p.blk[t.blk];
  const int i = t.i0 + (threadIdx.x & 31), j = t.j0 + (threadIdx.x >> 5);
  if (i > b.n1 || j > b.n2) return;
  for (int k = t.k0; k < t.k1; ++k) {
    const long long r = row(b, i, j, k);
    ur[r] = urb[r];
  }
}

// the local steps of the preconditioned system (Compute_dt_blk with prec) of every interior cell of P, before the ramp
// factor, into dtl (rows); reduce != 0: also their minimum into the case's clock
__global__ void __launch_bounds__(32 * TY_AUX) k_dt_prec(Params p, const DTile* __restrict__ tiles,
                                                         const double* __restrict__ P, double* __restrict__ dtl,
                                                         int reduce) {
  __shared__ double sred[32];
  const DTile t = tiles[blockIdx.x];
  const DBlk b = p.blk[t.blk];
  const int i = t.i0 + (threadIdx.x & 31), j = t.j0 + (threadIdx.x >> 5);
  double v = 1e300;
  if (i <= b.n1 && j <= b.n2) {
    for (int k = t.k0; k < t.k1; ++k) {
      const long long r = row(b, i, j, k);
      double pl[MB_NP];
#pragma unroll
      for (int s = 0; s < MB_NP; ++s) pl[s] = P[r + s * p.nc];
      const double dtc = cell_dt_t<double, true>(p, b, r - b.boff, pl, p.ur[r]);
      dtl[r] = dtc;
      v = mn(v, dtc);
    }
  }
  if (reduce) cta_min_dt(p.st + b.grp, v, sred);
}

// ---- launchers ----
cudaError_t prec_ur(const Params& p, const DTile* tiles, int ntiles, const double* P, double* ur, double* urb,
                    int nsmooth, cudaStream_t s, int* nl) {
  k_ur<<<ntiles, 32 * TY_AUX, 0, s>>>(p, tiles, P, ur);
  *nl = 1;
  for (int q = 0; q < nsmooth; ++q) {
    k_ur_smooth<<<ntiles, 32 * TY_AUX, 0, s>>>(p, tiles, ur, urb);
    k_ur_copy<<<ntiles, 32 * TY_AUX, 0, s>>>(p, tiles, urb, ur);
    *nl += 2;
  }
  return cudaGetLastError();
}

cudaError_t prec_dt(const Params& p, const DTile* tiles, int ntiles, const double* P, double* dtl, int reduce,
                    cudaStream_t s) {
  k_dt_prec<<<ntiles, 32 * TY_AUX, 0, s>>>(p, tiles, P, dtl, reduce);
  return cudaGetLastError();
}

}  // namespace mb
