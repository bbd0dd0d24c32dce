// mose_oracle.cpp -- CPU restatement (FP64) of MOSE-GPU's explicit residual evaluation and
// Runge-Kutta stage update, used ONLY as the correctness checker of the B200 engine and as the
// timed CPU baseline of bench.py. It is test infrastructure: nothing in the product links it.
//
// Parity status: the reference cannot be compiled or run here (Fortran/OpenACC/CUDA-Fortran with
// nvfortran; the FiNeR submodule is missing) and its tests ship no value-level golden vectors
// (test/reference_1it.md5 pins the md5 of ASCII output only). This restatement is therefore pinned
// by physics known-answers (exact Riemann solution of the Sod problem, conservation on periodic
// meshes, Taylor-Green kinetic-energy decay) -- PARITY WITH THE REFERENCE'S OWN OUTPUT IS UNPINNED.
//
// Each routine cites the reference statements it restates (paths relative to the reference root)
// and keeps their operation order (compile with -ffp-contract=off: no FMA contraction), because
// that order is what fixes the last bits of the result:
//   convective face         src/lib/gpu/conv_physics.inc:1-179, Mod_Convective.f90:288-412
//   limiter                 src/lib/numerics/space/Lib_Limiters.f90:65-97 (Mod_Convective.f90:161-191)
//   AUSM+, LMRoe            src/lib/numerics/fluxes/riemann_open_body.inc:100-150, 679-730, 965-1091
//   LLF, SLAU2, exact,      src/lib/numerics/fluxes/riemann_open_body.inc:244-347, 348-516, 518-676
//   MiczekRoe
//   HLLC, HLLE at records   src/lib/numerics/fluxes/Lib_Riemann_HLL.f90:21-198, 209-310
//   HLLE, SLAU interior     src/lib/gpu/conv_physics.inc:116-159
//   SLAU at records         src/lib/numerics/fluxes/Lib_Riemann.f90:138-197
//   face thermo + viscous   src/lib/numerics/fluxes/Mod_Diffusive.f90:248-373, gpu/diff_cuf_kernels.inc:11-87,
//                           gpu/diff_physics.inc:1-161
//   pass 2                  src/lib/gpu/pass2_body.inc:1-61
//   boundary records        numerics/fluxes/bc/bc_record_body.inc, bc_record_apply.inc, Mod_BC.f90:400-572,
//                           Lib_BC.f90:1770-1867 (connection, Euler), 2113-2178 (connection, viscous),
//                           1119-1165 (extrapolation), 640-737 (symmetry, Euler part of the adiabatic wall),
//                           879-982 (adiabatic wall, viscous), 1519-1597 + 1247-1330 (405 supersonic inlet),
//                           741-861 (symmetry, viscous), 997-1115 (isothermal wall), 1604-1658 + 1166-1240
//                           (406 outlet),
//                           physics/turbulence/Mod_Fluid.f90:20-44 (wall stress)
//   ghost fill              bc/Lib_Extrapolation.f90:558-641 (symmetry, ZG, cubic), 643-730, 859-879, 1023-1191
//   thermo cache            src/lib/physics/Mod_Thermo_Cache.f90:291-425
//   state update            src/lib/gpu/newstate_cons_body.inc:1-89, explicit/Lib_Newstate.f90:257-307,
//                           348-531 (primitive)
//   residual smoothing      explicit/Lib_IRS.f90:57-236
//   RK coefficients         explicit/Lib_RK.f90:6-9; classical RK4 with a conserved accumulator (no reference)
//   local dt                src/lib/gpu/dt_blk.inc:11-222, numerics/time/Mod_dt.f90:15-106
//   thermo leaves           lib/FLINT/src/lib/Lib_ThermoTransport_dev.f90:54-300
//   the step                explicit/Mod_Explicit.f90:52-279
//   residual diagnostic     src/lib/diagnostic/Mod_Diagnostic.f90:64-104, Mod_Explicit.f90:325-358
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include "../include/mose_b200.h"

namespace {

constexpr int GC = MB_GC;
constexpr int NP = MB_NPRIM;
constexpr int IU = 1, IV = 2, IW = 3, IP = 4;  // 0-based nu, nv, nw, np (nsc = 1: species slot 0)
constexpr double RUNIV = 8314.46261815324;     // Lib_ThermoTransport.f90:13

struct Thermo {
  int tmin, tmax;
  double wm, ri;                    // Ri_tab = Runiv / wm_tab (Load_ThermoTransport.f90:54)
  std::vector<double> cp_, h_, mu_, k_;
  const double* cp;  // indexed by the table row (T index), tmin..tmax
  const double* h;
  const double* mu;
  const double* k;
};

struct Blk {
  int n1, n2, n3, pi, pj;
  int64_t boff;
  const double *fm1, *fm2, *fm3, *dl, *m, *vol;
  bool ext = false;  // mb_block.group < 0: a copy of a block another rank owns (its rows are donor values the halo
                     // exchange writes); nothing is computed on it
};

struct Ctx {
  std::vector<Blk> blk;
  std::vector<mb_bc> rec;
  std::vector<mb_conn> conn;
  int64_t ncell;
  mb_scheme sc;
  int sd = 0;               // the shock sensor (sd_dev): 0 none, 1 Tramel, 2 Chen
  Thermo th;
  std::vector<double> pg;  // bc_pg(nprim, 6, nrec) of the connection records
  std::vector<double> acc4; // RK4: the conserved accumulator Un + dt (k1/6 + k2/3 + ...), (ncell, nprim)
  std::vector<double> ur;   // prec: Ur of every row (ur_f; the ghost rows stay 0, Lib_Preconditioning.f90:146-153)
  bool ur_ready = false;    // Ur computed (the first Compute_dt, then after every stage's update)
  mb_status st;
};

inline bool prec_on(const Ctx& c) { return c.sc.intvar == 2; }
inline double ur_at(const Ctx& c, int64_t r) { return prec_on(c) ? c.ur[r] : 0.0; }

// ---- indexing (MOSE_Field_m.f90:78-109; geometry shapes Mod_Convective.f90:594-596) ----
inline int64_t row(const Blk& b, int i, int j, int k) {
  return b.boff + (int64_t)(i + GC - 1) + (int64_t)(j + GC - 1) * b.pi + (int64_t)(k + GC - 1) * b.pi * b.pj;
}
inline int64_t lin(const Blk& b, int i, int j, int k) {
  return (int64_t)(i + GC - 1) + (int64_t)(j + GC - 1) * b.pi + (int64_t)(k + GC - 1) * b.pi * b.pj;
}
inline const double* fm1p(const Blk& b, int i, int j, int k) {  // fm1(1:4, i, j, k), i in 0..n1
  return b.fm1 + 4 * ((int64_t)i + (int64_t)(b.n1 + 1) * ((j - 1) + (int64_t)b.n2 * (k - 1)));
}
inline const double* fm2p(const Blk& b, int i, int j, int k) {
  return b.fm2 + 4 * ((int64_t)(i - 1) + (int64_t)b.n1 * (j + (int64_t)(b.n2 + 1) * (k - 1)));
}
inline const double* fm3p(const Blk& b, int i, int j, int k) {
  return b.fm3 + 4 * ((int64_t)(i - 1) + (int64_t)b.n1 * ((j - 1) + (int64_t)b.n2 * k));
}
inline double dlv(const Blk& b, int d, int i, int j, int k) { return b.dl[d + 3 * lin(b, i, j, k)]; }
inline double mv(const Blk& b, int a, int c, int i, int j, int k) { return b.m[a + 3 * c + 9 * lin(b, i, j, k)]; }

// ---- FLINT leaves ----
// f_tabT_expr: Vij + (Viij - Vij) * Tdiff (Lib_ThermoTransport_dev.f90:306-314)
inline double tabT(const double* t, int ti, double td) { return t[ti] + (t[ti + 1] - t[ti]) * td; }

// The table row of a temperature: int(T), kept inside [tmin, tmax-1]. The reference clamps at some
// call sites and indexes unchecked at others; on the table the two agree, off it (a state the thermo
// guard / state check rejects) the unchecked form reads outside the table, which the engine must
// never do on the GPU, so both the engine and this restatement clamp everywhere (NaN -> tmin).
inline int tidx(const Thermo& th, double T) {
  if (!(T >= (double)th.tmin)) return th.tmin;
  if (T >= (double)(th.tmax - 1)) return th.tmax - 1;
  return (int)T;
}

// co_rotot_Rtot_dev (Lib_ThermoTransport_dev.f90:107-115): rho = sum(rhoi), R = sum(Ri rhoi / rho)
inline void rotot_rtot(const Thermo& th, double rhoi, double& rho, double& R) {
  rho = 0.0 + rhoi;
  R = 0.0 + th.ri * rhoi / rho;
}

// f_cp_dev (Lib_ThermoTransport_dev.f90:280-300)
inline double f_cp(const Thermo& th, double rhoi, int ti, double td, double rho) {
  double cpi = tabT(th.cp, ti, td);
  return 0.0 + rhoi / rho * cpi;
}

// f_ss_dev (Lib_ThermoTransport_dev.f90:76-90): no clamp of the T index
inline double f_ss(const Thermo& th, double rhoi, double p, double rho, double Rtot) {
  double T = p / (Rtot * rho);
  int ti = tidx(th, T);
  double td = T - ti;
  double cp = f_cp(th, rhoi, ti, td, rho);
  double gam = cp / (cp - Rtot);
  return std::sqrt(gam * Rtot * T);
}

// H0_dev (Lib_ThermoTransport_dev.f90:54-73)
inline double H0(const Thermo& th, double p, double rhoi, double u) {
  double rho = 0.0 + rhoi;
  double Rgas = 0.0 + th.ri * rhoi / rho;
  double T = p / (Rgas * rho);
  int ti = tidx(th, T);
  double td = T - ti;
  double e = 0.0 + tabT(th.h, ti, td) * rhoi / rho;
  return e + 0.5 * u * u;
}

// f_molecularWeight + co_fiij_dev + co_k_mi_lam_Wilke_dev for one species
// (Lib_ThermoTransport_dev.f90:118-184, 316-345)
inline void wilke(const Thermo& th, double rhoi, double rho, int ti, double td, double& mil, double& kl) {
  double rho_ = 0.0 + rhoi;
  double wmt = 0.0 + (rhoi / rho_ / th.wm);
  wmt = 1.0 / wmt;
  double xi = rhoi * wmt / (rho * th.wm);
  double mi = tabT(th.mu, ti, td);
  double ki = tabT(th.k, ti, td);
  // co_fiij_dev: Mi_Mj_pow_m025(1,1) = 1, inv_sqrt8_1p(1,1) = 1/sqrt(16)
  double sq_num = std::sqrt(mi);
  double inv_den = 1.0 / std::sqrt(mi + 1e-20);
  const double pw = std::pow(th.wm / th.wm, -0.25);
  const double is8 = 1.0 / std::sqrt(8.0 * (1.0 + th.wm / th.wm));
  double ratio = sq_num * inv_den * pw;
  double one_plus = 1.0 + ratio;
  double fi = one_plus * one_plus * is8;
  double lam_den = 0.0 + xi * fi;
  double inv_ld = 1.0 / lam_den;
  mil = 0.0 + xi * mi * inv_ld;
  kl = 0.0 + xi * ki * inv_ld;
}

// ---- limiter (Lib_Limiters.f90:65-97) ----
inline double rlimiter(int lim, double x, double y) {
  double ru, phi;
  switch (lim) {
    case 1: {
      if (x * y < 0.0) return 0.0;
      double r = x;
      if (std::fabs(x) > std::fabs(y)) r = y;
      return r;
    }
    case 2:
      ru = y / (x + 1e-30);
      phi = (ru + std::fabs(ru)) / (1.0 + std::fabs(ru));
      return phi * x;
    case 3:
      ru = y / (x + 1e-30);
      phi = (ru * ru + ru) / (1.0 + ru * ru);
      return phi * x;
    case 4:
      ru = y / (x + 1e-30);
      phi = std::max(0.0, std::min(std::min(2.0 * ru, 0.5 * (1.0 + ru)), 2.0));
      return phi * x;
    case 5:
      ru = y / (x + 1e-30);
      phi = std::max(std::max(0.0, std::min(2.0 * ru, 1.0)), std::min(ru, 2.0));
      return phi * x;
    default:
      return 0.0;
  }
}

inline double fsign_half(double f) { return std::copysign(0.5, f); }

// SLAU flux from the two states and their total enthalpies h0l / h0r (Liou-Shima: riemann_SLAU_base +
// riemann_SLAU; the statements of conv_physics.inc:125-159 and Lib_Riemann.f90:167-196, which are the same)
void slau_flux(double ul, double vl, double wl, double pl, double al, double dltot, double h0l, double ur, double vr,
               double wr, double pr, double ar, double drtot, double h0r, double unl, double unr, double nx, double ny,
               double nz, double& F_r, double& F_u, double& F_v, double& F_w, double& F_E) {
  double af_ = 0.5 * (al + ar);
  double ml_ = unl / af_, mr_ = unr / af_;
  double mt_ = std::min(1.0, std::sqrt(0.5 * ((ul * ul + vl * vl + wl * wl) + (ur * ur + vr * vr + wr * wr))) / af_);
  double chi_ = (1.0 - mt_) * (1.0 - mt_);
  double vnm_ = (dltot * std::fabs(unl) + drtot * std::fabs(unr)) / (dltot + drtot);
  double frho_ = -std::max(std::min(ml_, 0.0), -1.0) * std::min(std::max(mr_, 0.0), 1.0);
  double vnl_ = (1.0 - frho_) * vnm_ + frho_ * std::fabs(unl);
  double vnr_ = (1.0 - frho_) * vnm_ + frho_ * std::fabs(unr);
  F_r = 0.5 * (dltot * (unl + vnl_) + drtot * (unr - vnr_) - (chi_ / af_) * (pr - pl));
  double bl_, br_;
  if (std::fabs(ml_) < 1.0) bl_ = 0.25 * (2.0 - ml_) * ((ml_ + 1.0) * (ml_ + 1.0));
  else if (ml_ >= 0.0) bl_ = 1.0;
  else bl_ = 0.0;
  if (std::fabs(mr_) < 1.0) br_ = 0.25 * (2.0 + mr_) * ((mr_ - 1.0) * (mr_ - 1.0));
  else if (mr_ >= 0.0) br_ = 0.0;
  else br_ = 1.0;
  double ph_ = 0.5 * (pl + pr) + 0.5 * (bl_ - br_) * (pl - pr) + (1.0 - chi_) * (bl_ + br_ - 1.0) * 0.5 * (pl + pr);
  if (F_r >= 0.0) {
    F_u = F_r * ul + nx * ph_; F_v = F_r * vl + ny * ph_; F_w = F_r * wl + nz * ph_; F_E = F_r * h0l;
  } else {
    F_u = F_r * ur + nx * ph_; F_v = F_r * vr + ny * ph_; F_w = F_r * wr + nz * ph_; F_E = F_r * h0r;
  }
}

// HLLE two-wave flux with the Batten signal speeds S1, S4 (Lib_Riemann_HLL.f90:176-196 = conv_physics.inc:116-124)
void hlle_flux(double ul, double vl, double wl, double pl, double dltot, double h0l, double ur, double vr, double wr,
               double pr, double drtot, double h0r, double unl, double unr, double S1, double S4, double nx, double ny,
               double nz, double& F_r, double& F_u, double& F_v, double& F_w, double& F_E) {
  double inv_denom = 1.0 / (S4 - S1);
  double FrL = dltot * unl, FrR = drtot * unr;
  F_r = (S4 * FrL - S1 * FrR + S1 * S4 * (drtot - dltot)) * inv_denom;
  F_u = (S4 * (FrL * ul + pl * nx) - S1 * (FrR * ur + pr * nx) + S1 * S4 * (drtot * ur - dltot * ul)) * inv_denom;
  F_v = (S4 * (FrL * vl + pl * ny) - S1 * (FrR * vr + pr * ny) + S1 * S4 * (drtot * vr - dltot * vl)) * inv_denom;
  F_w = (S4 * (FrL * wl + pl * nz) - S1 * (FrR * wr + pr * nz) + S1 * S4 * (drtot * wr - dltot * wl)) * inv_denom;
  F_E = (S4 * (FrL * h0l) - S1 * (FrR * h0r) + S1 * S4 * (drtot * (h0r - pr / drtot) - dltot * (h0l - pl / dltot))) *
        inv_denom;
}

// ---- the MOSE_open solvers of riemann_open_body.inc used here: AUSM+ (4), LLF (8), SLAU2 (9), LMRoe (12) ----
// Thermo as written there: T clamped to [tmin, tmax-1] before the table lookup (H / H0 of FLINT).
inline double h_static(const Thermo& th, double rhoi, double p) {
  double rho_ = 0.0 + rhoi;
  double rg = 0.0 + th.ri * rhoi / rho_;
  double T = p / (rg * rho_);
  double Tc = std::max((double)th.tmin, std::min(T, (double)(th.tmax - 1)));
  int ti = (int)Tc;
  double td = Tc - ti;
  int t1 = std::max(th.tmin, std::min(ti, th.tmax));
  int t2 = std::max(th.tmin, std::min(ti + 1, th.tmax));
  double hs = th.h[t1] + (th.h[t2] - th.h[t1]) * td;
  return 0.0 + hs * rhoi / rho_;
}

// gamma of a state as riemann_open_body.inc writes f_gamma out (:349-366): T from p / (R rho_tot), the table row
// int(T) with both rows held to the table
inline double gam_state(const Thermo& th, double d, double p, double dtot) {
  double rho_ = 0.0 + d;
  double rg_ = 0.0 + th.ri * d / rho_;
  double T_ = p / (rg_ * dtot);
  int Ti = (int)T_;
  double Td = T_ - Ti;
  int t1 = std::max(th.tmin, std::min(Ti, th.tmax)), t2 = std::max(th.tmin, std::min(Ti + 1, th.tmax));
  double cp_ = 0.0 + d / dtot * (th.cp[t1] + (th.cp[t2] - th.cp[t1]) * Td);
  return cp_ / (cp_ - rg_);
}

void riemann_open(const Thermo& th, int rs, double mco, double bet, double dl, double ul, double vl, double wl,
                  double pl, double al, double dltot, double dr, double ur, double vr, double wr, double pr,
                  double ar, double drtot, double nx, double ny, double nz, double& F_r, double& F_u,
                  double& F_v, double& F_w, double& F_E, double urL_ = 0.0, double urR_ = 0.0) {
  double unl = ul * nx + vl * ny + wl * nz;
  double unr = ur * nx + vr * ny + wr * nz;
  if (rs == 14) {  // HLLC-PC (riemann_open_body.inc:1092-1175, Riemann_HLLCprec): HLLC Batten with the signal speeds of
                   // the preconditioned system, Vr = min(Ur, a) of each side and of the sqrt(rho) average
    const double hL = h_static(th, dl, pl), hR = h_static(th, dr, pr);
    const double eL = hL - pl / dltot, eR = hR - pr / drtot;
    const double h0l = hL + 0.5 * (ul * ul + vl * vl + wl * wl), h0r = hR + 0.5 * (ur * ur + vr * vr + wr * wr);
    const double EtL = eL + 0.5 * (ul * ul + vl * vl + wl * wl), EtR = eR + 0.5 * (ur * ur + vr * vr + wr * wr);
    const double FrL = dltot * unl;
    const double Ful = FrL * ul + pl * nx, Fvl = FrL * vl + pl * ny, Fwl = FrL * wl + pl * nz, Fel = FrL * h0l;
    const double FrR = drtot * unr;
    const double Fur = FrR * ur + pr * nx, Fvr = FrR * vr + pr * ny, Fwr = FrR * wr + pr * nz, Fer = FrR * h0r;
    const double srL = std::sqrt(dltot), srR = std::sqrt(drtot), den = srL + srR;
    const double u_roe = (srL * ul + srR * ur) / den, v_roe = (srL * vl + srR * vr) / den;
    const double w_roe = (srL * wl + srR * wr) / den, a_roe = (srL * al + srR * ar) / den;
    const double un_roe = u_roe * nx + v_roe * ny + w_roe * nz;
    const double VrL = std::min(urL_, al), VrR = std::min(urR_, ar), VrRoe = (srL * VrL + srR * VrR) / den;
    const double alL = (1.0 - (VrL * VrL) / (al * al)) / 2.0, alR = (1.0 - (VrR * VrR) / (ar * ar)) / 2.0;
    const double alRoe = (1.0 - (VrRoe * VrRoe) / (a_roe * a_roe)) / 2.0;
    const double vLs = unl * (1.0 - alL), vRs = unr * (1.0 - alR), vRoes = un_roe * (1.0 - alRoe);
    const double cLs = std::sqrt(std::max(alL * alL * (unl * unl) + VrL * VrL, 0.0));
    const double cRs = std::sqrt(std::max(alR * alR * (unr * unr) + VrR * VrR, 0.0));
    const double cRoes = std::sqrt(std::max(alRoe * alRoe * (un_roe * un_roe) + VrRoe * VrRoe, 0.0));
    const double S1 = std::min(std::min(0.0, vLs - cLs), vRoes - cRoes);
    const double S4 = std::max(std::max(0.0, vRs + cRs), vRoes + cRoes);
    const double Sstar = (pr - pl + dltot * unl * (S1 - unl) - drtot * unr * (S4 - unr)) /
                         (dltot * (S1 - unl) - drtot * (S4 - unr));
    const double pstar = dltot * (unl - S1) * (unl - Sstar) + pl;
    if (S1 >= 0.0) {
      F_r = FrL; F_u = Ful; F_v = Fvl; F_w = Fwl; F_E = Fel;
    } else if (S4 <= 0.0) {
      F_r = FrR; F_u = Fur; F_v = Fvr; F_w = Fwr; F_E = Fer;
    } else if (Sstar >= 0.0) {
      const double q = S1 - Sstar;
      const double U1S = dltot * (S1 - unl) / q;
      const double U2S = ((S1 - unl) * dltot * ul + (pstar - pl) * nx) / q;
      const double U3S = ((S1 - unl) * dltot * vl + (pstar - pl) * ny) / q;
      const double U4S = ((S1 - unl) * dltot * wl + (pstar - pl) * nz) / q;
      const double U5S = ((S1 - unl) * dltot * EtL - pl * unl + pstar * Sstar) / q;
      F_r = FrL + S1 * (U1S - dltot); F_u = Ful + S1 * (U2S - dltot * ul); F_v = Fvl + S1 * (U3S - dltot * vl);
      F_w = Fwl + S1 * (U4S - dltot * wl); F_E = Fel + S1 * (U5S - dltot * EtL);
    } else {
      const double q = S4 - Sstar;
      const double U1S = drtot * (S4 - unr) / q;
      const double U2S = ((S4 - unr) * drtot * ur + (pstar - pr) * nx) / q;
      const double U3S = ((S4 - unr) * drtot * vr + (pstar - pr) * ny) / q;
      const double U4S = ((S4 - unr) * drtot * wr + (pstar - pr) * nz) / q;
      const double U5S = ((S4 - unr) * drtot * EtR - pr * unr + pstar * Sstar) / q;
      F_r = FrR + S4 * (U1S - drtot); F_u = Fur + S4 * (U2S - drtot * ur); F_v = Fvr + S4 * (U3S - drtot * vr);
      F_w = Fwr + S4 * (U4S - drtot * wr); F_E = Fer + S4 * (U5S - drtot * EtR);
    }
    return;
  }
  if (rs == 4) {  // riemann_open_body.inc:100-150
    const double ab = 0.125, aa = 0.1875;
    double vel = std::sqrt(ul * ul + vl * vl + wl * wl);
    double H_L = h_static(th, dl, pl) + 0.5 * vel * vel;
    vel = std::sqrt(ur * ur + vr * vr + wr * wr);
    double H_R = h_static(th, dr, pr) + 0.5 * vel * vel;
    double a_half = std::sqrt(al * ar);
    double ML = unl / a_half, MR = unr / a_half;
    double MplusL, pplusL, MminusR, pminusR;
    if (std::fabs(ML) < 1.0) {
      MplusL = 0.25 * ((ML + 1.0) * (ML + 1.0)) + ab * ((ML * ML - 1.0) * (ML * ML - 1.0));
      pplusL = 0.25 * ((ML + 1.0) * (ML + 1.0)) * (2.0 - ML) + aa * ML * ((ML * ML - 1.0) * (ML * ML - 1.0));
    } else {
      MplusL = 0.5 * (ML + std::fabs(ML));
      pplusL = 0.5 * (1.0 + std::copysign(1.0, ML));
    }
    if (std::fabs(MR) < 1.0) {
      MminusR = -0.25 * ((MR - 1.0) * (MR - 1.0)) - ab * ((MR * MR - 1.0) * (MR * MR - 1.0));
      pminusR = 0.25 * ((MR - 1.0) * (MR - 1.0)) * (2.0 + MR) - aa * MR * ((MR * MR - 1.0) * (MR * MR - 1.0));
    } else {
      MminusR = 0.5 * (MR - std::fabs(MR));
      pminusR = 0.5 * (1.0 - std::copysign(1.0, MR));
    }
    double Mhalf = MplusL + MminusR;
    double phalf = pplusL * pl + pminusR * pr;
    double mdotp = dltot * a_half * 0.5 * (Mhalf + std::fabs(Mhalf));
    double mdotm = drtot * a_half * 0.5 * (Mhalf - std::fabs(Mhalf));
    F_r = mdotp + mdotm;
    F_u = mdotp * ul + mdotm * ur + nx * phalf;
    F_v = mdotp * vl + mdotm * vr + ny * phalf;
    F_w = mdotp * wl + mdotm * wr + nz * phalf;
    F_E = mdotp * H_L + mdotm * H_R;
    return;
  }
  if (rs == 5) {  // AUSM+M (riemann_open_body.inc:152-242, Chen et al. 2020): the AUSMPW+ sound speed, Mach-number
                  // function f and the shock gate g of the face sensor bet
    const double ab = 0.125, aa = 0.1875, pi_ = 3.141592653589793;
    double Vl2 = ul * ul + vl * vl + wl * wl, Vr2 = ur * ur + vr * vr + wr * wr;
    double Hs_L = h_static(th, dl, pl);
    double vel_ = std::sqrt(Vl2);
    double H_L = Hs_L + 0.5 * vel_ * vel_;
    double gam_L = gam_state(th, dl, pl, dltot);
    double Hs_R = h_static(th, dr, pr);
    vel_ = std::sqrt(Vr2);
    double H_R = Hs_R + 0.5 * vel_ * vel_;
    double gam_R = gam_state(th, dr, pr, drtot);
    double gam = 0.5 * (gam_L + gam_R);
    double hnorm = 0.5 * (Hs_L + Hs_R);
    double cs = std::sqrt(2.0 * (gam - 1.0) / (gam + 1.0) * hnorm);
    double c12 = (unl + unr >= 0.0) ? cs * cs / std::max(std::fabs(unl), cs) : cs * cs / std::max(std::fabs(unr), cs);
    double ML = unl / c12, MR = unr / c12;
    double MplusL, pplusL, MminusR, pminusR;
    if (std::fabs(ML) < 1.0) {
      MplusL = 0.25 * ((ML + 1.0) * (ML + 1.0)) + ab * ((ML * ML - 1.0) * (ML * ML - 1.0));
      pplusL = 0.25 * ((ML + 1.0) * (ML + 1.0)) * (2.0 - ML) + aa * ML * ((ML * ML - 1.0) * (ML * ML - 1.0));
    } else {
      MplusL = 0.5 * (ML + std::fabs(ML));
      pplusL = 0.5 * (1.0 + std::copysign(1.0, ML));
    }
    if (std::fabs(MR) < 1.0) {
      MminusR = -0.25 * ((MR - 1.0) * (MR - 1.0)) - ab * ((MR * MR - 1.0) * (MR * MR - 1.0));
      pminusR = 0.25 * ((MR - 1.0) * (MR - 1.0)) * (2.0 + MR) - aa * MR * ((MR * MR - 1.0) * (MR * MR - 1.0));
    } else {
      MminusR = 0.5 * (MR - std::fabs(MR));
      pminusR = 0.5 * (1.0 - std::copysign(1.0, MR));
    }
    double f_ = 0.5 * (1.0 - std::cos(pi_ * std::min(1.0, std::max(std::fabs(ML), std::fabs(MR)))));
    double g_ = 0.5 * (1.0 + std::cos(pi_ * bet));
    double rho12 = 0.5 * (dltot + drtot);
    double Mp = -0.5 * (1.0 - f_) * (pr - pl) / (rho12 * c12 * c12) * (1.0 - g_);
    double M12 = MplusL + MminusR + Mp;
    double mdot = M12 * c12 * ((M12 >= 0.0) ? dltot : drtot);
    double fo = std::min(1.0, std::max(f_, mco));
    double ps = 0.5 * (pl + pr) + 0.5 * (pplusL - pminusR) * (pl - pr) + fo * (pplusL + pminusR - 1.0) * 0.5 * (pl + pr);
    double gfac = g_ * gam * (pl + pr) / (2.0 * c12) * pplusL * pminusR;
    double pux = -gfac * (ur - ul), puy = -gfac * (vr - vl), puz = -gfac * (wr - wl);
    F_r = mdot;
    if (M12 >= 0.0) {
      F_u = mdot * ul + ps * nx + pux; F_v = mdot * vl + ps * ny + puy; F_w = mdot * wl + ps * nz + puz; F_E = mdot * H_L;
    } else {
      F_u = mdot * ur + ps * nx + pux; F_v = mdot * vr + ps * ny + puy; F_w = mdot * wr + ps * nz + puz; F_E = mdot * H_R;
    }
    return;
  }
  if (rs == 11) {  // exact Godunov (riemann_open_body.inc:348-516): Newton on the star velocity, gamma of each state
    double gam_L = gam_state(th, dl, pl, dltot), gam_R = gam_state(th, dr, pr, drtot);
    double gm1 = gam_L - 1.0, gm4 = gam_R - 1.0;
    double d1 = 0.5 * gm1, d4 = 0.5 * gm4;
    double e1 = gam_L / d1, e4 = gam_R / d4;
    double un1 = ul * nx + vl * ny + wl * nz;
    double ut1 = ul - un1 * nx, vt1 = vl - un1 * ny, wt1 = wl - un1 * nz;
    double un4 = ur * nx + vr * ny + wr * nz;
    double ut4 = ur - un4 * nx, vt4 = vr - un4 * ny, wt4 = wr - un4 * nz;
    double r2i = un1 + (2.0 / gm1) * al;
    double r1iv = un4 - (2.0 / gm4) * ar;
    double dum = (pl < pr) ? gm4 / (2.0 * gam_R) : gm1 / (2.0 * gam_L);
    double z = (gm1 / gm4) * (ar / al) * std::pow(pl / pr, dum);
    double vel = (z * r2i + r1iv) / (1.0 + z);
    double p3 = 1.0, p2 = 2.0 * p3, dpr = 0.0, dpl = 0.0;
    int iter = 0;
    double swl = 0.0, swr = 0.0, vw1 = 0.0, vw2 = 0.0, vw3 = 0.0, vw4 = 0.0, a2 = al, a3 = ar;
    while (std::fabs(1.0 - (p2 / p3)) >= 1e-5 && iter <= 1000) {
      if (vel < un1) {  // shock on the left
        double x = (gam_L + 1.0) * (vel - un1) / (4.0 * al);
        double mrel = x - std::sqrt(1.0 + x * x);
        double c = gam_L * pl / al;
        p2 = pl + c * (vel - un1) * mrel;
        dpr = 2.0 * c * std::pow(mrel, 3.0) / (1.0 + mrel * mrel);
        double rp = p2 / pl;
        swl = un1 + al * mrel;
        a2 = al * std::sqrt((gam_L + 1.0 + (gam_L - 1.0) * rp) / (gam_L + 1.0 + (gam_L - 1.0) / rp));
      } else {  // rarefaction on the left
        double delta = 0.5 * (gam_L - 1.0);
        double dum1 = 2.0 * gam_L / (gam_L - 1.0);
        a2 = al - delta * (vel - un1);
        p2 = pl * std::pow(a2 / al, dum1);
        dpr = -gam_L * p2 / a2;
        vw1 = un1 - al;
        vw2 = vel - a2;
      }
      if (vel > un4) {  // shock on the right
        double x = (gam_R + 1.0) * (vel - un4) / (4.0 * ar);
        double mrel = x + std::sqrt(1.0 + x * x);
        double c = gam_R * pr / ar;
        p3 = pr + c * (vel - un4) * mrel;
        dpl = 2.0 * c * std::pow(mrel, 3.0) / (1.0 + mrel * mrel);
        double rp = p3 / pr;
        swr = un4 + ar * mrel;
        a3 = ar * std::sqrt((gam_R + 1.0 + (gam_R - 1.0) * rp) / (gam_R + 1.0 + (gam_R - 1.0) / rp));
      } else {  // rarefaction on the right
        double delta = 0.5 * (gam_R - 1.0);
        double dum1 = 2.0 * gam_R / (gam_R - 1.0);
        a3 = ar + delta * (vel - un4);
        p3 = pr * std::pow(a3 / ar, dum1);
        dpl = gam_R * p3 / a3;
        vw3 = vel + a3;
        vw4 = un4 + ar;
      }
      vel = vel - ((p2 - p3) / (dpr - dpl));
      iter = iter + 1;
    }
    double af, pf, rhof, uf, vf, wf, Hs;
    if (vel > 0.0) {
      af = a2; pf = p2;
      if (vel <= un1) {
        if (swl > 0.0) { af = al; vel = un1; pf = pl; }
      } else if (vw1 > 0.0) {
        vel = un1; af = al; pf = pl;
      } else if (vw2 > 0.0) {
        af = (un1 + al / d1) / (1.0 + 1.0 / d1);
        vel = af;
        pf = pl * std::pow(af / al, e1);
      }
      rhof = gam_L * pf / (af * af);
      uf = vel * nx + ut1; vf = vel * ny + vt1; wf = vel * nz + wt1;
      Hs = h_static(th, dl / dltot * rhof, pf);
    } else {
      af = a3; pf = p3;
      if (vel >= un4) {
        if (swr < 0.0) { af = ar; vel = un4; pf = pr; }
      } else if (vw4 < 0.0) {
        af = ar; vel = un4; pf = pr;
      } else if (vw3 < 0.0) {
        af = -(un4 - ar / d4) / (1.0 + 1.0 / d4);
        vel = -af;
        pf = pr * std::pow(af / ar, e4);
      }
      rhof = gam_R * pf / (af * af);
      uf = vel * nx + ut4; vf = vel * ny + vt4; wf = vel * nz + wt4;
      Hs = h_static(th, dr / drtot * rhof, pf);
    }
    F_r = rhof * vel;
    F_u = F_r * uf + pf * nx;
    F_v = F_r * vf + pf * ny;
    F_w = F_r * wf + pf * nz;
    double uu = std::sqrt(vel * vel);
    F_E = F_r * (Hs + 0.5 * uu * uu);
    return;
  }
  if (rs == 13) {  // MiczekRoe (riemann_open_body.inc:518-676): the Miczek et al. 2015 preconditioned Roe flux
    double nmag = std::sqrt(nx * nx + ny * ny + nz * nz);
    if (nmag <= 0.0) { F_r = 0.0; F_u = 0.0; F_v = 0.0; F_w = 0.0; F_E = 0.0; return; }
    double n1 = nx / nmag, n2 = ny / nmag, n3 = nz / nmag;
    double tx = 1.0, ty = 0.0, tz = 0.0;
    if (!(std::fabs(n1) < 0.9)) { tx = 0.0; ty = 1.0; }
    double dot = tx * n1 + ty * n2 + tz * n3;
    double t1x = tx - dot * n1, t1y = ty - dot * n2, t1z = tz - dot * n3;
    double tmag = std::sqrt(t1x * t1x + t1y * t1y + t1z * t1z);
    if (tmag <= 0.0) {
      t1x = -n2; t1y = n1; t1z = 0.0;
      tmag = std::sqrt(t1x * t1x + t1y * t1y + t1z * t1z);
    }
    t1x = t1x / tmag; t1y = t1y / tmag; t1z = t1z / tmag;
    double t2x = n2 * t1z - n3 * t1y, t2y = n3 * t1x - n1 * t1z, t2z = n1 * t1y - n2 * t1x;
    double unL = ul * n1 + vl * n2 + wl * n3, unR = ur * n1 + vr * n2 + wr * n3;
    double ut1L = ul * t1x + vl * t1y + wl * t1z, ut1R = ur * t1x + vr * t1y + wr * t1z;
    double ut2L = ul * t2x + vl * t2y + wl * t2z, ut2R = ur * t2x + vr * t2y + wr * t2z;
    double hL = h_static(th, dl, pl), hR = h_static(th, dr, pr);
    double H0L = hL + 0.5 * (ul * ul + vl * vl + wl * wl);
    double H0R = hR + 0.5 * (ur * ur + vr * vr + wr * wr);
    double FL1 = dltot * unL, FL2 = dltot * unL * ul + pl * n1, FL3 = dltot * unL * vl + pl * n2,
           FL4 = dltot * unL * wl + pl * n3, FL5 = dltot * unL * H0L;
    double FR1 = drtot * unR, FR2 = drtot * unR * ur + pr * n1, FR3 = drtot * unR * vr + pr * n2,
           FR4 = drtot * unR * wr + pr * n3, FR5 = drtot * unR * H0R;
    double sRL = std::sqrt(dltot), sRR = std::sqrt(drtot), den = sRL + sRR;
    double u = (sRL * ul + sRR * ur) / den, v = (sRL * vl + sRR * vr) / den, w = (sRL * wl + sRR * wr) / den;
    double H = (sRL * H0L + sRR * H0R) / den;
    double un = u * n1 + v * n2 + w * n3;
    double rho = sRL * sRR;
    double u2 = u * u + v * v + w * w;
    double gam_L = gam_state(th, dl, pl, dltot), gam_R = gam_state(th, dr, pr, drtot);
    double kL = gam_L - 1.0, kR = gam_R - 1.0;
    double chiL = al * al - kL * hL, chiR = ar * ar - kR * hR;
    double kRoe = (sRL * kL + sRR * kR) / den, chiRoe = (sRL * chiL + sRR * chiR) / den;
    double cc = std::sqrt(std::max(1e-30, chiRoe + kRoe * (H - 0.5 * u2)));
    double Mcut = std::max(1e-6, mco);
    double Mloc = std::sqrt(u2) / cc;
    double mu = std::min(1.0, std::max(Mloc, Mcut));
    double del = 1.0 / mu - 1.0, del2 = del * del, om = 1.0 / (1.0 + del2);
    double drho = drtot - dltot, dp = pr - pl, dun = unR - unL, dut1 = ut1R - ut1L, dut2 = ut2R - ut2L;
    double p11 = un, p12 = rho * (1.0 + del * un / cc), p13 = del / cc, p22 = un - del * cc;
    double p23 = (1.0 - del * un / cc) / rho, p32 = rho * cc * (cc + del * un), p33 = un + cc * del;
    double s2 = (1.0 + del2) * cc * cc - del2 * un * un;
    double s = std::sqrt(std::max(1e-30, s2));
    s2 = s * s;
    double le = un, lp = un + s, lm = un - s;
    double va1 = (p11 - lm) * drho + p12 * dun + p13 * dp, va2 = (p22 - lm) * dun + p23 * dp,
           va3 = p32 * dun + (p33 - lm) * dp;
    double vb1 = (p11 - lp) * drho + p12 * dun + p13 * dp, vb2 = (p22 - lp) * dun + p23 * dp,
           vb3 = p32 * dun + (p33 - lp) * dp;
    double w1 = (p11 - lp) * va1 + p12 * va2 + p13 * va3, w2 = (p22 - lp) * va2 + p23 * va3,
           w3 = p32 * va2 + (p33 - lp) * va3;
    double x1 = (p11 - le) * va1 + p12 * va2 + p13 * va3, x2 = (p22 - le) * va2 + p23 * va3,
           x3 = p32 * va2 + (p33 - le) * va3;
    double z1 = (p11 - le) * vb1 + p12 * vb2 + p13 * vb3, z2 = (p22 - le) * vb2 + p23 * vb3,
           z3 = p32 * vb2 + (p33 - le) * vb3;
    double c1 = std::fabs(le) / (-s2), c2 = std::fabs(lp) / (2.0 * s2), c3 = std::fabs(lm) / (2.0 * s2);
    double g1 = c1 * w1 + c2 * x1 + c3 * z1, g2 = c1 * w2 + c2 * x2 + c3 * z2, g3 = c1 * w3 + c2 * x3 + c3 * z3;
    double ddrho = g1 - (rho * del / cc) * om * g2 - (del2 / (cc * cc)) * om * g3;
    double ddun = om * (g2 + (del / (rho * cc)) * g3);
    double ddp = om * (-rho * cc * del * g2 + g3);
    double ddut1 = std::fabs(un) * dut1, ddut2 = std::fabs(un) * dut2;
    double ddux = ddun * n1 + ddut1 * t1x + ddut2 * t2x;
    double dduy = ddun * n2 + ddut1 * t1y + ddut2 * t2y;
    double dduz = ddun * n3 + ddut1 * t1z + ddut2 * t2z;
    F_r = 0.5 * (FL1 + FR1) - 0.5 * (ddrho);
    F_u = 0.5 * (FL2 + FR2) - 0.5 * (u * ddrho + rho * ddux);
    F_v = 0.5 * (FL3 + FR3) - 0.5 * (v * ddrho + rho * dduy);
    F_w = 0.5 * (FL4 + FR4) - 0.5 * (w * ddrho + rho * dduz);
    F_E = 0.5 * (FL5 + FR5) - 0.5 * (0.5 * u2 * ddrho + rho * (u * ddux + v * dduy + w * dduz) + ddp / kRoe);
    return;
  }
  if (rs == 8) {  // LLF / Rusanov (riemann_open_body.inc:244-278)
    double lf_a = std::max(std::max(std::fabs(unl - al), std::fabs(unr - ar)),
                           std::max(std::fabs(unl + al), std::fabs(unr + ar)));
    double rho_ = 0.0 + dr;
    double Hs_R = h_static(th, dr, pr);
    double vel_ = std::sqrt(ur * ur + vr * vr + wr * wr);
    double FrR = rho_ * (ur * nx + vr * ny + wr * nz);
    double Fur = FrR * ur + pr * nx, Fvr = FrR * vr + pr * ny, Fwr = FrR * wr + pr * nz;
    double Fer = FrR * (Hs_R + 0.5 * vel_ * vel_);
    double e0r_ = (Hs_R - pr / rho_) + 0.5 * vel_ * vel_;
    rho_ = 0.0 + dl;
    double Hs_L = h_static(th, dl, pl);
    vel_ = std::sqrt(ul * ul + vl * vl + wl * wl);
    double FrL = rho_ * (ul * nx + vl * ny + wl * nz);
    double Ful = FrL * ul + pl * nx, Fvl = FrL * vl + pl * ny, Fwl = FrL * wl + pl * nz;
    double Fel = FrL * (Hs_L + 0.5 * vel_ * vel_);
    double e0l_ = (Hs_L - pl / rho_) + 0.5 * vel_ * vel_;
    F_r = 0.5 * (FrL + FrR - lf_a * (drtot - dltot));
    F_u = 0.5 * (Fur + Ful - lf_a * (drtot * ur - dltot * ul));
    F_v = 0.5 * (Fvr + Fvl - lf_a * (drtot * vr - dltot * vl));
    F_w = 0.5 * (Fwr + Fwl - lf_a * (drtot * wr - dltot * wl));
    F_E = 0.5 * (Fel + Fer - lf_a * (drtot * e0r_ - dltot * e0l_));
    return;
  }
  if (rs == 9) {  // SLAU2 (riemann_open_body.inc:280-347): SLAU with the Kitamura-Shima 2013 pressure flux
    double Vl2 = ul * ul + vl * vl + wl * wl;
    double Vr2 = ur * ur + vr * vr + wr * wr;
    double af = 0.5 * (al + ar);
    double ml = unl / af, mr = unr / af;
    double mt = std::min(1.0, std::sqrt(0.5 * (Vl2 + Vr2)) / af);
    double chi = (1.0 - mt) * (1.0 - mt);
    double vnm = (dltot * std::fabs(unl) + drtot * std::fabs(unr)) / (dltot + drtot);
    double frho = -std::max(std::min(ml, 0.0), -1.0) * std::min(std::max(mr, 0.0), 1.0);
    double vnl = (1.0 - frho) * vnm + frho * std::fabs(unl);
    double vnr = (1.0 - frho) * vnm + frho * std::fabs(unr);
    F_r = 0.5 * (dltot * (unl + vnl) + drtot * (unr - vnr) - (chi / af) * (pr - pl));
    F_r = std::max(-1.0e150, std::min(F_r, 1.0e150));
    double bl, br;
    if (std::fabs(ml) < 1.0) bl = 0.25 * (2.0 - ml) * ((ml + 1.0) * (ml + 1.0));
    else if (ml >= 0.0) bl = 1.0;
    else bl = 0.0;
    if (std::fabs(mr) < 1.0) br = 0.25 * (2.0 + mr) * ((mr - 1.0) * (mr - 1.0));
    else if (mr >= 0.0) br = 0.0;
    else br = 1.0;
    double ph = 0.5 * (pl + pr) + 0.5 * (bl - br) * (pl - pr) +
                std::sqrt(0.5 * (Vl2 + Vr2)) * (bl + br - 1.0) * af * 0.5 * (dltot + drtot);
    ph = std::max(-1.0e150, std::min(ph, 1.0e150));
    double Hs_L = h_static(th, dl, pl);
    double Hs_R = h_static(th, dr, pr);
    double H_L = Hs_L + 0.5 * std::sqrt(Vl2) * std::sqrt(Vl2);
    double H_R = Hs_R + 0.5 * std::sqrt(Vr2) * std::sqrt(Vr2);
    H_L = std::max(-1.0e150, std::min(H_L, 1.0e150));
    H_R = std::max(-1.0e150, std::min(H_R, 1.0e150));
    if (F_r >= 0.0) {
      F_u = F_r * ul + nx * ph; F_v = F_r * vl + ny * ph; F_w = F_r * wl + nz * ph; F_E = F_r * H_L;
    } else {
      F_u = F_r * ur + nx * ph; F_v = F_r * vr + ny * ph; F_w = F_r * wr + nz * ph; F_E = F_r * H_R;
    }
    return;
  }
  // rs 6, 7, 10, 12: Roe averages (riemann_open_body.inc:679-730), then HLLE++, HLLC+Tramel, HLLC+Chen or LMRoe
  double rho_ = 0.0 + dl;
  double Rl = 0.0 + th.ri * dl / rho_;
  rho_ = 0.0 + dr;
  double Rr = 0.0 + th.ri * dr / rho_;
  double inv_dltot = 1.0 / dltot, inv_drtot = 1.0 / drtot;
  double Tl = pl * inv_dltot / Rl, Tr = pr * inv_drtot / Rr;
  int Til = tidx(th, Tl);
  int Tir = tidx(th, Tr);
  double dTl = Tl - Til, dTr = Tr - Tir;
  double srL = std::sqrt(dltot), srR = std::sqrt(drtot);
  double inv_sr = 1.0 / (srL + srR);
  double rho_roe = srL * srR;
  double u_roe = (srR * ur + srL * ul) * inv_sr;
  double v_roe = (srR * vr + srL * vl) * inv_sr;
  double w_roe = (srR * wr + srL * wl) * inv_sr;
  double R_roe = (srR * Rr + srL * Rl) * inv_sr;
  double T_roe = (srR * Tr + srL * Tl) * inv_sr;
  double h0l = 0.0, h0r = 0.0, cv_roe = 0.0, sum_ei = 0.0;
  {
    double invW = RUNIV / th.wm;
    double hl = th.h[Til] + (th.h[Til + 1] - th.h[Til]) * dTl;
    double hr = th.h[Tir] + (th.h[Tir + 1] - th.h[Tir]) * dTr;
    double el = hl - invW * Tl, er = hr - invW * Tr;
    h0l = h0l + hl * dl * inv_dltot;
    h0r = h0r + hr * dr * inv_drtot;
    double d_roe = (srR * dr * inv_drtot + srL * dl * inv_dltot) * inv_sr;
    cv_roe = cv_roe + d_roe * (0.5 * (th.cp[Til] + (th.cp[Til + 1] - th.cp[Til]) * dTl + th.cp[Tir] +
                                      (th.cp[Tir + 1] - th.cp[Tir]) * dTr) - invW);
    sum_ei = sum_ei + d_roe * (srR * er + srL * el) * inv_sr;
  }
  h0l = h0l + 0.5 * (ul * ul + vl * vl + wl * wl);
  h0r = h0r + 0.5 * (ur * ur + vr * vr + wr * wr);
  double h0_roe = (srR * h0r + srL * h0l) * inv_sr;
  double gam_roe = 1.0 + R_roe / cv_roe;
  double vel2 = u_roe * u_roe + v_roe * v_roe + w_roe * w_roe;
  double a_roe = std::sqrt((gam_roe - 1.0) * (h0_roe - 0.5 * vel2 + cv_roe * T_roe - sum_ei));
  double un_roe = u_roe * nx + v_roe * ny + w_roe * nz;
  if (rs == 6) {  // HLLE++ (riemann_open_body.inc:728-810): HLLE and Roe wave speeds blended by the face sensor
    double S1 = std::min(std::min(0.0, unl - al), un_roe - a_roe);
    double S4 = std::max(std::max(0.0, unr + ar), un_roe + a_roe);
    double inv_denom = 1.0 / (S4 - S1);
    double lam1_hlle = std::fabs((S4 + S1) * un_roe * inv_denom - 2.0 * S4 * S1 * inv_denom);
    double lam2_hlle = std::fabs((S4 + S1) * (un_roe - a_roe) * inv_denom - 2.0 * S4 * S1 * inv_denom);
    double lam3_hlle = std::fabs((S4 + S1) * (un_roe + a_roe) * inv_denom - 2.0 * S4 * S1 * inv_denom);
    double eps_ = 0.3 * (std::fabs(un_roe) + a_roe);
    double lam1_roe = std::fabs(un_roe);
    double vv = un_roe - a_roe;
    double lam2_roe = std::fabs(vv);
    if (std::fabs(vv) <= eps_) lam2_roe = (vv * vv + eps_ * eps_) / (2.0 * eps_);
    vv = un_roe + a_roe;
    double lam3_roe = std::fabs(vv);
    if (std::fabs(vv) <= eps_) lam3_roe = (vv * vv + eps_ * eps_) / (2.0 * eps_);
    double lam1_pp = bet * lam1_roe + (1.0 - bet) * lam1_hlle;
    double lam2_pp = bet * lam2_roe + (1.0 - bet) * lam2_hlle;
    double lam3_pp = bet * lam3_roe + (1.0 - bet) * lam3_hlle;
    double rL = 0.0 + dl;
    double FrL = rL * (ul * nx + vl * ny + wl * nz);
    double Ful = FrL * ul + pl * nx, Fvl = FrL * vl + pl * ny, Fwl = FrL * wl + pl * nz;
    double Hs_L = h_static(th, dl, pl);
    double vel_ = std::sqrt(ul * ul + vl * vl + wl * wl);
    double Fel = FrL * (Hs_L + 0.5 * vel_ * vel_);
    double rR = 0.0 + dr;
    double FrR = rR * (ur * nx + vr * ny + wr * nz);
    double Fur = FrR * ur + pr * nx, Fvr = FrR * vr + pr * ny, Fwr = FrR * wr + pr * nz;
    double Hs_R = h_static(th, dr, pr);
    vel_ = std::sqrt(ur * ur + vr * vr + wr * wr);
    double Fer = FrR * (Hs_R + 0.5 * vel_ * vel_);
    F_r = 0.5 * (FrL + FrR); F_u = 0.5 * (Ful + Fur); F_v = 0.5 * (Fvl + Fvr); F_w = 0.5 * (Fwl + Fwr);
    F_E = 0.5 * (Fel + Fer);
    double drho = drtot - dltot, dp = pr - pl, du = ur - ul, dv = vr - vl, dw = wr - wl, dun = unr - unl;
    double t1x, t1y, t1z;
    if (std::fabs(nx) < 0.9) { t1x = 0.0; t1y = -nz; t1z = ny; } else { t1x = -nz; t1y = 0.0; t1z = nx; }
    double normt = std::sqrt(t1x * t1x + t1y * t1y + t1z * t1z);
    t1x = t1x / normt; t1y = t1y / normt; t1z = t1z / normt;
    double t2x = ny * t1z - nz * t1y, t2y = nz * t1x - nx * t1z, t2z = nx * t1y - ny * t1x;
    double alpha_m = (dp - rho_roe * a_roe * dun) / (2.0 * a_roe * a_roe);
    double alpha_c = drho - dp / (a_roe * a_roe);
    double alpha_s1 = rho_roe * (du * t1x + dv * t1y + dw * t1z);
    double alpha_s2 = rho_roe * (du * t2x + dv * t2y + dw * t2z);
    double alpha_p = (dp + rho_roe * a_roe * dun) / (2.0 * a_roe * a_roe);
    F_r = F_r - 0.5 * (alpha_c * lam1_pp + alpha_m * lam2_pp + alpha_p * lam3_pp);
    F_u = F_u - 0.5 * (alpha_c * lam1_pp * u_roe);
    F_v = F_v - 0.5 * (alpha_c * lam1_pp * v_roe);
    F_w = F_w - 0.5 * (alpha_c * lam1_pp * w_roe);
    F_u = F_u - 0.5 * lam1_pp * (alpha_s1 * t1x + alpha_s2 * t2x);
    F_v = F_v - 0.5 * lam1_pp * (alpha_s1 * t1y + alpha_s2 * t2y);
    F_w = F_w - 0.5 * lam1_pp * (alpha_s1 * t1z + alpha_s2 * t2z);
    F_u = F_u - 0.5 * (alpha_m * lam2_pp * (u_roe - a_roe * nx) + alpha_p * lam3_pp * (u_roe + a_roe * nx));
    F_v = F_v - 0.5 * (alpha_m * lam2_pp * (v_roe - a_roe * ny) + alpha_p * lam3_pp * (v_roe + a_roe * ny));
    F_w = F_w - 0.5 * (alpha_m * lam2_pp * (w_roe - a_roe * nz) + alpha_p * lam3_pp * (w_roe + a_roe * nz));
    F_E = F_E - 0.5 * lam1_pp * (alpha_c * 0.5 * (u_roe * u_roe + v_roe * v_roe + w_roe * w_roe));
    F_E = F_E - 0.5 * lam1_pp *
                    (alpha_s1 * (u_roe * t1x + v_roe * t1y + w_roe * t1z) + alpha_s2 * (u_roe * t2x + v_roe * t2y + w_roe * t2z));
    F_E = F_E - 0.5 * (alpha_m * lam2_pp * (h0_roe - a_roe * un_roe) + alpha_p * lam3_pp * (h0_roe + a_roe * un_roe));
    return;
  }
  if (rs == 7 || rs == 10) {  // HLLC+Tramel (:811-880) and HLLC+Chen (:881-964): HLLC with the face sensor
    double S1 = std::min(std::min(0.0, unl - al), un_roe - a_roe);
    double S4 = std::max(std::max(0.0, unr + ar), un_roe + a_roe);
    double FrE = 0.0, FuE = 0.0, FvE = 0.0, FwE = 0.0, FeE = 0.0;
    if (rs == 7) {  // riemann_HLLE
      double inv_denom = 1.0 / (S4 - S1);
      double FrL = dltot * unl, FrR = drtot * unr;
      FrE = (S4 * FrL - S1 * FrR + S1 * S4 * (drtot - dltot)) * inv_denom;
      FuE = (S4 * (FrL * ul + pl * nx) - S1 * (FrR * ur + pr * nx) + S1 * S4 * (drtot * ur - dltot * ul)) * inv_denom;
      FvE = (S4 * (FrL * vl + pl * ny) - S1 * (FrR * vr + pr * ny) + S1 * S4 * (drtot * vr - dltot * vl)) * inv_denom;
      FwE = (S4 * (FrL * wl + pl * nz) - S1 * (FrR * wr + pr * nz) + S1 * S4 * (drtot * wr - dltot * wl)) * inv_denom;
      FeE = (S4 * (FrL * h0l) - S1 * (FrR * h0r) + S1 * S4 * (drtot * (h0r - pr / drtot) - dltot * (h0l - pl / dltot))) *
            inv_denom;
    }
    double e0l = h0l - pl / dltot, e0r = h0r - pr / drtot;
    double inv_denom = 1.0 / (dltot * (S1 - unl) - drtot * (S4 - unr));
    double Sstar = (pr - pl + dltot * unl * (S1 - unl) - drtot * unr * (S4 - unr)) * inv_denom;
    double pstar = dltot * (unl - S1) * (unl - Sstar) + pl;
    double ch_pref = 0.0, ch_fstar = 0.0, ch_g = 0.0, ch_dU = 0.0, ch_dutx = 0.0, ch_duty = 0.0, ch_dutz = 0.0;
    if (rs == 10) {  // the Chen all-speed terms (the sensor h of the face is bet)
      double ch_phiL = dltot * (S1 - unl), ch_phiR = drtot * (S4 - unr);
      ch_pref = ch_phiL * ch_phiR / (ch_phiR - ch_phiL);
      double ch_Mloc = std::min(1.0, std::max(std::sqrt(ul * ul + vl * vl + wl * wl) / al,
                                              std::sqrt(ur * ur + vr * vr + wr * wr) / ar));
      ch_Mloc = std::max(mco, ch_Mloc);
      double om = 1.0 - ch_Mloc * ch_Mloc;
      double ch_fM = ch_Mloc * std::sqrt(4.0 + om * om) / (1.0 + ch_Mloc * ch_Mloc);
      ch_g = 1.0 - std::pow(bet, ch_Mloc);
      ch_fstar = ch_fM + ch_g * (1.0 - ch_fM);
      ch_dU = unr - unl;
      ch_dutx = (ur - ul) - ch_dU * nx; ch_duty = (vr - vl) - ch_dU * ny; ch_dutz = (wr - wl) - ch_dU * nz;
    }
    double FrC, FuC, FvC, FwC, FeC;
    if (S1 >= 0.0) {
      FrC = dltot * unl; FuC = FrC * ul + pl * nx; FvC = FrC * vl + pl * ny; FwC = FrC * wl + pl * nz; FeC = FrC * h0l;
    } else if (Sstar >= 0.0) {
      FrC = dltot * unl; FuC = FrC * ul + pl * nx; FvC = FrC * vl + pl * ny; FwC = FrC * wl + pl * nz; FeC = FrC * h0l;
      double id = 1.0 / (S1 - Sstar);
      double U1S = dltot * (S1 - unl) * id;
      double U2S = ((S1 - unl) * dltot * ul + (pstar - pl) * nx) * id;
      double U3S = ((S1 - unl) * dltot * vl + (pstar - pl) * ny) * id;
      double U4S = ((S1 - unl) * dltot * wl + (pstar - pl) * nz) * id;
      double U5S = ((S1 - unl) * dltot * e0l - pl * unl + pstar * Sstar) * id;
      FrC = FrC + S1 * (U1S - dltot); FuC = FuC + S1 * (U2S - dltot * ul); FvC = FvC + S1 * (U3S - dltot * vl);
      FwC = FwC + S1 * (U4S - dltot * wl); FeC = FeC + S1 * (U5S - dltot * e0l);
      if (rs == 10) {
        double ch_SK = S1;
        double ch_lm = ch_pref * (ch_fstar - 1.0) * ch_dU;
        double ch_sh = ch_pref * (ch_SK / (ch_SK - Sstar)) * ch_g;
        FuC = FuC + ch_lm * nx + ch_sh * ch_dutx;
        FvC = FvC + ch_lm * ny + ch_sh * ch_duty;
        FwC = FwC + ch_lm * nz + ch_sh * ch_dutz;
        FeC = FeC + ch_lm * Sstar;
      }
    } else if (S4 > 0.0) {
      FrC = drtot * unr; FuC = FrC * ur + pr * nx; FvC = FrC * vr + pr * ny; FwC = FrC * wr + pr * nz; FeC = FrC * h0r;
      double id = 1.0 / (S4 - Sstar);
      double U1S = drtot * (S4 - unr) * id;
      double U2S = ((S4 - unr) * drtot * ur + (pstar - pr) * nx) * id;
      double U3S = ((S4 - unr) * drtot * vr + (pstar - pr) * ny) * id;
      double U4S = ((S4 - unr) * drtot * wr + (pstar - pr) * nz) * id;
      double U5S = ((S4 - unr) * drtot * e0r - pr * unr + pstar * Sstar) * id;
      FrC = FrC + S4 * (U1S - drtot); FuC = FuC + S4 * (U2S - drtot * ur); FvC = FvC + S4 * (U3S - drtot * vr);
      FwC = FwC + S4 * (U4S - drtot * wr); FeC = FeC + S4 * (U5S - drtot * e0r);
      if (rs == 10) {
        double ch_SK = S4;
        double ch_lm = ch_pref * (ch_fstar - 1.0) * ch_dU;
        double ch_sh = ch_pref * (ch_SK / (ch_SK - Sstar)) * ch_g;
        FuC = FuC + ch_lm * nx + ch_sh * ch_dutx;
        FvC = FvC + ch_lm * ny + ch_sh * ch_duty;
        FwC = FwC + ch_lm * nz + ch_sh * ch_dutz;
        FeC = FeC + ch_lm * Sstar;
      }
    } else {
      FrC = drtot * unr; FuC = FrC * ur + pr * nx; FvC = FrC * vr + pr * ny; FwC = FrC * wr + pr * nz; FeC = FrC * h0r;
    }
    if (rs == 10 || bet >= 1.0) {
      F_r = FrC; F_u = FuC; F_v = FvC; F_w = FwC; F_E = FeC;
    } else if (bet == 0.0) {
      F_r = FrE; F_u = FuE; F_v = FvE; F_w = FwE; F_E = FeE;
    } else {
      F_r = bet * FrC + (1.0 - bet) * FrE; F_u = bet * FuC + (1.0 - bet) * FuE; F_v = bet * FvC + (1.0 - bet) * FvE;
      F_w = bet * FwC + (1.0 - bet) * FwE; F_E = bet * FeC + (1.0 - bet) * FeE;
    }
    return;
  }
  double nmag = std::sqrt(nx * nx + ny * ny + nz * nz);
  if (nmag <= 0.0) { F_r = F_u = F_v = F_w = F_E = 0.0; return; }
  double n1 = nx / nmag, n2 = ny / nmag, n3 = nz / nmag;
  double tx, ty, tz;
  if (std::fabs(n1) < 0.9) { tx = 1.0; ty = 0.0; tz = 0.0; } else { tx = 0.0; ty = 1.0; tz = 0.0; }
  double t1x = tx - (tx * n1 + ty * n2 + tz * n3) * n1;
  double t1y = ty - (tx * n1 + ty * n2 + tz * n3) * n2;
  double t1z = tz - (tx * n1 + ty * n2 + tz * n3) * n3;
  double tmag = std::sqrt(t1x * t1x + t1y * t1y + t1z * t1z);
  if (tmag <= 0.0) { t1x = -n2; t1y = n1; t1z = 0.0; tmag = std::sqrt(t1x * t1x + t1y * t1y + t1z * t1z); }
  t1x = t1x / tmag; t1y = t1y / tmag; t1z = t1z / tmag;
  double t2x = n2 * t1z - n3 * t1y;
  double t2y = n3 * t1x - n1 * t1z;
  double t2z = n1 * t1y - n2 * t1x;
  double unL = ul * n1 + vl * n2 + wl * n3, unR = ur * n1 + vr * n2 + wr * n3;
  double ut1L = ul * t1x + vl * t1y + wl * t1z, ut1R = ur * t1x + vr * t1y + wr * t1z;
  double ut2L = ul * t2x + vl * t2y + wl * t2z, ut2R = ur * t2x + vr * t2y + wr * t2z;
  double hL = h_static(th, dl, pl), hR = h_static(th, dr, pr);
  double H0L = hL + 0.5 * (ul * ul + vl * vl + wl * wl);
  double H0R = hR + 0.5 * (ur * ur + vr * vr + wr * wr);
  double FL1 = dltot * unL, FL2 = dltot * unL * ul + pl * n1, FL3 = dltot * unL * vl + pl * n2;
  double FL4 = dltot * unL * wl + pl * n3, FL5 = dltot * unL * H0L;
  double FR1 = drtot * unR, FR2 = drtot * unR * ur + pr * n1, FR3 = drtot * unR * vr + pr * n2;
  double FR4 = drtot * unR * wr + pr * n3, FR5 = drtot * unR * H0R;
  double unRoe = u_roe * n1 + v_roe * n2 + w_roe * n3;
  double u2 = u_roe * u_roe + v_roe * v_roe + w_roe * w_roe;
  double utmag = std::sqrt(std::max(0.0, u2 - unRoe * unRoe));
  double Ma = (a_roe > 0.0) ? (std::fabs(unRoe) + utmag) / a_roe : 1.0;
  double phi = std::max(mco, std::min(1.0, Ma));
  double drho = drtot - dltot, dp = pr - pl, dun = unR - unL;
  double dut1 = ut1R - ut1L, dut2 = ut2R - ut2L;
  double dunmod = phi * dun;
  double abs1 = std::fabs(unRoe - a_roe), abs2 = std::fabs(unRoe), abs3 = std::fabs(unRoe),
         abs4 = std::fabs(unRoe), abs5 = std::fabs(unRoe + a_roe);
  double a2 = a_roe * a_roe, inva = 1.0 / a_roe, inva2 = 1.0 / a2;
  double al4 = drho - dp * inva2;
  double al2 = rho_roe * dut1, al3 = rho_roe * dut2;
  double al1 = 0.5 * (dp * inva2 - rho_roe * dunmod * inva);
  double al5 = 0.5 * (dp * inva2 + rho_roe * dunmod * inva);
  double r1[5] = {1.0, u_roe - a_roe * n1, v_roe - a_roe * n2, w_roe - a_roe * n3, h0_roe - a_roe * unRoe};
  double r5[5] = {1.0, u_roe + a_roe * n1, v_roe + a_roe * n2, w_roe + a_roe * n3, h0_roe + a_roe * unRoe};
  double r4[5] = {1.0, u_roe, v_roe, w_roe, 0.5 * u2};
  double r2[5] = {0.0, t1x, t1y, t1z, u_roe * t1x + v_roe * t1y + w_roe * t1z};
  double r3[5] = {0.0, t2x, t2y, t2z, u_roe * t2x + v_roe * t2y + w_roe * t2z};
  double d[5];
  for (int q = 0; q < 5; ++q)
    d[q] = abs1 * al1 * r1[q] + abs2 * al2 * r2[q] + abs3 * al3 * r3[q] + abs4 * al4 * r4[q] + abs5 * al5 * r5[q];
  F_r = 0.5 * (FL1 + FR1) - 0.5 * d[0];
  F_u = 0.5 * (FL2 + FR2) - 0.5 * d[1];
  F_v = 0.5 * (FL3 + FR3) - 0.5 * d[2];
  F_w = 0.5 * (FL4 + FR4) - 0.5 * d[3];
  F_E = 0.5 * (FL5 + FR5) - 0.5 * d[4];
}

// HLLC (rs 1) / HLLE (rs 2) of Lib_Riemann_HLL.f90:21-134 / 137-198 with roe_averages :209-310 (boundary records;
// no T clamp)
void riemann_hllc_bc(const Thermo& th, int rs, double dl, double ul, double vl, double wl, double pl, double al,
                     double dltot, double dr, double ur, double vr, double wr, double pr, double ar, double drtot,
                     double nx, double ny, double nz, double& F_r, double& F_u, double& F_v, double& F_w,
                     double& F_E) {
  double unl = ul * nx + vl * ny + wl * nz;
  double unr = ur * nx + vr * ny + wr * nz;
  double Rl = 0.0 + th.ri * dl / (0.0 + dl);
  double Rr = 0.0 + th.ri * dr / (0.0 + dr);
  double inv_dltot = 1.0 / dltot, inv_drtot = 1.0 / drtot;
  double Tl = pl * inv_dltot / Rl, Tr = pr * inv_drtot / Rr;
  int Til = tidx(th, Tl), Tir = tidx(th, Tr);
  double dTl = Tl - Til, dTr = Tr - Tir;
  double srL = std::sqrt(dltot), srR = std::sqrt(drtot);
  double inv_sr = 1.0 / (srL + srR);
  double u_roe = (srR * ur + srL * ul) * inv_sr;
  double v_roe = (srR * vr + srL * vl) * inv_sr;
  double w_roe = (srR * wr + srL * wl) * inv_sr;
  double R_roe = (srR * Rr + srL * Rl) * inv_sr;
  double T_roe = (srR * Tr + srL * Tl) * inv_sr;
  double h0l = 0.0, h0r = 0.0, cv_roe = 0.0, sum_ei = 0.0;
  {
    double invW = RUNIV / th.wm;
    double hl = th.h[Til] + (th.h[Til + 1] - th.h[Til]) * dTl;
    double hr = th.h[Tir] + (th.h[Tir + 1] - th.h[Tir]) * dTr;
    double el = hl - invW * Tl, er = hr - invW * Tr;
    h0l = h0l + hl * dl * inv_dltot;
    h0r = h0r + hr * dr * inv_drtot;
    double d_roe = (srR * dr * inv_drtot + srL * dl * inv_dltot) * inv_sr;
    cv_roe = cv_roe + d_roe * (0.5 * (th.cp[Til] + (th.cp[Til + 1] - th.cp[Til]) * dTl + th.cp[Tir] +
                                      (th.cp[Tir + 1] - th.cp[Tir]) * dTr) - invW);
    sum_ei = sum_ei + d_roe * (srR * er + srL * el) * inv_sr;
  }
  h0l = h0l + 0.5 * (ul * ul + vl * vl + wl * wl);
  h0r = h0r + 0.5 * (ur * ur + vr * vr + wr * wr);
  double h0_roe = (srR * h0r + srL * h0l) * inv_sr;
  double gam_roe = 1.0 + R_roe / cv_roe;
  double vel2 = u_roe * u_roe + v_roe * v_roe + w_roe * w_roe;
  double a_roe = std::sqrt((gam_roe - 1.0) * (h0_roe - 0.5 * vel2 + cv_roe * T_roe - sum_ei));
  double un_roe = u_roe * nx + v_roe * ny + w_roe * nz;
  double e0l = h0l - pl / dltot, e0r = h0r - pr / drtot;
  double S1 = std::min(std::min(0.0, unl - al), un_roe - a_roe);
  double S4 = std::max(std::max(0.0, unr + ar), un_roe + a_roe);
  if (rs == 2) {
    hlle_flux(ul, vl, wl, pl, dltot, h0l, ur, vr, wr, pr, drtot, h0r, unl, unr, S1, S4, nx, ny, nz, F_r, F_u, F_v, F_w,
              F_E);
    return;
  }
  double inv_denom = 1.0 / (dltot * (S1 - unl) - drtot * (S4 - unr));
  double Sstar = (pr - pl + dltot * unl * (S1 - unl) - drtot * unr * (S4 - unr)) * inv_denom;
  double pstar = dltot * (unl - S1) * (unl - Sstar) + pl;
  if (S1 >= 0.0) {
    F_r = dltot * unl; F_u = F_r * ul + pl * nx; F_v = F_r * vl + pl * ny; F_w = F_r * wl + pl * nz; F_E = F_r * h0l;
  } else if (Sstar >= 0.0) {
    F_r = dltot * unl; F_u = F_r * ul + pl * nx; F_v = F_r * vl + pl * ny; F_w = F_r * wl + pl * nz; F_E = F_r * h0l;
    inv_denom = 1.0 / (S1 - Sstar);
    double U1S = dltot * (S1 - unl) * inv_denom;
    double U2S = ((S1 - unl) * dltot * ul + (pstar - pl) * nx) * inv_denom;
    double U3S = ((S1 - unl) * dltot * vl + (pstar - pl) * ny) * inv_denom;
    double U4S = ((S1 - unl) * dltot * wl + (pstar - pl) * nz) * inv_denom;
    double U5S = ((S1 - unl) * dltot * e0l - pl * unl + pstar * Sstar) * inv_denom;
    F_r = F_r + S1 * (U1S - dltot); F_u = F_u + S1 * (U2S - dltot * ul); F_v = F_v + S1 * (U3S - dltot * vl);
    F_w = F_w + S1 * (U4S - dltot * wl); F_E = F_E + S1 * (U5S - dltot * e0l);
  } else if (S4 > 0.0) {
    F_r = drtot * unr; F_u = F_r * ur + pr * nx; F_v = F_r * vr + pr * ny; F_w = F_r * wr + pr * nz; F_E = F_r * h0r;
    inv_denom = 1.0 / (S4 - Sstar);
    double U1S = drtot * (S4 - unr) * inv_denom;
    double U2S = ((S4 - unr) * drtot * ur + (pstar - pr) * nx) * inv_denom;
    double U3S = ((S4 - unr) * drtot * vr + (pstar - pr) * ny) * inv_denom;
    double U4S = ((S4 - unr) * drtot * wr + (pstar - pr) * nz) * inv_denom;
    double U5S = ((S4 - unr) * drtot * e0r - pr * unr + pstar * Sstar) * inv_denom;
    F_r = F_r + S4 * (U1S - drtot); F_u = F_u + S4 * (U2S - drtot * ur); F_v = F_v + S4 * (U3S - drtot * vr);
    F_w = F_w + S4 * (U4S - drtot * wr); F_E = F_E + S4 * (U5S - drtot * e0r);
  } else {
    F_r = drtot * unr; F_u = F_r * ur + pr * nx; F_v = F_r * vr + pr * ny; F_w = F_r * wr + pr * nz; F_E = F_r * h0r;
  }
}

// SLAU at the records (Lib_Riemann.f90:140-197): T = p / (rho R) and H0 = h(T) + V^2/2 of each state from the
// tables (no T clamp), then the SLAU flux
void riemann_slau_bc(const Thermo& th, double dl, double ul, double vl, double wl, double pl, double al, double dltot,
                     double dr, double ur, double vr, double wr, double pr, double ar, double drtot, double nx,
                     double ny, double nz, double& F_r, double& F_u, double& F_v, double& F_w, double& F_E) {
  double unl = ul * nx + vl * ny + wl * nz;
  double unr = ur * nx + vr * ny + wr * nz;
  double Rl = 0.0 + th.ri * dl / dltot;
  double Rr = 0.0 + th.ri * dr / drtot;
  double Tl = pl / (dltot * Rl), Tr = pr / (drtot * Rr);
  int Til = (int)Tl, Tir = (int)Tr;
  double dTl = Tl - Til, dTr = Tr - Tir;
  double h0l = 0.0 + (th.h[Til] + (th.h[Til + 1] - th.h[Til]) * dTl) * dl / dltot;
  double h0r = 0.0 + (th.h[Tir] + (th.h[Tir + 1] - th.h[Tir]) * dTr) * dr / drtot;
  h0l = h0l + 0.5 * (ul * ul + vl * vl + wl * wl);
  h0r = h0r + 0.5 * (ur * ur + vr * vr + wr * wr);
  slau_flux(ul, vl, wl, pl, al, dltot, h0l, ur, vr, wr, pr, ar, drtot, h0r, unl, unr, nx, ny, nz, F_r, F_u, F_v, F_w,
            F_E);
}

// The shock sensor of a cell from its pressure and its six face neighbours' (SD_beta, Lib_Shock_Detector.f90:51-81):
// 1 Tramel (1 smooth, 0 at a shock), 2 Chen (the smallest neighbour pressure ratio)
double sd_beta(int id, double p, double p1, double p2, double p3, double p4, double p5, double p6) {
  const double DELTA = 20.0;
  if (id == 1) {
    double kp1 = std::fabs((p2 - 2.0 * p + p1) / (p2 + 2.0 * p + p1));
    double kp2 = std::fabs((p4 - 2.0 * p + p3) / (p4 + 2.0 * p + p3));
    double kp3 = std::fabs((p6 - 2.0 * p + p5) / (p6 + 2.0 * p + p5));
    double sw = std::max(std::max(kp1, kp2), kp3);
    if (sw < 1.0 / DELTA) {
      double phi = std::max(sw / DELTA, 0.0);
      return 1.0 - std::tanh(10.0 * phi * phi * phi);
    }
    return 0.0;
  }
  if (id == 2) {
    double beta = 1.0;
    beta = std::min(beta, std::min(p, p1) / std::max(p, p1));
    beta = std::min(beta, std::min(p, p2) / std::max(p, p2));
    beta = std::min(beta, std::min(p, p3) / std::max(p, p3));
    beta = std::min(beta, std::min(p, p4) / std::max(p, p4));
    beta = std::min(beta, std::min(p, p5) / std::max(p, p5));
    beta = std::min(beta, std::min(p, p6) / std::max(p, p6));
    return beta;
  }
  return 1.0;
}

// beta of the cell (i,j,k) from the filled state (Fluxes_blk, Mod_Fluxes.f90:282-294), 1 without a sensor
double cell_beta(const Ctx& c, const Blk& b, const double* P, int i, int j, int k) {
  if (!c.sd) return 1.0;
  const int64_t o = IP * c.ncell;
  return sd_beta(c.sd, P[row(b, i, j, k) + o], P[row(b, i - 1, j, k) + o], P[row(b, i + 1, j, k) + o],
                 P[row(b, i, j - 1, k) + o], P[row(b, i, j + 1, k) + o], P[row(b, i, j, k - 1) + o],
                 P[row(b, i, j, k + 1) + o]);
}

// ---- one interior convective face: conv_physics.inc:1-179 ----
void conv_face(const Ctx& c, const double* pm1, const double* p0, const double* pp1, const double* pp2,
               const double* dlc, const double* nrm, double area, double* res0, double bet, double urL = 0.0,
               double urR = 0.0) {
  const Thermo& th = c.th;
  const int limv = c.sc.limiter, rsv = c.sc.riemann;
  double l0 = 0.5 * (dlc[0] + dlc[1]), l1 = 0.5 * (dlc[1] + dlc[2]), l2 = 0.5 * (dlc[2] + dlc[3]);
  double lm = 0.5 * dlc[1], lp = 0.5 * dlc[2];
  const double beta_order = c.sd ? bet : 1.0;  // SD_space_order: the slopes scaled by the face sensor
  double idl0 = 1.0 / l0, idl1 = 1.0 / l1, idl2 = 1.0 / l2;
  double P1[NP], P4[NP];
  for (int s = 0; s < NP; ++s) {
    double slope0 = (p0[s] - pm1[s]) * idl0;
    double slope1 = (pp1[s] - p0[s]) * idl1;
    double slope2 = (pp2[s] - pp1[s]) * idl2;
    double slopel = rlimiter(limv, slope1, slope0);
    double sloper = rlimiter(limv, slope2, slope1);
    P1[s] = p0[s] + beta_order * slopel * lm;
    P4[s] = pp1[s] - beta_order * sloper * lp;
  }
  P1[0] = std::max(P1[0], 1e-20);
  P4[0] = std::max(P4[0], 1e-20);
  double rotot1 = 0.0 + P1[0];
  double Rtot1 = 0.0 + th.ri * P1[0] / rotot1;
  double rotot4 = 0.0 + P4[0];
  double Rtot4 = 0.0 + th.ri * P4[0] / rotot4;
  double T1d = P1[IP] / (Rtot1 * rotot1);
  int Ti1 = tidx(th, T1d);
  double Tdiffd = T1d - Ti1;
  double cpd = 0.0 + P1[0] / rotot1 * (th.cp[Ti1] + (th.cp[Ti1 + 1] - th.cp[Ti1]) * Tdiffd);
  double gamd = cpd / (cpd - Rtot1);
  double a1 = std::sqrt(gamd * Rtot1 * T1d);
  double T4d = P4[IP] / (Rtot4 * rotot4);
  int Ti4 = tidx(th, T4d);
  Tdiffd = T4d - Ti4;
  cpd = 0.0 + P4[0] / rotot4 * (th.cp[Ti4] + (th.cp[Ti4 + 1] - th.cp[Ti4]) * Tdiffd);
  gamd = cpd / (cpd - Rtot4);
  double a4 = std::sqrt(gamd * Rtot4 * T4d);
  double dltot = rotot1, drtot = rotot4;
  double ul = P1[IU], vl = P1[IV], wl = P1[IW], pl = P1[IP], al = a1;
  double ur = P4[IU], vr = P4[IV], wr = P4[IW], pr = P4[IP], ar = a4;
  double nx = nrm[0], ny = nrm[1], nz = nrm[2];
  double F_r, F_u, F_v, F_w, F_E;
  if (rsv == 1 || rsv == 2 || rsv == 3) {  // the prologue of conv_physics.inc:49-86, then the solver's flux
    double unl = ul * nx + vl * ny + wl * nz;
    double unr = ur * nx + vr * ny + wr * nz;
    double Rl = Rtot1, Rr = Rtot4;
    double inv_dltot = 1.0 / dltot, inv_drtot = 1.0 / drtot;
    double Tl = pl * inv_dltot / Rl, Tr = pr * inv_drtot / Rr;
    int Til = tidx(th, Tl);
    int Tir = tidx(th, Tr);
    double dTl = Tl - Til, dTr = Tr - Tir;
    double srL = std::sqrt(dltot), srR = std::sqrt(drtot), inv_sr = 1.0 / (srL + srR);
    double u_roe = (srR * ur + srL * ul) * inv_sr, v_roe = (srR * vr + srL * vl) * inv_sr,
           w_roe = (srR * wr + srL * wl) * inv_sr;
    double R_roe = (srR * Rr + srL * Rl) * inv_sr, T_roe = (srR * Tr + srL * Tl) * inv_sr;
    double h0l = 0.0, h0r = 0.0, cv_roe = 0.0, sum_ei = 0.0;
    {
      double invW = RUNIV / th.wm;
      double hl = th.h[Til] + (th.h[Til + 1] - th.h[Til]) * dTl;
      double hr = th.h[Tir] + (th.h[Tir + 1] - th.h[Tir]) * dTr;
      double el = hl - invW * Tl, er = hr - invW * Tr;
      h0l = h0l + hl * P1[0] * inv_dltot;
      h0r = h0r + hr * P4[0] * inv_drtot;
      double d_roe = (srR * P4[0] * inv_drtot + srL * P1[0] * inv_dltot) * inv_sr;
      cv_roe = cv_roe + d_roe * (0.5 * (th.cp[Til] + (th.cp[Til + 1] - th.cp[Til]) * dTl + th.cp[Tir] +
                                        (th.cp[Tir + 1] - th.cp[Tir]) * dTr) - invW);
      sum_ei = sum_ei + d_roe * (srR * er + srL * el) * inv_sr;
    }
    h0l = h0l + 0.5 * (ul * ul + vl * vl + wl * wl);
    h0r = h0r + 0.5 * (ur * ur + vr * vr + wr * wr);
    double h0_roe = (srR * h0r + srL * h0l) * inv_sr;
    double gam_roe = 1.0 + R_roe / cv_roe;
    double vel2 = u_roe * u_roe + v_roe * v_roe + w_roe * w_roe;
    double a_roe = std::sqrt((gam_roe - 1.0) * (h0_roe - 0.5 * vel2 + cv_roe * T_roe - sum_ei));
    double un_roe = u_roe * nx + v_roe * ny + w_roe * nz;
    double e0l = h0l - pl / dltot, e0r = h0r - pr / drtot;
    double S1 = std::min(std::min(0.0, unl - al), un_roe - a_roe);
    double S4 = std::max(std::max(0.0, unr + ar), un_roe + a_roe);
    double inv_denom = 1.0 / (dltot * (S1 - unl) - drtot * (S4 - unr));
    double Sstar = (pr - pl + dltot * unl * (S1 - unl) - drtot * unr * (S4 - unr)) * inv_denom;
    double pstar = dltot * (unl - S1) * (unl - Sstar) + pl;
    if (rsv == 2) {
      hlle_flux(ul, vl, wl, pl, dltot, h0l, ur, vr, wr, pr, drtot, h0r, unl, unr, S1, S4, nx, ny, nz, F_r, F_u, F_v,
                F_w, F_E);
    } else if (rsv == 3) {
      slau_flux(ul, vl, wl, pl, al, dltot, h0l, ur, vr, wr, pr, ar, drtot, h0r, unl, unr, nx, ny, nz, F_r, F_u, F_v,
                F_w, F_E);
    } else if (S1 >= 0.0) {
      F_r = dltot * unl; F_u = F_r * ul + pl * nx; F_v = F_r * vl + pl * ny; F_w = F_r * wl + pl * nz; F_E = F_r * h0l;
    } else if (Sstar >= 0.0) {
      F_r = dltot * unl; F_u = F_r * ul + pl * nx; F_v = F_r * vl + pl * ny; F_w = F_r * wl + pl * nz; F_E = F_r * h0l;
      inv_denom = 1.0 / (S1 - Sstar);
      double U1S = dltot * (S1 - unl) * inv_denom;
      double U2S = ((S1 - unl) * dltot * ul + (pstar - pl) * nx) * inv_denom;
      double U3S = ((S1 - unl) * dltot * vl + (pstar - pl) * ny) * inv_denom;
      double U4S = ((S1 - unl) * dltot * wl + (pstar - pl) * nz) * inv_denom;
      double U5S = ((S1 - unl) * dltot * e0l - pl * unl + pstar * Sstar) * inv_denom;
      F_r = F_r + S1 * (U1S - dltot); F_u = F_u + S1 * (U2S - dltot * ul); F_v = F_v + S1 * (U3S - dltot * vl);
      F_w = F_w + S1 * (U4S - dltot * wl); F_E = F_E + S1 * (U5S - dltot * e0l);
    } else if (S4 > 0.0) {
      F_r = drtot * unr; F_u = F_r * ur + pr * nx; F_v = F_r * vr + pr * ny; F_w = F_r * wr + pr * nz; F_E = F_r * h0r;
      inv_denom = 1.0 / (S4 - Sstar);
      double U1S = drtot * (S4 - unr) * inv_denom;
      double U2S = ((S4 - unr) * drtot * ur + (pstar - pr) * nx) * inv_denom;
      double U3S = ((S4 - unr) * drtot * vr + (pstar - pr) * ny) * inv_denom;
      double U4S = ((S4 - unr) * drtot * wr + (pstar - pr) * nz) * inv_denom;
      double U5S = ((S4 - unr) * drtot * e0r - pr * unr + pstar * Sstar) * inv_denom;
      F_r = F_r + S4 * (U1S - drtot); F_u = F_u + S4 * (U2S - drtot * ur); F_v = F_v + S4 * (U3S - drtot * vr);
      F_w = F_w + S4 * (U4S - drtot * wr); F_E = F_E + S4 * (U5S - drtot * e0r);
    } else {
      F_r = drtot * unr; F_u = F_r * ur + pr * nx; F_v = F_r * vr + pr * ny; F_w = F_r * wr + pr * nz; F_E = F_r * h0r;
    }
  } else {
    // HLLC-PC takes the Ur of the face's two cells (conv_physics.inc:159-163)
    riemann_open(th, rsv, c.sc.mco, bet, P1[0], ul, vl, wl, pl, al, dltot, P4[0], ur, vr, wr, pr, ar, drtot, nx, ny, nz,
                 F_r, F_u, F_v, F_w, F_E, urL, urR);
  }
  double su = fsign_half(F_r), sp = 0.5 + su, sm = su - 0.5;
  double irotot1 = 1.0 / rotot1, irotot4 = 1.0 / rotot4;
  res0[0] = F_r * area * (sp * (P1[0] * irotot1) - sm * (P4[0] * irotot4));
  res0[IU] = F_u * area; res0[IV] = F_v * area; res0[IW] = F_w * area; res0[IP] = F_E * area;
}

// face thermo of the diffusive flux: Diffusive_Face_Thermo_Fill (Mod_Diffusive.f90:311-325)
// and Diffusive_Face_State (Mod_Diffusive.f90:748-776): the same statements
void face_thermo(const Ctx& c, double rhoi, double p, double& rho, double& T, int& ti, double& td, double& cp,
                 double& mil, double& kl) {
  double Rgas;
  rotot_rtot(c.th, rhoi, rho, Rgas);
  T = p / (rho * Rgas);
  ti = tidx(c.th, T);
  td = T - ti;
  cp = f_cp(c.th, rhoi, ti, td, rho);
  wilke(c.th, rhoi, rho, ti, td, mil, kl);
  if (c.sc.prandtl > 0.0) kl = mil * cp / c.sc.prandtl;
}

// the cell temperature / density of the thermo cache (Mod_Thermo_Cache.f90:327-330,378-380)
inline void cell_rho_T(const Ctx& c, const double* P, int64_t nc, int64_t r, double& rho, double& T) {
  double Rg;
  rotot_rtot(c.th, P[r], rho, Rg);
  T = P[r + IP * nc] / (rho * Rg);
}

// ---- one interior viscous face: diff_cuf_kernels.inc:11-87 + diff_physics.inc:1-161 (laminar) ----
// cells: 1,2 the face pair; 3,4 (-/+ along axis ib) of cell 1; 5,6 of cell 2; 7,8 along ic of cell 1; 9,10 of cell 2
void visc_face(const Ctx& c, const Blk& b, const double* P, int dir, int i, int j, int k, double* res0) {
  const int64_t nc = c.ncell;
  const Thermo& th = c.th;
  int ia, ib, ic;
  int o[3] = {0, 0, 0};
  o[dir] = 1;
  if (dir == 0) { ia = 0; ib = 1; ic = 2; } else if (dir == 1) { ia = 1; ib = 0; ic = 2; } else { ia = 2; ib = 0; ic = 1; }
  int eb[3] = {0, 0, 0}, ec[3] = {0, 0, 0};
  eb[ib] = 1; ec[ic] = 1;
  int64_t cc[10];
  cc[0] = row(b, i, j, k);
  cc[1] = row(b, i + o[0], j + o[1], k + o[2]);
  cc[2] = row(b, i - eb[0], j - eb[1], k - eb[2]);
  cc[3] = row(b, i + eb[0], j + eb[1], k + eb[2]);
  cc[4] = row(b, i + o[0] - eb[0], j + o[1] - eb[1], k + o[2] - eb[2]);
  cc[5] = row(b, i + o[0] + eb[0], j + o[1] + eb[1], k + o[2] + eb[2]);
  cc[6] = row(b, i - ec[0], j - ec[1], k - ec[2]);
  cc[7] = row(b, i + ec[0], j + ec[1], k + ec[2]);
  cc[8] = row(b, i + o[0] - ec[0], j + o[1] - ec[1], k + o[2] - ec[2]);
  cc[9] = row(b, i + o[0] + ec[0], j + o[1] + ec[1], k + o[2] + ec[2]);
  double rho_n[10], T_n[10];
  for (int q = 0; q < 10; ++q) cell_rho_T(c, P, nc, cc[q], rho_n[q], T_n[q]);
  auto w = [&](int q, int s) { return P[cc[q] + (int64_t)s * nc]; };
  double G[NP][3];
  double irho1 = 1.0 / rho_n[0], irho2 = 1.0 / rho_n[1];
  G[0][ia] = w(1, 0) * irho2 - w(0, 0) * irho1;
  G[IP][ia] = T_n[1] - T_n[0];
  for (int s = IU; s <= IW; ++s) G[s][ia] = w(1, s) - w(0, s);
  double irt1 = 1.0 / rho_n[2], irt2 = 1.0 / rho_n[3], irt3 = 1.0 / rho_n[4], irt4 = 1.0 / rho_n[5];
  G[0][ib] = (w(3, 0) * irt2 - w(2, 0) * irt1 + w(5, 0) * irt4 - w(4, 0) * irt3) * 0.25;
  G[IP][ib] = (T_n[3] - T_n[2] + T_n[5] - T_n[4]) * 0.25;
  for (int s = IU; s <= IW; ++s) G[s][ib] = (w(3, s) - w(2, s) + w(5, s) - w(4, s)) * 0.25;
  irt1 = 1.0 / rho_n[6]; irt2 = 1.0 / rho_n[7]; irt3 = 1.0 / rho_n[8]; irt4 = 1.0 / rho_n[9];
  G[0][ic] = (w(7, 0) * irt2 - w(6, 0) * irt1 + w(9, 0) * irt4 - w(8, 0) * irt3) * 0.25;
  G[IP][ic] = (T_n[7] - T_n[6] + T_n[9] - T_n[8]) * 0.25;
  for (int s = IU; s <= IW; ++s) G[s][ic] = (w(7, s) - w(6, s) + w(9, s) - w(8, s)) * 0.25;
  double Mav[3][3];
  for (int a = 0; a < 3; ++a)
    for (int q = 0; q < 3; ++q)
      Mav[a][q] = 0.5 * (mv(b, a, q, i, j, k) + mv(b, a, q, i + o[0], j + o[1], k + o[2]));
  for (int iv = 0; iv < NP; ++iv) {
    double g1 = G[iv][0], g2 = G[iv][1], g3 = G[iv][2];
    G[iv][0] = g1 * Mav[0][0] + g2 * Mav[1][0] + g3 * Mav[2][0];
    G[iv][1] = g1 * Mav[0][1] + g2 * Mav[1][1] + g3 * Mav[2][1];
    G[iv][2] = g1 * Mav[0][2] + g2 * Mav[1][2] + g3 * Mav[2][2];
  }
  double Pf[NP];
  for (int iv = 0; iv < NP; ++iv) Pf[iv] = 0.5 * (w(0, iv) + w(1, iv));
  // face thermo from the face-averaged species density and pressure (tface)
  double frs = 0.5 * (w(0, 0) + w(1, 0));
  double fp = 0.5 * (w(0, IP) + w(1, IP));
  double drho, dT, dcp, dmil, dkl;
  int tint; double tdf0;
  face_thermo(c, frs, fp, drho, dT, tint, tdf0, dcp, dmil, dkl);
  const double* nrm;
  if (dir == 0) nrm = fm1p(b, i, j, k); else if (dir == 1) nrm = fm2p(b, i, j, k); else nrm = fm3p(b, i, j, k);
  double area = nrm[3];
  int Ti = tidx(th, dT);
  double Tdf = dT - Ti;
  double Gv[3][3];
  for (int dd = 0; dd < 3; ++dd) { Gv[0][dd] = G[IU][dd]; Gv[1][dd] = G[IV][dd]; Gv[2][dd] = G[IW][dd]; }
  const double mie = 0.0;
  const double sct = 0.9, prt = 0.85;
  double Dm = (dmil / c.sc.schmidt + mie / sct) / drho;
  double kappaf = dkl + mie * dcp / prt;
  double dmi = dmil + mie;
  const double ntt = -2.0 / 3.0;
  double dlam = ntt * dmi;
  double Diver = Gv[0][0] + Gv[1][1] + Gv[2][2];
  double lamDiv = dlam * Diver;
  const double rhokd = 0.0;
  double Txx = lamDiv + 2.0 * dmi * Gv[0][0] + rhokd;
  double Tyy = lamDiv + 2.0 * dmi * Gv[1][1] + rhokd;
  double Tzz = lamDiv + 2.0 * dmi * Gv[2][2] + rhokd;
  double Txy = dmi * (Gv[0][1] + Gv[1][0]), Txz = dmi * (Gv[0][2] + Gv[2][0]), Tyz = dmi * (Gv[1][2] + Gv[2][1]);
  double S1 = Txx * nrm[0] + Txy * nrm[1] + Txz * nrm[2];
  double S2 = Txy * nrm[0] + Tyy * nrm[1] + Tyz * nrm[2];
  double S3 = Txz * nrm[0] + Tyz * nrm[1] + Tzz * nrm[2];
  double DiffH = 0.0;
  double Flx[NP] = {0, 0, 0, 0, 0};
  double DmGY = Dm * (G[0][0] * nrm[0] + G[0][1] * nrm[1] + G[0][2] * nrm[2]);
  Flx[0] = drho * area * DmGY;
  double hh1 = th.h[Ti], hh2 = th.h[Ti + 1];
  double hh = hh1 + Tdf * (hh2 - hh1);
  DiffH = DiffH + DmGY * hh;
  double sflx = 0.0 + Flx[0];
  Flx[0] = Flx[0] - sflx * Pf[0] / drho;
  Flx[IU] = area * S1; Flx[IV] = area * S2; Flx[IW] = area * S3;
  Flx[IP] = area * ((S1 * Pf[IU] + S2 * Pf[IV] + S3 * Pf[IW]) +
                    kappaf * (G[IP][0] * nrm[0] + G[IP][1] * nrm[1] + G[IP][2] * nrm[2]) + DiffH * drho);
  for (int s = 0; s < NP; ++s) res0[s] = Flx[s];
}

// ---- boundary records (bc_record_body.inc + bc_record_apply.inc) ----
// Compute_Diffusive_Flux_St (Mod_Diffusive.f90:781-867), laminar
void diff_flux_st(const Ctx& c, const double* Pa, const double G[NP][3], double area, const double* nrm, double rho,
                  int ti, double td, double cp, double mil, double kl, double* F) {
  const double mie = 0.0, sct = 0.9, prt = 0.85;
  double Gv[3][3];
  for (int dd = 0; dd < 3; ++dd) { Gv[0][dd] = G[IU][dd]; Gv[1][dd] = G[IV][dd]; Gv[2][dd] = G[IW][dd]; }
  double Dm = (mil / c.sc.schmidt + mie / sct) / rho;
  double kappa = kl + mie * cp / prt;
  // Stress_Vector_Std (physics/turbulence/Mod_Fluid.f90:20-44)
  double mi = mil + mie;
  double lam = (-2.0 / 3.0) * mi;
  double Div = Gv[0][0] + Gv[1][1] + Gv[2][2];
  double lamDiv = lam * Div;
  double Txx = lamDiv + 2.0 * mi * Gv[0][0], Tyy = lamDiv + 2.0 * mi * Gv[1][1], Tzz = lamDiv + 2.0 * mi * Gv[2][2];
  double Txy = mi * (Gv[0][1] + Gv[1][0]), Txz = mi * (Gv[0][2] + Gv[2][0]), Tyz = mi * (Gv[1][2] + Gv[2][1]);
  double S[3];
  S[0] = Txx * nrm[0] + Txy * nrm[1] + Txz * nrm[2];
  S[1] = Txy * nrm[0] + Tyy * nrm[1] + Tyz * nrm[2];
  S[2] = Txz * nrm[0] + Tyz * nrm[1] + Tzz * nrm[2];
  double DiffH = 0.0;
  for (int s = 0; s < NP; ++s) F[s] = 0.0;
  double DmG = Dm * (G[0][0] * nrm[0] + G[0][1] * nrm[1] + G[0][2] * nrm[2]);
  F[0] = rho * area * DmG;
  double hh1 = c.th.h[ti], hh2 = c.th.h[ti + 1];
  double hh = hh1 + td * (hh2 - hh1);
  DiffH = DiffH + DmG * hh;
  double sum = 0.0 + F[0];
  F[0] = F[0] - sum * Pa[0] / rho;
  F[IU] = area * S[0]; F[IV] = area * S[1]; F[IW] = area * S[2];
  F[IP] = area * ((S[0] * Pa[IU] + S[1] * Pa[IV] + S[2] * Pa[IW]) +
                  kappa * (G[IP][0] * nrm[0] + G[IP][1] * nrm[1] + G[IP][2] * nrm[2]) + DiffH * rho);
}

void bc_face_geom(const Blk& b, int Im, int Jm, int Km, int Fm, double* nrm, double& area) {
  int dir = (Fm + 1) / 2, modfm = Fm % 2;
  const double* f;
  if (dir == 1) f = fm1p(b, Im - modfm, Jm, Km);
  else if (dir == 2) f = fm2p(b, Im, Jm - modfm, Km);
  else f = fm3p(b, Im, Jm, Km - modfm);
  nrm[0] = f[0]; nrm[1] = f[1]; nrm[2] = f[2]; area = f[3];
}

void riemann_rec(const Ctx& c, double dl, double ul, double vl, double wl, double pl, double al, double dltot,
                 double dr, double ur, double vr, double wr, double pr, double ar, double drtot, double nx, double ny,
                 double nz, double& F_r, double& F_u, double& F_v, double& F_w, double& F_E, double bet = 1.0,
                 double urL = 0.0, double urR = 0.0);

// BC_Connection_Eul_lean (Lib_BC.f90:1770-1867)
void bc_connection_eul(const Ctx& c, const Blk& b, const double* P, double* R, int Im, int Jm, int Km, int Fm) {
  const int64_t nc = c.ncell;
  const Thermo& th = c.th;
  int dir = (Fm + 1) / 2, modfm = Fm % 2, modfm1 = 1 - modfm, modfm2 = 1 - 2 * modfm, gstep = 2 * modfm - 1;
  int o1 = modfm * (-gstep * GC) + modfm1 * (gstep), o2 = modfm * (-gstep), o3 = modfm1 * (-gstep),
      o4 = modfm1 * (-gstep * GC) + modfm * (gstep);
  int e[3] = {0, 0, 0};
  e[dir - 1] = 1;
  int64_t r1 = row(b, Im + o1 * e[0], Jm + o1 * e[1], Km + o1 * e[2]);
  int64_t r2 = row(b, Im + o2 * e[0], Jm + o2 * e[1], Km + o2 * e[2]);
  int64_t r3 = row(b, Im + o3 * e[0], Jm + o3 * e[1], Km + o3 * e[2]);
  int64_t r4 = row(b, Im + o4 * e[0], Jm + o4 * e[1], Km + o4 * e[2]);
  double dlc4[4];
  dlc4[0] = dlv(b, dir - 1, Im + o1 * e[0], Jm + o1 * e[1], Km + o1 * e[2]);
  dlc4[1] = dlv(b, dir - 1, Im + o2 * e[0], Jm + o2 * e[1], Km + o2 * e[2]);
  dlc4[2] = dlv(b, dir - 1, Im + o3 * e[0], Jm + o3 * e[1], Km + o3 * e[2]);
  dlc4[3] = dlv(b, dir - 1, Im + o4 * e[0], Jm + o4 * e[1], Km + o4 * e[2]);
  double nrm[3], area;
  bc_face_geom(b, Im, Jm, Km, Fm, nrm, area);
  const double beta_ = cell_beta(c, b, P, Im, Jm, Km);  // Lib_BC.f90:1811-1818
  double Dl1 = dlc4[0] * 0.5, Dl2 = dlc4[1] * 0.5, Dl3 = dlc4[2] * 0.5, Dl4 = dlc4[3] * 0.5;
  double D12 = Dl1 + Dl2, D23 = Dl2 + Dl3, D34 = Dl3 + Dl4;
  double PL[NP], PR[NP];
  for (int s = 0; s < NP; ++s) {
    double q1 = P[r1 + s * nc], q2 = P[r2 + s * nc], q3 = P[r3 + s * nc], q4 = P[r4 + s * nc];
    double d21 = (q2 - q1) / D12, d32 = (q3 - q2) / D23, d43 = (q4 - q3) / D34;
    PL[s] = q2 + beta_ * rlimiter(c.sc.limiter, d32, d21) * Dl2;
    PR[s] = q3 - beta_ * rlimiter(c.sc.limiter, d43, d32) * Dl3;
  }
  double rhoL, RL, rhoR, RR;
  rotot_rtot(th, PL[0], rhoL, RL);
  double aL = f_ss(th, PL[0], PL[IP], rhoL, RL);
  rotot_rtot(th, PR[0], rhoR, RR);
  double aR = f_ss(th, PR[0], PR[IP], rhoR, RR);
  double F_r, F_u, F_v, F_w, F_E;
  // HLLC-PC: the Ur of the two cells of the face, the ghost's 0 (never filled, Lib_BC.f90:1739-1742)
  riemann_rec(c, PL[0], PL[IU], PL[IV], PL[IW], PL[IP], aL, rhoL, PR[0], PR[IU], PR[IV], PR[IW], PR[IP], aR, rhoR,
              nrm[0], nrm[1], nrm[2], F_r, F_u, F_v, F_w, F_E, beta_, ur_at(c, r2), ur_at(c, r3));
  double su = fsign_half(F_r), selL = 0.5 + su, selR = su - 0.5;
  double Fmass = F_r * area;
  int64_t rm = row(b, Im, Jm, Km);
  double sg = (double)modfm2;
  R[rm] = R[rm] + sg * Fmass * (selL * PL[0] / rhoL - selR * PR[0] / rhoR);
  R[rm + IU * nc] = R[rm + IU * nc] + sg * F_u * area;
  R[rm + IV * nc] = R[rm + IV * nc] + sg * F_v * area;
  R[rm + IW * nc] = R[rm + IW * nc] + sg * F_w * area;
  R[rm + IP * nc] = R[rm + IP * nc] + sg * F_E * area;
}

// BC_Connection_Visc_lean (Lib_BC.f90:2113-2178): pg = bc_pg(:, 1:6) of the record
void bc_connection_visc(const Ctx& c, const Blk& b, const double* P, double* R, int Im, int Jm, int Km, int Fm,
                        const double* pg) {
  const int64_t nc = c.ncell;
  int dir = (Fm + 1) / 2, modfm2 = 1 - 2 * (Fm % 2), gstep = 2 * (Fm % 2) - 1;
  int ia = dir - 1, ib, ic;
  int bm[3] = {Im, Jm, Km}, bp[3] = {Im, Jm, Km}, cm[3] = {Im, Jm, Km}, cp[3] = {Im, Jm, Km};
  if (dir == 1) { ib = 1; ic = 2; bm[1] = Jm - 1; bp[1] = Jm + 1; cm[2] = Km - 1; cp[2] = Km + 1; }
  else if (dir == 2) { ib = 0; ic = 2; bm[0] = Im - 1; bp[0] = Im + 1; cm[2] = Km - 1; cp[2] = Km + 1; }
  else { ib = 0; ic = 1; bm[0] = Im - 1; bp[0] = Im + 1; cm[1] = Jm - 1; cp[1] = Jm + 1; }
  int g[3] = {Im, Jm, Km};
  g[dir - 1] -= gstep;
  double M[3][3];
  for (int q = 0; q < 3; ++q)
    for (int a = 0; a < 3; ++a) M[a][q] = 0.5 * (mv(b, a, q, Im, Jm, Km) + mv(b, a, q, g[0], g[1], g[2]));
  int64_t r1 = row(b, Im, Jm, Km), r3 = row(b, bp[0], bp[1], bp[2]), r4 = row(b, bm[0], bm[1], bm[2]),
          r5 = row(b, cp[0], cp[1], cp[2]), r6 = row(b, cm[0], cm[1], cm[2]);
  auto pv = [&](int q, int s) -> double {
    switch (q) {
      case 0: return P[r1 + s * nc];
      case 1: return pg[s + NP * 0];
      case 2: return P[r3 + s * nc];
      case 3: return P[r4 + s * nc];
      case 4: return P[r5 + s * nc];
      case 5: return P[r6 + s * nc];
      default: return pg[s + NP * (q - 4)];  // q = 6..9 -> Pg(:,3..6)
    }
  };
  double rh[10], rg[10];
  for (int q = 0; q < 10; ++q) rotot_rtot(c.th, pv(q, 0), rh[q], rg[q]);
  double G2l[NP][3], G2g[NP][3], Pa[NP];
  for (int s = 0; s < NP; ++s) {
    double vv[10];
    for (int q = 0; q < 10; ++q) {
      double x = pv(q, s);
      if (s >= IU && s <= IW) vv[q] = x;
      else if (s == IP) vv[q] = x / (rh[q] * rg[q]);
      else vv[q] = x / rh[q];
    }
    double gl[3], gg[3];
    gl[ia] = (vv[1] - vv[0]) * (double)modfm2;
    gl[ib] = (vv[2] - vv[3]) * 0.5;
    gl[ic] = (vv[4] - vv[5]) * 0.5;
    gg[ia] = (vv[0] - vv[1]) * (double)(-modfm2);
    gg[ib] = (vv[7] - vv[6]) * 0.5;
    gg[ic] = (vv[9] - vv[8]) * 0.5;
    for (int kk = 0; kk < 3; ++kk) {
      G2l[s][kk] = gl[0] * M[0][kk] + gl[1] * M[1][kk] + gl[2] * M[2][kk];
      G2g[s][kk] = gg[0] * M[0][kk] + gg[1] * M[1][kk] + gg[2] * M[2][kk];
    }
    Pa[s] = 0.5 * (pv(0, s) + pv(1, s));
  }
  double rho_f, T_f, td, cp_f, mil_f, kl_f;
  int ti;
  face_thermo(c, Pa[0], Pa[IP], rho_f, T_f, ti, td, cp_f, mil_f, kl_f);
  double nrm[3], area;
  bc_face_geom(b, Im, Jm, Km, Fm, nrm, area);
  double Fl[NP], Fg[NP];
  diff_flux_st(c, Pa, G2l, area, nrm, rho_f, ti, td, cp_f, mil_f, kl_f, Fl);
  diff_flux_st(c, Pa, G2g, area, nrm, rho_f, ti, td, cp_f, mil_f, kl_f, Fg);
  for (int s = 0; s < NP; ++s) R[r1 + s * nc] = R[r1 + s * nc] - 0.5 * (double)modfm2 * (Fl[s] + Fg[s]);
}

// BC_Extrapolation (Lib_BC.f90:1119-1165)
void bc_extrapolation(const Ctx& c, const Blk& b, const double* P, double* R, int Im, int Jm, int Km, int Fm) {
  const int64_t nc = c.ncell;
  int64_t r = row(b, Im, Jm, Km);
  double Pr[NP];
  for (int s = 0; s < NP; ++s) Pr[s] = P[r + s * nc];
  double nrm[3], area;
  bc_face_geom(b, Im, Jm, Km, Fm, nrm, area);
  double Un = Pr[IU] * nrm[0] + Pr[IV] * nrm[1] + Pr[IW] * nrm[2];
  double F[NP];
  double Fmass = 0.0;
  F[0] = Pr[0] * Un * area;
  Fmass = Fmass + F[0];
  F[IU] = Fmass * Pr[IU] + Pr[IP] * area * nrm[0];
  F[IV] = Fmass * Pr[IV] + Pr[IP] * area * nrm[1];
  F[IW] = Fmass * Pr[IW] + Pr[IP] * area * nrm[2];
  double vmag = std::sqrt(Pr[IU] * Pr[IU] + Pr[IV] * Pr[IV] + Pr[IW] * Pr[IW]);
  F[IP] = Fmass * H0(c.th, Pr[IP], Pr[0], vmag);
  double sg = (double)(1 - 2 * (Fm % 2));
  for (int s = 0; s < NP; ++s) R[r + s * nc] = R[r + s * nc] + sg * F[s];
}

// The Riemann dispatch of the record routines (Lib_Riemann.f90:114-136, `Riemann`): HLLC Batten for rs 1, HLLE for
// 2, SLAU for 3, the MOSE_open solvers for rs 4..14 (the face sensor argument is 1 at these records)
void riemann_rec(const Ctx& c, double dl, double ul, double vl, double wl, double pl, double al, double dltot,
                 double dr, double ur, double vr, double wr, double pr, double ar, double drtot, double nx, double ny,
                 double nz, double& F_r, double& F_u, double& F_v, double& F_w, double& F_E, double bet, double urL,
                 double urR) {
  if (c.sc.riemann == 1 || c.sc.riemann == 2)
    riemann_hllc_bc(c.th, c.sc.riemann, dl, ul, vl, wl, pl, al, dltot, dr, ur, vr, wr, pr, ar, drtot, nx, ny, nz, F_r,
                    F_u, F_v, F_w, F_E);
  else if (c.sc.riemann == 3)
    riemann_slau_bc(c.th, dl, ul, vl, wl, pl, al, dltot, dr, ur, vr, wr, pr, ar, drtot, nx, ny, nz, F_r, F_u, F_v, F_w,
                    F_E);
  else
    riemann_open(c.th, c.sc.riemann, c.sc.mco, bet, dl, ul, vl, wl, pl, al, dltot, dr, ur, vr, wr, pr, ar, drtot, nx, ny, nz,
                 F_r, F_u, F_v, F_w, F_E, urL, urR);
}

// BC_Symmetry_Eul (Lib_BC.f90:640-737): the boundary cell mirrored about the face (Un_wall = 0), a limited
// one-sided reconstruction to the face, and the Riemann problem between the face state and its mirror;
// only the momentum rows change. Also the Euler part of the adiabatic wall (bc_record_apply.inc, case 5).
void bc_symmetry_eul(const Ctx& c, const Blk& b, const double* P, double* R, int Im, int Jm, int Km, int Fm) {
  const int64_t nc = c.ncell;
  const Thermo& th = c.th;
  int dir = (Fm + 1) / 2, modfm = Fm % 2, modfm1 = 1 - modfm, modfm2 = 1 - 2 * modfm, gstep = 2 * modfm - 1;
  int In[3] = {Im, Jm, Km};
  In[dir - 1] += gstep;
  int64_t rb = row(b, Im, Jm, Km), ri = row(b, In[0], In[1], In[2]);
  double nrm[3], area;
  bc_face_geom(b, Im, Jm, Km, Fm, nrm, area);
  double Bound_Dl = 0.5 * dlv(b, dir - 1, Im, Jm, Km);
  double Int_Dl = 0.5 * dlv(b, dir - 1, In[0], In[1], In[2]);
  double B[NP], I[NP], G[NP], P1[NP], P3[NP], F[NP], Sl[NP];
  for (int s = 0; s < NP; ++s) { B[s] = P[rb + s * nc]; I[s] = P[ri + s * nc]; }
  double Un = B[IU] * nrm[0] + B[IV] * nrm[1] + B[IW] * nrm[2];
  for (int s = 0; s < NP; ++s) G[s] = B[s];
  G[IU] = B[IU] - 2.0 * Un * nrm[0];
  G[IV] = B[IV] - 2.0 * Un * nrm[1];
  G[IW] = B[IW] - 2.0 * Un * nrm[2];
  for (int s = 0; s < NP; ++s) {
    P1[s] = (double)modfm * G[s] + (double)modfm1 * I[s];
    P3[s] = (double)modfm * I[s] + (double)modfm1 * G[s];
  }
  double Dist12 = 2.0 * Bound_Dl * (double)modfm + (Bound_Dl + Int_Dl) * (double)modfm1;
  double Dist23 = (Bound_Dl + Int_Dl) * (double)modfm + 2.0 * Bound_Dl * (double)modfm1;
  for (int s = 0; s < NP; ++s) {
    double s32 = (P3[s] - B[s]) / Dist23;
    double s21 = (B[s] - P1[s]) / Dist12;
    Sl[s] = rlimiter(c.sc.limiter, s32, s21);
  }
  double Dist = Bound_Dl * (double)modfm2;
  for (int s = 0; s < NP; ++s) F[s] = B[s] + Sl[s] * Dist;
  double rotot, Rtot;
  rotot_rtot(th, F[0], rotot, Rtot);
  double Sound = f_ss(th, F[0], F[IP], rotot, Rtot);
  Un = F[IU] * nrm[0] + F[IV] * nrm[1] + F[IW] * nrm[2];
  double Vt[3] = {F[IU] - Un * nrm[0], F[IV] - Un * nrm[1], F[IW] - Un * nrm[2]};
  double Un1 = Un * (double)modfm2;
  double U1[3], U4[3];
  for (int a = 0; a < 3; ++a) { U1[a] = Un1 * nrm[a] + Vt[a]; U4[a] = -Un1 * nrm[a] + Vt[a]; }
  double F_r, F_u, F_v, F_w, F_E;
  // HLLC-PC: the Ur of the cell on both sides (Lib_BC.f90:720-723)
  riemann_rec(c, F[0], U1[0], U1[1], U1[2], F[IP], Sound, rotot, F[0], U4[0], U4[1], U4[2], F[IP], Sound, rotot,
              nrm[0], nrm[1], nrm[2], F_r, F_u, F_v, F_w, F_E, 1.0, ur_at(c, rb), ur_at(c, rb));
  R[rb + IU * nc] = R[rb + IU * nc] + (double)modfm2 * F_u * area;
  R[rb + IV * nc] = R[rb + IV * nc] + (double)modfm2 * F_v * area;
  R[rb + IW * nc] = R[rb + IW * nc] + (double)modfm2 * F_w * area;
}

// BC_Wall_Heat_dev (Lib_BC.f90:879-982), laminar: the wall-normal velocity gradient of the boundary cell
// (wall velocity 0), Grad . M of the cell, the stress vector of Stress_Vector_Std (Mod_Fluid.f90:20-44) with
// mu_t = 0; adiabatic, so the energy row is untouched.
void bc_wall_heat(const Ctx& c, const Blk& b, const double* P, double* R, int Im, int Jm, int Km, int Fm) {
  const int64_t nc = c.ncell;
  int dir = (Fm + 1) / 2, modfm = Fm % 2, modfm2 = 1 - 2 * modfm, modfm3 = 2 * (2 * modfm - 1);
  int64_t rb = row(b, Im, Jm, Km);
  double Pb[NP];
  for (int s = 0; s < NP; ++s) Pb[s] = P[rb + s * nc];
  double M[3][3];
  for (int a = 0; a < 3; ++a)
    for (int q = 0; q < 3; ++q) M[a][q] = mv(b, a, q, Im, Jm, Km);
  double rho, Rgas;
  rotot_rtot(c.th, Pb[0], rho, Rgas);
  double T = Pb[IP] / (rho * Rgas);
  int ti = tidx(c.th, T);
  double Tdiff = T - ti;
  double mil, kl;
  wilke(c.th, Pb[0], rho, ti, Tdiff, mil, kl);
  double Grad[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int a = 0; a < 3; ++a) Grad[a][dir - 1] = Pb[IU + a] * (double)modfm3;
  double G2[3][3];
  for (int kk = 0; kk < 3; ++kk)
    for (int ii = 0; ii < 3; ++ii)
      G2[ii][kk] = Grad[ii][0] * M[0][kk] + Grad[ii][1] * M[1][kk] + Grad[ii][2] * M[2][kk];
  double nrm[3], area;
  bc_face_geom(b, Im, Jm, Km, Fm, nrm, area);
  const double ntt = -2.0 / 3.0;  // negativetwothird (Mod_Fluid.f90:4)
  double mi = mil + 0.0;
  double lam = ntt * mi;
  double Div = G2[0][0] + G2[1][1] + G2[2][2];
  double lamDiv = lam * Div;
  double txx = lamDiv + 2.0 * mi * G2[0][0], tyy = lamDiv + 2.0 * mi * G2[1][1], tzz = lamDiv + 2.0 * mi * G2[2][2];
  double txy = mi * (G2[0][1] + G2[1][0]), txz = mi * (G2[0][2] + G2[2][0]), tyz = mi * (G2[1][2] + G2[2][1]);
  double S1 = txx * nrm[0] + txy * nrm[1] + txz * nrm[2];
  double S2 = txy * nrm[0] + tyy * nrm[1] + tyz * nrm[2];
  double S3 = txz * nrm[0] + tyz * nrm[1] + tzz * nrm[2];
  R[rb + IU * nc] = R[rb + IU * nc] - (double)modfm2 * area * S1;
  R[rb + IV * nc] = R[rb + IV * nc] - (double)modfm2 * area * S2;
  R[rb + IW * nc] = R[rb + IW * nc] - (double)modfm2 * area * S3;
}

// Stress_Vector_Std (Mod_Fluid.f90:20-44) with mu_t = 0: the stress vector tau . n of the gradient G2 (Grad . M)
void stress_std(const double G2[3][3], const double* nrm, double mil, double* S) {
  const double ntt = -2.0 / 3.0;
  double mi = mil + 0.0;
  double lam = ntt * mi;
  double Div = G2[0][0] + G2[1][1] + G2[2][2];
  double lamDiv = lam * Div;
  double txx = lamDiv + 2.0 * mi * G2[0][0], tyy = lamDiv + 2.0 * mi * G2[1][1], tzz = lamDiv + 2.0 * mi * G2[2][2];
  double txy = mi * (G2[0][1] + G2[1][0]), txz = mi * (G2[0][2] + G2[2][0]), tyz = mi * (G2[1][2] + G2[2][1]);
  S[0] = txx * nrm[0] + txy * nrm[1] + txz * nrm[2];
  S[1] = txy * nrm[0] + tyy * nrm[1] + tyz * nrm[2];
  S[2] = txz * nrm[0] + tyz * nrm[1] + tzz * nrm[2];
}

// BC_Symmetry_Visc (Lib_BC.f90:741-861), laminar: the boundary cell and its four transverse neighbours mirrored
// about the face give the normal and the two transverse velocity gradients; the stress of Grad . M and its work on
// the face-mean velocity leave the momentum and energy rows.
void bc_symmetry_visc(const Ctx& c, const Blk& b, const double* P, double* R, int Im, int Jm, int Km, int Fm) {
  const int64_t nc = c.ncell;
  int modfm = Fm % 2, modfm2 = 1 - 2 * modfm;
  int64_t rb = row(b, Im, Jm, Km);
  double Pb[NP];
  for (int s = 0; s < NP; ++s) Pb[s] = P[rb + s * nc];
  double M[3][3];
  for (int a = 0; a < 3; ++a)
    for (int q = 0; q < 3; ++q) M[a][q] = mv(b, a, q, Im, Jm, Km);
  double rho, Rgas;
  rotot_rtot(c.th, Pb[0], rho, Rgas);
  double T = Pb[IP] / (rho * Rgas);
  int ti = tidx(c.th, T);
  double Tdiff = T - ti;
  double mil, kl;
  wilke(c.th, Pb[0], rho, ti, Tdiff, mil, kl);
  int o3[3] = {0, 0, 0}, o4[3] = {0, 0, 0}, o7[3] = {0, 0, 0}, o8[3] = {0, 0, 0};
  int a, bb, cc;
  if (Fm <= 2) { o3[1] = -1; o4[1] = 1; o7[2] = -1; o8[2] = 1; a = 0; bb = 1; cc = 2; }
  else if (Fm <= 4) { o3[0] = -1; o4[0] = 1; o7[2] = -1; o8[2] = 1; a = 1; bb = 0; cc = 2; }
  else { o3[0] = -1; o4[0] = 1; o7[1] = -1; o8[1] = 1; a = 2; bb = 0; cc = 1; }
  auto vel = [&](const int* o, double* v) {
    int64_t r = row(b, Im + o[0], Jm + o[1], Km + o[2]);
    v[0] = P[r + IU * nc]; v[1] = P[r + IV * nc]; v[2] = P[r + IW * nc];
  };
  double V1[3] = {Pb[IU], Pb[IV], Pb[IW]}, V3[3], V4[3], V7[3], V8[3];
  vel(o3, V3); vel(o4, V4); vel(o7, V7); vel(o8, V8);
  double nrm[3], area;
  bc_face_geom(b, Im, Jm, Km, Fm, nrm, area);
  double d1 = V1[0] * nrm[0] + V1[1] * nrm[1] + V1[2] * nrm[2];
  double d3 = V3[0] * nrm[0] + V3[1] * nrm[1] + V3[2] * nrm[2];
  double d4 = V4[0] * nrm[0] + V4[1] * nrm[1] + V4[2] * nrm[2];
  double d7 = V7[0] * nrm[0] + V7[1] * nrm[1] + V7[2] * nrm[2];
  double d8 = V8[0] * nrm[0] + V8[1] * nrm[1] + V8[2] * nrm[2];
  double V2[3], V5[3], V6[3], V9[3], V10[3];
  for (int s = 0; s < 3; ++s) {
    V2[s] = V1[s] - 2.0 * d1 * nrm[s];
    V5[s] = V3[s] - 2.0 * d3 * nrm[s];
    V6[s] = V4[s] - 2.0 * d4 * nrm[s];
    V9[s] = V7[s] - 2.0 * d7 * nrm[s];
    V10[s] = V8[s] - 2.0 * d8 * nrm[s];
  }
  double Grad[3][3];
  for (int s = 0; s < 3; ++s) {
    Grad[s][a] = (V2[s] - V1[s]) * (double)modfm2;
    Grad[s][bb] = (V4[s] - V3[s] + V6[s] - V5[s]) * 0.25;
    Grad[s][cc] = (V8[s] - V7[s] + V10[s] - V9[s]) * 0.25;
  }
  double G2[3][3];
  for (int kk = 0; kk < 3; ++kk)
    for (int ii = 0; ii < 3; ++ii)
      G2[ii][kk] = Grad[ii][0] * M[0][kk] + Grad[ii][1] * M[1][kk] + Grad[ii][2] * M[2][kk];
  double S[3];
  stress_std(G2, nrm, mil, S);
  double Vf[3] = {0.5 * (V1[0] + V2[0]), 0.5 * (V1[1] + V2[1]), 0.5 * (V1[2] + V2[2])};
  R[rb + IU * nc] = R[rb + IU * nc] - (double)modfm2 * area * S[0];
  R[rb + IV * nc] = R[rb + IV * nc] - (double)modfm2 * area * S[1];
  R[rb + IW * nc] = R[rb + IW * nc] - (double)modfm2 * area * S[2];
  R[rb + IP * nc] = R[rb + IP * nc] - (double)modfm2 * area * (Vf[0] * S[0] + Vf[1] * S[1] + Vf[2] * S[2]);
}

// BC_Wall_Temperature_dev (Lib_BC.f90:997-1115), laminar no-slip wall at T_wall: the wall state p(wall) = p(cell)
// at T_wall gives mu and k (k = mu cp / Pr when Pr > 0), the wall-normal velocity and temperature gradients of the
// boundary cell give the stress (momentum rows) and the conducted heat (energy row).
void bc_wall_temperature(const Ctx& c, const Blk& b, const double* P, double* R, int Im, int Jm, int Km, int Fm,
                         double Tw) {
  const int64_t nc = c.ncell;
  int dir = (Fm + 1) / 2, modfm = Fm % 2, modfm2 = 1 - 2 * modfm, modfm3 = 2 * (2 * modfm - 1);
  int64_t rb = row(b, Im, Jm, Km);
  double Pb[NP];
  for (int s = 0; s < NP; ++s) Pb[s] = P[rb + s * nc];
  double M[3][3];
  for (int a = 0; a < 3; ++a)
    for (int q = 0; q < 3; ++q) M[a][q] = mv(b, a, q, Im, Jm, Km);
  double rho, Rgas;
  rotot_rtot(c.th, Pb[0], rho, Rgas);
  double T = Pb[IP] / (rho * Rgas);
  double rho_wall = Pb[IP] / (Rgas * Tw);
  double Pw0 = Pb[0] * rho_wall / rho;
  int ti = tidx(c.th, Tw);
  double Tdiff = Tw - ti;
  double mil, kl;
  wilke(c.th, Pw0, rho_wall, ti, Tdiff, mil, kl);
  if (c.sc.prandtl > 0.0) kl = mil * f_cp(c.th, Pw0, ti, Tdiff, rho_wall) / c.sc.prandtl;
  double Grad[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int a = 0; a < 3; ++a) Grad[a][dir - 1] = Pb[IU + a] * (double)modfm3;
  double G2[3][3];
  for (int kk = 0; kk < 3; ++kk)
    for (int ii = 0; ii < 3; ++ii)
      G2[ii][kk] = Grad[ii][0] * M[0][kk] + Grad[ii][1] * M[1][kk] + Grad[ii][2] * M[2][kk];
  double nrm[3], area;
  bc_face_geom(b, Im, Jm, Km, Fm, nrm, area);
  double S[3];
  stress_std(G2, nrm, mil, S);
  double Gnp_dir = (T - Tw) * (double)modfm3;
  double Gnp[3];
  for (int kk = 0; kk < 3; ++kk) Gnp[kk] = Gnp_dir * M[dir - 1][kk];
  double Flux_np = area * kl * (Gnp[0] * nrm[0] + Gnp[1] * nrm[1] + Gnp[2] * nrm[2]);
  R[rb + IU * nc] = R[rb + IU * nc] - (double)modfm2 * area * S[0];
  R[rb + IV * nc] = R[rb + IV * nc] - (double)modfm2 * area * S[1];
  R[rb + IW * nc] = R[rb + IW * nc] - (double)modfm2 * area * S[2];
  R[rb + IP * nc] = R[rb + IP * nc] - (double)modfm2 * Flux_np;
}

// The inflow / outflow record (type 4), BC_Inflow_Outflow (Lib_BC.f90:1519-1597). q = mach, T0, p0, alpha, beta,
// rel_fac, open code, pamb, t (3): the open code selects the closure as IO_BC_Open.f90:229-307 sets it up -- 0 or 405
// the supersonic static inlet (any Mach; the face closes on outward flow), 401 the subsonic stagnation inlet (T0, p0),
// 403 the mass-flux inlet with total T (p0 = the mass flux), 404 the mass-flux inlet with static T, 407 the ambient
// boundary (stagnation inlet on inward flow, outflow to pamb = q[7] on outward flow). t is the unit tangent of the
// face (Mod_BC.f90:226-240: the diagonal of its nodes). Outward flow at a 401-405 face closes it (BC_Symmetry_Eul).
void outflow_flux(const Thermo& th, const double* Bp, double Brho, double BRgas, double BSound, double Un,
                  double BGamma, double Riem, const double* nrm, double area, double p_Amb, double BC_Sign,
                  double* Flux);
void inflow_resolve(const double* q, double& mach, double& pamb) {
  const int code = (int)q[6];
  mach = q[0];
  pamb = -2.71;  // PAMB_FORCE_SUPERSONIC
  if (code == 401) { mach = 0.0; pamb = -3.14; }
  else if (code == 403) { mach = -10.0; pamb = -3.14; }
  else if (code == 404) { mach = -1.0; pamb = -3.14; }
  else if (code == 407) { mach = 0.0; pamb = q[7]; }
}

// BC_Subsonic_Inflow (Lib_BC.f90:1335-1512), one species: the face state from the outgoing Riemann invariant and the
// stagnation (mach >= 0) or mass-flux (mach < 0) conditions; its flux into Flux
void subsonic_inflow_flux(const Thermo& th, const double* Bp, double Un, double Sound, double Gamma, double Riem,
                          double BC_alpha, double BC_beta, double BC_Mach, double BC_T0, double BC_p0, double rel,
                          double BC_Sign, const double* t, const double* n, double area, double* Flux) {
  double bv[3] = {n[1] * t[2] - n[2] * t[1], n[2] * t[0] - n[0] * t[2], n[0] * t[1] - n[1] * t[0]};
  double bmod = std::sqrt(bv[0] * bv[0] + bv[1] * bv[1] + bv[2] * bv[2]);
  bv[0] = bv[0] / bmod; bv[1] = bv[1] / bmod; bv[2] = bv[2] / bmod;
  double alpha, beta;
  if (BC_alpha == 0.0 && BC_beta == 0.0) {
    alpha = std::atan(n[1] / (n[0] + 1e-20));
    beta = std::atan(n[2] / (n[0] + 1e-20));
  } else {
    alpha = BC_alpha; beta = BC_beta;
  }
  const double ta = std::tan(alpha), tb = std::tan(beta);
  double XA = n[1] - n[0] * ta, XB = t[1] - t[0] * ta, XC = bv[1] - bv[0] * ta;
  double XD = n[2] - n[0] * tb, XE = t[2] - t[0] * tb, XF = bv[2] - bv[0] * tb;
  double check = (XC * XE - XF * XB);
  double E1 = (XF * XA - XC * XD) / check;
  double E2 = (XD * XB - XE * XA) / check;
  double Fp[NP], Frho, FRgas, Fun;
  if (BC_Mach >= 0.0) {
    double Discr = -1.0, p0_try = BC_p0, Sound0 = 0.0, Coef_D = 0.0, YA = 0.0, YB = 0.0;
    int iter = 0;
    while (Discr < 0.0) {
      iter = iter + 1;
      FRgas = 0.0 + 1.0 * th.ri;
      Sound0 = std::sqrt(Gamma * FRgas * BC_T0);
      Coef_D = (1.0 + E1 * E1 + E2 * E2) * (Gamma - 1.0) / 2.0;
      double Coef_C = std::pow(p0_try / Bp[IP], (Gamma - 1.0) / Gamma);
      Coef_C = Coef_C * ((Sound / Sound0) * (Sound / Sound0));
      const double g2 = (Gamma - 1.0) / 2.0;
      YA = g2 * g2 + Coef_C * Coef_D;
      YB = BC_Sign * Riem * ((Gamma - 1.0) / 2.0);
      double YC = Riem * Riem - Coef_C * (Sound0 * Sound0);
      Discr = YB * YB - YA * YC;
      if (Discr < 0.0 && std::fabs(Discr) < 1e-2) Discr = 0.0;
      if (Discr < 0.0 && std::fabs(Discr) > 1e-2) {
        if (rel == 1.0) { Discr = 0.0; break; }
        p0_try = rel * p0_try + (1.0 - rel) * Bp[IP];
      }
      if (iter > 1000) { Discr = 0.0; break; }
    }
    double Un_Sign = std::copysign(1.0, Un);
    double Un3 = (YB + Un_Sign * std::sqrt(Discr)) / YA;
    double Sound3 = std::sqrt(Sound0 * Sound0 - Coef_D * (Un3 * Un3));
    double p3 = p0_try * std::pow(Sound3 / Sound0, 2.0 * Gamma / (Gamma - 1.0));
    double Ut3 = Un3 * E1, Ub3 = Un3 * E2;
    Fp[IP] = p3;
    Frho = Gamma * Fp[IP] / (Sound3 * Sound3);
    Fp[0] = 1.0 * Frho;
    Fp[IU] = Un3 * n[0] + Ut3 * t[0] + Ub3 * bv[0];
    Fp[IV] = Un3 * n[1] + Ut3 * t[1] + Ub3 * bv[1];
    Fp[IW] = Un3 * n[2] + Ut3 * t[2] + Ub3 * bv[2];
    Fun = Un3;
  } else {  // mass flux (p0 column) and temperature: total (mach -10) or static
    double mdot = BC_p0, p3 = Bp[IP];
    int Ti = tidx(th, BC_T0);
    double Td = BC_T0 - Ti;
    double cp3 = 0.0 + 1.0 * tabT(th.cp, Ti, Td);
    double Rgas3 = 0.0 + 1.0 * th.ri;
    double T3 = BC_T0;
    if (BC_Mach == -10.0) {
      double x = mdot * Rgas3 / p3, y = p3 / (mdot * Rgas3);
      T3 = (-cp3 + std::sqrt(cp3 * cp3 + 2.0 * cp3 * BC_T0 * (x * x))) * (y * y);
    }
    double rho3 = p3 / (Rgas3 * T3);
    double Un3 = mdot / rho3;
    double Ut3 = Un3 * E1, Ub3 = Un3 * E2;
    FRgas = Rgas3;
    Frho = rho3;
    Fp[0] = Frho * 1.0;
    Fp[IU] = Un3 * n[0] + Ut3 * t[0] + Ub3 * bv[0];
    Fp[IV] = Un3 * n[1] + Ut3 * t[1] + Ub3 * bv[1];
    Fp[IW] = Un3 * n[2] + Ut3 * t[2] + Ub3 * bv[2];
    Fp[IP] = p3;
    Fun = Un3;
  }
  double FEnth = 0.0;
  double FT = Fp[IP] / (FRgas * Frho);
  int Ti = tidx(th, FT);
  double Td = FT - Ti;
  FEnth = FEnth + Fp[0] / Frho * tabT(th.h, Ti, Td);
  Flux[0] = Fp[0] * Fun * area;
  double Fmass = Frho * Fun * area;
  Flux[IU] = Fmass * Fp[IU] + Fp[IP] * area * n[0];
  Flux[IV] = Fmass * Fp[IV] + Fp[IP] * area * n[1];
  Flux[IW] = Fmass * Fp[IW] + Fp[IP] * area * n[2];
  double vt2 = Fp[IU] * Fp[IU] + Fp[IV] * Fp[IV] + Fp[IW] * Fp[IW];
  Flux[IP] = Fmass * (0.5 * vt2 + FEnth);
}

void bc_inflow_405(const Ctx& c, const Blk& b, const double* P, double* R, int Im, int Jm, int Km, int Fm,
                   const double* q) {
  const int64_t nc = c.ncell;
  const Thermo& th = c.th;
  int dir = (Fm + 1) / 2, modfm = Fm % 2, modfm1 = 1 - modfm, modfm2 = 1 - 2 * modfm, gstep = 2 * modfm - 1;
  int In[3] = {Im, Jm, Km};
  In[dir - 1] += gstep;
  int64_t rb = row(b, Im, Jm, Km), ri = row(b, In[0], In[1], In[2]);
  double P2[NP], Ip[NP];
  for (int s = 0; s < NP; ++s) { P2[s] = P[rb + s * nc]; Ip[s] = P[ri + s * nc]; }
  double nrm[3], area;
  bc_face_geom(b, Im, Jm, Km, Fm, nrm, area);
  double BC_Mach, pamb;
  inflow_resolve(q, BC_Mach, pamb);
  const double BC_T0 = q[1], BC_p0 = q[2], rel = q[5];
  const double BC_Sign = (double)modfm2;
  double Un = P2[IU] * nrm[0] + P2[IV] * nrm[1] + P2[IW] * nrm[2];
  double Brho, BRgas;
  rotot_rtot(th, P2[0], Brho, BRgas);
  double BSound = f_ss(th, P2[0], P2[IP], Brho, BRgas);
  double T = P2[IP] / (Brho * BRgas);
  int tiB = tidx(th, T);
  double cpB = f_cp(th, P2[0], tiB, T - tiB, Brho);
  double BGamma = cpB / (cpB - BRgas);
  double Riem = BSound + BC_Sign * 0.5 * (BGamma - 1.0) * Un;
  double InOut = BC_Sign * Un;
  if (BC_Mach < 0.0) InOut = -1.0;
  if (InOut >= 0.0) {
    if (pamb == -3.14 || pamb == -2.71) {  // an inlet: error = 1, the caller applies the symmetry flux
      bc_symmetry_eul(c, b, P, R, Im, Jm, Km, Fm);
      return;
    }
    double Flux[NP];
    outflow_flux(th, P2, Brho, BRgas, BSound, Un, BGamma, Riem, nrm, area, pamb, BC_Sign, Flux);
    for (int s = 0; s < NP; ++s) R[rb + s * nc] = R[rb + s * nc] + (double)modfm2 * Flux[s];
    return;
  }
  if (!(BC_Mach > 1.0 || pamb == -2.71)) {
    if (BC_Mach < 1.0) {
      double Flux[NP];
      subsonic_inflow_flux(th, P2, Un, BSound, BGamma, Riem, q[3], q[4], BC_Mach, BC_T0, BC_p0, rel, BC_Sign, q + 8,
                           nrm, area, Flux);
      for (int s = 0; s < NP; ++s) R[rb + s * nc] = R[rb + s * nc] + (double)modfm2 * Flux[s];
    }
    return;
  }
  // BC_Supersonic_Inflow
  double fR, frho;
  rotot_rtot(th, P2[0], frho, fR);  // f_Rtot
  double vmag2 = P2[IU] * P2[IU] + P2[IV] * P2[IV] + P2[IW] * P2[IW];
  double fS = f_ss(th, P2[0], P2[IP], P2[0], fR);
  double fM = std::sqrt(vmag2) / fS;
  double Mach_l = rel * BC_Mach + (1.0 - rel) * fM;
  double p0_l = rel * BC_p0 + (1.0 - rel) * P2[IP];
  double Sup[NP];
  Sup[IP] = p0_l;
  double Sup_T = BC_T0;
  double Sup_Rgas = 0.0 + 1.0 * th.ri;
  double Sup_rho = Sup[IP] / (Sup_Rgas * Sup_T);
  Sup[0] = Sup_rho * 1.0;
  double Sup_Sound = f_ss(th, Sup[0], Sup[IP], Sup_rho, Sup_Rgas);
  const double ca = std::cos(q[3]), sa = std::sin(q[3]), cb = std::cos(q[4]), sb = std::sin(q[4]);
  Sup[IU] = Mach_l * Sup_Sound * ca * cb;
  Sup[IV] = Mach_l * Sup_Sound * sa * cb;
  Sup[IW] = Mach_l * Sup_Sound * sb;
  double PL[NP], PR[NP];
  for (int s = 0; s < NP; ++s) {
    double p1 = (double)modfm * Sup[s] + (double)modfm1 * Ip[s];
    double p3 = (double)modfm * Ip[s] + (double)modfm1 * Sup[s];
    double Slope = rlimiter(c.sc.limiter, p3 - P2[s], P2[s] - p1);
    double Face = P2[s] + 0.5 * Slope * (double)modfm2;
    PL[s] = (double)modfm * Sup[s] + (double)modfm1 * Face;
    PR[s] = (double)modfm * Face + (double)modfm1 * Sup[s];
  }
  double rL, RL, rR, RR;
  rotot_rtot(th, PL[0], rL, RL);
  double aL = f_ss(th, PL[0], PL[IP], rL, RL);
  rotot_rtot(th, PR[0], rR, RR);
  double aR = f_ss(th, PR[0], PR[IP], rR, RR);
  double F_r, F_u, F_v, F_w, F_E;
  // Ur = a on both sides: no preconditioning at the inlet (Lib_BC.f90:1308-1310)
  riemann_rec(c, PL[0], PL[IU], PL[IV], PL[IW], PL[IP], aL, rL, PR[0], PR[IU], PR[IV], PR[IW], PR[IP], aR, rR, nrm[0],
              nrm[1], nrm[2], F_r, F_u, F_v, F_w, F_E, 1.0, aL, aR);
  double su = std::copysign(1.0, F_r);
  double selL = (1.0 + su) / 2.0, selR = (su - 1.0) / 2.0;
  double Fmass = F_r * area;
  double Fl[NP];
  Fl[0] = Fmass * (selL * PL[0] / rL - selR * PR[0] / rR);
  Fl[IU] = F_u * area; Fl[IV] = F_v * area; Fl[IW] = F_w * area; Fl[IP] = F_E * area;
  for (int s = 0; s < NP; ++s) R[rb + s * nc] = R[rb + s * nc] + (double)modfm2 * Fl[s];
}

// BC_Outflow (Lib_BC.f90:1166-1240): the face state of an outflow to the pressure p_Amb (isentropic when the normal
// Mach number is below 1 and p_Amb > 0, the boundary cell itself otherwise) and its flux
void outflow_flux(const Thermo& th, const double* Bp, double Brho, double BRgas, double BSound, double Un,
                  double BGamma, double Riem, const double* nrm, double area, double p_Amb, double BC_Sign,
                  double* Flux) {
  double vmag = std::sqrt(Bp[IU] * Bp[IU] + Bp[IV] * Bp[IV] + Bp[IW] * Bp[IW]);
  double VT[3] = {Bp[IU] - Un * nrm[0], Bp[IV] - Un * nrm[1], Bp[IW] - Un * nrm[2]};
  double Mach_abs = vmag / BSound;
  (void)Mach_abs;
  double Mach_N = std::fabs(Un / BSound);
  double pe = p_Amb;
  double Fp[NP], Fun, Frho, FRgas;
  if (Mach_N < 1.0 && p_Amb > 0.0) {
    double delta = 0.5 * (BGamma - 1.0);
    double denom = 1.0 / std::pow(1.0 + delta, BGamma / (BGamma - 1.0));
    double pstar = Bp[IP] * denom * std::pow(1.0 + delta * (Mach_N * Mach_N), BGamma / (BGamma - 1.0));
    if (pstar >= p_Amb) pe = pstar;
    double Isentropic = (BGamma - 1.0) / (2.0 * BGamma);
    double FSound = BSound * std::pow(pe / Bp[IP], Isentropic);
    Fun = (Riem - FSound) / (BC_Sign * 0.5 * (BGamma - 1.0));
    Fp[IP] = pe;
    Frho = BGamma * Fp[IP] / (FSound * FSound);
    Fp[0] = Bp[0] / Brho * Frho;
    Fp[IU] = VT[0] + Fun * nrm[0];
    Fp[IV] = VT[1] + Fun * nrm[1];
    Fp[IW] = VT[2] + Fun * nrm[2];
    FRgas = BRgas;
  } else {
    for (int s = 0; s < NP; ++s) Fp[s] = Bp[s];
    Fun = Un; Frho = Brho; FRgas = BRgas;
  }
  double FEnth = 0.0;
  double FT = Fp[IP] / (FRgas * Frho);
  int Ti = tidx(th, FT);
  double Td = FT - Ti;
  FEnth = FEnth + Fp[0] / Frho * tabT(th.h, Ti, Td);
  Flux[0] = Fp[0] * area * Fun;
  double Fmass = Frho * area * Fun;
  Flux[IU] = Fp[IU] * Fmass + Fp[IP] * area * nrm[0];
  Flux[IV] = Fp[IV] * Fmass + Fp[IP] * area * nrm[1];
  Flux[IW] = Fp[IW] * Fmass + Fp[IP] * area * nrm[2];
  double vt2 = Fp[IU] * Fp[IU] + Fp[IV] * Fp[IV] + Fp[IW] * Fp[IW];
  Flux[IP] = Fmass * (0.5 * vt2 + FEnth);
}

// BC_Outlet (Lib_BC.f90:1604-1658) of a 406 record, q = exit pressure, relaxation factor: inward flow closes the
// face (BC_Symmetry_Eul); otherwise the Riemann invariant towards the face and the relaxed exit pressure give the
// face state of BC_Outflow (Lib_BC.f90:1166-1240): isentropic to p_exit when the normal Mach number is below 1 and
// p_exit > 0, the boundary cell itself otherwise.
void bc_outlet(const Ctx& c, const Blk& b, const double* P, double* R, int Im, int Jm, int Km, int Fm,
               const double* q) {
  const int64_t nc = c.ncell;
  const Thermo& th = c.th;
  int modfm = Fm % 2, modfm2 = 1 - 2 * modfm;
  int64_t rb = row(b, Im, Jm, Km);
  double Bp[NP];
  for (int s = 0; s < NP; ++s) Bp[s] = P[rb + s * nc];
  double nrm[3], area;
  bc_face_geom(b, Im, Jm, Km, Fm, nrm, area);
  const double BC_pExit = q[0], BC_rel_fac = q[1];
  double BC_Sign = (double)modfm2;
  double Un = Bp[IU] * nrm[0] + Bp[IV] * nrm[1] + Bp[IW] * nrm[2];
  if (BC_Sign * Un < 0.0) {
    bc_symmetry_eul(c, b, P, R, Im, Jm, Km, Fm);
    return;
  }
  double Brho, BRgas;
  rotot_rtot(th, Bp[0], Brho, BRgas);
  double BSound = f_ss(th, Bp[0], Bp[IP], Brho, BRgas);
  double T = Bp[IP] / (Brho * BRgas);
  int ti = tidx(th, T);
  double Tdiff = T - ti;
  double cp = f_cp(th, Bp[0], ti, Tdiff, Brho);
  double BGamma = cp / (cp - BRgas);
  double Riem = BSound + BC_Sign * 0.5 * (BGamma - 1.0) * Un;
  double p_exit = BC_rel_fac * BC_pExit + (1.0 - BC_rel_fac) * Bp[IP];
  double Flux[NP];
  outflow_flux(th, Bp, Brho, BRgas, BSound, Un, BGamma, Riem, nrm, area, p_exit, BC_Sign, Flux);
  for (int s = 0; s < NP; ++s) R[rb + s * nc] = R[rb + s * nc] + (double)modfm2 * Flux[s];
}

// ---- ghost fill ----
inline int64_t rowg(const Ctx& c, int blk, int i, int j, int k) { return row(c.blk[blk], i, j, k); }

void fill_ghosts(Ctx& c, double* P) {
  const int64_t nc = c.ncell;
  // Fill_Ghost_Cell_blk: symmetry for type 3, zero-gradient for types 11 / 4 / 24, cubic extrapolation for the walls
  // 5 / 6 (Lib_Extrapolation.f90:643-730)
  for (const mb_bc& r : c.rec) {
    const Blk& b = c.blk[r.blk];
    int dir = (r.face + 1) / 2, gstep = 2 * (r.face % 2) - 1;
    int e[3] = {0, 0, 0};
    e[dir - 1] = 1;
    if (r.type == MB_BC_SYMMETRY) {  // Ghost_Symmetry (:558-587): the first layer only, normal velocity reversed
      double nrm[3], area;
      bc_face_geom(b, r.i, r.j, r.k, r.face, nrm, area);
      int64_t src = row(b, r.i, r.j, r.k);
      int64_t dst = row(b, r.i - gstep * e[0], r.j - gstep * e[1], r.k - gstep * e[2]);
      double vel[3] = {P[src + IU * nc], P[src + IV * nc], P[src + IW * nc]};
      double udotn = vel[0] * nrm[0] + vel[1] * nrm[1] + vel[2] * nrm[2];
      for (int a = 0; a < 3; ++a) vel[a] = vel[a] - 2.0 * udotn * nrm[a];
      P[dst] = P[src];
      P[dst + IU * nc] = vel[0]; P[dst + IV * nc] = vel[1]; P[dst + IW * nc] = vel[2];
      P[dst + IP * nc] = P[src + IP * nc];
    } else if (r.type == MB_BC_EXTRAPOLATION || r.type == MB_BC_INFLOW || r.type == MB_BC_OUTLET ||
               r.type == MB_BC_NONE) {  // type 0 (no condition): zero-gradient ghost (Lib_Extrapolation.f90:692)
      int64_t src = row(b, r.i, r.j, r.k);
      for (int g = 1; g <= GC; ++g) {
        int64_t dst = row(b, r.i - gstep * g * e[0], r.j - gstep * g * e[1], r.k - gstep * g * e[2]);
        for (int s = 0; s < NP; ++s) P[dst + s * nc] = P[src + s * nc];
      }
    } else if (r.type == MB_BC_WALL || r.type == MB_BC_WALL_T) {
      int step = -gstep;
      for (int g = 1; g <= GC; ++g) {
        int64_t d0 = row(b, r.i + g * step * e[0], r.j + g * step * e[1], r.k + g * step * e[2]);
        int64_t a1 = row(b, r.i + (g - 1) * step * e[0], r.j + (g - 1) * step * e[1], r.k + (g - 1) * step * e[2]);
        int64_t a2 = row(b, r.i + (g - 2) * step * e[0], r.j + (g - 2) * step * e[1], r.k + (g - 2) * step * e[2]);
        int64_t a3 = row(b, r.i + (g - 3) * step * e[0], r.j + (g - 3) * step * e[1], r.k + (g - 3) * step * e[2]);
        for (int s = 0; s < NP; ++s)
          P[d0 + s * nc] = 3.0 * P[a1 + s * nc] - 3.0 * P[a2 + s * nc] + P[a3 + s * nc];
      }
    }
  }
  // extrapolation-ghost = cubic on the 400 faces (Fill_Ghost_Cubic_Extrapolation_blk, :859-879)
  for (const mb_bc& r : c.rec) {
    if (r.type != MB_BC_EXTRAPOLATION) continue;
    const Blk& b = c.blk[r.blk];
    int dir = (r.face + 1) / 2, gstep = 2 * (r.face % 2) - 1, step = -gstep;
    int e[3] = {0, 0, 0};
    e[dir - 1] = 1;
    for (int g = 1; g <= GC; ++g) {
      int64_t d0 = row(b, r.i + g * step * e[0], r.j + g * step * e[1], r.k + g * step * e[2]);
      int64_t a1 = row(b, r.i + (g - 1) * step * e[0], r.j + (g - 1) * step * e[1], r.k + (g - 1) * step * e[2]);
      int64_t a2 = row(b, r.i + (g - 2) * step * e[0], r.j + (g - 2) * step * e[1], r.k + (g - 2) * step * e[2]);
      int64_t a3 = row(b, r.i + (g - 3) * step * e[0], r.j + (g - 3) * step * e[1], r.k + (g - 3) * step * e[2]);
      for (int s = 0; s < NP; ++s) P[d0 + s * nc] = 3.0 * P[a1 + s * nc] - 3.0 * P[a2 + s * nc] + P[a3 + s * nc];
    }
  }
  // connection / periodic copies (Ghost_Connection_pair, :1023-1134): receiver ghost layer g <- donor layer g
  // guide(F) = the inward unit step of face F
  auto guide = [](int F, int ax) { int d = (F + 1) / 2 - 1; return ax == d ? ((F % 2) ? 1 : -1) : 0; };
  for (const mb_conn& cn : c.conn) {
    const mb_bc& r = c.rec[cn.rec];
    for (int g = 1; g <= GC; ++g) {
      int64_t dst = rowg(c, r.blk, r.i - guide(r.face, 0) * g, r.j - guide(r.face, 1) * g, r.k - guide(r.face, 2) * g);
      int64_t src = rowg(c, cn.bs, cn.is + guide(cn.fs, 0) * (g - 1), cn.js + guide(cn.fs, 1) * (g - 1),
                         cn.ks + guide(cn.fs, 2) * (g - 1));
      for (int s = 0; s < NP; ++s) P[dst + s * nc] = P[src + s * nc];
    }
  }
  // bc_pg: layers 1-2 and the four transverse neighbours of the donor face cell, after every ghost write
  // (Ghost_Connection_pairs_B, :1136-1191)
  for (size_t q = 0; q < c.conn.size(); ++q) {
    const mb_conn& cn = c.conn[q];
    double* pg = &c.pg[(size_t)cn.rec * 6 * NP];
    int64_t s1 = rowg(c, cn.bs, cn.is, cn.js, cn.ks);
    int64_t s2 = rowg(c, cn.bs, cn.is + guide(cn.fs, 0), cn.js + guide(cn.fs, 1), cn.ks + guide(cn.fs, 2));
    int I = cn.is, J = cn.js, K = cn.ks;
    int t[4][3];
    if (cn.fs <= 2) {
      int a[4][3] = {{I, J - cn.d11, K - cn.d12}, {I, J + cn.d11, K + cn.d12}, {I, J - cn.d21, K - cn.d22}, {I, J + cn.d21, K + cn.d22}};
      std::memcpy(t, a, sizeof(t));
    } else if (cn.fs <= 4) {
      int a[4][3] = {{I - cn.d11, J, K - cn.d12}, {I + cn.d11, J, K + cn.d12}, {I - cn.d21, J, K - cn.d22}, {I + cn.d21, J, K + cn.d22}};
      std::memcpy(t, a, sizeof(t));
    } else {
      int a[4][3] = {{I - cn.d11, J - cn.d12, K}, {I + cn.d11, J + cn.d12, K}, {I - cn.d21, J - cn.d22, K}, {I + cn.d21, J + cn.d22, K}};
      std::memcpy(t, a, sizeof(t));
    }
    for (int s = 0; s < NP; ++s) {
      pg[s + NP * 0] = P[s1 + s * nc];
      pg[s + NP * 1] = P[s2 + s * nc];
      for (int m = 0; m < 4; ++m) pg[s + NP * (2 + m)] = P[rowg(c, cn.bs, t[m][0], t[m][1], t[m][2]) + s * nc];
    }
  }
}

// ---- residual: pass 1 + pass 2 (Mod_Fluxes.f90:188-390) + BC_Fluxes (Mod_BC.f90:646-800) ----
void residual(Ctx& c, const double* P, double* R) {
  const int64_t nc = c.ncell;
  const bool visc = c.sc.visc != 0;
  for (const Blk& b : c.blk) {
    if (b.ext) continue;
    const int n1 = b.n1, n2 = b.n2, n3 = b.n3;
    const int64_t nf1 = (int64_t)(n1 - 1) * n2 * n3, nf2 = (int64_t)n1 * (n2 - 1) * n3, nf3 = (int64_t)n1 * n2 * (n3 - 1);
    std::vector<double> fh[3], dfh[3];
    fh[0].assign(std::max<int64_t>(nf1, 0) * NP, 0.0);
    fh[1].assign(std::max<int64_t>(nf2, 0) * NP, 0.0);
    fh[2].assign(std::max<int64_t>(nf3, 0) * NP, 0.0);
    if (visc) { dfh[0].assign(fh[0].size(), 0.0); dfh[1].assign(fh[1].size(), 0.0); dfh[2].assign(fh[2].size(), 0.0); }
    // pass 1: the interior faces of each direction (conv_cuf_i/j/k, diff_cuf_i/j/k)
    for (int d = 0; d < 3; ++d) {
      int h1 = n1, h2 = n2, h3 = n3;
      if (d == 0) h1 = n1 - 1; else if (d == 1) h2 = n2 - 1; else h3 = n3 - 1;
      if (h1 < 1 || h2 < 1 || h3 < 1) continue;
#pragma omp parallel for collapse(2) schedule(static)
      for (int k = 1; k <= h3; ++k)
        for (int j = 1; j <= h2; ++j)
          for (int i = 1; i <= h1; ++i) {
            int e[3] = {0, 0, 0};
            e[d] = 1;
            double pm1[NP], p0[NP], pp1[NP], pp2[NP], dlc[4], res0[NP];
            int64_t r0 = row(b, i, j, k);
            int64_t st = e[0] + (int64_t)e[1] * b.pi + (int64_t)e[2] * b.pi * b.pj;
            for (int s = 0; s < NP; ++s) {
              pm1[s] = P[r0 - st + s * nc]; p0[s] = P[r0 + s * nc];
              pp1[s] = P[r0 + st + s * nc]; pp2[s] = P[r0 + 2 * st + s * nc];
            }
            for (int q = -1; q <= 2; ++q) dlc[q + 1] = dlv(b, d, i + q * e[0], j + q * e[1], k + q * e[2]);
            const double* f = (d == 0) ? fm1p(b, i, j, k) : (d == 1) ? fm2p(b, i, j, k) : fm3p(b, i, j, k);
            conv_face(c, pm1, p0, pp1, pp2, dlc, f, f[3], res0, cell_beta(c, b, P, i, j, k), ur_at(c, r0),
                      ur_at(c, r0 + st));
            int64_t fi;
            if (d == 0) fi = (i - 1) + (int64_t)(j - 1) * (n1 - 1) + (int64_t)(k - 1) * (n1 - 1) * n2;
            else if (d == 1) fi = (i - 1) + (int64_t)(j - 1) * n1 + (int64_t)(k - 1) * n1 * (n2 - 1);
            else fi = (i - 1) + (int64_t)(j - 1) * n1 + (int64_t)(k - 1) * n1 * n2;
            for (int s = 0; s < NP; ++s) fh[d][fi * NP + s] = res0[s];
            if (visc) {
              visc_face(c, b, P, d, i, j, k, res0);
              for (int s = 0; s < NP; ++s) dfh[d][fi * NP + s] = res0[s];
            }
          }
    }
    // pass 2 (pass2_body.inc): R of every interior cell, written once
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= n3; ++k)
      for (int j = 1; j <= n2; ++j)
        for (int i = 1; i <= n1; ++i) {
          double t[NP] = {0, 0, 0, 0, 0};
          auto add = [&](const std::vector<double>& v, int64_t f, double sg) {
            for (int s = 0; s < NP; ++s) t[s] = (sg > 0) ? t[s] + v[f * NP + s] : t[s] - v[f * NP + s];
          };
          auto f1 = [&](int ii) { return (ii - 1) + (int64_t)(j - 1) * (n1 - 1) + (int64_t)(k - 1) * (n1 - 1) * n2; };
          auto f2 = [&](int jj) { return (i - 1) + (int64_t)(jj - 1) * n1 + (int64_t)(k - 1) * n1 * (n2 - 1); };
          auto f3 = [&](int kk) { return (i - 1) + (int64_t)(j - 1) * n1 + (int64_t)(kk - 1) * n1 * n2; };
          if (i < n1) add(fh[0], f1(i), 1); if (i > 1) add(fh[0], f1(i - 1), -1);
          if (j < n2) add(fh[1], f2(j), 1); if (j > 1) add(fh[1], f2(j - 1), -1);
          if (k < n3) add(fh[2], f3(k), 1); if (k > 1) add(fh[2], f3(k - 1), -1);
          if (visc) {
            if (i < n1) add(dfh[0], f1(i), -1); if (i > 1) add(dfh[0], f1(i - 1), 1);
            if (j < n2) add(dfh[1], f2(j), -1); if (j > 1) add(dfh[1], f2(j - 1), 1);
            if (k < n3) add(dfh[2], f3(k), -1); if (k > 1) add(dfh[2], f3(k - 1), 1);
          }
          int64_t r0 = row(b, i, j, k);
          for (int s = 0; s < NP; ++s) R[r0 + s * nc] = t[s];
        }
  }
  // boundary records, one face index at a time (the per-cell add order of Mod_BC.f90:449-485)
  for (int f = 1; f <= 6; ++f) {
    const int nr = (int)c.rec.size();
#pragma omp parallel for schedule(static)
    for (int q = 0; q < nr; ++q) {
      const mb_bc& r = c.rec[q];
      if (r.face != f) continue;
      const Blk& b = c.blk[r.blk];
      switch (r.type) {
        case MB_BC_CONNECTION:
          bc_connection_eul(c, b, P, R, r.i, r.j, r.k, r.face);
          if (visc) bc_connection_visc(c, b, P, R, r.i, r.j, r.k, r.face, &c.pg[(size_t)q * 6 * NP]);
          break;
        case MB_BC_EXTRAPOLATION:
          bc_extrapolation(c, b, P, R, r.i, r.j, r.k, r.face);
          break;
        case MB_BC_WALL:
          bc_symmetry_eul(c, b, P, R, r.i, r.j, r.k, r.face);
          if (visc) bc_wall_heat(c, b, P, R, r.i, r.j, r.k, r.face);
          break;
        case MB_BC_INFLOW:
          bc_inflow_405(c, b, P, R, r.i, r.j, r.k, r.face, r.q);
          break;
        case MB_BC_SYMMETRY:
          bc_symmetry_eul(c, b, P, R, r.i, r.j, r.k, r.face);
          if (visc) bc_symmetry_visc(c, b, P, R, r.i, r.j, r.k, r.face);
          break;
        case MB_BC_WALL_T:
          bc_symmetry_eul(c, b, P, R, r.i, r.j, r.k, r.face);
          if (visc) bc_wall_temperature(c, b, P, R, r.i, r.j, r.k, r.face, r.q[0]);
          break;
        case MB_BC_OUTLET:
          bc_outlet(c, b, P, R, r.i, r.j, r.k, r.face, r.q);
          break;
        default:
          break;
      }
    }
  }
}

// ---- state update: newstate_cons_body.inc ----
static const double RKC[4][4] = {{1.0, 0.0, 0.0, 0.0}, {1.0, 0.50, 0.0, 0.0}, {1.0, 0.25, 2.0 / 3.0, 0.0}, {0, 0, 0, 0}};

// RK4 (n_rk = 4, no reference): stage weights of the new state from Un and of the accumulator
static const double RK4_C[4] = {0.5, 0.5, 1.0, 0.0};
static const double RK4_W[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};

// rk4 = 0: the SSP form of the reference, cons = cold + (cons - cold + rl) * rkc. rk4 = stage 1..4 of RK4 with
// the cell's accumulator a4: stage 1 a4 = cold + rl/6, stages 2-3 a4 += rl/3, new = cold + C rl; stage 4
// new = a4 + rl/6 (rl = -R / vol * dt).
void update_cell(const Ctx& c, const double* po, double* p, const double* res, double vol, double dt, double rkc,
                 double tc, int rk4 = 0, double* a4 = nullptr, bool prescaled = false) {
  const Thermo& th = c.th;
  const double strang = 1.0;
  double cons[NP], cold[NP], rl[NP];
  auto prim2cons = [&](const double* q, double* u) {
    double rho = 0.0 + q[0];
    double Rg = 0.0 + th.ri * q[0] / rho;
    double vmag = 0.0;
    for (int s = IU; s <= IW; ++s) vmag = vmag + q[s] * q[s];
    double Tl = q[IP] / (Rg * rho);
    int ti = tidx(th, Tl);
    double Td = Tl - ti;
    double hs = th.h[ti] + Td * (th.h[ti + 1] - th.h[ti]);
    double hmix = 0.0 + hs * q[0] / rho;
    double E0 = hmix - q[IP] / rho + 0.5 * vmag;
    u[0] = q[0];
    for (int s = IU; s <= IW; ++s) u[s] = rho * q[s];
    u[IP] = rho * E0;
  };
  prim2cons(po, cold);
  prim2cons(p, cons);
  // IRS: the residual arrives scaled (-R / vol * dt * strang) and smoothed (newstate_cons_body.inc, ps_)
  for (int s = 0; s < NP; ++s) rl[s] = prescaled ? res[s] : -res[s] / vol * dt * strang;
  if (rk4 == 0) {
    for (int s = 0; s < NP; ++s) cons[s] = cold[s] + (cons[s] - cold[s] + rl[s]) * rkc;
  } else if (rk4 < 4) {
    for (int s = 0; s < NP; ++s) {
      a4[s] = (rk4 == 1) ? cold[s] + rl[s] * RK4_W[0] : a4[s] + rl[s] * RK4_W[rk4 - 1];
      cons[s] = cold[s] + rl[s] * RK4_C[rk4 - 1];
    }
  } else {
    for (int s = 0; s < NP; ++s) cons[s] = a4[s] + rl[s] * RK4_W[3];
  }
  double rho = 0.0 + cons[0];
  double Rg = 0.0 + th.ri * cons[0] / rho;
  p[0] = cons[0];
  for (int s = IU; s <= IW; ++s) p[s] = cons[s] / rho;
  double vmag = 0.0;
  for (int s = IU; s <= IW; ++s) vmag = vmag + (cons[s] / rho) * (cons[s] / rho);
  double energy = cons[IP] / rho - 0.5 * vmag;
  double diff_en = 1e3, T_it = tc;
  int it = 1;
  while ((std::fabs(diff_en / energy) >= 1e-6) && (it <= 20)) {
    int ti = tidx(th, T_it);
    double Td = T_it - ti;
    double cv = -Rg, enth = 0.0;
    double cps = th.cp[ti] + Td * (th.cp[ti + 1] - th.cp[ti]);
    double hs = th.h[ti] + Td * (th.h[ti + 1] - th.h[ti]);
    cv = cv + cons[0] / rho * cps;
    enth = enth + cons[0] / rho * hs;
    double p_it = rho * Rg * T_it;
    diff_en = std::fabs((enth - p_it / rho) - energy);
    T_it = T_it + (energy - (enth - p_it / rho)) / cv;
    it = it + 1;
  }
  p[IP] = rho * Rg * T_it;
  if (p[0] < 1e-20) p[0] = 1e-20;
}

// Newstate_Primitive_blk (Lib_Newstate.f90:348-531), one species: the conservative residual taken to the primitive
// variables by the inverse of the prim -> cons Jacobian (Theta = rho_p: no preconditioning), then the RK stage on the
// primitive state: new = old + (state - old + res dt / vol) rkc, rho floored at 1e-20
void update_cell_prim(const Ctx& c, const double* po, double* p, const double* res, double vol, double dt, double rkc,
                      double urc = 0.0) {
  const Thermo& th = c.th;
  const double strang = 1.0;
  double rho, Rgas;
  rotot_rtot(th, p[0], rho, Rgas);
  double temperature = p[IP] / (rho * Rgas);
  int T_i = tidx(th, temperature);
  double Tdiff = temperature - T_i;
  double inv_rho = 1.0 / rho;
  double vel[3] = {p[IU], p[IV], p[IW]};
  double modvel = std::sqrt(vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
  double q2 = modvel * modvel;
  double cp = f_cp(th, p[0], T_i, Tdiff, rho);
  double rho_T = -rho / temperature;
  double rho_p = 1.0 / (Rgas * temperature);
  double enthalpy = H0(th, p[IP], p[0], modvel);
  double Theta = rho_p;
  if (prec_on(c)) {  // Weiss-Smith: Theta from the cell's Ur (Lib_Newstate.f90:399-402)
    const double gam = cp / (cp - Rgas);
    const double sound = std::sqrt(gam * Rgas * temperature);
    const double a2 = sound * sound;
    const double beta2 = std::max(urc * urc / a2, 1.0e-6);
    Theta = 1.0 / (beta2 * a2) + 1.0 / (cp * temperature);
  }
  double Denom = 1.0 / (rho * cp * Theta + rho_T);
  double G[5][5];
  G[0][0] = (rho_T * (enthalpy - q2) + rho * cp) * Denom;
  G[0][1] = rho_T * vel[0] * Denom; G[0][2] = rho_T * vel[1] * Denom; G[0][3] = rho_T * vel[2] * Denom;
  G[0][4] = -rho_T * Denom;
  for (int a = 0; a < 3; ++a) {
    G[1 + a][0] = -vel[a] * inv_rho;
    for (int q = 1; q < 5; ++q) G[1 + a][q] = 0.0;
    G[1 + a][1 + a] = inv_rho;
  }
  G[4][0] = -(Theta * (enthalpy - q2) - 1.0) * Denom;
  G[4][1] = -vel[0] * Theta * Denom; G[4][2] = -vel[1] * Theta * Denom; G[4][3] = -vel[2] * Theta * Denom;
  G[4][4] = Theta * Denom;
  double cres[5] = {-res[0], -res[IU], -res[IV], -res[IW], -res[IP]}, pres[5];
  for (int r_ = 0; r_ < 5; ++r_) {
    pres[r_] = 0.0;
    for (int c_ = 0; c_ < 5; ++c_) pres[r_] = pres[r_] + G[r_][c_] * cres[c_];
  }
  double rl[NP];
  rl[IU] = pres[1]; rl[IV] = pres[2]; rl[IW] = pres[3];
  rl[IP] = pres[0];
  rl[0] = rho_p * pres[0] + rho_T * pres[4];
  for (int s = 0; s < NP; ++s) rl[s] = rl[s] * dt / vol * strang;
  for (int s = 0; s < NP; ++s) p[s] = po[s] + (p[s] - po[s] + rl[s]) * rkc;
  if (p[0] < 1e-20) p[0] = 1e-20;
}

void update(Ctx& c, double* P, const double* PO, const double* R, int irk, double dt, bool prescaled = false,
            const double* dtl = nullptr) {
  const int64_t nc = c.ncell;
  const double rkc = c.sc.n_rk == 4 ? 0.0 : RKC[c.sc.n_rk - 1][irk - 1];
  const bool guard = c.sc.visc != 0;
  int nbad = 0, nth = 0;
  for (size_t bi = 0; bi < c.blk.size(); ++bi) {
    const Blk& b = c.blk[bi];
    if (b.ext) continue;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : nbad, nth)
    for (int k = 1; k <= b.n3; ++k)
      for (int j = 1; j <= b.n2; ++j)
        for (int i = 1; i <= b.n1; ++i) {
          int64_t r = row(b, i, j, k);
          double p[NP], po[NP], res[NP];
          for (int s = 0; s < NP; ++s) { p[s] = P[r + s * nc]; po[s] = PO[r + s * nc]; res[s] = R[r + s * nc]; }
          double rho, T;
          cell_rho_T(c, P, nc, r, rho, T);
          if (guard && !(T > 1.0 && T < 9990.0)) {  // thermo guard (Mod_Thermo_Cache.f90:317-327)
            ++nth;
            if (T != T) T = 300.0;
            T = std::min(std::max(T, 1.0), 9990.0);
          }
          const double dtc = dtl ? dtl[r] : dt;  // time-accurate = false: the cell's own dtlocal
          if (c.sc.intvar >= 1)
            update_cell_prim(c, po, p, res, b.vol[lin(b, i, j, k)], dtc, rkc, ur_at(c, r));
          else if (c.sc.n_rk == 4)
            update_cell(c, po, p, res, b.vol[lin(b, i, j, k)], dtc, rkc, T, irk, &c.acc4[(size_t)r * NP]);
          else
            update_cell(c, po, p, res, b.vol[lin(b, i, j, k)], dtc, rkc, T, 0, nullptr, prescaled);
          bool bad = !(p[IP] >= 0.0);
          for (int s = 0; s < NP; ++s) if (!std::isfinite(p[s])) bad = true;
          if (bad) ++nbad;
          for (int s = 0; s < NP; ++s) P[r + s * nc] = p[s];
        }
  }
  c.st.n_bad_state += nbad;
  c.st.n_bad_thermo += nth;
  if (nth && c.st.code == MB_OK) c.st.code = MB_E_THERMO;
  if (nbad && c.sc.state_check && c.st.code == MB_OK) c.st.code = MB_E_STATE;
}

// ---- implicit residual smoothing: IRS_apply (Lib_IRS.f90:57-105) ----

// Ghost_Residual_Extrapolation (irs_ghost_residual, :119-177): the first ghost layer of every face of every block
// takes the adjacent cell's residual, then every connection record's ghost takes its donor face cell's
void irs_ghost_residual(const Ctx& c, double* R) {
  const int64_t nc = c.ncell;
  for (const Blk& b : c.blk) {
    if (b.ext) continue;
    auto cp = [&](int64_t g, int64_t m) { for (int s = 0; s < NP; ++s) R[g + s * nc] = R[m + s * nc]; };
    for (int k = 1; k <= b.n3; ++k)
      for (int j = 1; j <= b.n2; ++j) {
        cp(row(b, 0, j, k), row(b, 1, j, k));
        cp(row(b, b.n1 + 1, j, k), row(b, b.n1, j, k));
      }
    for (int k = 1; k <= b.n3; ++k)
      for (int i = 1; i <= b.n1; ++i) {
        cp(row(b, i, 0, k), row(b, i, 1, k));
        cp(row(b, i, b.n2 + 1, k), row(b, i, b.n2, k));
      }
    for (int j = 1; j <= b.n2; ++j)
      for (int i = 1; i <= b.n1; ++i) {
        cp(row(b, i, j, 0), row(b, i, j, 1));
        cp(row(b, i, j, b.n3 + 1), row(b, i, j, b.n3));
      }
  }
  // irs_ghost_conn (:180-200): r(receiver ghost behind its face cell) = r(donor face cell)
  for (const mb_conn& q : c.conn) {
    const mb_bc& r = c.rec[q.rec];
    const Blk& bm = c.blk[r.blk];
    const int gstep = 2 * (r.face % 2) - 1;
    int ig = r.i, jg = r.j, kg = r.k;
    if (r.face <= 2) ig -= gstep; else if (r.face <= 4) jg -= gstep; else kg -= gstep;
    const int64_t cg = row(bm, ig, jg, kg), cd = row(c.blk[q.bs], q.is, q.js, q.ks);
    for (int s = 0; s < NP; ++s) R[cg + s * nc] = R[cd + s * nc];
  }
}

// IRS_apply: scale (Scale_Residual_Cons, irs_scale_blk :108-116: R = -R / vol * dt * strang on the interior, the
// conservative path only), then per direction the ghost residual and njacobi Jacobi sweeps of
// R* = (R + beta (R*(c - off) + R*(c + off))) / (1 + 2 beta) over the interior (irs_smooth_blk, :204-236)
void irs_apply(Ctx& c, double* R, double dt, bool scale, const double* dtl = nullptr) {
  const int64_t nc = c.ncell;
  const double strang = 1.0, beta = c.sc.irs_beta;
  const int njacobi = c.sc.irs;
  if (scale)
    for (const Blk& b : c.blk)
      if (!b.ext)
      for (int k = 1; k <= b.n3; ++k)
        for (int j = 1; j <= b.n2; ++j)
          for (int i = 1; i <= b.n1; ++i) {
            const int64_t r = row(b, i, j, k);
            const double vol_ = b.vol[lin(b, i, j, k)], dtl_ = dtl ? dtl[r] : dt;
            for (int s = 0; s < NP; ++s) R[r + s * nc] = -R[r + s * nc] / vol_ * dtl_ * strang;
          }
  std::vector<double> rs1((size_t)nc * NP), rs2((size_t)nc * NP);
  for (int d = 1; d <= c.sc.ndir; ++d) {
    irs_ghost_residual(c, R);
    for (const Blk& b : c.blk) {
    if (b.ext) continue;
      const int64_t off = (d == 1) ? 1 : (d == 2 ? (int64_t)b.pi : (int64_t)b.pi * b.pj);
      const int64_t nflat = (int64_t)b.pi * b.pj * (b.n3 + 2 * GC);
      for (int s = 0; s < NP; ++s)
        for (int64_t q = 0; q < nflat; ++q) rs1[b.boff + q + s * nc] = R[b.boff + q + s * nc];
      for (int jac = 0; jac < njacobi; ++jac) {
        for (int k = 1; k <= b.n3; ++k)
          for (int j = 1; j <= b.n2; ++j)
            for (int i = 1; i <= b.n1; ++i) {
              const int64_t c0 = row(b, i, j, k);
              for (int s = 0; s < NP; ++s) {
                const int64_t x = c0 + s * nc;
                rs2[x] = (R[x] + beta * (rs1[x - off] + rs1[x + off])) / (1.0 + 2.0 * beta);
              }
            }
        for (int k = 1; k <= b.n3; ++k)
          for (int j = 1; j <= b.n2; ++j)
            for (int i = 1; i <= b.n1; ++i) {
              const int64_t c0 = row(b, i, j, k);
              for (int s = 0; s < NP; ++s) rs1[c0 + s * nc] = rs2[c0 + s * nc];
            }
      }
      for (int k = 1; k <= b.n3; ++k)
        for (int j = 1; j <= b.n2; ++j)
          for (int i = 1; i <= b.n1; ++i) {
            const int64_t c0 = row(b, i, j, k);
            for (int s = 0; s < NP; ++s) R[c0 + s * nc] = rs1[c0 + s * nc];
          }
    }
  }
}

// ---- local dt: dt_blk.inc (min rule) + Thermo_Cache_rrt_blk / _visc_blk ----
// ---- integration-variables = prec: the reference velocity Ur (Lib_Preconditioning.f90) ----

// comp_Ur (:84-142): mode 1 a uniform Uref (the sound speed above it), mode 2 the target preconditioned Mach number
// (the root w < 1 of A w^2 + B w + A = 0, w = (Ur / a)^2), mode 3 Weiss-Smith (|u| Ur-factor between eps_min a and a);
// the viscous floor in modes 2 and 3, then Ur-min
double comp_ur(const mb_scheme& sc, double vel, double sound, double ur_visc) {
  double Ur;
  const double eps = sc.prec_eps_min;
  if (sc.prec_uref > 0.0) {
    Ur = (vel > sc.prec_uref) ? sound : sc.prec_uref;
  } else if (sc.prec_mach > 0.0) {
    const double Mt = sc.prec_mach, m = vel / sound;
    const double A_q = 0.25 * m * m * (Mt * Mt - 1.0);
    const double B_q = Mt * Mt - 0.5 * m * m * (Mt * Mt + 1.0);
    if (std::fabs(A_q) > 1.0e-30) {
      const double S_q = -B_q / A_q, disc = S_q * S_q - 4.0;
      if (disc > 0.0 && S_q > 2.0) Ur = sound * std::sqrt(2.0 / (S_q + std::sqrt(disc)));
      else Ur = sound;
    } else {
      Ur = sound * eps;
    }
    Ur = std::max(Ur, eps * sound);
    Ur = std::min(Ur, sound);
    Ur = std::max(Ur, ur_visc);
  } else {
    if (vel < eps * sound) Ur = sound * eps;
    else if (vel >= sound) Ur = sound;
    else Ur = vel * sc.prec_ur_factor;
    Ur = std::max(Ur, ur_visc);
  }
  if (sc.prec_ur_min > 0.0) Ur = std::max(Ur, sc.prec_ur_min);
  return Ur;
}

// Update_Derived_Variables (:158-184): Ur_Blk (:187-264) of every interior cell of P, the viscous floor
// max(mu / (rho dx_min), k / (rho cp dx_min)) with mu and k of the Wilke rule, then Smooth_Ur_Blk (:269-295): passes of
// the max over the cell and its six face neighbours, the ghost neighbours 0
void update_ur(Ctx& c, const double* P) {
  const int64_t nc = c.ncell;
  const Thermo& th = c.th;
  for (const Blk& b : c.blk) {
    if (b.ext) continue;
    for (int k = 1; k <= b.n3; ++k)
      for (int j = 1; j <= b.n2; ++j)
        for (int i = 1; i <= b.n1; ++i) {
          const int64_t r = row(b, i, j, k);
          double pl[NP];
          for (int s = 0; s < NP; ++s) pl[s] = P[r + s * nc];
          double rho, R;
          rotot_rtot(th, pl[0], rho, R);
          const double T = pl[IP] / (rho * R);
          const double vel_mag = std::sqrt(pl[IU] * pl[IU] + pl[IV] * pl[IV] + pl[IW] * pl[IW]);
          double ur_visc = 0.0;
          if (c.sc.visc) {
            double dx_min = dlv(b, 0, i, j, k);
            for (int d = 1; d < c.sc.ndir; ++d) dx_min = std::min(dx_min, dlv(b, d, i, j, k));
            const int ti = tidx(th, T);
            const double td = T - ti;
            const double cp = f_cp(th, pl[0], ti, td, rho);
            double mu, lambda;
            wilke(th, pl[0], rho, ti, td, mu, lambda);
            ur_visc = std::max(mu / (rho * dx_min), lambda / (rho * cp * dx_min));
          }
          const double sound = f_ss(th, pl[0], pl[IP], rho, R);
          c.ur[r] = comp_ur(c.sc, vel_mag, sound, ur_visc);
        }
    std::vector<double> urb((size_t)b.n1 * b.n2 * b.n3);
    for (int pass = 0; pass < c.sc.prec_smooth; ++pass) {
      const int64_t si = 1, sj = b.pi, sk = (int64_t)b.pi * b.pj;
      size_t q = 0;
      for (int k = 1; k <= b.n3; ++k)
        for (int j = 1; j <= b.n2; ++j)
          for (int i = 1; i <= b.n1; ++i, ++q) {
            const int64_t r = row(b, i, j, k);
            double m = c.ur[r];
            m = std::max(m, c.ur[r - si]); m = std::max(m, c.ur[r + si]);
            m = std::max(m, c.ur[r - sj]); m = std::max(m, c.ur[r + sj]);
            m = std::max(m, c.ur[r - sk]); m = std::max(m, c.ur[r + sk]);
            urb[q] = m;
          }
      q = 0;
      for (int k = 1; k <= b.n3; ++k)
        for (int j = 1; j <= b.n2; ++j)
          for (int i = 1; i <= b.n1; ++i, ++q) c.ur[row(b, i, j, k)] = urb[q];
    }
  }
  c.ur_ready = true;
}

// the local step of one interior cell of P (Compute_dt_blk, dt_blk.inc:11-191), before the ramp factor
double cell_dt(const Ctx& c, const Blk& b, const double* P, int i, int j, int k) {
  const int64_t nc = c.ncell;
  const Thermo& th = c.th;
  int64_t r = row(b, i, j, k);
  double pl[NP];
  for (int s = 0; s < NP; ++s) pl[s] = P[r + s * nc];
  double rho, Rg;
  rotot_rtot(th, pl[0], rho, Rg);
  double Tc = pl[IP] / (rho * Rg);
  double Sound = f_ss(th, pl[0], pl[IP], rho, Rg);
  double dtc = 1e8;
  const bool prec = prec_on(c);
  double Alpha_ = 0.0, urc = 0.0;
  if (prec) {  // the pseudo-acoustic speed of the preconditioned system (dt_blk.inc:72-75)
    urc = c.ur[r];
    const double Beta_ = 1.0 / (Sound * Sound);
    Alpha_ = 0.5 * (1.0 - Beta_ * (urc * urc));
  }
  if (c.sc.dt_additive) {  // dt-rule = additive (dt_blk.inc:79-155)
    double ra_c = 0.0, ra_v = 0.0;
    for (int d = 0; d < c.sc.ndir; ++d) {
      double m0 = mv(b, d, 0, i, j, k), m1 = mv(b, d, 1, i, j, k), m2 = mv(b, d, 2, i, j, k);
      double gn = std::sqrt(m0 * m0 + m1 * m1 + m2 * m2);
      double vel_ = std::fabs(pl[IU] * m0 + pl[IV] * m1 + pl[IW] * m2) / gn;
      double lambda;
      if (prec) lambda = vel_ * (1.0 - Alpha_) + std::sqrt(Alpha_ * Alpha_ * (vel_ * vel_) + urc * urc);
      else lambda = vel_ + Sound;
      ra_c = ra_c + lambda * gn;
      ra_v = ra_v + gn * gn;
    }
    if (c.sc.visc) {
      if (c.sc.ndir == 3) {
        double g[3][3];
        for (int d = 0; d < 3; ++d) for (int a = 0; a < 3; ++a) g[d][a] = mv(b, d, a, i, j, k);
        auto dot = [&](int p, int q) { return g[p][0] * g[q][0] + g[p][1] * g[q][1] + g[p][2] * g[q][2]; };
        auto nr = [&](int p) { return std::sqrt(g[p][0] * g[p][0] + g[p][1] * g[p][1] + g[p][2] * g[p][2]); };
        double c12 = dot(0, 1) / (nr(0) * nr(1)), c13 = dot(0, 2) / (nr(0) * nr(2)), c23 = dot(1, 2) / (nr(1) * nr(2));
        double ss = c12 * c12 + c13 * c13 + c23 * c23;
        double qp = c12 * c13 * c23;
        if (ss + 2.0 * qp > 1.0) {
          double mr = 2.0 * std::sqrt(ss / 3.0) *
                      std::cos(std::acos(std::max(-1.0, std::min(1.0, 3.0 * std::sqrt(3.0) * qp / std::pow(ss, 1.5)))) / 3.0);
          ra_v = ra_v * 0.25 * (2.0 + mr + 1.0 / mr);
        }
      }
      double Ta = pl[IP] / (rho * Rg);
      int ta = tidx(th, Ta);
      double tda = Ta - ta;
      double cpa = f_cp(th, pl[0], ta, tda, rho);
      double cva = cpa - Rg;
      double mila, kla;
      wilke(th, pl[0], rho, ta, tda, mila, kla);
      if (c.sc.prandtl > 0.0) kla = mila * cpa / c.sc.prandtl;
      const double mie = 0.0, prt = 0.85;
      double Dmx = std::max(4.0 / 3.0 * (mila + mie) / rho, (kla + mie * cpa / prt) / (rho * cva));
      dtc = 1.0 / (ra_c / c.sc.cfl + Dmx * ra_v / c.sc.vnn);
    } else {
      dtc = c.sc.cfl / ra_c;
    }
  } else {
  for (int d = 0; d < c.sc.ndir; ++d) {
    double m0 = mv(b, d, 0, i, j, k), m1 = mv(b, d, 1, i, j, k), m2 = mv(b, d, 2, i, j, k);
    double nrm = std::sqrt(m0 * m0 + m1 * m1 + m2 * m2);
    double v0 = m0 / nrm, v1 = m1 / nrm, v2 = m2 / nrm;
    double vel_ = std::fabs(pl[IU] * v0 + pl[IV] * v1 + pl[IW] * v2);
    double lambda;
    if (prec) {
      const double cst_ = std::sqrt(Alpha_ * Alpha_ * (vel_ * vel_) + urc * urc);
      vel_ = vel_ * (1.0 - Alpha_);
      lambda = vel_ + cst_;
    } else {
      lambda = vel_ + Sound;
    }
    double dtd = dlv(b, d, i, j, k) / lambda * c.sc.cfl;
    dtc = std::min(dtd, dtc);
  }
  if (c.sc.visc) {
    int ti = tidx(th, Tc);
    double td = Tc - ti, mil, kl;
    wilke(th, pl[0], rho, ti, td, mil, kl);
    double mi = 0.0 + mil;
    for (int d = 0; d < c.sc.ndir; ++d) {
      double dl = dlv(b, d, i, j, k);
      double dtd = (rho * (dl * dl) * c.sc.vnn) / mi;
      dtc = std::min(dtd, dtc);
    }
  }
  }
  return dtc;
}

// cfl-rise-threshold (rampa_iter, Mod_dt.f90:57-58): the step's dt factor iter / rampa_iter while iter < rampa_iter, iter
// counting this step
double ramp_factor(const Ctx& c) {
  const int iter = c.st.steps + 1;
  return (iter < c.sc.cfl_rise) ? (double)iter / c.sc.cfl_rise : 1.0;
}

// Compute_dt: dtglobal = min(1e5, the cells' local steps times the ramp factor); with local time stepping (time-accurate
// = false) the cells' own steps, in dtl (per row of P, interior cells), are the step of each cell
double compute_dt(Ctx& c, const double* P, std::vector<double>* dtl = nullptr) {
  double dtglobal = 1e5;  // Mod_Explicit.f90:122
  const double rampa = ramp_factor(c);
  for (const Blk& b : c.blk) {
    if (b.ext) continue;
#pragma omp parallel for collapse(2) schedule(static) reduction(min : dtglobal)
    for (int k = 1; k <= b.n3; ++k)
      for (int j = 1; j <= b.n2; ++j)
        for (int i = 1; i <= b.n1; ++i) {
          double dtc = cell_dt(c, b, P, i, j, k) * rampa;
          if (dtl) (*dtl)[row(b, i, j, k)] = dtc;
          dtglobal = std::min(dtc, dtglobal);
        }
  }
  return dtglobal;
}

}  // namespace

extern "C" {

struct orc_ctx { Ctx c; };

int orc_init(const mb_mesh* mesh, const mb_scheme* sc, const mb_thermo* th, orc_ctx** out) {
  if (!mesh || !sc || !th || !out) return MB_E_ARG;
  if (sc->riemann < 1 || sc->riemann > 14 || sc->sensor < 0 || sc->sensor > 3 || sc->intvar < 0 || sc->intvar > 2 ||
      (sc->intvar >= 1 && sc->n_rk == 4) || (sc->riemann == 14) != (sc->intvar == 2) ||
      (sc->intvar == 2 && sc->local_dt != 1) || sc->irs < 0 || sc->irs > 4 || (sc->irs > 0 && sc->n_rk == 4))
    return MB_E_UNSUPPORTED;
  if (sc->irs > 0 && !(sc->irs_beta >= 0.0 && std::isfinite(sc->irs_beta))) return MB_E_ARG;
  if (sc->local_dt < 0 || sc->local_dt > 1 || sc->cfl_rise < 0) return MB_E_ARG;
  if (sc->intvar == 2 && !(sc->prec_eps_min > 0.0 && sc->prec_eps_min < 1.0 && sc->prec_smooth >= 0)) return MB_E_ARG;
  if (sc->limiter < 1 || sc->limiter > 6) return MB_E_UNSUPPORTED;
  if (sc->n_rk < 1 || sc->n_rk > 4) return MB_E_UNSUPPORTED;
  orc_ctx* o = new orc_ctx();
  Ctx& c = o->c;
  c.sc = *sc;
  c.sd = mb_effective_sensor(sc->riemann, sc->sensor);
  c.ncell = mesh->ncell_total;
  for (int b = 0; b < mesh->nblk; ++b) {
    const mb_block& q = mesh->blk[b];
    Blk k;
    k.n1 = q.n[0]; k.n2 = q.n[1]; k.n3 = q.n[2];
    k.pi = q.n[0] + 2 * GC; k.pj = q.n[1] + 2 * GC;
    k.boff = q.boff;
    k.fm1 = q.fm1; k.fm2 = q.fm2; k.fm3 = q.fm3; k.dl = q.dl; k.m = q.m; k.vol = q.vol;
    k.ext = q.group < 0;
    c.blk.push_back(k);
  }
  c.rec.assign(mesh->rec, mesh->rec + mesh->nrec);
  c.conn.assign(mesh->conn, mesh->conn + mesh->nconn);
  for (const mb_bc& r : c.rec)
    if (r.type != MB_BC_CONNECTION && r.type != MB_BC_EXTRAPOLATION && r.type != MB_BC_WALL &&
        r.type != MB_BC_INFLOW && r.type != MB_BC_SYMMETRY && r.type != MB_BC_WALL_T && r.type != MB_BC_OUTLET &&
        r.type != MB_BC_NONE) {
      delete o;
      return MB_E_UNSUPPORTED;
    }
  c.pg.assign((size_t)c.rec.size() * 6 * NP, 0.0);
  if (sc->n_rk == 4) c.acc4.assign((size_t)c.ncell * NP, 0.0);
  if (sc->intvar == 2) c.ur.assign((size_t)c.ncell, 0.0);
  Thermo& t = c.th;
  t.tmin = th->tmin; t.tmax = th->tmax; t.wm = th->wm; t.ri = RUNIV / th->wm;
  size_t nt = (size_t)(th->tmax - th->tmin + 1);
  t.cp_.assign(th->cp, th->cp + nt); t.h_.assign(th->h, th->h + nt);
  t.mu_.assign(th->mu, th->mu + nt); t.k_.assign(th->k, th->k + nt);
  t.cp = t.cp_.data() - th->tmin; t.h = t.h_.data() - th->tmin;
  t.mu = t.mu_.data() - th->tmin; t.k = t.k_.data() - th->tmin;
  std::memset(&c.st, 0, sizeof(c.st));
  *out = o;
  return MB_OK;
}

void orc_destroy(orc_ctx* o) { delete o; }

int orc_fill_ghosts(orc_ctx* o, double* P) { fill_ghosts(o->c, P); return MB_OK; }
// prec: an entry point that reads Ur computes it from the state it is given when nothing has yet (the reference's first
// Compute_dt); the time loop refreshes it after every stage's update (Mod_Explicit.f90:273-277)
static void ur_first(Ctx& c, const double* P) {
  if (prec_on(c) && !c.ur_ready) update_ur(c, P);
}

int orc_residual(orc_ctx* o, const double* P, double* R) {
  ur_first(o->c, P);
  residual(o->c, P, R);
  return MB_OK;
}
int orc_update(orc_ctx* o, double* P, const double* PO, const double* R, int irk, double dt) {
  Ctx& c = o->c;
  ur_first(c, P);
  // time-accurate = false: each cell's dtlocal, from the state at the start of the step (PO)
  std::vector<double> dtl;
  if (c.sc.local_dt) {
    dtl.assign((size_t)c.ncell, 0.0);
    compute_dt(c, PO, &dtl);
  }
  const double* dl = c.sc.local_dt ? dtl.data() : nullptr;
  if (c.sc.irs > 0) {  // RK_Newstate with IRS: the smoothing on a copy of R (Newstate_Conservative / _Primitive)
    std::vector<double> Rs(R, R + c.ncell * NP);
    irs_apply(c, Rs.data(), dt, c.sc.intvar == 0, dl);
    update(c, P, PO, Rs.data(), irk, dt, c.sc.intvar == 0, dl);
  } else {
    update(c, P, PO, R, irk, dt, false, dl);
  }
  return c.st.code;
}
int orc_dt(orc_ctx* o, const double* P, double* dt) {
  ur_first(o->c, P);
  *dt = compute_dt(o->c, P);
  return MB_OK;
}

// nsteps explicit steps (Mod_Explicit.f90:52-279): dt, PO <- P, then per stage ghost fill, residual, update.
int orc_step(orc_ctx* o, double* P, double* PO, double* R, int nsteps) {
  Ctx& c = o->c;
  const int64_t n = c.ncell * NP;
  for (int st = 0; st < nsteps; ++st) {
    if (c.st.done) return MB_OK;  // the residual end test stopped the case (Mod_Explicit.f90:363-370)
    ur_first(c, P);
    std::vector<double> dtl;
    if (c.sc.local_dt) dtl.assign((size_t)c.ncell, 0.0);
    double dt = compute_dt(c, P, c.sc.local_dt ? &dtl : nullptr);
    const double* dl = c.sc.local_dt ? dtl.data() : nullptr;
    if (!c.sc.local_dt) {  // time-accurate: Set_Global_dt and the clock (Mod_Explicit.f90:124-128)
      if (c.sc.time_clip) {  // Clip_dt_To_Timemax (Mod_dt.f90:283-296)
        double rem = c.sc.time_threshold - c.st.time;
        if (rem > 0.0 && dt > rem) dt = rem * (1.0 + 1e-12);
      }
      c.st.time += dt;
    }
    c.st.dt = dt;
    std::memcpy(PO, P, sizeof(double) * n);
    for (int irk = 1; irk <= c.sc.n_rk; ++irk) {
      fill_ghosts(c, P);
      residual(c, P, R);
      if (c.sc.irs > 0) irs_apply(c, R, dt, c.sc.intvar == 0, dl);
      update(c, P, PO, R, irk, dt, c.sc.irs > 0 && c.sc.intvar == 0, dl);
      if (prec_on(c)) update_ur(c, P);  // Ur of the updated state
    }
    // the residual diagnostic of the step (Compute_Residual_blk, Mod_Diagnostic.f90:64-104; the L2 norm of
    // Mod_Explicit.f90:325-358): sqrt of the sum over the interior cells of (new - old)^2 per primitive variable
    double r2[NP] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (const Blk& b : c.blk)
      if (!b.ext)
      for (int k = 1; k <= b.n3; ++k)
        for (int j = 1; j <= b.n2; ++j)
          for (int i = 1; i <= b.n1; ++i) {
            const int64_t r = row(b, i, j, k);
            for (int v = 0; v < NP; ++v) {
              const double d = P[r + v * c.ncell] - PO[r + v * c.ncell];
              r2[v] = r2[v] + d * d;
            }
          }
    for (int v = 0; v < NP; ++v) c.st.res[v] = std::sqrt(r2[v]);
    c.st.steps += 1;
    if (c.sc.res_stop > 0.0 && c.st.res[0] <= c.sc.res_stop) c.st.done = 1;
    if (c.st.code != MB_OK) return c.st.code;
  }
  return MB_OK;
}

int orc_get_status(orc_ctx* o, mb_status* st) { *st = o->c.st; return MB_OK; }

int orc_set_record_params(orc_ctx* o, int rec, const double* q) {
  if (rec < 0 || rec >= (int)o->c.rec.size()) return MB_E_ARG;
  for (int s = 0; s < MB_BC_NQ; ++s) o->c.rec[rec].q[s] = q[s];
  return MB_OK;
}

}  // extern "C"
