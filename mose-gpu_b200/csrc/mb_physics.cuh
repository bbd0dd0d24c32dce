// mb_physics.cuh -- device arithmetic of the face fluxes, boundary records, state update and local
// dt of the B200 engine. Templated on the flux arithmetic type R: double for the plain FP64 form,
// float for the mixed form (reconstruction, Riemann and viscous flux arithmetic in FP32; state,
// RK accumulation, T/p recovery and dt stay FP64 -- those routines are not templated).
//
// The FP64 instantiation keeps the reference's operation order statement by statement and is built
// with --fmad=false, so it rounds exactly as written. Sources (paths relative to the reference root):
//   convective face       src/lib/gpu/conv_physics.inc:1-179
//   limiters              src/lib/numerics/space/Lib_Limiters.f90:65-97
//   AUSM+ / LMRoe         src/lib/numerics/fluxes/riemann_open_body.inc:100-150, 679-730, 965-1091
//   HLLC (records)        src/lib/numerics/fluxes/Lib_Riemann_HLL.f90:21-134, 209-310
//   viscous face          src/lib/gpu/diff_cuf_kernels.inc:11-87, diff_physics.inc:1-161,
//                         Mod_Diffusive.f90:311-325 (face thermo)
//   connection records    src/lib/numerics/fluxes/bc/Lib_BC.f90:1770-1867, 2113-2178
//   extrapolation record  src/lib/numerics/fluxes/bc/Lib_BC.f90:1119-1165
//   state update          src/lib/gpu/newstate_cons_body.inc:1-89
//   local dt              src/lib/gpu/dt_blk.inc:11-222
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define MB_NP 5
#define MB_IU 1
#define MB_IV 2
#define MB_IW 3
#define MB_IPR 4

// the arithmetic is callable from host code as well (host-side debugging of the device arithmetic)
#define MB_HD __host__ __device__ __forceinline__
#define MB_HD_NOINLINE __host__ __device__ __noinline__

namespace mb {

constexpr int GC = 2;
constexpr double RUNIV = 8314.46261815324;  // lib/FLINT/src/lib/Lib_ThermoTransport.f90:13
constexpr int MB_E_TIMEOUT_DEV = -7;  // MB_E_TIMEOUT of the C ABI: a bounded device wait gave up

struct DBlk {
  int n1, n2, n3, pi, pj;
  int grp;              // the case of the block (its clock: Params::st[grp])
  int ndir;             // computational directions of the case (the dt rule)
  int kmirror;          // one cell deep in k with extrapolation (type 11) records on every cell of both k faces,
                        // or with no k-face record at all (taken as the same): its k ghosts equal the k = 1 values
                        // exactly (zero-gradient then cubic: 3a - 3a + a = a),
                        // so readers take the k = 1 cell and the fused stage does not fill them
  int rmap[6];          // offset of each face's record map in Params::rec_map (-1: none)
  long long boff;
  const double *fm1, *fm2, *fm3, *dl, *m, *vol;
  // FP32 copies of the face and cell geometry, made once by mb_init for the mixed form (null otherwise)
  const float *fm1f, *fm2f, *fm3f, *dlf, *mf;
};

// the geometry arrays in the flux arithmetic type
template <typename R> struct Geo;
template <> struct Geo<double> {
  MB_HD static const double* fm(const DBlk& b, int d) { return d == 0 ? b.fm1 : (d == 1 ? b.fm2 : b.fm3); }
  MB_HD static const double* dl(const DBlk& b) { return b.dl; }
  MB_HD static const double* m(const DBlk& b) { return b.m; }
};
template <> struct Geo<float> {
  MB_HD static const float* fm(const DBlk& b, int d) { return d == 0 ? b.fm1f : (d == 1 ? b.fm2f : b.fm3f); }
  MB_HD static const float* dl(const DBlk& b) { return b.dlf; }
  MB_HD static const float* m(const DBlk& b) { return b.mf; }
};

struct DRec {
  int type;
  int pg;               // row of the record in the transverse-stencil table (connections), -1 otherwise
  // type 4: mach, T0, p0, rel_fac, cos alpha, sin alpha, cos beta, sin beta (the angles' cos / sin taken once on the
  // host, so that every form uses the same values), the closure code (0 / 401 / 403 / 404 / 405 / 407), pamb, alpha,
  // beta, the face's unit tangent (3); type 6: T_wall; type 24: exit pressure, relaxation factor
  double q[16];
};

// device status + clock of the time loop (one per context)
struct DevState {
  unsigned long long dtmin_bits;  // min of the local dt of the step being computed (positive doubles order as u64)
  double dt;                      // dt of the current step
  double time;
  int steps;
  int code;
  int n_bad_state;
  int n_bad_thermo;
  int bad_blk, bad_i, bad_j, bad_k;
  int first_bad_claimed;
  int time_clip;                  // the case's stop rule: clip the last step onto t_end
  int done;                       // the case reached t_end: its tiles are skipped
  double t_end;                   // 0: no stop
  double res2[MB_NP];             // sum over the case's interior cells of (new - old)^2 of the step's primitive state
                                  // (the fused last stage accumulates it; zeroed at the step's start)
  double res_stop;                // the case stops once sqrt(res2[0]) of a step is <= res_stop (0: never)
  double rampf;                   // cfl-rise-threshold factor of the current step (1 without a ramp)
};

struct Params {
  const DBlk* blk;
  const int* rec_map;
  const DRec* rec;
  const long long* pgsrc;  // [connection][6]: the rows of P that bc_pg(:,1:6) of the connection record copies
  const double *cp, *h, *mu, *k;      // FP64 tables, indexed by the table row (pointer shifted by -tmin)
  const float *cpf, *hf, *muf, *kf;   // FP32 copies for the mixed form
  DevState* st;            // one clock per case: st[DBlk::grp]
  int ngroups;
  long long nc;
  int tmin, tmax;
  double wm, ri;
  double iri;              // 1 / ri (the mixed form's state update multiplies by it)
  int sd;                  // the shock sensor in effect (sd_dev): 0 none, 1 Tramel, 2 Chen
  int intvar;              // integration variables: 0 conservative, 1 primitive
  int local_dt;            // time-accurate = false: each cell's own step (from the state at the start of the step)
  int prec;                // integration-variables = prec: Ur of every row in ur (ghost rows 0), the local steps of
                           // the step in dtl (rows; fixed at the start of the step), HLLC-PC (14) reads ur
  const double* ur;
  const double* dtl;
  double prec_eps_min, prec_uref, prec_mach, prec_ur_factor, prec_ur_min;  // the preconditioning keys (comp_Ur)
  int cfl_rise;            // cfl-rise-threshold (0: no ramp)
  int lim, rs, visc, ndir, dt_additive, guard, state_check;
  double cfl, vnn, prandtl, schmidt, mco;
  void* recflux;           // boundary-record contributions [record][10] in the flux type (k_records)
  int stg;                 // mixed form: the tile staging of the sweep (STG_PLAIN 0, STG_TMA 1 of mb_engine.cuh)
  const void* tmap;        // STG_TMA: the TMA tensor map (CUtensorMap, device memory) of the sweep's input state as a
                           // 2-D tensor of (ncell_total rows, 5 variables), or null (the same tile by plain loads)
  int* queue;              // persistent sweep: the tile counter (null: one CTA per tile)
  int ntiles_run;          // tiles of the launch (persistent sweep)
  int pgrid;               // CTAs of a persistent launch (resident CTAs per SM x SMs)
  int pgrid_km;            // the same for the tiles of mirrored one-plane blocks (their own occupancy)
  int n_rk;                // 4: classical RK4 through the accumulator acc4
  int irk;                 // stage of the launch (1-based; set per launch)
  double* acc4;            // RK4: conserved accumulator (nc, 5), null otherwise
};

// The mixed form (R = float) applies the single-species identities of the reference's mixture formulas
// exactly: rho = rho_s, Y = rho_s / rho = 1, R_mix = Ri, cp_mix = cp(T), h_mix = h(T), the Wilke mixture
// viscosity / conductivity = the table values, and a zero species-diffusion flux. The FP64 form keeps the
// literal statements (their rounding is what the parity gate compares).
// The algebraically simplified flux path (single-species identities, one-quotient van Albada, net face fluxes, the
// reciprocal state update): the mixed form's FP32 arithmetic, and the FP64 production form's (its translation units
// define MB_FAST64 = 1 and are built with FMA contraction). The FP64 parity form keeps the reference's statements.
#ifndef MB_FAST64
#define MB_FAST64 0
#endif
template <typename R> struct Fast { static constexpr bool on = sizeof(R) == 4 || MB_FAST64; };

template <typename R> struct Tab;
template <> struct Tab<double> {
  MB_HD static const double* cp(const Params& p) { return p.cp; }
  MB_HD static const double* h(const Params& p) { return p.h; }
  MB_HD static const double* mu(const Params& p) { return p.mu; }
  MB_HD static const double* k(const Params& p) { return p.k; }
};
template <> struct Tab<float> {
  MB_HD static const float* cp(const Params& p) { return p.cpf; }
  MB_HD static const float* h(const Params& p) { return p.hf; }
  MB_HD static const float* mu(const Params& p) { return p.muf; }
  MB_HD static const float* k(const Params& p) { return p.kf; }
};

template <typename R> MB_HD R rsqrt_(R x);
template <> MB_HD double rsqrt_(double x) { return sqrt(x); }
template <> MB_HD float rsqrt_(float x) { return sqrtf(x); }

// ---- indexing (gpu/MOSE_Field_m.f90:78-109) ----
MB_HD long long lin(const DBlk& b, int i, int j, int k) {
  return (long long)(i + GC - 1) + (long long)(j + GC - 1) * b.pi + (long long)(k + GC - 1) * b.pi * b.pj;
}
MB_HD long long row(const DBlk& b, int i, int j, int k) { return b.boff + lin(b, i, j, k); }
MB_HD const double* fm1p(const DBlk& b, int i, int j, int k) {
  return b.fm1 + 4 * ((long long)i + (long long)(b.n1 + 1) * ((j - 1) + (long long)b.n2 * (k - 1)));
}
MB_HD const double* fm2p(const DBlk& b, int i, int j, int k) {
  return b.fm2 + 4 * ((long long)(i - 1) + (long long)b.n1 * (j + (long long)(b.n2 + 1) * (k - 1)));
}
MB_HD const double* fm3p(const DBlk& b, int i, int j, int k) {
  return b.fm3 + 4 * ((long long)(i - 1) + (long long)b.n1 * ((j - 1) + (long long)b.n2 * k));
}
MB_HD const double* fmp(const DBlk& b, int d, int i, int j, int k) {
  return d == 0 ? fm1p(b, i, j, k) : (d == 1 ? fm2p(b, i, j, k) : fm3p(b, i, j, k));
}
// index (in values) of the face (i,j,k) of direction d in its fm array
MB_HD long long fmi(const DBlk& b, int d, int i, int j, int k) {
  if (d == 0) return 4 * ((long long)i + (long long)(b.n1 + 1) * ((j - 1) + (long long)b.n2 * (k - 1)));
  if (d == 1) return 4 * ((long long)(i - 1) + (long long)b.n1 * (j + (long long)(b.n2 + 1) * (k - 1)));
  return 4 * ((long long)(i - 1) + (long long)b.n1 * ((j - 1) + (long long)b.n2 * k));
}
// 32-bit forms of lin and fmi for the sweep's hot path: mb_init rejects a block whose padded cells x 9 or face
// values reach 2^31, so every intra-block offset fits an int
MB_HD int lin32(const DBlk& b, int i, int j, int k) {
  return (i + GC - 1) + (j + GC - 1) * b.pi + (k + GC - 1) * b.pi * b.pj;
}
MB_HD int fmi32(const DBlk& b, int d, int i, int j, int k) {
  if (d == 0) return 4 * (i + (b.n1 + 1) * ((j - 1) + b.n2 * (k - 1)));
  if (d == 1) return 4 * ((i - 1) + b.n1 * (j + (b.n2 + 1) * (k - 1)));
  return 4 * ((i - 1) + b.n1 * ((j - 1) + b.n2 * k));
}
MB_HD double ld(const double* p) {
#ifdef __CUDA_ARCH__
  return __ldg(p);
#else
  return *p;
#endif
}
MB_HD float ld(const float* p) {
#ifdef __CUDA_ARCH__
  return __ldg(p);
#else
  return *p;
#endif
}

// min / max with the semantics of std::min / std::max of the CPU restatement ((b < a) ? b : a and
// (a < b) ? b : a): the same operand is returned for equal values, so signed zeros match as well
template <typename R> MB_HD R mn(R a, R b) { return (b < a) ? b : a; }
template <typename R> MB_HD R mx(R a, R b) { return (a < b) ? b : a; }

// ---- table lookups ----
// The table row of a temperature, kept inside [tmin, tmax-1] (NaN -> tmin): on the table this is
// int(T) as in the reference; off it the reference would index outside the table, which must never
// happen on the GPU (the thermo guard / state check report such a state).
template <typename R>
MB_HD int tidx(const Params& p, R T) {
  if (!(T >= (R)p.tmin)) return p.tmin;
  if (T >= (R)(p.tmax - 1)) return p.tmax - 1;
  return (int)T;
}
template <typename R>
MB_HD R tabT(const R* t, int ti, R td) {
  R a = t[ti];
  R b = t[ti + 1];
  return a + (b - a) * td;
}

// ---- FLINT leaves (Lib_ThermoTransport_dev.f90) ----
template <typename R>
MB_HD void rotot_rtot(const Params& p, R rhoi, R& rho, R& Rg) {
  if (Fast<R>::on) { rho = rhoi; Rg = (R)p.ri; return; }
  rho = (R)0 + rhoi;
  Rg = (R)0 + (R)p.ri * rhoi / rho;
}
template <typename R>
MB_HD R f_cp(const Params& p, R rhoi, int ti, R td, R rho) {
  R cpi = tabT(Tab<R>::cp(p), ti, td);
  if (Fast<R>::on) return cpi;
  return (R)0 + rhoi / rho * cpi;
}
template <typename R>
MB_HD R f_ss(const Params& p, R rhoi, R pr, R rho, R Rtot) {
  R T = pr / (Rtot * rho);
  int ti = tidx(p, T);
  R td = T - (R)ti;
  R cp = f_cp(p, rhoi, ti, td, rho);
  R gam = cp / (cp - Rtot);
  return rsqrt_(gam * Rtot * T);
}
template <typename R>
MB_HD R H0(const Params& p, R pr, R rhoi, R u) {
  R rho, Rg;
  rotot_rtot(p, rhoi, rho, Rg);
  R T = pr / (Rg * rho);
  int ti = tidx(p, T);
  R td = T - (R)ti;
  R e = Fast<R>::on ? tabT(Tab<R>::h(p), ti, td) : (R)0 + tabT(Tab<R>::h(p), ti, td) * rhoi / rho;
  return e + (R)0.5 * u * u;
}
// f_molecularWeight + co_fiij_dev + co_k_mi_lam_Wilke_dev, one species
template <typename R>
MB_HD void wilke(const Params& p, R rhoi, R rho, int ti, R td, R& mil, R& kl) {
  if (Fast<R>::on) { mil = tabT(Tab<R>::mu(p), ti, td); kl = tabT(Tab<R>::k(p), ti, td); return; }
  const R wm = (R)p.wm;
  R rho_ = (R)0 + rhoi;
  R wmt = (R)0 + (rhoi / rho_ / wm);
  wmt = (R)1 / wmt;
  R xi = rhoi * wmt / (rho * wm);
  R mi = tabT(Tab<R>::mu(p), ti, td);
  R ki = tabT(Tab<R>::k(p), ti, td);
  R sq_num = rsqrt_(mi);
  R inv_den = (R)1 / rsqrt_(mi + (R)1e-20);
  const R pw = (R)1;     // Mi_Mj_pow_m025(1,1) = (wm/wm)**(-0.25) = 1
  const R is8 = (R)0.25; // inv_sqrt8_1p(1,1) = 1/sqrt(8 (1 + 1))
  R ratio = sq_num * inv_den * pw;
  R one_plus = (R)1 + ratio;
  R fi = one_plus * one_plus * is8;
  R lam_den = (R)0 + xi * fi;
  R inv_ld = (R)1 / lam_den;
  mil = (R)0 + xi * mi * inv_ld;
  kl = (R)0 + xi * ki * inv_ld;
}

// ---- limiter (Lib_Limiters.f90:65-97) ----
// The ratio ru = y / (x + 1e-30) reaches ~1e27 where a slope is exactly zero (a velocity component
// that is zero, a symmetry point); ru*ru then overflows FP32 and van Albada turns into inf/inf = NaN,
// where FP64 gives phi = 1 (and the limited slope phi*x = 0). The FP32 form therefore holds |ru| to
// 1e18, beyond which every limiter function below has reached its FP32 limit value; the FP64 form
// is untouched.
template <typename R> MB_HD R hold_ratio(R ru) { return ru; }
template <> MB_HD float hold_ratio<float>(float ru) { return mx(mn(ru, 1e18f), -1e18f); }

template <typename R>
MB_HD R rlimiter(int lim, R x, R y) {
  R ru, phi;
  switch (lim) {
    case 1: {
      if (x * y < (R)0) return (R)0;
      R r = x;
      if (fabs(x) > fabs(y)) r = y;
      return r;
    }
    case 2:
      ru = hold_ratio(y / (x + (R)1e-30));
      phi = (ru + fabs(ru)) / ((R)1 + fabs(ru));
      return phi * x;
    case 3:
      if (Fast<R>::on)  // the same function as one quotient: x y (x + y) / (x^2 + y^2)
        return x * y * (x + y) / (x * x + y * y + (R)1e-30);
      ru = hold_ratio(y / (x + (R)1e-30));
      phi = (ru * ru + ru) / ((R)1 + ru * ru);
      return phi * x;
    case 4:
      ru = hold_ratio(y / (x + (R)1e-30));
      phi = mx((R)0, mn(mn((R)2 * ru, (R)0.5 * ((R)1 + ru)), (R)2));
      return phi * x;
    case 5:
      ru = hold_ratio(y / (x + (R)1e-30));
      phi = mx(mx((R)0, mn((R)2 * ru, (R)1)), mn(ru, (R)2));
      return phi * x;
    default:
      return (R)0;
  }
}

// ---- MOSE_open solvers of riemann_open_body.inc: AUSM+ (4), LMRoe (12) ----
template <typename R>
MB_HD R h_static(const Params& p, R rhoi, R pr) {
  R rho_, rg;
  rotot_rtot(p, rhoi, rho_, rg);
  R T = pr / (rg * rho_);
  R Tc = mx((R)p.tmin, mn(T, (R)(p.tmax - 1)));
  if (Tc != Tc) Tc = (R)p.tmin;
  int ti = (int)Tc;
  R td = Tc - (R)ti;
  int t1 = max(p.tmin, min(ti, p.tmax));
  int t2 = max(p.tmin, min(ti + 1, p.tmax));
  const R* h = Tab<R>::h(p);
  R hs = h[t1] + (h[t2] - h[t1]) * td;
  if (Fast<R>::on) return hs;
  return (R)0 + hs * rhoi / rho_;
}

template <typename R> MB_HD R powr(R x, R y);
template <> MB_HD double powr(double x, double y) { return pow(x, y); }
template <> MB_HD float powr(float x, float y) { return powf(x, y); }

// gamma of a state as riemann_open_body.inc writes f_gamma out (:349-366): T from p / (R rho_tot), the table row
// int(T) with both rows held to the table
template <typename R>
MB_HD R gam_state(const Params& p, R d, R pr, R dtot) {
  const R* CP = Tab<R>::cp(p);
  R rho_ = (R)0 + d;
  R rg_ = (R)0 + (R)p.ri * d / rho_;
  R T_ = pr / (rg_ * dtot);
  int Ti = (int)T_;
  R Td = T_ - (R)Ti;
  int t1 = max(p.tmin, min(Ti, p.tmax)), t2 = max(p.tmin, min(Ti + 1, p.tmax));
  R cp_ = (R)0 + d / dtot * (CP[t1] + (CP[t2] - CP[t1]) * Td);
  return cp_ / (cp_ - rg_);
}

template <typename R>
MB_HD void riemann_open(const Params& p, int rs, R bet, R dl, R ul, R vl, R wl, R pl, R al, R dltot,
                                             R dr, R ur, R vr, R wr, R pr, R ar, R drtot, R nx, R ny, R nz,
                                             R& F_r, R& F_u, R& F_v, R& F_w, R& F_E, R urL = (R)0, R urR = (R)0) {
  R unl = ul * nx + vl * ny + wl * nz;
  R unr = ur * nx + vr * ny + wr * nz;
  if (rs == 14) {  // HLLC-PC (riemann_open_body.inc:1092-1175, Riemann_HLLCprec): HLLC Batten with the signal speeds of
                   // the preconditioned system, Vr = min(Ur, a) of each side (urL, urR) and of the sqrt(rho) average
    const R hL = h_static(p, dl, pl), hR = h_static(p, dr, pr);
    const R eL = hL - pl / dltot, eR = hR - pr / drtot;
    const R kL = (R)0.5 * (ul * ul + vl * vl + wl * wl), kR = (R)0.5 * (ur * ur + vr * vr + wr * wr);
    const R h0l = hL + kL, h0r = hR + kR, EtL = eL + kL, EtR = eR + kR;
    const R FrL = dltot * unl;
    const R Ful = FrL * ul + pl * nx, Fvl = FrL * vl + pl * ny, Fwl = FrL * wl + pl * nz, Fel = FrL * h0l;
    const R FrR = drtot * unr;
    const R Fur = FrR * ur + pr * nx, Fvr = FrR * vr + pr * ny, Fwr = FrR * wr + pr * nz, Fer = FrR * h0r;
    const R srL = rsqrt_(dltot), srR = rsqrt_(drtot), den = srL + srR;
    const R u_roe = (srL * ul + srR * ur) / den, v_roe = (srL * vl + srR * vr) / den;
    const R w_roe = (srL * wl + srR * wr) / den, a_roe = (srL * al + srR * ar) / den;
    const R un_roe = u_roe * nx + v_roe * ny + w_roe * nz;
    const R VrL = mn(urL, al), VrR = mn(urR, ar), VrRoe = (srL * VrL + srR * VrR) / den;
    const R alL = ((R)1 - (VrL * VrL) / (al * al)) / (R)2, alR = ((R)1 - (VrR * VrR) / (ar * ar)) / (R)2;
    const R alRoe = ((R)1 - (VrRoe * VrRoe) / (a_roe * a_roe)) / (R)2;
    const R vLs = unl * ((R)1 - alL), vRs = unr * ((R)1 - alR), vRoes = un_roe * ((R)1 - alRoe);
    const R cLs = rsqrt_(mx(alL * alL * (unl * unl) + VrL * VrL, (R)0));
    const R cRs = rsqrt_(mx(alR * alR * (unr * unr) + VrR * VrR, (R)0));
    const R cRoes = rsqrt_(mx(alRoe * alRoe * (un_roe * un_roe) + VrRoe * VrRoe, (R)0));
    const R S1 = mn(mn((R)0, vLs - cLs), vRoes - cRoes);
    const R S4 = mx(mx((R)0, vRs + cRs), vRoes + cRoes);
    const R Sstar = (pr - pl + dltot * unl * (S1 - unl) - drtot * unr * (S4 - unr)) /
                    (dltot * (S1 - unl) - drtot * (S4 - unr));
    const R pstar = dltot * (unl - S1) * (unl - Sstar) + pl;
    if (S1 >= (R)0) {
      F_r = FrL; F_u = Ful; F_v = Fvl; F_w = Fwl; F_E = Fel;
    } else if (S4 <= (R)0) {
      F_r = FrR; F_u = Fur; F_v = Fvr; F_w = Fwr; F_E = Fer;
    } else if (Sstar >= (R)0) {
      const R q = S1 - Sstar;
      const R U1S = dltot * (S1 - unl) / q;
      const R U2S = ((S1 - unl) * dltot * ul + (pstar - pl) * nx) / q;
      const R U3S = ((S1 - unl) * dltot * vl + (pstar - pl) * ny) / q;
      const R U4S = ((S1 - unl) * dltot * wl + (pstar - pl) * nz) / q;
      const R U5S = ((S1 - unl) * dltot * EtL - pl * unl + pstar * Sstar) / q;
      F_r = FrL + S1 * (U1S - dltot); F_u = Ful + S1 * (U2S - dltot * ul); F_v = Fvl + S1 * (U3S - dltot * vl);
      F_w = Fwl + S1 * (U4S - dltot * wl); F_E = Fel + S1 * (U5S - dltot * EtL);
    } else {
      const R q = S4 - Sstar;
      const R U1S = drtot * (S4 - unr) / q;
      const R U2S = ((S4 - unr) * drtot * ur + (pstar - pr) * nx) / q;
      const R U3S = ((S4 - unr) * drtot * vr + (pstar - pr) * ny) / q;
      const R U4S = ((S4 - unr) * drtot * wr + (pstar - pr) * nz) / q;
      const R U5S = ((S4 - unr) * drtot * EtR - pr * unr + pstar * Sstar) / q;
      F_r = FrR + S4 * (U1S - drtot); F_u = Fur + S4 * (U2S - drtot * ur); F_v = Fvr + S4 * (U3S - drtot * vr);
      F_w = Fwr + S4 * (U4S - drtot * wr); F_E = Fer + S4 * (U5S - drtot * EtR);
    }
    return;
  }
  if (rs == 4) {
    const R ab = (R)0.125, aa = (R)0.1875;
    R vel = rsqrt_(ul * ul + vl * vl + wl * wl);
    R H_L = h_static(p, dl, pl) + (R)0.5 * vel * vel;
    vel = rsqrt_(ur * ur + vr * vr + wr * wr);
    R H_R = h_static(p, dr, pr) + (R)0.5 * vel * vel;
    R a_half = rsqrt_(al * ar);
    R ML = unl / a_half, MR = unr / a_half;
    R MplusL, pplusL, MminusR, pminusR;
    if (fabs(ML) < (R)1) {
      MplusL = (R)0.25 * ((ML + (R)1) * (ML + (R)1)) + ab * ((ML * ML - (R)1) * (ML * ML - (R)1));
      pplusL = (R)0.25 * ((ML + (R)1) * (ML + (R)1)) * ((R)2 - ML) + aa * ML * ((ML * ML - (R)1) * (ML * ML - (R)1));
    } else {
      MplusL = (R)0.5 * (ML + fabs(ML));
      pplusL = (R)0.5 * ((R)1 + copysign((R)1, ML));
    }
    if (fabs(MR) < (R)1) {
      MminusR = (R)(-0.25) * ((MR - (R)1) * (MR - (R)1)) - ab * ((MR * MR - (R)1) * (MR * MR - (R)1));
      pminusR = (R)0.25 * ((MR - (R)1) * (MR - (R)1)) * ((R)2 + MR) - aa * MR * ((MR * MR - (R)1) * (MR * MR - (R)1));
    } else {
      MminusR = (R)0.5 * (MR - fabs(MR));
      pminusR = (R)0.5 * ((R)1 - copysign((R)1, MR));
    }
    R Mhalf = MplusL + MminusR;
    R phalf = pplusL * pl + pminusR * pr;
    R mdotp = dltot * a_half * (R)0.5 * (Mhalf + fabs(Mhalf));
    R mdotm = drtot * a_half * (R)0.5 * (Mhalf - fabs(Mhalf));
    F_r = mdotp + mdotm;
    F_u = mdotp * ul + mdotm * ur + nx * phalf;
    F_v = mdotp * vl + mdotm * vr + ny * phalf;
    F_w = mdotp * wl + mdotm * wr + nz * phalf;
    F_E = mdotp * H_L + mdotm * H_R;
    return;
  }
  if (rs == 5) {  // AUSM+M (riemann_open_body.inc:152-242, Chen et al. 2020): the AUSMPW+ sound speed, Mach-number
                  // function f and the shock gate g of the face sensor bet
    const R ab = (R)0.125, aa = (R)0.1875, pi_ = (R)3.141592653589793;
    R Vl2 = ul * ul + vl * vl + wl * wl, Vr2 = ur * ur + vr * vr + wr * wr;
    R Hs_L = h_static(p, dl, pl);
    R vel_ = rsqrt_(Vl2);
    R H_L = Hs_L + (R)0.5 * vel_ * vel_;
    R gam_L = gam_state(p, dl, pl, dltot);
    R Hs_R = h_static(p, dr, pr);
    vel_ = rsqrt_(Vr2);
    R H_R = Hs_R + (R)0.5 * vel_ * vel_;
    R gam_R = gam_state(p, dr, pr, drtot);
    R gam = (R)0.5 * (gam_L + gam_R);
    R hnorm = (R)0.5 * (Hs_L + Hs_R);
    R cs = rsqrt_((R)2.0 * (gam - (R)1.0) / (gam + (R)1.0) * hnorm);
    R c12 = (unl + unr >= (R)0.0) ? cs * cs / mx(fabs(unl), cs) : cs * cs / mx(fabs(unr), cs);
    R ML = unl / c12, MR = unr / c12;
    R MplusL, pplusL, MminusR, pminusR;
    if (fabs(ML) < (R)1.0) {
      MplusL = (R)0.25 * ((ML + (R)1.0) * (ML + (R)1.0)) + ab * ((ML * ML - (R)1.0) * (ML * ML - (R)1.0));
      pplusL = (R)0.25 * ((ML + (R)1.0) * (ML + (R)1.0)) * ((R)2.0 - ML) + aa * ML * ((ML * ML - (R)1.0) * (ML * ML - (R)1.0));
    } else {
      MplusL = (R)0.5 * (ML + fabs(ML));
      pplusL = (R)0.5 * ((R)1.0 + copysign((R)1.0, ML));
    }
    if (fabs(MR) < (R)1.0) {
      MminusR = (R)-0.25 * ((MR - (R)1.0) * (MR - (R)1.0)) - ab * ((MR * MR - (R)1.0) * (MR * MR - (R)1.0));
      pminusR = (R)0.25 * ((MR - (R)1.0) * (MR - (R)1.0)) * ((R)2.0 + MR) - aa * MR * ((MR * MR - (R)1.0) * (MR * MR - (R)1.0));
    } else {
      MminusR = (R)0.5 * (MR - fabs(MR));
      pminusR = (R)0.5 * ((R)1.0 - copysign((R)1.0, MR));
    }
    R f_ = (R)0.5 * ((R)1.0 - cos(pi_ * mn((R)1.0, mx(fabs(ML), fabs(MR)))));
    R g_ = (R)0.5 * ((R)1.0 + cos(pi_ * bet));
    R rho12 = (R)0.5 * (dltot + drtot);
    R Mp = (R)-0.5 * ((R)1.0 - f_) * (pr - pl) / (rho12 * c12 * c12) * ((R)1.0 - g_);
    R M12 = MplusL + MminusR + Mp;
    R mdot = M12 * c12 * ((M12 >= (R)0.0) ? dltot : drtot);
    R fo = mn((R)1.0, mx(f_, (R)p.mco));
    R ps = (R)0.5 * (pl + pr) + (R)0.5 * (pplusL - pminusR) * (pl - pr) + fo * (pplusL + pminusR - (R)1.0) * (R)0.5 * (pl + pr);
    R gfac = g_ * gam * (pl + pr) / ((R)2.0 * c12) * pplusL * pminusR;
    R pux = -gfac * (ur - ul), puy = -gfac * (vr - vl), puz = -gfac * (wr - wl);
    F_r = mdot;
    if (M12 >= (R)0.0) {
      F_u = mdot * ul + ps * nx + pux; F_v = mdot * vl + ps * ny + puy; F_w = mdot * wl + ps * nz + puz; F_E = mdot * H_L;
    } else {
      F_u = mdot * ur + ps * nx + pux; F_v = mdot * vr + ps * ny + puy; F_w = mdot * wr + ps * nz + puz; F_E = mdot * H_R;
    }
    return;
  }
  if (rs == 11) {  // exact Godunov (riemann_open_body.inc:348-516): Newton on the star velocity, gamma of each state
    R gam_L = gam_state(p, dl, pl, dltot), gam_R = gam_state(p, dr, pr, drtot);
    R gm1 = gam_L - (R)1.0, gm4 = gam_R - (R)1.0;
    R d1 = (R)0.5 * gm1, d4 = (R)0.5 * gm4;
    R e1 = gam_L / d1, e4 = gam_R / d4;
    R un1 = ul * nx + vl * ny + wl * nz;
    R ut1 = ul - un1 * nx, vt1 = vl - un1 * ny, wt1 = wl - un1 * nz;
    R un4 = ur * nx + vr * ny + wr * nz;
    R ut4 = ur - un4 * nx, vt4 = vr - un4 * ny, wt4 = wr - un4 * nz;
    R r2i = un1 + ((R)2.0 / gm1) * al;
    R r1iv = un4 - ((R)2.0 / gm4) * ar;
    R dum = (pl < pr) ? gm4 / ((R)2.0 * gam_R) : gm1 / ((R)2.0 * gam_L);
    R z = (gm1 / gm4) * (ar / al) * powr(pl / pr, dum);
    R vel = (z * r2i + r1iv) / ((R)1.0 + z);
    R p3 = (R)1.0, p2 = (R)2.0 * p3, dpr = (R)0.0, dpl = (R)0.0;
    int iter = 0;
    R swl = (R)0.0, swr = (R)0.0, vw1 = (R)0.0, vw2 = (R)0.0, vw3 = (R)0.0, vw4 = (R)0.0, a2 = al, a3 = ar;
    while (fabs((R)1.0 - (p2 / p3)) >= (R)1e-5 && iter <= 1000) {
      if (vel < un1) {  // shock on the left
        R x = (gam_L + (R)1.0) * (vel - un1) / ((R)4.0 * al);
        R mrel = x - rsqrt_((R)1.0 + x * x);
        R c = gam_L * pl / al;
        p2 = pl + c * (vel - un1) * mrel;
        dpr = (R)2.0 * c * powr(mrel, (R)3.0) / ((R)1.0 + mrel * mrel);
        R rp = p2 / pl;
        swl = un1 + al * mrel;
        a2 = al * rsqrt_((gam_L + (R)1.0 + (gam_L - (R)1.0) * rp) / (gam_L + (R)1.0 + (gam_L - (R)1.0) / rp));
      } else {  // rarefaction on the left
        R delta = (R)0.5 * (gam_L - (R)1.0);
        R dum1 = (R)2.0 * gam_L / (gam_L - (R)1.0);
        a2 = al - delta * (vel - un1);
        p2 = pl * powr(a2 / al, dum1);
        dpr = -gam_L * p2 / a2;
        vw1 = un1 - al;
        vw2 = vel - a2;
      }
      if (vel > un4) {  // shock on the right
        R x = (gam_R + (R)1.0) * (vel - un4) / ((R)4.0 * ar);
        R mrel = x + rsqrt_((R)1.0 + x * x);
        R c = gam_R * pr / ar;
        p3 = pr + c * (vel - un4) * mrel;
        dpl = (R)2.0 * c * powr(mrel, (R)3.0) / ((R)1.0 + mrel * mrel);
        R rp = p3 / pr;
        swr = un4 + ar * mrel;
        a3 = ar * rsqrt_((gam_R + (R)1.0 + (gam_R - (R)1.0) * rp) / (gam_R + (R)1.0 + (gam_R - (R)1.0) / rp));
      } else {  // rarefaction on the right
        R delta = (R)0.5 * (gam_R - (R)1.0);
        R dum1 = (R)2.0 * gam_R / (gam_R - (R)1.0);
        a3 = ar + delta * (vel - un4);
        p3 = pr * powr(a3 / ar, dum1);
        dpl = gam_R * p3 / a3;
        vw3 = vel + a3;
        vw4 = un4 + ar;
      }
      vel = vel - ((p2 - p3) / (dpr - dpl));
      iter = iter + 1;
    }
    R af, pf, rhof, uf, vf, wf, Hs;
    if (vel > (R)0.0) {
      af = a2; pf = p2;
      if (vel <= un1) {
        if (swl > (R)0.0) { af = al; vel = un1; pf = pl; }
      } else if (vw1 > (R)0.0) {
        vel = un1; af = al; pf = pl;
      } else if (vw2 > (R)0.0) {
        af = (un1 + al / d1) / ((R)1.0 + (R)1.0 / d1);
        vel = af;
        pf = pl * powr(af / al, e1);
      }
      rhof = gam_L * pf / (af * af);
      uf = vel * nx + ut1; vf = vel * ny + vt1; wf = vel * nz + wt1;
      Hs = h_static(p, dl / dltot * rhof, pf);
    } else {
      af = a3; pf = p3;
      if (vel >= un4) {
        if (swr < (R)0.0) { af = ar; vel = un4; pf = pr; }
      } else if (vw4 < (R)0.0) {
        af = ar; vel = un4; pf = pr;
      } else if (vw3 < (R)0.0) {
        af = -(un4 - ar / d4) / ((R)1.0 + (R)1.0 / d4);
        vel = -af;
        pf = pr * powr(af / ar, e4);
      }
      rhof = gam_R * pf / (af * af);
      uf = vel * nx + ut4; vf = vel * ny + vt4; wf = vel * nz + wt4;
      Hs = h_static(p, dr / drtot * rhof, pf);
    }
    F_r = rhof * vel;
    F_u = F_r * uf + pf * nx;
    F_v = F_r * vf + pf * ny;
    F_w = F_r * wf + pf * nz;
    R uu = rsqrt_(vel * vel);
    F_E = F_r * (Hs + (R)0.5 * uu * uu);
    return;
  }
  if (rs == 13) {  // MiczekRoe (riemann_open_body.inc:518-676): the Miczek et al. 2015 preconditioned Roe flux
    R nmag = rsqrt_(nx * nx + ny * ny + nz * nz);
    if (nmag <= (R)0.0) { F_r = (R)0.0; F_u = (R)0.0; F_v = (R)0.0; F_w = (R)0.0; F_E = (R)0.0; return; }
    R n1 = nx / nmag, n2 = ny / nmag, n3 = nz / nmag;
    R tx = (R)1.0, ty = (R)0.0, tz = (R)0.0;
    if (!(fabs(n1) < (R)0.9)) { tx = (R)0.0; ty = (R)1.0; }
    R dot = tx * n1 + ty * n2 + tz * n3;
    R t1x = tx - dot * n1, t1y = ty - dot * n2, t1z = tz - dot * n3;
    R tmag = rsqrt_(t1x * t1x + t1y * t1y + t1z * t1z);
    if (tmag <= (R)0.0) {
      t1x = -n2; t1y = n1; t1z = (R)0.0;
      tmag = rsqrt_(t1x * t1x + t1y * t1y + t1z * t1z);
    }
    t1x = t1x / tmag; t1y = t1y / tmag; t1z = t1z / tmag;
    R t2x = n2 * t1z - n3 * t1y, t2y = n3 * t1x - n1 * t1z, t2z = n1 * t1y - n2 * t1x;
    R unL = ul * n1 + vl * n2 + wl * n3, unR = ur * n1 + vr * n2 + wr * n3;
    R ut1L = ul * t1x + vl * t1y + wl * t1z, ut1R = ur * t1x + vr * t1y + wr * t1z;
    R ut2L = ul * t2x + vl * t2y + wl * t2z, ut2R = ur * t2x + vr * t2y + wr * t2z;
    R hL = h_static(p, dl, pl), hR = h_static(p, dr, pr);
    R H0L = hL + (R)0.5 * (ul * ul + vl * vl + wl * wl);
    R H0R = hR + (R)0.5 * (ur * ur + vr * vr + wr * wr);
    R FL1 = dltot * unL, FL2 = dltot * unL * ul + pl * n1, FL3 = dltot * unL * vl + pl * n2,
           FL4 = dltot * unL * wl + pl * n3, FL5 = dltot * unL * H0L;
    R FR1 = drtot * unR, FR2 = drtot * unR * ur + pr * n1, FR3 = drtot * unR * vr + pr * n2,
           FR4 = drtot * unR * wr + pr * n3, FR5 = drtot * unR * H0R;
    R sRL = rsqrt_(dltot), sRR = rsqrt_(drtot), den = sRL + sRR;
    R u = (sRL * ul + sRR * ur) / den, v = (sRL * vl + sRR * vr) / den, w = (sRL * wl + sRR * wr) / den;
    R H = (sRL * H0L + sRR * H0R) / den;
    R un = u * n1 + v * n2 + w * n3;
    R rho = sRL * sRR;
    R u2 = u * u + v * v + w * w;
    R gam_L = gam_state(p, dl, pl, dltot), gam_R = gam_state(p, dr, pr, drtot);
    R kL = gam_L - (R)1.0, kR = gam_R - (R)1.0;
    R chiL = al * al - kL * hL, chiR = ar * ar - kR * hR;
    R kRoe = (sRL * kL + sRR * kR) / den, chiRoe = (sRL * chiL + sRR * chiR) / den;
    R cc = rsqrt_(mx((R)1e-30, chiRoe + kRoe * (H - (R)0.5 * u2)));
    R Mcut = mx((R)1e-6, (R)p.mco);
    R Mloc = rsqrt_(u2) / cc;
    R mu = mn((R)1.0, mx(Mloc, Mcut));
    R del = (R)1.0 / mu - (R)1.0, del2 = del * del, om = (R)1.0 / ((R)1.0 + del2);
    R drho = drtot - dltot, dp = pr - pl, dun = unR - unL, dut1 = ut1R - ut1L, dut2 = ut2R - ut2L;
    R p11 = un, p12 = rho * ((R)1.0 + del * un / cc), p13 = del / cc, p22 = un - del * cc;
    R p23 = ((R)1.0 - del * un / cc) / rho, p32 = rho * cc * (cc + del * un), p33 = un + cc * del;
    R s2 = ((R)1.0 + del2) * cc * cc - del2 * un * un;
    R s = rsqrt_(mx((R)1e-30, s2));
    s2 = s * s;
    R le = un, lp = un + s, lm = un - s;
    R va1 = (p11 - lm) * drho + p12 * dun + p13 * dp, va2 = (p22 - lm) * dun + p23 * dp,
           va3 = p32 * dun + (p33 - lm) * dp;
    R vb1 = (p11 - lp) * drho + p12 * dun + p13 * dp, vb2 = (p22 - lp) * dun + p23 * dp,
           vb3 = p32 * dun + (p33 - lp) * dp;
    R w1 = (p11 - lp) * va1 + p12 * va2 + p13 * va3, w2 = (p22 - lp) * va2 + p23 * va3,
           w3 = p32 * va2 + (p33 - lp) * va3;
    R x1 = (p11 - le) * va1 + p12 * va2 + p13 * va3, x2 = (p22 - le) * va2 + p23 * va3,
           x3 = p32 * va2 + (p33 - le) * va3;
    R z1 = (p11 - le) * vb1 + p12 * vb2 + p13 * vb3, z2 = (p22 - le) * vb2 + p23 * vb3,
           z3 = p32 * vb2 + (p33 - le) * vb3;
    R c1 = fabs(le) / (-s2), c2 = fabs(lp) / ((R)2.0 * s2), c3 = fabs(lm) / ((R)2.0 * s2);
    R g1 = c1 * w1 + c2 * x1 + c3 * z1, g2 = c1 * w2 + c2 * x2 + c3 * z2, g3 = c1 * w3 + c2 * x3 + c3 * z3;
    R ddrho = g1 - (rho * del / cc) * om * g2 - (del2 / (cc * cc)) * om * g3;
    R ddun = om * (g2 + (del / (rho * cc)) * g3);
    R ddp = om * (-rho * cc * del * g2 + g3);
    R ddut1 = fabs(un) * dut1, ddut2 = fabs(un) * dut2;
    R ddux = ddun * n1 + ddut1 * t1x + ddut2 * t2x;
    R dduy = ddun * n2 + ddut1 * t1y + ddut2 * t2y;
    R dduz = ddun * n3 + ddut1 * t1z + ddut2 * t2z;
    F_r = (R)0.5 * (FL1 + FR1) - (R)0.5 * (ddrho);
    F_u = (R)0.5 * (FL2 + FR2) - (R)0.5 * (u * ddrho + rho * ddux);
    F_v = (R)0.5 * (FL3 + FR3) - (R)0.5 * (v * ddrho + rho * dduy);
    F_w = (R)0.5 * (FL4 + FR4) - (R)0.5 * (w * ddrho + rho * dduz);
    F_E = (R)0.5 * (FL5 + FR5) - (R)0.5 * ((R)0.5 * u2 * ddrho + rho * (u * ddux + v * dduy + w * dduz) + ddp / kRoe);
    return;
  }
  if (rs == 8) {  // LLF / Rusanov (riemann_open_body.inc:244-278)
    R lf_a = mx(mx(fabs(unl - al), fabs(unr - ar)), mx(fabs(unl + al), fabs(unr + ar)));
    R rho_ = (R)0 + dr;
    R Hs_R = h_static(p, dr, pr);
    R vel_ = rsqrt_(ur * ur + vr * vr + wr * wr);
    R FrR = rho_ * (ur * nx + vr * ny + wr * nz);
    R Fur = FrR * ur + pr * nx, Fvr = FrR * vr + pr * ny, Fwr = FrR * wr + pr * nz;
    R Fer = FrR * (Hs_R + (R)0.5 * vel_ * vel_);
    R e0r_ = (Hs_R - pr / rho_) + (R)0.5 * vel_ * vel_;
    rho_ = (R)0 + dl;
    R Hs_L = h_static(p, dl, pl);
    vel_ = rsqrt_(ul * ul + vl * vl + wl * wl);
    R FrL = rho_ * (ul * nx + vl * ny + wl * nz);
    R Ful = FrL * ul + pl * nx, Fvl = FrL * vl + pl * ny, Fwl = FrL * wl + pl * nz;
    R Fel = FrL * (Hs_L + (R)0.5 * vel_ * vel_);
    R e0l_ = (Hs_L - pl / rho_) + (R)0.5 * vel_ * vel_;
    F_r = (R)0.5 * (FrL + FrR - lf_a * (drtot - dltot));
    F_u = (R)0.5 * (Fur + Ful - lf_a * (drtot * ur - dltot * ul));
    F_v = (R)0.5 * (Fvr + Fvl - lf_a * (drtot * vr - dltot * vl));
    F_w = (R)0.5 * (Fwr + Fwl - lf_a * (drtot * wr - dltot * wl));
    F_E = (R)0.5 * (Fel + Fer - lf_a * (drtot * e0r_ - dltot * e0l_));
    return;
  }
  if (rs == 9) {  // SLAU2 (riemann_open_body.inc:280-347): SLAU with the Kitamura-Shima 2013 pressure flux
    // the reference holds F_r, the pressure flux and H to +-1e150; FP32 holds them to +-3e38 (1e150 is inf there)
    const R big = (R)(sizeof(R) == 4 ? 3.0e38 : 1.0e150);
    R Vl2 = ul * ul + vl * vl + wl * wl;
    R Vr2 = ur * ur + vr * vr + wr * wr;
    R af = (R)0.5 * (al + ar);
    R ml = unl / af, mr = unr / af;
    R mt = mn((R)1, rsqrt_((R)0.5 * (Vl2 + Vr2)) / af);
    R chi = ((R)1 - mt) * ((R)1 - mt);
    R vnm = (dltot * fabs(unl) + drtot * fabs(unr)) / (dltot + drtot);
    R frho = -mx(mn(ml, (R)0), (R)(-1)) * mn(mx(mr, (R)0), (R)1);
    R vnl = ((R)1 - frho) * vnm + frho * fabs(unl);
    R vnr = ((R)1 - frho) * vnm + frho * fabs(unr);
    F_r = (R)0.5 * (dltot * (unl + vnl) + drtot * (unr - vnr) - (chi / af) * (pr - pl));
    F_r = mx(-big, mn(F_r, big));
    R bl, br;
    if (fabs(ml) < (R)1) bl = (R)0.25 * ((R)2 - ml) * ((ml + (R)1) * (ml + (R)1));
    else if (ml >= (R)0) bl = (R)1;
    else bl = (R)0;
    if (fabs(mr) < (R)1) br = (R)0.25 * ((R)2 + mr) * ((mr - (R)1) * (mr - (R)1));
    else if (mr >= (R)0) br = (R)0;
    else br = (R)1;
    R ph = (R)0.5 * (pl + pr) + (R)0.5 * (bl - br) * (pl - pr) +
           rsqrt_((R)0.5 * (Vl2 + Vr2)) * (bl + br - (R)1) * af * (R)0.5 * (dltot + drtot);
    ph = mx(-big, mn(ph, big));
    R Hs_L = h_static(p, dl, pl);
    R Hs_R = h_static(p, dr, pr);
    R H_L = Hs_L + (R)0.5 * rsqrt_(Vl2) * rsqrt_(Vl2);
    R H_R = Hs_R + (R)0.5 * rsqrt_(Vr2) * rsqrt_(Vr2);
    H_L = mx(-big, mn(H_L, big));
    H_R = mx(-big, mn(H_R, big));
    if (F_r >= (R)0) {
      F_u = F_r * ul + nx * ph; F_v = F_r * vl + ny * ph; F_w = F_r * wl + nz * ph; F_E = F_r * H_L;
    } else {
      F_u = F_r * ur + nx * ph; F_v = F_r * vr + ny * ph; F_w = F_r * wr + nz * ph; F_E = F_r * H_R;
    }
    return;
  }
  const R* H = Tab<R>::h(p);
  const R* CP = Tab<R>::cp(p);
  R rho_, Rl, Rr;
  rotot_rtot(p, dl, rho_, Rl);
  rotot_rtot(p, dr, rho_, Rr);
  R inv_dltot = (R)1 / dltot, inv_drtot = (R)1 / drtot;
  R Tl = pl * inv_dltot / Rl, Tr = pr * inv_drtot / Rr;
  int Til = tidx(p, Tl);
  int Tir = tidx(p, Tr);
  R dTl = Tl - (R)Til, dTr = Tr - (R)Tir;
  R srL = rsqrt_(dltot), srR = rsqrt_(drtot);
  R inv_sr = (R)1 / (srL + srR);
  R rho_roe = srL * srR;
  R u_roe = (srR * ur + srL * ul) * inv_sr;
  R v_roe = (srR * vr + srL * vl) * inv_sr;
  R w_roe = (srR * wr + srL * wl) * inv_sr;
  R R_roe = (srR * Rr + srL * Rl) * inv_sr;
  R T_roe = (srR * Tr + srL * Tl) * inv_sr;
  R h0l = (R)0, h0r = (R)0, cv_roe = (R)0, sum_ei = (R)0;
  {
    R invW = (R)(RUNIV / p.wm);
    R hl = H[Til] + (H[Til + 1] - H[Til]) * dTl;
    R hr = H[Tir] + (H[Tir + 1] - H[Tir]) * dTr;
    R el = hl - invW * Tl, er = hr - invW * Tr;
    if (Fast<R>::on) {  // one species: Y = 1, d_roe = 1
      h0l = hl;
      h0r = hr;
      cv_roe = (R)0.5 * (CP[Til] + (CP[Til + 1] - CP[Til]) * dTl + CP[Tir] + (CP[Tir + 1] - CP[Tir]) * dTr) - invW;
      sum_ei = (srR * er + srL * el) * inv_sr;
    } else {
    h0l = h0l + hl * dl * inv_dltot;
    h0r = h0r + hr * dr * inv_drtot;
    R d_roe = (srR * dr * inv_drtot + srL * dl * inv_dltot) * inv_sr;
    cv_roe = cv_roe + d_roe * ((R)0.5 * (CP[Til] + (CP[Til + 1] - CP[Til]) * dTl + CP[Tir] +
                                         (CP[Tir + 1] - CP[Tir]) * dTr) - invW);
    sum_ei = sum_ei + d_roe * (srR * er + srL * el) * inv_sr;
    }
  }
  h0l = h0l + (R)0.5 * (ul * ul + vl * vl + wl * wl);
  h0r = h0r + (R)0.5 * (ur * ur + vr * vr + wr * wr);
  R h0_roe = (srR * h0r + srL * h0l) * inv_sr;
  R gam_roe = (R)1 + R_roe / cv_roe;
  R vel2 = u_roe * u_roe + v_roe * v_roe + w_roe * w_roe;
  R a_roe = rsqrt_((gam_roe - (R)1) * (h0_roe - (R)0.5 * vel2 + cv_roe * T_roe - sum_ei));
  R un_roe = u_roe * nx + v_roe * ny + w_roe * nz;
  if (rs == 6) {  // HLLE++ (riemann_open_body.inc:728-810): HLLE and Roe wave speeds blended by the face sensor
    R S1 = mn(mn((R)0.0, unl - al), un_roe - a_roe);
    R S4 = mx(mx((R)0.0, unr + ar), un_roe + a_roe);
    R inv_denom = (R)1.0 / (S4 - S1);
    R lam1_hlle = fabs((S4 + S1) * un_roe * inv_denom - (R)2.0 * S4 * S1 * inv_denom);
    R lam2_hlle = fabs((S4 + S1) * (un_roe - a_roe) * inv_denom - (R)2.0 * S4 * S1 * inv_denom);
    R lam3_hlle = fabs((S4 + S1) * (un_roe + a_roe) * inv_denom - (R)2.0 * S4 * S1 * inv_denom);
    R eps_ = (R)0.3 * (fabs(un_roe) + a_roe);
    R lam1_roe = fabs(un_roe);
    R vv = un_roe - a_roe;
    R lam2_roe = fabs(vv);
    if (fabs(vv) <= eps_) lam2_roe = (vv * vv + eps_ * eps_) / ((R)2.0 * eps_);
    vv = un_roe + a_roe;
    R lam3_roe = fabs(vv);
    if (fabs(vv) <= eps_) lam3_roe = (vv * vv + eps_ * eps_) / ((R)2.0 * eps_);
    R lam1_pp = bet * lam1_roe + ((R)1.0 - bet) * lam1_hlle;
    R lam2_pp = bet * lam2_roe + ((R)1.0 - bet) * lam2_hlle;
    R lam3_pp = bet * lam3_roe + ((R)1.0 - bet) * lam3_hlle;
    R rL = (R)0.0 + dl;
    R FrL = rL * (ul * nx + vl * ny + wl * nz);
    R Ful = FrL * ul + pl * nx, Fvl = FrL * vl + pl * ny, Fwl = FrL * wl + pl * nz;
    R Hs_L = h_static(p, dl, pl);
    R vel_ = rsqrt_(ul * ul + vl * vl + wl * wl);
    R Fel = FrL * (Hs_L + (R)0.5 * vel_ * vel_);
    R rR = (R)0.0 + dr;
    R FrR = rR * (ur * nx + vr * ny + wr * nz);
    R Fur = FrR * ur + pr * nx, Fvr = FrR * vr + pr * ny, Fwr = FrR * wr + pr * nz;
    R Hs_R = h_static(p, dr, pr);
    vel_ = rsqrt_(ur * ur + vr * vr + wr * wr);
    R Fer = FrR * (Hs_R + (R)0.5 * vel_ * vel_);
    F_r = (R)0.5 * (FrL + FrR); F_u = (R)0.5 * (Ful + Fur); F_v = (R)0.5 * (Fvl + Fvr); F_w = (R)0.5 * (Fwl + Fwr);
    F_E = (R)0.5 * (Fel + Fer);
    R drho = drtot - dltot, dp = pr - pl, du = ur - ul, dv = vr - vl, dw = wr - wl, dun = unr - unl;
    R t1x, t1y, t1z;
    if (fabs(nx) < (R)0.9) { t1x = (R)0.0; t1y = -nz; t1z = ny; } else { t1x = -nz; t1y = (R)0.0; t1z = nx; }
    R normt = rsqrt_(t1x * t1x + t1y * t1y + t1z * t1z);
    t1x = t1x / normt; t1y = t1y / normt; t1z = t1z / normt;
    R t2x = ny * t1z - nz * t1y, t2y = nz * t1x - nx * t1z, t2z = nx * t1y - ny * t1x;
    R alpha_m = (dp - rho_roe * a_roe * dun) / ((R)2.0 * a_roe * a_roe);
    R alpha_c = drho - dp / (a_roe * a_roe);
    R alpha_s1 = rho_roe * (du * t1x + dv * t1y + dw * t1z);
    R alpha_s2 = rho_roe * (du * t2x + dv * t2y + dw * t2z);
    R alpha_p = (dp + rho_roe * a_roe * dun) / ((R)2.0 * a_roe * a_roe);
    F_r = F_r - (R)0.5 * (alpha_c * lam1_pp + alpha_m * lam2_pp + alpha_p * lam3_pp);
    F_u = F_u - (R)0.5 * (alpha_c * lam1_pp * u_roe);
    F_v = F_v - (R)0.5 * (alpha_c * lam1_pp * v_roe);
    F_w = F_w - (R)0.5 * (alpha_c * lam1_pp * w_roe);
    F_u = F_u - (R)0.5 * lam1_pp * (alpha_s1 * t1x + alpha_s2 * t2x);
    F_v = F_v - (R)0.5 * lam1_pp * (alpha_s1 * t1y + alpha_s2 * t2y);
    F_w = F_w - (R)0.5 * lam1_pp * (alpha_s1 * t1z + alpha_s2 * t2z);
    F_u = F_u - (R)0.5 * (alpha_m * lam2_pp * (u_roe - a_roe * nx) + alpha_p * lam3_pp * (u_roe + a_roe * nx));
    F_v = F_v - (R)0.5 * (alpha_m * lam2_pp * (v_roe - a_roe * ny) + alpha_p * lam3_pp * (v_roe + a_roe * ny));
    F_w = F_w - (R)0.5 * (alpha_m * lam2_pp * (w_roe - a_roe * nz) + alpha_p * lam3_pp * (w_roe + a_roe * nz));
    F_E = F_E - (R)0.5 * lam1_pp * (alpha_c * (R)0.5 * (u_roe * u_roe + v_roe * v_roe + w_roe * w_roe));
    F_E = F_E - (R)0.5 * lam1_pp *
                    (alpha_s1 * (u_roe * t1x + v_roe * t1y + w_roe * t1z) + alpha_s2 * (u_roe * t2x + v_roe * t2y + w_roe * t2z));
    F_E = F_E - (R)0.5 * (alpha_m * lam2_pp * (h0_roe - a_roe * un_roe) + alpha_p * lam3_pp * (h0_roe + a_roe * un_roe));
    return;
  }
  if (rs == 7 || rs == 10) {  // HLLC+Tramel (:811-880) and HLLC+Chen (:881-964): HLLC with the face sensor
    R S1 = mn(mn((R)0.0, unl - al), un_roe - a_roe);
    R S4 = mx(mx((R)0.0, unr + ar), un_roe + a_roe);
    R FrE = (R)0.0, FuE = (R)0.0, FvE = (R)0.0, FwE = (R)0.0, FeE = (R)0.0;
    if (rs == 7) {  // riemann_HLLE
      R inv_denom = (R)1.0 / (S4 - S1);
      R FrL = dltot * unl, FrR = drtot * unr;
      FrE = (S4 * FrL - S1 * FrR + S1 * S4 * (drtot - dltot)) * inv_denom;
      FuE = (S4 * (FrL * ul + pl * nx) - S1 * (FrR * ur + pr * nx) + S1 * S4 * (drtot * ur - dltot * ul)) * inv_denom;
      FvE = (S4 * (FrL * vl + pl * ny) - S1 * (FrR * vr + pr * ny) + S1 * S4 * (drtot * vr - dltot * vl)) * inv_denom;
      FwE = (S4 * (FrL * wl + pl * nz) - S1 * (FrR * wr + pr * nz) + S1 * S4 * (drtot * wr - dltot * wl)) * inv_denom;
      FeE = (S4 * (FrL * h0l) - S1 * (FrR * h0r) + S1 * S4 * (drtot * (h0r - pr / drtot) - dltot * (h0l - pl / dltot))) *
            inv_denom;
    }
    R e0l = h0l - pl / dltot, e0r = h0r - pr / drtot;
    R inv_denom = (R)1.0 / (dltot * (S1 - unl) - drtot * (S4 - unr));
    R Sstar = (pr - pl + dltot * unl * (S1 - unl) - drtot * unr * (S4 - unr)) * inv_denom;
    R pstar = dltot * (unl - S1) * (unl - Sstar) + pl;
    R ch_pref = (R)0.0, ch_fstar = (R)0.0, ch_g = (R)0.0, ch_dU = (R)0.0, ch_dutx = (R)0.0, ch_duty = (R)0.0, ch_dutz = (R)0.0;
    if (rs == 10) {  // the Chen all-speed terms (the sensor h of the face is bet)
      R ch_phiL = dltot * (S1 - unl), ch_phiR = drtot * (S4 - unr);
      ch_pref = ch_phiL * ch_phiR / (ch_phiR - ch_phiL);
      R ch_Mloc = mn((R)1.0, mx(rsqrt_(ul * ul + vl * vl + wl * wl) / al,
                                              rsqrt_(ur * ur + vr * vr + wr * wr) / ar));
      ch_Mloc = mx((R)p.mco, ch_Mloc);
      R om = (R)1.0 - ch_Mloc * ch_Mloc;
      R ch_fM = ch_Mloc * rsqrt_((R)4.0 + om * om) / ((R)1.0 + ch_Mloc * ch_Mloc);
      ch_g = (R)1.0 - powr(bet, ch_Mloc);
      ch_fstar = ch_fM + ch_g * ((R)1.0 - ch_fM);
      ch_dU = unr - unl;
      ch_dutx = (ur - ul) - ch_dU * nx; ch_duty = (vr - vl) - ch_dU * ny; ch_dutz = (wr - wl) - ch_dU * nz;
    }
    R FrC, FuC, FvC, FwC, FeC;
    if (S1 >= (R)0.0) {
      FrC = dltot * unl; FuC = FrC * ul + pl * nx; FvC = FrC * vl + pl * ny; FwC = FrC * wl + pl * nz; FeC = FrC * h0l;
    } else if (Sstar >= (R)0.0) {
      FrC = dltot * unl; FuC = FrC * ul + pl * nx; FvC = FrC * vl + pl * ny; FwC = FrC * wl + pl * nz; FeC = FrC * h0l;
      R id = (R)1.0 / (S1 - Sstar);
      R U1S = dltot * (S1 - unl) * id;
      R U2S = ((S1 - unl) * dltot * ul + (pstar - pl) * nx) * id;
      R U3S = ((S1 - unl) * dltot * vl + (pstar - pl) * ny) * id;
      R U4S = ((S1 - unl) * dltot * wl + (pstar - pl) * nz) * id;
      R U5S = ((S1 - unl) * dltot * e0l - pl * unl + pstar * Sstar) * id;
      FrC = FrC + S1 * (U1S - dltot); FuC = FuC + S1 * (U2S - dltot * ul); FvC = FvC + S1 * (U3S - dltot * vl);
      FwC = FwC + S1 * (U4S - dltot * wl); FeC = FeC + S1 * (U5S - dltot * e0l);
      if (rs == 10) {
        R ch_SK = S1;
        R ch_lm = ch_pref * (ch_fstar - (R)1.0) * ch_dU;
        R ch_sh = ch_pref * (ch_SK / (ch_SK - Sstar)) * ch_g;
        FuC = FuC + ch_lm * nx + ch_sh * ch_dutx;
        FvC = FvC + ch_lm * ny + ch_sh * ch_duty;
        FwC = FwC + ch_lm * nz + ch_sh * ch_dutz;
        FeC = FeC + ch_lm * Sstar;
      }
    } else if (S4 > (R)0.0) {
      FrC = drtot * unr; FuC = FrC * ur + pr * nx; FvC = FrC * vr + pr * ny; FwC = FrC * wr + pr * nz; FeC = FrC * h0r;
      R id = (R)1.0 / (S4 - Sstar);
      R U1S = drtot * (S4 - unr) * id;
      R U2S = ((S4 - unr) * drtot * ur + (pstar - pr) * nx) * id;
      R U3S = ((S4 - unr) * drtot * vr + (pstar - pr) * ny) * id;
      R U4S = ((S4 - unr) * drtot * wr + (pstar - pr) * nz) * id;
      R U5S = ((S4 - unr) * drtot * e0r - pr * unr + pstar * Sstar) * id;
      FrC = FrC + S4 * (U1S - drtot); FuC = FuC + S4 * (U2S - drtot * ur); FvC = FvC + S4 * (U3S - drtot * vr);
      FwC = FwC + S4 * (U4S - drtot * wr); FeC = FeC + S4 * (U5S - drtot * e0r);
      if (rs == 10) {
        R ch_SK = S4;
        R ch_lm = ch_pref * (ch_fstar - (R)1.0) * ch_dU;
        R ch_sh = ch_pref * (ch_SK / (ch_SK - Sstar)) * ch_g;
        FuC = FuC + ch_lm * nx + ch_sh * ch_dutx;
        FvC = FvC + ch_lm * ny + ch_sh * ch_duty;
        FwC = FwC + ch_lm * nz + ch_sh * ch_dutz;
        FeC = FeC + ch_lm * Sstar;
      }
    } else {
      FrC = drtot * unr; FuC = FrC * ur + pr * nx; FvC = FrC * vr + pr * ny; FwC = FrC * wr + pr * nz; FeC = FrC * h0r;
    }
    if (rs == 10 || bet >= (R)1.0) {
      F_r = FrC; F_u = FuC; F_v = FvC; F_w = FwC; F_E = FeC;
    } else if (bet == (R)0.0) {
      F_r = FrE; F_u = FuE; F_v = FvE; F_w = FwE; F_E = FeE;
    } else {
      F_r = bet * FrC + ((R)1.0 - bet) * FrE; F_u = bet * FuC + ((R)1.0 - bet) * FuE; F_v = bet * FvC + ((R)1.0 - bet) * FvE;
      F_w = bet * FwC + ((R)1.0 - bet) * FwE; F_E = bet * FeC + ((R)1.0 - bet) * FeE;
    }
    return;
  }
  if (Fast<R>::on) {
    // The mixed form evaluates the same flux with fewer operations: the face normal is already a unit vector,
    // the two tangential waves together are the tangential part of the velocity jump, (du - dun n), and the
    // static enthalpies of the two states are the ones interpolated above.
    if (nx == (R)0 && ny == (R)0 && nz == (R)0) { F_r = F_u = F_v = F_w = F_E = (R)0; return; }
    const R unL = unl, unR = unr;
    const R FL1 = dltot * unL, FR1 = drtot * unR;
    const R unRoe = u_roe * nx + v_roe * ny + w_roe * nz;
    const R u2 = u_roe * u_roe + v_roe * v_roe + w_roe * w_roe;
    const R utmag = rsqrt_(mx((R)0, u2 - unRoe * unRoe));
    const R Ma = (a_roe > (R)0) ? (fabs(unRoe) + utmag) / a_roe : (R)1;
    const R phi = mx((R)p.mco, mn((R)1, Ma));
    const R drho = drtot - dltot, dp = pr - pl, dun = unR - unL;
    const R abs1 = fabs(unRoe - a_roe), abs2 = fabs(unRoe), abs5 = fabs(unRoe + a_roe);
    const R inva = (R)1 / a_roe, inva2 = inva * inva;
    const R al4 = drho - dp * inva2;
    const R al1 = (R)0.5 * (dp * inva2 - rho_roe * phi * dun * inva);
    const R al5 = (R)0.5 * (dp * inva2 + rho_roe * phi * dun * inva);
    const R k1 = abs1 * al1, k5 = abs5 * al5, k4 = abs2 * al4, kt = abs2 * rho_roe;
    const R dtx = (ur - ul) - dun * nx, dty = (vr - vl) - dun * ny, dtz = (wr - wl) - dun * nz;
    const R d1 = k1 + k4 + k5;
    const R d2 = k1 * (u_roe - a_roe * nx) + kt * dtx + k4 * u_roe + k5 * (u_roe + a_roe * nx);
    const R d3 = k1 * (v_roe - a_roe * ny) + kt * dty + k4 * v_roe + k5 * (v_roe + a_roe * ny);
    const R d4 = k1 * (w_roe - a_roe * nz) + kt * dtz + k4 * w_roe + k5 * (w_roe + a_roe * nz);
    const R d5 = k1 * (h0_roe - a_roe * unRoe) + kt * (u_roe * dtx + v_roe * dty + w_roe * dtz) +
                 k4 * ((R)0.5 * u2) + k5 * (h0_roe + a_roe * unRoe);
    F_r = (R)0.5 * (FL1 + FR1) - (R)0.5 * d1;
    F_u = (R)0.5 * (FL1 * ul + pl * nx + FR1 * ur + pr * nx) - (R)0.5 * d2;
    F_v = (R)0.5 * (FL1 * vl + pl * ny + FR1 * vr + pr * ny) - (R)0.5 * d3;
    F_w = (R)0.5 * (FL1 * wl + pl * nz + FR1 * wr + pr * nz) - (R)0.5 * d4;
    F_E = (R)0.5 * (FL1 * h0l + FR1 * h0r) - (R)0.5 * d5;
    return;
  }
  R nmag = rsqrt_(nx * nx + ny * ny + nz * nz);
  if (!(nmag > (R)0)) { F_r = F_u = F_v = F_w = F_E = (R)0; return; }
  R n1 = nx / nmag, n2 = ny / nmag, n3 = nz / nmag;
  R tx, ty, tz;
  if (fabs(n1) < (R)0.9) { tx = (R)1; ty = (R)0; tz = (R)0; } else { tx = (R)0; ty = (R)1; tz = (R)0; }
  R t1x = tx - (tx * n1 + ty * n2 + tz * n3) * n1;
  R t1y = ty - (tx * n1 + ty * n2 + tz * n3) * n2;
  R t1z = tz - (tx * n1 + ty * n2 + tz * n3) * n3;
  R tmag = rsqrt_(t1x * t1x + t1y * t1y + t1z * t1z);
  if (tmag <= (R)0) { t1x = -n2; t1y = n1; t1z = (R)0; tmag = rsqrt_(t1x * t1x + t1y * t1y + t1z * t1z); }
  t1x = t1x / tmag; t1y = t1y / tmag; t1z = t1z / tmag;
  R t2x = n2 * t1z - n3 * t1y;
  R t2y = n3 * t1x - n1 * t1z;
  R t2z = n1 * t1y - n2 * t1x;
  R unL = ul * n1 + vl * n2 + wl * n3, unR = ur * n1 + vr * n2 + wr * n3;
  R ut1L = ul * t1x + vl * t1y + wl * t1z, ut1R = ur * t1x + vr * t1y + wr * t1z;
  R ut2L = ul * t2x + vl * t2y + wl * t2z, ut2R = ur * t2x + vr * t2y + wr * t2z;
  R hL = h_static(p, dl, pl), hR = h_static(p, dr, pr);
  R H0L = hL + (R)0.5 * (ul * ul + vl * vl + wl * wl);
  R H0R = hR + (R)0.5 * (ur * ur + vr * vr + wr * wr);
  R FL1 = dltot * unL, FL2 = dltot * unL * ul + pl * n1, FL3 = dltot * unL * vl + pl * n2;
  R FL4 = dltot * unL * wl + pl * n3, FL5 = dltot * unL * H0L;
  R FR1 = drtot * unR, FR2 = drtot * unR * ur + pr * n1, FR3 = drtot * unR * vr + pr * n2;
  R FR4 = drtot * unR * wr + pr * n3, FR5 = drtot * unR * H0R;
  R unRoe = u_roe * n1 + v_roe * n2 + w_roe * n3;
  R u2 = u_roe * u_roe + v_roe * v_roe + w_roe * w_roe;
  R utmag = rsqrt_(mx((R)0, u2 - unRoe * unRoe));
  R Ma = (a_roe > (R)0) ? (fabs(unRoe) + utmag) / a_roe : (R)1;
  R phi = mx((R)p.mco, mn((R)1, Ma));
  R drho = drtot - dltot, dp = pr - pl, dun = unR - unL;
  R dut1 = ut1R - ut1L, dut2 = ut2R - ut2L;
  R dunmod = phi * dun;
  R abs1 = fabs(unRoe - a_roe), abs2 = fabs(unRoe), abs5 = fabs(unRoe + a_roe);
  R a2 = a_roe * a_roe, inva = (R)1 / a_roe, inva2 = (R)1 / a2;
  R al4 = drho - dp * inva2;
  R al2 = rho_roe * dut1, al3 = rho_roe * dut2;
  R al1 = (R)0.5 * (dp * inva2 - rho_roe * dunmod * inva);
  R al5 = (R)0.5 * (dp * inva2 + rho_roe * dunmod * inva);
  R d1 = abs1 * al1 * (R)1 + abs2 * al2 * (R)0 + abs2 * al3 * (R)0 + abs2 * al4 * (R)1 + abs5 * al5 * (R)1;
  R d2 = abs1 * al1 * (u_roe - a_roe * n1) + abs2 * al2 * t1x + abs2 * al3 * t2x + abs2 * al4 * u_roe +
         abs5 * al5 * (u_roe + a_roe * n1);
  R d3 = abs1 * al1 * (v_roe - a_roe * n2) + abs2 * al2 * t1y + abs2 * al3 * t2y + abs2 * al4 * v_roe +
         abs5 * al5 * (v_roe + a_roe * n2);
  R d4 = abs1 * al1 * (w_roe - a_roe * n3) + abs2 * al2 * t1z + abs2 * al3 * t2z + abs2 * al4 * w_roe +
         abs5 * al5 * (w_roe + a_roe * n3);
  R d5 = abs1 * al1 * (h0_roe - a_roe * unRoe) + abs2 * al2 * (u_roe * t1x + v_roe * t1y + w_roe * t1z) +
         abs2 * al3 * (u_roe * t2x + v_roe * t2y + w_roe * t2z) + abs2 * al4 * ((R)0.5 * u2) +
         abs5 * al5 * (h0_roe + a_roe * unRoe);
  F_r = (R)0.5 * (FL1 + FR1) - (R)0.5 * d1;
  F_u = (R)0.5 * (FL2 + FR2) - (R)0.5 * d2;
  F_v = (R)0.5 * (FL3 + FR3) - (R)0.5 * d3;
  F_w = (R)0.5 * (FL4 + FR4) - (R)0.5 * d4;
  F_E = (R)0.5 * (FL5 + FR5) - (R)0.5 * d5;
}

// The mixed form's LMRoe (Mco floor) from the states' thermo already evaluated by the caller (T, its table row and
// fraction, cp): the Roe averages of riemann_open_body.inc:679-730 with the single-species identities, then the
// dissipation of the fast path of riemann_open.
template <typename R>
MB_HD void lmroe_fast(const Params& p, R dl, R ul, R vl, R wl, R pl, R Tl, int Til, R dTl, R cpl, R dr, R ur, R vr,
                      R wr, R pr, R Tr, int Tir, R dTr, R cpr, R nx, R ny, R nz, R& F_r, R& F_u, R& F_v, R& F_w,
                      R& F_E) {
  const R* H = Tab<R>::h(p);
  const R Rg = (R)p.ri;
  const R srL = rsqrt_(dl), srR = rsqrt_(dr);
  const R inv_sr = (R)1 / (srL + srR);
  const R rho_roe = srL * srR;
  const R u_roe = (srR * ur + srL * ul) * inv_sr;
  const R v_roe = (srR * vr + srL * vl) * inv_sr;
  const R w_roe = (srR * wr + srL * wl) * inv_sr;
  const R T_roe = (srR * Tr + srL * Tl) * inv_sr;
  const R hl = H[Til] + (H[Til + 1] - H[Til]) * dTl;
  const R hr = H[Tir] + (H[Tir + 1] - H[Tir]) * dTr;
  const R el = hl - Rg * Tl, er = hr - Rg * Tr;
  const R cv_roe = (R)0.5 * (cpl + cpr) - Rg;
  const R sum_ei = (srR * er + srL * el) * inv_sr;
  const R h0l = hl + (R)0.5 * (ul * ul + vl * vl + wl * wl);
  const R h0r = hr + (R)0.5 * (ur * ur + vr * vr + wr * wr);
  const R h0_roe = (srR * h0r + srL * h0l) * inv_sr;
  const R gam_roe = (R)1 + Rg / cv_roe;
  const R u2 = u_roe * u_roe + v_roe * v_roe + w_roe * w_roe;
  const R a_roe = rsqrt_((gam_roe - (R)1) * (h0_roe - (R)0.5 * u2 + cv_roe * T_roe - sum_ei));
  if (nx == (R)0 && ny == (R)0 && nz == (R)0) { F_r = F_u = F_v = F_w = F_E = (R)0; return; }
  const R unL = ul * nx + vl * ny + wl * nz, unR = ur * nx + vr * ny + wr * nz;
  const R FL1 = dl * unL, FR1 = dr * unR;
  const R unRoe = u_roe * nx + v_roe * ny + w_roe * nz;
  const R utmag = rsqrt_(mx((R)0, u2 - unRoe * unRoe));
  const R Ma = (a_roe > (R)0) ? (fabs(unRoe) + utmag) / a_roe : (R)1;
  const R phi = mx((R)p.mco, mn((R)1, Ma));
  const R drho = dr - dl, dp = pr - pl, dun = unR - unL;
  const R abs1 = fabs(unRoe - a_roe), abs2 = fabs(unRoe), abs5 = fabs(unRoe + a_roe);
  const R inva = (R)1 / a_roe, inva2 = inva * inva;
  const R al4 = drho - dp * inva2;
  const R al1 = (R)0.5 * (dp * inva2 - rho_roe * phi * dun * inva);
  const R al5 = (R)0.5 * (dp * inva2 + rho_roe * phi * dun * inva);
  const R k1 = abs1 * al1, k5 = abs5 * al5, k4 = abs2 * al4, kt = abs2 * rho_roe;
  const R dtx = (ur - ul) - dun * nx, dty = (vr - vl) - dun * ny, dtz = (wr - wl) - dun * nz;
  const R d1 = k1 + k4 + k5;
  const R d2 = k1 * (u_roe - a_roe * nx) + kt * dtx + k4 * u_roe + k5 * (u_roe + a_roe * nx);
  const R d3 = k1 * (v_roe - a_roe * ny) + kt * dty + k4 * v_roe + k5 * (v_roe + a_roe * ny);
  const R d4 = k1 * (w_roe - a_roe * nz) + kt * dtz + k4 * w_roe + k5 * (w_roe + a_roe * nz);
  const R d5 = k1 * (h0_roe - a_roe * unRoe) + kt * (u_roe * dtx + v_roe * dty + w_roe * dtz) +
               k4 * ((R)0.5 * u2) + k5 * (h0_roe + a_roe * unRoe);
  F_r = (R)0.5 * (FL1 + FR1) - (R)0.5 * d1;
  F_u = (R)0.5 * (FL1 * ul + pl * nx + FR1 * ur + pr * nx) - (R)0.5 * d2;
  F_v = (R)0.5 * (FL1 * vl + pl * ny + FR1 * vr + pr * ny) - (R)0.5 * d3;
  F_w = (R)0.5 * (FL1 * wl + pl * nz + FR1 * wr + pr * nz) - (R)0.5 * d4;
  F_E = (R)0.5 * (FL1 * h0l + FR1 * h0r) - (R)0.5 * d5;
}

// Roe averages shared by the two HLLC forms: the inline one of conv_physics.inc (clamped T row, Rl/Rr
// taken from the caller) and riemann_HLLC / roe_averages of Lib_Riemann_HLL.f90 (boundary records).
// SLAU flux from the two states and their total enthalpies (riemann_SLAU_base + riemann_SLAU: conv_physics.inc:125-159
// = Lib_Riemann.f90:167-196, the same statements)
template <typename R>
MB_HD void slau_flux(R ul, R vl, R wl, R pl, R al, R dltot, R h0l, R ur, R vr, R wr, R pr, R ar, R drtot, R h0r, R unl,
                     R unr, R nx, R ny, R nz, R& F_r, R& F_u, R& F_v, R& F_w, R& F_E) {
  R af_ = (R)0.5 * (al + ar);
  R ml_ = unl / af_, mr_ = unr / af_;
  R mt_ = mn((R)1, rsqrt_((R)0.5 * ((ul * ul + vl * vl + wl * wl) + (ur * ur + vr * vr + wr * wr))) / af_);
  R chi_ = ((R)1 - mt_) * ((R)1 - mt_);
  R vnm_ = (dltot * fabs(unl) + drtot * fabs(unr)) / (dltot + drtot);
  R frho_ = -mx(mn(ml_, (R)0), (R)(-1)) * mn(mx(mr_, (R)0), (R)1);
  R vnl_ = ((R)1 - frho_) * vnm_ + frho_ * fabs(unl);
  R vnr_ = ((R)1 - frho_) * vnm_ + frho_ * fabs(unr);
  F_r = (R)0.5 * (dltot * (unl + vnl_) + drtot * (unr - vnr_) - (chi_ / af_) * (pr - pl));
  R bl_, br_;
  if (fabs(ml_) < (R)1) bl_ = (R)0.25 * ((R)2 - ml_) * ((ml_ + (R)1) * (ml_ + (R)1));
  else if (ml_ >= (R)0) bl_ = (R)1;
  else bl_ = (R)0;
  if (fabs(mr_) < (R)1) br_ = (R)0.25 * ((R)2 + mr_) * ((mr_ - (R)1) * (mr_ - (R)1));
  else if (mr_ >= (R)0) br_ = (R)0;
  else br_ = (R)1;
  R ph_ = (R)0.5 * (pl + pr) + (R)0.5 * (bl_ - br_) * (pl - pr) + ((R)1 - chi_) * (bl_ + br_ - (R)1) * (R)0.5 * (pl + pr);
  if (F_r >= (R)0) {
    F_u = F_r * ul + nx * ph_; F_v = F_r * vl + ny * ph_; F_w = F_r * wl + nz * ph_; F_E = F_r * h0l;
  } else {
    F_u = F_r * ur + nx * ph_; F_v = F_r * vr + ny * ph_; F_w = F_r * wr + nz * ph_; F_E = F_r * h0r;
  }
}

// HLLE two-wave flux with the Batten signal speeds (Lib_Riemann_HLL.f90:176-196 = conv_physics.inc:116-124)
template <typename R>
MB_HD void hlle_flux(R ul, R vl, R wl, R pl, R dltot, R h0l, R ur, R vr, R wr, R pr, R drtot, R h0r, R unl, R unr, R S1,
                     R S4, R nx, R ny, R nz, R& F_r, R& F_u, R& F_v, R& F_w, R& F_E) {
  R inv_denom = (R)1 / (S4 - S1);
  R FrL = dltot * unl, FrR = drtot * unr;
  F_r = (S4 * FrL - S1 * FrR + S1 * S4 * (drtot - dltot)) * inv_denom;
  F_u = (S4 * (FrL * ul + pl * nx) - S1 * (FrR * ur + pr * nx) + S1 * S4 * (drtot * ur - dltot * ul)) * inv_denom;
  F_v = (S4 * (FrL * vl + pl * ny) - S1 * (FrR * vr + pr * ny) + S1 * S4 * (drtot * vr - dltot * vl)) * inv_denom;
  F_w = (S4 * (FrL * wl + pl * nz) - S1 * (FrR * wr + pr * nz) + S1 * S4 * (drtot * wr - dltot * wl)) * inv_denom;
  F_E = (S4 * (FrL * h0l) - S1 * (FrR * h0r) + S1 * S4 * (drtot * (h0r - pr / drtot) - dltot * (h0l - pl / dltot))) *
        inv_denom;
}

// SLAU at the boundary records (Lib_Riemann.f90:140-197): T = p / (rho R) and H0 = h(T) + V^2/2 of each state from
// the tables (no T clamp), then the SLAU flux
template <typename R>
MB_HD void slau_rec(const Params& p, R dl, R ul, R vl, R wl, R pl, R al, R dltot, R dr, R ur, R vr, R wr, R pr, R ar,
                    R drtot, R nx, R ny, R nz, R& F_r, R& F_u, R& F_v, R& F_w, R& F_E) {
  const R* H = Tab<R>::h(p);
  const R ri = (R)(RUNIV / p.wm);
  R unl = ul * nx + vl * ny + wl * nz;
  R unr = ur * nx + vr * ny + wr * nz;
  R Rl = (R)0 + ri * dl / dltot;
  R Rr = (R)0 + ri * dr / drtot;
  R Tl = pl / (dltot * Rl), Tr = pr / (drtot * Rr);
  int Til = (int)Tl, Tir = (int)Tr;
  R dTl = Tl - (R)Til, dTr = Tr - (R)Tir;
  R h0l = (R)0 + (H[Til] + (H[Til + 1] - H[Til]) * dTl) * dl / dltot;
  R h0r = (R)0 + (H[Tir] + (H[Tir + 1] - H[Tir]) * dTr) * dr / drtot;
  h0l = h0l + (R)0.5 * (ul * ul + vl * vl + wl * wl);
  h0r = h0r + (R)0.5 * (ur * ur + vr * vr + wr * wr);
  slau_flux(ul, vl, wl, pl, al, dltot, h0l, ur, vr, wr, pr, ar, drtot, h0r, unl, unr, nx, ny, nz, F_r, F_u, F_v, F_w,
            F_E);
}

template <typename R>
MB_HD void hllc(const Params& p, R dl, R ul, R vl, R wl, R pl, R al, R dltot, R Rl, R dr, R ur,
                                     R vr, R wr, R pr, R ar, R drtot, R Rr, R nx, R ny, R nz, R& F_r, R& F_u,
                                     R& F_v, R& F_w, R& F_E, const R* thL = nullptr, const R* thR = nullptr,
                                     int tiL = 0, int tiR = 0, int tail = 1) {
  // thL / thR (the mixed form, from the caller's reconstruction): T, its table fraction and cp of each state
  const R* H = Tab<R>::h(p);
  const R* CP = Tab<R>::cp(p);
  const bool given = Fast<R>::on && thL != nullptr;
  R unl = ul * nx + vl * ny + wl * nz;
  R unr = ur * nx + vr * ny + wr * nz;
  R inv_dltot = given ? (R)0 : (R)1 / dltot, inv_drtot = given ? (R)0 : (R)1 / drtot;
  R Tl = given ? thL[0] : pl * inv_dltot / Rl, Tr = given ? thR[0] : pr * inv_drtot / Rr;
  int Til = given ? tiL : tidx(p, Tl);
  int Tir = given ? tiR : tidx(p, Tr);
  R dTl = given ? thL[1] : Tl - (R)Til, dTr = given ? thR[1] : Tr - (R)Tir;
  R srL = rsqrt_(dltot), srR = rsqrt_(drtot), inv_sr = (R)1 / (srL + srR);
  R u_roe = (srR * ur + srL * ul) * inv_sr, v_roe = (srR * vr + srL * vl) * inv_sr,
    w_roe = (srR * wr + srL * wl) * inv_sr;
  R R_roe = (srR * Rr + srL * Rl) * inv_sr, T_roe = (srR * Tr + srL * Tl) * inv_sr;
  R h0l = (R)0, h0r = (R)0, cv_roe = (R)0, sum_ei = (R)0;
  {
    R invW = (R)(RUNIV / p.wm);
    R hl = H[Til] + (H[Til + 1] - H[Til]) * dTl;
    R hr = H[Tir] + (H[Tir + 1] - H[Tir]) * dTr;
    R el = hl - invW * Tl, er = hr - invW * Tr;
    if (Fast<R>::on) {  // one species: Y = 1, d_roe = 1
      h0l = hl;
      h0r = hr;
      cv_roe = given ? (R)0.5 * (thL[2] + thR[2]) - invW
                     : (R)0.5 * (CP[Til] + (CP[Til + 1] - CP[Til]) * dTl + CP[Tir] + (CP[Tir + 1] - CP[Tir]) * dTr) - invW;
      sum_ei = (srR * er + srL * el) * inv_sr;
    } else {
    h0l = h0l + hl * dl * inv_dltot;
    h0r = h0r + hr * dr * inv_drtot;
    R d_roe = (srR * dr * inv_drtot + srL * dl * inv_dltot) * inv_sr;
    cv_roe = cv_roe + d_roe * ((R)0.5 * (CP[Til] + (CP[Til + 1] - CP[Til]) * dTl + CP[Tir] +
                                         (CP[Tir + 1] - CP[Tir]) * dTr) - invW);
    sum_ei = sum_ei + d_roe * (srR * er + srL * el) * inv_sr;
    }
  }
  h0l = h0l + (R)0.5 * (ul * ul + vl * vl + wl * wl);
  h0r = h0r + (R)0.5 * (ur * ur + vr * vr + wr * wr);
  R h0_roe = (srR * h0r + srL * h0l) * inv_sr;
  R gam_roe = (R)1 + R_roe / cv_roe;
  R vel2 = u_roe * u_roe + v_roe * v_roe + w_roe * w_roe;
  R a_roe = rsqrt_((gam_roe - (R)1) * (h0_roe - (R)0.5 * vel2 + cv_roe * T_roe - sum_ei));
  R un_roe = u_roe * nx + v_roe * ny + w_roe * nz;
  R e0l = h0l - pl / dltot, e0r = h0r - pr / drtot;
  R S1 = mn(mn((R)0, unl - al), un_roe - a_roe);
  R S4 = mx(mx((R)0, unr + ar), un_roe + a_roe);
  if (tail == 2) {  // HLLE
    hlle_flux(ul, vl, wl, pl, dltot, h0l, ur, vr, wr, pr, drtot, h0r, unl, unr, S1, S4, nx, ny, nz, F_r, F_u, F_v, F_w,
              F_E);
    return;
  }
  if (tail == 3) {  // SLAU (the interior face: the total enthalpies of this prologue)
    slau_flux(ul, vl, wl, pl, al, dltot, h0l, ur, vr, wr, pr, ar, drtot, h0r, unl, unr, nx, ny, nz, F_r, F_u, F_v, F_w,
              F_E);
    return;
  }
  R inv_denom = (R)1 / (dltot * (S1 - unl) - drtot * (S4 - unr));
  R Sstar = (pr - pl + dltot * unl * (S1 - unl) - drtot * unr * (S4 - unr)) * inv_denom;
  R pstar = dltot * (unl - S1) * (unl - Sstar) + pl;
  if (S1 >= (R)0) {
    F_r = dltot * unl; F_u = F_r * ul + pl * nx; F_v = F_r * vl + pl * ny; F_w = F_r * wl + pl * nz; F_E = F_r * h0l;
  } else if (Sstar >= (R)0) {
    F_r = dltot * unl; F_u = F_r * ul + pl * nx; F_v = F_r * vl + pl * ny; F_w = F_r * wl + pl * nz; F_E = F_r * h0l;
    inv_denom = (R)1 / (S1 - Sstar);
    R U1S = dltot * (S1 - unl) * inv_denom;
    R U2S = ((S1 - unl) * dltot * ul + (pstar - pl) * nx) * inv_denom;
    R U3S = ((S1 - unl) * dltot * vl + (pstar - pl) * ny) * inv_denom;
    R U4S = ((S1 - unl) * dltot * wl + (pstar - pl) * nz) * inv_denom;
    R U5S = ((S1 - unl) * dltot * e0l - pl * unl + pstar * Sstar) * inv_denom;
    F_r = F_r + S1 * (U1S - dltot); F_u = F_u + S1 * (U2S - dltot * ul); F_v = F_v + S1 * (U3S - dltot * vl);
    F_w = F_w + S1 * (U4S - dltot * wl); F_E = F_E + S1 * (U5S - dltot * e0l);
  } else if (S4 > (R)0) {
    F_r = drtot * unr; F_u = F_r * ur + pr * nx; F_v = F_r * vr + pr * ny; F_w = F_r * wr + pr * nz; F_E = F_r * h0r;
    inv_denom = (R)1 / (S4 - Sstar);
    R U1S = drtot * (S4 - unr) * inv_denom;
    R U2S = ((S4 - unr) * drtot * ur + (pstar - pr) * nx) * inv_denom;
    R U3S = ((S4 - unr) * drtot * vr + (pstar - pr) * ny) * inv_denom;
    R U4S = ((S4 - unr) * drtot * wr + (pstar - pr) * nz) * inv_denom;
    R U5S = ((S4 - unr) * drtot * e0r - pr * unr + pstar * Sstar) * inv_denom;
    F_r = F_r + S4 * (U1S - drtot); F_u = F_u + S4 * (U2S - drtot * ur); F_v = F_v + S4 * (U3S - drtot * vr);
    F_w = F_w + S4 * (U4S - drtot * wr); F_E = F_E + S4 * (U5S - drtot * e0r);
  } else {
    F_r = drtot * unr; F_u = F_r * ur + pr * nx; F_v = F_r * vr + pr * ny; F_w = F_r * wr + pr * nz; F_E = F_r * h0r;
  }
}

// The shock sensor of a cell from its pressure and its six face neighbours' (SD_beta, Lib_Shock_Detector.f90:51-81):
// 1 Tramel (1 smooth, 0 at a shock), 2 Chen (the smallest neighbour pressure ratio), 1 otherwise
template <typename R>
MB_HD R sd_beta(int id, R pc, R p1, R p2, R p3, R p4, R p5, R p6) {
  if (id == 1) {
    const R DELTA = (R)20;
    R kp1 = fabs((p2 - (R)2 * pc + p1) / (p2 + (R)2 * pc + p1));
    R kp2 = fabs((p4 - (R)2 * pc + p3) / (p4 + (R)2 * pc + p3));
    R kp3 = fabs((p6 - (R)2 * pc + p5) / (p6 + (R)2 * pc + p5));
    R sw = mx(mx(kp1, kp2), kp3);
    if (sw < (R)1 / DELTA) {
      R phi = mx(sw / DELTA, (R)0);
      return (R)1 - tanh((R)10 * phi * phi * phi);
    }
    return (R)0;
  }
  if (id == 2) {
    R beta = (R)1;
    beta = mn(beta, mn(pc, p1) / mx(pc, p1));
    beta = mn(beta, mn(pc, p2) / mx(pc, p2));
    beta = mn(beta, mn(pc, p3) / mx(pc, p3));
    beta = mn(beta, mn(pc, p4) / mx(pc, p4));
    beta = mn(beta, mn(pc, p5) / mx(pc, p5));
    beta = mn(beta, mn(pc, p6) / mx(pc, p6));
    return beta;
  }
  return (R)1;
}

// ---- interior convective face from the 4-cell stencil (conv_physics.inc) ----
// RS / LIM: the Riemann solver and limiter ids fixed at compile time (0: read p.rs / p.lim at run time)
template <typename R, int RS = 0, int LIM = 0>
MB_HD void conv_face(const Params& p, const R* pm1, const R* p0, const R* pp1, const R* pp2,
                                          const R* dlc, R nx, R ny, R nz, R area, R* res0, R bet = (R)1,
                                          R urL = (R)0, R urR = (R)0) {
  const int rs = RS ? RS : p.rs;
  const int lim = LIM ? LIM : p.lim;
  R l0 = (R)0.5 * (dlc[0] + dlc[1]), l1 = (R)0.5 * (dlc[1] + dlc[2]), l2 = (R)0.5 * (dlc[2] + dlc[3]);
  R lm = (R)0.5 * dlc[1], lp = (R)0.5 * dlc[2];
  const R beta_order = (RS == 0 && p.sd) ? bet : (R)1;  // SD_space_order: the slopes scaled by the face sensor
  R idl0 = (R)1 / l0, idl1 = (R)1 / l1, idl2 = (R)1 / l2;
  R P1[MB_NP], P4[MB_NP];
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) {
    R slope0 = (p0[s] - pm1[s]) * idl0;
    R slope1 = (pp1[s] - p0[s]) * idl1;
    R slope2 = (pp2[s] - pp1[s]) * idl2;
    R slopel = rlimiter(lim, slope1, slope0);
    R sloper = rlimiter(lim, slope2, slope1);
    P1[s] = p0[s] + beta_order * slopel * lm;
    P4[s] = pp1[s] - beta_order * sloper * lp;
  }
  P1[0] = mx(P1[0], (R)1e-20);
  P4[0] = mx(P4[0], (R)1e-20);
  R rotot1, Rtot1, rotot4, Rtot4;
  rotot_rtot(p, P1[0], rotot1, Rtot1);
  rotot_rtot(p, P4[0], rotot4, Rtot4);
  const R* CP = Tab<R>::cp(p);
  R T1d = P1[MB_IPR] / (Rtot1 * rotot1);
  int Ti1 = tidx(p, T1d);
  R Tdiffd = T1d - (R)Ti1;
  const R Td1 = Tdiffd;
  R cpd = Fast<R>::on ? CP[Ti1] + (CP[Ti1 + 1] - CP[Ti1]) * Tdiffd
                       : (R)0 + P1[0] / rotot1 * (CP[Ti1] + (CP[Ti1 + 1] - CP[Ti1]) * Tdiffd);
  R gamd = cpd / (cpd - Rtot1);
  R a1 = rsqrt_(gamd * Rtot1 * T1d);
  R T4d = P4[MB_IPR] / (Rtot4 * rotot4);
  int Ti4 = tidx(p, T4d);
  Tdiffd = T4d - (R)Ti4;
  cpd = Fast<R>::on ? CP[Ti4] + (CP[Ti4 + 1] - CP[Ti4]) * Tdiffd
                   : (R)0 + P4[0] / rotot4 * (CP[Ti4] + (CP[Ti4 + 1] - CP[Ti4]) * Tdiffd);
  gamd = cpd / (cpd - Rtot4);
  R a4 = rsqrt_(gamd * Rtot4 * T4d);
  R F_r, F_u, F_v, F_w, F_E;
  if (Fast<R>::on && rs == 12) {  // the mixed form's LMRoe takes the thermo of the two states evaluated above
    const R cp1 = CP[Ti1] + (CP[Ti1 + 1] - CP[Ti1]) * Td1;
    lmroe_fast(p, P1[0], P1[MB_IU], P1[MB_IV], P1[MB_IW], P1[MB_IPR], T1d, Ti1, Td1, cp1, P4[0], P4[MB_IU],
               P4[MB_IV], P4[MB_IW], P4[MB_IPR], T4d, Ti4, Tdiffd, cpd, nx, ny, nz, F_r, F_u, F_v, F_w, F_E);
  } else if (rs == 1 || rs == 2 || rs == 3) {  // HLLC, HLLE, SLAU after the Roe-average prologue of conv_physics.inc
    const R th1[3] = {T1d, Td1, CP[Ti1] + (CP[Ti1 + 1] - CP[Ti1]) * Td1}, th4[3] = {T4d, Tdiffd, cpd};
    hllc(p, P1[0], P1[MB_IU], P1[MB_IV], P1[MB_IW], P1[MB_IPR], a1, rotot1, Rtot1, P4[0], P4[MB_IU], P4[MB_IV],
         P4[MB_IW], P4[MB_IPR], a4, rotot4, Rtot4, nx, ny, nz, F_r, F_u, F_v, F_w, F_E,
         Fast<R>::on ? th1 : nullptr, Fast<R>::on ? th4 : nullptr, Ti1, Ti4, rs);
  }
  else
    riemann_open(p, rs, bet, P1[0], P1[MB_IU], P1[MB_IV], P1[MB_IW], P1[MB_IPR], a1, rotot1, P4[0], P4[MB_IU],
                 P4[MB_IV], P4[MB_IW], P4[MB_IPR], a4, rotot4, nx, ny, nz, F_r, F_u, F_v, F_w, F_E, urL, urR);
  if (Fast<R>::on) {
    res0[0] = F_r * area;  // one species: the upwinded mass fraction is 1
  } else {
    R su = copysign((R)0.5, F_r), sp = (R)0.5 + su, sm = su - (R)0.5;
    R irotot1 = (R)1 / rotot1, irotot4 = (R)1 / rotot4;
    res0[0] = F_r * area * (sp * (P1[0] * irotot1) - sm * (P4[0] * irotot4));
  }
  res0[MB_IU] = F_u * area; res0[MB_IV] = F_v * area; res0[MB_IW] = F_w * area; res0[MB_IPR] = F_E * area;
}

// the Riemann dispatch of the record routines (Lib_Riemann.f90:114-136, `Riemann`): HLLC Batten for rs 1, HLLE for
// 2 (both after roe_averages), SLAU for 3, the MOSE_open solvers otherwise
template <typename R, int RS = 0>
MB_HD void riemann_rec(const Params& p, R dl, R ul, R vl, R wl, R pl, R al, R dltot, R Rl, R dr, R ur, R vr, R wr,
                       R pr, R ar, R drtot, R Rr, R nx, R ny, R nz, R& F_r, R& F_u, R& F_v, R& F_w, R& F_E,
                       R bet = (R)1, R urL = (R)0, R urR = (R)0) {
  const int rs = RS ? RS : p.rs;
  if (rs == 1 || rs == 2)
    hllc(p, dl, ul, vl, wl, pl, al, dltot, Rl, dr, ur, vr, wr, pr, ar, drtot, Rr, nx, ny, nz, F_r, F_u, F_v, F_w, F_E,
         (const R*)nullptr, (const R*)nullptr, 0, 0, rs);
  else if (rs == 3)
    slau_rec(p, dl, ul, vl, wl, pl, al, dltot, dr, ur, vr, wr, pr, ar, drtot, nx, ny, nz, F_r, F_u, F_v, F_w, F_E);
  else
    riemann_open(p, rs, bet, dl, ul, vl, wl, pl, al, dltot, dr, ur, vr, wr, pr, ar, drtot, nx, ny, nz, F_r, F_u, F_v, F_w,
                 F_E, urL, urR);
}

// face thermo (Diffusive_Face_Thermo_Fill, Mod_Diffusive.f90:311-325 = Diffusive_Face_State :748-776)
template <typename R>
MB_HD void face_thermo(const Params& p, R rhoi, R pr, R& rho, R& T, int& ti, R& td, R& cp,
                                            R& mil, R& kl) {
  R Rgas;
  rotot_rtot(p, rhoi, rho, Rgas);
  T = pr / (rho * Rgas);
  ti = tidx(p, T);
  td = T - (R)ti;
  cp = f_cp(p, rhoi, ti, td, rho);
  wilke(p, rhoi, rho, ti, td, mil, kl);
  if (p.prandtl > 0.0) kl = mil * cp / (R)p.prandtl;
}

// the laminar viscous flux of a face from its gradients (diff_physics.inc:88-161 with mie = 0);
// Stress_Vector_Std (physics/turbulence/Mod_Fluid.f90:20-44) is the same arithmetic
template <typename R>
MB_HD void visc_flux(const Params& p, const R G[MB_NP][3], const R* Pf, R nx, R ny, R nz,
                                          R area, R drho, R dT, R dcp, R dmil, R dkl, R* F) {
  int Ti = tidx(p, dT);
  R Tdf = dT - (R)Ti;
  const R mie = (R)0, sct = (R)0.9, prt = (R)0.85;
  R Dm = (dmil / (R)p.schmidt + mie / sct) / drho;
  R kappaf = dkl + mie * dcp / prt;
  R dmi = dmil + mie;
  const R ntt = (R)(-2.0 / 3.0);
  R dlam = ntt * dmi;
  R Diver = G[MB_IU][0] + G[MB_IV][1] + G[MB_IW][2];
  R lamDiv = dlam * Diver;
  const R rhokd = (R)0;
  R Txx = lamDiv + (R)2 * dmi * G[MB_IU][0] + rhokd;
  R Tyy = lamDiv + (R)2 * dmi * G[MB_IV][1] + rhokd;
  R Tzz = lamDiv + (R)2 * dmi * G[MB_IW][2] + rhokd;
  R Txy = dmi * (G[MB_IU][1] + G[MB_IV][0]), Txz = dmi * (G[MB_IU][2] + G[MB_IW][0]),
    Tyz = dmi * (G[MB_IV][2] + G[MB_IW][1]);
  R S1 = Txx * nx + Txy * ny + Txz * nz;
  R S2 = Txy * nx + Tyy * ny + Tyz * nz;
  R S3 = Txz * nx + Tyz * ny + Tzz * nz;
  R DiffH = (R)0;
  if (Fast<R>::on) {
    F[0] = (R)0;  // one species: no species diffusion, no enthalpy diffusion
  } else {
  R DmGY = Dm * (G[0][0] * nx + G[0][1] * ny + G[0][2] * nz);
  R F0 = drho * area * DmGY;
  const R* H = Tab<R>::h(p);
  R hh1 = H[Ti], hh2 = H[Ti + 1];
  R hh = hh1 + Tdf * (hh2 - hh1);
  DiffH = DiffH + DmGY * hh;
  R sflx = (R)0 + F0;
  F[0] = F0 - sflx * Pf[0] / drho;
  }
  F[MB_IU] = area * S1; F[MB_IV] = area * S2; F[MB_IW] = area * S3;
  if (Fast<R>::on)
    F[MB_IPR] = area * ((S1 * Pf[MB_IU] + S2 * Pf[MB_IV] + S3 * Pf[MB_IW]) +
                        kappaf * (G[MB_IPR][0] * nx + G[MB_IPR][1] * ny + G[MB_IPR][2] * nz));
  else
    F[MB_IPR] = area * ((S1 * Pf[MB_IU] + S2 * Pf[MB_IV] + S3 * Pf[MB_IW]) +
                        kappaf * (G[MB_IPR][0] * nx + G[MB_IPR][1] * ny + G[MB_IPR][2] * nz) + DiffH * drho);
}

// the cell density / temperature of the thermo cache (Mod_Thermo_Cache.f90:327-330,378-380)
template <typename R>
MB_HD void cell_rho_T(const Params& p, R rhoi, R pr, R& rho, R& T) {
  R Rg;
  rotot_rtot(p, rhoi, rho, Rg);
  T = pr / (rho * Rg);
}

MB_HD int face_sign(int F) { return 1 - 2 * (F % 2); }  // modfm2 / FluxSign

}  // namespace mb
