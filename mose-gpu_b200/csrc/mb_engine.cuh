// mb_engine.cuh -- kernels of the B200 engine.
//
//   k_sweep      the fused stage: every interior face flux of a tile computed ONCE (one thread per
//                face), exchanged through shared memory, summed per cell in the reference's pass-2
//                order (src/lib/gpu/pass2_body.inc), the boundary records of the cell added in face
//                order 1..6 (numerics/fluxes/bc/Mod_BC.f90:449-485), then either the residual is
//                written (parity hook, mode RESIDUAL) or the conservative RK update is applied
//                (gpu/newstate_cons_body.inc) with, on the last stage, the local dt of the new state
//                reduced into the device clock (gpu/dt_blk.inc; warp shuffles, one atomic per CTA).
//   k_ghost_*    the ghost fill (numerics/fluxes/bc/Lib_Extrapolation.f90:1370-1528)
//   k_dt         Compute_dt on its own (numerics/time/Mod_dt.f90:15-106)
//   k_update     RK_Newstate on its own (explicit/Lib_Newstate.f90:257-307)
//
// Tiling: a CTA owns a tile of 32 (i) x TY (j) cells of one block and marches over a chunk of k
// planes. Per plane it computes the (32+1) x TY i-faces, 32 x (TY+1) j-faces and the 32 x TY
// k-faces above the plane (the k-face below is the previous plane's), so only the tile's left i-faces
// and bottom j-faces are computed twice across CTAs. Warps run the face tasks through one call
// site, which keeps a single copy of the flux code in the kernel.
#pragma once
#include "mb_physics.cuh"

namespace mb {

struct DTile {
  int blk, i0, j0, k0, k1;  // cells i0..i0+31, j0..j0+TY-1, planes k0..k1-1 (1-based)
};

enum { MODE_RESIDUAL = 0, MODE_UPDATE = 1 };

template <typename R> MB_HD R cvt(double x) { return (R)x; }

// ---------------------------------------------------------------------------------------------
// The state tile of a CTA in shared memory: 4 k-planes (a rolling window), each (32+4) x (TY+4) cells
// (two halo cells on each side in i and j), converted to the flux arithmetic type once per cell, with the
// thermo-cache temperature T = p / (rho Rg) (Mod_Thermo_Cache.f90:327-330). The FP64 forms keep 6 values per cell:
// rho_s, u, v, w, p, T. The mixed form keeps 5: rho_s, u, v, w, T, and takes p = rho Rg T where it reads it (one
// value less per cell leaves room in shared memory for the TMA staging buffer at 3 CTAs per SM).
// Layout [slot][value][jj][ii], ii fastest.
constexpr int TXH = 36;
// The staging of a sweep's state tile, a template parameter of the sweep (STG) chosen per context (mb_autotune,
// mb_set_staging): STG_PLAIN, per-thread coalesced loads into a 6-value tile (rho_s, u, v, w, p, T) with the k-face
// fluxes of two planes in shared memory; STG_TMA (the mixed form), TMA boxes of the state arena landing on an mbarrier
// in a staging buffer, converted into a 5-value tile (rho_s, u, v, w, T; p = rho Rg T where it is read) with the
// k-face fluxes carried in registers, which together leave room for the staging buffer at 3 CTAs per SM.
enum { STG_PLAIN = 0, STG_TMA = 1 };
template <typename R, int STG> struct Stg {
  static constexpr bool tma = STG == STG_TMA && sizeof(R) == 4;
  static constexpr int nv = tma ? 5 : 6;   // values per staged cell
  static constexpr bool kreg = tma;        // k-face fluxes in registers
};

template <typename R, int TY, int NV_ = 6>
struct Tile {
  R* base;
  R rg;                                              // the gas constant of the single species (5-value tile)
  static constexpr int NVT = NV_;
  static constexpr int VS = (TY + 4) * TXH;          // stride between the values of one cell
  MB_HD int off(int slot, int jj, int ii) const { return slot * NVT * VS + jj * TXH + ii; }
  // value var (0..4: rho_s, u, v, w, p; 5: T) of the cell at offset o
  MB_HD R v(int o, int var) const {
    if (NVT == 6 || var < 4) return base[o + var * VS];
    if (var == 5) return base[o + 4 * VS];
    return base[o] * rg * base[o + 4 * VS];
  }
};

// the plane slot of plane kk (kk >= -1); the tile of a mirrored one-plane block (KM) holds its one plane only
template <bool KM = false>
MB_HD int slot_of(int kk) { return KM ? 0 : (kk + 8) & 3; }
// planes held by the state tile
template <bool KM>
MB_HD constexpr int tile_planes() { return KM ? 1 : 4; }

// One interior face of direction d between cell (i,j,k) and its +d neighbour, from the state tile: the
// convective flux (conv_physics.inc) into out[0..4] and, for Navier-Stokes, the viscous flux
// (diff_cuf_kernels.inc:11-87 + diff_physics.inc) into out[5..9]. (ii, jj) are the tile coordinates of the
// cell, sk the slot of plane k. The gradients are built per variable in registers and placed on the
// axes by d (ia = d; the two tangential axes in increasing order), as the reference's Grad(:, ia/ib/ic).
template <typename R, int TY, bool VISC, int RS = 0, int LIM = 0, bool KM = false, int NVT = 6>
MB_HD void face_flux(const Params& p, const DBlk& b, const Tile<R, TY, NVT>& T, int d, int i, int j, int k, int ii,
                     int jj, R* out) {
  // a mirrored block (one cell deep in k, extrapolated k faces) reads its k = 1 plane for the k ghosts
  const int skm = slot_of<KM>(k - 1), sk = slot_of<KM>(k), sk1 = slot_of<KM>(k + 1), sk2 = slot_of<KM>(k + 2);
  const int l0 = lin32(b, i, j, k);
  const int st = (d == 0) ? 1 : (d == 1 ? b.pi : b.pi * b.pj);
  // the 4-cell stencil along d
  int o4[4];
  if (d == 0) { o4[0] = T.off(sk, jj, ii - 1); o4[1] = T.off(sk, jj, ii); o4[2] = T.off(sk, jj, ii + 1); o4[3] = T.off(sk, jj, ii + 2); }
  else if (d == 1) { o4[0] = T.off(sk, jj - 1, ii); o4[1] = T.off(sk, jj, ii); o4[2] = T.off(sk, jj + 1, ii); o4[3] = T.off(sk, jj + 2, ii); }
  else { o4[0] = T.off(skm, jj, ii); o4[1] = T.off(sk, jj, ii); o4[2] = T.off(sk1, jj, ii); o4[3] = T.off(sk2, jj, ii); }
  R pm1[MB_NP], p0[MB_NP], pp1[MB_NP], pp2[MB_NP], dlc[4];
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) {
    pm1[s] = T.v(o4[0], s); p0[s] = T.v(o4[1], s); pp1[s] = T.v(o4[2], s); pp2[s] = T.v(o4[3], s);
  }
  const auto* gdl = Geo<R>::dl(b);
#pragma unroll
  for (int q = 0; q < 4; ++q) dlc[q] = (R)ld(gdl + d + 3 * (l0 + (q - 1) * st));
  const auto* f = Geo<R>::fm(b, d) + fmi32(b, d, i, j, k);
  R nx = (R)ld(f), ny = (R)ld(f + 1), nz = (R)ld(f + 2), area = (R)ld(f + 3);
  R bet = (R)1;
  if (RS == 0 && p.sd) {  // the sensor of the face's left cell (Mod_Fluxes.f90:282-294; conv_cuf: bet = beta(i,j,k))
    bet = sd_beta<R>(p.sd, p0[MB_IPR], T.v(T.off(sk, jj, ii - 1), MB_IPR), T.v(T.off(sk, jj, ii + 1), MB_IPR),
                     T.v(T.off(sk, jj - 1, ii), MB_IPR), T.v(T.off(sk, jj + 1, ii), MB_IPR),
                     T.v(T.off(skm, jj, ii), MB_IPR), T.v(T.off(sk1, jj, ii), MB_IPR));
  }
  R urL = (R)0, urR = (R)0;
  if (RS == 0 && p.prec) {  // HLLC-PC: the Ur of the face's two cells (conv_physics.inc:159-163)
    urL = (R)ld(p.ur + b.boff + l0);
    urR = (R)ld(p.ur + b.boff + l0 + st);
  }
  conv_face<R, RS, LIM>(p, pm1, p0, pp1, pp2, dlc, nx, ny, nz, area, out, bet, urL, urR);
  if (!VISC) return;
  // ---- viscous face: cells 1,2 = (c, c+d); 3,4 = c -/+ b-axis; 5,6 = c+d -/+ b; 7,8 = c -/+ c-axis; 9,10 = c+d -/+ c
  int oc[10];
  oc[0] = o4[1];
  oc[1] = o4[2];
  if (d == 0) {
    oc[2] = T.off(sk, jj - 1, ii); oc[3] = T.off(sk, jj + 1, ii); oc[4] = T.off(sk, jj - 1, ii + 1); oc[5] = T.off(sk, jj + 1, ii + 1);
    oc[6] = T.off(skm, jj, ii); oc[7] = T.off(sk1, jj, ii); oc[8] = T.off(skm, jj, ii + 1); oc[9] = T.off(sk1, jj, ii + 1);
  } else if (d == 1) {
    oc[2] = T.off(sk, jj, ii - 1); oc[3] = T.off(sk, jj, ii + 1); oc[4] = T.off(sk, jj + 1, ii - 1); oc[5] = T.off(sk, jj + 1, ii + 1);
    oc[6] = T.off(skm, jj, ii); oc[7] = T.off(sk1, jj, ii); oc[8] = T.off(skm, jj + 1, ii); oc[9] = T.off(sk1, jj + 1, ii);
  } else {
    oc[2] = T.off(sk, jj, ii - 1); oc[3] = T.off(sk, jj, ii + 1); oc[4] = T.off(sk1, jj, ii - 1); oc[5] = T.off(sk1, jj, ii + 1);
    oc[6] = T.off(sk, jj - 1, ii); oc[7] = T.off(sk, jj + 1, ii); oc[8] = T.off(sk1, jj - 1, ii); oc[9] = T.off(sk1, jj + 1, ii);
  }
  auto w = [&](int q, int s) -> R { return T.v(oc[q], s); };
  // rho_c = sum(rho_s) = rho_s (one species); T_c from the tile
  R G[MB_NP][3];
  {
    R ga[MB_NP], gb[MB_NP], gc[MB_NP];
    if (Fast<R>::on) {  // one species: the mass-fraction gradient is zero
      ga[0] = gb[0] = gc[0] = (R)0;
    } else {
      R irho1 = (R)1 / w(0, 0), irho2 = (R)1 / w(1, 0);
      R irt1 = (R)1 / w(2, 0), irt2 = (R)1 / w(3, 0), irt3 = (R)1 / w(4, 0), irt4 = (R)1 / w(5, 0);
      R jrt1 = (R)1 / w(6, 0), jrt2 = (R)1 / w(7, 0), jrt3 = (R)1 / w(8, 0), jrt4 = (R)1 / w(9, 0);
      ga[0] = w(1, 0) * irho2 - w(0, 0) * irho1;
      gb[0] = (w(3, 0) * irt2 - w(2, 0) * irt1 + w(5, 0) * irt4 - w(4, 0) * irt3) * (R)0.25;
      gc[0] = (w(7, 0) * jrt2 - w(6, 0) * jrt1 + w(9, 0) * jrt4 - w(8, 0) * jrt3) * (R)0.25;
    }
    ga[MB_IPR] = w(1, 5) - w(0, 5);
    gb[MB_IPR] = (w(3, 5) - w(2, 5) + w(5, 5) - w(4, 5)) * (R)0.25;
    gc[MB_IPR] = (w(7, 5) - w(6, 5) + w(9, 5) - w(8, 5)) * (R)0.25;
#pragma unroll
    for (int s = MB_IU; s <= MB_IW; ++s) {
      ga[s] = w(1, s) - w(0, s);
      gb[s] = (w(3, s) - w(2, s) + w(5, s) - w(4, s)) * (R)0.25;
      gc[s] = (w(7, s) - w(6, s) + w(9, s) - w(8, s)) * (R)0.25;
    }
#pragma unroll
    for (int s = 0; s < MB_NP; ++s) {
      G[s][0] = (d == 0) ? ga[s] : gb[s];
      G[s][1] = (d == 0) ? gb[s] : (d == 1 ? ga[s] : gc[s]);
      G[s][2] = (d == 2) ? ga[s] : gc[s];
    }
  }
  R Mav[3][3];
  const auto* m1 = Geo<R>::m(b) + 9 * l0;
  const auto* m2 = Geo<R>::m(b) + 9 * (l0 + st);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int q = 0; q < 3; ++q) Mav[a][q] = (R)0.5 * ((R)ld(m1 + a + 3 * q) + (R)ld(m2 + a + 3 * q));
#pragma unroll
  for (int iv = 0; iv < MB_NP; ++iv) {
    R g1 = G[iv][0], g2 = G[iv][1], g3 = G[iv][2];
    G[iv][0] = g1 * Mav[0][0] + g2 * Mav[1][0] + g3 * Mav[2][0];
    G[iv][1] = g1 * Mav[0][1] + g2 * Mav[1][1] + g3 * Mav[2][1];
    G[iv][2] = g1 * Mav[0][2] + g2 * Mav[1][2] + g3 * Mav[2][2];
  }
  R Pf[MB_NP];
#pragma unroll
  for (int iv = 0; iv < MB_NP; ++iv) Pf[iv] = (R)0.5 * (w(0, iv) + w(1, iv));
  R frs = (R)0.5 * (w(0, 0) + w(1, 0));
  R fp = (R)0.5 * (w(0, MB_IPR) + w(1, MB_IPR));
  R drho, dT, dcp, dmil, dkl, tdf0;
  int tint;
  face_thermo<R>(p, frs, fp, drho, dT, tint, tdf0, dcp, dmil, dkl);
  visc_flux<R>(p, G, Pf, nx, ny, nz, area, drho, dT, dcp, dmil, dkl, out + MB_NP);
}

// ---------------------------------------------------------------------------------------------
// The boundary record of the cell (i,j,k) on face F, added into acc (the R_flat row of the cell).
MB_HD void bc_face_geom(const DBlk& b, int Im, int Jm, int Km, int F, double* g) {
  int dir = (F + 1) / 2, modfm = F % 2;
  const double* f = (dir == 1) ? fm1p(b, Im - modfm, Jm, Km) : (dir == 2 ? fm2p(b, Im, Jm - modfm, Km) : fm3p(b, Im, Jm, Km - modfm));
  g[0] = ld(f); g[1] = ld(f + 1); g[2] = ld(f + 2); g[3] = ld(f + 3);
}

// BC_Connection_Eul_lean (Lib_BC.f90:1770-1867)
template <typename R, int RS = 0, int LIM = 0>
MB_HD void bc_conn_eul(const Params& p, const DBlk& b, const double* __restrict__ P, int Im, int Jm,
                                         int Km, int Fm, R* A) {
  const long long nc = p.nc;
  const int rs = RS ? RS : p.rs;
  const int lim = LIM ? LIM : p.lim;
  int dir = (Fm + 1) / 2, modfm = Fm % 2, modfm1 = 1 - modfm, modfm2 = 1 - 2 * modfm, gstep = 2 * modfm - 1;
  int o[4] = {modfm * (-gstep * GC) + modfm1 * gstep, modfm * (-gstep), modfm1 * (-gstep),
              modfm1 * (-gstep * GC) + modfm * gstep};
  const long long st = (dir == 1) ? 1 : (dir == 2 ? (long long)b.pi : (long long)b.pi * b.pj);
  const long long rm = row(b, Im, Jm, Km);
  const long long lm = rm - b.boff;
  R dlc4[4];
  long long rr[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    rr[q] = rm + o[q] * st;
    dlc4[q] = cvt<R>(ld(b.dl + (dir - 1) + 3 * (lm + o[q] * st)));
  }
  double g[4];
  bc_face_geom(b, Im, Jm, Km, Fm, g);
  R nx = cvt<R>(g[0]), ny = cvt<R>(g[1]), nz = cvt<R>(g[2]), area = cvt<R>(g[3]);
  R beta_ = (R)1;
  if (RS == 0 && p.sd) {  // the sensor of the record's cell (Lib_BC.f90:1811-1818); a mirrored block's k ghosts are
                          // its k = 1 cells
    const double* pp = P + MB_IPR * nc;
    const long long sj = b.pi, sk = b.kmirror ? 0 : (long long)b.pi * b.pj;
    beta_ = sd_beta<R>(p.sd, cvt<R>(ld(pp + rm)), cvt<R>(ld(pp + rm - 1)), cvt<R>(ld(pp + rm + 1)),
                       cvt<R>(ld(pp + rm - sj)), cvt<R>(ld(pp + rm + sj)), cvt<R>(ld(pp + rm - sk)),
                       cvt<R>(ld(pp + rm + sk)));
  }
  R Dl1 = dlc4[0] * (R)0.5, Dl2 = dlc4[1] * (R)0.5, Dl3 = dlc4[2] * (R)0.5, Dl4 = dlc4[3] * (R)0.5;
  R D12 = Dl1 + Dl2, D23 = Dl2 + Dl3, D34 = Dl3 + Dl4;
  R PL[MB_NP], PR[MB_NP];
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) {
    R q1 = cvt<R>(ld(P + rr[0] + s * nc)), q2 = cvt<R>(ld(P + rr[1] + s * nc)), q3 = cvt<R>(ld(P + rr[2] + s * nc)),
      q4 = cvt<R>(ld(P + rr[3] + s * nc));
    R d21 = (q2 - q1) / D12, d32 = (q3 - q2) / D23, d43 = (q4 - q3) / D34;
    PL[s] = q2 + beta_ * rlimiter(lim, d32, d21) * Dl2;
    PR[s] = q3 - beta_ * rlimiter(lim, d43, d32) * Dl3;
  }
  R rhoL, RL, rhoR, RRr;
  rotot_rtot(p, PL[0], rhoL, RL);
  R aL = f_ss(p, PL[0], PL[MB_IPR], rhoL, RL);
  rotot_rtot(p, PR[0], rhoR, RRr);
  R aR = f_ss(p, PR[0], PR[MB_IPR], rhoR, RRr);
  R F_r, F_u, F_v, F_w, F_E;
  // HLLC-PC: the Ur of cells 2 and 3, the ghost's 0 (never filled, Lib_BC.f90:1739-1742)
  const R urL = (RS == 0 && p.prec) ? (R)ld(p.ur + rr[1]) : (R)0, urR = (RS == 0 && p.prec) ? (R)ld(p.ur + rr[2]) : (R)0;
  riemann_rec<R, RS>(p, PL[0], PL[MB_IU], PL[MB_IV], PL[MB_IW], PL[MB_IPR], aL, rhoL, RL, PR[0], PR[MB_IU], PR[MB_IV],
                     PR[MB_IW], PR[MB_IPR], aR, rhoR, RRr, nx, ny, nz, F_r, F_u, F_v, F_w, F_E, beta_, urL, urR);
  R su = copysign((R)0.5, F_r), selL = (R)0.5 + su, selR = su - (R)0.5;
  R Fmass = F_r * area;
  R sg = (R)modfm2;
  A[0] = sg * Fmass * (selL * PL[0] / rhoL - selR * PR[0] / rhoR);
  A[MB_IU] = sg * F_u * area;
  A[MB_IV] = sg * F_v * area;
  A[MB_IW] = sg * F_w * area;
  A[MB_IPR] = sg * F_E * area;
}

// BC_Connection_Visc_lean (Lib_BC.f90:2113-2178). The reference reads bc_pg(:,1:6), a copy of six donor cells taken
// after the ghost fill (Ghost_Connection_pairs_B, Lib_Extrapolation.f90:1136-1191); the records run on the same
// filled state, so this reads those cells of P in place: pgr = the six donor rows of the record (the same values,
// without the copy pass and its nconn x 30 FP64 buffer).
template <typename R>
MB_HD void bc_conn_visc(const Params& p, const DBlk& b, const double* __restrict__ P, int Im, int Jm,
                                          int Km, int Fm, const long long* __restrict__ pgr, R* S) {
  const long long nc = p.nc;
  int dir = (Fm + 1) / 2, modfm2 = 1 - 2 * (Fm % 2), gstep = 2 * (Fm % 2) - 1;
  int ia = dir - 1, ib, ic;
  long long sb, sc;
  if (dir == 1) { ib = 1; ic = 2; sb = b.pi; sc = (long long)b.pi * b.pj; }
  else if (dir == 2) { ib = 0; ic = 2; sb = 1; sc = (long long)b.pi * b.pj; }
  else { ib = 0; ic = 1; sb = 1; sc = b.pi; }
  const long long st = (dir == 1) ? 1 : (dir == 2 ? (long long)b.pi : (long long)b.pi * b.pj);
  const long long r1 = row(b, Im, Jm, Km);
  const long long l1 = r1 - b.boff;
  const long long lg = l1 - gstep * st;  // the ghost cell Im - gstep along dir
  R M[3][3];
#pragma unroll
  for (int q = 0; q < 3; ++q)
#pragma unroll
    for (int a = 0; a < 3; ++a)
      M[a][q] = (R)0.5 * (cvt<R>(ld(b.m + a + 3 * q + 9 * l1)) + cvt<R>(ld(b.m + a + 3 * q + 9 * lg)));
  // cells: 0 loc, 1 ghost (Pg(:,1)), 2 b+, 3 b-, 4 c+, 5 c-, 6..9 Pg(:,3..6)
  const long long scm = (b.kmirror && ic == 2) ? 0 : sc;  // a mirrored block's k ghosts are its k = 1 cells
  const long long rc[6] = {r1, 0, r1 + sb, r1 - sb, r1 + scm, r1 - scm};
  auto pv = [&](int q, int s) -> R {
    if (q == 1) return cvt<R>(ld(P + pgr[0] + s * nc));
    if (q >= 6) return cvt<R>(ld(P + pgr[q - 4] + s * nc));
    return cvt<R>(ld(P + rc[q] + s * nc));
  };
  R rh[10], rg[10];
#pragma unroll
  for (int q = 0; q < 10; ++q) rotot_rtot(p, pv(q, 0), rh[q], rg[q]);
  R G2l[MB_NP][3], G2g[MB_NP][3], Pa[MB_NP];
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) {
    R vv[10];
#pragma unroll
    for (int q = 0; q < 10; ++q) {
      R x = pv(q, s);
      if (s >= MB_IU && s <= MB_IW) vv[q] = x;
      else if (s == MB_IPR) vv[q] = x / (rh[q] * rg[q]);
      else vv[q] = x / rh[q];
    }
    R gl[3], gg[3];
    gl[ia] = (vv[1] - vv[0]) * (R)modfm2;
    gl[ib] = (vv[2] - vv[3]) * (R)0.5;
    gl[ic] = (vv[4] - vv[5]) * (R)0.5;
    gg[ia] = (vv[0] - vv[1]) * (R)(-modfm2);
    gg[ib] = (vv[7] - vv[6]) * (R)0.5;
    gg[ic] = (vv[9] - vv[8]) * (R)0.5;
#pragma unroll
    for (int kk = 0; kk < 3; ++kk) {
      G2l[s][kk] = gl[0] * M[0][kk] + gl[1] * M[1][kk] + gl[2] * M[2][kk];
      G2g[s][kk] = gg[0] * M[0][kk] + gg[1] * M[1][kk] + gg[2] * M[2][kk];
    }
    Pa[s] = (R)0.5 * (pv(0, s) + pv(1, s));
  }
  R rho_f, T_f, td, cp_f, mil_f, kl_f;
  int ti;
  face_thermo(p, Pa[0], Pa[MB_IPR], rho_f, T_f, ti, td, cp_f, mil_f, kl_f);
  double g[4];
  bc_face_geom(b, Im, Jm, Km, Fm, g);
  R nx = cvt<R>(g[0]), ny = cvt<R>(g[1]), nz = cvt<R>(g[2]), area = cvt<R>(g[3]);
  R Fl[MB_NP], Fg[MB_NP];
  visc_flux(p, G2l, Pa, nx, ny, nz, area, rho_f, T_f, cp_f, mil_f, kl_f, Fl);
  visc_flux(p, G2g, Pa, nx, ny, nz, area, rho_f, T_f, cp_f, mil_f, kl_f, Fg);
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) S[s] = (R)0.5 * (R)modfm2 * (Fl[s] + Fg[s]);
}

// BC_Extrapolation (Lib_BC.f90:1119-1165)
template <typename R>
MB_HD void bc_extrap(const Params& p, const DBlk& b, const double* __restrict__ P, int Im, int Jm,
                                       int Km, int Fm, R* A) {
  const long long nc = p.nc;
  const long long r = row(b, Im, Jm, Km);
  R Pr[MB_NP];
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) Pr[s] = cvt<R>(ld(P + r + s * nc));
  double g[4];
  bc_face_geom(b, Im, Jm, Km, Fm, g);
  R nx = cvt<R>(g[0]), ny = cvt<R>(g[1]), nz = cvt<R>(g[2]), area = cvt<R>(g[3]);
  R Un = Pr[MB_IU] * nx + Pr[MB_IV] * ny + Pr[MB_IW] * nz;
  R F[MB_NP];
  R Fmass = (R)0;
  F[0] = Pr[0] * Un * area;
  Fmass = Fmass + F[0];
  F[MB_IU] = Fmass * Pr[MB_IU] + Pr[MB_IPR] * area * nx;
  F[MB_IV] = Fmass * Pr[MB_IV] + Pr[MB_IPR] * area * ny;
  F[MB_IW] = Fmass * Pr[MB_IW] + Pr[MB_IPR] * area * nz;
  R vmag = rsqrt_(Pr[MB_IU] * Pr[MB_IU] + Pr[MB_IV] * Pr[MB_IV] + Pr[MB_IW] * Pr[MB_IW]);
  F[MB_IPR] = Fmass * H0(p, Pr[MB_IPR], Pr[0], vmag);
  R sg = (R)face_sign(Fm);
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) A[s] = sg * F[s];
}

// BC_Symmetry_Eul (Lib_BC.f90:640-737): mirror of the boundary cell about the face, limited one-sided
// reconstruction, Riemann problem between the face state and its mirror; momentum rows only. The Euler part of
// the adiabatic wall and the closed-inlet fallback of the 405 record.
template <typename R, int RS = 0, int LIM = 0>
MB_HD void bc_sym_eul(const Params& p, const DBlk& b, const double* __restrict__ P, int Im, int Jm, int Km,
                               int Fm, R* A) {
  const long long nc = p.nc;
  const int lim = LIM ? LIM : p.lim;
  int dir = (Fm + 1) / 2, modfm = Fm % 2, modfm1 = 1 - modfm, modfm2 = 1 - 2 * modfm, gstep = 2 * modfm - 1;
  const long long st = (dir == 1) ? 1 : (dir == 2 ? (long long)b.pi : (long long)b.pi * b.pj);
  const long long rb = row(b, Im, Jm, Km), ri = rb + gstep * st;
  double g[4];
  bc_face_geom(b, Im, Jm, Km, Fm, g);
  R nrm[3] = {cvt<R>(g[0]), cvt<R>(g[1]), cvt<R>(g[2])};
  R area = cvt<R>(g[3]);
  R Bound_Dl = (R)0.5 * cvt<R>(ld(b.dl + (dir - 1) + 3 * (rb - b.boff)));
  R Int_Dl = (R)0.5 * cvt<R>(ld(b.dl + (dir - 1) + 3 * (ri - b.boff)));
  R B[MB_NP], I[MB_NP], G[MB_NP], F[MB_NP];
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) { B[s] = cvt<R>(ld(P + rb + s * nc)); I[s] = cvt<R>(ld(P + ri + s * nc)); }
  R Un = B[MB_IU] * nrm[0] + B[MB_IV] * nrm[1] + B[MB_IW] * nrm[2];
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) G[s] = B[s];
  G[MB_IU] = B[MB_IU] - (R)2 * Un * nrm[0];
  G[MB_IV] = B[MB_IV] - (R)2 * Un * nrm[1];
  G[MB_IW] = B[MB_IW] - (R)2 * Un * nrm[2];
  const R fm = (R)modfm, fm1 = (R)modfm1;
  R Dist12 = (R)2 * Bound_Dl * fm + (Bound_Dl + Int_Dl) * fm1;
  R Dist23 = (Bound_Dl + Int_Dl) * fm + (R)2 * Bound_Dl * fm1;
  R Dist = Bound_Dl * (R)modfm2;
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) {
    R P1 = fm * G[s] + fm1 * I[s];
    R P3 = fm * I[s] + fm1 * G[s];
    R s32 = (P3 - B[s]) / Dist23;
    R s21 = (B[s] - P1) / Dist12;
    F[s] = B[s] + rlimiter(lim, s32, s21) * Dist;
  }
  R rotot, Rtot;
  rotot_rtot(p, F[0], rotot, Rtot);
  R Sound = f_ss(p, F[0], F[MB_IPR], rotot, Rtot);
  Un = F[MB_IU] * nrm[0] + F[MB_IV] * nrm[1] + F[MB_IW] * nrm[2];
  R Vt[3] = {F[MB_IU] - Un * nrm[0], F[MB_IV] - Un * nrm[1], F[MB_IW] - Un * nrm[2]};
  R Un1 = Un * (R)modfm2;
  R U1[3], U4[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) { U1[a] = Un1 * nrm[a] + Vt[a]; U4[a] = -Un1 * nrm[a] + Vt[a]; }
  R F_r, F_u, F_v, F_w, F_E;
  const R urc = (RS == 0 && p.prec) ? (R)ld(p.ur + rb) : (R)0;  // HLLC-PC: the cell's Ur on both sides (:720-723)
  riemann_rec<R, RS>(p, F[0], U1[0], U1[1], U1[2], F[MB_IPR], Sound, rotot, Rtot, F[0], U4[0], U4[1], U4[2],
                     F[MB_IPR], Sound, rotot, Rtot, nrm[0], nrm[1], nrm[2], F_r, F_u, F_v, F_w, F_E, (R)1, urc, urc);
  A[0] = (R)-0.0;  // an exact no-op when added: only the momentum rows change
  A[MB_IU] = (R)modfm2 * F_u * area;
  A[MB_IV] = (R)modfm2 * F_v * area;
  A[MB_IW] = (R)modfm2 * F_w * area;
  A[MB_IPR] = (R)-0.0;
}

// BC_Wall_Heat_dev (Lib_BC.f90:879-982), laminar adiabatic no-slip wall: the wall-normal velocity gradient of the
// boundary cell, Grad . M of the cell, Stress_Vector_Std (Mod_Fluid.f90:20-44) with mu_t = 0; momentum rows only.
template <typename R>
MB_HD void bc_wall_heat(const Params& p, const DBlk& b, const double* __restrict__ P, int Im, int Jm, int Km,
                                 int Fm, R* S) {
  const long long nc = p.nc;
  int dir = (Fm + 1) / 2, modfm = Fm % 2, modfm2 = 1 - 2 * modfm, modfm3 = 2 * (2 * modfm - 1);
  const long long rb = row(b, Im, Jm, Km), l = rb - b.boff;
  R Pb[MB_NP];
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) Pb[s] = cvt<R>(ld(P + rb + s * nc));
  R M[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int q = 0; q < 3; ++q) M[a][q] = cvt<R>(ld(b.m + a + 3 * q + 9 * l));
  R rho, Rgas;
  rotot_rtot(p, Pb[0], rho, Rgas);
  R T = Pb[MB_IPR] / (rho * Rgas);
  int ti = tidx(p, T);
  R Tdiff = T - (R)ti;
  R mil, kl;
  wilke(p, Pb[0], rho, ti, Tdiff, mil, kl);
  R Grad[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int d = 0; d < 3; ++d) Grad[a][d] = (d == dir - 1) ? Pb[MB_IU + a] * (R)modfm3 : (R)0;
  R G2[3][3];
#pragma unroll
  for (int kk = 0; kk < 3; ++kk)
#pragma unroll
    for (int ii = 0; ii < 3; ++ii) G2[ii][kk] = Grad[ii][0] * M[0][kk] + Grad[ii][1] * M[1][kk] + Grad[ii][2] * M[2][kk];
  double g[4];
  bc_face_geom(b, Im, Jm, Km, Fm, g);
  R nx = cvt<R>(g[0]), ny = cvt<R>(g[1]), nz = cvt<R>(g[2]), area = cvt<R>(g[3]);
  const R ntt = (R)(-2.0 / 3.0);
  R mi = mil + (R)0;
  R lam = ntt * mi;
  R Div = G2[0][0] + G2[1][1] + G2[2][2];
  R lamDiv = lam * Div;
  R txx = lamDiv + (R)2 * mi * G2[0][0], tyy = lamDiv + (R)2 * mi * G2[1][1], tzz = lamDiv + (R)2 * mi * G2[2][2];
  R txy = mi * (G2[0][1] + G2[1][0]), txz = mi * (G2[0][2] + G2[2][0]), tyz = mi * (G2[1][2] + G2[2][1]);
  R S1 = txx * nx + txy * ny + txz * nz;
  R S2 = txy * nx + tyy * ny + tyz * nz;
  R S3 = txz * nx + tyz * ny + tzz * nz;
  S[0] = (R)0;  // an exact no-op when subtracted: only the momentum rows change
  S[MB_IU] = (R)modfm2 * area * S1;
  S[MB_IV] = (R)modfm2 * area * S2;
  S[MB_IW] = (R)modfm2 * area * S3;
  S[MB_IPR] = (R)0;
}

// Stress_Vector_Std (Mod_Fluid.f90:20-44) with mu_t = 0: the stress vector tau . n of the gradient G2 (Grad . M)
template <typename R>
MB_HD void stress_std(const R G2[3][3], R nx, R ny, R nz, R mil, R* S) {
  const R ntt = (R)(-2.0 / 3.0);
  R mi = mil + (R)0;
  R lam = ntt * mi;
  R Div = G2[0][0] + G2[1][1] + G2[2][2];
  R lamDiv = lam * Div;
  R txx = lamDiv + (R)2 * mi * G2[0][0], tyy = lamDiv + (R)2 * mi * G2[1][1], tzz = lamDiv + (R)2 * mi * G2[2][2];
  R txy = mi * (G2[0][1] + G2[1][0]), txz = mi * (G2[0][2] + G2[2][0]), tyz = mi * (G2[1][2] + G2[2][1]);
  S[0] = txx * nx + txy * ny + txz * nz;
  S[1] = txy * nx + tyy * ny + tyz * nz;
  S[2] = txz * nx + tyz * ny + tzz * nz;
}

// BC_Symmetry_Visc (Lib_BC.f90:741-861), laminar: the boundary cell and its four transverse neighbours mirrored about
// the face give the normal and transverse velocity gradients; the stress of Grad . M (momentum rows) and its work on
// the face-mean velocity (energy row), subtracted.
template <typename R>
MB_HD void bc_sym_visc(const Params& p, const DBlk& b, const double* __restrict__ P, int Im, int Jm, int Km, int Fm,
                       R* S) {
  const long long nc = p.nc;
  const int modfm = Fm % 2, modfm2 = 1 - 2 * modfm;
  const long long rb = row(b, Im, Jm, Km), l = rb - b.boff;
  R Pb[MB_NP];
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) Pb[s] = cvt<R>(ld(P + rb + s * nc));
  R M[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int q = 0; q < 3; ++q) M[a][q] = cvt<R>(ld(b.m + a + 3 * q + 9 * l));
  R rho, Rgas;
  rotot_rtot(p, Pb[0], rho, Rgas);
  R T = Pb[MB_IPR] / (rho * Rgas);
  int ti = tidx(p, T);
  R Tdiff = T - (R)ti;
  R mil, kl;
  wilke(p, Pb[0], rho, ti, Tdiff, mil, kl);
  // transverse strides: b then c axis of the face (Fm 1-2: j, k; 3-4: i, k; 5-6: i, j); a = the face axis
  const long long sj = b.pi, sk = (long long)b.pi * b.pj;
  const long long sb = (Fm <= 2) ? sj : 1, sc = (Fm <= 4) ? sk : sj;
  const int a = (Fm - 1) >> 1, bb = (Fm <= 2) ? 1 : 0, cc = (Fm <= 4) ? 2 : 1;
  R V1[3] = {Pb[MB_IU], Pb[MB_IV], Pb[MB_IW]}, V3[3], V4[3], V7[3], V8[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    V3[q] = cvt<R>(ld(P + rb - sb + (MB_IU + q) * nc));
    V4[q] = cvt<R>(ld(P + rb + sb + (MB_IU + q) * nc));
    V7[q] = cvt<R>(ld(P + rb - sc + (MB_IU + q) * nc));
    V8[q] = cvt<R>(ld(P + rb + sc + (MB_IU + q) * nc));
  }
  double g[4];
  bc_face_geom(b, Im, Jm, Km, Fm, g);
  const R nrm[3] = {cvt<R>(g[0]), cvt<R>(g[1]), cvt<R>(g[2])};
  const R area = cvt<R>(g[3]);
  R d1 = V1[0] * nrm[0] + V1[1] * nrm[1] + V1[2] * nrm[2];
  R d3 = V3[0] * nrm[0] + V3[1] * nrm[1] + V3[2] * nrm[2];
  R d4 = V4[0] * nrm[0] + V4[1] * nrm[1] + V4[2] * nrm[2];
  R d7 = V7[0] * nrm[0] + V7[1] * nrm[1] + V7[2] * nrm[2];
  R d8 = V8[0] * nrm[0] + V8[1] * nrm[1] + V8[2] * nrm[2];
  R V2[3], Grad[3][3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    V2[q] = V1[q] - (R)2 * d1 * nrm[q];
    R V5 = V3[q] - (R)2 * d3 * nrm[q], V6 = V4[q] - (R)2 * d4 * nrm[q];
    R V9 = V7[q] - (R)2 * d7 * nrm[q], V10 = V8[q] - (R)2 * d8 * nrm[q];
    R ga = (V2[q] - V1[q]) * (R)modfm2;
    R gb = (V4[q] - V3[q] + V6 - V5) * (R)0.25;
    R gc = (V8[q] - V7[q] + V10 - V9) * (R)0.25;
#pragma unroll
    for (int d = 0; d < 3; ++d) Grad[q][d] = (d == a) ? ga : ((d == bb) ? gb : gc);
    (void)cc;
  }
  R G2[3][3];
#pragma unroll
  for (int kk = 0; kk < 3; ++kk)
#pragma unroll
    for (int ii = 0; ii < 3; ++ii) G2[ii][kk] = Grad[ii][0] * M[0][kk] + Grad[ii][1] * M[1][kk] + Grad[ii][2] * M[2][kk];
  R St[3];
  stress_std(G2, nrm[0], nrm[1], nrm[2], mil, St);
  R Vf[3] = {(R)0.5 * (V1[0] + V2[0]), (R)0.5 * (V1[1] + V2[1]), (R)0.5 * (V1[2] + V2[2])};
  S[0] = (R)0;
  S[MB_IU] = (R)modfm2 * area * St[0];
  S[MB_IV] = (R)modfm2 * area * St[1];
  S[MB_IW] = (R)modfm2 * area * St[2];
  S[MB_IPR] = (R)modfm2 * area * (Vf[0] * St[0] + Vf[1] * St[1] + Vf[2] * St[2]);
}

// BC_Wall_Temperature_dev (Lib_BC.f90:997-1115), laminar no-slip wall at T_wall: mu and k of the wall state
// (p of the cell at T_wall; k = mu cp / Pr when Pr > 0), the wall-normal velocity and temperature gradients of the
// boundary cell: stress (momentum rows) and conducted heat (energy row), subtracted.
template <typename R>
MB_HD void bc_wall_temp(const Params& p, const DBlk& b, const double* __restrict__ P, int Im, int Jm, int Km, int Fm,
                        double Tw_, R* S) {
  const long long nc = p.nc;
  int dir = (Fm + 1) / 2, modfm = Fm % 2, modfm2 = 1 - 2 * modfm, modfm3 = 2 * (2 * modfm - 1);
  const long long rb = row(b, Im, Jm, Km), l = rb - b.boff;
  const R Tw = cvt<R>(Tw_);
  R Pb[MB_NP];
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) Pb[s] = cvt<R>(ld(P + rb + s * nc));
  R M[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int q = 0; q < 3; ++q) M[a][q] = cvt<R>(ld(b.m + a + 3 * q + 9 * l));
  R rho, Rgas;
  rotot_rtot(p, Pb[0], rho, Rgas);
  R T = Pb[MB_IPR] / (rho * Rgas);
  R rho_wall = Pb[MB_IPR] / (Rgas * Tw);
  R Pw0 = Pb[0] * rho_wall / rho;
  int ti = tidx(p, Tw);
  R Tdiff = Tw - (R)ti;
  R mil, kl;
  wilke(p, Pw0, rho_wall, ti, Tdiff, mil, kl);
  if (p.prandtl > 0.0) kl = mil * f_cp(p, Pw0, ti, Tdiff, rho_wall) / (R)p.prandtl;
  R G2[3][3];
#pragma unroll
  for (int kk = 0; kk < 3; ++kk)
#pragma unroll
    for (int ii = 0; ii < 3; ++ii) {
      R g1 = (dir == 1) ? Pb[MB_IU + ii] * (R)modfm3 : (R)0, g2 = (dir == 2) ? Pb[MB_IU + ii] * (R)modfm3 : (R)0,
        g3 = (dir == 3) ? Pb[MB_IU + ii] * (R)modfm3 : (R)0;
      G2[ii][kk] = g1 * M[0][kk] + g2 * M[1][kk] + g3 * M[2][kk];
    }
  double g[4];
  bc_face_geom(b, Im, Jm, Km, Fm, g);
  R nx = cvt<R>(g[0]), ny = cvt<R>(g[1]), nz = cvt<R>(g[2]), area = cvt<R>(g[3]);
  R St[3];
  stress_std(G2, nx, ny, nz, mil, St);
  R Gnp_dir = (T - Tw) * (R)modfm3;
  R Gnp[3];
#pragma unroll
  for (int kk = 0; kk < 3; ++kk) Gnp[kk] = Gnp_dir * M[dir - 1][kk];
  R Flux_np = area * kl * (Gnp[0] * nx + Gnp[1] * ny + Gnp[2] * nz);
  S[0] = (R)0;
  S[MB_IU] = (R)modfm2 * area * St[0];
  S[MB_IV] = (R)modfm2 * area * St[1];
  S[MB_IW] = (R)modfm2 * area * St[2];
  S[MB_IPR] = (R)modfm2 * Flux_np;
}

template <typename R> MB_HD R pw_(R x, R y);
template <> MB_HD double pw_(double x, double y) { return pow(x, y); }
template <> MB_HD float pw_(float x, float y) { return powf(x, y); }

// BC_Outflow (Lib_BC.f90:1166-1240): the face state of an outflow to the pressure p_Amb (isentropic when the normal
// Mach number is below 1 and p_Amb > 0, the boundary cell itself otherwise) and its flux Fl
template <typename R>
MB_HD void outflow_face(const Params& p, const R* Bp, R Brho, R BRgas, R BSound, R Un, R BGamma, R Riem,
                        const R* nrm, R area, R p_Amb, R BC_Sign, R* Fl) {
  R VT[3] = {Bp[MB_IU] - Un * nrm[0], Bp[MB_IV] - Un * nrm[1], Bp[MB_IW] - Un * nrm[2]};
  R Mach_N = fabs(Un / BSound);
  R pe = p_Amb;
  R Fp[MB_NP], Fun, Frho, FRgas;
  if (Mach_N < (R)1 && p_Amb > (R)0) {
    R delta = (R)0.5 * (BGamma - (R)1);
    R denom = (R)1 / pw_((R)1 + delta, BGamma / (BGamma - (R)1));
    R pstar = Bp[MB_IPR] * denom * pw_((R)1 + delta * (Mach_N * Mach_N), BGamma / (BGamma - (R)1));
    if (pstar >= p_Amb) pe = pstar;
    R Isentropic = (BGamma - (R)1) / ((R)2 * BGamma);
    R FSound = BSound * pw_(pe / Bp[MB_IPR], Isentropic);
    Fun = (Riem - FSound) / (BC_Sign * (R)0.5 * (BGamma - (R)1));
    Fp[MB_IPR] = pe;
    Frho = BGamma * Fp[MB_IPR] / (FSound * FSound);
    Fp[0] = Bp[0] / Brho * Frho;
    Fp[MB_IU] = VT[0] + Fun * nrm[0];
    Fp[MB_IV] = VT[1] + Fun * nrm[1];
    Fp[MB_IW] = VT[2] + Fun * nrm[2];
    FRgas = BRgas;
  } else {
#pragma unroll
    for (int s = 0; s < MB_NP; ++s) Fp[s] = Bp[s];
    Fun = Un; Frho = Brho; FRgas = BRgas;
  }
  R FT = Fp[MB_IPR] / (FRgas * Frho);
  int Ti = tidx(p, FT);
  R Td = FT - (R)Ti;
  const R* H = Tab<R>::h(p);
  R FEnth = (R)0 + Fp[0] / Frho * (H[Ti] + (H[Ti + 1] - H[Ti]) * Td);
  Fl[0] = Fp[0] * area * Fun;
  R Fmass = Frho * area * Fun;
  Fl[MB_IU] = Fp[MB_IU] * Fmass + Fp[MB_IPR] * area * nrm[0];
  Fl[MB_IV] = Fp[MB_IV] * Fmass + Fp[MB_IPR] * area * nrm[1];
  Fl[MB_IW] = Fp[MB_IW] * Fmass + Fp[MB_IPR] * area * nrm[2];
  R vt2 = Fp[MB_IU] * Fp[MB_IU] + Fp[MB_IV] * Fp[MB_IV] + Fp[MB_IW] * Fp[MB_IW];
  Fl[MB_IPR] = Fmass * ((R)0.5 * vt2 + FEnth);
}

// BC_Subsonic_Inflow (Lib_BC.f90:1335-1512), one species: the face state from the outgoing Riemann invariant and the
// stagnation (mach >= 0) or mass-flux (mach < 0: p0 = the mass flux; mach -10: T0 total) conditions, and its flux Fl
template <typename R>
MB_HD void subsonic_inflow_face(const Params& p, const R* Bp, R Un, R Sound, R Gamma, R Riem, R BC_alpha, R BC_beta,
                                R BC_Mach, R BC_T0, R BC_p0, R rel, R BC_Sign, const R* t, const R* n, R area, R* Fl) {
  R bv[3] = {n[1] * t[2] - n[2] * t[1], n[2] * t[0] - n[0] * t[2], n[0] * t[1] - n[1] * t[0]};
  R bmod = rsqrt_(bv[0] * bv[0] + bv[1] * bv[1] + bv[2] * bv[2]);
  bv[0] = bv[0] / bmod; bv[1] = bv[1] / bmod; bv[2] = bv[2] / bmod;
  R alpha, beta;
  if (BC_alpha == (R)0 && BC_beta == (R)0) {
    alpha = atan(n[1] / (n[0] + (R)1e-20));
    beta = atan(n[2] / (n[0] + (R)1e-20));
  } else {
    alpha = BC_alpha; beta = BC_beta;
  }
  const R ta = tan(alpha), tb = tan(beta);
  R XA = n[1] - n[0] * ta, XB = t[1] - t[0] * ta, XC = bv[1] - bv[0] * ta;
  R XD = n[2] - n[0] * tb, XE = t[2] - t[0] * tb, XF = bv[2] - bv[0] * tb;
  R check = (XC * XE - XF * XB);
  R E1 = (XF * XA - XC * XD) / check;
  R E2 = (XD * XB - XE * XA) / check;
  const R ri = (R)p.ri;
  R Fp[MB_NP], Frho, FRgas, Fun;
  if (BC_Mach >= (R)0) {
    R Discr = (R)-1, p0_try = BC_p0, Sound0 = (R)0, Coef_D = (R)0, YA = (R)1, YB = (R)0;
    int iter = 0;
    FRgas = (R)0 + (R)1 * ri;
    while (Discr < (R)0) {  // at most 1001 passes
      iter = iter + 1;
      FRgas = (R)0 + (R)1 * ri;
      Sound0 = rsqrt_(Gamma * FRgas * BC_T0);
      Coef_D = ((R)1 + E1 * E1 + E2 * E2) * (Gamma - (R)1) / (R)2;
      R Coef_C = powr(p0_try / Bp[MB_IPR], (Gamma - (R)1) / Gamma);
      Coef_C = Coef_C * ((Sound / Sound0) * (Sound / Sound0));
      const R g2 = (Gamma - (R)1) / (R)2;
      YA = g2 * g2 + Coef_C * Coef_D;
      YB = BC_Sign * Riem * ((Gamma - (R)1) / (R)2);
      R YC = Riem * Riem - Coef_C * (Sound0 * Sound0);
      Discr = YB * YB - YA * YC;
      if (Discr < (R)0 && fabs(Discr) < (R)1e-2) Discr = (R)0;
      if (Discr < (R)0 && fabs(Discr) > (R)1e-2) {
        if (rel == (R)1) { Discr = (R)0; break; }
        p0_try = rel * p0_try + ((R)1 - rel) * Bp[MB_IPR];
      }
      if (iter > 1000) { Discr = (R)0; break; }
    }
    R Un_Sign = copysign((R)1, Un);
    R Un3 = (YB + Un_Sign * rsqrt_(Discr)) / YA;
    R Sound3 = rsqrt_(Sound0 * Sound0 - Coef_D * (Un3 * Un3));
    R p3 = p0_try * powr(Sound3 / Sound0, (R)2 * Gamma / (Gamma - (R)1));
    R Ut3 = Un3 * E1, Ub3 = Un3 * E2;
    Fp[MB_IPR] = p3;
    Frho = Gamma * Fp[MB_IPR] / (Sound3 * Sound3);
    Fp[0] = (R)1 * Frho;
    Fp[MB_IU] = Un3 * n[0] + Ut3 * t[0] + Ub3 * bv[0];
    Fp[MB_IV] = Un3 * n[1] + Ut3 * t[1] + Ub3 * bv[1];
    Fp[MB_IW] = Un3 * n[2] + Ut3 * t[2] + Ub3 * bv[2];
    Fun = Un3;
  } else {
    R mdot = BC_p0, p3 = Bp[MB_IPR];
    int Ti = tidx(p, BC_T0);
    R Td = BC_T0 - (R)Ti;
    const R* CP = Tab<R>::cp(p);
    R cp3 = (R)0 + (R)1 * (CP[Ti] + (CP[Ti + 1] - CP[Ti]) * Td);
    R Rgas3 = (R)0 + (R)1 * ri;
    R T3 = BC_T0;
    if (BC_Mach == (R)-10) {
      R x = mdot * Rgas3 / p3, y = p3 / (mdot * Rgas3);
      T3 = (-cp3 + rsqrt_(cp3 * cp3 + (R)2 * cp3 * BC_T0 * (x * x))) * (y * y);
    }
    R rho3 = p3 / (Rgas3 * T3);
    R Un3 = mdot / rho3;
    R Ut3 = Un3 * E1, Ub3 = Un3 * E2;
    FRgas = Rgas3;
    Frho = rho3;
    Fp[0] = Frho * (R)1;
    Fp[MB_IU] = Un3 * n[0] + Ut3 * t[0] + Ub3 * bv[0];
    Fp[MB_IV] = Un3 * n[1] + Ut3 * t[1] + Ub3 * bv[1];
    Fp[MB_IW] = Un3 * n[2] + Ut3 * t[2] + Ub3 * bv[2];
    Fp[MB_IPR] = p3;
    Fun = Un3;
  }
  R FT = Fp[MB_IPR] / (FRgas * Frho);
  int Ti = tidx(p, FT);
  R Td = FT - (R)Ti;
  const R* H = Tab<R>::h(p);
  R FEnth = (R)0 + Fp[0] / Frho * (H[Ti] + (H[Ti + 1] - H[Ti]) * Td);
  Fl[0] = Fp[0] * Fun * area;
  R Fmass = Frho * Fun * area;
  Fl[MB_IU] = Fmass * Fp[MB_IU] + Fp[MB_IPR] * area * n[0];
  Fl[MB_IV] = Fmass * Fp[MB_IV] + Fp[MB_IPR] * area * n[1];
  Fl[MB_IW] = Fmass * Fp[MB_IW] + Fp[MB_IPR] * area * n[2];
  R vt2 = Fp[MB_IU] * Fp[MB_IU] + Fp[MB_IV] * Fp[MB_IV] + Fp[MB_IW] * Fp[MB_IW];
  Fl[MB_IPR] = Fmass * ((R)0.5 * vt2 + FEnth);
}

// The inflow / outflow record (type 4), BC_Inflow_Outflow (Lib_BC.f90:1519-1597). The record's closure code (q[8]:
// 0 / 405, 401, 403, 404, 407, as IO_BC_Open.f90:229-307 sets them up) gives mach and pamb: outward flow closes an
// inlet face (BC_Symmetry_Eul) or leaves to pamb (BC_Outflow, 407); inward flow takes the supersonic static inlet
// (405, or mach > 1: BC_Supersonic_Inflow, Lib_BC.f90:1247-1330) or the subsonic closure (BC_Subsonic_Inflow).
template <typename R, int RS = 0, int LIM = 0>
MB_HD void bc_inflow(const Params& p, const DBlk& b, const double* __restrict__ P, int Im, int Jm, int Km,
                              int Fm, const double* __restrict__ q, R* A) {
  const long long nc = p.nc;
  const int lim = LIM ? LIM : p.lim;
  int dir = (Fm + 1) / 2, modfm = Fm % 2, modfm1 = 1 - modfm, modfm2 = 1 - 2 * modfm, gstep = 2 * modfm - 1;
  const long long st = (dir == 1) ? 1 : (dir == 2 ? (long long)b.pi : (long long)b.pi * b.pj);
  const long long rb = row(b, Im, Jm, Km), ri = rb + gstep * st;
  R P2[MB_NP], Ip[MB_NP];
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) { P2[s] = cvt<R>(ld(P + rb + s * nc)); Ip[s] = cvt<R>(ld(P + ri + s * nc)); }
  double g[4];
  bc_face_geom(b, Im, Jm, Km, Fm, g);
  R nx = cvt<R>(g[0]), ny = cvt<R>(g[1]), nz = cvt<R>(g[2]), area = cvt<R>(g[3]);
  const int code = (int)ld(q + 8);
  R BC_Mach = cvt<R>(ld(q + 0));
  R pamb = (R)-2.71;  // PAMB_FORCE_SUPERSONIC
  if (code == 401) { BC_Mach = (R)0; pamb = (R)-3.14; }
  else if (code == 403) { BC_Mach = (R)-10; pamb = (R)-3.14; }
  else if (code == 404) { BC_Mach = (R)-1; pamb = (R)-3.14; }
  else if (code == 407) { BC_Mach = (R)0; pamb = cvt<R>(ld(q + 9)); }
  const R BC_T0 = cvt<R>(ld(q + 1)), BC_p0 = cvt<R>(ld(q + 2)), rel = cvt<R>(ld(q + 3));
  const R BC_Sign = (R)modfm2;
  R Un = P2[MB_IU] * nx + P2[MB_IV] * ny + P2[MB_IW] * nz;
  R Brho, BRgas;
  rotot_rtot(p, P2[0], Brho, BRgas);
  R BSound = f_ss(p, P2[0], P2[MB_IPR], Brho, BRgas);
  R Tb = P2[MB_IPR] / (Brho * BRgas);
  int tiB = tidx(p, Tb);
  R cpB = f_cp(p, P2[0], tiB, Tb - (R)tiB, Brho);
  R BGamma = cpB / (cpB - BRgas);
  R Riem = BSound + BC_Sign * (R)0.5 * (BGamma - (R)1) * Un;
  R InOut = BC_Sign * Un;
  if (BC_Mach < (R)0) InOut = (R)-1;
  const R nrm[3] = {nx, ny, nz};
  if (InOut >= (R)0) {
    if (pamb == (R)-3.14 || pamb == (R)-2.71) {  // an inlet: the face closes
      bc_sym_eul<R, RS, LIM>(p, b, P, Im, Jm, Km, Fm, A);
      return;
    }
    R Fo[MB_NP];
    outflow_face<R>(p, P2, Brho, BRgas, BSound, Un, BGamma, Riem, nrm, area, pamb, BC_Sign, Fo);
#pragma unroll
    for (int s = 0; s < MB_NP; ++s) A[s] = (R)modfm2 * Fo[s];
    return;
  }
  if (!(BC_Mach > (R)1 || pamb == (R)-2.71)) {
    R Fo[MB_NP];
#pragma unroll
    for (int s = 0; s < MB_NP; ++s) Fo[s] = (R)0;
    if (BC_Mach < (R)1) {
      const R tv[3] = {cvt<R>(ld(q + 12)), cvt<R>(ld(q + 13)), cvt<R>(ld(q + 14))};
      subsonic_inflow_face<R>(p, P2, Un, BSound, BGamma, Riem, cvt<R>(ld(q + 10)), cvt<R>(ld(q + 11)), BC_Mach, BC_T0,
                              BC_p0, rel, BC_Sign, tv, nrm, area, Fo);
    }
#pragma unroll
    for (int s = 0; s < MB_NP; ++s) A[s] = (R)modfm2 * Fo[s];
    return;
  }
  R frho, fR;
  rotot_rtot(p, P2[0], frho, fR);
  R vmag2 = P2[MB_IU] * P2[MB_IU] + P2[MB_IV] * P2[MB_IV] + P2[MB_IW] * P2[MB_IW];
  R fS = f_ss(p, P2[0], P2[MB_IPR], P2[0], fR);
  R fM = rsqrt_(vmag2) / fS;
  R Mach_l = rel * BC_Mach + ((R)1 - rel) * fM;
  R p0_l = rel * BC_p0 + ((R)1 - rel) * P2[MB_IPR];
  R Sup[MB_NP];
  Sup[MB_IPR] = p0_l;
  R Sup_Rgas = (R)0 + (R)1 * (R)p.ri;
  R Sup_rho = Sup[MB_IPR] / (Sup_Rgas * BC_T0);
  Sup[0] = Sup_rho * (R)1;
  R Sup_Sound = f_ss(p, Sup[0], Sup[MB_IPR], Sup_rho, Sup_Rgas);
  const R ca = cvt<R>(ld(q + 4)), sa = cvt<R>(ld(q + 5)), cb = cvt<R>(ld(q + 6)), sb = cvt<R>(ld(q + 7));
  Sup[MB_IU] = Mach_l * Sup_Sound * ca * cb;
  Sup[MB_IV] = Mach_l * Sup_Sound * sa * cb;
  Sup[MB_IW] = Mach_l * Sup_Sound * sb;
  const R fm = (R)modfm, fm1 = (R)modfm1;
  R PL[MB_NP], PR[MB_NP];
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) {
    R p1 = fm * Sup[s] + fm1 * Ip[s];
    R p3 = fm * Ip[s] + fm1 * Sup[s];
    R Slope = rlimiter(lim, p3 - P2[s], P2[s] - p1);
    R Face = P2[s] + (R)0.5 * Slope * (R)modfm2;
    PL[s] = fm * Sup[s] + fm1 * Face;
    PR[s] = fm * Face + fm1 * Sup[s];
  }
  R rL, RL, rR, RRr;
  rotot_rtot(p, PL[0], rL, RL);
  R aL = f_ss(p, PL[0], PL[MB_IPR], rL, RL);
  rotot_rtot(p, PR[0], rR, RRr);
  R aR = f_ss(p, PR[0], PR[MB_IPR], rR, RRr);
  R F_r, F_u, F_v, F_w, F_E;
  // Ur = a on both sides: no preconditioning at the inlet (Lib_BC.f90:1308-1310)
  riemann_rec<R, RS>(p, PL[0], PL[MB_IU], PL[MB_IV], PL[MB_IW], PL[MB_IPR], aL, rL, RL, PR[0], PR[MB_IU], PR[MB_IV],
                     PR[MB_IW], PR[MB_IPR], aR, rR, RRr, nx, ny, nz, F_r, F_u, F_v, F_w, F_E, (R)1, aL, aR);
  R su = copysign((R)1, F_r);
  R selL = ((R)1 + su) / (R)2, selR = (su - (R)1) / (R)2;
  R Fmass = F_r * area;
  R Fl[MB_NP];
  Fl[0] = Fmass * (selL * PL[0] / rL - selR * PR[0] / rR);
  Fl[MB_IU] = F_u * area; Fl[MB_IV] = F_v * area; Fl[MB_IW] = F_w * area; Fl[MB_IPR] = F_E * area;
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) A[s] = (R)modfm2 * Fl[s];
}


// BC_Outlet (Lib_BC.f90:1604-1658) of a 406 record (q = exit pressure, relaxation factor): inward flow closes the face
// (BC_Symmetry_Eul); otherwise the face state of BC_Outflow (Lib_BC.f90:1166-1240) from the Riemann invariant towards
// the face and the relaxed exit pressure (isentropic when the normal Mach number is below 1 and p_exit > 0).
template <typename R, int RS = 0, int LIM = 0>
MB_HD void bc_outlet(const Params& p, const DBlk& b, const double* __restrict__ P, int Im, int Jm, int Km, int Fm,
                     const double* __restrict__ q, R* A) {
  const long long nc = p.nc;
  const int modfm = Fm % 2, modfm2 = 1 - 2 * modfm;
  const long long rb = row(b, Im, Jm, Km);
  R Bp[MB_NP];
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) Bp[s] = cvt<R>(ld(P + rb + s * nc));
  double g[4];
  bc_face_geom(b, Im, Jm, Km, Fm, g);
  const R nrm[3] = {cvt<R>(g[0]), cvt<R>(g[1]), cvt<R>(g[2])};
  const R area = cvt<R>(g[3]);
  const R pExit = cvt<R>(ld(q + 0)), rel = cvt<R>(ld(q + 1));
  const R BC_Sign = (R)modfm2;
  R Un = Bp[MB_IU] * nrm[0] + Bp[MB_IV] * nrm[1] + Bp[MB_IW] * nrm[2];
  if (BC_Sign * Un < (R)0) {
    bc_sym_eul<R, RS, LIM>(p, b, P, Im, Jm, Km, Fm, A);
    return;
  }
  R Brho, BRgas;
  rotot_rtot(p, Bp[0], Brho, BRgas);
  R BSound = f_ss(p, Bp[0], Bp[MB_IPR], Brho, BRgas);
  R T = Bp[MB_IPR] / (Brho * BRgas);
  int ti = tidx(p, T);
  R Tdiff = T - (R)ti;
  R cp = f_cp(p, Bp[0], ti, Tdiff, Brho);
  R BGamma = cp / (cp - BRgas);
  R Riem = BSound + BC_Sign * (R)0.5 * (BGamma - (R)1) * Un;
  R p_Amb = rel * pExit + ((R)1 - rel) * Bp[MB_IPR];
  R Fl[MB_NP];
  outflow_face<R>(p, Bp, Brho, BRgas, BSound, Un, BGamma, Riem, nrm, area, p_Amb, BC_Sign, Fl);
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) A[s] = (R)modfm2 * Fl[s];
}

// The record (type, id) of the cell (i,j,k) on face F, -1 if none.
MB_HD int record_of(const Params& p, const DBlk& b, int F, int i, int j, int k) {
  if (b.rmap[F - 1] < 0) return -1;
  const int ax = (F - 1) >> 1;
  const int t = (ax == 0) ? (j - 1) + (k - 1) * b.n2 : (ax == 1 ? (i - 1) + (k - 1) * b.n1 : (i - 1) + (j - 1) * b.n1);
  return p.rec_map[b.rmap[F - 1] + t];
}

// One boundary record (bc_record_apply.inc): its contributions to the cell's R row, in the flux type. A is added
// and then, in Navier-Stokes, S is subtracted (the order of the reference's statements); components a record leaves
// alone hold exact no-ops (-0 in A, +0 in S).
template <typename R, bool VISC, int RS = 0, int LIM = 0>
MB_HD void bc_record(const Params& p, const DBlk& b, const double* __restrict__ P, int rid, int i, int j, int k, int F,
                     R* A, R* S) {
  const DRec& rc = p.rec[rid];
  if (VISC)
    for (int s = 0; s < MB_NP; ++s) S[s] = (R)0;
  if (rc.type == 1) {
    bc_conn_eul<R, RS, LIM>(p, b, P, i, j, k, F, A);
    if (VISC) bc_conn_visc<R>(p, b, P, i, j, k, F, p.pgsrc + (long long)rc.pg * 6, S);
  } else if (rc.type == 11) {
    bc_extrap<R>(p, b, P, i, j, k, F, A);
  } else if (rc.type == 5) {
    bc_sym_eul<R, RS, LIM>(p, b, P, i, j, k, F, A);
    if (VISC) bc_wall_heat<R>(p, b, P, i, j, k, F, S);
  } else if (rc.type == 4) {
    bc_inflow<R, RS, LIM>(p, b, P, i, j, k, F, rc.q, A);
  } else if (rc.type == 3) {
    bc_sym_eul<R, RS, LIM>(p, b, P, i, j, k, F, A);
    if (VISC) bc_sym_visc<R>(p, b, P, i, j, k, F, S);
  } else if (rc.type == 6) {
    bc_sym_eul<R, RS, LIM>(p, b, P, i, j, k, F, A);
    if (VISC) bc_wall_temp<R>(p, b, P, i, j, k, F, rc.q[0], S);
  } else if (rc.type == 24) {
    bc_outlet<R, RS, LIM>(p, b, P, i, j, k, F, rc.q, A);
  } else {
    for (int s = 0; s < MB_NP; ++s) A[s] = (R)-0.0;
  }
}

// Every boundary record of the mesh, one thread each, from the stage input P (ghosts filled): the contributions
// (A, S) of record q go to recflux[q][0..9] in the flux type; the sweep adds them in face order after the interior
// sum (BC_Fluxes after Fluxes, Mod_Explicit.f90:187-189).
// VAR tells apart the instantiations of the same types built with different flags (the FP64 production form's units)
template <typename R, bool VISC, int RS, int LIM, int VAR = 0>
__global__ void __launch_bounds__(128) k_records(Params p, const int* __restrict__ brec, const int* __restrict__ bcell,
                                               int nrec, const double* __restrict__ P) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nrec) return;
  const int rid = brec[q];
  const int* c = bcell + 5 * q;  // blk, i, j, k, face
  const DBlk b = p.blk[c[0]];
  if (p.st[b.grp].done) return;
  R v[2 * MB_NP];
  bc_record<R, VISC, RS, LIM>(p, b, P, rid, c[1], c[2], c[3], c[4], v, v + MB_NP);
  R* out = reinterpret_cast<R*>(p.recflux) + (long long)rid * 2 * MB_NP;
#pragma unroll
  for (int s = 0; s < 2 * MB_NP; ++s) out[s] = (VISC || s < MB_NP) ? v[s] : (R)0;
}

// adds the record contributions of slot v (A = v[0..4], S = v[5..9]) into acc
template <typename R, bool VISC>
MB_HD void bc_apply(const R* v, double* acc) {
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) acc[s] = acc[s] + (double)v[s];
  if (VISC) {
#pragma unroll
    for (int s = 0; s < MB_NP; ++s) acc[s] = acc[s] - (double)v[MB_NP + s];
  }
}

// ---------------------------------------------------------------------------------------------
// The conservative state update of one cell (newstate_cons_body.inc), FP64. Returns the new
// primitive state in pn.
// RK4 (n_rk = 4, no reference): weight C of rl in the new state from Un (stages 1-3: 1/2, 1/2, 1) and weight W
// of rl in the accumulator a4 (stage 1: a4 = Un + rl/6; 2-3: a4 += rl/3; 4: new state = a4 + rl/6), rl = -R/vol*dt

MB_HD void cons_update(const Params& p, const double* pc, const double* po, const double* res,
                                            double vol, double dt, double rkc, double tc, double* pn,
                                            long long row_ = -1, bool prescaled = false) {
  const double strang = 1.0;
  double cons[MB_NP], cold[MB_NP], rl[MB_NP];
  auto prim2cons = [&](const double* q, double* u) {
    double rho = 0.0 + q[0];
    double Rg = 0.0 + p.ri * q[0] / rho;
    double vmag = 0.0;
#pragma unroll
    for (int s = MB_IU; s <= MB_IW; ++s) vmag = vmag + q[s] * q[s];
    double Tl = q[MB_IPR] / (Rg * rho);
    int ti = tidx(p, Tl);
    double Td = Tl - (double)ti;
    double hs = p.h[ti] + Td * (p.h[ti + 1] - p.h[ti]);
    double hmix = 0.0 + hs * q[0] / rho;
    double E0 = hmix - q[MB_IPR] / rho + 0.5 * vmag;
    u[0] = q[0];
#pragma unroll
    for (int s = MB_IU; s <= MB_IW; ++s) u[s] = rho * q[s];
    u[MB_IPR] = rho * E0;
  };
  prim2cons(po, cold);
  prim2cons(pc, cons);
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) rl[s] = prescaled ? res[s] : -res[s] / vol * dt * strang;  // IRS: prescaled
  if (p.n_rk != 4) {
#pragma unroll
    for (int s = 0; s < MB_NP; ++s) cons[s] = cold[s] + (cons[s] - cold[s] + rl[s]) * rkc;
  } else {
    double* a4 = p.acc4 + row_;
    const int q = p.irk - 1;
    const double W = (q == 0 || q == 3) ? 1.0 / 6.0 : 1.0 / 3.0;
    if (q < 3) {
      const double Cq = (q == 2) ? 1.0 : 0.5;
#pragma unroll
      for (int s = 0; s < MB_NP; ++s) {
        const double prev = (q == 0) ? cold[s] : a4[s * p.nc];
        a4[s * p.nc] = prev + rl[s] * W;
        cons[s] = cold[s] + rl[s] * Cq;
      }
    } else {
#pragma unroll
      for (int s = 0; s < MB_NP; ++s) cons[s] = a4[s * p.nc] + rl[s] * W;
    }
  }
  double rho = 0.0 + cons[0];
  double Rg = 0.0 + p.ri * cons[0] / rho;
  pn[0] = cons[0];
#pragma unroll
  for (int s = MB_IU; s <= MB_IW; ++s) pn[s] = cons[s] / rho;
  double vmag = 0.0;
#pragma unroll
  for (int s = MB_IU; s <= MB_IW; ++s) vmag = vmag + (cons[s] / rho) * (cons[s] / rho);
  double energy = cons[MB_IPR] / rho - 0.5 * vmag;
  double diff_en = 1e3, T_it = tc;
  int it = 1;
  while ((fabs(diff_en / energy) >= 1e-6) && (it <= 20)) {
    int ti = tidx(p, T_it);
    double Td = T_it - (double)ti;
    double cv = -Rg, enth = 0.0;
    double cps = p.cp[ti] + Td * (p.cp[ti + 1] - p.cp[ti]);
    double hs = p.h[ti] + Td * (p.h[ti + 1] - p.h[ti]);
    cv = cv + cons[0] / rho * cps;
    enth = enth + cons[0] / rho * hs;
    double p_it = rho * Rg * T_it;
    diff_en = fabs((enth - p_it / rho) - energy);
    T_it = T_it + (energy - (enth - p_it / rho)) / cv;
    it = it + 1;
  }
  pn[MB_IPR] = rho * Rg * T_it;
  if (pn[0] < 1e-20) pn[0] = 1e-20;
}

// Newstate_Primitive_blk (Lib_Newstate.f90:348-531), one species, FP64 in both forms: the conservative residual taken
// to the primitive variables by the inverse of the prim -> cons Jacobian (Theta = rho_p), then the RK stage on the
// primitive state, rho floored at 1e-20
MB_HD void prim_update(const Params& p, const double* pc, const double* po, const double* res, double vol, double dt,
                       double rkc, double* pn, double urc = 0.0) {
  const double strang = 1.0;
  double rho, Rgas;
  rotot_rtot(p, pc[0], rho, Rgas);
  const double temperature = pc[MB_IPR] / (rho * Rgas);
  const int T_i = tidx(p, temperature);
  const double Tdiff = temperature - (double)T_i;
  const double inv_rho = 1.0 / rho;
  const double vel[3] = {pc[MB_IU], pc[MB_IV], pc[MB_IW]};
  const double modvel = sqrt(vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
  const double q2 = modvel * modvel;
  const double cp = f_cp(p, pc[0], T_i, Tdiff, rho);
  const double rho_T = -rho / temperature;
  const double rho_p = 1.0 / (Rgas * temperature);
  const double enthalpy = H0(p, pc[MB_IPR], pc[0], modvel);
  double Theta = rho_p;
  if (p.prec) {  // Weiss-Smith: Theta from the cell's Ur (Lib_Newstate.f90:399-402)
    const double gam = cp / (cp - Rgas);
    const double sound = sqrt(gam * Rgas * temperature);
    const double a2 = sound * sound;
    const double beta2 = mx(urc * urc / a2, 1.0e-6);
    Theta = 1.0 / (beta2 * a2) + 1.0 / (cp * temperature);
  }
  const double Denom = 1.0 / (rho * cp * Theta + rho_T);
  double G[5][5];
  G[0][0] = (rho_T * (enthalpy - q2) + rho * cp) * Denom;
  G[0][1] = rho_T * vel[0] * Denom; G[0][2] = rho_T * vel[1] * Denom; G[0][3] = rho_T * vel[2] * Denom;
  G[0][4] = -rho_T * Denom;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    G[1 + a][0] = -vel[a] * inv_rho;
#pragma unroll
    for (int q = 1; q < 5; ++q) G[1 + a][q] = 0.0;
    G[1 + a][1 + a] = inv_rho;
  }
  G[4][0] = -(Theta * (enthalpy - q2) - 1.0) * Denom;
  G[4][1] = -vel[0] * Theta * Denom; G[4][2] = -vel[1] * Theta * Denom; G[4][3] = -vel[2] * Theta * Denom;
  G[4][4] = Theta * Denom;
  const double cres[5] = {-res[0], -res[MB_IU], -res[MB_IV], -res[MB_IW], -res[MB_IPR]};
  double pres[5];
#pragma unroll
  for (int r_ = 0; r_ < 5; ++r_) {
    pres[r_] = 0.0;
#pragma unroll
    for (int c_ = 0; c_ < 5; ++c_) pres[r_] = pres[r_] + G[r_][c_] * cres[c_];
  }
  double rl[MB_NP];
  rl[MB_IU] = pres[1]; rl[MB_IV] = pres[2]; rl[MB_IW] = pres[3];
  rl[MB_IPR] = pres[0];
  rl[0] = rho_p * pres[0] + rho_T * pres[4];
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) rl[s] = rl[s] * dt / vol * strang;
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) pn[s] = po[s] + (pc[s] - po[s] + rl[s]) * rkc;
  if (pn[0] < 1e-20) pn[0] = 1e-20;
}

// The state update of the mixed form: the arithmetic of cons_update, in FP64, with the single-species identities
// (rho = rho_s, R_mix = R, h_mix = h(T)) applied exactly and each division by rho, vol or R taken once as a
// reciprocal: p / rho = R T in the Newton iteration for T, its stop test |de| < 1e-6 |e| without a division. About
// 30 FP64 divisions fewer per cell; the rounding differs from the parity form's at the last bits.
MB_HD void cons_update_fast(const Params& p, const double* pc, const double* po, const double* res, double vol,
                            double dt, double rkc, double tc, double* pn, long long row_) {
  const double Rg = p.ri;
  double cons[MB_NP], cold[MB_NP], rl[MB_NP];
  auto prim2cons = [&](const double* q, double* u) {
    const double irho = 1.0 / q[0];
    const double vmag = q[MB_IU] * q[MB_IU] + q[MB_IV] * q[MB_IV] + q[MB_IW] * q[MB_IW];
    const double Tl = q[MB_IPR] * irho * p.iri;
    const int ti = tidx(p, Tl);
    const double Td = Tl - (double)ti;
    const double hs = p.h[ti] + Td * (p.h[ti + 1] - p.h[ti]);
    const double E0 = hs - q[MB_IPR] * irho + 0.5 * vmag;
    u[0] = q[0];
#pragma unroll
    for (int s = MB_IU; s <= MB_IW; ++s) u[s] = q[0] * q[s];
    u[MB_IPR] = q[0] * E0;
  };
  prim2cons(po, cold);
  prim2cons(pc, cons);
  const double f = dt / vol;
#pragma unroll
  for (int s = 0; s < MB_NP; ++s) rl[s] = -res[s] * f;
  if (p.n_rk != 4) {
#pragma unroll
    for (int s = 0; s < MB_NP; ++s) cons[s] = cold[s] + (cons[s] - cold[s] + rl[s]) * rkc;
  } else {
    double* a4 = p.acc4 + row_;
    const int q = p.irk - 1;
    const double W = (q == 0 || q == 3) ? 1.0 / 6.0 : 1.0 / 3.0;
    if (q < 3) {
      const double Cq = (q == 2) ? 1.0 : 0.5;
#pragma unroll
      for (int s = 0; s < MB_NP; ++s) {
        const double prev = (q == 0) ? cold[s] : a4[s * p.nc];
        a4[s * p.nc] = prev + rl[s] * W;
        cons[s] = cold[s] + rl[s] * Cq;
      }
    } else {
#pragma unroll
      for (int s = 0; s < MB_NP; ++s) cons[s] = a4[s * p.nc] + rl[s] * W;
    }
  }
  const double rho = cons[0], irho = 1.0 / rho;
  pn[0] = rho;
  double vmag = 0.0;
#pragma unroll
  for (int s = MB_IU; s <= MB_IW; ++s) {
    pn[s] = cons[s] * irho;
    vmag = vmag + pn[s] * pn[s];
  }
  const double energy = cons[MB_IPR] * irho - 0.5 * vmag;
  double diff_en = 1e3, T_it = tc;
  int it = 1;
  while ((fabs(diff_en) >= 1e-6 * fabs(energy)) && (it <= 20)) {
    const int ti = tidx(p, T_it);
    const double Td = T_it - (double)ti;
    const double cps = p.cp[ti] + Td * (p.cp[ti + 1] - p.cp[ti]);
    const double hs = p.h[ti] + Td * (p.h[ti + 1] - p.h[ti]);
    const double e_T = hs - Rg * T_it;
    diff_en = fabs(e_T - energy);
    T_it = T_it + (energy - e_T) / (cps - Rg);
    it = it + 1;
  }
  pn[MB_IPR] = rho * Rg * T_it;
  if (pn[0] < 1e-20) pn[0] = 1e-20;
}

// local dt of one cell (dt_blk.inc: min rule :156-191, additive rule :79-155) in the arithmetic type R: FP64 for the
// parity form and the standalone Compute_dt, FP32 (geometry and tables in FP32) for the fused dt of the mixed form.
// PREC: integration-variables = prec, the pseudo-acoustic speed c* = sqrt(alpha^2 u^2 + Ur^2) of the preconditioned
// system with the cell's Ur (urc) in place of the sound speed (dt_blk.inc:72-75, 89-92, 138-142)
template <typename R, bool PREC = false>
MB_HD R cell_dt_t(const Params& p, const DBlk& b, long long l, const R* pl, R urc = (R)0) {
  R rho, Rg;
  rotot_rtot(p, pl[0], rho, Rg);
  R Tc = pl[MB_IPR] / (rho * Rg);
  R Sound = f_ss(p, pl[0], pl[MB_IPR], rho, Rg);
  const auto* m = Geo<R>::m(b) + 9 * l;
  const auto* dl = Geo<R>::dl(b) + 3 * l;
  R dtc = (R)1e8;
  R Alpha_ = (R)0;
  if (PREC) {
    const R Beta_ = (R)1 / (Sound * Sound);
    Alpha_ = (R)0.5 * ((R)1 - Beta_ * (urc * urc));
  }
  if (p.dt_additive) {
    R ra_c = (R)0, ra_v = (R)0;
    for (int d = 0; d < b.ndir; ++d) {
      R m0 = cvt<R>(ld(m + d)), m1 = cvt<R>(ld(m + d + 3)), m2 = cvt<R>(ld(m + d + 6));
      R gn = rsqrt_(m0 * m0 + m1 * m1 + m2 * m2);
      R vel_ = fabs(pl[MB_IU] * m0 + pl[MB_IV] * m1 + pl[MB_IW] * m2) / gn;
      R lambda = vel_ + Sound;
      if (PREC) lambda = vel_ * ((R)1 - Alpha_) + rsqrt_(Alpha_ * Alpha_ * (vel_ * vel_) + urc * urc);
      ra_c = ra_c + lambda * gn;
      ra_v = ra_v + gn * gn;
    }
    if (p.visc) {
      if (b.ndir == 3) {
        R g[3][3];
        for (int d = 0; d < 3; ++d)
          for (int a = 0; a < 3; ++a) g[d][a] = cvt<R>(ld(m + d + 3 * a));
        auto dot = [&](int x, int y) { return g[x][0] * g[y][0] + g[x][1] * g[y][1] + g[x][2] * g[y][2]; };
        auto nr = [&](int x) { return rsqrt_(g[x][0] * g[x][0] + g[x][1] * g[x][1] + g[x][2] * g[x][2]); };
        R c12 = dot(0, 1) / (nr(0) * nr(1)), c13 = dot(0, 2) / (nr(0) * nr(2)), c23 = dot(1, 2) / (nr(1) * nr(2));
        R ss = c12 * c12 + c13 * c13 + c23 * c23;
        R qp = c12 * c13 * c23;
        if (ss + (R)2.0 * qp > (R)1.0) {
          R mr = (R)2.0 * rsqrt_(ss / (R)3.0) *
                 cos(acos(mx((R)-1.0, mn((R)1.0, (R)3.0 * rsqrt_((R)3.0) * qp / pow(ss, (R)1.5)))) / (R)3.0);
          ra_v = ra_v * (R)0.25 * ((R)2.0 + mr + (R)1.0 / mr);
        }
      }
      int ta = tidx(p, Tc);
      R tda = Tc - (R)ta;
      R cpa = f_cp(p, pl[0], ta, tda, rho);
      R cva = cpa - Rg;
      R mila, kla;
      wilke(p, pl[0], rho, ta, tda, mila, kla);
      if (p.prandtl > 0.0) kla = mila * cpa / (R)p.prandtl;
      const R mie = (R)0.0, prt = (R)0.85;
      R Dmx = mx((R)4.0 / (R)3.0 * (mila + mie) / rho, (kla + mie * cpa / prt) / (rho * cva));
      dtc = (R)1.0 / (ra_c / (R)p.cfl + Dmx * ra_v / (R)p.vnn);
    } else {
      dtc = (R)p.cfl / ra_c;
    }
  } else {
    for (int d = 0; d < b.ndir; ++d) {
      R m0 = cvt<R>(ld(m + d)), m1 = cvt<R>(ld(m + d + 3)), m2 = cvt<R>(ld(m + d + 6));
      R nrm = rsqrt_(m0 * m0 + m1 * m1 + m2 * m2);
      R v0 = m0 / nrm, v1 = m1 / nrm, v2 = m2 / nrm;
      R vel_ = fabs(pl[MB_IU] * v0 + pl[MB_IV] * v1 + pl[MB_IW] * v2);
      R lambda = vel_ + Sound;
      if (PREC) {
        const R cst_ = rsqrt_(Alpha_ * Alpha_ * (vel_ * vel_) + urc * urc);
        vel_ = vel_ * ((R)1 - Alpha_);
        lambda = vel_ + cst_;
      }
      R dtd = cvt<R>(ld(dl + d)) / lambda * (R)p.cfl;
      dtc = mn(dtd, dtc);
    }
    if (p.visc) {
      int ti = tidx(p, Tc);
      R td = Tc - (R)ti, mil, kl;
      wilke(p, pl[0], rho, ti, td, mil, kl);
      R mi = (R)0.0 + mil;
      for (int d = 0; d < b.ndir; ++d) {
        R dlv = cvt<R>(ld(dl + d));
        R dtd = (rho * (dlv * dlv) * (R)p.vnn) / mi;
        dtc = mn(dtd, dtc);
      }
    }
  }
  return dtc * (R)1.0;
}
MB_HD double cell_dt(const Params& p, const DBlk& b, long long l, const double* pl) {
  return cell_dt_t<double>(p, b, l, pl);
}

// the step of a cell in the state update: the case's dt, or with local time stepping (time-accurate = false) the
// cell's own dtlocal, from its state at the start of the step, times the step's ramp factor (dt_blk.inc: dtlocal =
// dtc * rampa_fac)
__device__ __forceinline__ double step_dt(const Params& p, const DBlk& b, const DevState* st, long long l,
                                          const double* po, double dt) {
  if (p.prec) return p.dtl[b.boff + l] * st->rampf;  // prec: the steps of the start of the step, with its Ur
  return p.local_dt ? cell_dt(p, b, l, po) * st->rampf : dt;
}

// min over the CTA of a positive double, then one atomic into the device clock
__device__ __forceinline__ void cta_min_dt(DevState* st, double v, double* sred) {
  const unsigned full = 0xffffffffu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = mn(v, __shfl_xor_sync(full, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) sred[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = (lane < nw) ? sred[lane] : 1e300;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = mn(v, __shfl_xor_sync(full, v, o));
    if (lane == 0 && v < 1e300) atomicMin(&st->dtmin_bits, (unsigned long long)__double_as_longlong(v));
  }
}

// ---- Compute_dt alone: the local dt of every interior cell in the form's arithmetic (FP64; FP32 for the mixed
// form, as its fused dt), reduced into the case's clock. only_group >= 0: the cells of that case only (its first
// dt after mb_group_reset). Tiles of 32 x TY_AUX cells (8 rows).
template <typename R, int VAR = 0>
__global__ void __launch_bounds__(256) k_dt_t(Params p, const DTile* __restrict__ tiles, const double* P,
                                             int only_group) {
  __shared__ double sred[32];
  const DTile t = tiles[blockIdx.x];
  const DBlk b = p.blk[t.blk];
  if (only_group >= 0 && b.grp != only_group) return;
  const int i = t.i0 + (threadIdx.x & 31), j = t.j0 + (threadIdx.x >> 5);
  double v = 1e300;
  if (i <= b.n1 && j <= b.n2) {
    for (int k = t.k0; k < t.k1; ++k) {
      const long long r = row(b, i, j, k);
      R pl[MB_NP];
      for (int s = 0; s < MB_NP; ++s) pl[s] = cvt<R>(P[r + s * p.nc]);
      v = mn(v, (double)cell_dt_t<R>(p, b, r - b.boff, pl));
    }
  }
  cta_min_dt(p.st + b.grp, v, sred);
}

__device__ __forceinline__ void report_bad_state(DevState* st, int blk, int i, int j, int k) {
  atomicAdd(&st->n_bad_state, 1);
  if (atomicCAS(&st->first_bad_claimed, 0, 1) == 0) {
    st->bad_blk = blk; st->bad_i = i; st->bad_j = j; st->bad_k = k;
  }
}

// ---------------------------------------------------------------------------------------------
// Stage plane kk of the tile window: cells (i0-2 .. i0+33) x (j0-2 .. j0+TY+1), those inside the padded block and
// within jext rows of the interior (jext < 2 for a block one cell deep in j: no j-faces, so only the viscous
// transverse stencil reads the ghost rows); the others hold zeros.
template <typename R, int TY, int NVT>
__device__ __forceinline__ void put_cell(const Params& p, const Tile<R, TY, NVT>& T, int o, R* vals) {
  R rho, Tc;
  cell_rho_T<R>(p, vals[0], vals[MB_IPR], rho, Tc);
  constexpr int VS = Tile<R, TY, NVT>::VS;
#pragma unroll
  for (int v = 0; v < 4; ++v) T.base[o + v * VS] = vals[v];
  if (NVT == 6) {
    T.base[o + 4 * VS] = vals[MB_IPR];
    T.base[o + 5 * VS] = Tc;
  } else {
    T.base[o + 4 * VS] = Tc;
  }
}

template <typename R, int TY, int NVT, bool KM>
__device__ __forceinline__ void stage_plane(const Params& p, const DBlk& b, const double* __restrict__ P,
                                            const Tile<R, TY, NVT>& T, int i0, int j0, int kk, int jext) {
  const int sl = slot_of<KM>(kk);
  const long long nc = p.nc;
  for (int c = threadIdx.x; c < TXH * (TY + 4); c += blockDim.x) {
    const int jj = c / TXH, ii = c - jj * TXH;
    const int i = i0 - 2 + ii, j = j0 - 2 + jj;
    const int o = T.off(sl, jj, ii);
    R vals[MB_NP] = {(R)0, (R)0, (R)0, (R)0, (R)0};
    if (i >= 1 - GC && i <= b.n1 + GC && j >= 1 - jext && j <= b.n2 + jext) {
      const long long r = row(b, i, j, kk);
#pragma unroll
      for (int s = 0; s < MB_NP; ++s) vals[s] = cvt<R>(ld(P + r + s * nc));
      put_cell<R, TY, NVT>(p, T, o, vals);
    } else {
#pragma unroll
      for (int v = 0; v < NVT; ++v) T.base[o + v * Tile<R, TY, NVT>::VS] = (R)0;
    }
  }
}

// ---- TMA staging of the mixed form (sm_100a). The state arena is a 2-D tensor of ncell_total rows x 5 variables
// (var-last, the reference's P_flat); one staged j-row of a plane is one box of 38 consecutive rows x 5 variables,
// its first row rounded down to an even row (the 16-byte rule of the innermost coordinate), so the 36 cells of the
// row sit at offset (row & 1). The TY+4 boxes of a plane land in the raw buffer ([jj][var][38] FP64, one 1536-byte
// slot per j-row) and complete one phase of a shared-memory mbarrier; stage_plane_raw then converts them to the tile.
constexpr int TMA_BOX_ROWS = 38;
constexpr int TMA_ROW_BYTES = 1536;                  // 5 x 38 x 8 = 1520, padded to a multiple of 128
constexpr unsigned TMA_WAIT_LIMIT = 1u << 22;        // try_wait rounds before a wait gives up (seconds)

__device__ __forceinline__ unsigned smem_addr(const void* q) { return (unsigned)__cvta_generic_to_shared(q); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_test(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred q;\n mbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n selp.u32 %0, 1, 0, q;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait of every thread for the phase `parity` of bar; false if it gave up (the caller's threads then agree
// through a barrier and leave)
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  for (unsigned q = 0; q < TMA_WAIT_LIMIT; ++q)
    if (mbar_test(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int x, int y, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_addr(dst)), "l"(tmap), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// warp 0 issues the TY+4 row boxes of plane kk into raw (lane 0 arms the barrier first)
template <int TY>
__device__ __forceinline__ void tma_issue_plane(const Params& p, const DBlk& b, unsigned char* raw,
                                                unsigned long long* bar, int i0, int j0, int kk) {
  if (threadIdx.x >= 32) return;
  if (threadIdx.x == 0) mbar_expect(bar, (unsigned)((TY + 4) * MB_NP * TMA_BOX_ROWS * sizeof(double)));
  __syncwarp();
  const int jj = threadIdx.x;
  if (jj < TY + 4) {
    const long long r = row(b, i0 - 2, j0 - 2 + jj, kk);
    tma_load_2d(raw + jj * TMA_ROW_BYTES, p.tmap, (int)(r & ~1LL), 0, bar);
  }
}

// the TMA staging state of a CTA: the staging buffer of the landing plane, its mbarrier and the parity it is waited
// for next
struct TmaStage {
  unsigned char* halo;
  unsigned long long* bar_halo;
  unsigned ph_halo;
};

// convert the landed raw plane into the tile slot of plane kk (the same cells and values as stage_plane)
template <typename R, int TY, int NVT, bool KM>
__device__ __forceinline__ void stage_plane_raw(const Params& p, const DBlk& b, const unsigned char* raw,
                                                const Tile<R, TY, NVT>& T, int i0, int j0, int kk, int jext) {
  const int sl = slot_of<KM>(kk);
  for (int c = threadIdx.x; c < TXH * (TY + 4); c += blockDim.x) {
    const int jj = c / TXH, ii = c - jj * TXH;
    const int i = i0 - 2 + ii, j = j0 - 2 + jj;
    const int o = T.off(sl, jj, ii);
    R vals[MB_NP] = {(R)0, (R)0, (R)0, (R)0, (R)0};
    if (i >= 1 - GC && i <= b.n1 + GC && j >= 1 - jext && j <= b.n2 + jext) {
      const int sh = (int)(row(b, i0 - 2, j, kk) & 1);
      const double* src = reinterpret_cast<const double*>(raw + jj * TMA_ROW_BYTES) + sh + ii;
#pragma unroll
      for (int s = 0; s < MB_NP; ++s) vals[s] = cvt<R>(src[s * TMA_BOX_ROWS]);
      put_cell<R, TY, NVT>(p, T, o, vals);
    } else {
#pragma unroll
      for (int v = 0; v < NVT; ++v) T.base[o + v * Tile<R, TY, NVT>::VS] = (R)0;
    }
  }
}

// One tile of the fused stage (the body of k_sweep).
// With TMA staging (the mixed form, p.tmap set) raw is the staging buffer and bar its mbarrier, phase the parity the
// CTA waits for next; false: a bounded wait gave up (the clock's code is set to MB_E_TIMEOUT) and the CTA must stop.
template <typename R, int TY, bool VISC, int MODE, int RS, int LIM, bool KM, int STG>
__device__ __forceinline__ bool sweep_tile(const Params& p, const DTile t, const double* __restrict__ Pin,
                                           const double* Pold, double* Pout, double* Rout, double rkc, int last,
                                           unsigned char* smem_raw, double* sred, double* s_res, TmaStage& ts) {
  unsigned char* raw = ts.halo;
  unsigned long long* bar = ts.bar_halo;
  unsigned& phase = ts.ph_halo;
  constexpr int NF = VISC ? 2 * MB_NP : MB_NP;  // values a face task computes (convective, viscous)
  // values a face keeps in shared memory: both fluxes in the FP64 form (pass 2 sums them in the reference's
  // order); the net flux (convective - viscous) in the mixed form
  constexpr bool NET = VISC && Fast<R>::on;
  constexpr int NS = NET ? MB_NP : NF;
  typedef R RowI[33][NS];
  typedef R RowJ[32][NS];
  constexpr int NVT = Stg<R, STG>::nv;
  Tile<R, TY, NVT> T;
  T.base = reinterpret_cast<R*>(smem_raw);                                       // [4][NVT][TY+4][36]
  T.rg = (R)p.ri;
  unsigned char* fbase = smem_raw + sizeof(R) * tile_planes<KM>() * NVT * (TY + 4) * TXH;
  RowI* sFi = reinterpret_cast<RowI*>(fbase);                                     // [TY][33][NS]
  RowJ* sFj = reinterpret_cast<RowJ*>(fbase + sizeof(R) * TY * 33 * NS);          // [TY+1][32][NS]
  // the k-faces: the face above a cell is computed by the thread of that cell and is the face below it on the next
  // plane, so the mixed form carries both in that thread's registers (kup, kdn: no shared buffer, which leaves room
  // for the TMA staging buffer at 3 CTAs per SM); the FP64 forms keep them in shared memory (two planes)
  constexpr bool KREG = Stg<R, STG>::kreg;
  RowJ* sFk0 = reinterpret_cast<RowJ*>(fbase + sizeof(R) * (TY * 33 + (TY + 1) * 32) * NS);  // [2][TY][32][NS]
  R kup[NS], kdn[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) kup[q] = kdn[q] = (R)0;
  const DBlk b = p.blk[t.blk];
  DevState* st = p.st + b.grp;
  if (MODE == MODE_UPDATE && st->done) return true;  // the case has reached its stop time (uniform over the CTA)
  // TMA staging (uniform over the CTA; without a map the TMA form stages the same tile values by plain loads)
  const bool tma = Stg<R, STG>::tma && p.tmap != nullptr;
  const int tid = threadIdx.x;
  const int tx = tid & 31, ty = tid >> 5;
  const int i = t.i0 + tx, j = t.j0 + ty;
  const bool own = (i <= b.n1) && (j <= b.n2);
  const double dt = (MODE == MODE_UPDATE) ? st->dt : 0.0;
  double dtloc = 1e300;
  if (MODE == MODE_UPDATE && last && tid < 8 * MB_NP) s_res[tid] = 0.0;  // used after the prologue's barrier
  int kb = 0;  // buffer of the k-face above the current plane
  // ghost layers the stencils read: 2 along an axis with faces; for a block one cell deep along j or k (2-D,
  // 1-D) no face of that axis exists and only the viscous transverse gradient reads one ghost layer
  const bool sens = RS == 0 && p.sd;  // the shock sensor reads the six face neighbours of a cell
  const int jext = (b.n2 > 1) ? GC : ((VISC || sens) ? 1 : 0);
  const int kext = (b.n3 > 1) ? GC : (((VISC || sens) && !KM) ? 1 : 0);
  // a TMA wait that gave up: every thread learns it at the same barrier, the clock records it, the CTA stops
  auto gave_up = [&](bool ok) -> bool {
    if (!__syncthreads_or(!ok)) return false;
    if (tid == 0) atomicCAS(&st->code, 0, MB_E_TIMEOUT_DEV);
    return true;
  };
  // prologue: planes k0-2 .. k0+1, and the k-face below the first plane
  for (int kk = t.k0 - 2; kk <= t.k0 + 1; ++kk) {
    if (kk < 1 - kext || kk > b.n3 + kext) continue;
    if (tma) {
      tma_issue_plane<TY>(p, b, raw, bar, t.i0, t.j0, kk);
      const bool ok = mbar_wait(bar, phase);
      phase ^= 1u;
      if (gave_up(ok)) return false;
      stage_plane_raw<R, TY, NVT, KM>(p, b, raw, T, t.i0, t.j0, kk, jext);
      __syncthreads();  // the staging buffer is free again
    } else {
      stage_plane<R, TY, NVT, KM>(p, b, Pin, T, t.i0, t.j0, kk, jext);
    }
  }
  // the first plane of the loop in flight while the k-face below is computed
  if (tma && t.k0 + 2 <= b.n3 + kext) tma_issue_plane<TY>(p, b, raw, bar, t.i0, t.j0, t.k0 + 2);
  __syncthreads();
  if (own && t.k0 > 1) {
    R out[NF];
    face_flux<R, TY, VISC, RS, LIM, KM, NVT>(p, b, T, 2, i, j, t.k0 - 1, tx + 2, ty + 2, out);
    if (KREG) {
#pragma unroll
      for (int q = 0; q < NS; ++q) kdn[q] = NET ? out[q] - out[MB_NP + q] : out[q];
    } else {
      R* dst = &sFk0[(kb ^ 1) * TY + ty][tx][0];
#pragma unroll
      for (int q = 0; q < NS; ++q) dst[q] = NET ? out[q] - out[MB_NP + q] : out[q];
    }
  }
  for (int k = t.k0; k < t.k1; ++k) {
    // the slot of plane k-2 is free: its last readers, the faces of plane k-1, finished before the barrier that
    // preceded pass 2 of plane k-1; so a thread stages plane k+2 as soon as its own pass 2 of plane k-1 is done
    if (k + 2 <= b.n3 + kext) {
      if (tma) {
        const bool ok = mbar_wait(bar, phase);
        phase ^= 1u;
        if (gave_up(ok)) return false;
        stage_plane_raw<R, TY, NVT, KM>(p, b, raw, T, t.i0, t.j0, k + 2, jext);
      } else {
        stage_plane<R, TY, NVT, KM>(p, b, Pin, T, t.i0, t.j0, k + 2, jext);
      }
    }
    __syncthreads();  // plane k+2 staged, and every pass 2 of plane k-1 done (the flux buffers are free)
    // the next plane's boxes fly under this plane's faces and pass 2 (the staging buffer was read before the barrier)
    if (tma && k + 3 <= b.n3 + kext && k + 1 < t.k1) tma_issue_plane<TY>(p, b, raw, bar, t.i0, t.j0, k + 3);
    // ---- face tasks of this plane through one call site: 0 = i-face #tid, 1 = extra i-faces (last warp,
    // lanes < TY), 2 = j-face #tid, 3 = extra j-face row (warp 0), 4 = the k-face above
#pragma unroll 1
    for (int task = 0; task < 5; ++task) {
      int d = -1, fi = 0, fj = 0, ii = 0, jj = 0;
      R* dst = nullptr;
      if (task == 0 || task == 1) {
        int f;
        if (task == 0) f = tid;
        else { if (ty != TY - 1 || tx >= TY) continue; f = 32 * TY + tx; }
        const int rw = f / 33, cl = f - rw * 33;
        fi = t.i0 + cl - 1; fj = t.j0 + rw; ii = cl + 1; jj = rw + 2;
        if (fi >= 1 && fi <= b.n1 - 1 && fj <= b.n2) { d = 0; dst = &sFi[rw][cl][0]; }
      } else if (task == 2 || task == 3) {
        int f;
        if (task == 2) f = tid;
        else { if (ty != 0) continue; f = 32 * TY + tx; }
        const int rw = f >> 5, cl = f & 31;
        fi = t.i0 + cl; fj = t.j0 + rw - 1; ii = cl + 2; jj = rw + 1;
        if (fj >= 1 && fj <= b.n2 - 1 && fi <= b.n1) { d = 1; dst = &sFj[rw][cl][0]; }
      } else {
        if (!own || k >= b.n3) continue;
        fi = i; fj = j; ii = tx + 2; jj = ty + 2; d = 2; dst = KREG ? nullptr : &sFk0[kb * TY + ty][tx][0];
      }
      if (d < 0) continue;
      R out[NF];
      face_flux<R, TY, VISC, RS, LIM, KM, NVT>(p, b, T, d, fi, fj, k, ii, jj, out);
      if (KREG && task == 4) {
#pragma unroll
        for (int q = 0; q < NS; ++q) kup[q] = NET ? out[q] - out[MB_NP + q] : out[q];
      } else {
#pragma unroll
        for (int q = 0; q < NS; ++q) dst[q] = NET ? out[q] - out[MB_NP + q] : out[q];
      }
    }
    __syncthreads();
    // the residual diagnostic of the last stage: (new - old)^2 of this thread's cell, in the flux type (the warps'
    // partial sums in FP32 in the mixed form: the diagnostic to FP32 accuracy there)
    R rsq[MB_NP];
#pragma unroll
    for (int v = 0; v < MB_NP; ++v) rsq[v] = (R)0;
    if (own) {
      // ---- pass 2 (pass2_body.inc): convective i +,-, j +,-, k +,-, then viscous i -,+, j -,+, k -,+
      double acc[MB_NP];
      const R* fr = (i < b.n1) ? &sFi[ty][tx + 1][0] : nullptr;
      const R* fl = (i > 1) ? &sFi[ty][tx][0] : nullptr;
      const R* gr = (j < b.n2) ? &sFj[ty + 1][tx][0] : nullptr;
      const R* gl = (j > 1) ? &sFj[ty][tx][0] : nullptr;
      const bool hr_on = k < b.n3, hl_on = k > 1;
      const R* hr = (!KREG && hr_on) ? &sFk0[kb * TY + ty][tx][0] : nullptr;
      const R* hl = (!KREG && hl_on) ? &sFk0[(kb ^ 1) * TY + ty][tx][0] : nullptr;
      // the sum runs in the flux type (the FP64 form: FP64 in the reference's order; the mixed form: the six FP32
      // net face fluxes summed in FP32 and converted once), the boundary records and the update in FP64
#pragma unroll
      for (int s = 0; s < MB_NP; ++s) {
        R a = (R)0;
        if (fr) a = a + fr[s];
        if (fl) a = a - fl[s];
        if (gr) a = a + gr[s];
        if (gl) a = a - gl[s];
        if (KREG) {
          if (hr_on) a = a + kup[s];
          if (hl_on) a = a - kdn[s];
        } else {
          if (hr) a = a + hr[s];
          if (hl) a = a - hl[s];
        }
        if (VISC && !NET) {
          if (fr) a = a - fr[MB_NP + s];
          if (fl) a = a + fl[MB_NP + s];
          if (gr) a = a - gr[MB_NP + s];
          if (gl) a = a + gl[MB_NP + s];
          if (hr) a = a - hr[MB_NP + s];
          if (hl) a = a + hl[MB_NP + s];
        }
        acc[s] = (double)a;
      }
      // ---- boundary records of the cell, face order 1..6 (computed before the sweep by k_records)
      if (i == 1 || i == b.n1 || j == 1 || j == b.n2 || k == 1 || k == b.n3) {
        const R* rf = reinterpret_cast<const R*>(p.recflux);
        const int on = (i == 1) | (i == b.n1) << 1 | (j == 1) << 2 | (j == b.n2) << 3 | (k == 1) << 4 | (k == b.n3) << 5;
        constexpr int nF = KM ? 4 : 6;  // a mirrored block's k-face records follow below
#pragma unroll 1
        for (int F = 1; F <= nF; ++F) {
          if (!((on >> (F - 1)) & 1)) continue;
          const int rid = record_of(p, b, F, i, j, k);
          if (rid >= 0) bc_apply<R, VISC>(rf + (long long)rid * 2 * MB_NP, acc);
        }
        if (KM) {  // faces 5 and 6 of a mirrored block: the extrapolation records of every cell, computed here
          R A[MB_NP];
#pragma unroll 1
          for (int F = 5; F <= 6; ++F) {
            bc_extrap<R>(p, b, Pin, i, j, k, F, A);
#pragma unroll
            for (int s = 0; s < MB_NP; ++s) acc[s] = acc[s] + (double)A[s];
          }
        }
      }
      const long long r = row(b, i, j, k);
      if (MODE == MODE_RESIDUAL) {
#pragma unroll
        for (int s = 0; s < MB_NP; ++s) Rout[r + s * p.nc] = acc[s];
      } else {
        double pc[MB_NP], po[MB_NP], pn[MB_NP];
#pragma unroll
#pragma unroll
        for (int s = 0; s < MB_NP; ++s) { pc[s] = ld(Pin + r + s * p.nc); po[s] = Pold[r + s * p.nc]; }
        double rho, Tc;
        if (Fast<R>::on) Tc = pc[MB_IPR] / pc[0] * p.iri;  // one species: R_mix = R
        else cell_rho_T(p, pc[0], pc[MB_IPR], rho, Tc);
        if (p.guard && !(Tc > 1.0 && Tc < 9990.0)) {  // thermo guard (Mod_Thermo_Cache.f90:317-327)
          atomicAdd(&st->n_bad_thermo, 1);
          if (Tc != Tc) Tc = 300.0;
          Tc = mn(mx(Tc, 1.0), 9990.0);
        }
        const double vol = ld(b.vol + (r - b.boff));
        double dtc = dt;
        if (RS == 0 && p.prec) {
          dtc = ld(p.dtl + r) * st->rampf;  // the steps of the start of the step (Ur of that state)
        } else if (RS == 0 && p.local_dt) {  // the cell's own step in the flux type (FP64 in the parity form)
          R pr[MB_NP];
#pragma unroll
          for (int s = 0; s < MB_NP; ++s) pr[s] = cvt<R>(po[s]);
          dtc = (double)cell_dt_t<R>(p, b, r - b.boff, pr) * st->rampf;
        }
        if (RS == 0 && p.intvar) prim_update(p, pc, po, acc, vol, dtc, rkc, pn, p.prec ? ld(p.ur + r) : 0.0);
        else if (Fast<R>::on) cons_update_fast(p, pc, po, acc, vol, dtc, rkc, Tc, pn, r);
        else cons_update(p, pc, po, acc, vol, dtc, rkc, Tc, pn, r);
        bool bad = !(pn[MB_IPR] >= 0.0);
#pragma unroll
        for (int s = 0; s < MB_NP; ++s) bad = bad || !isfinite(pn[s]);
        if (bad) report_bad_state(st, t.blk, i, j, k);
#pragma unroll
        for (int s = 0; s < MB_NP; ++s) Pout[r + s * p.nc] = pn[s];
        if (last) {  // the new state's local dt, in the flux type (FP64 in the parity form)
#pragma unroll
          for (int v = 0; v < MB_NP; ++v) {
            const R dv = (R)(pn[v] - po[v]);
            rsq[v] = dv * dv;
          }
          R pr[MB_NP];
#pragma unroll
          for (int s = 0; s < MB_NP; ++s) pr[s] = cvt<R>(pn[s]);
          dtloc = mn(dtloc, (double)cell_dt_t<R>(p, b, r - b.boff, pr));
        }
      }
    }
    if (MODE == MODE_UPDATE && last) {  // uniform over the CTA: each warp adds its plane sums into its own slots
#pragma unroll
      for (int v = 0; v < MB_NP; ++v) {
        R x = rsq[v];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((tid & 31) == 0) s_res[8 * v + (tid >> 5)] += (double)x;
      }
    }
    kb ^= 1;
    if (KREG) {
#pragma unroll
      for (int q = 0; q < NS; ++q) kdn[q] = kup[q];
    }
  }
  if (MODE == MODE_UPDATE && last) {
    cta_min_dt(st, dtloc, sred);  // its barrier also orders the warps' sums before their reads below
    if (tid < MB_NP) {
      double x = 0.0;
      for (int w = 0; w < (TY < 8 ? TY : 8); ++w) x += s_res[8 * tid + w];
      atomicAdd(&st->res2[tid], x);
    }
  }
  return true;
}

// shared memory of the sweep: the state tile and the face-flux buffers (sweep_smem_core), and in the mixed form the
// TMA staging buffer of one plane (TY+4 row slots) with its 128-byte alignment slack. The tiles of mirrored one-plane
// blocks (KM) hold one plane and have no k faces (no k-face buffers): a quarter of the tile, more CTAs per SM
template <typename R, int TY, bool VISC, int STG = STG_PLAIN, bool KM = false>
MB_HD constexpr size_t sweep_smem_core() {
  return sizeof(R) * ((size_t)tile_planes<KM>() * Stg<R, STG>::nv * (TY + 4) * TXH +
                      (size_t)(TY * 33 + (TY + 1) * 32 + ((Stg<R, STG>::kreg || KM) ? 0 : 2 * TY * 32)) *
                          ((VISC && !Fast<R>::on) ? 2 * MB_NP : MB_NP));
}
template <typename R, int TY, bool VISC, int STG = STG_PLAIN, bool KM = false>
MB_HD constexpr size_t sweep_smem() {
  return sweep_smem_core<R, TY, VISC, STG, KM>() +
         (Stg<R, STG>::tma ? (size_t)128 + (size_t)(TY + 4) * TMA_ROW_BYTES : 0);
}

// The fused stage over a tile list (KM: the tiles of mirrored one-plane blocks, a separate instantiation so that
// the other blocks' code carries none of their special cases). p.queue == null: one CTA per tile (grid = ntiles).
// Otherwise a persistent
// work queue: a grid of about one wave of CTAs, each taking the next tile from the counter p.queue (zeroed
// before the launch) until the list is exhausted. MINB: resident CTAs per SM the register allocation must
// allow (launch bounds).
template <typename R, int TY, bool VISC, int MODE, int RS, int LIM, int MINB, bool KM = false, int VAR = 0,
          int STG = STG_PLAIN>
__global__ void __launch_bounds__(32 * TY, MINB)
k_sweep(Params p, const DTile* __restrict__ tiles, const double* __restrict__ Pin, const double* Pold, double* Pout,
        double* Rout, double rkc, int last) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sred[32];
  __shared__ double s_res[8 * MB_NP];  // per warp (at most 8) and variable: the tile's residual sums
  __shared__ int s_next;
  __shared__ __align__(8) unsigned long long s_bar;  // TMA staging: the mbarrier of the landing plane
  static_assert(TY <= 8, "one residual slot per warp");
  TmaStage ts{nullptr, &s_bar, 0u};
  if (Stg<R, STG>::tma) {  // the staging buffer after the tile and the flux buffers, 128-byte aligned
    unsigned char* q = smem_raw + sweep_smem_core<R, TY, VISC, STG, KM>();
    ts.halo = q + ((128u - (smem_addr(q) & 127u)) & 127u);
    if (p.tmap) {
      if (threadIdx.x == 0) mbar_init(&s_bar);
      // the map was written to device memory by a host copy: the lanes that issue copies order it into the
      // tensor-map proxy before their first use
      if (threadIdx.x < 32)
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(p.tmap) : "memory");
      __syncthreads();
    }
  }
  if (!p.queue) {
    sweep_tile<R, TY, VISC, MODE, RS, LIM, KM, STG>(p, tiles[blockIdx.x], Pin, Pold, Pout, Rout, rkc, last, smem_raw,
                                                     sred, s_res, ts);
    return;
  }
  for (;;) {
    if (threadIdx.x == 0) s_next = atomicAdd(p.queue, 1);
    __syncthreads();
    const int tix = s_next;
    if (tix >= p.ntiles_run) break;
    if (!sweep_tile<R, TY, VISC, MODE, RS, LIM, KM, STG>(p, tiles[tix], Pin, Pold, Pout, Rout, rkc, last, smem_raw,
                                                          sred, s_res, ts))
      break;
    __syncthreads();  // the tile's shared memory is free and s_next may be overwritten
  }
}

}  // namespace mb
