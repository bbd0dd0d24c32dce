/*
 * mose_b200.h -- C ABI of the B200 residual / stage-update engine for the multi-block structured
 * compressible Euler / Navier-Stokes solver MOSE-GPU.
 *
 * The reference drives one explicit Runge-Kutta step from Explicit_Step
 * (src/lib/numerics/time/explicit/Mod_Explicit.f90:52-397). Inside it, per stage, it calls
 *   Fill_Ghost_Cell        (Mod_Explicit.f90:173 -> bc/Lib_Extrapolation.f90:1370-1528)
 *   Refresh_Thermo_Cache   (Mod_Explicit.f90:179 -> physics/Mod_Thermo_Cache.f90:25-111)
 *   Fluxes                 (Mod_Explicit.f90:187 -> numerics/fluxes/Mod_Fluxes.f90:10-98)
 *   BC_Fluxes              (Mod_Explicit.f90:189 -> numerics/fluxes/bc/Mod_BC.f90:646-800)
 *   RK_Newstate            (Mod_Explicit.f90:262 -> explicit/Lib_Newstate.f90:77-143)
 * and once per step Compute_dt (Mod_Explicit.f90:123 -> numerics/time/Mod_dt.f90:15-243) and
 * Copy_State (Mod_Explicit.f90:157 -> gpu/MOSE_Field_m.f90:321-330).
 * The entry points below replace those calls. Every data pointer handed to an entry point that
 * launches work is a DEVICE pointer borrowed from the caller (the reference's OpenACC-resident
 * arrays, obtained with `host_data use_device`), in the reference's own layouts:
 *   P_flat, PO_flat, R_flat : (ncell_total, nprim) FP64, column-major, var-last, one padded block
 *                             after the other (gpu/MOSE_Field_m.f90:42-47,128-167); the row of the
 *                             interior or ghost cell (i,j,k) of block b (i,j,k 1-based, ghosts 1-gc..n+gc) is
 *                             boff(b) + (i+gc-1) + (j+gc-1)*pi + (k+gc-1)*pi*pj, 0-based,
 *                             pi = n1+2gc, pj = n2+2gc (MOSE_Field_m.f90:78-109).
 *   fm1/fm2/fm3             : face normal + area (4, 0:n1, n2, n3) etc. (Mod_Convective.f90:594-596)
 *   dl, m, vol              : dl_f(3, padded), m_f(3,3, padded), vol(padded) (Mod_Fluxes.f90:222-227,
 *                             Lib_Newstate.f90:266)
 * Host-side descriptions (blocks, boundary records, connections, thermo tables) are read once by
 * mb_init, which builds its own device tables from them (Setup_BC_Device, Mod_BC.f90:99-338).
 *
 * Error behaviour: the reference stops the process (`error stop`) on a bad scheme id, a
 * non-physical state or an off-table temperature (Lib_Newstate.f90:234-246,
 * Mod_Thermo_Cache.f90:509-536, Mod_Convective.f90:759-766). Here every call returns an int
 * status (MB_OK = 0, negative on error) and device code never traps; mb_get_status reports the
 * first bad cell so that a Fortran shim can print the reference's message and stop.
 */
#ifndef MOSE_B200_H
#define MOSE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* compile-time dimensions of the reference build for the configurations served here:
 * single-species air, laminar (nsc = 1, nrans = 0 -> nprim = 5), gc = 2
 * (src/lib/base/Global_m.f90:8,15,18; src/lib/CMakeLists.txt:64-72) */
#define MB_GC 2
#define MB_NSC 1
#define MB_NPRIM 5

/* status codes */
#define MB_OK 0
#define MB_E_ARG (-1)          /* bad argument (null pointer, size, index) */
#define MB_E_UNSUPPORTED (-2)  /* scheme id or boundary type not served (Convective_assert_scheme) */
#define MB_E_CUDA (-3)         /* a CUDA runtime call failed */
#define MB_E_STATE (-4)        /* state check: p < 0 or a non-finite primitive (State_Check_blk) */
#define MB_E_THERMO (-5)       /* thermo guard: T outside (1, 9990) K in a viscous run */
#define MB_E_BUDGET (-6)       /* serving: a case does not fit the HBM budget */
#define MB_E_TIMEOUT (-7)      /* a bounded device wait gave up */
#define MB_E_NOMEM (-8)        /* device allocation failed */
#define MB_E_NODEV (-9)        /* no CUDA device */

/* boundary record types after Setup_BC_Device (IO_BC_Open.f90:155-390 maps the bc.txt codes):
 * 1 = 1:1 / periodic connection (101, 201), 4 = inflow/outflow as bc.txt 405 sets it up (the supersonic
 * static-state inlet, pamb = PAMB_FORCE_SUPERSONIC, IO_BC_Open.f90:286-303: the supersonic closure
 * whatever the Mach, the face closed to a symmetry face on outward flow), 5 = adiabatic no-slip wall
 * (301 with q = 0), 11 = extrapolation (400), 3 = symmetry (300), 6 = no-slip wall at a prescribed temperature
 * (302; q[0] = T_wall), 24 = back-pressure outlet (406; q[0] = exit pressure, q[1] = relaxation factor) */
#define MB_BC_NONE 0 /* no boundary condition (bc.txt 0 / 100, IO_BC_Open.f90:155-156): the degenerate faces of a 1-D or
                        2-D mesh; zero-gradient ghosts and no face flux (Mod_BC.f90:55-59, Lib_Extrapolation.f90:692) */
#define MB_BC_CONNECTION 1
#define MB_BC_SYMMETRY 3
#define MB_BC_INFLOW 4
#define MB_BC_WALL 5
#define MB_BC_WALL_T 6
#define MB_BC_EXTRAPOLATION 11
#define MB_BC_OUTLET 24
#define MB_BC_NQ 12 /* parameters of a record (mb_bc.q) */

/* limiter ids = lim_dev (numerics/space/Lib_Limiters.f90:21-61) */
#define MB_LIM_MINMOD 1
#define MB_LIM_VANLEER 2
#define MB_LIM_VANALBADA 3
#define MB_LIM_MC 4
#define MB_LIM_SUPERBEE 5
#define MB_LIM_FIRST_ORDER 6
/* Riemann solver ids = rs_dev (numerics/fluxes/Lib_Riemann.f90:23-107) */
#define MB_RS_HLLC 1
#define MB_RS_HLLE 2
#define MB_RS_SLAU 3
#define MB_RS_AUSMP 4
#define MB_RS_AUSMPM 5
#define MB_RS_HLLEPP 6
#define MB_RS_HLLC_TRAMEL 7
#define MB_RS_LLF 8
#define MB_RS_SLAU2 9
#define MB_RS_HLLC_CHEN 10
#define MB_RS_EXACT 11
#define MB_RS_LMROE 12
#define MB_RS_MICZEKROE 13
#define MB_RS_HLLC_PC 14 /* with intvar = 2 (prec) only */

/* the sensor id in effect (sd_dev): 0 none, 1 Tramel, 2 Chen */
static inline int mb_effective_sensor(int riemann, int sensor) {
  if (sensor == 1 || sensor == 2) return sensor;
  if (sensor == 3) return 0;
  if (riemann == 6 || riemann == 7) return 1;
  if (riemann == 5 || riemann == 10) return 2;
  return 0;
}

#define MB_PREC_FP64 0
#define MB_PREC_MIXED 1 /* reconstruction + Riemann + viscous flux arithmetic in FP32; state,
                           RK accumulation, T/p recovery and dt in FP64 */
#define MB_PREC_FP64_FAST 2 /* the FP64 production form: every value FP64 as in MB_PREC_FP64, but the flux path of the
                               mixed form (single-species identities applied exactly, van Albada as one quotient, net
                               face fluxes, reciprocals in the state update) built with FMA contraction. It meets the
                               parity gates against the reference's statement order (1e-12 relative after one step,
                               1e-9 after many) without being bit-identical to it; MB_PREC_FP64 is the bit-parity form */

/* One block: interior extents, row offset in the arena, geometry (device pointers). */
typedef struct mb_block {
  int32_t n[3];      /* interior cells n1, n2, n3 (blk%dim) */
  int32_t group;     /* the independent case (time step, clock, status) the block belongs to: 0 .. ngroups-1;
                        -1: an external block, the local copy of a block another rank owns when the blocks are
                        partitioned over GPUs: its rows hold the donor cells the halo exchange writes (mb_unpack_rows),
                        the connection records of the local blocks may name it as donor, and nothing is computed on
                        it (no tiles, records, ghost fill, time step or status); it carries no records itself */
  int64_t boff;      /* 0-based first row of the padded block in P_flat (field_block_index_params) */
  const double* fm1; /* (4, 0:n1, n2, n3): nx, ny, nz, area of the i-faces */
  const double* fm2; /* (4, n1, 0:n2, n3) */
  const double* fm3; /* (4, n1, n2, 0:n3) */
  const double* dl;  /* dl_f(3, 1-gc:n1+gc, 1-gc:n2+gc, 1-gc:n3+gc) */
  const double* m;   /* m_f(3, 3, padded): m(d, a) = d xi_d / d x_a */
  const double* vol; /* vol(padded) */
} mb_block;

/* One boundary record (domain%bc_bi/bj/bk/bf/typ, Mod_BC.f90:400-437): the interior cell that
 * owns a boundary face, the face 1..6 (odd = low side), and its type. */
typedef struct mb_bc {
  int32_t blk;   /* 0-based block */
  int32_t i, j, k;
  int32_t face;  /* 1..6 */
  int32_t type;  /* MB_BC_* */
  int32_t conn;  /* type 1: index into mb_mesh.conn; -1 otherwise */
  int32_t pad0;
  double q[MB_BC_NQ]; /* type 4: q[0..5] = mach, T0, p0, alpha, beta (flow angles, radians), rel_fac (bc%mach, %T0,
                         %p0, %alpha, %beta, %rel_fac); q[6] = the bc.txt code of the closure, as IO_BC_Open.f90:229-307
                         maps it: 0 or 405 the static inlet (T0, p0 static; the supersonic closure at any Mach),
                         401 the stagnation inlet (T0, p0 total), 403 the mass-flux inlet with total T (p0 = the mass
                         flux), 404 the mass-flux inlet with static T (rel_fac 1), 407 the ambient boundary (stagnation
                         inlet inwards, outflow to q[7] = pamb outwards); q[8..10] = the unit tangent of the face (the
                         diagonal of its nodes, Mod_BC.f90:226-240; read by 401-404 and 407);
                         type 6: q[0] = T_wall; type 24: q[0] = exit pressure, q[1] = rel_fac; unused otherwise */
} mb_bc;

/* One connection (domain%conn_*, Lib_Extrapolation.f90:1023-1134): the donor face cell of a
 * type-1 record and the orientation of the two transverse axes (d11 d12 d21 d22 of bc.txt). */
typedef struct mb_conn {
  int32_t rec;               /* the receiving record (index into mb_mesh.rec) */
  int32_t bs, is, js, ks, fs; /* donor block (0-based), donor face cell (1-based), donor face 1..6 */
  int32_t d11, d12, d21, d22;
} mb_conn;

typedef struct mb_mesh {
  int32_t nblk;
  int32_t nrec;
  int32_t nconn;
  int32_t ngroups;       /* independent cases in the context (0 or 1: one case). Each case has its own dt (the
                            minimum over its own cells), clock, stop time and status, so a batch of cases advances
                            exactly as each case alone; mb_init reserves this many clocks for later
                            mb_reconfigure calls */
  int64_t ncell_total;   /* rows of P_flat */
  const mb_block* blk;   /* host array [nblk] (the geometry pointers in it are device pointers) */
  const mb_bc* rec;      /* host array [nrec], grouped per block and ordered by face within it. A block one cell
                            deep in k (n[2] = 1) with no record on faces 5 and 6 is taken as having extrapolation
                            (type 11) records on every cell of both (the reference's 2-D meshes): the results are
                            the same, with 2 n1 n2 records fewer; its k ghost rows are then never filled (nothing
                            reads them) */
  const mb_conn* conn;   /* host array [nconn] */
} mb_mesh;

/* Single-species thermo and transport tables on the reference's 1 K grid
 * (lib/FLINT/src/lib/Load_ThermoTransport.f90:82-97,173-188): rows tmin..tmax of h, cp, mu, k
 * (host pointers; copied to the device by mb_init). */
typedef struct mb_thermo {
  int32_t tmin, tmax;
  double wm;          /* molar mass [kg/kmol]; R = Runiv / wm */
  const double* cp;
  const double* h;
  const double* mu;
  const double* k;
} mb_thermo;

typedef struct mb_scheme {
  int32_t limiter;    /* lim_dev */
  int32_t riemann;    /* rs_dev */
  int32_t visc;       /* 0 Euler, 1 laminar Navier-Stokes */
  int32_t n_rk;       /* 1 euler, 2 RK2, 3 SSP-RK3 (Lib_RK.f90:6-9); 4 classical RK4 (no reference: the
                         reference's two-register update cannot express it; the engine keeps a conserved
                         accumulator, U1 = Un + dt/2 k1, U2 = Un + dt/2 k2, U3 = Un + dt k3,
                         Un+1 = Un + dt/6 (k1 + 2 k2 + 2 k3 + k4)) */
  int32_t precision;  /* MB_PREC_* */
  int32_t ndir;       /* computational directions (Lib_Metrics.f90:152-172) */
  int32_t time_clip;  /* clip the last step onto time_threshold (Mod_dt.f90:283-296) */
  int32_t state_check;/* [MOSE-scheme] state-check (Lib_Newstate.f90:14) */
  int32_t dt_additive;/* dt-rule = additive (dt_blk.inc:79-155; 3-D): the convective and diffusive rates of
                         the three directions add up; 0 = the default min rule (dt_blk.inc:156-191) */
  int32_t sensor;     /* [MOSE-scheme] shock-detector (Assign_SD, Lib_Shock_Detector.f90:22-46): 0 the solver's own
                         (Tramel for HLLE++ / HLLC+Tramel, Chen for AUSM+M / HLLC+Chen, none otherwise), 1 Tramel,
                         2 Chen, 3 none. A limiter name with the SD suffix is the Tramel sensor. With a sensor the
                         cell's beta scales the reconstruction slopes of its faces and goes to their Riemann solver */
  int32_t intvar;     /* integration-variables (Assign_Integration_Variables, Lib_Newstate.f90:43-60): 0 cons
                         (Newstate_Conservative), 1 prim (Newstate_Primitive: the residual taken to the primitive
                         variables through the inverse of the prim -> cons Jacobian, Lib_Newstate.f90:348-531; with
                         n_rk <= 3), 2 prec (the primitive update with the Weiss-Smith low-Mach preconditioning of
                         Lib_Preconditioning.f90: the reference velocity Ur of every cell sets Theta, the local step
                         with the pseudo-acoustic speed and the HLLC-PC solver 14; steady runs only: local_dt = 1) */
  int32_t irs;        /* implicit residual smoothing (IRS = t of [MOSE-scheme], Lib_IRS.f90:57-105): the number of Jacobi
                         sweeps of R* = R + beta d2(R*) along each direction (the reference runs 2); 0 = off, at most
                         4, with n_rk <= 3. Conservative variables: the residual is scaled to -dt R / vol first and
                         the update takes it as it is; primitive variables: the raw residual is smoothed */
  double cfl;
  double vnn;         /* default 0.3 (MOSE_Types_m.f90:268) */
  double prandtl;     /* > 0: kl = mu cp / Pr (Mod_Diffusive.f90:303) */
  double schmidt;     /* laminar Schmidt (Lib_RANS.f90:25), 0.7 */
  double mco;         /* riemann-options-Mco (LMRoe low-Mach floor; 1 = plain Roe) */
  double time_threshold;
  double res_stop;    /* [MOSE-parameters] res-threshold (MOSE_Types_m.f90:247-250, default 1e-10 there): the case
                         stops once the residual diagnostic of rho (mb_status.res[0]) of a step is <= res_stop, as
                         Explicit_Step's end test (Mod_Explicit.f90:363-370); 0 = no residual stop */
  double irs_beta;    /* [MOSE-scheme] beta of the smoothing (Lib_IRS.f90:41-42, default 0.5), >= 0 */
  int32_t local_dt;   /* time-accurate = false (Mod_Explicit.f90:122-128): every cell advances with its own local step
                         (dtlocal of Compute_dt, taken from the state at the start of the step), the simulated time
                         does not advance (a steady run ends by res_stop or by the step count); 0 = time-accurate, the
                         global minimum step */
  int32_t cfl_rise;   /* [MOSE-parameters] cfl-rise-threshold (rampa_iter, Mod_dt.f90:57-58): the local steps are scaled
                         by iter / cfl_rise while the step count iter (1 for the first step of mb_init or
                         mb_group_reset) is below it; 0 = no ramp */
  int32_t prec_smooth;    /* integration-variables = prec (intvar 2): preconditioning-Ur-smooth, passes of max over the
                             six face neighbours (Lib_Preconditioning.f90:269-295) */
  int32_t pad2;
  double prec_eps_min;    /* preconditioning-eps-min, in (0, 1) (default 0.05) */
  double prec_uref;       /* preconditioning-Uref (> 0: mode 1, a uniform reference velocity) */
  double prec_mach;       /* preconditioning-Mach (> 0: mode 2, the target preconditioned Mach number) */
  double prec_ur_factor;  /* preconditioning-Ur-factor (mode 3, Weiss-Smith; default 1) */
  double prec_ur_min;     /* preconditioning-Ur-min (> 0: a floor of Ur) */
} mb_scheme;

typedef struct mb_status {
  int32_t code;        /* first error seen (MB_OK if none) */
  int32_t n_bad_state; /* cells that failed the state check */
  int32_t n_bad_thermo;/* cells that failed the thermo guard */
  int32_t bad_blk, bad_i, bad_j, bad_k; /* first offender */
  int32_t steps;       /* steps taken by mb_step since mb_init (or the case's mb_group_reset) */
  double time;         /* simulated time (sum of dt) */
  double dt;           /* dt of the last step */
  int32_t done;        /* the case reached its stop time (t_end) or residual (res_stop) and no longer advances */
  int32_t pad0;
  double res[5];       /* residual diagnostic of the last step taken by mb_step / mb_stage (Compute_Residual_blk,
                          Mod_Diagnostic.f90:64-104, as the L2 norm of Mod_Explicit.f90:325-358): sqrt of the sum
                          over the case's interior cells of (new - old)^2 of rho, u, v, w, p; in the mixed form the
                          partial sums of a warp are FP32 */
} mb_status;

/* The stop rule of one case of a batch (mb_group_reset): the reference's time loop stops at time >= timemax
 * (Mod_Explicit.f90:52-397) and Clip_dt_To_Timemax (Mod_dt.f90:283-296) clips the last step onto it. */
typedef struct mb_group {
  int32_t time_clip;  /* clip the last step onto t_end */
  int32_t pad0;
  double t_end;       /* the case stops advancing once its time reaches t_end (0: never) */
  double res_stop;    /* ... or once a step's residual of rho (mb_status.res[0]) is <= res_stop (0: never) */
} mb_group;

typedef struct mb_ctx mb_ctx;

/* Reads the mesh, scheme and tables, checks the scheme ids, builds the device tables (ghost
 * gather lists, record maps, tile lists) and the scratch state buffer. Replaces the device part of
 * MOSE_setup (Setup_BC_Device Mod_BC.f90:99, Setup_Device_Residency Mod_Explicit.f90:404-482,
 * cuf_init_tables Mod_Convective.f90:57-75). */
int mb_init(const mb_mesh* mesh, const mb_scheme* scheme, const mb_thermo* thermo, int device,
            mb_ctx** out);
void mb_destroy(mb_ctx* ctx);

/* Fill_Ghost_Cell on P (device pointer): physical ghosts, connection / periodic copies and the
 * transverse viscous stencil of the connection records (Lib_Extrapolation.f90:1370-1528). */
int mb_fill_ghosts(mb_ctx* ctx, double* P, void* stream);

/* Fluxes + BC_Fluxes: R = sum of the face fluxes of every interior cell, in the reference's order
 * (pass2_body.inc, then the boundary records face 1..6), from P whose ghosts are filled
 * (Mod_Fluxes.f90:10-98, Mod_BC.f90:646-800). The parity hook: nothing else is written. */
int mb_residual(mb_ctx* ctx, const double* P, double* R, void* stream);

/* RK_Newstate (conservative form) of stage irk (1-based) with residual R and time step dt:
 * P <- update(P, PO, R) at every interior cell (Lib_Newstate.f90:77-143, newstate_cons_body.inc).
 * With implicit residual smoothing (mb_scheme.irs > 0) the smoothing of IRS_apply runs first on a copy
 * of R in the engine's own buffers (Lib_IRS.f90:57-105); R itself is not written. */
int mb_update(mb_ctx* ctx, double* P, const double* PO, const double* R, int irk, double dt,
              void* stream);

/* Compute_dt: the global minimum local step of P (interior cells), written to *dt_host
 * (Mod_dt.f90:15-243, dt_blk.inc:11-222), with the cfl-rise factor of case 0's next step. Synchronises
 * the stream. With local time stepping (mb_scheme.local_dt) mb_update takes each cell's own step from PO
 * and ignores its dt argument. */
int mb_dt(mb_ctx* ctx, const double* P, double* dt_host, void* stream);

/* One fused stage: ghost fill of the stage input, then ONE sweep that computes every face flux once,
 * accumulates the divergence in registers and applies the RK update (and on the last stage the next
 * step's local dt). Stage input and output buffers are chosen by the engine so that, after the last
 * stage of a step, P holds the new state; PO is used as the engine's second buffer. */
int mb_stage(mb_ctx* ctx, double* P, double* PO, int irk, void* stream);

/* nsteps whole time steps on P (dt + stages), the dt kept on the device between steps; with
 * use_graph != 0 one step is captured once as a CUDA graph and replayed. */
int mb_step(mb_ctx* ctx, double* P, double* PO, int nsteps, int use_graph, void* stream);

/* Sets the step's dt on the device clock from the minimum of the local steps of P (Compute_dt +
 * Set_Global_dt + Clip_dt_To_Timemax), without a host read. Called before the first mb_stage. */
int mb_begin_step(mb_ctx* ctx, const double* P, void* stream);

/* Measurement hook: runs stage irk (ghost fill + boundary records + fused sweep, as mb_stage) nrep times on the
 * stream and returns the average device time of the surface work (ghost fill and boundary records) and of the
 * sweep kernel in milliseconds, each taken with CUDA events recorded around the launches on that stream.
 * Advances the state like mb_stage. */
int mb_profile_stage(mb_ctx* ctx, double* P, double* PO, int irk, int nrep, float* ms_ghost, float* ms_sweep,
                     void* stream);

/* ---- Blocks partitioned over several GPUs (one process and context per GPU; the reference's MPI decomposition by
 * blocks, src/lib/parallel/Mod_MPI.f90:147-258 and the halo exchange of Mod_GhostExchange.f90:217-383,685-957).
 * Each rank's mesh holds its own blocks and, as external blocks (group -1), copies of the remote donor blocks of its
 * connection records. A step is then
 *   mb_step_prepare -> MIN all-reduce of the clock's minimum local step (mb_copy_dtmin out, all-reduce, back in;
 *   mpi_allreduce_min_r8 of Mod_MPI.f90:571-581) -> mb_step_start -> per stage:
 *   halo rows of the donors' interior cells (mb_pack_rows on the owner, mb_unpack_rows into the external block)
 *   -> mb_stage_begin (ghost fill of the stage input) -> for Navier-Stokes, the donor rows the viscous connection
 *   records read, after the owners' own ghost fill -> mb_stage_end (records, sweep, update).
 * mb_begin_step = mb_step_prepare + mb_step_start and mb_stage = mb_stage_begin + mb_stage_end on one rank. */

/* Makes the minimum local step of P available in the case clocks (Compute_dt over this context's blocks; nothing
 * to do when the last stage of the previous step computed it). No host synchronisation. */
int mb_step_prepare(mb_ctx* ctx, const double* P, void* stream);

/* Copies case g's minimum local step between its clock and a caller device buffer of 8 bytes, ordered on `stream`:
 * to_clock = 0 clock -> buf, 1 buf -> clock. The value is the IEEE bit pattern of a positive double, so an integer
 * MIN all-reduce of the 64-bit patterns (signed or unsigned) is the MIN of the steps. */
int mb_copy_dtmin(mb_ctx* ctx, int g, void* buf, int to_clock, void* stream);

/* Starts the step on every case clock from the minimum in the clock (the ramp, the clip onto t_end, time and step
 * count, Set_Global_dt + Clip_dt_To_Timemax). */
int mb_step_start(mb_ctx* ctx, void* stream);

/* Stage irk split at the halo exchange point: mb_stage_begin fills the ghosts of the stage input (Fill_Ghost_Cell),
 * mb_stage_end computes the boundary records and runs the fused sweep and update. */
int mb_stage_begin(mb_ctx* ctx, double* P, double* PO, int irk, void* stream);
/* The device buffer stage irk reads (P, PO or the engine's own stage buffer: the engine rotates three buffers through
 * the stages): the buffer whose halo rows the exchange of that stage packs and unpacks. */
int mb_stage_input(mb_ctx* ctx, double* P, double* PO, int irk, double** in);
int mb_stage_end(mb_ctx* ctx, double* P, double* PO, int irk, void* stream);

/* Halo rows of a partitioned mesh: buf[v * n + q] = P[rows[q] + v * ncell] (pack) and its inverse (unpack), for the
 * five primitive variables v; rows (int64) and buf are device arrays. Ordered on `stream`; no context needed. */
int mb_pack_rows(const double* P, int64_t ncell, const int64_t* rows, int32_t n, double* buf, void* stream);
int mb_unpack_rows(double* P, int64_t ncell, const int64_t* rows, int32_t n, const double* buf, void* stream);

/* The same halo rows moved in one kernel from the owner's stage input into the receiver's, without a buffer or a
 * send / receive: dst[dst_rows[q] + v * ndst] = src[src_rows[q] + v * nsrc], launched on the owner's stream. dst is
 * the receiver's arena: on the same GPU, or on a peer GPU of the same node with peer access enabled (the stores
 * cross NVLink; a pointer from cudaIpcOpenMemHandle in a multi-process host). src_rows and dst_rows are device arrays
 * on the owner's GPU. The receiver's next launch must be ordered after this one (an event, or a barrier between the
 * processes). */
int mb_push_rows(const double* src, int64_t nsrc, const int64_t* src_rows, double* dst, int64_t ndst,
                 const int64_t* dst_rows, int32_t n, void* stream);

/* Lets kernels running on `device` store into `peer`'s memory (cudaDeviceEnablePeerAccess, once per ordered pair of
 * devices and process; already enabled is success, the same device is success): the precondition of mb_push_rows
 * into a peer GPU's arena from one process. MB_E_UNSUPPORTED where the two GPUs have no peer path. */
int mb_enable_peer(int device, int peer);

/* CUDA IPC of a stage buffer, for mb_push_rows between processes (one per GPU, or several on one GPU): mb_ipc_export
 * writes the 64-byte handle of the allocation that ptr lies in, ptr's byte offset inside it and the allocation's size
 * (a receiver checks that its arena fits); the owner's process maps it with mb_ipc_open (the base of the allocation,
 * on `device`; add the offset) and unmaps it with mb_ipc_close. A handle cannot be opened in the process that exported
 * it. */
int mb_ipc_export(const void* ptr, void* handle, int64_t* offset, int64_t* size);
int mb_ipc_open(const void* handle, int device, void** base);
int mb_ipc_close(void* base);

/* Status of case 0 (state check, thermo guard, first offender, simulated time, last dt). Synchronises. */
int mb_get_status(mb_ctx* ctx, mb_status* st);

/* Compute_dt of one block without allocating any device memory. No counterpart in the reference.
 * For callers that cannot allocate device memory when they need a time step: a Fortran host whose device
 * arrays belong to the OpenACC runtime, a serving loop already at its HBM budget, or code that must not
 * synchronise the device or is capturing a CUDA graph (cudaMalloc / cudaFree synchronise and are not
 * allowed during capture). Everything is caller-owned: P (the arena, ncell_total rows), the block's
 * padded dl and m, the FP64 cp, mu and k tables (rows tmin..tmax) on the device, the scheme (host
 * struct: cfl, vnn, prandtl, ndir, visc, dt_additive) and dt_out, one device double that receives
 * min(1e5, min over the block's interior cells of the local dt).
 * What it computes differs from mb_dt in two stated ways: the local dt is always the FP64 rule of the parity
 * form (mb_dt of a mixed-precision context takes it in FP32), and the cfl-rise ramp is NOT applied (during the
 * ramp, iteration iter < cfl_rise, the caller multiplies dt_out by iter / cfl_rise as mb_dt does).
 * integration-variables = prec (intvar 2) takes its steps from the context's Ur field: MB_E_UNSUPPORTED.
 * The only scratch is a file-scope device array of 65536 doubles (512 KB) of per-CTA partial minima, held by
 * every GPU that loads the library until exit; a block whose 32 x 8-cell (i, j) tiles exceed 65536 is rejected
 * with MB_E_ARG. The first call on a device looks up the array's device address (cudaGetSymbolAddress), so make
 * that first call before any stream capture (a first call on a capturing stream returns MB_E_ARG). Calls share
 * the array: calls that overlap on the GPU (different streams, no ordering between them) race and must not be
 * issued. */
int mb_dt_block_noalloc(const double* P, int64_t ncell_total, int64_t boff, const int32_t n[3], const double* dl,
                        const double* m, const double* cp, const double* mu, const double* k, int32_t tmin,
                        int32_t tmax, double wm, const mb_scheme* sc, double* dt_out, void* stream);

/* The launch shape mb_dt_block_noalloc uses for a block of n[3] interior cells, without launching anything (a
 * host-only query): the k chunk *kc (16 planes, doubled until one partial minimum per tile fits the 65536 of the
 * static array) and the tile count *ntiles = ceil(n1/32) ceil(n2/8) ceil(n3/kc). MB_E_ARG when even one plane
 * needs more than 65536 tiles. No counterpart in the reference. */
int mb_dt_block_noalloc_tiles(const int32_t n[3], int32_t* kc, int32_t* ntiles);

/* Batched cases (no counterpart in the reference, whose process runs one case): mb_init with
 * mesh->ngroups = G reserves G case clocks; the blocks of every case sit in one arena of ncell_total rows and
 * every fused stage is ONE sweep over the tiles of all of them, each case with its own dt. */

/* Replaces the blocks, records and connections of the context (cases admitted or retired) while keeping its
 * buffers, the state arena layout rules (ncell_total may not grow) and the clocks of the cases that stay.
 * Synchronises the device; invalidates the captured step graph. */
int mb_reconfigure(mb_ctx* ctx, const mb_mesh* mesh);

/* The same, ordered on `stream` (the stream every call of this context runs on) without synchronising the device:
 * the new tables are allocated and copied in stream order (the stream-ordered allocator) and the old ones released
 * after the work already queued on the stream, so other contexts (other serving lanes) keep running. Invalidates
 * the captured step graph (a replay in flight completes on the old tables). No counterpart in the reference. */
int mb_reconfigure_async(mb_ctx* ctx, const mb_mesh* mesh, void* stream);

/* Starts case g afresh: time 0, no steps, cleared status, its stop rule, and its first dt from the cells of P
 * that belong to it (the other cases' clocks are untouched). */
/* Replaces the parameters (mb_bc.q, same meaning as at mb_init) of record `rec` from the next stage on, ordered on
 * `stream`: a time-dependent boundary driven by the host, as the reference's 402 inlet interpolates p0(t) from its file
 * table each step (Mod_BC_Time.f90) and hands the value to the record. Validated as at mb_init. */
int mb_set_record_params(mb_ctx* ctx, int rec, const double* q, void* stream);
int mb_group_reset(mb_ctx* ctx, int g, const mb_group* spec, const double* P, void* stream);

/* Status of cases g0 .. g0+n-1 (one device read). Synchronises. */
int mb_get_group_status(mb_ctx* ctx, int g0, int n, mb_status* out);

/* The same, ordered on `stream` (the stream the context's steps run on): waits for that stream only, so that
 * several contexts on their own streams keep running. */
int mb_read_group_status(mb_ctx* ctx, int g0, int n, mb_status* out, void* stream);

/* The sweep's autotuner (no counterpart in the reference): times, on the state P and the current mesh, the
 * k-chunk of the tiles of 3-D blocks (8 / 16 / 32 / 64 planes) and a plain grid (one CTA per tile) against the
 * persistent work queue (one wave of CTAs taking the largest tiles first from a counter), and keeps the
 * fastest for every later sweep. Does not change P or the clocks; call between steps. */
int mb_autotune(mb_ctx* ctx, const double* P, void* stream);

/* Sets the sweep configuration by hand: the k-chunk of 3-D tiles and the persistent work queue (1) or the plain
 * grid (0). Synchronises; invalidates the captured step graph. */
int mb_set_tuning(mb_ctx* ctx, int kchunk, int persistent);

/* The configuration chosen by mb_autotune (k-chunk 16 and the plain grid before any call) and its sweep time. */
int mb_get_tuning(const mb_ctx* ctx, int* kchunk, int* persistent, float* ms);

/* The tile staging of the mixed form's sweep (no counterpart in the reference): tma = 1 (the default) stages each
 * plane of a tile by TMA, cp.async.bulk.tensor boxes of 38 rows x 5 variables of the state arena landing on an
 * mbarrier (bounded waits; a wait that gives up sets MB_E_TIMEOUT in the case status), converted into a 5-value
 * FP32 tile (rho, u, v, w, T; p = rho R T where it is read) with the k-face fluxes carried in registers; tma = 0
 * stages by per-thread coalesced loads into a 6-value tile (rho, u, v, w, p, T). The two differ in the FP32
 * rounding of p (within the mixed form's accuracy); mb_autotune keeps the faster for each tile list (this call sets
 * both lists: the blocks with several k planes, and the mirrored one-plane blocks). TMA is used where a tensor map of
 * the state buffer can be made: the buffer 16-byte aligned, ncell_total even, the map made outside any stream
 * capture (at the first mb_stage / mb_step / mb_residual / mb_autotune on that buffer), MB_NO_TMA unset at
 * mb_init. Invalidates the captured step graph when it changes the staging. */
int mb_set_staging(mb_ctx* ctx, int tma);

/* Failure-detection check of the staging's bounded waits (no counterpart in the reference): one CTA on `device` waits
 * for an mbarrier phase that nothing completes, with a limit of `tries` rounds of mbarrier.try_wait, and the kernel
 * returns; *gave_up = 1 when the wait ran out (as a sweep's would, which then sets MB_E_TIMEOUT in the case status
 * and stops), the device staying usable. Synchronises. */
int mb_selftest_bounded_wait(int device, int tries, int* gave_up);

/* The mixed form's sweep launches of this context so far by staging: *tma_sweeps by TMA, *plain_sweeps by plain
 * loads (launches recorded into a CUDA graph count once, at capture). */
int mb_get_staging(const mb_ctx* ctx, int64_t* tma_sweeps, int64_t* plain_sweeps);

/* The mixed sweep's configured staging (mb_set_staging, or mb_autotune's choice, which tunes the tile list of
 * mirrored one-plane blocks separately): *tma = 1 for the 5-value tile (staged by TMA where the state buffer has a
 * tensor map, by plain loads where it has none), 0 for the 6-value tile by plain loads; of the main tile list, or of
 * the one-plane list when the mesh has no other blocks. */
int mb_get_staging_mode(const mb_ctx* ctx, int* tma);

/* Number of kernel launches this context has issued (for launch accounting). */
int64_t mb_launch_count(const mb_ctx* ctx);

/* Version string of the built library. */
const char* mb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MOSE_B200_H */
