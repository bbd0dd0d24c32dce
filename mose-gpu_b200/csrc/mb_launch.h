// mb_launch.h -- launchers of the engine kernels, shared by the host API (mb_api.cu) and the two
// kernel translation units (mb_f64.cu: FP64 form, built without FMA contraction; mb_f32.cu: mixed
// form, FP32 flux arithmetic with FMA).
#pragma once
#include <cuda_runtime.h>
#include "mb_engine.cuh"

namespace mb {

// a boundary record as the ghost fill needs it
struct GRec {
  int blk, i, j, k, face, type;
};

// the ghost-fill work lists, built by mb_init (device pointers)
struct GhostLists {
  const GRec* rec;        // every record
  const int* phys;        // records with zero-gradient (types 4, 11) or wall-extrapolated (5) ghosts
  int nphys;
  const int* cubic;       // records of type 11 (cubic extrapolation ghost)
  int ncubic;
  const long long* cdst;  // connection ghost copies: row cdst[q] <- row csrc[q]
  const long long* csrc;
  int ncopy;
  const long long* pgsrc; // [nconn][6] source rows of bc_pg
  int nconn;
  // ordered != 0: the phys and cubic lists are split in two halves, off[0]..off[1] and off[1]..off[2], the second
  // holding the records whose opposite-face partner on the same column comes earlier in record order; each pass then
  // runs as two launches (only on blocks with an axis of at most two cells does the order change values)
  int ordered;
  int phys_off[3];
  int cubic_off[3];
};

constexpr int TY_F64 = 4;    // tile rows of the FP64 sweep (128 threads)
constexpr int TY_F32 = 8;    // tile rows of the mixed sweep (256 threads)
constexpr int MINB_F64 = 2;  // resident CTAs per SM the FP64 sweep's registers must allow
constexpr int MINB_F32 = 3;  // resident CTAs per SM the mixed sweep's registers must allow (80 registers)
constexpr int TY_AUX = 8;    // tile rows of the per-cell kernels (dt, update)

#define MB_CAT2(a, b) a##b
#define MB_CAT(a, b) MB_CAT2(a, b)

#define MB_DECLARE_SWEEP(name)                                                                                    \
  cudaError_t name(const Params& p, const DTile* tiles, int ntiles, int mode, const double* Pin, const double* Pold, \
                   double* Pout, double* Rout, double rkc, int last, int km, cudaStream_t s);                      \
  cudaError_t name##_setup();                                                                                    \
  cudaError_t name##_records(const Params& p, const int* brec, const int* bcell, int nrec, const double* P,      \
                             cudaStream_t s);                                                                    \
  cudaError_t name##_dt(const Params& p, const DTile* tiles, int ntiles, const double* P, int only_group,       \
                        cudaStream_t s);                                                                         \
  int name##_occupancy(int visc);                                                                            \
  int name##_occupancy_km(int visc);
MB_DECLARE_SWEEP(sweep_f64_rs1)
MB_DECLARE_SWEEP(sweep_f64_rs4)
MB_DECLARE_SWEEP(sweep_f64_rs12)
MB_DECLARE_SWEEP(sweep_f32_rs1)
MB_DECLARE_SWEEP(sweep_f32_rs4)
MB_DECLARE_SWEEP(sweep_f32_rs12)
MB_DECLARE_SWEEP(sweep_f64_rs0)
MB_DECLARE_SWEEP(sweep_f32_rs0)
// the FP64 production form: the simplified flux path in FP64, built with FMA contraction
MB_DECLARE_SWEEP(sweep_f64f_rs1)
MB_DECLARE_SWEEP(sweep_f64f_rs4)
MB_DECLARE_SWEEP(sweep_f64f_rs12)
MB_DECLARE_SWEEP(sweep_f64f_rs0)
// the sweep unit of a Riemann solver id: one unit per benchmarked solver (the id a compile-time constant there), the
// rs0 units (the id read at run time) for the others
// the unit of the scheme's precision form (MB_PREC_MIXED: f32, MB_PREC_FP64_FAST: f64f, MB_PREC_FP64: f64)
#define MB_BY_FORM(prec, rs, fn, args)                                                                     \
  ((prec) == MB_PREC_MIXED ? MB_BY_RS(f32, rs, fn, args)                                                  \
                           : (prec) == MB_PREC_FP64_FAST ? MB_BY_RS(f64f, rs, fn, args) : MB_BY_RS(f64, rs, fn, args))
#define MB_BY_RS(form, rs, fn, args)                                                                        \
  ((rs) == 1 ? sweep_##form##_rs1##fn args                                                                  \
             : (rs) == 4 ? sweep_##form##_rs4##fn args : (rs) == 12 ? sweep_##form##_rs12##fn args : sweep_##form##_rs0##fn args)

// ghost fill; *nl receives the number of kernels launched
cudaError_t ghost_fill(const Params& p, const GhostLists& g, double* P, cudaStream_t s, int* nl);
cudaError_t dt_cells(const Params& p, const DTile* tiles, int ntiles, const double* P, cudaStream_t s,
                     int only_group = -1);
cudaError_t update_cells(const Params& p, const DTile* tiles, int ntiles, double* P, const double* PO,
                         const double* R, double rkc, double dt, cudaStream_t s, int prescaled = 0);
cudaError_t reset_dt(const Params& p, cudaStream_t s, int only_group = -1);
// integration-variables = prec (mb_prec.cu): Ur of the interior cells of P with nsmooth smoothing passes (urb: the
// second buffer; *nl: kernels launched), and the local steps of P into dtl (reduce: their minimum into the clocks)
cudaError_t prec_ur(const Params& p, const DTile* tiles, int ntiles, const double* P, double* ur, double* urb,
                    int nsmooth, cudaStream_t s, int* nl);
cudaError_t prec_dt(const Params& p, const DTile* tiles, int ntiles, const double* P, double* dtl, int reduce,
                    cudaStream_t s);
// implicit residual smoothing (mb_irs.cu)
cudaError_t irs_scale(const Params& p, const DTile* tiles, int ntiles, double* R, double dt, const double* Pold,
                      cudaStream_t s);
cudaError_t irs_ghosts(const Params& p, const long long* dst, const long long* src, int n, double* R, cudaStream_t s);
cudaError_t irs_smooth(const Params& p, const DTile* tiles, int ntiles, const double* Rin, double* Rout, int d,
                       int njacobi, double beta, cudaStream_t s);
cudaError_t irs_stage_update(const Params& p, const DTile* tiles, int ntiles, const double* Pin, const double* Pold,
                             double* Pout, const double* R, double rkc, int last, cudaStream_t s);
cudaError_t to_float(const double* src, float* dst, long long n, cudaStream_t s);
// halo rows of a partitioned mesh: buf[v * n + q] <-> P[rows[q] + v * ncell] (mb_pack_rows / mb_unpack_rows)
cudaError_t pack_rows(const double* P, long long ncell, const long long* rows, int n, double* buf, cudaStream_t s);
cudaError_t unpack_rows(double* P, long long ncell, const long long* rows, int n, const double* buf, cudaStream_t s);
// dst[drows[q] + v * ndst] = src[srows[q] + v * nsrc] (mb_push_rows; dst may be a peer GPU's memory)
cudaError_t push_rows(const double* src, long long nsrc, const long long* srows, double* dst, long long ndst,
                      const long long* drows, int n, cudaStream_t s);
cudaError_t clock_step(const Params& p, cudaStream_t s);
// the TMA staging's bounded mbarrier wait, made to run out (mb_selftest_bounded_wait)
cudaError_t wait_selftest(unsigned tries, int* gave_up, cudaStream_t s);
cudaError_t group_reset(const Params& p, int g, int time_clip, double t_end, double res_stop, cudaStream_t s);

}  // namespace mb
