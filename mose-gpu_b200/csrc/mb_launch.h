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
  double* pg;             // [nconn][6][5]
};

constexpr int TY_F64 = 4;    // default tile rows of the FP64 sweep (4 or 8; MB_SWEEP_TY overrides)
constexpr int TY_F32 = 8;    // default tile rows of the mixed sweep
constexpr int TY_AUX = 8;    // tile rows of the per-cell kernels (dt, update)

cudaError_t sweep_f64(const Params& p, const DTile* tiles, int ntiles, int ty, int mode, const double* Pin,
                      const double* Pold, double* Pout, double* Rout, double rkc, int last, cudaStream_t s);
cudaError_t sweep_f32(const Params& p, const DTile* tiles, int ntiles, int ty, int mode, const double* Pin,
                      const double* Pold, double* Pout, double* Rout, double rkc, int last, cudaStream_t s);
// ghost fill; *nl receives the number of kernels launched
cudaError_t ghost_fill(const Params& p, const GhostLists& g, double* P, cudaStream_t s, int* nl);
cudaError_t dt_cells(const Params& p, const DTile* tiles, int ntiles, const double* P, cudaStream_t s);
cudaError_t update_cells(const Params& p, const DTile* tiles, int ntiles, double* P, const double* PO,
                         const double* R, double rkc, double dt, cudaStream_t s);
cudaError_t reset_dt(const Params& p, cudaStream_t s);
cudaError_t clock_step(const Params& p, int time_clip, double threshold, cudaStream_t s);
cudaError_t sweep_setup_f64();
cudaError_t sweep_setup_f32();

}  // namespace mb
