// mb_f32.cu -- the mixed form of the fused sweep: reconstruction, Riemann and viscous flux arithmetic
// in FP32 (with FMA), the residual accumulated and the state updated in FP64.
#include "mb_launch.h"

namespace mb {

template <int TY, bool VISC, int MODE>
static cudaError_t sweep_one(const Params& p, const DTile* tiles, int ntiles, const double* Pin, const double* Pold,
                             double* Pout, double* Rout, double rkc, int last, cudaStream_t s) {
  const size_t sm = sweep_smem<float, TY, VISC>();
  k_sweep<float, TY, VISC, MODE><<<ntiles, 32 * TY, sm, s>>>(p, tiles, Pin, Pold, Pout, Rout, rkc, last);
  return cudaGetLastError();
}

template <int TY, bool VISC, int MODE>
static cudaError_t set_attr() {
  return cudaFuncSetAttribute(k_sweep<float, TY, VISC, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sweep_smem<float, TY, VISC>());
}

cudaError_t sweep_setup_f32() {
  cudaError_t e;
  if ((e = set_attr<4, true, MODE_RESIDUAL>()) != cudaSuccess) return e;
  if ((e = set_attr<4, true, MODE_UPDATE>()) != cudaSuccess) return e;
  if ((e = set_attr<4, false, MODE_RESIDUAL>()) != cudaSuccess) return e;
  if ((e = set_attr<4, false, MODE_UPDATE>()) != cudaSuccess) return e;
  if ((e = set_attr<8, true, MODE_RESIDUAL>()) != cudaSuccess) return e;
  if ((e = set_attr<8, true, MODE_UPDATE>()) != cudaSuccess) return e;
  if ((e = set_attr<8, false, MODE_RESIDUAL>()) != cudaSuccess) return e;
  return set_attr<8, false, MODE_UPDATE>();
}

template <int TY>
static cudaError_t sweep_ty(const Params& p, const DTile* tiles, int ntiles, int mode, const double* Pin,
                            const double* Pold, double* Pout, double* Rout, double rkc, int last, cudaStream_t s) {
  if (p.visc) {
    if (mode == MODE_RESIDUAL) return sweep_one<TY, true, MODE_RESIDUAL>(p, tiles, ntiles, Pin, Pold, Pout, Rout, rkc, last, s);
    return sweep_one<TY, true, MODE_UPDATE>(p, tiles, ntiles, Pin, Pold, Pout, Rout, rkc, last, s);
  }
  if (mode == MODE_RESIDUAL) return sweep_one<TY, false, MODE_RESIDUAL>(p, tiles, ntiles, Pin, Pold, Pout, Rout, rkc, last, s);
  return sweep_one<TY, false, MODE_UPDATE>(p, tiles, ntiles, Pin, Pold, Pout, Rout, rkc, last, s);
}

cudaError_t sweep_f32(const Params& p, const DTile* tiles, int ntiles, int ty, int mode, const double* Pin,
                      const double* Pold, double* Pout, double* Rout, double rkc, int last, cudaStream_t s) {
  if (ty == 8) return sweep_ty<8>(p, tiles, ntiles, mode, Pin, Pold, Pout, Rout, rkc, last, s);
  if (ty == 4) return sweep_ty<4>(p, tiles, ntiles, mode, Pin, Pold, Pout, Rout, rkc, last, s);
  return cudaErrorInvalidValue;
}

}  // namespace mb
