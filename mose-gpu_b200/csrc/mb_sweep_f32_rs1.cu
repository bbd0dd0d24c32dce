// Fused sweep of the mixed form (FP32 flux arithmetic), Riemann solver id 1.
#define MB_R float
#define MB_RS 1
#define MB_TY TY_F32
#define MB_MINB MINB_F32
#define MB_MINB_KM 4  // the one-plane tiles: a quarter of the shared memory, 4 CTAs per SM at 64 registers
#define MB_NAME sweep_f32_rs1
#include "mb_sweep_inst.inc"
