// Fused sweep of the mixed form (FP32 flux arithmetic), Riemann solver id 1.
#define MB_R float
#define MB_RS 1
#define MB_TY TY_F32
#define MB_MINB MINB_F32
#define MB_NAME sweep_f32_rs1
#include "mb_sweep_inst.inc"
