// Fused sweep of the mixed form (FP32 flux arithmetic), the Riemann solver id read at run time (HLLE, SLAU, LLF,
// SLAU2, exact, MiczekRoe: the solvers of no benchmarked case).
#define MB_R float
#define MB_RS 0
#define MB_TY TY_F32
#define MB_MINB MINB_F32
#define MB_NAME sweep_f32_rs0
#include "mb_sweep_inst.inc"
