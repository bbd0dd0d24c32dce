// Fused sweep of the FP64 form, the Riemann solver id read at run time (HLLE, SLAU, LLF,
// SLAU2, exact, MiczekRoe: the solvers of no benchmarked case).
#define MB_R double
#define MB_RS 0
#define MB_TY TY_F64
#define MB_MINB MINB_F64
#define MB_NAME sweep_f64_rs0
#include "mb_sweep_inst.inc"
