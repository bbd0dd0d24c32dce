// Fused sweep of the FP64 form (built with --fmad=false), Riemann solver id 12.
#define MB_R double
#define MB_RS 12
#define MB_TY TY_F64
#define MB_MINB MINB_F64
#define MB_NAME sweep_f64_rs12
#include "mb_sweep_inst.inc"
