// Fused sweep of the FP64 production form (the simplified flux path in FP64, built with FMA contraction), Riemann
// solver id 4.
#define MB_FAST64 1
#define MB_VAR 1
#define MB_R double
#define MB_RS 4
#define MB_TY TY_F64
#define MB_MINB MINB_F64
#define MB_NAME sweep_f64f_rs4
#include "mb_sweep_inst.inc"
