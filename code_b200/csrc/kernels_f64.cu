// kernels_f64.cu -- FP64 instantiation of the hot-path kernels. Built with --fmad=false: no
// contraction into fused multiply-adds, so each expression rounds exactly as written -- the
// same rounding as the reference's double-precision CPU routines evaluated in source order.
#define GB_REAL double
#include "kernels_inst.cuh"
