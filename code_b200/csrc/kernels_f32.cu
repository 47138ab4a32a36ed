// kernels_f32.cu -- FP32 instantiation of the hot-path kernels (the mixed-precision variant's
// fluxes, limiters and vertical solves). Built with FMA contraction enabled.
#define GB_REAL float
#define GB_REAL_IS_FLOAT 1
#include "kernels_inst.cuh"
