// kernels_f32.cu -- FP32 instantiation of the hot-path kernels (the mixed-precision variant's
// fluxes, limiters and vertical solves). Built with FMA contraction enabled.
#define GB_REAL float
#include "kernels_inst.cuh"
