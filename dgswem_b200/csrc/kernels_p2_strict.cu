// kernels_p2_strict.cu -- the p=2 stage without contraction (nvcc
// -fmad=false): every product and sum separately rounded, the evaluation
// the FP64 oracle uses.
#define DGSWEM_VARIANT strict_p2
#include "hydro_kernels.cuh"
#include "hydro_p2.cuh"
