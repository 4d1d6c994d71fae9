// kernels_p2_fast.cu -- the p=2 stage with fused multiply-add contraction
// (nvcc -fmad=true), the production p=2 variant.
#define DGSWEM_VARIANT fast_p2
#define DGSWEM_FAST_MATH 1
#include "hydro_kernels.cuh"
#include "hydro_p2.cuh"
