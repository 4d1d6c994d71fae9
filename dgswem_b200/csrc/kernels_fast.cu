// kernels_fast.cu -- the production variant: the compiler may contract
// a*b+c into a fused multiply-add (nvcc -fmad=true, the default).
#define DGSWEM_VARIANT fast
#include "hydro_kernels.cuh"
#include "kernel_launch.inc"
