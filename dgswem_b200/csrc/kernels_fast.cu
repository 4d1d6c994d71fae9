// kernels_fast.cu -- the production variant: the compiler may contract
// a*b+c into a fused multiply-add (nvcc -fmad=true, the default), and the
// Manning depth factor uses cbrt instead of pow(x, 1/3).
#define DGSWEM_VARIANT fast
#define DGSWEM_FAST_MATH 1
#include "hydro_kernels.cuh"
#include "kernel_launch.inc"
