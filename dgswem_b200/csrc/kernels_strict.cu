// kernels_strict.cu -- the parity variant, compiled with nvcc -fmad=false:
// every product and sum is rounded separately, in the evaluation order of
// the FP64 CPU restatement, so results match it bit for bit wherever no
// device transcendental (pow in Manning / hybrid friction) is involved.
#define DGSWEM_VARIANT strict
#include "hydro_kernels.cuh"
#include "kernel_launch.inc"
