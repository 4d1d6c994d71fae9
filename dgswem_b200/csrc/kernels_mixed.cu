// kernels_mixed.cu -- the mixed-precision variant: the fast variant with the
// stage kernel's edge traces, numerical fluxes, boundary ghost states,
// volume fluxes and sources and the per-mode right-hand-side sums in FP32,
// and the slope limiter's sweeps in FP32 on deviations from the element
// mean (a variable whose vertex values lie within their node bounds keeps
// its FP64 modes).  The state, the SSP-RK combination (so the element-mean
// elevation accumulates across stages in FP64), the node bounds, the ocean
// depth-positivity fix and WETDRY stay FP64.
#define DGSWEM_VARIANT mixed
#define DGSWEM_FAST_MATH 1
#define DGSWEM_MIXED 1
// FP32 terms need fewer registers and a smaller tile in shared memory:
// 1152 resident stage threads per SM (three blocks of 384, 56 registers)
#define DGSWEM_STAGE_RESIDENT_THREADS 1152
#include "hydro_kernels.cuh"
#include "kernel_launch.inc"
