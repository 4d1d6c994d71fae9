// kernels_p2_mixed.cu -- the p=2 stage in mixed precision: edge traces,
// numerical fluxes, the edge-point flux slots, volume fluxes and sources in
// FP32; the right-hand-side sums and their weights, the state, the SSP-RK
// combination (the element-mean elevation accumulates across stages in
// FP64) and the ocean depth-positivity fix in FP64.
#define DGSWEM_VARIANT mixed_p2
#define DGSWEM_FAST_MATH 1
#define DGSWEM_MIXED 1
#include "hydro_kernels.cuh"
#include "hydro_p2.cuh"
