// partition.h -- element partition of the mesh for partitioned handles
// (one per GPU) and the device element order of every handle.
#pragma once

#include <vector>

#include "dgswem_cuda.h"

namespace dgswem {

// Indices sorting points along a Morton (Z-order) curve (stable: ties keep
// the input order).
std::vector<int> morton_order(const std::vector<double>& px, const std::vector<double>& py);

// Partition `part` of `nparts`: the elements at positions
// [part*NE/nparts, (part+1)*NE/nparts) of the global Morton order of the
// element centroids, plus the ghost elements its stage needs from other
// partitions.  Halo kinds:
//   kHaloMeans (0): elements sharing a node with an owned element -- the
//     limiter's node min/max reads their element means after the stage RHS;
//   kHaloFull  (1): elements sharing an edge with an owned element, and
//     internal-barrier partners -- the next stage's fluxes read their full
//     state and wet/dry flag after the limiter and WETDRY.
// send[k][q] / recv[k][q]: input element ids (0-based, ascending) this
// partition sends to / receives from partition q; the two sides derive them
// from the same adjacency, so send[k][q] of p equals recv[k][p] of q.
struct PartPlan {
  int part = 0, nparts = 1;
  std::vector<int> order;   // global Morton order (input ids)
  std::vector<int> owner;   // owning partition of each input element
  std::vector<int> local;   // this partition's elements: owned (Morton order), then ghosts (Morton order)
  int n_own = 0;
  std::vector<std::vector<int>> send[2], recv[2];
};
constexpr int kHaloMeans = 0, kHaloFull = 1;

PartPlan make_part_plan(const dgswem_cuda_setup* s, int part, int nparts);

}  // namespace dgswem
