// partition.h -- element partition of the mesh for partitioned handles
// (one per GPU) and the device element order of every handle.
#pragma once

#include <vector>

#include "dgswem_cuda.h"

namespace dgswem {

// Indices sorting points along a Morton (Z-order) curve (stable: ties keep
// the input order).  With `group` (one id per point, 0..G-1), points are
// sorted by group first and along the curve of their group's own bounding
// box within it, so that disjoint meshes sharing the same coordinates (the
// members of a merged ensemble) stay contiguous.
std::vector<int> morton_order(const std::vector<double>& px, const std::vector<double>& py,
                              const std::vector<int>& group = {});

// The setup's integer mesh tables checked against their ranges before any
// of them indexes an array: NM in 1..NP, NELED in 1..NEDGES, NEDEL in
// 0..NE (0: no element on that side), NEDSD in 1..3 where NEDEL names an
// element, and the boundary lists' edge numbers in 1..NEDGES.  A host that
// passes an inconsistent mesh gets DGSWEM_ERR_ARG (a Failure) instead of a
// fault in the setup or the kernels.
void validate_mesh_ids(const dgswem_cuda_setup* s);

// Connected components of the mesh (elements joined by shared nodes),
// numbered by their first element in input order: one id per element, and
// per node in *node_comp when given.  A connected mesh is one component.
std::vector<int> mesh_components(const dgswem_cuda_setup* s, std::vector<int>* node_comp);

// Partition `part` of `nparts`: the elements at positions
// [part*NE/nparts, (part+1)*NE/nparts) of the global order of the element
// centroids (by component, then Morton), plus the ghost elements its stage needs from other
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
