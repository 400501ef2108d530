// Stand-in for raft::sparse::solver::lanczos_compute_smallest_eigenvectors
// (see ../../../README.txt): it always reports failure (status -1).
// TEST INFRASTRUCTURE ONLY.
#pragma once
#include "../../core/resources.hpp"
#include "lanczos_types.hpp"
namespace raft {
namespace sparse {
namespace solver {
template <typename IndexT, typename ValueT, typename... Views>
int lanczos_compute_smallest_eigenvectors(const raft::resources&,
                                          const lanczos_solver_config<ValueT>&, Views&&...) {
  return -1;
}
}  // namespace solver
}  // namespace sparse
}  // namespace raft
