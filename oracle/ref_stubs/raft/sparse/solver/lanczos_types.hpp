// Stand-in for raft::sparse::solver::lanczos_solver_config (see
// ../../../README.txt). TEST INFRASTRUCTURE ONLY.
#pragma once
#include <cstdint>
namespace raft {
namespace sparse {
namespace solver {
enum class LANCZOS_WHICH { LA, LM, SA, SM };
template <typename ValueT>
struct lanczos_solver_config {
  int n_components;
  int max_iterations;
  int ncv;
  ValueT tolerance;
  LANCZOS_WHICH which;
  uint64_t seed;
};
}  // namespace solver
}  // namespace sparse
}  // namespace raft
