// Stand-in for raft::resource::get_cuda_stream (see ../../../README.txt).
// TEST INFRASTRUCTURE ONLY.
#pragma once
#include <cuda_runtime.h>

#include "../resources.hpp"

namespace raft {
namespace resource {
struct stream_ref {
  cudaStream_t s = nullptr;
  cudaStream_t value() const { return s; }
};
inline stream_ref get_cuda_stream(const resources&) { return stream_ref{}; }
}  // namespace resource
}  // namespace raft
