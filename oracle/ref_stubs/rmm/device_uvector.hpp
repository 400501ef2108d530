// Stand-in for rmm::device_uvector (see ../README.txt): holds no memory.
// TEST INFRASTRUCTURE ONLY.
#pragma once
#include <cstddef>
namespace rmm {
template <typename T>
class device_uvector {
 public:
  template <typename Stream>
  device_uvector(std::size_t, Stream) {}
  T* data() { return nullptr; }
};
}  // namespace rmm
