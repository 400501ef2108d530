// Stand-in views for raft::make_device_{vector,matrix}_view (see
// ../../README.txt). TEST INFRASTRUCTURE ONLY.
#pragma once
namespace raft {
struct row_major {};
struct col_major {};
template <typename T, typename IdxT>
struct device_view {
  T* ptr;
  IdxT rows, cols;
};
template <typename T, typename IdxT, typename Layout = row_major>
device_view<T, IdxT> make_device_vector_view(T* p, IdxT n) {
  return device_view<T, IdxT>{p, n, IdxT(1)};
}
template <typename T, typename IdxT, typename Layout = row_major>
device_view<T, IdxT> make_device_matrix_view(T* p, IdxT r, IdxT c) {
  return device_view<T, IdxT>{p, r, c};
}
}  // namespace raft
