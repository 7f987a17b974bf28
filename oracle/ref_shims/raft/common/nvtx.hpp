// Stand-in for RAFT's NVTX helpers: ranges are no-ops (see ../../README.md).
#pragma once
namespace raft::common::nvtx {
struct range {
  template <typename... A>
  explicit range(A&&...)
  {
  }
};
template <typename... A>
inline void push_range(A&&...)
{
}
inline void pop_range() {}
}  // namespace raft::common::nvtx
