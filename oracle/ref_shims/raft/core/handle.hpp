// Stand-in for RAFT's resource handle: the dual simplex only stores a pointer to it.
#pragma once
namespace raft {
class handle_t {};
}  // namespace raft
