// Stand-in for raft::resources (see ../../README.txt). TEST INFRASTRUCTURE ONLY.
#pragma once
namespace raft {
class resources {};
}  // namespace raft
