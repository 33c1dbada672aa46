// C entry points into the reference's own GatherChase implementation
// (lib/kascade/local_pointer_chasing.cpp, compiled from the reference source
// tree by oracle/Makefile).  Test and baseline infrastructure only.
#include <cstdint>
#include <span>

#include "kascade/types.hpp"

namespace kascade {
void local_pointer_chasing(std::span<idx_t> succ_array, std::span<rank_t> rank_array);
}

extern "C" __attribute__((visibility("default"))) void ref_local_pointer_chasing(
    std::uint64_t* succ, std::int64_t* rank, std::uint64_t n) {
  kascade::local_pointer_chasing(std::span<kascade::idx_t>(succ, n),
                                 std::span<kascade::rank_t>(rank, n));
}

// GatherRank (bench/detail/algorithm_impl.hpp:81-89) on one rank:
// set_initial_ranking_state (list_ranking.cpp:60-80) then the chase.
extern "C" __attribute__((visibility("default"))) void ref_gather_rank(
    const std::uint64_t* succ, std::uint64_t n, std::uint64_t* root, std::int64_t* rank) {
  for (std::uint64_t i = 0; i < n; ++i) {
    root[i] = succ[i];
    rank[i] = (succ[i] == i) ? 0 : 1;
  }
  ref_local_pointer_chasing(root, rank, n);
}
