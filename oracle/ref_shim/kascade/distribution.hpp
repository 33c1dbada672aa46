// Shim for the reference's kascade/distribution.hpp (which needs kamping/MPI):
// a single-rank block distribution, i.e. the identity index maps that the
// one-GPU setting collapses the distribution to.  Only the three members that
// local_pointer_chasing.cpp calls are provided.
#pragma once
#include <cstddef>
#include "kascade/types.hpp"
namespace kascade {
class Distribution {
 public:
  [[nodiscard]] bool is_local(idx_t, std::size_t) const { return true; }
  [[nodiscard]] idx_t get_global_idx(idx_t i, std::size_t) const { return i; }
  [[nodiscard]] idx_t get_local_idx(idx_t i, std::size_t) const { return i; }
};
}  // namespace kascade
