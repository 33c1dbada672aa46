// C++ host interface of kascade_b200, shaped like the reference's lib/kascade
// free functions (niklas-uhl/kascade) minus the MPI Distribution and
// Communicator arguments.  Header-only over the C ABI in kascade_b200.h.
//
//  reference                                      here
//  kascade::set_initial_ranking_state(...)        set_initial_ranking_state(ctx, ...)
//    (lib/kascade/list_ranking.hpp:47-50)
//  kascade::sparse_ruling_set(cfg, succ, rank..)  sparse_ruling_set(ctx, opts, succ, rank)
//    (lib/kascade/sparse_ruling_set.hpp:13-18)
//  kascade::pointer_doubling(cfg, succ, rank..)   pointer_doubling(ctx, opts, succ, rank)
//    (lib/kascade/pointer_doubling.hpp:18-23)
//  kascade::rank_on_root / local_pointer_chasing  rank_on_root(ctx, succ, rank)
//    (lib/kascade/list_ranking.hpp:19-28)
//  kascade::rank_via_euler_tour(cfg, succ, rank)  rank_via_euler_tour(ctx, opts, succ, rank)
//    (lib/kascade/eulertour.hpp:22-27)
//  kascade::compute_euler_tour(parent, comm, hd)  compute_euler_tour(ctx, parent, tour)
//    (lib/kascade/eulertour.hpp:32-34)
//  kascade::is_list(succ, comm)                   is_list(ctx, succ)
//    (lib/kascade/successor_utils.hpp:19-24)
//  AbstractAlgorithm (bench/detail/algorithm.hpp:7-20)  B200Ranking
//
// Spans passed to the device functions must point to device memory; the
// B200Ranking plug-in works on host vectors like the reference's.
#pragma once

#include <cstdint>
#include <span>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "kascade_b200.h"

namespace kascade::b200 {

using idx_t = std::uint64_t;   // lib/kascade/types.hpp:8
using rank_t = std::int64_t;   // lib/kascade/types.hpp:9

enum class Algorithm : std::uint8_t {  // lib/kascade/configuration.hpp:9-18
  GatherChase = KASCADE_ALGO_GATHER_CHASE,
  PointerDoubling = KASCADE_ALGO_POINTER_DOUBLING,
  AsyncPointerDoubling = KASCADE_ALGO_ASYNC_POINTER_DOUBLING,
  RMAPointerDoubling = KASCADE_ALGO_RMA_POINTER_DOUBLING,
  SparseRulingSet = KASCADE_ALGO_SPARSE_RULING_SET,
  EulerTour = KASCADE_ALGO_EULER_TOUR,
};

class Error : public std::runtime_error {
 public:
  Error(kascade_status s, const char* where)
      : std::runtime_error(std::string(where) + ": " + kascade_status_string(s)), status_(s) {}
  [[nodiscard]] kascade_status status() const noexcept { return status_; }

 private:
  kascade_status status_;
};

inline void check(kascade_status s, const char* where) {
  if (s != KASCADE_OK) throw Error(s, where);
}

inline kascade_opts default_opts(Algorithm a = Algorithm::SparseRulingSet) {
  kascade_opts o;
  kascade_opts_init(&o);
  o.algorithm = static_cast<std::uint32_t>(a);
  return o;
}

class Context {
 public:
  explicit Context(int device = 0) { check(kascade_ctx_create(device, &ctx_), "kascade_ctx_create"); }
  ~Context() { kascade_ctx_destroy(ctx_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  Context(Context&& o) noexcept : ctx_(std::exchange(o.ctx_, nullptr)) {}
  [[nodiscard]] kascade_ctx* get() const noexcept { return ctx_; }

 private:
  kascade_ctx* ctx_ = nullptr;
};

// ---- device spans ---------------------------------------------------------
inline void set_initial_ranking_state(Context& c, std::span<const idx_t> succ, std::span<idx_t> root,
                                      std::span<rank_t> rank, void* stream = nullptr) {
  check(kascade_set_initial_ranking_state(c.get(), succ.data(), root.data(), rank.data(), succ.size(), stream),
        "set_initial_ranking_state");
}

inline void sparse_ruling_set(Context& c, const kascade_opts& o, std::span<idx_t> succ, std::span<rank_t> rank,
                              void* stream = nullptr) {
  check(kascade_sparse_ruling_set(c.get(), &o, succ.data(), rank.data(), succ.size(), stream), "sparse_ruling_set");
}

inline void pointer_doubling(Context& c, const kascade_opts& o, std::span<idx_t> succ, std::span<rank_t> rank,
                             void* stream = nullptr) {
  check(kascade_pointer_doubling(c.get(), &o, succ.data(), rank.data(), succ.size(), stream), "pointer_doubling");
}

inline void rank_on_root(Context& c, std::span<idx_t> succ, std::span<rank_t> rank, void* stream = nullptr) {
  check(kascade_rank_on_root(c.get(), succ.data(), rank.data(), succ.size(), stream), "rank_on_root");
}

inline void local_pointer_chasing(Context& c, std::span<idx_t> succ, std::span<rank_t> rank,
                                  void* stream = nullptr) {
  rank_on_root(c, succ, rank, stream);
}

inline void rank_via_euler_tour(Context& c, const kascade_opts& o, std::span<idx_t> succ, std::span<rank_t> rank,
                                void* stream = nullptr) {
  check(kascade_rank_via_euler_tour(c.get(), &o, succ.data(), rank.data(), succ.size(), stream),
        "rank_via_euler_tour");
}

// tour must hold 2 * parent.size() entries; returns the tour length m.
inline std::uint64_t compute_euler_tour(Context& c, std::span<const idx_t> parent, std::span<idx_t> tour,
                                        void* stream = nullptr) {
  if (tour.size() < 2 * parent.size()) throw Error(KASCADE_ERR_INVALID_ARG, "compute_euler_tour");
  std::uint64_t m = 0;
  check(kascade_compute_euler_tour(c.get(), parent.data(), parent.size(), tour.data(), &m, stream),
        "compute_euler_tour");
  return m;
}

// The reference's use_high_degree_handling argument: on one rank its proxy
// construction (lib/kascade/successor_utils.cpp:302-418) creates no proxy and
// builds the same tour, so the flag does not change the result.
inline std::uint64_t compute_euler_tour(Context& c, std::span<const idx_t> parent, std::span<idx_t> tour,
                                        bool /*use_high_degree_handling*/, void* stream = nullptr) {
  return compute_euler_tour(c, parent, tour, stream);
}

inline bool is_list(Context& c, std::span<const idx_t> succ, void* stream = nullptr) {
  int ok = 0;
  check(kascade_is_list(c.get(), succ.data(), succ.size(), &ok, stream), "is_list");
  return ok != 0;
}

// ---- host vectors ---------------------------------------------------------
struct Ranked {
  std::vector<idx_t> root;
  std::vector<std::uint64_t> rank;
};

inline Ranked rank_list_host(Context& c, std::span<const idx_t> succ, std::span<const std::uint32_t> weights = {},
                             const kascade_opts* o = nullptr) {
  Ranked r{std::vector<idx_t>(succ.size()), std::vector<std::uint64_t>(succ.size())};
  check(kascade_rank_list_host(c.get(), succ.data(), weights.empty() ? nullptr : weights.data(), succ.size(),
                               r.root.data(), r.rank.data(), o, nullptr),
        "rank_list_host");
  return r;
}

inline Ranked root_forest_host(Context& c, std::span<const idx_t> parent, const kascade_opts* o = nullptr) {
  Ranked r{std::vector<idx_t>(parent.size()), std::vector<std::uint64_t>(parent.size())};
  check(kascade_root_forest_host(c.get(), parent.data(), parent.size(), r.root.data(), r.rank.data(), o, nullptr),
        "root_forest_host");
  return r;
}

// The reference benchmark's plug-in interface (bench/detail/algorithm.hpp:
// 7-20), implemented on the GPU: ingest a successor (or, for EulerTour, a
// parent) array, run, read roots and ranks -- exactly what GatherRank
// (bench/detail/algorithm_impl.hpp:81-89) produces for the same input.
class B200Ranking {
 public:
  explicit B200Ranking(Algorithm a = Algorithm::SparseRulingSet, int device = 0) : algo_(a), ctx_(device) {}
  void ingest(std::span<const idx_t> succ_array) { succ_.assign(succ_array.begin(), succ_array.end()); }
  void run() {
    Ranked r;
    if (algo_ == Algorithm::EulerTour) {
      r = root_forest_host(ctx_, succ_);
    } else {
      kascade_opts o = default_opts(algo_);
      r = rank_list_host(ctx_, succ_, {}, &o);
    }
    root_ = std::move(r.root);
    rank_.assign(r.rank.begin(), r.rank.end());
  }
  [[nodiscard]] auto get_rank_array() -> std::vector<rank_t> const& { return rank_; }
  [[nodiscard]] auto get_root_array() -> std::vector<idx_t> const& { return root_; }

 private:
  Algorithm algo_;
  Context ctx_;
  std::vector<idx_t> succ_;
  std::vector<idx_t> root_;
  std::vector<rank_t> rank_;
};

}  // namespace kascade::b200
