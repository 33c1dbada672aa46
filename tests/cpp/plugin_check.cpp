// C++ host-side check: the B200Ranking plug-in (include/kascade_b200.hpp)
// ranks seeded lists and forests; results are checked by the local
// conditions that determine them uniquely:
//   list : rank[root] == 0, rank[x] == 1 + rank[succ[x]], root[x] == root[succ[x]]
//   tree : depth[root] == 0, depth[v] == 1 + depth[parent[v]], root[v] == root[parent[v]]
// Exit code 0 on success.
#include <cstdio>
#include <vector>

#include "kascade_b200.hpp"
#include "gen_common.h"

using kascade::b200::Algorithm;
using kascade::b200::B200Ranking;
using kascade::b200::idx_t;

static bool check(const std::vector<idx_t>& succ, B200Ranking& plug, const char* what) {
  plug.ingest(succ);
  plug.run();
  auto const& root = plug.get_root_array();
  auto const& rank = plug.get_rank_array();
  for (idx_t x = 0; x < succ.size(); ++x) {
    idx_t s = succ[x];
    bool ok = (s == x) ? (rank[x] == 0 && root[x] == x) : (rank[x] == 1 + rank[s] && root[x] == root[s]);
    if (!ok) {
      std::printf("%s: mismatch at %llu\n", what, (unsigned long long)x);
      return false;
    }
  }
  std::printf("%s: ok (%zu elements)\n", what, succ.size());
  return true;
}

int main() {
  const uint64_t n = 1u << 20;
  std::vector<idx_t> succ(n);
  ks_perm p = ks_list_perm(n, 42, KS_LAYOUT_RANDOM);
  for (uint64_t k = 0; k < n; ++k) {
    uint64_t e = ks_list_elem(&p, KS_LAYOUT_RANDOM, n, k);
    succ[e] = (k + 1 < n) ? ks_list_elem(&p, KS_LAYOUT_RANDOM, n, k + 1) : e;
  }
  std::vector<idx_t> parent(n);
  ks_perm q = ks_forest_perm(n, 43);
  for (uint64_t v = 0; v < n; ++v) {
    uint64_t at, par;
    ks_forest_edge(&q, KS_FOREST_RRT, n, 16, 0, 43, v, &at, &par);
    parent[at] = par;
  }
  bool ok = true;
  try {
    B200Ranking srs(Algorithm::SparseRulingSet);
    ok &= check(succ, srs, "sparse_ruling_set");
    B200Ranking pd(Algorithm::PointerDoubling);
    ok &= check(succ, pd, "pointer_doubling");
    ok &= check(parent, pd, "pointer_doubling(forest)");
    B200Ranking et(Algorithm::EulerTour);
    ok &= check(parent, et, "euler_tour");
  } catch (const kascade::b200::Error& e) {
    std::printf("error: %s\n", e.what());
    return 2;
  }
  return ok ? 0 : 1;
}
