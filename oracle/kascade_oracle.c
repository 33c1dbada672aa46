/*
 * kascade CPU oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-rank restatement of the reference's list-ranking and
 * tree-rooting algorithms (niklas-uhl/kascade, lib/kascade).  It exists to
 * check the CUDA library: only the tests, the smoke entry and the bench's CPU
 * baseline leg load it.  The product library never links or calls it.
 *
 * Parity pin: oracle_local_pointer_chasing is checked against the reference's
 * own lib/kascade/local_pointer_chasing.cpp, compiled from its source by
 * oracle/Makefile into oracle/_ref (see ref_entry.cpp), and the pack/unpack
 * restatement against the known answers of tests/pack_test.cpp.
 *
 * Conventions: idx_t = uint64_t, rank_t = int64_t (lib/kascade/types.hpp:8-9).
 * A root is an element whose successor is itself
 * (lib/kascade/successor_utils.cpp:65-70).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../kascade_b200/csrc/gen_common.h"

#define ORACLE_API __attribute__((visibility("default")))

/* list_ranking.cpp:60-80 (set_initial_ranking_state): root := succ,
 * rank := 1, and 0 for roots. */
ORACLE_API void oracle_set_initial_ranking_state(const uint64_t* succ, uint64_t n, uint64_t* root,
                                                 int64_t* rank) {
  for (uint64_t i = 0; i < n; ++i) {
    root[i] = succ[i];
    rank[i] = (succ[i] == i) ? 0 : 1;
  }
}

/* local_pointer_chasing.cpp:18-59 (single rank, identity index maps).
 * Marks every element that has a predecessor, then walks from every leaf to
 * its root, and writes back along the walked path in reverse, skipping the
 * last path element (whose successor already is the root): each element adds
 * the (already final) rank of its successor and then points at the root.
 * Works for forests of lists and of trees.  Returns 0, or -1 when a walk
 * exceeds n steps (a cycle without a root, which the reference would loop on). */
ORACLE_API int oracle_local_pointer_chasing(uint64_t* succ, int64_t* rank, uint64_t n) {
  uint8_t* has_pred = (uint8_t*)calloc(n ? n : 1, 1);
  uint64_t* path = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
  int rc = 0;
  for (uint64_t i = 0; i < n; ++i) has_pred[succ[i]] = 1;
  for (uint64_t leaf = 0; leaf < n; ++leaf) {
    if (has_pred[leaf]) continue;
    uint64_t len = 0;
    uint64_t cur = leaf;
    while (succ[cur] != cur) {
      if (len >= n) {
        rc = -1;
        goto done;
      }
      path[len++] = cur;
      cur = succ[cur];
    }
    uint64_t root = cur;
    /* reverse order, dropping the first element of the reversed path */
    if (len >= 2) {
      for (uint64_t j = len - 1; j-- > 0;) {
        uint64_t idx = path[j];
        rank[idx] += rank[succ[idx]];
        succ[idx] = root;
      }
    }
  }
done:
  free(path);
  free(has_pred);
  return rc;
}

/* Synchronous pointer doubling, restating pointer_doubling_generic.hpp:
 * initialize_active_vertices (:418-438) flags roots with the MSB, every round
 * each active element reads (succ, rank) of its successor as it was at the
 * start of the round (the request/reply exchange, :171-212 and
 * update_via_read_offsets :43-60): rank += rank[s], succ = succ[s]; an element
 * leaves the active set once its new successor carries the root flag; the flag
 * is cleared at the end (:690-692).  Returns the number of rounds, or -1 if it
 * exceeds 64 rounds (a cycle). */
#define ROOT_FLAG (1ull << 63)
ORACLE_API int oracle_pointer_doubling(uint64_t* succ, int64_t* rank, uint64_t n) {
  uint64_t* s2 = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
  int64_t* r2 = (int64_t*)malloc(sizeof(int64_t) * (n ? n : 1));
  uint8_t* active = (uint8_t*)malloc(n ? n : 1);
  uint64_t num_active = 0;
  int rounds = 0;
  for (uint64_t i = 0; i < n; ++i) {
    if (succ[i] == i) {
      succ[i] |= ROOT_FLAG;
      active[i] = 0;
    } else {
      active[i] = 1;
      num_active++;
    }
  }
  while (num_active > 0) {
    if (rounds >= 64) {
      rounds = -1;
      break;
    }
    memcpy(s2, succ, sizeof(uint64_t) * n);
    memcpy(r2, rank, sizeof(int64_t) * n);
    num_active = 0;
    for (uint64_t i = 0; i < n; ++i) {
      if (!active[i]) continue;
      uint64_t s = succ[i] & ~ROOT_FLAG;
      s2[i] = succ[s];
      r2[i] = rank[i] + rank[s];
      if (s2[i] & ROOT_FLAG)
        active[i] = 0;
      else
        num_active++;
    }
    memcpy(succ, s2, sizeof(uint64_t) * n);
    memcpy(rank, r2, sizeof(int64_t) * n);
    rounds++;
  }
  for (uint64_t i = 0; i < n; ++i) succ[i] &= ~ROOT_FLAG;
  free(s2);
  free(r2);
  free(active);
  return rounds;
}

/* Weighted list ranking in the clean form: weight[i] is the distance from i to
 * succ[i] (NULL = unit weights); a root's weight is ignored.  Output:
 * root[i], rank[i] = sum of weights on the path from i to its root, excluding
 * the root (0 at roots).  Initial state as list_ranking.cpp:60-80 with
 * weights instead of 1, then the GatherChase walk. */
ORACLE_API int oracle_rank_list(const uint64_t* succ, const uint32_t* weight, uint64_t n,
                                uint64_t* root, uint64_t* rank) {
  int64_t* r = (int64_t*)rank;
  for (uint64_t i = 0; i < n; ++i) {
    root[i] = succ[i];
    r[i] = (succ[i] == i) ? 0 : (weight ? (int64_t)weight[i] : 1);
  }
  int rc = oracle_local_pointer_chasing(root, r, n);
  /* A cycle no leaf leads into is never walked; it shows as an element whose
   * final root is not a root. */
  for (uint64_t i = 0; rc == 0 && i < n; ++i)
    if (root[root[i]] != root[i]) rc = -1;
  return rc;
}

/* Tree rooting by GatherRank (bench/detail/algorithm_impl.hpp:81-89): the
 * same initial state and chase on a parent array gives each vertex its root
 * and its depth (edge count). */
ORACLE_API int oracle_root_forest(const uint64_t* parent, uint64_t n, uint64_t* root,
                                  uint64_t* depth) {
  return oracle_rank_list(parent, NULL, n, root, depth);
}

/* successor_utils.cpp:31-63 (is_list): no element is the successor of two
 * different non-root elements. */
ORACLE_API int oracle_is_list(const uint64_t* succ, uint64_t n) {
  uint8_t* seen = (uint8_t*)calloc(n ? n : 1, 1);
  int ok = 1;
  for (uint64_t i = 0; i < n && ok; ++i) {
    if (succ[i] == i) continue;
    if (seen[succ[i]]) ok = 0;
    seen[succ[i]] = 1;
  }
  free(seen);
  return ok;
}

/* ---------------------------------------------------------------------------
 * Euler tour, single rank, in the reference's own element numbering.
 *
 *  - reverse_rooted_tree(add_back_edge = true), successor_utils.cpp:265-300:
 *    for i = 0..n-1 (non-roots) append edge (i -> parent) then (parent -> i).
 *  - make_graph, successor_utils.cpp:236-260: counting sort by source that
 *    fills each source's segment from its end, so a segment holds its edges in
 *    reverse insertion order.
 *  - compute_euler_tour_impl, eulertour.cpp:33-127: edge (v, nbr_i) gets the
 *    id xadj[v] + i; succ[(u_prev, v)] = (v, nbr_i) with
 *    u_prev = nbr_{(i-1) mod deg}; for a root v and i == 0 the successor is a
 *    dummy element (ids num_edges, num_edges+1, ... in root order) with weight
 *    0; weight +1 for (v, parent(v)) and -1 otherwise; the element array is
 *    num_edges + #roots long and starts as self loops.
 *
 * Outputs (m = 2 (n - #roots) + #roots elements): tour_succ[m], tour_w[m],
 * edge_src[m], edge_dst[m] (dummy elements: (v, v); isolated-root slots keep
 * (0, 0) as the reference's default-constructed pairs), is_up[m]. Returns m.
 * ------------------------------------------------------------------------ */
ORACLE_API uint64_t oracle_euler_tour_size(const uint64_t* parent, uint64_t n) {
  uint64_t roots = 0;
  for (uint64_t i = 0; i < n; ++i) roots += (parent[i] == i);
  return 2 * (n - roots) + roots;
}

ORACLE_API uint64_t oracle_euler_tour(const uint64_t* parent, uint64_t n, uint64_t* tour_succ,
                                      int64_t* tour_w, uint64_t* edge_src, uint64_t* edge_dst,
                                      uint8_t* is_up) {
  uint64_t roots = 0;
  for (uint64_t i = 0; i < n; ++i) roots += (parent[i] == i);
  uint64_t num_edges = 2 * (n - roots);
  uint64_t m = num_edges + roots;
  uint64_t* xadj = (uint64_t*)calloc(n + 1, sizeof(uint64_t));
  uint64_t* adj = (uint64_t*)malloc(sizeof(uint64_t) * (num_edges ? num_edges : 1));
  /* make_graph: count per source, inclusive scan, fill from the end */
  for (uint64_t i = 0; i < n; ++i) {
    if (parent[i] == i) continue;
    xadj[i]++;
    xadj[parent[i]]++;
  }
  for (uint64_t i = 1; i <= n; ++i) xadj[i] += xadj[i - 1];
  for (uint64_t i = 0; i < n; ++i) {
    if (parent[i] == i) continue;
    uint64_t p = parent[i];
    adj[--xadj[i]] = p; /* back edge (i -> p), inserted first   */
    adj[--xadj[p]] = i; /* edge (p -> i)                          */
  }
  for (uint64_t e = 0; e < m; ++e) {
    tour_succ[e] = e;
    tour_w[e] = 0;
    edge_src[e] = 0;
    edge_dst[e] = 0;
    is_up[e] = 0;
  }
  /* edge id of (v, u): position of u inside v's segment */
  uint64_t root_index = num_edges;
  for (uint64_t v = 0; v < n; ++v) {
    uint64_t b = xadj[v], deg = xadj[v + 1] - xadj[v];
    int v_root = (parent[v] == v);
    for (uint64_t i = 0; i < deg; ++i) {
      uint64_t u_prev = adj[b + (i + deg - 1) % deg];
      uint64_t u = adj[b + i];
      uint64_t id = b + i;
      edge_src[id] = v;
      edge_dst[id] = u;
      tour_w[id] = (parent[v] == u) ? 1 : -1;
      is_up[id] = (parent[v] == u);
      /* element (u_prev, v): position of v inside u_prev's segment */
      uint64_t pb = xadj[u_prev], pe = xadj[u_prev + 1], pos = pb;
      while (pos < pe && adj[pos] != v) pos++;
      if (v_root && i == 0) {
        tour_succ[pos] = root_index;
        tour_w[root_index] = 0;
        edge_src[root_index] = v;
        edge_dst[root_index] = v;
        root_index++;
      } else {
        tour_succ[pos] = id;
      }
    }
  }
  free(xadj);
  free(adj);
  return m;
}

/* rank_via_euler_tour (eulertour.cpp:337-377) with GatherChase as the list
 * ranker, and map_euler_tour_back (:230-313): for every up edge (v, parent)
 * root[v] = the vertex of the dummy its list ends in, rank[v] = its rank.
 * Roots keep their input values.  succ_array holds the parent array on input
 * and the roots on output; rank_array is written for non-roots only. */
ORACLE_API int oracle_rank_via_euler_tour(uint64_t* succ_array, int64_t* rank_array, uint64_t n) {
  uint64_t m = oracle_euler_tour_size(succ_array, n);
  uint64_t* ts = (uint64_t*)malloc(sizeof(uint64_t) * (m ? m : 1));
  int64_t* tw = (int64_t*)malloc(sizeof(int64_t) * (m ? m : 1));
  uint64_t* es = (uint64_t*)malloc(sizeof(uint64_t) * (m ? m : 1));
  uint64_t* ed = (uint64_t*)malloc(sizeof(uint64_t) * (m ? m : 1));
  uint8_t* up = (uint8_t*)malloc(m ? m : 1);
  oracle_euler_tour(succ_array, n, ts, tw, es, ed, up);
  int rc = oracle_local_pointer_chasing(ts, tw, m);
  if (rc == 0) {
    for (uint64_t e = 0; e < m; ++e) {
      if (!up[e]) continue;
      uint64_t v = es[e];
      succ_array[v] = ed[ts[e]];
      rank_array[v] = tw[e];
    }
  }
  free(ts);
  free(tw);
  free(es);
  free(ed);
  free(up);
  return rc;
}

/* ---------------------------------------------------------------------------
 * pack / unpack, pack.hpp:23-177 on one rank: the active elements (given in
 * increasing index order) are compacted to 0..k-1; a packed successor is the
 * packed index of the successor (which must be active); unpack writes the
 * packed result back, translating packed successors to original indices.
 * Returns 0, or -1 if an active element's successor is not active.
 * ------------------------------------------------------------------------ */
ORACLE_API int oracle_pack(const uint64_t* succ, const int64_t* rank, uint64_t n,
                           const uint64_t* active, uint64_t k, uint64_t* succ_packed,
                           int64_t* rank_packed) {
  uint64_t* to_packed = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
  int rc = 0;
  for (uint64_t i = 0; i < n; ++i) to_packed[i] = UINT64_MAX;
  for (uint64_t j = 0; j < k; ++j) to_packed[active[j]] = j;
  for (uint64_t j = 0; j < k; ++j) {
    uint64_t s = succ[active[j]];
    if (s >= n || to_packed[s] == UINT64_MAX) {
      rc = -1;
      break;
    }
    succ_packed[j] = to_packed[s];
    rank_packed[j] = rank[active[j]];
  }
  free(to_packed);
  return rc;
}

ORACLE_API void oracle_unpack(const uint64_t* succ_packed, const int64_t* rank_packed,
                              const uint64_t* active, uint64_t k, uint64_t* succ,
                              int64_t* rank) {
  for (uint64_t j = 0; j < k; ++j) {
    succ[active[j]] = active[succ_packed[j]];
    rank[active[j]] = rank_packed[j];
  }
}

/* ---------------------------------------------------------------------------
 * Seeded generators (the same code the CUDA generator kernels run).
 * ------------------------------------------------------------------------ */
ORACLE_API void oracle_gen_list(uint64_t n, uint64_t seed, uint32_t layout, uint64_t* succ) {
  if (n == 0) return;
  ks_perm p = ks_list_perm(n, seed, layout);
  for (uint64_t k = 0; k < n; ++k) {
    uint64_t e = ks_list_elem(&p, layout, n, k);
    succ[e] = (k + 1 < n) ? ks_list_elem(&p, layout, n, k + 1) : e;
  }
}

ORACLE_API void oracle_gen_weights(uint64_t n, uint64_t seed, uint32_t wbits, uint32_t* w) {
  for (uint64_t i = 0; i < n; ++i) w[i] = ks_weight(seed, i, wbits);
}

ORACLE_API void oracle_gen_forest(uint64_t n, uint64_t seed, uint32_t kind, uint64_t blocks,
                                  uint64_t spine, uint64_t* parent) {
  if (n == 0) return;
  ks_perm p = ks_forest_perm(n, seed);
  for (uint64_t v = 0; v < n; ++v) {
    uint64_t at, par;
    ks_forest_edge(&p, kind, n, blocks, spine, seed, v, &at, &par);
    parent[at] = par;
  }
}
