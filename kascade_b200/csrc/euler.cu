// Tree rooting via an Euler tour of the forest.
//
// Reference: rank_via_euler_tour / compute_euler_tour_impl / map_euler_tour_back
// (lib/kascade/eulertour.cpp:33-127, 235-278, 337-392) with the forest built
// by reverse_rooted_tree + make_graph (lib/kascade/successor_utils.cpp:236-300).
//
// Ranking needs each vertex's children grouped, in any order (depth and root
// are unique whatever the rotation), so no sort: one pass links every vertex
// into its parent's child list with one atomic exchange on the list head.
// The tour's rotation is the list order, which depends on the order of the
// exchanges; results do not.
//
// Layout for ranking a single forest (m = n + d elements): slot v (v < n) is
// the up edge v -> parent(v), and for a root r the tour's terminal element
// (weight 0, the reference's dummy root element).  The d non-root vertices
// with children also have a down edge parent(v) -> v, at slot n + (v's number
// among them).  A leaf's down edge would be followed at once by its own up
// edge (weights -1 and +1): the two are one element of weight 0 at slot v, so
// the tour is ~1.5n long instead of 2n, and a leaf's depth is its element's
// rank + 1.  Otherwise the depth of v is the rank of slot v, so the map-back
// is a coalesced pass over slots 0..n-1; the tour of a tree starts at the
// element entering the root's first child and ends in the root's terminal
// slot.  A batch of forests keeps one up and one down slot per vertex (slots
// by vertex, no compaction, so its record count does not depend on the
// forests' shapes) and contracts leaves the same way: a leaf's down slot,
// like a root's, is a dead self loop no element points to.
// compute_euler_tour (the reference's numbering) sorts the children.
#include <algorithm>

#include "ranker.cuh"
#include "sort.cuh"

namespace ks {

namespace {

constexpr int TB_ITEMS = 2;  // vertices per thread in the tour kernels (fewer registers, more resident warps)
constexpr int LINK_ITEMS = 8;  // vertices per thread in one linking round
constexpr int TB_BATCH_ITEMS = 1;  // vertices per thread in a batch's tour build (its forest search adds registers)

inline int bits_for(uint64_t n) {
  int b = 1;
  while (b < 63 && (1ull << b) < n) b++;
  return b;
}

// seg[v] = [start, end) of v's entries in the sorted children array
__global__ void __launch_bounds__(256) k_seg_bounds(const uint32_t* __restrict__ keys, uint32_t n,
                                                    uint2* __restrict__ seg) {
  for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t k = keys[q];
    if (q == 0 || keys[q - 1] != k) seg[k].x = (uint32_t)q;
    if (q + 1 == n || keys[q + 1] != k) seg[k].y = (uint32_t)(q + 1);
  }
}

constexpr uint32_t NO_CHILD = 0xFFFFFFFFu;

// Where a batch's forest tour records live, by vertex.  The forests are
// compacted into one vertex space with per-forest bases fd[j]:
// the up edge of compact vertex c of forest j at that vertex's position in
// the caller's concatenated arrays (foff[j] + c - fd[j]), the down edge into
// c after all input elements (down_base + c).  Ruler sampling thresholds can
// differ per forest (size classes).
struct SlotsBatch {
  const uint32_t* fd;       // nf + 1 compact starts
  const uint32_t* foff;     // nf concatenated offsets
  const uint32_t* fthresh;  // nf sampling thresholds
  const uint32_t* fhint;    // per 4096 compact vertices: the forest holding the first
  uint32_t nf;
  uint32_t down_base;
  __device__ __forceinline__ uint32_t seg_of(uint32_t c) const {
    // last j with fd[j] <= c, between the forests holding this block's first
    // vertex and the next block's
    uint32_t lo = __ldg(fhint + (c >> 12)), hi = min(__ldg(fhint + (c >> 12) + 1) + 1, nf);
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (__ldg(fd + mid) <= c)
        lo = mid;
      else
        hi = mid;
    }
    return lo;
  }
  __device__ __forceinline__ uint32_t up(uint32_t c, uint32_t j) const { return c - __ldg(fd + j) + __ldg(foff + j); }
  __device__ __forceinline__ uint32_t down(uint32_t c) const { return down_base + c; }
  __device__ __forceinline__ uint32_t thresh(uint32_t j) const { return __ldg(fthresh + j); }
};

// Exchange on a child-list head with an L2 evict-last hint: the head array is
// the one array linking reads at random, so its lines keep L2 ahead of the
// streamed parents and sibling links (2.47 -> 2.38 ms at 2^26 vertices).
__device__ __forceinline__ uint32_t exch_head(uint32_t* p, uint32_t v, uint64_t pol) {
  uint32_t old;
  asm volatile("atom.global.exch.L2::cache_hint.b32 %0, [%1], %2, %3;" : "=r"(old) : "l"(p), "r"(v), "l"(pol) : "memory");
  return old;
}

// Child lists of a forest: fc[p] = one child of p (NO_CHILD: a leaf),
// nsib[v] = v's next sibling (NO_CHILD: the last one), one atomic exchange on
// the parent's list head per vertex.  GROUP: a warp's vertices that share a
// parent first link to each other in lane order and the group's first lane
// exchanges the head once (a star then costs n/32 exchanges on one word
// instead of n).  Also writes the root bits (warp ballots over 32 consecutive
// vertices) and a packed 32-bit copy of the parents; an out-of-range parent
// is reported and the vertex treated as a root.
template <bool GROUP>
__global__ void __launch_bounds__(256) k_link_children(const uint64_t* __restrict__ parent, uint32_t n,
                                                       uint32_t* __restrict__ p32, uint32_t* __restrict__ fc,
                                                       uint32_t* __restrict__ nsib, uint32_t* __restrict__ root_bits,
                                                       DevStatus* st) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t pol = l2_keep_policy();
  const uint64_t tile_sz = (uint64_t)blockDim.x * LINK_ITEMS;
  for (uint64_t tile = (uint64_t)blockIdx.x * tile_sz; tile < n; tile += (uint64_t)gridDim.x * tile_sz) {
    // tile and blockDim are multiples of 32: lane 0 of a warp handles a multiple of 32
    uint64_t p[LINK_ITEMS];
#pragma unroll
    for (int i = 0; i < LINK_ITEMS; ++i) {
      const uint64_t v = tile + (uint64_t)i * blockDim.x + threadIdx.x;
      p[i] = v < n ? __ldcs(reinterpret_cast<const unsigned long long*>(parent) + v) : v;
    }
    // every item's exchange is issued before any result is used
    uint32_t old[LINK_ITEMS], peers[LINK_ITEMS];
#pragma unroll
    for (int i = 0; i < LINK_ITEMS; ++i) {
      const uint64_t v = tile + (uint64_t)i * blockDim.x + threadIdx.x;
      const bool valid = v < n;
      if (valid && p[i] >= n) {
        set_error(st, KASCADE_ERR_OUT_OF_RANGE, v);
        p[i] = v;
      }
      const bool root = valid && p[i] == v;
      const uint32_t rb = __ballot_sync(0xffffffffu, root);
      if (lane == 0 && valid) root_bits[v >> 5] = rb;
      const bool link = valid && !root;
      old[i] = NO_CHILD;
      peers[i] = 1u << lane;
      if (GROUP) {
        // parents are below 2^31: lanes that do not link get distinct keys above
        const uint32_t key = link ? (uint32_t)p[i] : (0x80000000u | lane);
        peers[i] = __match_any_sync(0xffffffffu, key);
        if (link && (int)lane == __ffs(peers[i]) - 1) old[i] = exch_head(fc + p[i], (uint32_t)v, pol);
      } else if (link) {
        old[i] = exch_head(fc + p[i], (uint32_t)v, pol);
      }
    }
#pragma unroll
    for (int i = 0; i < LINK_ITEMS; ++i) {
      const uint64_t v = tile + (uint64_t)i * blockDim.x + threadIdx.x;
      const bool valid = v < n;
      const bool link = valid && p[i] != v;
      uint32_t next = old[i];
      if (GROUP) {
        next = __shfl_sync(0xffffffffu, old[i], __ffs(peers[i]) - 1);
        const uint32_t after = peers[i] & ~((2u << lane) - 1u);  // higher lanes of my group
        if (after) next = (uint32_t)(v - lane + (uint32_t)(__ffs(after) - 1));
      }
      if (valid) {
        __stcs(p32 + v, (uint32_t)p[i]);  // streamed past L2: the list heads keep it
        __stcs(nsib + v, link ? next : NO_CHILD);
      }
    }
  }
}

// Sets bit g of `bits` for every lane with `set`: one atomic per distinct word
// the warp touches.  Called by all lanes of the warp.
__device__ __forceinline__ void warp_set_bits(uint32_t* __restrict__ bits, bool set, uint32_t g, uint32_t lane) {
  uint32_t pending = __ballot_sync(0xffffffffu, set);
  while (pending != 0u) {
    const int l = __ffs(pending) - 1;
    const uint32_t w = __shfl_sync(0xffffffffu, g >> 5, l);
    const bool in = set && (g >> 5) == w;
    const uint32_t word = __reduce_or_sync(0xffffffffu, in ? 1u << (g & 31) : 0u);
    if ((int)lane == l) atomicOr(bits + w, word);
    pending &= ~__ballot_sync(0xffffffffu, in);
  }
}

// The tour records of a batch's forests at the slots `slots` gives, from the
// child lists, with leaf contraction as for single forests: a leaf's down and
// up edge are one element of weight 0 at its up slot (its output position),
// whose rank is one less than the leaf's depth (bit set in leaf_out, indexed
// by output position).  The down slot of a leaf or a root holds a dead self
// loop of weight 0 that no element points to: the slots keep one place per
// vertex, so the batch's record count stays fixed (a plan's shapes do not
// depend on its forests' shapes) while the chase visits ~1.5 elements per
// vertex instead of 2.  A tree's tour starts at the element entering its
// root's list head (head_bits), which is always a ruler; ibits (vertices with
// a down edge) tells which element a sibling or first child is entered by.
// A tile's loads are issued in two independent rounds; rulers are sampled
// among the slots and numbered with one atomic per tile.
template <class Slots>
__global__ void __launch_bounds__(256) k_tour_links(const uint32_t* __restrict__ p32, uint32_t n,
                                                    const uint32_t* __restrict__ fc,
                                                    const uint32_t* __restrict__ nsib,
                                                    const uint32_t* __restrict__ ibits,
                                                    const uint32_t* __restrict__ head_bits, Rec* __restrict__ rec,
                                                    uint32_t* __restrict__ ruler_elem, uint32_t* __restrict__ counter,
                                                    uint32_t* __restrict__ leaf_out, uint32_t salt, Slots slots,
                                                    DevStatus* st) {
  __shared__ uint32_t sm[33];
  __shared__ uint32_t sbase;
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t tile_sz = (uint64_t)blockDim.x * TB_BATCH_ITEMS;
  for (uint64_t tile = (uint64_t)blockIdx.x * tile_sz; tile < n; tile += (uint64_t)gridDim.x * tile_sz) {
    uint32_t pv[TB_BATCH_ITEMS], sib[TB_BATCH_ITEMS], first[TB_BATCH_ITEMS], hw[TB_BATCH_ITEMS], jv[TB_BATCH_ITEMS];
#pragma unroll
    for (int i = 0; i < TB_BATCH_ITEMS; ++i) {
      const uint64_t v = tile + (uint64_t)i * blockDim.x + threadIdx.x;
      pv[i] = (uint32_t)v;
      sib[i] = first[i] = NO_CHILD;
      hw[i] = jv[i] = 0;
      if (v < n) {
        pv[i] = __ldcs(p32 + v);  // in range: k_link_children made bad parents roots
        sib[i] = __ldcs(nsib + v);
        first[i] = __ldcs(fc + v);
        hw[i] = __ldg(head_bits + (v >> 5));
        jv[i] = slots.seg_of((uint32_t)v);  // v, its parent and its children belong to the same forest
      }
    }
    uint32_t wsib[TB_BATCH_ITEMS], wfirst[TB_BATCH_ITEMS];
#pragma unroll
    for (int i = 0; i < TB_BATCH_ITEMS; ++i) {
      const uint32_t v = (uint32_t)(tile + (uint64_t)i * blockDim.x + threadIdx.x);
      if (pv[i] >= n) pv[i] = v;
      wsib[i] = wfirst[i] = 0;
      if (v < n && pv[i] != v) {
        if (sib[i] != NO_CHILD) wsib[i] = __ldg(ibits + (sib[i] >> 5));
        if (first[i] != NO_CHILD) wfirst[i] = __ldg(ibits + (first[i] >> 5));
      }
    }
    Rec ru[TB_BATCH_ITEMS], rd[TB_BATCH_ITEMS];
    uint32_t su[TB_BATCH_ITEMS], sd[TB_BATCH_ITEMS];
    uint32_t rl = 0, cnt = 0;
#pragma unroll
    for (int i = 0; i < TB_BATCH_ITEMS; ++i) {
      const uint32_t v = (uint32_t)(tile + (uint64_t)i * blockDim.x + threadIdx.x);
      su[i] = sd[i] = 0;
      bool leaf = false;
      if (v < n) {
        const uint32_t j = jv[i], p = pv[i];
        const uint32_t th = slots.thresh(j);
        const uint32_t up = slots.up(v, j), down = slots.down(v);
        su[i] = up;
        sd[i] = down;
        rd[i].a = 0;  // a dead self loop unless v keeps a down edge
        rd[i].b = down;
        if (p == v) {  // a root: the tour's terminal element (or an isolated vertex)
          ru[i].a = 0;
          ru[i].b = up;
          rl |= 1u << (2 * i);
          cnt++;
        } else {
          // the element a walk enters child c by: its down edge, or its merged slot
          const uint32_t up_next = (sib[i] != NO_CHILD)
                                       ? (((wsib[i] >> (sib[i] & 31)) & 1u) ? slots.down(sib[i]) : slots.up(sib[i], j))
                                       : slots.up(p, j);
          const bool head = (hw[i] >> (v & 31)) & 1u;
          ru[i].b = up_next;
          if (first[i] != NO_CHILD) {
            ru[i].a = 1ull;
            rd[i].a = ~0ull;  // -1
            rd[i].b = ((wfirst[i] >> (first[i] & 31)) & 1u) ? slots.down(first[i]) : slots.up(first[i], j);
            if (sampled(up, salt, th)) {
              rl |= 1u << (2 * i);
              cnt++;
            }
            if (head || sampled(down, salt, th)) {
              rl |= 2u << (2 * i);
              cnt++;
            }
          } else {
            leaf = true;
            ru[i].a = 0;  // down (-1) and up (+1) in one element
            if (head || sampled(up, salt, th)) {
              rl |= 1u << (2 * i);
              cnt++;
            }
          }
        }
      }
      warp_set_bits(leaf_out, leaf, su[i], lane);
    }
    uint32_t total;
    uint32_t pre = block_exclusive_scan(cnt, sm, &total);
    if (threadIdx.x == 0) {
      uint32_t b = total ? atomicAdd(counter, total) : 0u;
      if ((uint64_t)b + total > MAX_RULERS) set_error(st, KASCADE_ERR_TOO_LARGE, b);
      sbase = b;
    }
    __syncthreads();
    uint32_t id = sbase + pre;
#pragma unroll
    for (int i = 0; i < TB_BATCH_ITEMS; ++i) {
      const uint64_t v = tile + (uint64_t)i * blockDim.x + threadIdx.x;
      if (v >= n) continue;
      ru[i].c = TAG_UNREACHED;
      rd[i].c = TAG_UNREACHED;
      if ((rl >> (2 * i)) & 1u) {
        if (id < MAX_RULERS) {
          ru[i].c = TAG_RULER | id;
          ruler_elem[id] = su[i];
        }
        id++;
      }
      if ((rl >> (2 * i)) & 2u) {
        if (id < MAX_RULERS) {
          rd[i].c = TAG_RULER | id;
          ruler_elem[id] = sd[i];
        }
        id++;
      }
      st_rec_cs(rec + su[i], ru[i]);
      st_rec_cs(rec + sd[i], rd[i]);  // every down slot, dead or not: the stores stay coalesced
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// compute_euler_tour in the reference's numbering (one rank).
// ---------------------------------------------------------------------------
// deg[v] = #children + (v not a root); droot[v] = 1 for roots with deg > 0
__global__ void __launch_bounds__(256) k_ref_degrees(const uint64_t* __restrict__ parent, uint32_t n,
                                                     const uint2* __restrict__ seg, uint32_t* __restrict__ deg,
                                                     uint32_t* __restrict__ droot) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const bool root = parent[v] == v;
    const uint2 sg = seg[v];
    const uint32_t children = (sg.y - sg.x) - (root ? 1u : 0u);
    const uint32_t d = children + (root ? 0u : 1u);
    deg[v] = d;
    droot[v] = (root && d > 0) ? 1u : 0u;
  }
}

__global__ void __launch_bounds__(256) k_iota64(uint64_t* __restrict__ out, uint64_t m) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = i;
}

// Per sorted child entry (p, c): the element (c, p) and the element (p, c).
// A vertex v's neighbours in the reference CSR are ordered by decreasing key,
// with key(child) = child id and key(parent) = v (successor_utils.cpp:281-293
// appends (i, parent) then (parent, i) for i ascending; make_graph fills each
// segment from its end).
__global__ void __launch_bounds__(256) k_ref_tour(const uint64_t* __restrict__ parent, const uint32_t* __restrict__ keys,
                                                  const uint32_t* __restrict__ vals, uint32_t n,
                                                  const uint2* __restrict__ seg, const uint32_t* __restrict__ deg,
                                                  const uint32_t* __restrict__ xadj, const uint32_t* __restrict__ didx,
                                                  uint32_t num_edges, uint64_t* __restrict__ tour) {
  for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t p = keys[q], c = vals[q];
    if (p == c) continue;
    const bool proot = parent[p] == p;
    const uint2 sp = seg[p], sc = seg[c];
    const uint32_t cc_p = (sp.y - sp.x) - (proot ? 1u : 0u);
    // index of c among p's children in increasing id order
    uint32_t j = (uint32_t)q - sp.x;
    if (proot && p < c) j -= 1;  // p's own entry sits before c
    const uint32_t pos_c_in_p = (cc_p - 1 - j) + ((!proot && p > c) ? 1u : 0u);
    // number of c's children with id > c (c is not a root: no own entry)
    uint32_t lo = sc.x, hi = sc.y;
    while (lo < hi) {
      uint32_t mid = (lo + hi) >> 1;
      if (vals[mid] <= c)
        lo = mid + 1;
      else
        hi = mid;
    }
    const uint32_t pos_p_in_c = sc.y - lo;
    const uint32_t dp = deg[p], dc = deg[c];
    const uint32_t id_up = xadj[c] + pos_p_in_c;
    const uint32_t id_down = xadj[p] + pos_c_in_p;
    // succ of (c, p): (p, nbr_p[(pos_c_in_p + 1) mod deg p]), or p's dummy
    uint32_t k = (pos_c_in_p + 1) % dp;
    tour[id_up] = (proot && k == 0) ? (uint64_t)num_edges + didx[p] : (uint64_t)xadj[p] + k;
    // succ of (p, c): (c, nbr_c[(pos_p_in_c + 1) mod deg c])
    k = (pos_p_in_c + 1) % dc;
    tour[id_down] = (uint64_t)xadj[c] + k;
  }
}

// The reference-numbered tour's children array: (parent, child) pairs
// sorted by parent (stable, so children in increasing id), and each
// vertex's segment of it.
kascade_status sort_children(kascade_ctx& ctx, const uint64_t* parent, uint32_t n, uint32_t** keys, uint32_t** vals,
                             uint2** seg, cudaStream_t s) {
  SortSource src;
  src.parent = parent;
  KS_TRY(radix_sort_pairs(ctx, src, n, bits_for(n), keys, vals, s));
  *seg = alloc<uint2>(ctx, n);
  if (!*seg) return KASCADE_ERR_OOM;
  KS_CUDA(cudaMemsetAsync(*seg, 0, sizeof(uint2) * (size_t)n, s));
  ProfScope ps(ctx, "seg_bounds", s);
  k_seg_bounds<<<grid_for(ctx, n, 256, 8), 256, 0, s>>>(*keys, n, *seg);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

// Leaf contraction of a single forest's tour.  A leaf's down edge is
// followed by its own up edge (weights -1 and +1), so the two become one
// element of weight 0 at the leaf's slot v: every other rank is unchanged
// and the leaf's depth is that element's rank + 1 (leaf_bits tells the
// output step).  Only non-root vertices with children keep a down edge, at
// the compacted slot n + (their number among those vertices): ibits marks
// them (one word per 32 vertices) and ipre counts them before each word, so
// the element a parent or a sibling continues into is found with one read of
// these L2-resident tables.  head_bits marks the first child of every root
// (the vertex the tree's tour enters first), so the tour build reads its own
// word instead of its parent's root bit and list head.
__global__ void __launch_bounds__(256) k_internal_words(const uint32_t* __restrict__ p32,
                                                        const uint32_t* __restrict__ fc, uint32_t n,
                                                        uint32_t* __restrict__ ibits, uint32_t* __restrict__ icount,
                                                        uint32_t* __restrict__ head_bits) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t tile_sz = (uint64_t)blockDim.x * TB_ITEMS;
  for (uint64_t tile = (uint64_t)blockIdx.x * tile_sz; tile < n; tile += (uint64_t)gridDim.x * tile_sz) {
    // both words of every item are loaded before any is used: 2 x TB_ITEMS loads in flight
    uint32_t pv[TB_ITEMS], fv[TB_ITEMS];
#pragma unroll
    for (int i = 0; i < TB_ITEMS; ++i) {
      const uint64_t v = tile + (uint64_t)i * blockDim.x + threadIdx.x;
      pv[i] = v < n ? __ldcs(p32 + v) : (uint32_t)v;
      fv[i] = v < n ? __ldcs(fc + v) : NO_CHILD;
    }
#pragma unroll
    for (int i = 0; i < TB_ITEMS; ++i) {
      const uint64_t v = tile + (uint64_t)i * blockDim.x + threadIdx.x;
      const uint32_t bits = __ballot_sync(0xffffffffu, v < n && pv[i] != (uint32_t)v && fv[i] != NO_CHILD);
      // a root's list head enters its tree first: the head of that tree's tour
      if (v < n && pv[i] == (uint32_t)v && fv[i] != NO_CHILD) atomicOr(head_bits + (fv[i] >> 5), 1u << (fv[i] & 31));
      if (lane == 0 && v < n) {
        ibits[v >> 5] = bits;
        icount[v >> 5] = (uint32_t)__popc(bits);
      }
    }
  }
}

// (bits, down edges before the word) of every word of 32 vertices
__global__ void __launch_bounds__(256) k_internal_pack(const uint32_t* __restrict__ ibits,
                                                       const uint32_t* __restrict__ ipre, uint32_t words,
                                                       uint2* __restrict__ iw) {
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += gridDim.x * blockDim.x)
    iw[w] = make_uint2(ibits[w], ipre[w]);
}

struct Entries {
  const uint2* iw;  // per word of 32 vertices: (down-edge bits, down edges before it)
  uint32_t n;
  __device__ __forceinline__ uint2 word(uint32_t c) const { return __ldg(iw + (c >> 5)); }
  // the element a walk enters vertex c by, from c's word: its down edge, or
  // its merged slot
  __device__ __forceinline__ uint32_t of(uint32_t c, uint2 w) const {
    const uint32_t below = w.x & ((1u << (c & 31)) - 1u);
    return ((w.x >> (c & 31)) & 1u) ? n + w.y + (uint32_t)__popc(below) : c;
  }
  __device__ __forceinline__ uint32_t down_slot(uint32_t v, uint2 w) const {  // v has a down edge
    return n + w.y + (uint32_t)__popc(w.x & ((1u << (v & 31)) - 1u));
  }
};

// One tile of TB_ITEMS vertices per thread in two rounds of independent loads
// (the vertex's own words; the table words of its sibling, its first child
// and itself), so a tile waits for two memory latencies rather than a chain
// of them per vertex.
__global__ void __launch_bounds__(256) k_tour_leaves(const uint32_t* __restrict__ p32, uint32_t n,
                                                     const uint32_t* __restrict__ fc,
                                                     const uint32_t* __restrict__ nsib,
                                                     const uint32_t* __restrict__ head_bits, Entries ent,
                                                     Rec* __restrict__ rec, uint32_t* __restrict__ ruler_elem,
                                                     uint32_t* __restrict__ counter, uint32_t salt, uint32_t th,
                                                     uint32_t* __restrict__ leaf_bits, DevStatus* st) {
  __shared__ uint32_t sm[33];
  __shared__ uint32_t sbase;
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t tile_sz = (uint64_t)blockDim.x * TB_ITEMS;
  for (uint64_t tile = (uint64_t)blockIdx.x * tile_sz; tile < n; tile += (uint64_t)gridDim.x * tile_sz) {
    uint32_t pv[TB_ITEMS], sib[TB_ITEMS], first[TB_ITEMS], hw[TB_ITEMS];
#pragma unroll
    for (int i = 0; i < TB_ITEMS; ++i) {
      const uint64_t v = tile + (uint64_t)i * blockDim.x + threadIdx.x;
      pv[i] = (uint32_t)v;
      sib[i] = first[i] = NO_CHILD;
      hw[i] = 0;
      if (v < n) {
        pv[i] = __ldcs(p32 + v);
        sib[i] = __ldcs(nsib + v);
        first[i] = __ldcs(fc + v);
        hw[i] = __ldg(head_bits + (v >> 5));
      }
    }
    uint2 wsib[TB_ITEMS], wfirst[TB_ITEMS], wown[TB_ITEMS];
#pragma unroll
    for (int i = 0; i < TB_ITEMS; ++i) {
      const uint32_t v = (uint32_t)(tile + (uint64_t)i * blockDim.x + threadIdx.x);
      if (pv[i] >= n) pv[i] = v;  // k_link_children made bad parents roots; keeps every read in range
      const bool child = v < n && pv[i] != v;
      wsib[i] = wfirst[i] = wown[i] = make_uint2(0, 0);
      if (child) {
        if (sib[i] != NO_CHILD) wsib[i] = ent.word(sib[i]);
        if (first[i] != NO_CHILD) {
          wfirst[i] = ent.word(first[i]);
          wown[i] = ent.word(v);
        }
      }
    }
    Rec ru[TB_ITEMS], rd[TB_ITEMS];
    uint32_t sd[TB_ITEMS];
    uint32_t rl = 0, cnt = 0, has_down = 0;
#pragma unroll
    for (int i = 0; i < TB_ITEMS; ++i) {
      const uint32_t v = (uint32_t)(tile + (uint64_t)i * blockDim.x + threadIdx.x);
      sd[i] = 0;
      bool leaf = false;
      if (v < n) {
        const uint32_t p = pv[i];
        if (p == v) {  // a root: the tour's terminal element (or an isolated vertex)
          ru[i].a = 0;
          ru[i].b = v;
          rl |= 1u << (2 * i);
          cnt++;
        } else {
          const uint32_t up_next = (sib[i] != NO_CHILD) ? ent.of(sib[i], wsib[i]) : p;
          const bool head = (hw[i] >> (v & 31)) & 1u;  // the down edge (or merged element) heading a tour
          if (first[i] != NO_CHILD) {
            sd[i] = ent.down_slot(v, wown[i]);
            ru[i].a = 1ull;
            ru[i].b = up_next;
            rd[i].a = ~0ull;  // -1
            rd[i].b = ent.of(first[i], wfirst[i]);
            has_down |= 1u << i;
            if (sampled(v, salt, th)) {
              rl |= 1u << (2 * i);
              cnt++;
            }
            if (head || sampled(sd[i], salt, th)) {
              rl |= 2u << (2 * i);
              cnt++;
            }
          } else {
            leaf = true;
            ru[i].a = 0;  // down (-1) and up (+1) in one element
            ru[i].b = up_next;
            if (head || sampled(v, salt, th)) {
              rl |= 1u << (2 * i);
              cnt++;
            }
          }
        }
      }
      // a warp's 32 consecutive vertices make one word of leaf bits
      const uint32_t lb = __ballot_sync(0xffffffffu, leaf);
      if (lane == 0 && v < n) leaf_bits[v >> 5] = lb;
    }
    uint32_t total;
    uint32_t pre = block_exclusive_scan(cnt, sm, &total);
    if (threadIdx.x == 0) {
      uint32_t b = total ? atomicAdd(counter, total) : 0u;
      if ((uint64_t)b + total > MAX_RULERS) set_error(st, KASCADE_ERR_TOO_LARGE, b);
      sbase = b;
    }
    __syncthreads();
    uint32_t id = sbase + pre;
#pragma unroll
    for (int i = 0; i < TB_ITEMS; ++i) {
      const uint64_t v = tile + (uint64_t)i * blockDim.x + threadIdx.x;
      if (v >= n) continue;
      ru[i].c = TAG_UNREACHED;
      rd[i].c = TAG_UNREACHED;
      if ((rl >> (2 * i)) & 1u) {
        if (id < MAX_RULERS) {
          ru[i].c = TAG_RULER | id;
          ruler_elem[id] = (uint32_t)v;
        }
        id++;
      }
      if ((rl >> (2 * i)) & 2u) {
        if (id < MAX_RULERS) {
          rd[i].c = TAG_RULER | id;
          ruler_elem[id] = sd[i];
        }
        id++;
      }
      st_rec_cs(rec + v, ru[i]);
      if ((has_down >> i) & 1u) st_rec_cs(rec + sd[i], rd[i]);
    }
    __syncthreads();
  }
}

// Child lists of the forest (parent[v], n vertices, one vertex space), the
// packed parents and the root bits.
kascade_status link_children(kascade_ctx& ctx, const uint64_t* parent, uint32_t n, uint32_t* fc, uint32_t* nsib,
                             uint32_t* p32, uint32_t* root_bits, cudaStream_t s) {
  ProfScope ps(ctx, "link_children", s);
  KS_CUDA(cudaMemsetAsync(fc, 0xFF, sizeof(uint32_t) * (size_t)n, s));
  k_link_children<true><<<grid_for(ctx, n, 256, 8), 256, 0, s>>>(parent, n, p32, fc, nsib, root_bits, ctx.d_status);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

// Child lists and the leaf-contracted tour records of every vertex at the
// slots `slots` gives (a batch's forests); ruler ids continue `counter`,
// leaves are marked in leaf_out (by output position, zeroed by the caller).
template <class Slots>
kascade_status build_tour(kascade_ctx& ctx, const uint64_t* parent, uint32_t n, const Slots& slots, Rec* rec,
                          uint32_t* ruler_elem, uint32_t* counter, uint32_t* leaf_out, uint32_t salt, cudaStream_t s) {
  const uint64_t words = ((uint64_t)n + 31) / 32;
  uint32_t* fc = alloc<uint32_t>(ctx, n);
  uint32_t* nsib = alloc<uint32_t>(ctx, n);
  uint32_t* p32 = alloc<uint32_t>(ctx, n);
  uint32_t* root_bits = alloc<uint32_t>(ctx, words);
  uint32_t* ibits = alloc<uint32_t>(ctx, words);
  uint32_t* icount = alloc<uint32_t>(ctx, words);
  uint32_t* head_bits = alloc<uint32_t>(ctx, words);
  if (!fc || !nsib || !p32 || !root_bits || !ibits || !icount || !head_bits) return KASCADE_ERR_OOM;
  KS_CUDA(cudaMemsetAsync(head_bits, 0, sizeof(uint32_t) * words, s));
  KS_TRY(link_children(ctx, parent, n, fc, nsib, p32, root_bits, s));
  ProfScope ps(ctx, "tour_build", s);
  k_internal_words<<<grid_for(ctx, n, 256, 8), 256, 0, s>>>(p32, fc, n, ibits, icount, head_bits);
  KS_CHECK_LAUNCH();
  const unsigned grid =
      grid_for(ctx, ((uint64_t)n + 256 * TB_BATCH_ITEMS - 1) / (256 * TB_BATCH_ITEMS) * 256, 256, 8);
  k_tour_links<Slots><<<grid, 256, 0, s>>>(p32, n, fc, nsib, ibits, head_bits, rec, ruler_elem, counter, leaf_out,
                                           salt, slots, ctx.d_status);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

}  // namespace

kascade_status root_forest_impl(kascade_ctx& ctx, const uint64_t* parent, uint32_t n, uint64_t* root_out,
                                uint64_t* depth_out, int keep_roots, const Params& p, cudaStream_t s,
                                bool device_levels) {
  if (n == 0) return KASCADE_OK;
  const uint32_t words = (uint32_t)(((uint64_t)n + 31) / 32);
  Rec* rec = alloc<Rec>(ctx, 2ull * n);
  uint32_t* ruler_elem = alloc<uint32_t>(ctx, 2ull * n);
  uint32_t* ctr = alloc<uint32_t>(ctx, 2);  // ruler count, down-edge count
  uint32_t* fc = alloc<uint32_t>(ctx, n);
  uint32_t* nsib = alloc<uint32_t>(ctx, n);
  uint32_t* p32 = alloc<uint32_t>(ctx, n);
  uint32_t* root_bits = alloc<uint32_t>(ctx, words);
  uint32_t* ibits = alloc<uint32_t>(ctx, words);
  uint32_t* icount = alloc<uint32_t>(ctx, words);
  uint32_t* ipre = alloc<uint32_t>(ctx, words);
  uint32_t* leaf_bits = alloc<uint32_t>(ctx, words);
  uint32_t* head_bits = alloc<uint32_t>(ctx, words);
  uint2* iw = alloc<uint2>(ctx, words);
  if (!rec || !ruler_elem || !ctr || !fc || !nsib || !p32 || !root_bits || !ibits || !icount || !ipre || !leaf_bits ||
      !head_bits || !iw)
    return KASCADE_ERR_OOM;
  KS_CUDA(cudaMemsetAsync(ctr, 0, 2 * sizeof(uint32_t), s));
  KS_CUDA(cudaMemsetAsync(head_bits, 0, sizeof(uint32_t) * (size_t)words, s));
  KS_TRY(link_children(ctx, parent, n, fc, nsib, p32, root_bits, s));
  {
    ProfScope ps(ctx, "tour_build", s);
    k_internal_words<<<grid_for(ctx, n, 256, 8), 256, 0, s>>>(p32, fc, n, ibits, icount, head_bits);
    KS_CHECK_LAUNCH();
    KS_TRY(exclusive_scan_u32(ctx, icount, ipre, words, ctr + 1, s));
    k_internal_pack<<<grid_for(ctx, words, 256, 8), 256, 0, s>>>(ibits, ipre, words, iw);
    KS_CHECK_LAUNCH();
  }
  {
    ProfScope ps(ctx, "tour_build", s);
    const unsigned grid = grid_for(ctx, ((uint64_t)n + 256 * TB_ITEMS - 1) / (256 * TB_ITEMS) * 256, 256, 8);
    const uint32_t th = (uint32_t)(4294967296.0 / (double)(p.spacing0 < 2 ? 2 : p.spacing0));
    k_tour_leaves<<<grid, 256, 0, s>>>(p32, n, fc, nsib, head_bits, Entries{iw, n}, rec, ruler_elem, ctr,
                                       mix32(p.seed ^ 0x70757254u), th, leaf_bits, ctx.d_status);
    KS_CHECK_LAUNCH();
  }
  SinkTour sink{root_out, depth_out, n, keep_roots, leaf_bits};
  // The tour's length m = n + (down edges) is on the device (ctr[1]).  The
  // device-driven recursion sizes for the bound 2n instead of reading it: no
  // element points into the unused slots [m, 2n), no chase visits them, and
  // outputs come only from slots below n; the write-free level 0 takes its
  // count of down-edge entries from ctr[1].  (Every element below m exists
  // and m >= n > base_max, so no path that reads every record is taken.)
  const uint32_t m_cap = 2 * n;  // n <= 2^31 - 1
  if (device_levels && n > p.base_max && p.max_levels > 0) {
    sink.downs_dev = ctr + 1;
    if (m_cap < p.level0_log_min)
      return rank_records_dev(ctx, rec, m_cap, ctr, dev_cap_next(m_cap, p.spacing0), ruler_elem, sink, p, s);
    if (!keep_roots)  // the write-free level 0 with the ruler count and the deeper levels on the device
      return rank_level0_log(ctx, rec, m_cap, dev_cap_next(m_cap, p.spacing0), ruler_elem,
                             sink.log_target(m_cap), p, s, ctr);
  }
  // the host-driven path: the tour's length and the ruler count (host reads)
  uint32_t downs = 0, r = 0;
  KS_TRY(read_u32(ctx, ctr + 1, &downs, s));
  KS_TRY(read_u32(ctx, ctr, &r, s));
  return rank_records(ctx, rec, n + downs, r, ruler_elem, sink, p, s);
}

// Tours of a batch of forests whose parents are given in one compact vertex
// space (fpar[c] = compact parent of compact vertex c); records go to the
// slots described by SlotsBatch, ruler ids continue `counter`.
kascade_status batch_tours(kascade_ctx& ctx, const uint64_t* fpar, uint32_t F, const uint32_t* fd, const uint32_t* foff,
                           const uint32_t* fthresh, const uint32_t* fhint, uint32_t nf, uint32_t down_base, Rec* rec,
                           uint32_t* ruler_elem, uint32_t* counter, uint32_t* leaf_out, uint32_t salt,
                           cudaStream_t s) {
  if (F == 0) return KASCADE_OK;
  const SlotsBatch slots{fd, foff, fthresh, fhint, nf, down_base};
  return build_tour(ctx, fpar, F, slots, rec, ruler_elem, counter, leaf_out, salt, s);
}

kascade_status compute_euler_tour_impl(kascade_ctx& ctx, const uint64_t* parent, uint32_t n, uint64_t* tour,
                                       uint64_t* m_out, cudaStream_t s) {
  *m_out = 0;
  if (n == 0) return KASCADE_OK;
  uint32_t *keys, *vals;
  uint2* seg;
  KS_TRY(sort_children(ctx, parent, n, &keys, &vals, &seg, s));
  uint32_t* deg = alloc<uint32_t>(ctx, n);
  uint32_t* droot = alloc<uint32_t>(ctx, n);
  uint32_t* xadj = alloc<uint32_t>(ctx, n);
  uint32_t* tot = alloc<uint32_t>(ctx, 2);
  if (!deg || !droot || !xadj || !tot) return KASCADE_ERR_OOM;
  const unsigned grid = grid_for(ctx, n, 256, 8);
  k_ref_degrees<<<grid, 256, 0, s>>>(parent, n, seg, deg, droot);
  KS_CHECK_LAUNCH();
  KS_TRY(exclusive_scan_u32(ctx, deg, xadj, n, tot, s));
  KS_TRY(exclusive_scan_u32(ctx, droot, droot, n, tot + 1, s));
  uint32_t num_edges = 0;
  KS_TRY(read_u32(ctx, tot, &num_edges, s));
  // m = num_edges + #roots; #roots = n - num_edges / 2
  const uint64_t roots = (uint64_t)n - num_edges / 2;
  const uint64_t m = (uint64_t)num_edges + roots;
  k_iota64<<<grid_for(ctx, m, 256, 8), 256, 0, s>>>(tour, m);
  KS_CHECK_LAUNCH();
  {
    ProfScope ps(ctx, "ref_tour", s);
    k_ref_tour<<<grid, 256, 0, s>>>(parent, keys, vals, n, seg, deg, xadj, droot, num_edges, tour);
    KS_CHECK_LAUNCH();
  }
  *m_out = m;
  return KASCADE_OK;
}

}  // namespace ks
