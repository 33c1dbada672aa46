// Sharded list ranking: one list spread over several GPUs by index ranges.
//
// The reference distributes a list by contiguous index ranges
// (lib/kascade/distribution.hpp:16-113) and runs the ruler chase in
// synchronous rounds, one all-to-all exchange of ruler messages per round
// (sparse_ruling_set_detail/ruler_chasing_engine.hpp:57-101, locality aware:
// a message whose target is local is worked on at once).  These kernels are
// one shard's part of that scheme on its own GPU; the host side
// (kascade_b200/shard.py) drives the rounds over torch.distributed (NCCL) and
// gathers the ruler sub-list.
//
//   prepare    records of the shard's elements (successor as a global index),
//              rulers = roots + a counter-hash sample by global index, local
//              ruler ids
//   chase      chains start at the shard's rulers (or at incoming messages)
//              and walk while their element is local, stamping (ruler,
//              distance) into each record; a chain that reaches a ruler ends
//              with a sub-list record (ruler -> next ruler, distance), one
//              that leaves the shard becomes a message to the owner of its
//              next element.  Messages are bucketed per destination shard and
//              packed contiguously for the exchange.
//   unreached  after the chase: elements no chain reached (list heads ahead of
//              the first ruler) become rulers, as fixup_unreached does
//              (sparse_ruling_set_detail/post_invert.hpp:195-264); their
//              chains are chased the same way
//   sublist    the gathered chain ends as dense arrays over global ruler ids
//   propagate  rank = rank(ruler) - distance, root = root(ruler)
//
// Global ruler ids: sampled rulers of shard s are ruler_base(s) + local id;
// fix-up rulers follow every shard's sampled ones: fixup_base(s) + (local id -
// num_sampled(s)).  Every device loop is bounded by the shard size.
#include <algorithm>
#include <cstring>
#include <vector>

#include "ranker.cuh"

namespace ks {
namespace {

constexpr int MAX_SHARDS = 1024;

struct ShardView {
  uint64_t lo, n_local;
  uint32_t num_shards, self;
  const uint64_t* offsets;  // device, num_shards + 1
  uint64_t ruler_base, num_sampled, fixup_base;
  __device__ __forceinline__ uint32_t gid(uint32_t lid) const {
    return lid < num_sampled ? (uint32_t)(ruler_base + lid) : (uint32_t)(fixup_base + (lid - num_sampled));
  }
  __device__ __forceinline__ uint32_t owner(uint64_t g) const {
    uint32_t a = 0, b = num_shards;  // last s with offsets[s] <= g
    while (b - a > 1) {
      const uint32_t m = (a + b) >> 1;
      if (__ldg(offsets + m) <= g)
        a = m;
      else
        b = m;
    }
    return a;
  }
};

ShardView view_of(const kascade_shard_desc& d) {
  return ShardView{d.lo, d.n_local, d.num_shards, d.self, d.offsets, d.ruler_base, d.num_sampled, d.fixup_base};
}

__global__ void __launch_bounds__(256) k_shard_prepare(const uint64_t* __restrict__ succ,
                                                       const uint32_t* __restrict__ w, ShardView v, uint64_t n_global,
                                                       uint32_t salt, uint32_t th, Rec* __restrict__ rec,
                                                       uint32_t* __restrict__ ruler_elem, uint32_t* __restrict__ count,
                                                       DevStatus* st) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < v.n_local;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t s = succ[i];
    const uint64_t g = v.lo + i;
    if (s >= n_global) {
      set_error(st, KASCADE_ERR_OUT_OF_RANGE, g);
      s = g;
    }
    const bool root = s == g;
    Rec r;
    r.a = root ? 0ull : (w ? (uint64_t)w[i] : 1ull);
    r.b = (uint32_t)s;
    r.c = TAG_UNREACHED;
    if (root || sampled((uint32_t)g, salt, th)) {
      const uint32_t lid = atomicAdd(count, 1u);
      ruler_elem[lid] = (uint32_t)i;
      r.c = TAG_RULER | lid;
    }
    st_rec_cs(rec + i, r);
  }
}

// One chain per thread: from a start ruler (local element start[k]) or an
// incoming message, walk while the element is local.
__global__ void __launch_bounds__(256) k_shard_chase(Rec* __restrict__ rec, ShardView v,
                                                     const uint32_t* __restrict__ starts, uint64_t n_start,
                                                     const kascade_shard_msg* __restrict__ in, uint64_t n_in,
                                                     kascade_shard_msg* __restrict__ regions, uint64_t region_cap,
                                                     uint32_t* __restrict__ sent, kascade_shard_end* __restrict__ ends,
                                                     uint32_t* __restrict__ end_count, uint64_t end_cap,
                                                     DevStatus* st) {
  const uint64_t total = n_start + n_in;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t cur;  // global index of the chain's next element
    uint32_t ruler;
    uint64_t dist;
    if (k < n_start) {
      const uint32_t x = starts[k];
      const Rec r = ld_rec_cg(rec + x);
      ruler = v.gid(tag_id(r.c));
      if ((uint64_t)r.b == v.lo + x) {  // a root: its sub-list record is a self loop
        const uint32_t e = atomicAdd(end_count, 1u);
        if (e < end_cap) ends[e] = kascade_shard_end{ruler, ruler, 0ull};
        else set_error(st, KASCADE_ERR_TOO_LARGE, e);
        continue;
      }
      cur = r.b;
      dist = r.a;
    } else {
      const kascade_shard_msg m = in[k - n_start];
      cur = m.target;
      ruler = m.ruler;
      dist = m.dist;
    }
    for (uint64_t hop = 0;; ++hop) {
      if (cur < v.lo || cur >= v.lo + v.n_local) {
        const uint32_t d = v.owner(cur);
        const uint32_t p = atomicAdd(sent + d, 1u);
        if (p < region_cap && d != v.self)
          regions[(uint64_t)d * region_cap + p] = kascade_shard_msg{(uint32_t)cur, ruler, dist};
        else
          set_error(st, KASCADE_ERR_TOO_LARGE, p);
        break;
      }
      const uint64_t x = cur - v.lo;
      const Rec r = ld_rec_cg(rec + x);
      if (tag_ruler(r.c)) {  // the chain ends at the next ruler
        if (v.gid(tag_id(r.c)) == ruler) set_error(st, KASCADE_ERR_CYCLE, cur);  // back at its own: rootless
        const uint32_t e = atomicAdd(end_count, 1u);
        if (e < end_cap) ends[e] = kascade_shard_end{ruler, v.gid(tag_id(r.c)), dist};
        else set_error(st, KASCADE_ERR_TOO_LARGE, e);
        break;
      }
      if (!tag_unreached(r.c) || hop >= v.n_local) {
        // a second visit: two predecessors (not a list), or a walk past the shard's size
        set_error(st, KASCADE_ERR_NOT_A_LIST, cur);
        break;
      }
      Rec o;
      o.a = dist;
      o.b = r.b;
      o.c = ruler;  // stamped: the ruler's global id (below TAG_RULER)
      st_rec_cg(rec + x, o);
      dist += r.a;
      cur = r.b;
    }
  }
}

// Elements no chain reached become fix-up rulers (local ids first_lid + k).
__global__ void __launch_bounds__(256) k_shard_unreached(Rec* __restrict__ rec, uint64_t n_local, uint32_t first_lid,
                                                         uint32_t* __restrict__ ruler_elem,
                                                         uint32_t* __restrict__ count) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_local;
       i += (uint64_t)gridDim.x * blockDim.x) {
    Rec r = ld_rec_cg(rec + i);
    if (!tag_unreached(r.c)) continue;
    const uint32_t lid = first_lid + atomicAdd(count, 1u);
    ruler_elem[lid] = (uint32_t)i;
    r.c = TAG_RULER | lid;
    st_rec_cg(rec + i, r);
  }
}

// Global element index of each local ruler, in local-id order.
__global__ void __launch_bounds__(256) k_shard_ruler_globals(const uint32_t* __restrict__ ruler_elem, uint64_t lo,
                                                             uint32_t first, uint32_t count,
                                                             uint64_t* __restrict__ out) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x)
    out[k] = lo + ruler_elem[first + k];
}

// Chain ends -> dense sub-list arrays over global ruler ids.  Every ruler
// starts exactly one chain; succ2 must be preset to NO_RULER.
constexpr uint64_t NO_RULER = ~0ull;
__global__ void __launch_bounds__(256) k_shard_sublist(const kascade_shard_end* __restrict__ ends, uint64_t m,
                                                       uint64_t r, unsigned long long* __restrict__ succ2,
                                                       int64_t* __restrict__ w2, DevStatus* st) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (uint64_t)gridDim.x * blockDim.x) {
    const kascade_shard_end e = ends[k];
    if (e.ruler >= r || e.next >= r) {
      set_error(st, KASCADE_ERR_OUT_OF_RANGE, k);
      continue;
    }
    if (atomicCAS(succ2 + e.ruler, NO_RULER, (unsigned long long)e.next) != NO_RULER) {
      set_error(st, KASCADE_ERR_NOT_A_LIST, e.ruler);
      continue;
    }
    w2[e.ruler] = (int64_t)e.dist;
  }
}

__global__ void __launch_bounds__(256) k_shard_missing(const unsigned long long* __restrict__ succ2, uint64_t r,
                                                       DevStatus* st) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < r; k += (uint64_t)gridDim.x * blockDim.x)
    if (succ2[k] == NO_RULER) set_error(st, KASCADE_ERR_CYCLE, k);  // a ruler whose chain never ended
}

__global__ void __launch_bounds__(256) k_shard_propagate(const Rec* __restrict__ rec, ShardView v,
                                                         const uint64_t* __restrict__ sub_root,
                                                         const int64_t* __restrict__ sub_rank,
                                                         const uint64_t* __restrict__ elem_of, uint64_t r,
                                                         uint64_t* __restrict__ root_out,
                                                         uint64_t* __restrict__ rank_out, DevStatus* st) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < v.n_local;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const Rec e = ld_rec_cs(rec + i);
    uint32_t g;
    uint64_t d = 0;
    if (tag_ruler(e.c)) {
      g = v.gid(tag_id(e.c));
    } else if (!tag_unreached(e.c)) {
      g = e.c;
      d = e.a;
    } else {
      set_error(st, KASCADE_ERR_CYCLE, v.lo + i);
      continue;
    }
    if (g >= r) {
      set_error(st, KASCADE_ERR_OUT_OF_RANGE, v.lo + i);
      continue;
    }
    const uint64_t rg = __ldg(reinterpret_cast<const unsigned long long*>(sub_root) + g);
    if (rg >= r) {
      set_error(st, KASCADE_ERR_OUT_OF_RANGE, v.lo + i);
      continue;
    }
    __stcs(reinterpret_cast<unsigned long long*>(root_out) + i,
           (unsigned long long)__ldg(reinterpret_cast<const unsigned long long*>(elem_of) + rg));
    __stcs(reinterpret_cast<unsigned long long*>(rank_out) + i,
           (unsigned long long)((uint64_t)__ldg(reinterpret_cast<const long long*>(sub_rank) + g) - d));
  }
}

inline unsigned grid_n(const kascade_ctx& ctx, uint64_t n) { return grid_for(ctx, n, 256, 8); }

kascade_status check_desc(const kascade_shard_desc* d) {
  if (!d || d->num_shards == 0 || d->num_shards > MAX_SHARDS || d->self >= d->num_shards || !d->offsets)
    return KASCADE_ERR_INVALID_ARG;
  if (d->lo + d->n_local > d->n_global || d->n_global > 0xFFFFFFFEull) return KASCADE_ERR_TOO_LARGE;
  return KASCADE_OK;
}

}  // namespace
}  // namespace ks

using namespace ks;

namespace {
inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

kascade_status begin(kascade_ctx* c, cudaStream_t s) {
  if (!c) return KASCADE_ERR_INVALID_ARG;
  KS_CUDA(ensure_device(c->device));
  KS_TRY(status_reset(*c, s));
  c->profile = false;
  return KASCADE_OK;
}

kascade_status finish(kascade_ctx* c, cudaStream_t s, kascade_status st) {
  if (st != KASCADE_OK) {
    cudaStreamSynchronize(s);
    return st;
  }
  return status_finish(*c, s);
}

// a device counter word of the context's arena, zeroed on the stream
kascade_status counters(kascade_ctx* c, uint32_t words, uint32_t** out, cudaStream_t s) {
  KS_TRY(arena_begin_call(*c, s));
  *out = alloc<uint32_t>(*c, words);
  if (!*out) return KASCADE_ERR_OOM;
  KS_CUDA(cudaMemsetAsync(*out, 0, sizeof(uint32_t) * words, s));
  return KASCADE_OK;
}
}  // namespace

extern "C" {

KASCADE_API kascade_status kascade_shard_prepare(kascade_ctx* c, const kascade_shard_desc* desc,
                                                 const uint64_t* succ, const uint32_t* weights, uint64_t n_global,
                                                 uint32_t spacing, uint32_t seed, void* rec, uint32_t* ruler_elem,
                                                 uint64_t* num_rulers, void* stream) {
  cudaStream_t s = as_stream(stream);
  KS_TRY(check_desc(desc));
  if (desc->n_global != n_global || (desc->n_local && (!succ || !rec || !ruler_elem)) || !num_rulers)
    return KASCADE_ERR_INVALID_ARG;
  KS_TRY(begin(c, s));
  uint32_t* cnt = nullptr;
  kascade_status st = counters(c, 1, &cnt, s);
  if (st == KASCADE_OK && desc->n_local) {
    const uint32_t th = (uint32_t)(4294967296.0 / (double)(spacing < 2 ? 2 : spacing));
    k_shard_prepare<<<grid_n(*c, desc->n_local), 256, 0, s>>>(succ, weights, view_of(*desc), n_global,
                                                               mix32(seed ^ 0x73686172u), th,
                                                               reinterpret_cast<Rec*>(rec), ruler_elem, cnt,
                                                               c->d_status);
    if (cudaGetLastError() != cudaSuccess) st = KASCADE_ERR_CUDA;
  }
  uint32_t r = 0;
  if (st == KASCADE_OK) st = read_u32(*c, cnt, &r, s);
  *num_rulers = r;
  return finish(c, s, st);
}

KASCADE_API kascade_status kascade_shard_chase(kascade_ctx* c, const kascade_shard_desc* desc, void* rec,
                                               const uint32_t* start_rulers, uint64_t num_start,
                                               const kascade_shard_msg* incoming, uint64_t num_in,
                                               kascade_shard_msg* regions, uint64_t region_cap,
                                               kascade_shard_msg* send, uint64_t* sent_counts,
                                               kascade_shard_end* ends, uint64_t* num_ends, uint64_t end_cap,
                                               void* stream) {
  cudaStream_t s = as_stream(stream);
  KS_TRY(check_desc(desc));
  if (!sent_counts || !num_ends || (num_start && !start_rulers) || (num_in && !incoming) || !regions || !send ||
      !ends || *num_ends > end_cap)
    return KASCADE_ERR_INVALID_ARG;
  KS_TRY(begin(c, s));
  const uint32_t P = desc->num_shards;
  uint32_t* cnt = nullptr;
  kascade_status st = counters(c, P + 1, &cnt, s);  // P destination counts, then the end count
  if (st == KASCADE_OK) {
    // the end count continues from the previous rounds' (a pageable copy:
    // staged before the call returns)
    const uint32_t e0 = (uint32_t)*num_ends;
    st = cuda_status(cudaMemcpyAsync(cnt + P, &e0, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  }
  if (st == KASCADE_OK && num_start + num_in) {
    k_shard_chase<<<grid_n(*c, num_start + num_in), 256, 0, s>>>(
        reinterpret_cast<Rec*>(rec), view_of(*desc), start_rulers, num_start, incoming, num_in, regions, region_cap,
        cnt, ends, cnt + P, end_cap, c->d_status);
    if (cudaGetLastError() != cudaSuccess) st = KASCADE_ERR_CUDA;
  }
  std::vector<uint32_t> h(P + 1, 0);
  if (st == KASCADE_OK)
    st = cuda_status(cudaMemcpyAsync(h.data(), cnt, sizeof(uint32_t) * (P + 1), cudaMemcpyDeviceToHost, s));
  if (st == KASCADE_OK) st = cuda_status(cudaStreamSynchronize(s));
  if (st == KASCADE_OK) st = status_finish(*c, s);
  if (st != KASCADE_OK) return finish(c, s, st);
  // pack the per-destination regions into one contiguous send buffer
  uint64_t off = 0;
  for (uint32_t d = 0; d < P; ++d) {
    const uint64_t k = std::min<uint64_t>(h[d], region_cap);
    sent_counts[d] = k;
    if (k && d != desc->self) {
      st = cuda_status(cudaMemcpyAsync(send + off, regions + (uint64_t)d * region_cap, k * sizeof(kascade_shard_msg),
                                       cudaMemcpyDeviceToDevice, s));
      if (st != KASCADE_OK) break;
    }
    off += k;
  }
  *num_ends = h[P];
  if (st == KASCADE_OK) st = cuda_status(cudaStreamSynchronize(s));
  return st;
}

KASCADE_API kascade_status kascade_shard_unreached(kascade_ctx* c, const kascade_shard_desc* desc, void* rec,
                                                   uint32_t* ruler_elem, uint64_t first_lid, uint64_t* count,
                                                   void* stream) {
  cudaStream_t s = as_stream(stream);
  KS_TRY(check_desc(desc));
  if (!count || (desc->n_local && (!rec || !ruler_elem))) return KASCADE_ERR_INVALID_ARG;
  KS_TRY(begin(c, s));
  uint32_t* cnt = nullptr;
  kascade_status st = counters(c, 1, &cnt, s);
  if (st == KASCADE_OK && desc->n_local) {
    k_shard_unreached<<<grid_n(*c, desc->n_local), 256, 0, s>>>(reinterpret_cast<Rec*>(rec), desc->n_local,
                                                                 (uint32_t)first_lid, ruler_elem, cnt);
    if (cudaGetLastError() != cudaSuccess) st = KASCADE_ERR_CUDA;
  }
  uint32_t u = 0;
  if (st == KASCADE_OK) st = read_u32(*c, cnt, &u, s);
  *count = u;
  return finish(c, s, st);
}

KASCADE_API kascade_status kascade_shard_ruler_globals(kascade_ctx* c, const uint32_t* ruler_elem, uint64_t lo,
                                                       uint64_t first, uint64_t count, uint64_t* out, void* stream) {
  cudaStream_t s = as_stream(stream);
  if (count && (!ruler_elem || !out)) return KASCADE_ERR_INVALID_ARG;
  KS_TRY(begin(c, s));
  if (count) {
    k_shard_ruler_globals<<<grid_n(*c, count), 256, 0, s>>>(ruler_elem, lo, (uint32_t)first, (uint32_t)count, out);
    KS_CHECK_LAUNCH();
  }
  return finish(c, s, KASCADE_OK);
}

KASCADE_API kascade_status kascade_shard_sublist(kascade_ctx* c, const kascade_shard_end* ends, uint64_t num_ends,
                                                 uint64_t num_rulers, uint64_t* succ2, int64_t* w2, void* stream) {
  cudaStream_t s = as_stream(stream);
  if (num_rulers > 0x7FFFFFFEull) return KASCADE_ERR_TOO_LARGE;
  if ((num_ends && !ends) || (num_rulers && (!succ2 || !w2))) return KASCADE_ERR_INVALID_ARG;
  KS_TRY(begin(c, s));
  kascade_status st = KASCADE_OK;
  if (num_ends != num_rulers) {
    st = num_ends < num_rulers ? KASCADE_ERR_CYCLE : KASCADE_ERR_NOT_A_LIST;
  } else if (num_rulers) {
    KS_CUDA(cudaMemsetAsync(succ2, 0xFF, sizeof(uint64_t) * num_rulers, s));
    k_shard_sublist<<<grid_n(*c, num_ends), 256, 0, s>>>(ends, num_ends, num_rulers,
                                                          reinterpret_cast<unsigned long long*>(succ2), w2,
                                                          c->d_status);
    KS_CHECK_LAUNCH();
    k_shard_missing<<<grid_n(*c, num_rulers), 256, 0, s>>>(reinterpret_cast<unsigned long long*>(succ2), num_rulers,
                                                            c->d_status);
    KS_CHECK_LAUNCH();
  }
  return finish(c, s, st);
}

KASCADE_API kascade_status kascade_shard_propagate(kascade_ctx* c, const kascade_shard_desc* desc, const void* rec,
                                                   const uint64_t* sub_root, const int64_t* sub_rank,
                                                   const uint64_t* elem_of_ruler, uint64_t num_rulers,
                                                   uint64_t* root_out, uint64_t* rank_out, void* stream) {
  cudaStream_t s = as_stream(stream);
  KS_TRY(check_desc(desc));
  if (desc->n_local && (!rec || !sub_root || !sub_rank || !elem_of_ruler || !root_out || !rank_out))
    return KASCADE_ERR_INVALID_ARG;
  KS_TRY(begin(c, s));
  if (desc->n_local) {
    k_shard_propagate<<<grid_n(*c, desc->n_local), 256, 0, s>>>(reinterpret_cast<const Rec*>(rec), view_of(*desc),
                                                                 sub_root, sub_rank, elem_of_ruler, num_rulers,
                                                                 root_out, rank_out, c->d_status);
    KS_CHECK_LAUNCH();
  }
  return finish(c, s, KASCADE_OK);
}

}  // extern "C"
